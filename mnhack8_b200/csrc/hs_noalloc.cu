// hs_noalloc.cu -- the dot product of two node vectors without any device
// allocation, for callers that cannot call cudaMalloc.
//
// The library's other entry points work through a solver handle whose
// hs_create allocates its buffers.  Some callers cannot allocate device
// memory at the point where they need a result: code that runs under a
// strict device-memory budget owned by a host application, or a
// latency-critical path that must not take the allocator's locks.  For them
// hs_dot_noalloc computes x.y in the library's fixed (flat) reduction order
// -- bit for bit the value hs_dot returns -- with its per-block partial sums
// in a file-scope static device array instead of allocated scratch.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/heat_b200.h"
#include "hs_host.h"
#include "hs_kernels.cuh"

namespace hs {

// Partial sums of the flat reduction order.  k_reduce stores two quantities
// per block of RT*KF nodes (partials[q*nflat + block], q = 0, 1; a dot uses
// only q = 0 but the slot of q = 1 is written all the same), so a grid of
// nflat blocks needs 2*nflat doubles.  Every GPU that loads the library holds
// this array (1 MiB) until exit.
constexpr long long kNoAllocMaxBlocks = 65536;                 // nflat limit: N <= 321
constexpr long long kNoAllocPartials = 2 * kNoAllocMaxBlocks;  // doubles in the array
static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

// final combination of the partials into *out (one value)
__global__ void __launch_bounds__(RT) k_final_dot_noalloc(long long nflat, double* out) {
    __shared__ double sh[MAXQ][8];
    double part[1];
    final_sums<1>(part, g_noalloc_partials, nflat, sh);
    if (threadIdx.x == 0) out[0] = part[0];
}

namespace {
std::mutex g_mu;
// Host-usable device address of the array, per device, looked up once.  A
// cudaDeviceReset unloads the module, after which the cached address is
// stale: do not call hs_dot_noalloc on a device after resetting it.
double* g_addr[128] = {nullptr};
}  // namespace

}  // namespace hs

extern "C" hs_status hs_dot_noalloc(int N, const double* x, const double* y, double* out) {
    using namespace hs;
    if (N < 1 || N > 1200 || !x || !y || !out) { set_error("hs_dot_noalloc: bad arguments"); return HS_ERR_ARG; }
    const long long NN = N + 1, Nn = NN * NN * NN;
    const long long nflat = (Nn + (long long)RT * KF - 1) / ((long long)RT * KF);
    if (2 * nflat > kNoAllocPartials) {
        set_error("hs_dot_noalloc: grid too large for the static scratch (N <= 321, i.e. at most "
                  "65536 blocks of 512 nodes)");
        return HS_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("hs_dot_noalloc: no current CUDA device: ") + cudaGetErrorString(e));
        return HS_ERR_CUDA;
    }
    if (dev < 0 || dev >= 128) {
        set_error("hs_dot_noalloc: device ordinal exceeds 128 (the per-device address cache)");
        return HS_ERR_CUDA;
    }
    double* scratch = nullptr;
    {
        // first call on a device: look up the array's device address with that
        // device current (the symbol's host-side name is not a device address)
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            e = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_addr[dev]), g_noalloc_partials);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                set_error(std::string("hs_dot_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
                return HS_ERR_CUDA;
            }
        }
        scratch = g_addr[dev];
    }
    // every partial slot read (q = 0, blocks 0..nflat-1) is written by this
    // call's k_reduce before k_final_dot_noalloc reads it: nothing to clear
    RedArgs r{Nn, nflat, N, RED_DOT, x, y, scratch, nullptr, nullptr};
    k_reduce<<<(int)nflat, RT, 0, 0>>>(r);
    k_final_dot_noalloc<<<1, RT, 0, 0>>>(nflat, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("hs_dot_noalloc: launch failed: ") + cudaGetErrorString(e));
        return HS_ERR_CUDA;
    }
    return HS_OK;
}
