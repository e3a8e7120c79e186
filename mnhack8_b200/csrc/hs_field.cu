// hs_field.cu -- lognormal conductivity fields generated on the device
// (included by hs_solver.cu; used by hs_field_lognormal and by the batched
// solver's hs_batch_add_lognormal).
//
// The reference's generator (scripts/gen_field.py:29-61) draws white noise on
// the n^3 element grid, filters it in Fourier space by the square root of the
// spectrum of the periodic covariance exp(-r^2/L^2), standardises the result
// to mean 0 and variance 1 and sets k = exp(mu + sigma g).  The square-root
// spectrum exp(-|k|^2 L^2 / 8) is, in real space, the Gaussian kernel
// exp(-2 r^2 / L^2) (standard deviation L/2), so the same filtering is a
// periodic convolution that separates into three 1-D passes (z, y, x); the
// kernel is cut at 6 standard deviations (weights below 1.6e-8 of the
// centre) and wraps around the period like the FFT's.  The white noise comes
// from a counter-based generator: SplitMix64 (G. L. Steele, D. Lea and C. H.
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014) of
// the seed and the element index, turned into a normal by the Box-Muller
// transform.  This is not NumPy's stream, so a field is not the reference
// generator's field bit for bit (the host restatement in fields.py is); it
// is a field of the same law, a fixed function of (N, seed, L, mu, sigma):
// the standardisation uses the library's fixed-order reductions.
#include <cuda_runtime.h>

namespace hs {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// uniform in (0, 1]: the top 53 bits of a 64-bit word
__device__ __forceinline__ double u01(unsigned long long w) { return ((double)(w >> 11) + 1.0) * 0x1.0p-53; }

// g[e] ~ N(0, 1), independent over e, a fixed function of (seed, e)
__global__ void k_field_noise(long long ne, unsigned long long seed, double* g) {
    const unsigned long long key = splitmix64(seed);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
        const unsigned long long c = key + 2ull * (unsigned long long)e;
        const double u1 = u01(splitmix64(c)), u2 = u01(splitmix64(c + 1ull));
        g[e] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
}

// one periodic 1-D Gaussian pass along axis (0: x, 1: y, 2: z) of an n^3
// grid: out[i] = sum_t w(t) in[i + t e_axis mod n], t = -R..R, w(t) =
// exp(-t^2 / (2 s^2)) (s in cells), weights built once per block
constexpr int kFieldMaxTaps = 4096;
__global__ void k_field_conv(int n, int axis, int R, double s, const double* in, double* out) {
    __shared__ double w[kFieldMaxTaps];
    const int taps = 2 * R + 1;
    for (int t = threadIdx.x; t < taps; t += blockDim.x) {
        const double d = (double)(t - R);
        w[t] = exp(-d * d / (2.0 * s * s));
    }
    __syncthreads();
    const long long nn = (long long)n * n, ne = nn * n;
    const long long stride = axis == 0 ? nn : axis == 1 ? (long long)n : 1;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(axis == 0 ? e / nn : axis == 1 ? (e / n) % n : e % n);
        const long long base = e - (long long)c * stride;
        int j = ((c - R) % n + n) % n;
        double acc = 0.0;
        for (int t = 0; t < taps; ++t) {
            acc = __fma_rn(w[t], __ldg(in + base + (long long)j * stride), acc);
            j = (j + 1 == n) ? 0 : j + 1;
        }
        out[e] = acc;
    }
}

// block partials of sum(g) (pass 0) or sum((g - mean)^2) (pass 1, mean from stats[0])
__global__ void __launch_bounds__(RT) k_field_moment(long long ne, int pass, const double* g, const double* stats,
                                                     double* partials, long long nblk) {
    __shared__ double sh[MAXQ][8];
    const double mean = pass ? stats[0] : 0.0;
    double v[1] = {0.0};
    const long long e0 = ((long long)blockIdx.x * RT + threadIdx.x) * KF;
#pragma unroll
    for (int k = 0; k < KF; ++k) {
        const long long e = e0 + k;
        if (e >= ne) break;
        const double x = g[e];
        if (pass) { const double d = dsub(x, mean); v[0] = dfma(d, d, v[0]); }
        else v[0] = dadd(v[0], x);
    }
    store_partials<1>(v, partials, nblk, sh);
}
// stats[0] = mean (pass 0) or stats[1] = standard deviation (pass 1)
__global__ void __launch_bounds__(RT) k_field_moment_final(long long ne, int pass, const double* partials,
                                                           long long nblk, double* stats) {
    __shared__ double sh[MAXQ][8];
    double v[1];
    final_sums<1>(v, partials, nblk, sh);
    if (threadIdx.x != 0) return;
    if (pass == 0) stats[0] = __ddiv_rn(v[0], (double)ne);
    else stats[1] = __dsqrt_rn(__ddiv_rn(v[0], (double)ne));
}
// k = exp(mu + sigma (g - mean) / std), rho*c = rhoc (g is read from rh)
__global__ void k_field_finish(long long ne, double mu, double sigma, double rhoc, const double* stats, double* k,
                               double* rh) {
    const double mean = stats[0], sd = stats[1];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
        const double g = __ddiv_rn(dsub(rh[e], mean), sd);
        k[e] = exp(dfma(sigma, g, mu));
        rh[e] = rhoc;
    }
}

struct FieldSpecDev {
    int N;
    double mu, sigma, L, rhoc;
    unsigned long long seed;
};

// Taps of the 1-D pass for correlation length L (domain units) on an n-cell period
inline void field_taps(int n, double L, int* R, double* s) {
    *s = 0.5 * L * n;                       // L/2 in cells
    int r = (int)std::ceil(6.0 * *s);
    if (r < 1) r = 1;
    const int rmax = (kFieldMaxTaps - 1) / 2;
    *R = r > rmax ? rmax : r;
}

// Enqueue a lognormal field on stream st into k and rh (N^3 doubles each; rh
// is also the working buffer).  partials: ceil(N^3 / (RT*KF)) doubles;
// stats: 2 doubles.
inline cudaError_t enqueue_field_lognormal(const FieldSpecDev& f, double* k, double* rh, double* partials,
                                           double* stats, cudaStream_t st) {
    const int n = f.N;
    const long long ne = (long long)n * n * n;
    const long long nblk = (ne + (long long)RT * KF - 1) / ((long long)RT * KF);
    int R = 1;
    double s = 1.0;
    field_taps(n, f.L, &R, &s);
    const int g = (int)std::min<long long>((ne + RT - 1) / RT, 148 * 32);
    k_field_noise<<<g, RT, 0, st>>>(ne, f.seed, k);
    k_field_conv<<<g, RT, 0, st>>>(n, 2, R, s, k, rh);    // z
    k_field_conv<<<g, RT, 0, st>>>(n, 1, R, s, rh, k);    // y
    k_field_conv<<<g, RT, 0, st>>>(n, 0, R, s, k, rh);    // x
    for (int pass = 0; pass < 2; ++pass) {
        k_field_moment<<<(int)nblk, RT, 0, st>>>(ne, pass, rh, stats, partials, nblk);
        k_field_moment_final<<<1, RT, 0, st>>>(ne, pass, partials, nblk, stats);
    }
    k_field_finish<<<g, RT, 0, st>>>(ne, f.mu, f.sigma, f.rhoc, stats, k, rh);
    return cudaGetLastError();
}

}  // namespace hs

extern "C" hs_status hs_field_lognormal(int N, double mu, double sigma, double L, unsigned long long seed,
                                        double rhoc, double* k_dev, double* rhoc_dev) {
    using namespace hs;
    if (N < 1 || N > 1200 || !(sigma >= 0) || !(L > 0) || !(rhoc > 0) || !k_dev || !rhoc_dev) {
        set_error("hs_field_lognormal: bad arguments");
        return HS_ERR_ARG;
    }
    const long long ne = (long long)N * N * N;
    const long long nblk = (ne + (long long)RT * KF - 1) / ((long long)RT * KF);
    double* scratch = nullptr;
    cudaError_t e = cudaMalloc(&scratch, (size_t)(nblk + 2) * sizeof(double));
    if (e != cudaSuccess) { set_error(std::string("hs_field_lognormal: ") + cudaGetErrorString(e)); return HS_ERR_CUDA; }
    FieldSpecDev f{N, mu, sigma, L, rhoc, seed};
    e = enqueue_field_lognormal(f, k_dev, rhoc_dev, scratch + 2, scratch, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    cudaFree(scratch);
    if (e != cudaSuccess) { set_error(std::string("hs_field_lognormal: ") + cudaGetErrorString(e)); return HS_ERR_CUDA; }
    return HS_OK;
}
