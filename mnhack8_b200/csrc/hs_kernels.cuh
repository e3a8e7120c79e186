// hs_kernels.cuh -- sm_100a kernels of libheat_b200 (included by hs_solver.cu).
//
// All arithmetic is spelled out with round-to-nearest intrinsics (__dadd_rn,
// __dmul_rn, __fma_rn, __ddiv_rn, __dsqrt_rn) and the file is compiled with
// --fmad=false, so no operation is contracted or reordered by the compiler:
// the deterministic ("colored") path is a fixed function of its inputs.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "hs_types.h"

namespace hs {

// element-operator constants, passed by value (kernel parameter space)
struct ElemConsts {
    double M[64];      // Gauss-built M^ (het.cu:661-676), local-node order
    double K[64];      // Gauss-built K^
    double cm[4];      // wht: mass eigenvalue / 8 by Walsh index weight
    double ck[4];      // wht: stiffness eigenvalue / 8
    double detJ;       // gauss form
    const double* gtab;  // gauss form: [4][8 points][8 nodes] N, dNx, dNy, dNz
};

// local node i <-> q = ox<<2 | oy<<1 | oz   (het.cu:261-264)
__device__ __constant__ int kQofLocal[8] = {0, 4, 6, 2, 1, 5, 7, 3};

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double flipbit(double x, int bit) {
    return __longlong_as_double(__double_as_longlong(x) ^ (long long)(1ULL << bit));
}

// ---- element operators; v[8] in q-order, in place --------------------------
__device__ __forceinline__ void butterfly(double* v, int bit) {
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (!(q & bit)) {
            double u = v[q], w = v[q | bit];
            v[q] = dadd(u, w);
            v[q | bit] = dsub(u, w);
        }
}

// A_e = (1/8) H diag(lambda) H with H the 8-point Walsh-Hadamard matrix: the
// Q1 cube element's M^ = m (x) m (x) m and K^ = k(x)m(x)m + m(x)k(x)m +
// m(x)m(x)k share the eigenvectors of the 1D factors m = h/6 [2 1; 1 2] and
// k = 1/h [1 -1; -1 1] ([1,1]: h/2 and 0; [1,-1]: h/6 and 2/h).
__device__ __forceinline__ void elem_wht(double* v, double rhoc, double dk, const ElemConsts& c) {
    butterfly(v, 1);
    butterfly(v, 2);
    butterfly(v, 4);
    const double l0 = dmul(rhoc, c.cm[0]);
    const double l1 = dfma(dk, c.ck[1], dmul(rhoc, c.cm[1]));
    const double l2 = dfma(dk, c.ck[2], dmul(rhoc, c.cm[2]));
    const double l3 = dfma(dk, c.ck[3], dmul(rhoc, c.cm[3]));
    v[0] = dmul(v[0], l0);
    v[1] = dmul(v[1], l1); v[2] = dmul(v[2], l1); v[4] = dmul(v[4], l1);
    v[3] = dmul(v[3], l2); v[5] = dmul(v[5], l2); v[6] = dmul(v[6], l2);
    v[7] = dmul(v[7], l3);
    butterfly(v, 1);
    butterfly(v, 2);
    butterfly(v, 4);
}

// het.cu:340-349 with the multiply-adds made explicit
__device__ __forceinline__ void elem_fast(double* v, double rhoc, double dk, const ElemConsts& c) {
    double xl[8], yl[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) xl[i] = v[kQofLocal[i]];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            double a = dfma(rhoc, c.M[i * 8 + j], dmul(dk, c.K[i * 8 + j]));
            acc = dfma(a, xl[j], acc);
        }
        yl[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[kQofLocal[i]] = yl[i];
}

// het.cu:310-338 with the multiply-adds made explicit
__device__ __forceinline__ void elem_gauss(double* v, double rhoc, double ke, double dt_eff, const ElemConsts& c) {
    const double* gN = c.gtab;
    const double* gx = c.gtab + 64;
    const double* gy = c.gtab + 128;
    const double* gz = c.gtab + 192;
    double xl[8], yl[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) { xl[i] = v[kQofLocal[i]]; yl[i] = 0.0; }
    for (int g = 0; g < 8; ++g) {
        for (int i = 0; i < 8; ++i) {
            double Mx = 0.0, Kx = 0.0;
            const double ni = __ldg(gN + g * 8 + i);
            const double xi = __ldg(gx + g * 8 + i), yi = __ldg(gy + g * 8 + i), zi = __ldg(gz + g * 8 + i);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                double tm = dmul(dmul(rhoc, ni), __ldg(gN + g * 8 + j));
                Mx = dfma(tm, xl[j], Mx);
                double gg = dfma(zi, __ldg(gz + g * 8 + j), dfma(yi, __ldg(gy + g * 8 + j), dmul(xi, __ldg(gx + g * 8 + j))));
                Kx = dfma(dmul(ke, gg), xl[j], Kx);
            }
            yl[i] = dfma(c.detJ, dfma(dt_eff, Kx, Mx), yl[i]);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[kQofLocal[i]] = yl[i];
}

template <int FORM>
__device__ __forceinline__ void elem_apply(double* v, double rhoc, double kc, double dt_eff, const ElemConsts& c) {
    if (FORM == FORM_WHT) elem_wht(v, rhoc, dmul(dt_eff, kc), c);
    else if (FORM == FORM_FAST) elem_fast(v, rhoc, dmul(dt_eff, kc), c);
    else elem_gauss(v, rhoc, kc, dt_eff, c);
}

// ---- partition helpers --------------------------------------------------------
struct Part {
    int N, NN, I;
    int NTX, NTY, NTZ;
    long long ntiles, NB, nbb, nblk;
};

__host__ __device__ inline Part make_part(int N) {
    Part p;
    p.N = N; p.NN = N + 1; p.I = N - 1;
    if (p.I > 0) {
        p.NTX = (p.I + CX - 1) / CX; p.NTY = (p.I + TY - 1) / TY; p.NTZ = (p.I + TZ - 1) / TZ;
        p.ntiles = (long long)p.NTX * p.NTY * p.NTZ;
    } else {
        p.NTX = p.NTY = p.NTZ = 0; p.ntiles = 0;
    }
    long long NN = p.NN;
    p.NB = NN * NN * NN - (long long)p.I * p.I * p.I;
    p.nbb = (p.NB + (long long)RT * BPT - 1) / ((long long)RT * BPT);
    p.nblk = p.ntiles + p.nbb;
    return p;
}

// j-th boundary node in increasing node index
__device__ __forceinline__ long long bnd_node(long long j, int N) {
    const long long NN = N + 1, P = NN * NN;
    if (j < P) return j;
    long long jj = j - P;
    const long long R = 4LL * N;
    if (jj < (long long)(N - 1) * R) {
        long long ix = 1 + jj / R, r = jj % R, iy, iz;
        if (r < NN) { iy = 0; iz = r; }
        else if (r < NN + 2LL * (N - 1)) { long long t = r - NN; iy = 1 + t / 2; iz = (t & 1) ? N : 0; }
        else { iy = N; iz = r - NN - 2LL * (N - 1); }
        return (ix * NN + iy) * NN + iz;
    }
    jj -= (long long)(N - 1) * R;
    return (long long)N * P + jj;
}

__device__ __forceinline__ bool is_bnd(long long n, int N) {
    const long long NN = N + 1;
    int ix = (int)(n / (NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
    return ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N;
}

// ---- canonical CTA tree ----------------------------------------------------------
// sum over the RT threads of the CTA: xor butterfly inside each warp, then an
// 8-way xor butterfly over the warp sums; result valid in thread 0.
template <int NQ>
__device__ __forceinline__ void cta_tree_sum(double (&v)[NQ], double (*sh)[8]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) v[q] = dadd(v[q], __shfl_xor_sync(0xffffffffu, v[q], off));
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) sh[q][warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double u = (lane < 8) ? sh[q][lane] : 0.0;
#pragma unroll
            for (int off = 4; off >= 1; off >>= 1) u = dadd(u, __shfl_xor_sync(0xffffffffu, u, off));
            v[q] = u;
        }
    }
}

template <int NQ>
__device__ __forceinline__ void cta_tree_minmax(double& mn, double& mx, double (*sh)[8]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, off));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    __syncthreads();
    if (lane == 0) { sh[0][warp] = mn; sh[1][warp] = mx; }
    __syncthreads();
    if (warp == 0) {
        double a = (lane < 8) ? sh[0][lane] : 1e300, b = (lane < 8) ? sh[1][lane] : -1e300;
#pragma unroll
        for (int off = 4; off >= 1; off >>= 1) {
            a = fmin(a, __shfl_xor_sync(0xffffffffu, a, off));
            b = fmax(b, __shfl_xor_sync(0xffffffffu, b, off));
        }
        mn = a; mx = b;
    }
}

// Write the CTA partials, take a ticket; returns true in the last CTA, which
// then holds the final canonical sums in v (thread 0).
template <int NQ>
__device__ __forceinline__ bool reduce_partials(double (&v)[NQ], double* partials, unsigned* ticket,
                                                long long nblk, double (*sh)[8]) {
    __shared__ unsigned s_last;
    cta_tree_sum<NQ>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[q * nblk + blockIdx.x] = v[q];
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        s_last = (t == (unsigned)(nblk - 1));
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double acc = 0.0;
        for (long long k = threadIdx.x; k < nblk; k += RT) acc = dadd(acc, __ldcg(partials + q * nblk + k));
        v[q] = acc;
    }
    cta_tree_sum<NQ>(v, sh);
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// ---- operator application: colored (deterministic gather) --------------------
struct ApplyArgs {
    int N, role, form_pad;
    double dt_eff;
    const double* x;        // input (roles other than LOOP)
    const double* z;        // LOOP: preconditioned residual
    double* pbuf0;          // LOOP: p double buffer, p_k in pbuf[k & 1]
    double* pbuf1;
    double* y;              // output
    const double* rhoc;
    const double* kc;
    const double* w;        // ABFT weight (w_M or w_A) or null
    const double* F;        // ROLE_RHS source (null: none)
    double dtF;
    int d1;                 // evaluate the D1 checksum
    int pad1;
    double* partials;
    unsigned* ticket;
    DevState* st;
    ElemConsts ec;
};

struct NodeLoader {
    int role, iter;
    double beta;
    const double* x;
    const double* z;
    const double* pin;
    int fi_p;
    long long fi_idx;
    int fi_bit;

    __device__ __forceinline__ void fetch(long long n, double& a, double& b) const {
        if (role == ROLE_LOOP) {
            a = __ldg(z + n);
            b = (iter > 0) ? __ldg(pin + n) : 0.0;
        } else {
            a = __ldg(x + n);
            b = 0.0;
        }
    }
    __device__ __forceinline__ double make(long long n, double a, double b) const {
        if (role != ROLE_LOOP) return a;
        double p = (iter > 0) ? dfma(beta, b, a) : a;
        if (fi_p && n == fi_idx) p = flipbit(p, fi_bit);
        return p;
    }
};

template <int FORM>
__global__ void __launch_bounds__(RT, 2) k_apply_colored(ApplyArgs a) {
    __shared__ double xs[3][LY][LZ];
    __shared__ double yes[8][NELEM];
    __shared__ double sh[MAXQ][8];

    DevState* st = a.st;
    const int N = a.N;
    const long long NN = N + 1;
    const Part P = make_part(N);
    const int tid = threadIdx.x;

    NodeLoader L;
    L.role = a.role; L.iter = 0; L.beta = 0.0; L.x = a.x; L.z = a.z; L.pin = nullptr;
    L.fi_p = 0; L.fi_idx = -1; L.fi_bit = 0;
    double* pout = nullptr;
    int fi_ap = 0, fi_r = 0;
    long long fi_idx = -1, fi_elem = -1;
    int fi_bit = 0;
    if (a.role == ROLE_LOOP) {
        if (st->done) return;                       // uniform: the loop has ended
        L.iter = st->iter; L.beta = st->beta;
        L.pin = (L.iter & 1) ? a.pbuf0 : a.pbuf1;   // p_{k-1}
        pout = (L.iter & 1) ? a.pbuf1 : a.pbuf0;    // p_k
        if (st->fi_vec && st->fi_iter == L.iter) {
            fi_idx = st->fi_idx; fi_bit = st->fi_bit;
            L.fi_p = (st->fi_vec == FI_P); L.fi_idx = fi_idx; L.fi_bit = fi_bit;
            fi_ap = (st->fi_vec == FI_AP);
        }
    } else if (a.role == ROLE_X0 && st->fi_armR) {
        fi_r = 1; fi_elem = st->fi_elem; fi_bit = st->fi_bit;
    }
    const bool d1 = a.d1 != 0;
    const bool rhs = (a.role == ROLE_RHS) && a.F != nullptr;
    double part[MAXQ] = {0.0, 0.0, 0.0, 0.0};   // pAp, s, c, nx

    if (blockIdx.x < P.ntiles) {
        // ---------------- interior tile ----------------
        const long long t = blockIdx.x;
        const int tz = (int)(t % P.NTZ), ty = (int)((t / P.NTZ) % P.NTY), tx = (int)(t / ((long long)P.NTZ * P.NTY));
        const int y0 = 1 + ty * TY, z0 = 1 + tz * TZ;
        const int xa = 1 + tx * CX, xb = min(tx * CX + CX, P.I);
        const int ly = tid / TZ, lz = tid % TZ;
        const int iy = y0 + ly, iz = z0 + lz;
        const bool node_ok = (iy <= P.I) && (iz <= P.I);

        // load slots s0 = tid, s1 = tid + RT
        const int s1 = tid + RT;
        const bool has_s1 = s1 < NLOAD;
        const int sy0 = tid / LZ, sz0 = tid % LZ;
        const int sy1 = s1 / LZ, sz1 = s1 % LZ;
        const int gy0 = y0 - 1 + sy0, gz0 = z0 - 1 + sz0;
        const int gy1 = y0 - 1 + sy1, gz1 = z0 - 1 + sz1;
        const bool ok0 = gy0 <= N && gz0 <= N;
        const bool ok1 = has_s1 && gy1 <= N && gz1 <= N;
        // element slots e0 = tid, e1 = tid + RT
        const int le1 = tid + RT;
        const bool has_e1 = le1 < NELEM;
        const int ey0 = y0 - 1 + tid / EZ, ez0 = z0 - 1 + tid % EZ;
        const int ey1 = y0 - 1 + le1 / EZ, ez1 = z0 - 1 + le1 % EZ;
        const bool ein0 = ey0 <= N - 1 && ez0 <= N - 1;
        const bool ein1 = has_e1 && ey1 <= N - 1 && ez1 <= N - 1;

        auto node_index = [&](int px, int gy, int gz) -> long long { return ((long long)px * NN + gy) * NN + gz; };
        auto fetch_plane = [&](int px, double& a0, double& b0, double& a1, double& b1) {
            a0 = b0 = a1 = b1 = 0.0;
            if (ok0) L.fetch(node_index(px, gy0, gz0), a0, b0);
            if (ok1) L.fetch(node_index(px, gy1, gz1), a1, b1);
        };
        auto store_plane = [&](int px, double a0, double b0, double a1, double b1) {
            double (*dst)[LZ] = xs[px % 3];
            dst[sy0][sz0] = ok0 ? L.make(node_index(px, gy0, gz0), a0, b0) : 0.0;
            if (has_s1) dst[sy1][sz1] = ok1 ? L.make(node_index(px, gy1, gz1), a1, b1) : 0.0;
        };
        auto fetch_coef = [&](int ex, double& r0, double& k0, double& r1, double& k1) {
            r0 = k0 = r1 = k1 = 0.0;
            const long long base = (long long)ex * N;
            if (ein0) { long long e = (base + ey0) * N + ez0; r0 = __ldg(a.rhoc + e); k0 = __ldg(a.kc + e); }
            if (ein1) { long long e = (base + ey1) * N + ez1; r1 = __ldg(a.rhoc + e); k1 = __ldg(a.kc + e); }
        };
        auto elem_one = [&](int ex, int le, int ey, int ez, bool in, double rc, double kk) {
            const int ley = le / EZ, lez = le % EZ;
            double v[8];
            const double (*lo)[LZ] = xs[ex % 3];
            const double (*hi)[LZ] = xs[(ex + 1) % 3];
            v[0] = lo[ley][lez];     v[1] = lo[ley][lez + 1];
            v[2] = lo[ley + 1][lez]; v[3] = lo[ley + 1][lez + 1];
            v[4] = hi[ley][lez];     v[5] = hi[ley][lez + 1];
            v[6] = hi[ley + 1][lez]; v[7] = hi[ley + 1][lez + 1];
            elem_apply<FORM>(v, rc, kk, a.dt_eff, a.ec);
            if (fi_r) {
                long long e = ((long long)ex * N + ey) * N + ez;
                if (e == fi_elem) v[0] = flipbit(v[0], fi_bit);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) yes[q][le] = in ? v[q] : 0.0;
        };
        auto elem_plane = [&](int ex, double r0, double k0, double r1, double k1) {
            elem_one(ex, tid, ey0, ez0, ein0, r0, k0);
            if (has_e1) elem_one(ex, le1, ey1, ez1, ein1, r1, k1);
        };
        // contributions of the element plane in yes[] to node (ly, lz): ox
        // selects the node plane (0: same plane as the elements, 1: next)
        auto gather4 = [&](double acc, int ox) -> double {
            const int base = ly * EZ + lz;
            acc = dadd(acc, yes[(ox << 2) | 3][base]);            // element (iy-1, iz-1)
            acc = dadd(acc, yes[(ox << 2) | 2][base + 1]);        // element (iy-1, iz)
            acc = dadd(acc, yes[(ox << 2) | 1][base + EZ]);       // element (iy,   iz-1)
            acc = dadd(acc, yes[(ox << 2) | 0][base + EZ + 1]);   // element (iy,   iz)
            return acc;
        };

        double pa0, pb0, pa1, pb1;   // prefetched node plane
        double cr0, ck0, cr1, ck1;   // prefetched coefficients
        // prologue: planes xa-1, xa into smem; element plane xa-1
        fetch_plane(xa - 1, pa0, pb0, pa1, pb1);
        store_plane(xa - 1, pa0, pb0, pa1, pb1);
        fetch_plane(xa, pa0, pb0, pa1, pb1);
        store_plane(xa, pa0, pb0, pa1, pb1);
        fetch_coef(xa - 1, cr0, ck0, cr1, ck1);
        fetch_plane(xa + 1, pa0, pb0, pa1, pb1);
        __syncthreads();
        elem_plane(xa - 1, cr0, ck0, cr1, ck1);
        fetch_coef(xa, cr0, ck0, cr1, ck1);
        __syncthreads();
        double acc = node_ok ? gather4(0.0, 1) : 0.0;
        __syncthreads();

        for (int ix = xa; ix <= xb; ++ix) {
            store_plane(ix + 1, pa0, pb0, pa1, pb1);
            double nr0, nk0, nr1, nk1;
            if (ix + 2 <= xb + 1) fetch_plane(ix + 2, pa0, pb0, pa1, pb1);
            if (ix + 1 <= xb) fetch_coef(ix + 1, nr0, nk0, nr1, nk1);
            __syncthreads();
            elem_plane(ix, cr0, ck0, cr1, ck1);
            cr0 = nr0; ck0 = nk0; cr1 = nr1; ck1 = nk1;
            __syncthreads();
            if (node_ok) {
                double yv = gather4(acc, 0);
                acc = gather4(0.0, 1);
                const long long n = ((long long)ix * NN + iy) * NN + iz;
                const double pv = xs[ix % 3][ly + 1][lz + 1];
                if (fi_ap && n == fi_idx) yv = flipbit(yv, fi_bit);
                if (a.role == ROLE_LOOP) part[0] = dfma(pv, yv, part[0]);
                if (d1) {
                    part[1] = dadd(part[1], yv);
                    part[2] = dfma(__ldg(a.w + n), pv, part[2]);
                    part[3] = dfma(pv, pv, part[3]);
                }
                if (rhs) yv = dfma(a.dtF, __ldg(a.F + n), yv);
                a.y[n] = yv;
                if (pout) pout[n] = pv;
            }
            __syncthreads();
        }
    } else {
        // ---------------- boundary block ----------------
        const long long b = blockIdx.x - P.ntiles;
#pragma unroll 1
        for (int k = 0; k < BPT; ++k) {
            const long long j = b * (long long)(RT * BPT) + (long long)k * RT + tid;
            if (j >= P.NB) break;
            const long long n = bnd_node(j, N);
            double va, vb;
            L.fetch(n, va, vb);
            const double pv = L.make(n, va, vb);
            double yv = 0.0;
            if (fi_ap && n == fi_idx) yv = flipbit(yv, fi_bit);
            if (a.role == ROLE_LOOP) part[0] = dfma(pv, yv, part[0]);
            if (d1) {
                part[1] = dfma(0.0, yv, part[1]);
                part[2] = dfma(__ldg(a.w + n), pv, part[2]);
                part[3] = dfma(pv, pv, part[3]);
            }
            if (rhs) yv = dfma(a.dtF, __ldg(a.F + n), yv);
            a.y[n] = yv;
            if (pout) pout[n] = pv;
        }
    }

    if (a.role != ROLE_LOOP && !d1) return;
    if (!reduce_partials<MAXQ>(part, a.partials, a.ticket, P.nblk, sh)) return;
    if (threadIdx.x != 0) return;
    // ---- last CTA: role logic ----
    if (d1) {
        const double nw = (a.role == ROLE_RHS) ? st->norm_wM : st->norm_wA;
        const double nx = __dsqrt_rn(part[3]);
        double rel = __ddiv_rn(fabs(dsub(part[1], part[2])), dfma(nw, nx, 1e-300));
        if (!isfinite(rel)) rel = 1e300;
        st->d1_last = rel;
        if (a.role != ROLE_USER) st->d1_step = fmax(st->d1_step, rel);
    }
    if (a.role == ROLE_LOOP) {
        const double pAp = part[0];
        st->pAp = pAp;
        if (fabs(pAp) < 1e-30) {
            st->broken = 1; st->done = 1; st->result = st->iter;
        } else {
            st->alpha = __ddiv_rn(st->rho, pAp);
        }
    }
}

// ---- PCG vector update (canonical partition) -----------------------------------
struct UpdateArgs {
    int N, role;
    double* x;
    const double* b;
    double* r;
    double* z;
    const double* Ap;
    const double* d;
    const double* pbuf0;
    const double* pbuf1;
    double* partials;
    unsigned* ticket;
    DevState* st;
    cudaGraphConditionalHandle cond;
    int use_cond, pad;
};

__global__ void __launch_bounds__(RT) k_update(UpdateArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const int N = a.N;
    const long long NN = N + 1;
    const Part P = make_part(N);
    const int tid = threadIdx.x;
    if (a.role == UPD_LOOP && st->done) {
        if (a.use_cond && blockIdx.x == 0 && tid == 0) cudaGraphSetConditional(a.cond, 0u);
        return;
    }
    int iter = 0;
    double alpha = 0.0;
    const double* p = nullptr;
    int fi_r = 0, fi_bit = 0;
    long long fi_idx = -1;
    if (a.role == UPD_LOOP) {
        iter = st->iter; alpha = st->alpha;
        p = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec == FI_RV && st->fi_iter == iter) { fi_r = 1; fi_idx = st->fi_idx; fi_bit = st->fi_bit; }
    }
    const double nalpha = -alpha;
    double part[3] = {0.0, 0.0, 0.0};   // PRE: bb, rz, rr   LOOP: rr, rz, -

    auto node = [&](long long n) {
        if (a.role == UPD_PRE) {
            const double bv = __ldg(a.b + n);
            const double rv = dfma(-1.0, __ldg(a.Ap + n), bv);
            const double zv = __ddiv_rn(rv, __ldg(a.d + n));
            a.r[n] = rv; a.z[n] = zv;
            part[0] = dfma(bv, bv, part[0]);
            part[1] = dfma(rv, zv, part[1]);
            part[2] = dfma(rv, rv, part[2]);
        } else {
            a.x[n] = dfma(alpha, __ldg(p + n), a.x[n]);
            double rv = dfma(nalpha, __ldg(a.Ap + n), a.r[n]);
            if (fi_r && n == fi_idx) rv = flipbit(rv, fi_bit);
            const double zv = __ddiv_rn(rv, __ldg(a.d + n));
            a.r[n] = rv; a.z[n] = zv;
            part[0] = dfma(rv, rv, part[0]);
            part[1] = dfma(rv, zv, part[1]);
        }
    };
    if (blockIdx.x < P.ntiles) {
        const long long t = blockIdx.x;
        const int tz = (int)(t % P.NTZ), ty = (int)((t / P.NTZ) % P.NTY), tx = (int)(t / ((long long)P.NTZ * P.NTY));
        const int iy = 1 + ty * TY + tid / TZ, iz = 1 + tz * TZ + tid % TZ;
        if (iy <= P.I && iz <= P.I) {
            const int xa = 1 + tx * CX, xb = min(tx * CX + CX, P.I);
            for (int ix = xa; ix <= xb; ++ix) node(((long long)ix * NN + iy) * NN + iz);
        }
    } else {
        const long long b = blockIdx.x - P.ntiles;
#pragma unroll 1
        for (int k = 0; k < BPT; ++k) {
            const long long j = b * (long long)(RT * BPT) + (long long)k * RT + tid;
            if (j >= P.NB) break;
            node(bnd_node(j, N));
        }
    }
    if (!reduce_partials<3>(part, a.partials, a.ticket, P.nblk, sh)) return;
    if (tid != 0) return;
    if (a.role == UPD_PRE) {
        double bnorm = __dsqrt_rn(part[0]);
        if (bnorm < 1e-30) bnorm = 1.0;
        st->bnorm = bnorm;
        st->rho = part[1];
        st->rel0 = __ddiv_rn(__dsqrt_rn(part[2]), bnorm);
        st->iter = 0; st->broken = 0; st->result = 0; st->beta = 0.0;
        st->done = (st->max_iter <= 0) ? 1 : 0;
    } else {
        const double rnorm = __dsqrt_rn(part[0]);
        const double rel = __ddiv_rn(rnorm, st->bnorm);
        const bool conv = rel < st->tol;
        double beta = 0.0;
        if (!conv) { beta = __ddiv_rn(part[1], st->rho); st->rho = part[1]; }
        if (st->log_rel && iter < st->log_cap) {
            st->log_rel[iter] = rel; st->log_alpha[iter] = alpha; st->log_beta[iter] = beta;
        }
        st->beta = beta;
        if (conv) { st->result = iter + 1; st->done = 1; }
        else {
            st->iter = iter + 1;
            if (iter + 1 >= st->max_iter) { st->done = 1; st->result = st->max_iter; }
        }
        if (a.use_cond) cudaGraphSetConditional(a.cond, st->done ? 0u : 1u);
    }
}

// ---- generic reductions over node vectors (canonical partition) ---------------
enum RedKind {
    RED_DOT = 0,        // q0 = x.y
    RED_RESID = 1,      // r = b - Ap: q0 = r.r, q1 = b.b
    RED_DIFF = 2,       // d = a - b: q0 = d.d, q1 = b.b
    RED_ABFT_S = 3      // q0 = 1_int . y
};
struct RedArgs {
    int N, kind;
    const double* a;
    const double* b;
    double* partials;
    unsigned* ticket;
    double* out;     // NQ results (device)
};

__global__ void __launch_bounds__(RT) k_reduce(RedArgs a) {
    __shared__ double sh[MAXQ][8];
    const int N = a.N;
    const long long NN = N + 1;
    const Part P = make_part(N);
    const int tid = threadIdx.x;
    double part[2] = {0.0, 0.0};
    auto node = [&](long long n, bool bnd) {
        switch (a.kind) {
            case RED_DOT: part[0] = dfma(__ldg(a.a + n), __ldg(a.b + n), part[0]); break;
            case RED_RESID: {
                const double bv = __ldg(a.b + n);
                const double rv = dfma(-1.0, __ldg(a.a + n), bv);
                part[0] = dfma(rv, rv, part[0]);
                part[1] = dfma(bv, bv, part[1]);
            } break;
            case RED_DIFF: {
                const double bv = __ldg(a.b + n);
                const double dv = dsub(__ldg(a.a + n), bv);
                part[0] = dfma(dv, dv, part[0]);
                part[1] = dfma(bv, bv, part[1]);
            } break;
            default: part[0] = dfma(bnd ? 0.0 : 1.0, __ldg(a.a + n), part[0]); break;
        }
    };
    if (blockIdx.x < P.ntiles) {
        const long long t = blockIdx.x;
        const int tz = (int)(t % P.NTZ), ty = (int)((t / P.NTZ) % P.NTY), tx = (int)(t / ((long long)P.NTZ * P.NTY));
        const int iy = 1 + ty * TY + tid / TZ, iz = 1 + tz * TZ + tid % TZ;
        if (iy <= P.I && iz <= P.I) {
            const int xa = 1 + tx * CX, xb = min(tx * CX + CX, P.I);
            for (int ix = xa; ix <= xb; ++ix) node(((long long)ix * NN + iy) * NN + iz, false);
        }
    } else {
        const long long b = blockIdx.x - P.ntiles;
#pragma unroll 1
        for (int k = 0; k < BPT; ++k) {
            const long long j = b * (long long)(RT * BPT) + (long long)k * RT + tid;
            if (j >= P.NB) break;
            node(bnd_node(j, N), true);
        }
    }
    if (!reduce_partials<2>(part, a.partials, a.ticket, P.nblk, sh)) return;
    if (tid == 0) { a.out[0] = part[0]; a.out[1] = part[1]; }
}

// min / max over all nodes with the reference's fmin/fmax semantics
// (het.cu:506-534: NaN entries are ignored, initial values +-1e300)
__global__ void __launch_bounds__(RT) k_minmax(int N, const double* x, double* partials, unsigned* ticket,
                                              double* out2) {
    __shared__ double sh[MAXQ][8];
    __shared__ unsigned s_last;
    const long long Nn = (long long)(N + 1) * (N + 1) * (N + 1);
    double mn = 1e300, mx = -1e300;
    for (long long n = (long long)blockIdx.x * RT + threadIdx.x; n < Nn; n += (long long)gridDim.x * RT) {
        const double v = __ldg(x + n);
        mn = fmin(mn, v); mx = fmax(mx, v);
    }
    cta_tree_minmax<2>(mn, mx, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = mn; partials[gridDim.x + blockIdx.x] = mx;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    mn = 1e300; mx = -1e300;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += RT) {
        mn = fmin(mn, __ldcg(partials + k)); mx = fmax(mx, __ldcg(partials + gridDim.x + k));
    }
    cta_tree_minmax<2>(mn, mx, sh);
    if (threadIdx.x == 0) { out2[0] = mn; out2[1] = mx; *ticket = 0u; }
}

// max |a-b| (NaN ignored) as an ordered bit pattern; then count |a-b| > thr*max
__global__ void k_absdiff_max(long long Nn, const double* a, const double* b, unsigned long long* out) {
    double m = 0.0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < Nn; n += (long long)gridDim.x * blockDim.x) {
        const double d = fabs(dsub(__ldg(a + n), __ldg(b + n)));
        if (d > m) m = d;
    }
    for (int off = 16; off >= 1; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
__global__ void k_absdiff_count(long long Nn, const double* a, const double* b, const unsigned long long* gmax,
                                double rel, unsigned long long* count) {
    const double thr = dmul(rel, __longlong_as_double((long long)*gmax));
    unsigned long long c = 0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < Nn; n += (long long)gridDim.x * blockDim.x) {
        const double d = fabs(dsub(__ldg(a + n), __ldg(b + n)));
        if (d > thr) ++c;
    }
    for (int off = 16; off >= 1; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// ---- node-parallel operator (every node, any projection) -------------------------
// Recomputes the eight elements around each node; bit-identical node values to
// k_apply_colored (same element arithmetic, same summation order).  Used for
// the unprojected set-up applies and the diagonal.
enum GenKind { GEN_APPLY = 0, GEN_DIAG = 1 };
struct GenArgs {
    int N, kind, project, fire_r;
    double dt_eff;
    const double* x;
    double* y;
    const double* rhoc;
    const double* kc;
    long long fi_elem;
    int fi_bit, pad;
    ElemConsts ec;
};

template <int FORM>
__global__ void __launch_bounds__(RT) k_apply_nodes(GenArgs a) {
    const int N = a.N;
    const long long NN = N + 1, Nn = NN * NN * NN;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nn) return;
    const int ix = (int)(n / (NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
    const bool bnd = ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N;
    double acc = 0.0;
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        const int ao = (s >> 2) & 1, bo = (s >> 1) & 1, co = s & 1;
        const int ex = ix - 1 + ao, ey = iy - 1 + bo, ez = iz - 1 + co;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= N || ey >= N || ez >= N) continue;
        const long long e = ((long long)ex * N + ey) * N + ez;
        const int qn = ((1 - ao) << 2) | ((1 - bo) << 1) | (1 - co);
        double c;
        if (a.kind == GEN_DIAG) {
            const int i = (qn == 0) ? 0 : (qn == 4) ? 1 : (qn == 6) ? 2 : (qn == 2) ? 3 : (qn == 1) ? 4 : (qn == 5) ? 5 : (qn == 7) ? 6 : 7;
            const double dk = dmul(a.dt_eff, __ldg(a.kc + e));
            c = dfma(__ldg(a.rhoc + e), a.ec.M[i * 9], dmul(dk, a.ec.K[i * 9]));
        } else {
            double v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                v[q] = __ldg(a.x + (((long long)(ex + ((q >> 2) & 1)) * NN + ey + ((q >> 1) & 1)) * NN + ez + (q & 1)));
            elem_apply<FORM>(v, __ldg(a.rhoc + e), __ldg(a.kc + e), a.dt_eff, a.ec);
            if (a.fire_r && e == a.fi_elem) v[0] = flipbit(v[0], a.fi_bit);
            c = v[qn];
        }
        acc = dadd(acc, c);
    }
    if (bnd && a.project) acc = (a.kind == GEN_DIAG) ? 1.0 : 0.0;
    a.y[n] = acc;
}

// ---- atomic scatter (nondeterministic, the reference's production pattern) ----
struct AtomArgs {
    int N, role;
    double dt_eff;
    const double* x;        // input (roles other than LOOP)
    const double* pbuf0;    // LOOP: p_k in pbuf[k & 1]
    const double* pbuf1;
    double* y;
    const double* rhoc;
    const double* kc;
    const DevState* st;
    ElemConsts ec;
};
template <int FORM>
__global__ void __launch_bounds__(RT) k_apply_atomic(AtomArgs a) {
    const DevState* st = a.st;
    const double* x = a.x;
    if (a.role == ROLE_LOOP) {
        if (st->done) return;
        x = (st->iter & 1) ? a.pbuf1 : a.pbuf0;
    }
    const bool fire_r = (a.role == ROLE_X0) && st->fi_armR;
    const int N = a.N;
    const long long NN = N + 1, Ne = (long long)N * N * N;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const int ex = (int)(e / ((long long)N * N)), ey = (int)((e / N) % N), ez = (int)(e % N);
    double v[8];
    long long g[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        g[q] = ((long long)(ex + ((q >> 2) & 1)) * NN + ey + ((q >> 1) & 1)) * NN + ez + (q & 1);
        v[q] = __ldg(x + g[q]);
    }
    elem_apply<FORM>(v, __ldg(a.rhoc + e), __ldg(a.kc + e), a.dt_eff, a.ec);
    if (fire_r && e == st->fi_elem) v[0] = flipbit(v[0], st->fi_bit);
#pragma unroll
    for (int q = 0; q < 8; ++q) atomicAdd(a.y + g[q], v[q]);
}

// After an atomic scatter: projection, p.Ap / D1 partials and role logic, on
// the canonical partition (p formed beforehand by k_form_p).
struct FinishArgs {
    int N, role, d1, pad;
    const double* p;     // the vector the operator was applied to (roles other than LOOP)
    const double* pbuf0; // LOOP: p_k in pbuf[k & 1]
    const double* pbuf1;
    double* y;
    const double* w;
    const double* F;
    double dtF;
    double* partials;
    unsigned* ticket;
    DevState* st;
};
__global__ void __launch_bounds__(RT) k_finish_atomic(FinishArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const int N = a.N;
    const long long NN = N + 1;
    const Part P = make_part(N);
    const int tid = threadIdx.x;
    int fi_ap = 0, fi_bit = 0;
    long long fi_idx = -1;
    int iter = 0;
    if (a.role == ROLE_LOOP) {
        if (st->done) return;
        iter = st->iter;
        if (st->fi_vec == FI_AP && st->fi_iter == iter) { fi_ap = 1; fi_idx = st->fi_idx; fi_bit = st->fi_bit; }
    }
    const double* p = (a.role == ROLE_LOOP) ? ((iter & 1) ? a.pbuf1 : a.pbuf0) : a.p;
    const bool rhs = (a.role == ROLE_RHS) && a.F != nullptr;
    double part[MAXQ] = {0.0, 0.0, 0.0, 0.0};
    auto node = [&](long long n, bool bnd) {
        double yv = bnd ? 0.0 : a.y[n];
        if (fi_ap && n == fi_idx) yv = flipbit(yv, fi_bit);
        const double pv = __ldg(p + n);
        if (a.role == ROLE_LOOP) part[0] = dfma(pv, yv, part[0]);
        if (a.d1) {
            part[1] = dfma(bnd ? 0.0 : 1.0, yv, part[1]);
            part[2] = dfma(__ldg(a.w + n), pv, part[2]);
            part[3] = dfma(pv, pv, part[3]);
        }
        if (rhs) yv = dfma(a.dtF, __ldg(a.F + n), yv);
        a.y[n] = yv;
    };
    if (blockIdx.x < P.ntiles) {
        const long long t = blockIdx.x;
        const int tz = (int)(t % P.NTZ), ty = (int)((t / P.NTZ) % P.NTY), tx = (int)(t / ((long long)P.NTZ * P.NTY));
        const int iy = 1 + ty * TY + tid / TZ, iz = 1 + tz * TZ + tid % TZ;
        if (iy <= P.I && iz <= P.I) {
            const int xa = 1 + tx * CX, xb = min(tx * CX + CX, P.I);
            for (int ix = xa; ix <= xb; ++ix) node(((long long)ix * NN + iy) * NN + iz, false);
        }
    } else {
        const long long b = blockIdx.x - P.ntiles;
#pragma unroll 1
        for (int k = 0; k < BPT; ++k) {
            const long long j = b * (long long)(RT * BPT) + (long long)k * RT + tid;
            if (j >= P.NB) break;
            node(bnd_node(j, N), true);
        }
    }
    if (a.role != ROLE_LOOP && !a.d1) return;
    if (!reduce_partials<MAXQ>(part, a.partials, a.ticket, P.nblk, sh)) return;
    if (tid != 0) return;
    if (a.d1) {
        const double nw = (a.role == ROLE_RHS) ? st->norm_wM : st->norm_wA;
        const double nx = __dsqrt_rn(part[3]);
        double rel = __ddiv_rn(fabs(dsub(part[1], part[2])), dfma(nw, nx, 1e-300));
        if (!isfinite(rel)) rel = 1e300;
        st->d1_last = rel;
        if (a.role != ROLE_USER) st->d1_step = fmax(st->d1_step, rel);
    }
    if (a.role == ROLE_LOOP) {
        const double pAp = part[0];
        st->pAp = pAp;
        if (fabs(pAp) < 1e-30) { st->broken = 1; st->done = 1; st->result = st->iter; }
        else st->alpha = __ddiv_rn(st->rho, pAp);
    }
}

// p_k = z (k = 0) or z + beta p_{k-1}, with the level-P fault (atomic path)
struct FormPArgs {
    long long Nn;
    const double* z;
    double* pbuf0;
    double* pbuf1;
    DevState* st;
};
__global__ void k_form_p(FormPArgs a) {
    const DevState* st = a.st;
    if (st->done) return;
    const int iter = st->iter;
    const double beta = st->beta;
    const double* pin = (iter & 1) ? a.pbuf0 : a.pbuf1;
    double* pout = (iter & 1) ? a.pbuf1 : a.pbuf0;
    const bool fp = st->fi_vec == FI_P && st->fi_iter == iter;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < a.Nn; n += (long long)gridDim.x * blockDim.x) {
        const double zv = __ldg(a.z + n);
        double p = (iter > 0) ? dfma(beta, __ldg(pin + n), zv) : zv;
        if (fp && n == st->fi_idx) p = flipbit(p, st->fi_bit);
        pout[n] = p;
    }
}

// ---- small kernels ------------------------------------------------------------------
__global__ void k_zero(long long n, double* v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) v[i] = 0.0;
}
__global__ void k_copy(long long n, const double* s, double* d) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) d[i] = s[i];
}
__global__ void k_jacobi(long long n, const double* r, const double* d, double* z) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        z[i] = __ddiv_rn(r[i], d[i]);
}
__global__ void k_set_boundary(int N, double* v, double val) {
    const long long NN = N + 1, Nn = NN * NN * NN;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < Nn; n += (long long)gridDim.x * blockDim.x)
        if (is_bnd(n, N)) v[n] = val;
}
__global__ void k_flip(double* v, long long idx, int bit) { v[idx] = flipbit(v[idx], bit); }
// step prologue: arm the step's fault, clear the step's checksum maximum
struct StepCtl {
    int armR, vec, iter, bit;
    long long elem, idx;
    int flipG, pad;
    long long gidx;
};
__global__ void k_step_begin(DevState* st, StepCtl c, double* T) {
    st->fi_armR = c.armR; st->fi_vec = c.vec; st->fi_iter = c.iter; st->fi_bit = c.bit;
    st->fi_elem = c.elem; st->fi_idx = c.idx;
    st->d1_step = 0.0;
    if (c.flipG) T[c.gidx] = flipbit(T[c.gidx], c.bit);
}
__global__ void k_disarm_R(DevState* st) { st->fi_armR = 0; }
__global__ void k_step_end(DevState* st, int* iters_out, double* d1_out) {
    st->fi_armR = 0; st->fi_vec = 0;
    *iters_out = st->result;
    *d1_out = st->d1_step;
}
__global__ void k_d2_finish(const double* red, double* d2_out) {
    double bn = __dsqrt_rn(red[1]);
    if (bn < 1e-300) bn = 1.0;
    *d2_out = __ddiv_rn(__dsqrt_rn(red[0]), bn);
}
__global__ void k_e_finish(const double* red, const unsigned long long* gmax, const unsigned long long* cnt,
                           long long Nn, double* E_out, double* spread_out) {
    double den = red[1];
    const double gm = __longlong_as_double((long long)*gmax);
    *spread_out = (gm > 0.0) ? __ddiv_rn((double)*cnt, (double)Nn) : 0.0;
    if (den < 1e-300) den = 1.0;
    *E_out = __dsqrt_rn(__ddiv_rn(red[0], den));
}

}  // namespace hs
