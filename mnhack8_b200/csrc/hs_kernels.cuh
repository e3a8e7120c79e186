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
// apply partition of an N-element grid (cx planes per tile)
struct Part {
    int N, NN, I, cx;
    int NTX, NTY, NTZ, pad;
    long long ntiles, NB, nbb, nblk;
    long long Nn, nflat;              // flat partition: blocks of RT*KF nodes
};

__host__ __device__ inline Part make_part(int N, int cx) {
    Part p;
    p.N = N; p.NN = N + 1; p.I = N - 1; p.cx = cx; p.pad = 0;
    if (p.I > 0) {
        p.NTX = (p.I + cx - 1) / cx; p.NTY = (p.I + TY - 1) / TY; p.NTZ = (p.I + TZ - 1) / TZ;
        p.ntiles = (long long)p.NTX * p.NTY * p.NTZ;
    } else {
        p.NTX = p.NTY = p.NTZ = 0; p.ntiles = 0;
    }
    long long NN = p.NN;
    p.Nn = NN * NN * NN;
    p.NB = p.Nn - (long long)p.I * p.I * p.I;
    p.nbb = (p.NB + (long long)RT * BPT - 1) / ((long long)RT * BPT);
    p.nblk = p.ntiles + p.nbb;
    p.nflat = (p.Nn + (long long)RT * KF - 1) / ((long long)RT * KF);
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
    if (lane == 0 && warp < 8) {       // threads beyond RT carry no values
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
        if (threadIdx.x < RT)
            for (long long k = threadIdx.x; k < nblk; k += RT) acc = dadd(acc, __ldcg(partials + q * nblk + k));
        v[q] = acc;
    }
    cta_tree_sum<NQ>(v, sh);
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// Combine the CTA's RT values (canonical tree) and store them as partial
// blockIdx.x of each quantity; the reduction is finished by a final kernel.
template <int NQ>
__device__ __forceinline__ void store_partials(double (&v)[NQ], double* partials, long long nblk, double (*sh)[8]) {
    cta_tree_sum<NQ>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[q * nblk + blockIdx.x] = v[q];
    }
}
// Final combination of nblk partials per quantity (one CTA of RT threads):
// RT strided sequential sums, then the canonical tree; valid in thread 0.
template <int NQ>
__device__ __forceinline__ void final_sums(double (&v)[NQ], const double* partials, long long nblk, double (*sh)[8]) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double acc = 0.0;
        for (long long k = threadIdx.x; k < nblk; k += RT) acc = dadd(acc, __ldcg(partials + q * nblk + k));
        v[q] = acc;
    }
    cta_tree_sum<NQ>(v, sh);
}

// ---- operator application: colored (deterministic gather) --------------------
struct ApplyArgs {
    Part part;
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

// cp.async (LDGSTS) 8-byte copies into shared memory; src-size 0 zero-fills
__device__ __forceinline__ void cp_async8(void* smem, const double* gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory"); }

// ---- colored operator, interior tiles: z-paired elements ----------------------
// A CTA of KT = 160 threads handles one TY x TZ tile of node columns streaming
// cx planes in x.  Element-pair thread p (< NPAIR) applies the two
// z-adjacent elements (ley, 2j) and (ley, 2j+1) of each plane, which share
// their common face; node-pair thread p (< NNPAIR) sums the contributions of
// node columns (ly, 2j) and (ly, 2j+1) in the canonical order (lower x-plane
// first, then (y, z)).  Node planes stream through a RING of shared-memory
// slots filled by cp.async, AHEAD planes in flight.
constexpr int KT = 160;
constexpr int PZ = TZ / 2 + 1;        // element pairs per row (the last one half outside the tile)
constexpr int NPAIR = EY * PZ;        // 153 element-pair threads
constexpr int NNPAIR = TY * TZ / 2;   // 128 node-pair threads
constexpr int LZ2 = 2 * PZ + 2;       // 36 node columns per loaded row (35 used, 16-byte rows)
constexpr int NL2 = LY * LZ2;         // 360 node values per loaded plane
constexpr int RING = 4;
constexpr int AHEAD = RING - 2;
static_assert(NPAIR <= KT && NNPAIR <= KT && KT % 32 == 0, "operator kernel thread count");
static_assert(TZ % 2 == 0 && TY * TZ == RT && TZ / 2 == 16, "pair layout: 16 node pairs per row (half a warp)");
struct __align__(16) ApplySmem {
    double raw_a[RING][NL2];    // x, or z in the PCG loop (cp.async ring)
    double raw_b[RING][NL2];    // p_{k-1} in the PCG loop
    double pf[2][NL2];          // formed input planes p (PCG loop)
    double2 yes[8][NPAIR];      // (element A, element B) outputs of each pair, by q
    double sh[MAXQ][8];
};
constexpr size_t kApplySmem = sizeof(ApplySmem);

__device__ __forceinline__ double2 lds2(const double* p) { return *reinterpret_cast<const double2*>(p); }

// MODE 0: input x as given; 1: PCG loop, p = z; 2: PCG loop, p = z + beta p_{k-1}
template <int FORM, int MODE>
__device__ __forceinline__ void apply_tile_pairs(const ApplyArgs& a, ApplySmem& S, int N, int xa, int xb, int y0,
                                                 int z0, const double* src_a, const double* src_b, double beta,
                                                 double* pout, bool loop, bool d1, bool rhs, int fi_p, int fi_ap,
                                                 int fi_r, int fi_bit, long long fi_idx, long long fi_elem,
                                                 double (&pa)[MAXQ], double (&pb)[MAXQ]) {
    constexpr bool FORMED = MODE > 0;
    constexpr bool TWO = MODE == 2;
    const int tid = threadIdx.x;
    const int NN = N + 1;
    const int plane = NN * NN, eplane = N * N;
    // ---- copy slots: t, t + KT, t + 2 KT (< NL2) of a LY x LZ2 halo plane
    int coff[3];
    bool cok[3], chas[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int sl = tid + k * KT;
        chas[k] = sl < NL2;
        const int row = sl / LZ2, col = sl % LZ2;
        const int gy = y0 - 1 + row, gz = z0 - 1 + col;
        cok[k] = chas[k] && col < LZ2 - 1 && gy <= N && gz <= N;
        coff[k] = cok[k] ? gy * NN + gz : 0;
    }
    // ---- element pair
    const bool has_e = tid < NPAIR;
    const int ley = tid / PZ, jp = tid % PZ;
    const int ey = y0 - 1 + ley, ez = z0 - 1 + 2 * jp;          // first element of the pair
    const bool einA = has_e && ey <= N - 1 && ez <= N - 1;
    const bool einB = has_e && ey <= N - 1 && ez + 1 <= N - 1;
    const int eoA = einA ? ey * N + ez : 0;
    const int eoB = einB ? ey * N + ez + 1 : 0;
    const int elo = ley * LZ2 + 2 * jp;                          // node (ey, ez) in a halo plane
    // ---- node pair
    const bool has_n = tid < NNPAIR;
    const int ly = tid / (TZ / 2), jn = tid % (TZ / 2);
    const int iy = y0 + ly, iz = z0 + 2 * jn;
    const bool nokA = has_n && iy <= N - 1 && iz <= N - 1;
    const bool nokB = has_n && iy <= N - 1 && iz + 1 <= N - 1;
    const int woff = iy * NN + iz;
    const int pr0 = ly * PZ + jn, pr1 = (ly + 1) * PZ + jn;      // pairs (iy-1, .) and (iy, .) in yes[]
    const int cidx = (ly + 1) * LZ2 + 2 * jn + 1;                // node (iy, iz) in a halo plane

    int next_plane = xa - 1, next_base = (xa - 1) * plane;
    auto issue_plane = [&]() {
        if (next_plane <= xb + 1) {
            const int slot = (next_plane - (xa - 1)) & (RING - 1);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (chas[k]) {
                    cp_async8(&S.raw_a[slot][tid + k * KT], src_a + (next_base + coff[k]), cok[k]);
                    if (TWO) cp_async8(&S.raw_b[slot][tid + k * KT], src_b + (next_base + coff[k]), cok[k]);
                }
            }
        }
        cp_async_commit();
        next_base += plane;
        ++next_plane;
    };
    // p = z (+ beta p_{k-1}) for the copy slots of node plane px (ring slot rs)
    auto form_plane = [&](int px, int rs) {
        double* dst = S.pf[px & 1];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (chas[k]) {
                const int sl = tid + k * KT;
                double p = TWO ? dfma(beta, S.raw_b[rs][sl], S.raw_a[rs][sl]) : S.raw_a[rs][sl];
                if (fi_p && cok[k] && (long long)px * plane + coff[k] == fi_idx) p = flipbit(p, fi_bit);
                dst[sl] = p;
            }
        }
    };
    // coefficients of element plane ix, prefetched one plane ahead
    int eb = (xa - 1) * eplane;
    double rA = 0, kA = 0, rB = 0, kB = 0;
    if (einA) { rA = __ldg(a.rhoc + eb + eoA); kA = __ldg(a.kc + eb + eoA); }
    if (einB) { rB = __ldg(a.rhoc + eb + eoB); kB = __ldg(a.kc + eb + eoB); }
    int nb = xa * plane + woff;      // node index of (ix, iy, iz) in the node phase
    double wA = 0, wB = 0;
    if (d1) { if (nokA) wA = __ldg(a.w + nb); if (nokB) wB = __ldg(a.w + nb + 1); }

    for (int k = 0; k <= AHEAD; ++k) issue_plane();    // planes xa-1 .. xa+AHEAD-1
    if (FORMED) {
        cp_async_wait<AHEAD>();                         // plane xa-1
        __syncthreads();
        form_plane(xa - 1, 0);
    }
    double accA = 0.0, accB = 0.0;
    for (int ix = xa - 1; ix <= xb; ++ix) {
        const int lo = (ix - (xa - 1)) & (RING - 1);   // node plane ix
        const int hi = (lo + 1) & (RING - 1);          // node plane ix+1
        cp_async_wait<AHEAD - 1>();
        __syncthreads();
        issue_plane();
        if (FORMED) {
            form_plane(ix + 1, hi);
            __syncthreads();
        }
        double rAn = 0, kAn = 0, rBn = 0, kBn = 0;     // element plane ix+1
        if (ix + 1 <= xb) {
            if (einA) { rAn = __ldg(a.rhoc + eb + eplane + eoA); kAn = __ldg(a.kc + eb + eplane + eoA); }
            if (einB) { rBn = __ldg(a.rhoc + eb + eplane + eoB); kBn = __ldg(a.kc + eb + eplane + eoB); }
        }
        if (has_e) {
            // 12 node values: columns c, c+1, c+2 of rows ley, ley+1 of planes ix, ix+1
            double n_[2][2][3];
#pragma unroll
            for (int pl = 0; pl < 2; ++pl)
#pragma unroll
                for (int rw = 0; rw < 2; ++rw) {
                    const double* src = FORMED ? &S.pf[(ix + pl) & 1][elo + rw * LZ2]
                                               : &S.raw_a[pl ? hi : lo][elo + rw * LZ2];
                    const double2 v01 = lds2(src);
                    n_[pl][rw][0] = v01.x; n_[pl][rw][1] = v01.y; n_[pl][rw][2] = src[2];
                }
            double vA[8], vB[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                vA[q] = n_[(q >> 2) & 1][(q >> 1) & 1][(q & 1)];
                vB[q] = n_[(q >> 2) & 1][(q >> 1) & 1][1 + (q & 1)];
            }
            elem_apply<FORM>(vA, rA, kA, a.dt_eff, a.ec);
            elem_apply<FORM>(vB, rB, kB, a.dt_eff, a.ec);
            if (fi_r) {
                if (einA && (long long)(eb + eoA) == fi_elem) vA[0] = flipbit(vA[0], fi_bit);
                if (einB && (long long)(eb + eoB) == fi_elem) vB[0] = flipbit(vB[0], fi_bit);
            }
            // elements outside the domain (tile edges) produce garbage that no
            // interior node reads
#pragma unroll
            for (int q = 0; q < 8; ++q) S.yes[q][tid] = make_double2(vA[q], vB[q]);
        }
        rA = rAn; kA = kAn; rB = rBn; kB = kBn;
        eb += eplane;
        __syncthreads();
        if (has_n) {
            // element pairs (iy-1 | iy, 2jn..2jn+1) by q; elements 2jn+1, 2jn+2 of
            // the odd q come from this pair (.y) and the next pair (.x, from the
            // next node-pair thread of the row, or loaded by the row's last one)
            auto take = [&](int q, int pr, double& a_, double& b_, bool odd) {
                const double2 v = S.yes[q][pr];
                if (!odd) { a_ = v.x; b_ = v.y; return; }
                double nxt = __shfl_down_sync(0xffffffffu, v.x, 1);
                if (jn == TZ / 2 - 1) nxt = S.yes[q][pr + 1].x;
                a_ = v.y; b_ = nxt;
            };
            if (ix >= xa) {
                double c3a, c3b, c2a, c2b, c1a, c1b, c0a, c0b;
                take(3, pr0, c3a, c3b, false);     // element (iy-1, iz-1) / (iy-1, iz)   for nodes A / B
                take(2, pr0, c2a, c2b, true);      // element (iy-1, iz)   / (iy-1, iz+1)
                take(1, pr1, c1a, c1b, false);     // element (iy,   iz-1) / (iy,   iz)
                take(0, pr1, c0a, c0b, true);      // element (iy,   iz)   / (iy,   iz+1)
                double yA = accA, yB = accB;
                yA = dadd(yA, c3a); yA = dadd(yA, c2a); yA = dadd(yA, c1a); yA = dadd(yA, c0a);
                yB = dadd(yB, c3b); yB = dadd(yB, c2b); yB = dadd(yB, c1b); yB = dadd(yB, c0b);
                const double* cp_ = FORMED ? &S.pf[ix & 1][cidx] : &S.raw_a[lo][cidx];
                const double pvA = cp_[0], pvB = cp_[1];
                if (fi_ap) {
                    if ((long long)nb == fi_idx) yA = flipbit(yA, fi_bit);
                    if ((long long)nb + 1 == fi_idx) yB = flipbit(yB, fi_bit);
                }
                if (nokA) {
                    if (loop) pa[0] = dfma(pvA, yA, pa[0]);
                    if (d1) { pa[1] = dadd(pa[1], yA); pa[2] = dfma(wA, pvA, pa[2]); pa[3] = dfma(pvA, pvA, pa[3]); }
                    if (rhs) yA = dfma(a.dtF, __ldg(a.F + nb), yA);
                    a.y[nb] = yA;
                    if (pout) pout[nb] = pvA;
                }
                if (nokB) {
                    if (loop) pb[0] = dfma(pvB, yB, pb[0]);
                    if (d1) { pb[1] = dadd(pb[1], yB); pb[2] = dfma(wB, pvB, pb[2]); pb[3] = dfma(pvB, pvB, pb[3]); }
                    if (rhs) yB = dfma(a.dtF, __ldg(a.F + nb + 1), yB);
                    a.y[nb + 1] = yB;
                    if (pout) pout[nb + 1] = pvB;
                }
                nb += plane;
                if (d1 && ix + 1 <= xb) {
                    if (nokA) wA = __ldg(a.w + nb);
                    if (nokB) wB = __ldg(a.w + nb + 1);
                }
            }
            // contributions from below to the next node plane (ox = 1)
            double c7a, c7b, c6a, c6b, c5a, c5b, c4a, c4b;
            take(7, pr0, c7a, c7b, false);
            take(6, pr0, c6a, c6b, true);
            take(5, pr1, c5a, c5b, false);
            take(4, pr1, c4a, c4b, true);
            double nA = 0.0, nB = 0.0;
            nA = dadd(nA, c7a); nA = dadd(nA, c6a); nA = dadd(nA, c5a); nA = dadd(nA, c4a);
            nB = dadd(nB, c7b); nB = dadd(nB, c6b); nB = dadd(nB, c5b); nB = dadd(nB, c4b);
            accA = nA; accB = nB;
        }
    }
    cp_async_wait<0>();
}

// canonical tree of a tile whose node-pair thread p holds the column values
// (ly, 2j) in va and (ly, 2j+1) in vb: the 32-lane butterfly of each row is a
// 16-thread butterfly on both values (offsets 8..1 <-> column offsets 16..2)
// followed by va + vb (column offset 1); rows are the canonical warps.
template <int NQ>
__device__ __forceinline__ void cta_tree_pairs(double (&va)[NQ], double (&vb)[NQ], double (*sh)[8]) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) {
            va[q] = dadd(va[q], __shfl_xor_sync(0xffffffffu, va[q], off));
            vb[q] = dadd(vb[q], __shfl_xor_sync(0xffffffffu, vb[q], off));
        }
        va[q] = dadd(va[q], vb[q]);
    }
    __syncthreads();
    if (tid < NNPAIR && (tid % (TZ / 2)) == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) sh[q][tid / (TZ / 2)] = va[q];
    }
    __syncthreads();
    if (tid < 32) {
        const int lane = tid;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double u = (lane < 8) ? sh[q][lane] : 0.0;
#pragma unroll
            for (int off = 4; off >= 1; off >>= 1) u = dadd(u, __shfl_xor_sync(0xffffffffu, u, off));
            va[q] = u;
        }
    }
}

// Colored operator, interior tiles (blocks 0 .. ntiles-1 of the apply partition).
template <int FORM>
__global__ void __launch_bounds__(KT, FORM == FORM_WHT ? 4 : 3) k_apply_colored(ApplyArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ApplySmem& S = *reinterpret_cast<ApplySmem*>(smem_raw);
    DevState* st = a.st;
    const Part& P = a.part;
    const bool loop = a.role == ROLE_LOOP;
    int iter = 0;
    double beta = 0.0;
    const double* src_a = a.x;
    const double* src_b = nullptr;
    double* pout = nullptr;
    int fi_p = 0, fi_ap = 0, fi_r = 0, fi_bit = 0;
    long long fi_idx = -1, fi_elem = -1;
    if (loop) {
        if (st->done) return;
        iter = st->iter; beta = st->beta;
        src_a = a.z;
        src_b = (iter > 0) ? ((iter & 1) ? a.pbuf0 : a.pbuf1) : nullptr;
        pout = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec && st->fi_iter == iter) {
            fi_idx = st->fi_idx; fi_bit = st->fi_bit;
            fi_p = (st->fi_vec == FI_P); fi_ap = (st->fi_vec == FI_AP);
        }
    } else if (a.role == ROLE_X0 && st->fi_armR) {
        fi_r = 1; fi_elem = st->fi_elem; fi_bit = st->fi_bit;
    }
    const bool d1 = a.d1 != 0;
    const bool rhs = (a.role == ROLE_RHS) && a.F != nullptr;
    double pa[MAXQ] = {0.0, 0.0, 0.0, 0.0}, pb[MAXQ] = {0.0, 0.0, 0.0, 0.0};
    const long long t = blockIdx.x;
    const int tz = (int)(t % P.NTZ), ty = (int)((t / P.NTZ) % P.NTY), tx = (int)(t / ((long long)P.NTZ * P.NTY));
    const int y0 = 1 + ty * TY, z0 = 1 + tz * TZ;
    const int xa = 1 + tx * P.cx, xb = min(tx * P.cx + P.cx, P.I);
    if (!loop)
        apply_tile_pairs<FORM, 0>(a, S, a.N, xa, xb, y0, z0, src_a, src_b, beta, pout, loop, d1, rhs, fi_p, fi_ap,
                                  fi_r, fi_bit, fi_idx, fi_elem, pa, pb);
    else if (!src_b)
        apply_tile_pairs<FORM, 1>(a, S, a.N, xa, xb, y0, z0, src_a, src_b, beta, pout, loop, d1, rhs, fi_p, fi_ap,
                                  fi_r, fi_bit, fi_idx, fi_elem, pa, pb);
    else
        apply_tile_pairs<FORM, 2>(a, S, a.N, xa, xb, y0, z0, src_a, src_b, beta, pout, loop, d1, rhs, fi_p, fi_ap,
                                  fi_r, fi_bit, fi_idx, fi_elem, pa, pb);
    if (!loop && !d1) return;
    cta_tree_pairs<MAXQ>(pa, pb, S.sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < MAXQ; ++q) a.partials[q * P.nblk + t] = pa[q];
    }
}

// Colored operator, boundary nodes (blocks ntiles .. nblk-1 of the apply
// partition; the projection makes their outputs zero): input formation, the
// fault hooks, the partials and the stores.
__global__ void __launch_bounds__(RT) k_apply_boundary(ApplyArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const Part& P = a.part;
    const int N = a.N;
    const int tid = threadIdx.x;
    const bool loop = a.role == ROLE_LOOP;
    int iter = 0;
    double beta = 0.0;
    const double* src_a = a.x;
    const double* src_b = nullptr;
    double* pout = nullptr;
    int fi_p = 0, fi_ap = 0, fi_bit = 0;
    long long fi_idx = -1;
    if (loop) {
        if (st->done) return;
        iter = st->iter; beta = st->beta;
        src_a = a.z;
        src_b = (iter > 0) ? ((iter & 1) ? a.pbuf0 : a.pbuf1) : nullptr;
        pout = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec && st->fi_iter == iter) {
            fi_idx = st->fi_idx; fi_bit = st->fi_bit;
            fi_p = (st->fi_vec == FI_P); fi_ap = (st->fi_vec == FI_AP);
        }
    }
    const bool d1 = a.d1 != 0;
    const bool rhs = (a.role == ROLE_RHS) && a.F != nullptr;
    const bool two = src_b != nullptr;
    double part[MAXQ] = {0.0, 0.0, 0.0, 0.0};
    const long long b = blockIdx.x;
    long long nk[BPT];
    double va[BPT], vb[BPT], wv[BPT];
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const long long j = b * (long long)(RT * BPT) + (long long)k * RT + tid;
        nk[k] = (j < P.NB) ? bnd_node(j, N) : -1;
    }
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const long long n = nk[k];
        va[k] = (n >= 0) ? __ldg(src_a + n) : 0.0;
        vb[k] = (n >= 0 && two) ? __ldg(src_b + n) : 0.0;
        wv[k] = (n >= 0 && d1) ? __ldg(a.w + n) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const long long n = nk[k];
        if (n < 0) break;
        double pv = two ? dfma(beta, vb[k], va[k]) : va[k];
        if (fi_p && n == fi_idx) pv = flipbit(pv, fi_bit);
        double yv = 0.0;
        if (fi_ap && n == fi_idx) yv = flipbit(yv, fi_bit);
        if (loop) part[0] = dfma(pv, yv, part[0]);
        if (d1) {
            part[1] = dfma(0.0, yv, part[1]);
            part[2] = dfma(wv[k], pv, part[2]);
            part[3] = dfma(pv, pv, part[3]);
        }
        if (rhs) yv = dfma(a.dtF, __ldg(a.F + n), yv);
        a.y[n] = yv;
        if (pout) pout[n] = pv;
    }
    if (!loop && !d1) return;
    cta_tree_sum<MAXQ>(part, sh);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < MAXQ; ++q) a.partials[q * P.nblk + P.ntiles + b] = part[q];
    }
}

// Role logic of an operator application once its partials are complete:
// the D1 checksum (relative mismatch of 1_int.(Ax) and w.x) and, in the PCG
// loop, alpha = rho / p.Ap (or the reference's breakdown exit).
struct FinalApplyArgs {
    const double* partials;
    long long nblk;
    DevState* st;
    int role, d1;
};
__global__ void __launch_bounds__(RT) k_final_apply(FinalApplyArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const bool loop = a.role == ROLE_LOOP;
    if (loop && st->done) return;
    double part[MAXQ];
    final_sums<MAXQ>(part, a.partials, a.nblk, sh);
    if (threadIdx.x != 0) return;
    if (a.d1) {
        const double nw = (a.role == ROLE_RHS) ? st->norm_wM : st->norm_wA;
        const double nx = __dsqrt_rn(part[3]);
        double rel = __ddiv_rn(fabs(dsub(part[1], part[2])), dfma(nw, nx, 1e-300));
        if (!isfinite(rel)) rel = 1e300;
        st->d1_last = rel;
        if (a.role != ROLE_USER) st->d1_step = fmax(st->d1_step, rel);
    }
    if (loop) {
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
    long long Nn, nflat;
    int role, pad0;
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

// PCG vector update on the flat partition: each thread updates its KF = 2
// consecutive nodes (128-bit loads and stores), in order.
__global__ void __launch_bounds__(RT, 6) k_update(UpdateArgs a) {
    static_assert(KF == 2, "two nodes per thread");
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const int tid = threadIdx.x;
    if (a.role == UPD_LOOP && st->done) return;
    const bool pre = a.role == UPD_PRE;
    int iter = 0;
    double alpha = 0.0;
    const double* p = nullptr;
    int fi_r = 0, fi_bit = 0;
    long long fi_idx = -1;
    if (!pre) {
        iter = st->iter; alpha = st->alpha;
        p = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec == FI_RV && st->fi_iter == iter) { fi_r = 1; fi_idx = st->fi_idx; fi_bit = st->fi_bit; }
    }
    const double nalpha = -alpha;
    double part[3] = {0.0, 0.0, 0.0};   // PRE: bb, rz, rr   LOOP: rr, rz, -
    const long long m0 = ((long long)blockIdx.x * RT + tid) * KF;
    const int cnt = (m0 + 1 < a.Nn) ? 2 : (m0 < a.Nn ? 1 : 0);
    auto ld2 = [&](const double* base, double& u, double& v) {
        if (cnt == 2) { const double2 t = __ldg(reinterpret_cast<const double2*>(base + m0)); u = t.x; v = t.y; }
        else { u = cnt ? __ldg(base + m0) : 0.0; v = 0.0; }
    };
    auto st2 = [&](double* base, double u, double v) {
        if (cnt == 2) *reinterpret_cast<double2*>(base + m0) = make_double2(u, v);
        else if (cnt == 1) base[m0] = u;
    };
    if (pre) {
        double b0, b1, q0, q1, d0, d1;
        ld2(a.b, b0, b1); ld2(a.Ap, q0, q1); ld2(a.d, d0, d1);
        double r_[2], z_[2];
        const double bb[2] = {b0, b1}, qq[2] = {q0, q1}, dd[2] = {d0, d1};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (k >= cnt) break;
            r_[k] = dfma(-1.0, qq[k], bb[k]);
            z_[k] = __ddiv_rn(r_[k], dd[k]);
            part[0] = dfma(bb[k], bb[k], part[0]);
            part[1] = dfma(r_[k], z_[k], part[1]);
            part[2] = dfma(r_[k], r_[k], part[2]);
        }
        st2(a.r, r_[0], r_[1]); st2(a.z, z_[0], z_[1]);
    } else {
        double x0, x1, p0, p1, q0, q1, r0, r1, d0, d1;
        ld2(a.x, x0, x1); ld2(p, p0, p1); ld2(a.Ap, q0, q1); ld2(a.r, r0, r1); ld2(a.d, d0, d1);
        const double xx[2] = {x0, x1}, pp[2] = {p0, p1}, qq[2] = {q0, q1}, rr[2] = {r0, r1}, dd[2] = {d0, d1};
        double xn[2], r_[2], z_[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (k >= cnt) break;
            xn[k] = dfma(alpha, pp[k], xx[k]);
            r_[k] = dfma(nalpha, qq[k], rr[k]);
            if (fi_r && m0 + k == fi_idx) r_[k] = flipbit(r_[k], fi_bit);
            z_[k] = __ddiv_rn(r_[k], dd[k]);
            part[0] = dfma(r_[k], r_[k], part[0]);
            part[1] = dfma(r_[k], z_[k], part[1]);
        }
        st2(a.x, xn[0], xn[1]); st2(a.r, r_[0], r_[1]); st2(a.z, z_[0], z_[1]);
    }
    store_partials<3>(part, a.partials, a.nflat, sh);
}

// PCG scalar logic after the vector update: the prologue's ||b||, rho and
// initial residual, or the loop's convergence test (||r||/||b|| < tol, the
// reference's recursive residual), beta = rho_new / rho and the iteration
// count; sets the graph's while condition.
struct FinalUpdateArgs {
    const double* partials;
    long long nflat;
    DevState* st;
    cudaGraphConditionalHandle cond;
    int role, use_cond;
};
__global__ void __launch_bounds__(RT) k_final_update(FinalUpdateArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const bool pre = a.role == UPD_PRE;
    if (!pre && st->done) {
        if (a.use_cond && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
        return;
    }
    double part[3];
    final_sums<3>(part, a.partials, a.nflat, sh);
    if (threadIdx.x != 0) return;
    if (pre) {
        double bnorm = __dsqrt_rn(part[0]);
        if (bnorm < 1e-30) bnorm = 1.0;
        st->bnorm = bnorm;
        st->rho = part[1];
        st->rel0 = __ddiv_rn(__dsqrt_rn(part[2]), bnorm);
        st->iter = 0; st->broken = 0; st->result = 0; st->beta = 0.0;
        st->done = (st->max_iter <= 0) ? 1 : 0;
    } else {
        const int iter = st->iter;
        const double rnorm = __dsqrt_rn(part[0]);
        const double rel = __ddiv_rn(rnorm, st->bnorm);
        const bool conv = rel < st->tol;
        double beta = 0.0;
        if (!conv) { beta = __ddiv_rn(part[1], st->rho); st->rho = part[1]; }
        if (st->log_rel && iter < st->log_cap) {
            st->log_rel[iter] = rel; st->log_alpha[iter] = st->alpha; st->log_beta[iter] = beta;
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
    long long Nn, nflat;
    int N, kind;
    const double* a;
    const double* b;
    double* partials;
    unsigned* ticket;
    double* out;     // 2 results (device)
};

__global__ void __launch_bounds__(RT) k_reduce(RedArgs a) {
    __shared__ double sh[MAXQ][8];
    const int tid = threadIdx.x;
    double part[2] = {0.0, 0.0};
    const long long n0 = ((long long)blockIdx.x * RT + tid) * KF;
    double va[KF], vb[KF];
#pragma unroll
    for (int k = 0; k < KF; ++k) {
        const long long m = n0 + k;
        va[k] = (m < a.Nn) ? __ldg(a.a + m) : 0.0;
        vb[k] = (m < a.Nn && a.kind != RED_ABFT_S) ? __ldg(a.b + m) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < KF; ++k) {
        const long long m = n0 + k;
        if (m >= a.Nn) break;
        switch (a.kind) {
            case RED_DOT: part[0] = dfma(va[k], vb[k], part[0]); break;
            case RED_RESID: {
                const double rv = dfma(-1.0, va[k], vb[k]);
                part[0] = dfma(rv, rv, part[0]);
                part[1] = dfma(vb[k], vb[k], part[1]);
            } break;
            case RED_DIFF: {
                const double dv = dsub(va[k], vb[k]);
                part[0] = dfma(dv, dv, part[0]);
                part[1] = dfma(vb[k], vb[k], part[1]);
            } break;
            default: part[0] = dfma(is_bnd(m, a.N) ? 0.0 : 1.0, va[k], part[0]); break;
        }
    }
    store_partials<2>(part, a.partials, a.nflat, sh);
}
__global__ void __launch_bounds__(RT) k_final_reduce(const double* partials, long long nflat, double* out) {
    __shared__ double sh[MAXQ][8];
    double part[2];
    final_sums<2>(part, partials, nflat, sh);
    if (threadIdx.x == 0) { out[0] = part[0]; out[1] = part[1]; }
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
    Part part;
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
    const Part& P = a.part;
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
            const int xa = 1 + tx * P.cx, xb = min(tx * P.cx + P.cx, P.I);
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
    store_partials<MAXQ>(part, a.partials, P.nblk, sh);
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
// reads a buffer larger than the L2 (clean lines replace whatever was cached)
__global__ void k_l2_scrub(const double* __restrict__ buf, long long n, double* sink) {
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc += __ldcg(buf + i);
    if (acc == 1.2345e300) *sink = acc;   // keeps the loads; never true for the zeroed buffer
}
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
