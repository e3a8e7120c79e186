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
// canonical node sum: the corner q of each contributing element, in order
__device__ __constant__ int kSumOrder[8] = {4, 7, 6, 5, 0, 3, 2, 1};

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double flipbit(double x, int bit) {
    return __longlong_as_double(__double_as_longlong(x) ^ (long long)(1ULL << bit));
}

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization may start while the kernel before it in the stream is still
// running; pdl_wait() returns once that kernel has completed and its memory
// operations are visible (a no-op for a kernel launched without the
// attribute).  Everything a PCG-loop kernel reads that the loop writes comes
// after it; before it a kernel only sets up geometry and reads loop-invariant
// data.  pdl_release() lets the next kernel in the stream be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

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
// slab partition of an N-element grid (operator tiles) and the flat partition
struct Part {
    int N, NN;
    int C, R, CX;                     // tile columns, rows, planes
    int Cw, Rw;                       // positions per row and rows per plane (halo included)
    int NCB, NRB, NXB;                // tiles per direction (z, y, x)
    long long ntiles, nblk;           // tiles = apply partials per quantity
    long long Nn, nflat;              // flat partition: blocks of RT*KF nodes
};

inline Part make_part(int N) {
    Part p{};
    const SlabLayout L = slab_layout(N);
    p.N = N; p.NN = N + 1;
    p.C = L.C; p.R = L.R; p.CX = L.CX;
    p.Cw = L.C + 2; p.Rw = L.R + 2;
    p.NCB = L.NCB; p.NRB = L.NRB; p.NXB = L.NXB;
    p.ntiles = L.ntiles; p.nblk = L.ntiles;
    const long long NN = p.NN;
    p.Nn = NN * NN * NN;
    p.nflat = (p.Nn + (long long)RT * KF - 1) / ((long long)RT * KF);
    return p;
}

__device__ __forceinline__ bool is_bnd(long long n, int N) {
    const long long NN = N + 1;
    int ix = (int)(n / (NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
    return ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N;
}

// tile t of the slab partition: first row y0, first column z0, planes xa..xb
struct SlabTile { int y0, z0, xa, xb; };
__device__ __forceinline__ SlabTile slab_tile(const Part& P, long long t) {
    const int cb = (int)(t % P.NCB), rb = (int)((t / P.NCB) % P.NRB), tx = (int)(t / ((long long)P.NCB * P.NRB));
    SlabTile s;
    s.y0 = rb * P.R; s.z0 = cb * P.C; s.xa = tx * P.CX;
    s.xb = min(s.xa + P.CX, P.NN) - 1;
    return s;
}

// geometry of the SK positions of this thread in a slab CTA.  flags: bit k
// node exists, bit 8+k element (lower corner at the position) exists, bit 16+k
// tile node (output), bit 24+k on a y or z boundary face.
struct SlabPos {
    int noff[SK];     // node offset within a plane
    int eoff[SK];     // element offset within an element layer
    unsigned fl;
};
__device__ __forceinline__ SlabPos slab_pos(const Part& P, const SlabTile& T, int tid) {
    SlabPos s;
    s.fl = 0u;
    const int N = P.N;
#pragma unroll
    for (int k = 0; k < SK; ++k) {
        const int j = tid + k * ST;
        const int lr = j / P.Cw, lc = j - lr * P.Cw;
        const int gy = T.y0 - 1 + lr, gz = T.z0 - 1 + lc;
        const bool in = j < P.Rw * P.Cw;
        const bool valid = in && gy >= 0 && gy <= N && gz >= 0 && gz <= N;
        const bool elem = in && lr <= P.Rw - 2 && lc <= P.Cw - 2 && gy >= 0 && gy < N && gz >= 0 && gz < N;
        const bool out = valid && lr >= 1 && lr <= P.Rw - 2 && lc >= 1 && lc <= P.Cw - 2;
        const bool yzb = gy == 0 || gy == N || gz == 0 || gz == N;
        s.noff[k] = valid ? gy * P.NN + gz : 0;
        s.eoff[k] = elem ? gy * N + gz : 0;
        s.fl |= (valid ? 1u : 0u) << k | (elem ? 1u : 0u) << (8 + k) | (out ? 1u : 0u) << (16 + k) |
                (yzb ? 1u : 0u) << (24 + k);
    }
    return s;
}
__device__ __forceinline__ bool sp_valid(unsigned fl, int k) { return (fl >> k) & 1u; }
__device__ __forceinline__ bool sp_elem(unsigned fl, int k) { return (fl >> (8 + k)) & 1u; }
__device__ __forceinline__ bool sp_out(unsigned fl, int k) { return (fl >> (16 + k)) & 1u; }
__device__ __forceinline__ bool sp_yzb(unsigned fl, int k) { return (fl >> (24 + k)) & 1u; }

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
// The strided sums take their partials in batches of FB per quantity: all the
// batch's loads are issued before the (in-order) adds, so the pass costs a
// few memory latencies instead of one per partial.
template <int NQ, int FB = 16>
__device__ __forceinline__ void final_sums(double (&v)[NQ], const double* partials, long long nblk, double (*sh)[8]) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    for (long long k0 = threadIdx.x; k0 < nblk; k0 += (long long)RT * FB) {
        double t[NQ][FB];
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int u = 0; u < FB; ++u) {
                const long long k = k0 + (long long)u * RT;
                t[q][u] = (k < nblk) ? __ldcg(partials + q * nblk + k) : 0.0;
            }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int u = 0; u < FB; ++u)
                if (k0 + (long long)u * RT < nblk) v[q] = dadd(v[q], t[q][u]);
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
    const double2* coef;    // per element (rho*c, k)
    const double* w;        // ABFT weight (w_M or w_A) or null
    const double* F;        // ROLE_RHS source (null: none)
    double dtF;
    int d1;                 // evaluate the D1 checksum
    int pad1;
    double* partials;
    DevState* st;
    ElemConsts ec;
};

// ---- colored operator: slab tiles ------------------------------------------------
// One CTA of ST threads streams a tile's node planes in increasing x.  Per
// element layer ix (between planes ix and ix+1):
//   1. plane ix+1 is formed (p = z + beta p_{k-1} in the PCG loop) from
//      registers loaded one layer ahead, kept in registers and published to
//      shared memory;
//   2. the element whose lower corner is a position (own column) gathers its
//      six other corners from the two published planes, applies the element
//      operator, folds its own-column outputs (q = 0 into the plane-ix node,
//      q = 4 into the plane-(ix+1) node) into per-position accumulators and
//      hands the other six to the three neighbouring positions;
//   3. each tile node of plane ix adds the three handed-in contributions
//      (q = 3, 2, 1), which completes its canonical node sum, and is
//      projected, checked and stored; the plane-(ix+1) accumulators take
//      q = 7, 6, 5.
// Per node and layer that is one shared store of p, six shared loads for the
// gather and three 16-byte stores and loads for the hand-over.
struct __align__(16) SlabSmem {
    double P[2][SPOS];      // formed planes, plane px in P[px & 1]
    double2 Y1[SPOS];       // from the element at position j-1:      (q1, q5)
    double2 Y2[SPOS];       // from the element at position j-Cw:     (q2, q6)
    double2 Y3[SPOS];       // from the element at position j-Cw-1:   (q3, q7)
    double sh[MAXQ][8];
};
constexpr size_t kSlabSmem = sizeof(SlabSmem);

// MODE 0: input x as given; 1: PCG loop, p = z; 2: PCG loop, p = z + beta p_{k-1}.
// FI false: no fault is armed for this launch (the per-node fault tests compile out).
template <int FORM, int MODE, bool FI = true>
__device__ __forceinline__ void slab_march(const ApplyArgs& a, SlabSmem& S, const SlabTile& T, const SlabPos& G,
                                           const double* src_a, const double* src_b, double beta, double* pout,
                                           bool loop, bool d1, bool rhs, int fi_p, int fi_ap, int fi_r, int fi_bit,
                                           long long fi_idx, long long fi_elem, double (&part)[MAXQ]) {
    constexpr bool TWO = MODE == 2;
    if (!FI) { fi_p = 0; fi_ap = 0; fi_r = 0; }
    const Part& P = a.part;
    const int N = P.N, Cw = P.Cw;
    // node and element indices fit in 32 bits (N <= 1200): one wide multiply-add per address
    const unsigned plane = (unsigned)P.NN * (unsigned)P.NN, eplane = (unsigned)N * (unsigned)N;
    const int tid = threadIdx.x;
    const unsigned fl = G.fl;
    const int xa = T.xa, xb = T.xb;

    double pA[SK], pB[SK], aA[SK], aB[SK], ra[SK], rb[SK], cr[SK], ck[SK], wv[SK], fv[SK];
    auto ld_raw = [&](int px) {
        const bool pv = px >= 0 && px <= N;
        const unsigned base = (unsigned)px * plane;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            const bool v = pv && sp_valid(fl, k);
            const unsigned n = base + (unsigned)G.noff[k];
            ra[k] = v ? __ldg(src_a + n) : 0.0;
            if (TWO) rb[k] = v ? __ldg(src_b + n) : 0.0;
        }
    };
    auto form = [&](int px, double (&p)[SK]) {
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            double v = TWO ? dfma(beta, rb[k], ra[k]) : ra[k];
            if (fi_p && sp_valid(fl, k) && (long long)px * plane + G.noff[k] == fi_idx) v = flipbit(v, fi_bit);
            p[k] = v;
        }
    };
    auto ld_coef = [&](int ex) {
        const bool ev = ex >= 0 && ex < N;
        const unsigned base = (unsigned)ex * eplane;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            const bool v = ev && sp_elem(fl, k);
            const double2 c = v ? __ldg(a.coef + (base + (unsigned)G.eoff[k])) : make_double2(0.0, 0.0);
            cr[k] = c.x; ck[k] = c.y;
        }
    };
    auto ld_w = [&](int px) {
        const bool pv = px >= xa && px <= xb;
        const unsigned base = (unsigned)px * plane;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            const bool v = pv && sp_out(fl, k);
            const unsigned n = base + (unsigned)G.noff[k];
            wv[k] = (v && d1) ? __ldg(a.w + n) : 0.0;
            if (MODE == 0) fv[k] = (v && rhs) ? __ldg(a.F + n) : 0.0;
        }
    };

    // One element layer ix (between planes ix and ix+1).  Plane px lives in
    // P[(px - xa + 1) & 1] (cur for plane ix); pc / pn hold planes ix / ix+1
    // of the own column, ac / an the node sums of planes ix / ix+1.
    auto layer = [&](int ix, int cur, double (&pc)[SK], double (&pn)[SK], double (&ac)[SK], double (&an)[SK]) {
        const int nxt = cur ^ 1;
        // 1. plane ix+1
        form(ix + 1, pn);
#pragma unroll
        for (int k = 0; k < SK; ++k) S.P[nxt][tid + k * ST] = pn[k];
        ld_raw(ix + 2 <= xb + 1 ? ix + 2 : -2);
        __syncthreads();
        // 2. element layer ix
        if (ix >= 0 && ix < N) {
#pragma unroll
            for (int k = 0; k < SK; ++k) {
                // every position computes its element (zero coefficients where there
                // is none), so the SK elements carry no branch between them; only the
                // hand-over stores are guarded
                const bool ev = sp_elem(fl, k);
                const int j = tid + k * ST;
                double v[8];
                v[0] = pc[k];
                v[1] = S.P[cur][j + 1];
                v[2] = S.P[cur][j + Cw];
                v[3] = S.P[cur][j + Cw + 1];
                v[4] = pn[k];
                v[5] = S.P[nxt][j + 1];
                v[6] = S.P[nxt][j + Cw];
                v[7] = S.P[nxt][j + Cw + 1];
                elem_apply<FORM>(v, cr[k], ck[k], a.dt_eff, a.ec);
                if (fi_r && (long long)ix * eplane + G.eoff[k] == fi_elem) v[0] = flipbit(v[0], fi_bit);
                ac[k] = dadd(ac[k], v[0]);
                an[k] = dadd(0.0, v[4]);
                if (ev) {
                    S.Y1[j + 1] = make_double2(v[1], v[5]);
                    S.Y2[j + Cw] = make_double2(v[2], v[6]);
                    S.Y3[j + Cw + 1] = make_double2(v[3], v[7]);
                }
            }
        }
        ld_coef(ix + 1 <= xb ? ix + 1 : -1);
        __syncthreads();
        // 3. tile nodes of plane ix; node sums of plane ix+1
        const unsigned base = (unsigned)ix * plane;
        const bool xbnd = ix == 0 || ix == N;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            if (!sp_out(fl, k)) continue;
            const int j = tid + k * ST;
            const bool yzin = !sp_yzb(fl, k);
            double2 y3 = make_double2(0.0, 0.0), y2 = y3, y1 = y3;
            if (yzin) { y3 = S.Y3[j]; y2 = S.Y2[j]; y1 = S.Y1[j]; }
            if (ix >= xa) {
                const unsigned n = base + (unsigned)G.noff[k];
                const bool bnd = !yzin || xbnd;
                double y = bnd ? 0.0 : dadd(dadd(dadd(ac[k], y3.x), y2.x), y1.x);
                if (fi_ap && (long long)n == fi_idx) y = flipbit(y, fi_bit);
                const double pv = pc[k];
                if (loop) part[0] = dfma(pv, y, part[0]);
                if (d1) {
                    part[1] = bnd ? dfma(0.0, y, part[1]) : dadd(part[1], y);
                    part[2] = dfma(wv[k], pv, part[2]);
                    part[3] = dfma(pv, pv, part[3]);
                }
                if (MODE == 0 && rhs) y = dfma(a.dtF, fv[k], y);
                a.y[n] = y;
                if (TWO || MODE == 1) pout[n] = pv;
            }
            an[k] = yzin ? dadd(dadd(dadd(an[k], y3.y), y2.y), y1.y) : 0.0;
        }
        ld_w(ix + 1);
    };

    // plane xa-1, then the inputs of plane xa and the coefficients of layer xa-1
    ld_raw(xa - 1);
    form(xa - 1, pA);
#pragma unroll
    for (int k = 0; k < SK; ++k) { S.P[0][tid + k * ST] = pA[k]; aA[k] = 0.0; aB[k] = 0.0; }
    ld_raw(xa);
    ld_coef(xa - 1);
    for (int ix = xa - 1; ix <= xb; ++ix) {
        layer(ix, (ix - xa + 1) & 1, pA, pB, aA, aB);
#pragma unroll
        for (int k = 0; k < SK; ++k) { pA[k] = pB[k]; aA[k] = aB[k]; }
    }
}

// Colored operator: tile blockIdx.x of the slab partition (every node of the
// grid belongs to exactly one tile; boundary nodes are projected to zero).
// LOOP: the PCG-loop role (p formed in the kernel); otherwise the roles that
// apply the operator to a given vector.
template <int FORM, bool LOOP>
__global__ void __launch_bounds__(ST, FORM == FORM_WHT ? 2 : 1) k_apply_slab(ApplyArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SlabSmem& S = *reinterpret_cast<SlabSmem*>(smem_raw);
    DevState* st = a.st;
    int fi_p = 0, fi_ap = 0, fi_r = 0, fi_bit = 0;
    long long fi_idx = -1, fi_elem = -1;
    const bool d1 = a.d1 != 0;
    double part[MAXQ] = {0.0, 0.0, 0.0, 0.0};
    const SlabTile T = slab_tile(a.part, blockIdx.x);
    const SlabPos G = slab_pos(a.part, T, threadIdx.x);
    if (LOOP) {
        pdl_wait();
        pdl_release();
        if (st->done) return;
        const int iter = st->iter;
        const double beta = st->beta;
        const double* src_b = (iter > 0) ? ((iter & 1) ? a.pbuf0 : a.pbuf1) : nullptr;
        double* pout = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec && st->fi_iter == iter) {
            fi_idx = st->fi_idx; fi_bit = st->fi_bit;
            fi_p = (st->fi_vec == FI_P); fi_ap = (st->fi_vec == FI_AP);
        }
        if (!src_b)
            slab_march<FORM, 1>(a, S, T, G, a.z, src_b, beta, pout, true, d1, false, fi_p, fi_ap, 0, fi_bit, fi_idx,
                                -1, part);
        else if (fi_p || fi_ap)
            slab_march<FORM, 2, true>(a, S, T, G, a.z, src_b, beta, pout, true, d1, false, fi_p, fi_ap, 0, fi_bit,
                                      fi_idx, -1, part);
        else
            slab_march<FORM, 2, false>(a, S, T, G, a.z, src_b, beta, pout, true, d1, false, 0, 0, 0, 0, -1, -1, part);
    } else {
        if (a.role == ROLE_X0 && st->fi_armR) { fi_r = 1; fi_elem = st->fi_elem; fi_bit = st->fi_bit; }
        const bool rhs = (a.role == ROLE_RHS) && a.F != nullptr;
        slab_march<FORM, 0>(a, S, T, G, a.x, nullptr, 0.0, nullptr, false, d1, rhs, 0, 0, fi_r, fi_bit, -1, fi_elem,
                            part);
        if (!d1) return;
    }
    store_partials<MAXQ>(part, a.partials, a.part.nblk, S.sh);
}

// The D1 checksum (relative mismatch of 1_int.(Ax) and w.x) of an operator
// application outside the PCG loop, once its partials are complete.  The loop
// role's reductions (p.Ap, alpha, D1, breakdown) are finished by k_update.
struct FinalApplyArgs {
    const double* partials;
    long long nblk;
    DevState* st;
    int role, d1;
};
__global__ void __launch_bounds__(RT) k_final_apply(FinalApplyArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    double part[MAXQ];
    final_sums<MAXQ>(part, a.partials, a.nblk, sh);
    if (threadIdx.x != 0 || !a.d1) return;
    const double nw = (a.role == ROLE_RHS) ? st->norm_wM : st->norm_wA;
    const double nx = __dsqrt_rn(part[3]);
    double rel = __ddiv_rn(fabs(dsub(part[1], part[2])), dfma(nw, nx, 1e-300));
    if (!isfinite(rel)) rel = 1e300;
    st->d1_last = rel;
    if (a.role != ROLE_USER) st->d1_step = fmax(st->d1_step, rel);
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
    int use_cond, d1;           // d1: the loop operator's checksum is evaluated (CTA 0)
    const double* apart;        // LOOP: the operator's tile partials (p.Ap, 1_int.Ap, w.p, p.p)
    long long nblk;             // LOOP: their count per quantity
};

// PCG scalar logic after the vector update, on the RUN-order sums: the
// prologue's ||b||, rho and initial residual, or the loop's convergence test
// (||r||/||b|| < tol, the reference's recursive residual), beta = rho_new /
// rho and the iteration count; sets the graph's while condition.
__device__ __forceinline__ void update_scalars(const UpdateArgs& a, const double (&part)[3]) {
    DevState* st = a.st;
    if (a.role == UPD_PRE) {
        double bnorm = __dsqrt_rn(part[0]);
        if (bnorm < 1e-30) bnorm = 1.0;
        st->bnorm = bnorm;
        st->rho = part[1];
        st->rel0 = __ddiv_rn(__dsqrt_rn(part[2]), bnorm);
        st->iter = 0; st->broken = 0; st->result = 0; st->beta = 0.0;
        st->done = (st->max_iter <= 0) ? 1 : 0;
        st->x_pend = 0;
    } else {
        const int iter = st->iter;
        st->x_pend = (iter & 1) ? 0 : 1;        // an even iteration leaves its x update owed
        st->x_pend_iter = iter;
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

// PCG vector update on the flat partition: each thread updates its KF
// consecutive nodes (KF / 2 aligned 128-bit loads and stores per vector), in
// order.  In the loop it first finishes the operator's reductions: every CTA
// sums p.Ap over the tile partials in the canonical order (so alpha = rho /
// p.Ap is the same bits everywhere), and CTA 0 records p.Ap, alpha, the D1
// checksum and a breakdown.
//
// It also finishes its own reductions, in the RUN order: CTA c of the
// G = min(nflat, UPD_SLOTS) CTAs takes the flat blocks c, c+G, c+2G, ..., each
// thread carrying one sum through its nodes of all of them, reduces the run
// with one block tree, and the last CTA to finish (an atomic ticket) combines
// the G run sums
// (final_sums) and runs the scalar logic, the work a separate single-CTA
// kernel would do after it.  G fits one resident wave (5 CTAs per SM), so the
// last CTA's pass reads at most UPD_SLOTS partials per quantity.
constexpr int kUpdateCtasPerSm = 5;
static_assert(UPD_SLOTS == 148 * kUpdateCtasPerSm, "one resident wave of update CTAs on 148 SMs");
__global__ void __launch_bounds__(RT, kUpdateCtasPerSm) k_update(UpdateArgs a) {
    static_assert(KF % 2 == 0, "pairs of nodes per thread");
    constexpr int NC = KF / 2;
    __shared__ double sh[MAXQ][8];
    __shared__ double s_pAp;
    __shared__ unsigned s_last;
    DevState* st = a.st;
    const int tid = threadIdx.x;
    const bool pre = a.role == UPD_PRE;
    pdl_wait();
    pdl_release();
    if (!pre && st->done) {
        // the solve ended (converged, capped or broken down): end the graph's while loop
        if (a.use_cond && blockIdx.x == 0 && tid == 0) cudaGraphSetConditional(a.cond, 0u);
        return;
    }
    int iter = 0;
    double alpha = 0.0;
    const double* p = nullptr;
    int fi_r = 0, fi_bit = 0;
    long long fi_idx = -1;
    if (!pre) {
        iter = st->iter;
        p = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec == FI_RV && st->fi_iter == iter) { fi_r = 1; fi_idx = st->fi_idx; fi_bit = st->fi_bit; }
        // alpha from the operator's partials, once per CTA (short load batches keep the registers low)
        if (blockIdx.x == 0) {
            double q[MAXQ];
            final_sums<MAXQ, 2>(q, a.apart, a.nblk, sh);
            if (tid == 0) {
                if (a.d1) {
                    const double nx = __dsqrt_rn(q[3]);
                    double rel = __ddiv_rn(fabs(dsub(q[1], q[2])), dfma(st->norm_wA, nx, 1e-300));
                    if (!isfinite(rel)) rel = 1e300;
                    st->d1_last = rel;
                    st->d1_step = fmax(st->d1_step, rel);
                }
                st->pAp = q[0];
                if (fabs(q[0]) < 1e-30) {
                    st->broken = 1; st->done = 1; st->result = st->iter;
                    if (a.use_cond) cudaGraphSetConditional(a.cond, 0u);
                } else {
                    st->alpha = __ddiv_rn(st->rho, q[0]);
                    st->alpha_hist[st->iter & 1] = st->alpha;
                }
                s_pAp = q[0];
            }
        } else {
            double q[1];
            final_sums<1, 8>(q, a.apart, a.nblk, sh);
            if (tid == 0) s_pAp = q[0];
        }
        __syncthreads();
        const double pAp = s_pAp;
        if (fabs(pAp) < 1e-30) return;          // breakdown: the reference stops before the update
        alpha = __ddiv_rn(st->rho, pAp);
    }
    const double nalpha = -alpha;
    // x += alpha p runs at odd iterations, for the previous iteration and this
    // one (the previous p is still in the other buffer, its alpha in alpha_hist)
    const bool xupd = !pre && (iter & 1);
    const double* p_prev = (iter & 1) ? a.pbuf0 : a.pbuf1;
    const double alpha_prev = xupd ? st->alpha_hist[(iter - 1) & 1] : 0.0;
    // one flat block: its 3 partials (PRE: bb, rz, rr   LOOP: rr, rz, -) into part
    auto block = [&](long long blk, double* part) {
        const long long m0 = (blk * RT + tid) * KF;
        int cnt[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const long long m = m0 + 2 * c;
            cnt[c] = (blk >= a.nflat) ? 0 : (m + 1 < a.Nn) ? 2 : (m < a.Nn ? 1 : 0);
        }
        auto ld = [&](const double* base, double (&v)[KF]) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const long long m = m0 + 2 * c;
                if (cnt[c] == 2) { const double2 t = __ldg(reinterpret_cast<const double2*>(base + m)); v[2 * c] = t.x; v[2 * c + 1] = t.y; }
                else { v[2 * c] = cnt[c] ? __ldg(base + m) : 0.0; v[2 * c + 1] = 0.0; }
            }
        };
        auto stv = [&](double* base, const double (&v)[KF]) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const long long m = m0 + 2 * c;
                if (cnt[c] == 2) *reinterpret_cast<double2*>(base + m) = make_double2(v[2 * c], v[2 * c + 1]);
                else if (cnt[c] == 1) base[m] = v[2 * c];
            }
        };
        auto has = [&](int k) { return k % 2 < cnt[k / 2]; };
        if (pre) {
            double bb[KF], qq[KF], dd[KF], r_[KF], z_[KF];
            ld(a.b, bb); ld(a.Ap, qq); ld(a.d, dd);
#pragma unroll
            for (int k = 0; k < KF; ++k) {
                r_[k] = 0.0; z_[k] = 0.0;
                if (!has(k)) continue;
                r_[k] = dfma(-1.0, qq[k], bb[k]);
                z_[k] = __ddiv_rn(r_[k], dd[k]);
                part[0] = dfma(bb[k], bb[k], part[0]);
                part[1] = dfma(r_[k], z_[k], part[1]);
                part[2] = dfma(r_[k], r_[k], part[2]);
            }
            stv(a.r, r_); stv(a.z, z_);
        } else {
            double qq[KF], rr[KF], dd[KF];
            ld(a.Ap, qq); ld(a.r, rr); ld(a.d, dd);
            if (xupd) {
                // x += alpha_{k-1} p_{k-1}, then x += alpha_k p_k: the same two
                // multiply-adds, in the same order, as one update per iteration
                double xx[KF], pp[KF], po[KF];
                ld(a.x, xx); ld(p_prev, po); ld(p, pp);
#pragma unroll
                for (int k = 0; k < KF; ++k)
                    if (has(k)) xx[k] = dfma(alpha, pp[k], dfma(alpha_prev, po[k], xx[k]));
                stv(a.x, xx);
            }
#pragma unroll
            for (int k = 0; k < KF; ++k) {
                if (!has(k)) continue;
                double rk = dfma(nalpha, qq[k], rr[k]);
                if (fi_r && m0 + k == fi_idx) rk = flipbit(rk, fi_bit);
                rr[k] = rk;
                dd[k] = __ddiv_rn(rk, dd[k]);          // z
                part[0] = dfma(rk, rk, part[0]);
                part[1] = dfma(rk, dd[k], part[1]);
            }
            stv(a.r, rr); stv(a.z, dd);
        }
    };
    // run blockIdx.x of the RUN order: flat blocks c, c+G, ...; each thread
    // carries one sum through its nodes of all the run's blocks, and the run
    // takes one block tree at the end
    const int G = gridDim.x, c = blockIdx.x;
    double part[3] = {0.0, 0.0, 0.0};
    for (int blk = c; blk < a.nflat; blk += G) block(blk, part);
    cta_tree_sum<3>(part, sh);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) a.partials[(long long)q * G + c] = part[q];
        __threadfence();
        const unsigned t = atomicAdd(a.ticket, 1u);
        s_last = (t == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    // the last CTA: the run sums' final combination, then the scalar logic
    __threadfence();
    double v[3];
    final_sums<3, 4>(v, a.partials, G, sh);            // one batch of loads per thread (G <= 740)
    if (tid == 0) {
        *a.ticket = 0u;
        update_scalars(a, v);
    }
}

// The solution update still owed when the PCG loop ends (its last update ran
// at an even iteration): x += alpha p of that iteration.
__global__ void __launch_bounds__(RT) k_update_finish(long long Nn, double* x, const double* pbuf0,
                                                     const double* pbuf1, const DevState* st) {
    if (!st->x_pend) return;
    const int k = st->x_pend_iter;
    const double* p = (k & 1) ? pbuf1 : pbuf0;
    const double alpha = st->alpha_hist[k & 1];
    for (long long i = (long long)blockIdx.x * RT + threadIdx.x; i < Nn; i += (long long)gridDim.x * RT)
        x[i] = dfma(alpha, p[i], x[i]);
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
// k_apply_slab (same element arithmetic, same summation order).  Used for
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
        const int qn = kSumOrder[s];
        const int ex = ix - ((qn >> 2) & 1), ey = iy - ((qn >> 1) & 1), ez = iz - (qn & 1);
        if (ex < 0 || ey < 0 || ez < 0 || ex >= N || ey >= N || ez >= N) continue;
        const long long e = ((long long)ex * N + ey) * N + ez;
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
// Bricks of AB_X x AB_Y x AB_Z elements, one element per thread: the element
// outputs are added into the brick's node block in shared memory (shared
// atomics), and only the nodes on the brick's faces, which neighbouring
// bricks also touch, are added to y with global atomics; the brick's inner
// nodes are stored.  y is zeroed beforehand.  The order of the additions is
// not fixed (the reference's atomic mode is not bit-reproducible either).
constexpr int AB_X = 4, AB_Y = 8, AB_Z = 8;
constexpr int AB_NODES = (AB_X + 1) * (AB_Y + 1) * (AB_Z + 1);
template <int FORM>
__global__ void __launch_bounds__(RT) k_apply_atomic(AtomArgs a) {
    static_assert(AB_X * AB_Y * AB_Z == RT, "one element per thread");
    __shared__ double acc[AB_NODES];
    const DevState* st = a.st;
    const double* x = a.x;
    if (a.role == ROLE_LOOP) {
        if (st->done) return;
        x = (st->iter & 1) ? a.pbuf1 : a.pbuf0;
    }
    const bool fire_r = (a.role == ROLE_X0) && st->fi_armR;
    const int N = a.N;
    const long long NN = N + 1;
    const int nbz = (N + AB_Z - 1) / AB_Z, nby = (N + AB_Y - 1) / AB_Y;
    const int bz = blockIdx.x % nbz, by = (blockIdx.x / nbz) % nby, bx = blockIdx.x / (nbz * nby);
    const int x0 = bx * AB_X, y0 = by * AB_Y, z0 = bz * AB_Z;
    for (int i = threadIdx.x; i < AB_NODES; i += RT) acc[i] = 0.0;
    __syncthreads();
    const int tz = threadIdx.x % AB_Z, ty = (threadIdx.x / AB_Z) % AB_Y, tx = threadIdx.x / (AB_Z * AB_Y);
    const int ex = x0 + tx, ey = y0 + ty, ez = z0 + tz;
    if (ex < N && ey < N && ez < N) {
        const long long e = ((long long)ex * N + ey) * N + ez;
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            v[q] = __ldg(x + ((long long)(ex + ((q >> 2) & 1)) * NN + ey + ((q >> 1) & 1)) * NN + ez + (q & 1));
        elem_apply<FORM>(v, __ldg(a.rhoc + e), __ldg(a.kc + e), a.dt_eff, a.ec);
        if (fire_r && e == st->fi_elem) v[0] = flipbit(v[0], st->fi_bit);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int lx = tx + ((q >> 2) & 1), ly = ty + ((q >> 1) & 1), lz = tz + (q & 1);
            atomicAdd(&acc[(lx * (AB_Y + 1) + ly) * (AB_Z + 1) + lz], v[q]);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < AB_NODES; i += RT) {
        const int lz = i % (AB_Z + 1), ly = (i / (AB_Z + 1)) % (AB_Y + 1), lx = i / ((AB_Z + 1) * (AB_Y + 1));
        const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
        if (gx > N || gy > N || gz > N) continue;
        const long long n = ((long long)gx * NN + gy) * NN + gz;
        const bool face = lx == 0 || lx == AB_X || ly == 0 || ly == AB_Y || lz == 0 || lz == AB_Z;
        if (face) atomicAdd(a.y + n, acc[i]);
        else a.y[n] = acc[i];
    }
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
__global__ void __launch_bounds__(ST) k_finish_atomic(FinishArgs a) {
    __shared__ double sh[MAXQ][8];
    DevState* st = a.st;
    const int N = a.N;
    const Part& P = a.part;
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
    const SlabTile T = slab_tile(P, blockIdx.x);
    const SlabPos G = slab_pos(P, T, threadIdx.x);
    const long long plane = (long long)P.NN * P.NN;
    for (int ix = T.xa; ix <= T.xb; ++ix) {
        const bool xbnd = ix == 0 || ix == N;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            if (!sp_out(G.fl, k)) continue;
            const long long n = (long long)ix * plane + G.noff[k];
            const bool bnd = xbnd || sp_yzb(G.fl, k);
            double yv = bnd ? 0.0 : a.y[n];
            if (fi_ap && n == fi_idx) yv = flipbit(yv, fi_bit);
            const double pv = __ldg(p + n);
            if (a.role == ROLE_LOOP) part[0] = dfma(pv, yv, part[0]);
            if (a.d1) {
                part[1] = bnd ? dfma(0.0, yv, part[1]) : dadd(part[1], yv);
                part[2] = dfma(__ldg(a.w + n), pv, part[2]);
                part[3] = dfma(pv, pv, part[3]);
            }
            if (rhs) yv = dfma(a.dtF, __ldg(a.F + n), yv);
            a.y[n] = yv;
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
