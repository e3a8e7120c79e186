// hs_batch_kernels.cuh -- kernels of the batched mixed-precision solver
// (hs_batch.cu).  Many independent transient-heat solves advance together:
// every launch covers the operator tiles (column partition) or flat blocks (vector work)
// of all instances, and a block finds its instance through a map.  Each
// implicit-Euler step solves (M + dt K) T = M T_old by defect correction:
// FP64 residual r = b - A T (the column-march operator in FP64, ABFT checked),
// an FP32 Jacobi-PCG solve of A d = r to a loose relative tolerance (FP32
// operator and preconditioner, FP64 dot products of the FP32 values), and
// T += d in FP64, until ||b - A T|| / ||b|| < rtol.
// The CG dot products, the outer residual and the ABFT checksum sums are
// accumulated in FP64 with compensation (hs_csum.h): every partial is a pair
// (hi, lo), stored as quantity q and q + NQ, and merged pair-wise.
#pragma once
#include "hs_kernels.cuh"
#include "hs_csum.h"

namespace hs {

// canonical block tree (as cta_tree_sum) over compensated pairs; sh holds
// 2*NQ rows of 8; result valid in thread 0
template <int NQ>
__device__ __forceinline__ void cta_tree_csum(CSum (&v)[NQ], double (*sh)[8]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            const CSum o{__shfl_xor_sync(0xffffffffu, v[q].hi, off), __shfl_xor_sync(0xffffffffu, v[q].lo, off)};
            csum_merge(v[q], o);
        }
    }
    __syncthreads();
    if (lane == 0 && warp < 8) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) { sh[q][warp] = v[q].hi; sh[NQ + q][warp] = v[q].lo; }
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            CSum u{(lane < 8) ? sh[q][lane] : 0.0, (lane < 8) ? sh[NQ + q][lane] : 0.0};
#pragma unroll
            for (int off = 4; off >= 1; off >>= 1) {
                const CSum o{__shfl_xor_sync(0xffffffffu, u.hi, off), __shfl_xor_sync(0xffffffffu, u.lo, off)};
                csum_merge(u, o);
            }
            v[q] = u;
        }
    }
}
// store a block's compensated partials: hi as quantity q, lo as q + NQ
template <int NQ>
__device__ __forceinline__ void store_cpartials(const CSum (&v)[NQ], double* base, long long stride, long long idx) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        base[q * stride + idx] = v[q].hi;
        base[(NQ + q) * stride + idx] = v[q].lo;
    }
}

// per-instance scalars, device resident
struct BState {
    // inner FP32 PCG
    double rho, alpha, beta, bn_in, tol_in;
    int iter, done, broken, pad0;
    // outer defect correction
    double bn64, rel64, d1_last, d1_max64, d1_max32;
    double norm_wA, norm_wM;
    int outer, odone, pad1, pad2;
    // counters over the run
    long long inner_total, outer_total, applies32, applies64;
    // armed vector fault of the current step: level 5 p32 (after formation),
    // 6 r32 (after its update), 7 Ap32 (after projection), at correction
    // fi_outer (1-based) and inner iteration fi_iter; 0 = none
    int fi_vec, fi_outer, fi_iter, fi_bit;
    long long fi_idx;
    int fi_fired;           // the armed fault has fired
    int stalls;             // steps that ended at max_outer without reaching rtol
    int inner_bad;          // the current inner solve went non-finite: its correction is discarded
    int inner_faults;       // inner solves discarded so far
    int has_prev;           // the previous step's field is kept (extrapolated start)
    int extrap;             // this step starts from 2 T - T_prev
};

__device__ __forceinline__ float flipf(float x, int bit) {
    return __uint_as_float(__float_as_uint(x) ^ (1u << bit));
}
// the armed fault of level `vec` fires in this inner iteration
__device__ __forceinline__ bool fi_now(const BState* st, int vec) {
    return st->fi_vec == vec && st->outer == st->fi_outer && st->iter == st->fi_iter;
}

// instance descriptor (device array, rewritten by the host between rounds)
struct BInst {
    Part part;                 // flat blocks of this instance (vector work)
    ColLayout col;             // operator tiles of this instance (column partition)
    long long tile0, flat0;    // first global tile / flat block
    double dt;
    double cm[4], ck[4];       // wht eigen-constants / 8 of this grid
    float cmf[4], ckf[4];
    int active, pad;
    double* T;                 // solution (updated in place)
    double* b;                 // right-hand side M T_old
    double* y64;               // FP64 operator output
    double* r64;               // FP64 residual
    double* Tm1;               // field at the start of the previous step (extrapolated start)
    const double2* coef64;     // (rho*c, k) per element
    const float2* coef32;
    const double* wA;          // ABFT weights A 1_int, M 1_int (FP64)
    const double* wM;
    const float* dinv32;       // 1 / diag, FP32
    float* r32;
    float* z32;
    float* p32a;
    float* p32b;
    float* Ap32;
    float* d32;                // correction
    BState* st;
};

struct BatchArgs {
    const BInst* inst;
    const int* tile2inst;      // global tile -> instance slot (-1: none)
    const int* flat2inst;      // global flat block -> instance slot
    int n_inst, pad;
    long long ntiles, nflat;   // capacity of the grids
    double* pa;                // apply partials: [q * ntiles + tile]
    double* pf;                // flat partials:  [q * nflat + block]
    double rtol, inner_tol;
    int max_outer, max_inner;
    int detect, extrapolate;
};

template <typename V> struct VTraits;
template <> struct VTraits<float> {
    using V2 = float2;
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
};
template <> struct VTraits<double> {
    using V2 = double2;
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
};

// the Walsh-Hadamard element operator in precision V (same structure as elem_wht)
template <typename V>
__device__ __forceinline__ void elem_wht_v(V* v, V rhoc, V dk, const V* cm, const V* ck) {
    using T = VTraits<V>;
#pragma unroll
    for (int bit = 1; bit <= 4; bit <<= 1)
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (!(q & bit)) { const V u = v[q], w = v[q | bit]; v[q] = T::add(u, w); v[q | bit] = T::sub(u, w); }
    const V l0 = T::mul(rhoc, cm[0]);
    const V l1 = T::fma(dk, ck[1], T::mul(rhoc, cm[1]));
    const V l2 = T::fma(dk, ck[2], T::mul(rhoc, cm[2]));
    const V l3 = T::fma(dk, ck[3], T::mul(rhoc, cm[3]));
    v[0] = T::mul(v[0], l0);
    v[1] = T::mul(v[1], l1); v[2] = T::mul(v[2], l1); v[4] = T::mul(v[4], l1);
    v[3] = T::mul(v[3], l2); v[5] = T::mul(v[5], l2); v[6] = T::mul(v[6], l2);
    v[7] = T::mul(v[7], l3);
#pragma unroll
    for (int bit = 1; bit <= 4; bit <<= 1)
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (!(q & bit)) { const V u = v[q], w = v[q | bit]; v[q] = T::add(u, w); v[q | bit] = T::sub(u, w); }
}

// Batched operator, column-march warps (the FP64 solver's k_apply_col design,
// hs_colop.cuh) in precision V on one instance's column partition.  KIND 0:
// y64 = A T (FP64, residual); 1: b = M T (FP64, right-hand side); 2: inner
// FP32 loop, p = z (+ beta p), Ap = A p.  Partials per tile, compensated
// (hi, lo): p.Ap (KIND 2) and D1: 1_int.y, w.x, x.x.
enum BKind { BK_RESID = 0, BK_RHS = 1, BK_LOOP = 2 };

template <typename V>
struct BColStep {
    V a0, a1, b0, b1, cr, ck;
    double w;
};

__device__ __forceinline__ float flipv(float x, int bit) { return flipf(x, bit); }
__device__ __forceinline__ double flipv(double x, int bit) { return flipbit(x, bit); }

// FI false: no vector fault is armed for this launch
template <typename V, int KIND, bool FI>
__device__ __forceinline__ void kb_col_march(const BatchArgs& B, const BInst& I, const ColLane& C,
                                             CSum (&part)[MAXQ]) {
    using VT = VTraits<V>;
    using V2 = typename VT::V2;
    constexpr int NS = CR + 2;
    static_assert(NS % 3 == 0, "three rotating load sets per layer");
    BState* st = I.st;
    const bool loop = KIND == BK_LOOP;
    const int N = I.col.N, NN = I.col.NN;
    const int ec = C.ec, r0 = C.r0, xa = C.xa, xb = C.xb;
    const V dtv = (V)((KIND == BK_RHS) ? 0.0 : I.dt);
    V cm[4], ck[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        cm[j] = (sizeof(V) == 4) ? (V)I.cmf[j] : (V)I.cm[j];
        ck[j] = (sizeof(V) == 4) ? (V)I.ckf[j] : (V)I.ck[j];
    }
    const int iter = loop ? st->iter : 0;
    const V beta = (V)(loop ? st->beta : 0.0);
    const V* srcA;
    const V* srcB = nullptr;
    V* pout = nullptr;
    V* yout;
    if constexpr (KIND == BK_LOOP) {
        srcA = reinterpret_cast<const V*>(I.z32);
        srcB = (iter > 0) ? reinterpret_cast<const V*>((iter & 1) ? I.p32a : I.p32b) : nullptr;
        pout = reinterpret_cast<V*>((iter & 1) ? I.p32b : I.p32a);
        yout = reinterpret_cast<V*>(I.Ap32);
    } else {
        srcA = reinterpret_cast<const V*>(I.T);
        yout = reinterpret_cast<V*>(KIND == BK_RHS ? I.b : I.y64);
    }
    const bool two = srcB != nullptr;
    const double* w = (KIND == BK_RHS) ? I.wM : I.wA;
    const bool d1 = B.detect != 0;
    int fi_p = 0, fi_ap = 0, fi_bit = 0;
    long long fi_idx = -1;
    if constexpr (KIND == BK_LOOP && FI) {
        fi_p = fi_now(st, FI_P); fi_ap = fi_now(st, FI_AP);
        fi_bit = st->fi_bit; fi_idx = st->fi_idx;
    }
    const bool live = C.fl & 1u;
    const bool own = (C.fl & 2u) && ec <= N;
    const bool colv = live && ec >= 0 && ec <= N;
    const bool colv1 = live && ec + 1 >= 0 && ec + 1 <= N;
    const bool ecv = live && ec >= 0 && ec < N;
    unsigned rowv = 0u, erowv = 0u, orow = 0u;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        const int r = r0 - 1 + i;
        if (r >= 0 && r <= N) rowv |= 1u << i;
        if (i >= 1 && r - 1 >= 0 && r - 1 < N) erowv |= 1u << i;
        if (own && i >= 1 && i <= CR && r <= N) orow |= 1u << i;
    }
    if (own && (C.fl & 4u)) orow |= 1u << (NS - 1);
    const int lane_n = (r0 - 1) * NN + ec;
    const int lane_e = (r0 - 2) * N + ec;

    auto load = [&](BColStep<V>& S, int x, int i) {
        const int xp = x + 1;
        const bool pv = xp >= 0 && xp <= N && xp <= xb + 1 && ((rowv >> i) & 1u);
        const int n = xp * NN * NN + lane_n + i * NN;
        const bool v0 = pv && colv, v1 = pv && colv1;
        S.a0 = v0 ? __ldg(srcA + n) : (V)0;
        S.a1 = v1 ? __ldg(srcA + n + 1) : (V)0;
        S.b0 = (v0 && two) ? __ldg(srcB + n) : (V)0;
        S.b1 = (v1 && two) ? __ldg(srcB + n + 1) : (V)0;
        S.w = (d1 && v0 && xp >= xa && xp <= xb && ((orow >> i) & 1u)) ? __ldg(w + n) : 0.0;
        const bool ev = i >= 1 && x >= xa - 1 && x >= 0 && x < N && ecv && ((erowv >> i) & 1u);
        const int e = x * N * N + lane_e + i * N;
        if constexpr (sizeof(V) == 4) {
            const float2 c = ev ? __ldg(I.coef32 + e) : make_float2(0.f, 0.f);
            S.cr = c.x; S.ck = c.y;
        } else {
            const double2 c = ev ? __ldg(I.coef64 + e) : make_double2(0.0, 0.0);
            S.cr = c.x; S.ck = c.y;
        }
    };

    V fp[CR + 1][4];
    V slo[CR + 1];
    V pk[CR + 1];
#pragma unroll
    for (int j = 0; j <= CR; ++j) {
        slo[j] = (V)0; pk[j] = (V)0;
        fp[j][0] = fp[j][1] = fp[j][2] = fp[j][3] = (V)0;
    }
    BColStep<V> B0, B1, B2;
    load(B0, xa - 2, 0);
    load(B1, xa - 2, 1);
    for (int x = xa - 2; x <= xb; ++x) {
        const bool el = x >= xa - 1 && x >= 0 && x < N;
        const bool cpl = x >= xa;
        const bool fown = x + 1 >= xa && x + 1 <= xb;
        V zsP_s = (V)0, zsP_d = (V)0, pnA = (V)0;
        V hq2 = (V)0, hL3 = (V)0, hq6 = (V)0, hL7 = (V)0;
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            BColStep<V>& S = (i % 3 == 0) ? B0 : (i % 3 == 1) ? B1 : B2;
            const V a0 = S.a0, a1 = S.a1, b0 = S.b0, b1 = S.b1, cr = S.cr, ckk = S.ck;
            const double wv = S.w;
            {
                BColStep<V>& SL = ((i + 2) % 3 == 0) ? B0 : ((i + 2) % 3 == 1) ? B1 : B2;
                if (i + 2 < NS) load(SL, x, i + 2);
                else load(SL, x + 1, i + 2 - NS);
            }
            const int r = r0 - 1 + i;
            V pA = two ? VT::fma(beta, b0, a0) : a0;
            V pB = two ? VT::fma(beta, b1, a1) : a1;
            const int nrow = (x + 1) * NN * NN + lane_n + i * NN;
            if constexpr (KIND == BK_LOOP && FI) {
                if (fi_p && x + 1 <= N && ((rowv >> i) & 1u)) {
                    if (colv && (long long)nrow == fi_idx) { pA = flipv(pA, fi_bit); st->fi_fired = 1; }
                    if (colv1 && (long long)nrow + 1 == fi_idx) { pB = flipv(pB, fi_bit); st->fi_fired = 1; }
                }
            }
            if (fown && ((orow >> i) & 1u)) {
                if (loop) __stwb(pout + nrow, pA);
                if (d1) {
                    const double pd = (double)pA;
                    csum_fma(part[2], wv, pd);
                    part[3].hi = dfma(pd, pd, part[3].hi);     // the norm only scales the threshold
                }
            }
            const V zs_s = VT::add(pA, pB), zs_d = VT::sub(pA, pB);
            if (i >= 1) {
                const int j = i - 1;
                V v[8];
                const V f0 = VT::add(zsP_s, zs_s), f1 = VT::add(zsP_d, zs_d);
                const V f2 = VT::sub(zsP_s, zs_s), f3 = VT::sub(zsP_d, zs_d);
                if (el) {
                    v[0] = VT::add(fp[j][0], f0); v[1] = VT::add(fp[j][1], f1);
                    v[2] = VT::add(fp[j][2], f2); v[3] = VT::add(fp[j][3], f3);
                    v[4] = VT::sub(fp[j][0], f0); v[5] = VT::sub(fp[j][1], f1);
                    v[6] = VT::sub(fp[j][2], f2); v[7] = VT::sub(fp[j][3], f3);
                    const V dk = VT::mul(dtv, ckk);
                    const V l0 = VT::mul(cr, cm[0]);
                    const V l1 = VT::fma(dk, ck[1], VT::mul(cr, cm[1]));
                    const V l2 = VT::fma(dk, ck[2], VT::mul(cr, cm[2]));
                    const V l3 = VT::fma(dk, ck[3], VT::mul(cr, cm[3]));
                    v[0] = VT::mul(v[0], l0);
                    v[1] = VT::mul(v[1], l1); v[2] = VT::mul(v[2], l1); v[4] = VT::mul(v[4], l1);
                    v[3] = VT::mul(v[3], l2); v[5] = VT::mul(v[5], l2); v[6] = VT::mul(v[6], l2);
                    v[7] = VT::mul(v[7], l3);
#pragma unroll
                    for (int bit = 1; bit <= 4; bit <<= 1)
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            if (!(q & bit)) { const V u = v[q], t = v[q | bit]; v[q] = VT::add(u, t); v[q | bit] = VT::sub(u, t); }
                } else {
#pragma unroll
                    for (int q = 0; q < 8; ++q) v[q] = (V)0;
                }
                fp[j][0] = f0; fp[j][1] = f1; fp[j][2] = f2; fp[j][3] = f3;
                const V L1 = __shfl_up_sync(0xffffffffu, v[1], 1), L3 = __shfl_up_sync(0xffffffffu, v[3], 1);
                const V L5 = __shfl_up_sync(0xffffffffu, v[5], 1), L7 = __shfl_up_sync(0xffffffffu, v[7], 1);
                if (j >= 1) {
                    const int oj = j - 1;
                    if (cpl && ((orow >> j) & 1u)) {
                        const int er = r - 1;
                        const int n = x * NN * NN + lane_n + j * NN;
                        const bool bnd = x == 0 || x == N || er == 0 || er == N || ec == 0 || ec == N;
                        V y = bnd ? (V)0 : VT::add(VT::add(VT::add(VT::add(slo[oj], v[0]), hL3), hq2), L1);
                        if constexpr (KIND == BK_LOOP && FI) {
                            if (fi_ap && (long long)n == fi_idx) { y = flipv(y, fi_bit); st->fi_fired = 1; }
                        }
                        const double yd = (double)y;
                        if (loop) csum_fma(part[0], (double)pk[oj], yd);
                        if (d1 && !bnd) csum_add(part[1], yd);
                        __stwb(yout + n, y);
                    }
                    slo[oj] = VT::add(VT::add(VT::add(VT::add((V)0, v[4]), hL7), hq6), L5);
                    pk[oj] = pnA;
                }
                hq2 = v[2]; hL3 = L3; hq6 = v[6]; hL7 = L7;
            }
            zsP_s = zs_s; zsP_d = zs_d;
            pnA = pA;
        }
        if (C.fl & 4u) {
            if (cpl && own) {
                const int n = (x * NN + N) * NN + ec;
                V y = (V)0;
                if constexpr (KIND == BK_LOOP && FI) {
                    if (fi_ap && (long long)n == fi_idx) { y = flipv(y, fi_bit); st->fi_fired = 1; }
                }
                if (loop) csum_fma(part[0], (double)pk[CR], (double)y);
                __stwb(yout + n, y);
            }
            pk[CR] = pnA;
        }
    }
}

template <typename V, int KIND>
__global__ void __launch_bounds__(RT, 1) kb_apply(BatchArgs B) {
    __shared__ double sh[2 * MAXQ][8];
    const long long t = blockIdx.x;
    if (t >= B.ntiles) return;
    const int slot = B.tile2inst[t];
    if (slot < 0) return;
    const BInst& I = B.inst[slot];
    if (!I.active) return;
    const BState* st = I.st;
    if constexpr (KIND == BK_LOOP) {
        if (st->odone || st->done) return;
    } else if constexpr (KIND == BK_RESID) {
        if (st->odone) return;
    }
    CSum part[MAXQ] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    const long long wt = (t - I.tile0) * CW + (threadIdx.x >> 5);
    const ColLane C = col_lane(I.col, wt, threadIdx.x & 31);
    if (wt < I.col.ntasks) {                       // warp-uniform
        if constexpr (KIND == BK_LOOP) {
            if (fi_now(st, FI_P) || fi_now(st, FI_AP)) kb_col_march<V, KIND, true>(B, I, C, part);
            else kb_col_march<V, KIND, false>(B, I, C, part);
        } else {
            kb_col_march<V, KIND, false>(B, I, C, part);
        }
    }
    if (KIND != BK_LOOP && !B.detect) return;
    cta_tree_csum<MAXQ>(part, sh);
    if (threadIdx.x == 0) store_cpartials<MAXQ>(part, B.pa, B.ntiles, t);
}

// compensated sums of one instance's partials: count (hi, lo) pairs per
// quantity, hi of quantity q at base + q*qstride, lo at base + (q+NQ)*qstride;
// RT strided sequential merges, then the block tree; valid in thread 0
template <int NQ>
__device__ __forceinline__ void inst_sums(double (&v)[NQ], const double* base, long long count, long long qstride,
                                          double (*sh)[8]) {
    constexpr int FB = 8;
    CSum acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = CSum{0.0, 0.0};
    for (long long k0 = threadIdx.x; k0 < count; k0 += (long long)RT * FB) {
        double th[NQ][FB], tl[NQ][FB];
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int u = 0; u < FB; ++u) {
                const long long k = k0 + (long long)u * RT;
                th[q][u] = (k < count) ? __ldcg(base + q * qstride + k) : 0.0;
                tl[q][u] = (k < count) ? __ldcg(base + (NQ + q) * qstride + k) : 0.0;
            }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int u = 0; u < FB; ++u)
                if (k0 + (long long)u * RT < count) csum_merge(acc[q], CSum{th[q][u], tl[q][u]});
    }
    cta_tree_csum<NQ>(acc, sh);
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = csum_value(acc[q]);
}

__device__ __forceinline__ double d1_rel(const double (&p)[MAXQ], double nw) {
    const double nx = __dsqrt_rn(p[3]);
    double rel = __ddiv_rn(fabs(dsub(p[1], p[2])), dfma(nw, nx, 1e-300));
    if (!isfinite(rel)) rel = 1e300;
    return rel;
}

// one block per instance: operator partials -> D1 (and alpha in the loop)
template <int KIND>
__global__ void __launch_bounds__(RT) kb_final_apply(BatchArgs B) {
    __shared__ double sh[2 * MAXQ][8];
    const int slot = blockIdx.x;
    if (slot >= B.n_inst) return;
    const BInst& I = B.inst[slot];
    if (!I.active) return;
    BState* st = I.st;
    if (KIND == BK_LOOP && (st->odone || st->done)) return;
    if (KIND == BK_RESID && st->odone) return;
    double p[MAXQ];
    inst_sums<MAXQ>(p, B.pa + I.tile0, I.col.ntiles, B.ntiles, sh);
    if (threadIdx.x != 0) return;
    if (B.detect) {
        const double rel = d1_rel(p, KIND == BK_RHS ? st->norm_wM : st->norm_wA);
        st->d1_last = rel;
        if (KIND == BK_LOOP) st->d1_max32 = fmax(st->d1_max32, rel);
        else st->d1_max64 = fmax(st->d1_max64, rel);
    }
    if (KIND == BK_LOOP) {
        st->applies32 += 1;
        if (!isfinite(p[0])) { st->inner_bad = 1; st->done = 1; }
        else if (fabs(p[0]) < 1e-30) { st->broken = 1; st->done = 1; }
        else st->alpha = __ddiv_rn(st->rho, p[0]);
    } else {
        st->applies64 += 1;
    }
}

// flat block of an instance: slot, local block, first node, node count (0..KF)
struct FlatPos { int slot; long long m0; int cnt; };
__device__ __forceinline__ FlatPos flat_pos(const BatchArgs& B) {
    FlatPos f{-1, 0, 0};
    const long long g = blockIdx.x;
    if (g >= B.nflat) return f;
    const int slot = B.flat2inst[g];
    if (slot < 0) return f;
    const BInst& I = B.inst[slot];
    const long long lb = g - I.flat0;
    f.slot = slot;
    f.m0 = (lb * RT + threadIdx.x) * KF;
    const long long Nn = I.part.Nn;
    f.cnt = (f.m0 + 1 < Nn) ? 2 : (f.m0 < Nn ? 1 : 0);
    return f;
}

// residual r = b - A T in FP64 and the start of an inner solve:
// r32 = r, z32 = r32 / d, d32 = 0; partials r.r, b.b (FP64), r32.z32, r32.r32
__global__ void __launch_bounds__(RT) kb_resid(BatchArgs B) {
    __shared__ double sh[2 * MAXQ][8];
    const FlatPos f = flat_pos(B);
    CSum part[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    if (f.slot >= 0) {
        const BInst& I = B.inst[f.slot];
        if (I.active && !I.st->odone) {
            for (int k = 0; k < f.cnt; ++k) {
                const long long m = f.m0 + k;
                const double bv = I.b[m];
                const double rv = dsub(bv, I.y64[m]);
                I.r64[m] = rv;
                const float r32 = (float)rv;
                const float z = __fmul_rn(r32, I.dinv32[m]);
                I.r32[m] = r32; I.z32[m] = z; I.d32[m] = 0.f;
                csum_fma(part[0], rv, rv);
                csum_fma(part[1], bv, bv);
                csum_add(part[2], dmul((double)r32, (double)z));     // products of FP32 values are exact
                csum_add(part[3], dmul((double)r32, (double)r32));
            }
        }
    }
    cta_tree_csum<4>(part, sh);
    if (threadIdx.x == 0 && blockIdx.x < B.nflat) store_cpartials<4>(part, B.pf, B.nflat, blockIdx.x);
}

// one block per instance: outer convergence test and the inner solve's start
__global__ void __launch_bounds__(RT) kb_outer_final(BatchArgs B) {
    __shared__ double sh[2 * MAXQ][8];
    const int slot = blockIdx.x;
    if (slot >= B.n_inst) return;
    const BInst& I = B.inst[slot];
    if (!I.active) return;
    BState* st = I.st;
    if (st->odone) return;
    double p[4];
    inst_sums<4>(p, B.pf + I.flat0, I.part.nflat, B.nflat, sh);
    if (threadIdx.x != 0) return;
    if (st->outer == 0) {
        double bn = __dsqrt_rn(p[1]);
        if (bn < 1e-30) bn = 1.0;
        st->bn64 = bn;
    }
    st->rel64 = __ddiv_rn(__dsqrt_rn(p[0]), st->bn64);
    const bool conv = st->rel64 < B.rtol;
    if (conv || st->outer >= B.max_outer) {
        if (!conv) st->stalls += 1;
        st->odone = 1; st->done = 1;
        return;
    }
    st->outer += 1;
    st->outer_total += 1;
    st->rho = p[2];
    st->bn_in = __dsqrt_rn(p[3]);
    // solve only as far as the outer target needs: max(inner_tol, rtol / (2 rel64))
    st->tol_in = fmax(B.inner_tol, __ddiv_rn(0.5 * B.rtol, st->rel64));
    st->iter = 0; st->broken = 0; st->beta = 0.0; st->inner_bad = 0;
    st->done = (st->bn_in < 1e-300 || !isfinite(st->bn_in) || !isfinite(p[2])) ? 1 : 0;
    if (!isfinite(st->bn_in) || !isfinite(p[2])) st->inner_bad = 1;
}

// inner FP32 update: d += alpha p, r -= alpha Ap, z = r / diag; partials r.r, r.z
__global__ void __launch_bounds__(RT) kb_update32(BatchArgs B) {
    __shared__ double sh[2 * MAXQ][8];
    const FlatPos f = flat_pos(B);
    CSum part[2] = {{0.0, 0.0}, {0.0, 0.0}};
    if (f.slot >= 0) {
        const BInst& I = B.inst[f.slot];
        const BState* st = I.st;
        if (I.active && !st->odone && !st->done) {
            const int iter = st->iter;
            const float alpha = (float)st->alpha;
            const float* p = (iter & 1) ? I.p32b : I.p32a;
            const bool fr = fi_now(st, FI_RV);
            // the thread's node pair as 8-byte vectors (m0 is even, the buffers 256-byte aligned)
            float dv[2], pv[2], qv[2], rv[2], iv[2];
            if (f.cnt == 2) {
                const float2 a = *reinterpret_cast<const float2*>(I.d32 + f.m0);
                const float2 b = *reinterpret_cast<const float2*>(p + f.m0);
                const float2 c = *reinterpret_cast<const float2*>(I.Ap32 + f.m0);
                const float2 d = *reinterpret_cast<const float2*>(I.r32 + f.m0);
                const float2 e = __ldg(reinterpret_cast<const float2*>(I.dinv32 + f.m0));
                dv[0] = a.x; dv[1] = a.y; pv[0] = b.x; pv[1] = b.y; qv[0] = c.x; qv[1] = c.y;
                rv[0] = d.x; rv[1] = d.y; iv[0] = e.x; iv[1] = e.y;
            } else {
                for (int k = 0; k < 2; ++k) {
                    const bool in = k < f.cnt;
                    const long long m = f.m0 + k;
                    dv[k] = in ? I.d32[m] : 0.f; pv[k] = in ? p[m] : 0.f; qv[k] = in ? I.Ap32[m] : 0.f;
                    rv[k] = in ? I.r32[m] : 0.f; iv[k] = in ? I.dinv32[m] : 0.f;
                }
            }
            float zv[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                dv[k] = __fmaf_rn(alpha, pv[k], dv[k]);
                float r = __fmaf_rn(-alpha, qv[k], rv[k]);
                if (fr && f.m0 + k == st->fi_idx && k < f.cnt) { r = flipf(r, st->fi_bit); I.st->fi_fired = 1; }
                rv[k] = r;
                zv[k] = __fmul_rn(r, iv[k]);
                if (k < f.cnt) {
                    csum_add(part[0], dmul((double)r, (double)r));         // exact products
                    csum_add(part[1], dmul((double)r, (double)zv[k]));
                }
            }
            if (f.cnt == 2) {
                *reinterpret_cast<float2*>(I.d32 + f.m0) = make_float2(dv[0], dv[1]);
                *reinterpret_cast<float2*>(I.r32 + f.m0) = make_float2(rv[0], rv[1]);
                *reinterpret_cast<float2*>(I.z32 + f.m0) = make_float2(zv[0], zv[1]);
            } else if (f.cnt == 1) {
                I.d32[f.m0] = dv[0]; I.r32[f.m0] = rv[0]; I.z32[f.m0] = zv[0];
            }
        }
    }
    cta_tree_csum<2>(part, sh);
    if (threadIdx.x == 0 && blockIdx.x < B.nflat) store_cpartials<2>(part, B.pf, B.nflat, blockIdx.x);
}

// one block per instance: inner convergence and beta
__global__ void __launch_bounds__(RT) kb_final_update32(BatchArgs B) {
    __shared__ double sh[2 * MAXQ][8];
    const int slot = blockIdx.x;
    if (slot >= B.n_inst) return;
    const BInst& I = B.inst[slot];
    if (!I.active) return;
    BState* st = I.st;
    if (st->odone || st->done) return;
    double p[2];
    inst_sums<2>(p, B.pf + I.flat0, I.part.nflat, B.nflat, sh);
    if (threadIdx.x != 0) return;
    st->inner_total += 1;
    const double rel = __ddiv_rn(__dsqrt_rn(p[0]), st->bn_in);
    if (!isfinite(rel) || !isfinite(p[1])) { st->inner_bad = 1; st->done = 1; return; }
    if (rel < st->tol_in || st->iter + 1 >= B.max_inner) { st->done = 1; return; }
    st->beta = __ddiv_rn(p[1], st->rho);
    st->rho = p[1];
    st->iter += 1;
}

// T += d (FP64) at the interior nodes, for the instances whose inner solve
// just finished; Dirichlet values are never changed, and a correction from an
// inner solve that went non-finite is discarded (the next correction re-solves)
__global__ void __launch_bounds__(RT) kb_correct(BatchArgs B) {
    const FlatPos f = flat_pos(B);
    if (f.slot < 0) return;
    const BInst& I = B.inst[f.slot];
    if (!I.active || I.st->odone || I.st->inner_bad) return;
    const int N = I.part.N;
    for (int k = 0; k < f.cnt; ++k) {
        const long long m = f.m0 + k;
        if (!is_bnd(m, N)) I.T[m] = dadd(I.T[m], (double)I.d32[m]);
    }
}

// count the discarded inner solves (one thread per instance, after kb_correct)
__global__ void kb_count_bad(BatchArgs B) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= B.n_inst) return;
    const BInst& I = B.inst[slot];
    if (!I.active || I.st->odone) return;
    if (I.st->inner_bad) I.st->inner_faults += 1;
}

// set-up helpers: FP32 reciprocal of the diagonal; the interior indicator
__global__ void k_recip32(long long n, const double* d, float* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)__ddiv_rn(1.0, d[i]);
}
// interleaved FP64 and FP32 element coefficients (rho*c, k)
__global__ void k_pack_coef(long long ne, const double* rhoc, const double* k, double2* c64, float2* c32) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (long long)gridDim.x * blockDim.x) {
        const double r = rhoc[i], kk = k[i];
        c64[i] = make_double2(r, kk);
        c32[i] = make_float2(__double2float_rn(r), __double2float_rn(kk));
    }
}
// fresh state of an added instance: checksum weight norms from their squared sums, nothing to iterate
__global__ void kb_init_state(BState* st, const double* sq) {
    BState s{};
    s.norm_wM = __dsqrt_rn(sq[0]);
    s.norm_wA = __dsqrt_rn(sq[2]);
    s.odone = 1; s.done = 1;
    *st = s;
}
__global__ void k_ones_interior(int N, double* v) {
    const long long NN = N + 1, Nn = NN * NN * NN;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < Nn; i += (long long)gridDim.x * blockDim.x)
        v[i] = is_bnd(i, N) ? 0.0 : 1.0;
}

// arm (vec > 0) or disarm (vec == 0) the vector fault of one instance
__global__ void kb_arm(BState* st, int vec, int outer, int iter, long long idx, int bit) {
    st->fi_vec = vec; st->fi_outer = outer; st->fi_iter = iter; st->fi_idx = idx; st->fi_bit = bit;
}

// step start: outer state of every active instance
__global__ void kb_step_begin(BatchArgs B) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= B.n_inst) return;
    const BInst& I = B.inst[slot];
    if (!I.active) return;
    BState* st = I.st;
    st->outer = 0; st->odone = 0; st->done = 1; st->iter = 0;
    st->extrap = B.extrapolate && st->has_prev;
    st->has_prev = 1;
}

// start of the step's solve (after b = M T): T <- 2 T - T_prev where a
// previous field exists, else T unchanged; T_prev <- T of this step's start
__global__ void __launch_bounds__(RT) kb_extrapolate(BatchArgs B) {
    const FlatPos f = flat_pos(B);
    if (f.slot < 0 || !B.extrapolate) return;
    const BInst& I = B.inst[f.slot];
    if (!I.active) return;
    const bool ex = I.st->extrap;
    for (int k = 0; k < f.cnt; ++k) {
        const long long m = f.m0 + k;
        const double t = I.T[m];
        if (ex) I.T[m] = dfma(2.0, t, -I.Tm1[m]);
        I.Tm1[m] = t;
    }
}

// loop conditions: any active instance still in its outer loop (WHICH 0) /
// in an inner solve (WHICH 1)
template <int WHICH>
__global__ void kb_cond(BatchArgs B, cudaGraphConditionalHandle h, int* flag) {
    int any = 0;
    for (int s = threadIdx.x; s < B.n_inst; s += blockDim.x) {
        const BInst& I = B.inst[s];
        if (!I.active) continue;
        const BState* st = I.st;
        if (WHICH == 0 ? !st->odone : (!st->odone && !st->done)) any = 1;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        if (flag) *flag = any;                      // direct launches: the host reads the flag
        else cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

}  // namespace hs
