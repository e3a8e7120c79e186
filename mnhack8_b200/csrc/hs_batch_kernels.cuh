// hs_batch_kernels.cuh -- kernels of the batched mixed-precision solver
// (hs_batch.cu).  Many independent transient-heat solves advance together:
// every launch covers the slab tiles (operator) or flat blocks (vector work)
// of all instances, and a block finds its instance through a map.  Each
// implicit-Euler step solves (M + dt K) T = M T_old by defect correction:
// FP64 residual r = b - A T (the slab operator in FP64, ABFT checked),
// an FP32 Jacobi-PCG solve of A d = r to a loose relative tolerance (FP32
// operator and preconditioner, FP64 dot products of the FP32 values), and
// T += d in FP64, until ||b - A T|| / ||b|| < rtol.
// The sums of the FP64 applies (the outer residual ||b - A T||, ||b||, the
// ABFT checksum sums of the FP64 applies) and the inner solve's starting r.z
// and r.r are accumulated in FP64 with compensation (hs_csum.h); the inner
// FP32 iterations' sums are plain FP64 sums of FP32 values.  Every partial is
// a pair (hi, lo), stored as quantity q and q + NQ, and merged pair-wise.
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
    Part part;                 // slab tiles and flat blocks of this instance
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

template <typename V>
struct __align__(16) BSlabSmem {
    V P[2][SPOS];
    typename VTraits<V>::V2 Y1[SPOS], Y2[SPOS], Y3[SPOS];
    double sh[2 * MAXQ][8];
};

// Batched slab operator.  KIND 0: y64 = A T (FP64, residual); 1: b = M T
// (FP64, right-hand side); 2: inner FP32 loop, p = z (+ beta p), Ap = A p.
// Partials per tile: p.Ap (KIND 2), and D1: 1_int.y, w.x, x.x.
enum BKind { BK_RESID = 0, BK_RHS = 1, BK_LOOP = 2 };

// tile t of instance I; FI false: no vector fault is armed for this launch
template <typename V, int KIND, bool FI>
__device__ __forceinline__ void kb_tile(const BatchArgs& B, BSlabSmem<V>& S, long long t, const BInst& I) {
    using T2 = typename VTraits<V>::V2;
    using VT = VTraits<V>;
    BState* st = I.st;
    const bool loop = KIND == BK_LOOP;
    if constexpr (KIND == BK_LOOP) {
        if (st->odone || st->done) return;
    } else if constexpr (KIND == BK_RESID) {
        if (st->odone) return;
    }
    const Part& P = I.part;
    const int N = P.N, Cw = P.Cw;
    // node and element indices fit in 32 bits (N <= 1200)
    const unsigned plane = (unsigned)P.NN * (unsigned)P.NN, eplane = (unsigned)N * (unsigned)N;
    const SlabTile Tt = slab_tile(P, t - I.tile0);
    const SlabPos G = slab_pos(P, Tt, threadIdx.x);
    const unsigned fl = G.fl;
    const int tid = threadIdx.x, xa = Tt.xa, xb = Tt.xb;
    const V dtv = (V)((KIND == BK_RHS) ? 0.0 : I.dt);
    V cm[4], ck[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        cm[j] = (sizeof(V) == 4) ? (V)I.cmf[j] : (V)I.cm[j];
        ck[j] = (sizeof(V) == 4) ? (V)I.ckf[j] : (V)I.ck[j];
    }
    // inputs
    const int iter = loop ? st->iter : 0;
    const double betad = loop ? st->beta : 0.0;
    const V beta = (V)betad;
    const V* src_a;
    const V* src_b = nullptr;
    V* pout = nullptr;
    V* yout;
    if constexpr (KIND == BK_LOOP) {
        src_a = reinterpret_cast<const V*>(I.z32);
        src_b = (iter > 0) ? reinterpret_cast<const V*>((iter & 1) ? I.p32a : I.p32b) : nullptr;
        pout = reinterpret_cast<V*>((iter & 1) ? I.p32b : I.p32a);
        yout = reinterpret_cast<V*>(I.Ap32);
    } else {
        src_a = reinterpret_cast<const V*>(I.T);
        yout = reinterpret_cast<V*>(KIND == BK_RHS ? I.b : I.y64);
    }
    const bool two = src_b != nullptr;
    const double* w = (KIND == BK_RHS) ? I.wM : I.wA;
    const bool d1 = B.detect != 0;
    CSum part[MAXQ] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};

    V pA[SK], pB[SK], aA[SK], aB[SK], ra[SK], rb[SK], cr[SK], ckk[SK];
    double wv[SK];
    auto ld_raw = [&](int px) {
        const bool pv = px >= 0 && px <= N;
        const unsigned base = (unsigned)px * plane;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            const bool v = pv && sp_valid(fl, k);
            const unsigned n = base + (unsigned)G.noff[k];
            ra[k] = v ? __ldg(src_a + n) : (V)0;
            rb[k] = (v && two) ? __ldg(src_b + n) : (V)0;
        }
    };
    int fi_p = 0, fi_ap = 0, fi_bit = 0;
    long long fi_idx = -1;
    if constexpr (KIND == BK_LOOP && FI) {
        fi_p = fi_now(st, FI_P); fi_ap = fi_now(st, FI_AP);
        fi_bit = st->fi_bit; fi_idx = st->fi_idx;
    }
    auto form = [&](V (&p)[SK], int px) {
#pragma unroll
        for (int k = 0; k < SK; ++k) p[k] = two ? VT::fma(beta, rb[k], ra[k]) : ra[k];
        if constexpr (KIND == BK_LOOP && FI) {
            if (fi_p) {
#pragma unroll
                for (int k = 0; k < SK; ++k)
                    if (sp_valid(fl, k) && (long long)px * plane + G.noff[k] == fi_idx) {
                        p[k] = flipf(p[k], fi_bit);
                        st->fi_fired = 1;
                    }
            }
        }
    };
    auto ld_coef = [&](int ex) {
        const bool ev = ex >= 0 && ex < N;
        const unsigned base = (unsigned)ex * eplane;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            const bool v = ev && sp_elem(fl, k);
            const unsigned e = base + (unsigned)G.eoff[k];
            if constexpr (sizeof(V) == 4) {
                const float2 c = v ? __ldg(I.coef32 + e) : make_float2(0.f, 0.f);
                cr[k] = c.x; ckk[k] = c.y;
            } else {
                const double2 c = v ? __ldg(I.coef64 + e) : make_double2(0.0, 0.0);
                cr[k] = c.x; ckk[k] = c.y;
            }
        }
    };
    auto ld_w = [&](int px) {
        const bool pv = px >= xa && px <= xb;
        const unsigned base = (unsigned)px * plane;
#pragma unroll
        for (int k = 0; k < SK; ++k)
            wv[k] = (pv && d1 && sp_out(fl, k)) ? __ldg(w + (base + (unsigned)G.noff[k])) : 0.0;
    };
    auto layer = [&](int ix, int cur, V (&pc)[SK], V (&pn)[SK], V (&ac)[SK], V (&an)[SK]) {
        const int nxt = cur ^ 1;
        form(pn, ix + 1);
#pragma unroll
        for (int k = 0; k < SK; ++k) S.P[nxt][tid + k * ST] = pn[k];
        ld_raw(ix + 2 <= xb + 1 ? ix + 2 : -2);
        __syncthreads();
        if (ix >= 0 && ix < N) {
#pragma unroll
            for (int k = 0; k < SK; ++k) {
                if (!sp_elem(fl, k)) continue;
                const int j = tid + k * ST;
                V v[8];
                v[0] = pc[k];
                v[1] = S.P[cur][j + 1];
                v[2] = S.P[cur][j + Cw];
                v[3] = S.P[cur][j + Cw + 1];
                v[4] = pn[k];
                v[5] = S.P[nxt][j + 1];
                v[6] = S.P[nxt][j + Cw];
                v[7] = S.P[nxt][j + Cw + 1];
                elem_wht_v<V>(v, cr[k], VT::mul(dtv, ckk[k]), cm, ck);
                ac[k] = VT::add(ac[k], v[0]);
                an[k] = VT::add((V)0, v[4]);
                S.Y1[j + 1] = T2{v[1], v[5]};
                S.Y2[j + Cw] = T2{v[2], v[6]};
                S.Y3[j + Cw + 1] = T2{v[3], v[7]};
            }
        }
        ld_coef(ix + 1 <= xb ? ix + 1 : -1);
        __syncthreads();
        const unsigned base = (unsigned)ix * plane;
        const bool xbnd = ix == 0 || ix == N;
#pragma unroll
        for (int k = 0; k < SK; ++k) {
            if (!sp_out(fl, k)) continue;
            const int j = tid + k * ST;
            const bool yzin = !sp_yzb(fl, k);
            T2 y3{(V)0, (V)0}, y2 = y3, y1 = y3;
            if (yzin) { y3 = S.Y3[j]; y2 = S.Y2[j]; y1 = S.Y1[j]; }
            if (ix >= xa) {
                const unsigned n = base + (unsigned)G.noff[k];
                const bool bnd = !yzin || xbnd;
                V y = bnd ? (V)0 : VT::add(VT::add(VT::add(ac[k], y3.x), y2.x), y1.x);
                if constexpr (KIND == BK_LOOP && FI) {
                    if (fi_ap && (long long)n == fi_idx) { y = flipf(y, fi_bit); st->fi_fired = 1; }
                }
                const double pv = (double)pc[k], yd = (double)y;
                if constexpr (sizeof(V) == 8) {
                    // FP64 applies (right-hand side, outer residual): compensated sums
                    if (loop) csum_fma(part[0], pv, yd);
                    if (d1) {
                        if (!bnd) csum_add(part[1], yd);
                        csum_fma(part[2], wv[k], pv);
                        part[3].hi = dfma(pv, pv, part[3].hi);  // the norm only scales the threshold
                    }
                } else {
                    // FP32 inner applies: FP64 sums of FP32 values; their rounding (~1e-16 n)
                    // is far below the FP32 operator's own (~1e-9), so no compensation
                    if (loop) part[0].hi = dfma(pv, yd, part[0].hi);
                    if (d1) {
                        if (!bnd) part[1].hi = dadd(part[1].hi, yd);
                        part[2].hi = dfma(wv[k], pv, part[2].hi);
                        part[3].hi = dfma(pv, pv, part[3].hi);
                    }
                }
                __stwb(yout + n, y);                      // global stores (the pointers come from global memory)
                if (loop) __stwb(pout + n, pc[k]);
            }
            an[k] = yzin ? VT::add(VT::add(VT::add(an[k], y3.y), y2.y), y1.y) : (V)0;
        }
        ld_w(ix + 1);
    };
    ld_raw(xa - 1);
    form(pA, xa - 1);
#pragma unroll
    for (int k = 0; k < SK; ++k) { S.P[0][tid + k * ST] = pA[k]; aA[k] = (V)0; aB[k] = (V)0; }
    ld_raw(xa);
    ld_coef(xa - 1);
    for (int ix = xa - 1; ix <= xb; ++ix) {
        layer(ix, (ix - xa + 1) & 1, pA, pB, aA, aB);
#pragma unroll
        for (int k = 0; k < SK; ++k) { pA[k] = pB[k]; aA[k] = aB[k]; }
    }
    if (!loop && !d1) return;
    if constexpr (sizeof(V) == 8) {
        cta_tree_csum<MAXQ>(part, S.sh);
        if (threadIdx.x == 0) store_cpartials<MAXQ>(part, B.pa, B.ntiles, t);
    } else {
        // FP32 applies: plain FP64 sums, stored with lo = 0 in the same layout
        double ph[MAXQ] = {part[0].hi, part[1].hi, part[2].hi, part[3].hi};
        cta_tree_sum<MAXQ>(ph, S.sh);
        if (threadIdx.x == 0) {
            const CSum pc[MAXQ] = {{ph[0], 0.0}, {ph[1], 0.0}, {ph[2], 0.0}, {ph[3], 0.0}};
            store_cpartials<MAXQ>(pc, B.pa, B.ntiles, t);
        }
    }
}

template <typename V, int KIND>
__global__ void __launch_bounds__(ST, 2) kb_apply(BatchArgs B) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BSlabSmem<V>& S = *reinterpret_cast<BSlabSmem<V>*>(smem_raw);
    const long long t = blockIdx.x;
    if (t >= B.ntiles) return;
    const int slot = B.tile2inst[t];
    if (slot < 0) return;
    const BInst& I = B.inst[slot];
    if (!I.active) return;
    if constexpr (KIND == BK_LOOP) {
        if (fi_now(I.st, FI_P) || fi_now(I.st, FI_AP)) kb_tile<V, KIND, true>(B, S, t, I);
        else kb_tile<V, KIND, false>(B, S, t, I);
    } else {
        kb_tile<V, KIND, false>(B, S, t, I);
    }
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

// plain sums of one instance's partials whose lo parts are zero (the FP32
// inner solve's): hi of quantity q at base + q*qstride; RT strided sequential
// sums, then the block tree; valid in thread 0
template <int NQ>
__device__ __forceinline__ void inst_sums_plain(double (&v)[NQ], const double* base, long long count,
                                                long long qstride, double (*sh)[8]) {
    constexpr int FB = 8;
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    for (long long k0 = threadIdx.x; k0 < count; k0 += (long long)RT * FB) {
        double th[NQ][FB];
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int u = 0; u < FB; ++u) {
                const long long k = k0 + (long long)u * RT;
                th[q][u] = (k < count) ? __ldcg(base + q * qstride + k) : 0.0;
            }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int u = 0; u < FB; ++u)
                if (k0 + (long long)u * RT < count) v[q] = dadd(v[q], th[q][u]);
    }
    cta_tree_sum<NQ>(v, sh);
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
    if (KIND == BK_LOOP) inst_sums_plain<MAXQ>(p, B.pa + I.tile0, I.part.ntiles, B.ntiles, sh);
    else inst_sums<MAXQ>(p, B.pa + I.tile0, I.part.ntiles, B.ntiles, sh);
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
                    // products of FP32 values are exact in FP64; plain FP64 sums suffice
                    // for the inner solve's 1e-4 relative tolerance
                    part[0].hi = dfma((double)r, (double)r, part[0].hi);
                    part[1].hi = dfma((double)r, (double)zv[k], part[1].hi);
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
    // plain FP64 block tree (the inner sums carry no compensation); the
    // partials keep the (hi, lo) layout of the compensated ones, lo = 0
    double ph[2] = {part[0].hi, part[1].hi};
    cta_tree_sum<2>(ph, sh);
    if (threadIdx.x == 0 && blockIdx.x < B.nflat) {
        const CSum pc[2] = {{ph[0], 0.0}, {ph[1], 0.0}};
        store_cpartials<2>(pc, B.pf, B.nflat, blockIdx.x);
    }
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
    inst_sums_plain<2>(p, B.pf + I.flat0, I.part.nflat, B.nflat, sh);
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
