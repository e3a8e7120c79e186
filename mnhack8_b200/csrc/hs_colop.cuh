// hs_colop.cuh -- the colored operator kernel of the FP64 solver (included by
// hs_kernels.cuh after ApplyArgs).
//
// Column-march warps on the COL partition (hs_types.h).  The 32 lanes of a
// warp hold consecutive element columns, so a lane's right-hand neighbour
// column is the next lane: element outputs at the oz = 1 corners travel one
// lane up by a shuffle, and nothing goes through shared memory.  Each lane
// marches its CR node rows in y (one "step" per row) inside a march over the
// planes of its x-slab, so the element rows and planes above and below are in
// its own registers.
//
// A slab's march starts one layer early, forming its lower halo plane xa-1.
// Step i of layer x (elements between planes x and x+1):
//   1. forms p at node row r = r0-1+i of plane x+1, columns c and c+1 (the
//      PCG loop's p = z + beta p_{k-1}, or the input vector), stores p and
//      accumulates w.p and p.p at the lane's own nodes;
//   2. for the wht form, the z butterfly of that row (shared by the four
//      elements around the edge), the y butterfly with the row below (shared
//      by the two elements of the face) and, with the face of plane x kept
//      from the previous layer, the x butterfly of element (x, r-1, c); the
//      other forms gather the element's 8 corners from registers;
//   3. the element operator, then the node sum of node (x, r-1, c) in the
//      canonical order 4, 7, 6, 5 (from layer x-1, kept as a "lower" sum) and
//      0, 3, 2, 1 (this layer), projection, p.Ap / D1 partials and the store.
// The inputs of layer x+1 are copied into shared memory while layer x runs
// (asynchronous 8-byte copies, cp.async, into per-lane slots of a two-layer
// ring), so a load has a whole layer of work to arrive and costs no register
// until it is used; a lane reads only its own slots, so no barrier is needed.
//
// Elements outside the domain (the first lane of the first segment, column
// -1; the element column N of the lane owning node column N; element rows -1
// and N; layers -1 and N) are computed on zero inputs or skipped.  They only
// touch boundary nodes, whose projected output is 0 whatever their sum, so
// no mask is needed beyond keeping loads inside the arrays.
#pragma once

struct ColLane {
    int ec, r0, xa, xb;   // element column (node column owned), first node row, planes of the slab
    unsigned fl;          // bit 0 live lane, bit 1 owns node column ec, bit 2 owns the extra row N
};

// The lane's place in the COL partition: warp task wt, lane 0..31.  Lanes
// left over in a warp of packed partial segments are not live, but they run
// the march (with the task's planes) so that the warp's shuffles stay whole.
__device__ __forceinline__ ColLane col_lane(const ColLayout& L, long long wt, int lane) {
    ColLane c{-1, 0, 0, -1, 0u};
    if (wt >= L.ntasks) return c;
    const int xs = (int)(wt / L.TPS), task = (int)(wt - (long long)xs * L.TPS);
    c.xa = xs * L.CX;
    c.xb = min(c.xa + L.CX, L.NN) - 1;
    int rb, sl, base;
    if (task < L.S * L.NRB) {
        const int s = task / L.NRB;
        rb = task - s * L.NRB;
        sl = lane;
        base = CSEG * s - 1;
    } else {
        const int k = task - L.S * L.NRB, slot = lane / L.psize;
        sl = lane - slot * L.psize;
        rb = k * L.P + slot;
        base = CSEG * L.S - 1;
        if (slot >= L.P || rb >= L.NRB) return c;
    }
    c.ec = base + sl;
    c.r0 = rb * CR;
    c.fl = 1u | (sl >= 1 ? 2u : 0u) | ((L.extra && rb == L.NRB - 1) ? 4u : 0u);
    return c;
}

__device__ __forceinline__ double shfl_up1(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }

// asynchronous 8-byte global -> shared copy; valid == false reads nothing and
// writes zeros (source size 0)
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int nbytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// fields of one step in the shared-memory ring (one double per lane each)
enum ColField { CF_A0 = 0, CF_A1, CF_B0, CF_B1, CF_W, CF_CR, CF_CK, CF_N };
constexpr int kColSteps = CR + 2;
// ring: [layer parity][step][field][RT threads]
constexpr size_t kColSmem = (size_t)2 * kColSteps * CF_N * RT * sizeof(double);

// MODE 0: input x as given; 1: PCG loop, p = z; 2: PCG loop, p = z + beta p_{k-1}.
// FI false: no fault is armed for this launch (the fault tests compile out).
template <int FORM, int MODE, bool FI>
__device__ __forceinline__ void col_march(const ApplyArgs& a, const ColLane& C, double* ring, const double* srcA,
                                          const double* srcB, double beta, double* pout, bool loop, bool d1,
                                          bool rhs, int fi_p, int fi_ap, int fi_r, int fi_bit, long long fi_idx,
                                          long long fi_elem, double (&part)[MAXQ]) {
    constexpr int NS = CR + 2;                      // steps per layer
    static_assert(NS % 3 == 0, "three rotating load sets per layer");
    constexpr bool WHT = FORM == FORM_WHT;
    if (!FI) { fi_p = 0; fi_ap = 0; fi_r = 0; }
    const int N = a.cp.N, NN = a.cp.NN;
    const int ec = C.ec, r0 = C.r0, xa = C.xa, xb = C.xb;
    const bool live = C.fl & 1u;
    const bool own = (C.fl & 2u) && ec <= N;
    const bool colv = live && ec >= 0 && ec <= N;
    const bool colv1 = live && ec + 1 >= 0 && ec + 1 <= N;
    const bool ecv = live && ec >= 0 && ec < N;
    // bit i: node row r0-1+i exists / element row r0-2+i exists / node row r0-1+i owned
    unsigned rowv = 0u, erowv = 0u, orow = 0u;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        const int r = r0 - 1 + i;
        if (r >= 0 && r <= N) rowv |= 1u << i;
        if (i >= 1 && r - 1 >= 0 && r - 1 < N) erowv |= 1u << i;
        if (own && i >= 1 && i <= CR && r <= N) orow |= 1u << i;
    }
    if (own && (C.fl & 4u)) orow |= 1u << (NS - 1);   // row r0+CR == N
    const int lane_n = (r0 - 1) * NN + ec;             // node index offset of row r0-1, column c
    const int lane_e = (r0 - 2) * N + ec;              // element index offset of row r0-2, column c

    const int tid = threadIdx.x;
    // copies of layer x's inputs (plane x+1 rows, coefficients of layer x) into ring half par
    auto issue_layer = [&](int x, int par) {
        const int xp = x + 1;
        const bool plane_ok = xp >= 0 && xp <= N && xp <= xb + 1;
        const bool w_ok = d1 && xp >= xa && xp <= xb;
        const bool el_ok = x >= xa - 1 && x >= 0 && x < N && ecv;
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            double* slot = ring + ((size_t)(par * NS + i) * CF_N) * RT + tid;
            const bool pv = plane_ok && ((rowv >> i) & 1u);
            const int n = xp * NN * NN + lane_n + i * NN;
            const bool v0 = pv && colv, v1 = pv && colv1;
            cp_async8(slot + CF_A0 * RT, v0 ? srcA + n : srcA, v0);
            cp_async8(slot + CF_A1 * RT, v1 ? srcA + n + 1 : srcA, v1);
            if (MODE == 2) {
                cp_async8(slot + CF_B0 * RT, v0 ? srcB + n : srcB, v0);
                cp_async8(slot + CF_B1 * RT, v1 ? srcB + n + 1 : srcB, v1);
            }
            const bool wv = w_ok && v0 && ((orow >> i) & 1u);
            cp_async8(slot + CF_W * RT, wv ? a.w + n : a.y, wv);
            const bool ev = i >= 1 && el_ok && ((erowv >> i) & 1u);
            const double* ce = reinterpret_cast<const double*>(a.coef) + 2 * (long long)(x * N * N + lane_e + i * N);
            cp_async8(slot + CF_CR * RT, ev ? ce : srcA, ev);
            cp_async8(slot + CF_CK * RT, ev ? ce + 1 : srcA, ev);
        }
        cp_async_commit();
    };

    double fp[CR + 1][4];     // wht: y-butterflied faces of plane x, element rows r0-1+j
    double pl[NS][2];         // other forms: p of plane x at rows r0-1+i, columns c, c+1
    double slo[CR + 1];       // lower node sums of plane x at the owned rows ([CR]: extra row)
    double pk[CR + 1];        // p of plane x at the owned rows
#pragma unroll
    for (int j = 0; j <= CR; ++j) {
        slo[j] = 0.0; pk[j] = 0.0;
        fp[j][0] = fp[j][1] = fp[j][2] = fp[j][3] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < NS; ++i) pl[i][0] = pl[i][1] = 0.0;
    issue_layer(xa - 2, 0);

    // layer xa-2 only forms plane xa-1 (the slab's lower halo plane); layers
    // xa-1 .. xb apply their elements
    for (int x = xa - 2; x <= xb; ++x) {
        const bool el = x >= xa - 1 && x >= 0 && x < N;   // element layer x is applied
        const bool cpl = x >= xa;                          // plane x is the task's: complete its nodes
        const bool fown = x + 1 >= xa && x + 1 <= xb;      // plane x+1 is the task's: store p, w.p, p.p
        double zsP_s = 0.0, zsP_d = 0.0;       // z butterfly of the previous row
        double pnA = 0.0, pnB = 0.0;           // p of the previous row (plane x+1)
        double hq2 = 0.0, hL3 = 0.0, hq6 = 0.0, hL7 = 0.0;   // element row below: its oy = 1 outputs
        const int par = (x - xa) & 1;          // ring half of this layer (layer xa-2 is half 0)
        // the next layer's inputs go out now; this layer's have arrived once at most one group is pending
        if (x + 1 <= xb) issue_layer(x + 1, par ^ 1);
        else cp_async_commit();                // an empty group keeps the count
        cp_async_wait_prior1();
        const double* lring = ring + ((size_t)par * NS * CF_N) * RT + tid;
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            const double* sl = lring + (size_t)i * CF_N * RT;
            const double a0 = sl[CF_A0 * RT], a1 = sl[CF_A1 * RT];
            const double b0 = (MODE == 2) ? sl[CF_B0 * RT] : 0.0, b1 = (MODE == 2) ? sl[CF_B1 * RT] : 0.0;
            const double wv = sl[CF_W * RT], cr = sl[CF_CR * RT], ck = sl[CF_CK * RT];
            const int r = r0 - 1 + i;                   // node row formed, plane x+1
            // 1. p at (x+1, r, c) and (x+1, r, c+1)
            double pA, pB;
            if (MODE == 2) { pA = dfma(beta, b0, a0); pB = dfma(beta, b1, a1); }
            else { pA = a0; pB = a1; }
            const int nrow = (x + 1) * NN * NN + lane_n + i * NN;   // node (x+1, r, c)
            if (FI && fi_p && x + 1 <= N && ((rowv >> i) & 1u)) {
                if (colv && (long long)nrow == fi_idx) pA = flipbit(pA, fi_bit);
                if (colv1 && (long long)nrow + 1 == fi_idx) pB = flipbit(pB, fi_bit);
            }
            if (fown && ((orow >> i) & 1u)) {
                if (pout) pout[nrow] = pA;
                if (d1) {
                    part[2] = dfma(wv, pA, part[2]);
                    part[3] = dfma(pA, pA, part[3]);
                }
            }
            // 2. z butterfly of the row
            const double zs_s = dadd(pA, pB), zs_d = dsub(pA, pB);
            if (i >= 1) {
                const int j = i - 1;                    // element row er = r - 1 = r0-1+j
                double v[8];
                if (WHT) {
                    const double f0 = dadd(zsP_s, zs_s), f1 = dadd(zsP_d, zs_d);
                    const double f2 = dsub(zsP_s, zs_s), f3 = dsub(zsP_d, zs_d);
                    if (el) {
                        v[0] = dadd(fp[j][0], f0); v[1] = dadd(fp[j][1], f1);
                        v[2] = dadd(fp[j][2], f2); v[3] = dadd(fp[j][3], f3);
                        v[4] = dsub(fp[j][0], f0); v[5] = dsub(fp[j][1], f1);
                        v[6] = dsub(fp[j][2], f2); v[7] = dsub(fp[j][3], f3);
                        const double dk = dmul(a.dt_eff, ck);
                        const double l0 = dmul(cr, a.ec.cm[0]);
                        const double l1 = dfma(dk, a.ec.ck[1], dmul(cr, a.ec.cm[1]));
                        const double l2 = dfma(dk, a.ec.ck[2], dmul(cr, a.ec.cm[2]));
                        const double l3 = dfma(dk, a.ec.ck[3], dmul(cr, a.ec.cm[3]));
                        v[0] = dmul(v[0], l0);
                        v[1] = dmul(v[1], l1); v[2] = dmul(v[2], l1); v[4] = dmul(v[4], l1);
                        v[3] = dmul(v[3], l2); v[5] = dmul(v[5], l2); v[6] = dmul(v[6], l2);
                        v[7] = dmul(v[7], l3);
                        butterfly(v, 1);
                        butterfly(v, 2);
                        butterfly(v, 4);
                    }
                    fp[j][0] = f0; fp[j][1] = f1; fp[j][2] = f2; fp[j][3] = f3;
                } else {
                    if (el) {
                        v[0] = pl[j][0]; v[1] = pl[j][1]; v[2] = pl[j + 1][0]; v[3] = pl[j + 1][1];
                        v[4] = pnA; v[5] = pnB; v[6] = pA; v[7] = pB;
                        elem_apply<FORM>(v, cr, ck, a.dt_eff, a.ec);
                    }
                    pl[j][0] = pnA; pl[j][1] = pnB;     // row r-1 of plane x+1 replaces that of plane x
                }
                if (!el) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) v[q] = 0.0;
                }
                if (FI && fi_r && el && ecv && ((erowv >> i) & 1u) &&
                    (long long)(x * N * N + lane_e + i * N) == fi_elem)
                    v[0] = flipbit(v[0], fi_bit);
                // oz = 1 outputs of the left neighbour's element (same row)
                const double L1 = shfl_up1(v[1]), L3 = shfl_up1(v[3]), L5 = shfl_up1(v[5]), L7 = shfl_up1(v[7]);
                // 3. node row r-1: complete plane x, lower sum of plane x+1
                if (j >= 1) {
                    const int oj = j - 1;               // owned row r0+oj == r-1
                    if (cpl && ((orow >> j) & 1u)) {
                        const int er = r - 1;
                        const int n = x * NN * NN + lane_n + j * NN;
                        const bool bnd = x == 0 || x == N || er == 0 || er == N || ec == 0 || ec == N;
                        double y = bnd ? 0.0 : dadd(dadd(dadd(dadd(slo[oj], v[0]), hL3), hq2), L1);
                        if (FI && fi_ap && (long long)n == fi_idx) y = flipbit(y, fi_bit);
                        const double pv = pk[oj];
                        if (loop) part[0] = dfma(pv, y, part[0]);
                        if (d1) part[1] = bnd ? dfma(0.0, y, part[1]) : dadd(part[1], y);
                        if (MODE == 0 && rhs) y = dfma(a.dtF, __ldg(a.F + n), y);
                        a.y[n] = y;
                    }
                    slo[oj] = dadd(dadd(dadd(dadd(0.0, v[4]), hL7), hq6), L5);
                    pk[oj] = pnA;                       // p of plane x+1 at row r-1
                }
                hq2 = v[2]; hL3 = L3; hq6 = v[6]; hL7 = L7;
            }
            zsP_s = zs_s; zsP_d = zs_d;
            pnA = pA; pnB = pB;
        }
        if (!WHT) { pl[NS - 1][0] = pnA; pl[NS - 1][1] = pnB; }
        // the extra row N (a boundary row: projected output 0)
        if (C.fl & 4u) {
            if (cpl && own) {
                const int n = (x * NN + N) * NN + ec;
                double y = 0.0;
                if (FI && fi_ap && (long long)n == fi_idx) y = flipbit(y, fi_bit);
                if (loop) part[0] = dfma(pk[CR], y, part[0]);
                if (d1) part[1] = dfma(0.0, y, part[1]);
                if (MODE == 0 && rhs) y = dfma(a.dtF, __ldg(a.F + n), y);
                a.y[n] = y;
            }
            pk[CR] = pnA;
        }
    }
}

// Colored operator on the COL partition: tile blockIdx.x (CW warp tasks).
// LOOP: the PCG-loop role (p formed in the kernel); otherwise the roles that
// apply the operator to a given vector.  One tile per SM (the 172 KB ring).
template <int FORM, bool LOOP>
__global__ void __launch_bounds__(RT, 1) k_apply_col(ApplyArgs a) {
    __shared__ double sh[MAXQ][8];
    extern __shared__ __align__(16) double col_ring[];     // kColSmem bytes
    DevState* st = a.st;
    int fi_p = 0, fi_ap = 0, fi_r = 0, fi_bit = 0;
    long long fi_idx = -1, fi_elem = -1;
    const bool d1 = a.d1 != 0;
    double part[MAXQ] = {0.0, 0.0, 0.0, 0.0};
    const long long wt = (long long)blockIdx.x * CW + (threadIdx.x >> 5);
    const bool wlive = wt < a.cp.ntasks;            // warp-uniform
    const ColLane C = col_lane(a.cp, wt, threadIdx.x & 31);
    if (LOOP) {
        if (st->done) return;
        const int iter = st->iter;
        const double beta = st->beta;
        const double* src_b = (iter > 0) ? ((iter & 1) ? a.pbuf0 : a.pbuf1) : nullptr;
        double* pout = (iter & 1) ? a.pbuf1 : a.pbuf0;
        if (st->fi_vec && st->fi_iter == iter) {
            fi_idx = st->fi_idx; fi_bit = st->fi_bit;
            fi_p = (st->fi_vec == FI_P); fi_ap = (st->fi_vec == FI_AP);
        }
        if (wlive) {
            if (!src_b)
                col_march<FORM, 1, true>(a, C, col_ring, a.z, nullptr, 0.0, pout, true, d1, false, fi_p, fi_ap, 0, fi_bit,
                                         fi_idx, -1, part);
            else if (fi_p || fi_ap)
                col_march<FORM, 2, true>(a, C, col_ring, a.z, src_b, beta, pout, true, d1, false, fi_p, fi_ap, 0, fi_bit,
                                         fi_idx, -1, part);
            else
                col_march<FORM, 2, false>(a, C, col_ring, a.z, src_b, beta, pout, true, d1, false, 0, 0, 0, 0, -1, -1, part);
        }
    } else {
        if (a.role == ROLE_X0 && st->fi_armR) { fi_r = 1; fi_elem = st->fi_elem; fi_bit = st->fi_bit; }
        const bool rhs = (a.role == ROLE_RHS) && a.F != nullptr;
        if (wlive) {
            if (fi_r)
                col_march<FORM, 0, true>(a, C, col_ring, a.x, nullptr, 0.0, nullptr, false, d1, rhs, 0, 0, 1, fi_bit, -1,
                                         fi_elem, part);
            else
                col_march<FORM, 0, false>(a, C, col_ring, a.x, nullptr, 0.0, nullptr, false, d1, rhs, 0, 0, 0, 0, -1, -1,
                                          part);
        }
        if (!d1) return;
    }
    store_partials<MAXQ>(part, a.partials, a.cp.ntiles, sh);
}
