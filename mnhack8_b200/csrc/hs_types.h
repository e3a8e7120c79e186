// hs_types.h -- types shared by the host driver and the kernels of libheat_b200.
#pragma once
#include <cstdint>

namespace hs {

// ---- canonical partitions and reduction orders ------------------------------
// SLAB partition (operator kernels and the p.Ap / ABFT partials): the node grid
// is cut into tiles of CX planes (x) x R rows (y) x C columns (z) (the last
// tile of each direction may be short).  Tile t = (tx * NRB + rb) * NCB + cb
// covers planes [tx*CX, ..), rows [rb*R, ..), columns [cb*C, ..).  Its CTA
// holds the tile's rows and columns plus a one-node halo on each side as
// Rw = R+2 rows of Cw = C+2 positions, position j = lr*Cw + lc <-> node row
// rb*R - 1 + lr, column cb*C - 1 + lc; thread t owns positions t + k*ST,
// k = 0..SK-1.  A thread accumulates the tile nodes among its positions, plane
// by plane in increasing x, positions in increasing k.
// FLAT partition (the other reductions and the PCG vector update): blocks of
// RT*KF consecutive nodes, thread t of block b taking the KF consecutive nodes
// b*RT*KF + t*KF + k.
// RUN order (the PCG vector update's b.b, r.z and r.r): the FLAT blocks are
// dealt to G = min(blocks, UPD_SLOTS) runs, run c taking blocks c, c+G, ...;
// thread t of a run accumulates its KF nodes of each of the run's blocks,
// block after block, in one sum; the run's RT sums go through the block tree
// and the G run sums are then combined like per-block partials.
// In all, a block combines its RT values by a 32-lane xor butterfly per warp
// and an 8-way xor butterfly over the warp sums, and a final pass combines the
// per-block partials by RT strided sequential sums and the same block tree.
// Every result is a fixed function of the inputs, independent of scheduling.
//
// Node sums (operator output at a node): starting from +0.0, the contributions
// of the elements around the node are added in the order of their local
// corner q = ox<<2 | oy<<1 | oz at which the node sits: 4, 7, 6, 5, 0, 3, 2, 1
// (the lower x layer first, each layer's own-column element first), skipping
// elements outside the domain.
constexpr int RT = 256;
constexpr int KF = 2;                 // nodes per thread of the flat partition
constexpr int ST = RT;                // threads per slab CTA
constexpr int SK = 4;                 // positions per thread
constexpr int SPOS = ST * SK;         // positions per plane of a slab CTA (halo included)
constexpr int SLAB_SLOTS = 296;       // co-resident slab CTAs assumed by the layout: 148 SMs x 2
constexpr int UPD_SLOTS = 740;        // runs of the RUN order: co-resident update CTAs, 148 SMs x 5

struct SlabLayout {
    int C, R, CX;          // tile columns, rows, planes
    int NCB, NRB, NXB;     // tiles per direction
    long long ntiles;
};

// The tile shape of an N-element grid: among C >= min(N+1, 30) with
// (R+2)(C+2) <= SPOS (R as large as that allows) and CX from the first waves
// of SLAB_SLOTS tiles, the one minimising waves x (CX+2) x
// ((R+2)(C+2) + 2(R+1)(C+1)) (planes streamed x positions loaded plus twice
// the elements applied per plane); ties keep the smaller C, then fewer waves.
inline SlabLayout slab_layout(int N) {
    const long long NN = N + 1;
    SlabLayout best{};
    long long best_cost = -1;
    const long long cmin = NN < 30 ? NN : 30;
    for (long long C = cmin; C <= NN; ++C) {
        const long long Cw = C + 2;
        const long long Rmax = SPOS / Cw - 2;
        if (Rmax < 1) break;
        const long long R = Rmax < NN ? Rmax : NN;
        const long long NCB = (NN + C - 1) / C, NRB = (NN + R - 1) / R, tyz = NCB * NRB;
        const long long work = Cw * (R + 2) + 2 * (C + 1) * (R + 1);
        const long long w0 = (tyz + SLAB_SLOTS - 1) / SLAB_SLOTS;
        for (long long w = w0; w < w0 + 4; ++w) {
            long long nx = w * SLAB_SLOTS / tyz;
            if (nx < 1) continue;
            if (nx > NN) nx = NN;
            const long long CX = (NN + nx - 1) / nx;
            const long long NXB = (NN + CX - 1) / CX;
            const long long waves = (tyz * NXB + SLAB_SLOTS - 1) / SLAB_SLOTS;
            const long long cost = waves * (CX + 2) * work;
            if (best_cost < 0 || cost < best_cost) {
                best_cost = cost;
                best.C = (int)C; best.R = (int)R; best.CX = (int)CX;
                best.NCB = (int)NCB; best.NRB = (int)NRB; best.NXB = (int)NXB;
                best.ntiles = tyz * NXB;
            }
        }
    }
    return best;
}

constexpr int MAXQ = 4;               // reduced quantities per pass

enum Form { FORM_FAST = 0, FORM_GAUSS = 1, FORM_WHT = 2 };

// roles of an operator application
enum Role {
    ROLE_RHS = 0,    // b = M T (+ dt F): D1 against w_M
    ROLE_X0 = 1,     // Ap = A x0, first matvec of PCG: D1 against w_A, level-R fault
    ROLE_LOOP = 2,   // p = z + beta p, Ap = A p: p.Ap, D1, vector faults
    ROLE_PLAIN = 3,  // y = A x, projected, no checksum (D2 matvec, user calls)
    ROLE_USER = 4    // y = A x, projected, D1 against w (user call with detect)
};

enum UpdRole { UPD_PRE = 0, UPD_LOOP = 1 };

enum FiLevel { FI_NONE = 0, FI_G = 1, FI_R = 2, FI_H = 3, FI_P = 5, FI_RV = 6, FI_AP = 7 };

// device-resident solver scalars (one per handle)
struct DevState {
    // PCG
    double rho, alpha, beta, bnorm, pAp, rel0, tol;
    int iter, done, broken, result, max_iter, pad0;
    // ABFT D1
    double norm_wM, norm_wA, d1_step, d1_last;
    // fault injection armed for the current step
    int fi_armR;            // level R armed (fires in the ROLE_X0 apply)
    int fi_vec;             // 5/6/7 armed
    int fi_iter, fi_bit;
    long long fi_elem;      // level R element
    long long fi_idx;       // vector entry
    // per-iteration log (diag-cg), may be null
    double* log_rel;
    double* log_alpha;
    double* log_beta;
    int log_cap, pad1;
    // the solution update x += alpha_k p_k runs every second CG iteration: at
    // an odd k for k-1 and k (alpha_hist[k & 1] holds alpha_k); x_pend marks a
    // last update (at x_pend_iter) still owed when the loop ends
    double alpha_hist[2];
    int x_pend, x_pend_iter;
    // scratch outputs of standalone reductions
    double red_out[MAXQ];
    double mm_out[2];       // min, max
};

}  // namespace hs
