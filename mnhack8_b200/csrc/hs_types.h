// hs_types.h -- types shared by the host driver and the kernels of libheat_b200.
#pragma once
#include <cstdint>

namespace hs {

// ---- canonical partitions and reduction orders ------------------------------
// APPLY partition (operator kernels): interior nodes [1, N-1]^3 are covered by
// tiles of TY rows x TZ columns streaming cx(N) planes in x, one node column
// per reduction thread; boundary nodes (any coordinate 0 or N), enumerated in
// increasing node index, by blocks of RT*BPT nodes, thread t taking nodes
// b*RT*BPT + k*RT + t for k = 0..BPT-1.  The p.Ap and ABFT partials follow it.
// FLAT partition (every other reduction and the PCG vector update): blocks of
// RT*KF consecutive nodes, thread t of block b taking the KF consecutive nodes
// b*RT*KF + t*KF + k.
// In both, a thread accumulates its nodes in order, a block combines its RT
// values by a 32-lane xor butterfly per warp and an 8-way xor butterfly over
// the warp sums, and the last block to finish combines the per-block partials
// (apply: tiles first, then boundary blocks) by RT strided sequential sums and
// the same block tree.  Every result is a fixed function of the inputs,
// independent of scheduling.
constexpr int TY = 8;
constexpr int TZ = 32;
constexpr int RT = 256;
constexpr int BPT = 8;
constexpr int KF = 2;
constexpr int APPLY_SLOTS = 592;   // co-resident operator tiles assumed by cx(N): 148 SMs x 4

// planes per apply tile: the cx in [8, 64] minimising (waves x (cx + 1) element
// planes) for APPLY_SLOTS co-resident tiles
inline int apply_cx(int N) {
    const long long I = N - 1;
    if (I <= 0) return 16;
    const long long col = ((I + TY - 1) / TY) * ((I + TZ - 1) / TZ);
    int best = 16;
    long long best_cost = -1;
    for (int cx = 8; cx <= 64; ++cx) {
        const long long chunks = (I + cx - 1) / cx;
        const long long blocks = col * chunks;
        const long long waves = (blocks + APPLY_SLOTS - 1) / APPLY_SLOTS;
        const long long cost = waves * ((cx < I ? cx : I) + 1);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = cx; }
    }
    return best;
}
constexpr int EY = TY + 1;            // element rows touched by a tile
constexpr int EZ = TZ + 1;            // element columns touched by a tile
constexpr int LY = TY + 2;            // node rows loaded per plane (with halo)
constexpr int LZ = TZ + 2;            // node columns loaded per plane
constexpr int NLOAD = LY * LZ;        // 340 node values per plane
constexpr int NELEM = EY * EZ;        // 297 elements per plane
static_assert(TY * TZ == RT, "one node column per thread");
static_assert(NLOAD <= 2 * RT && NELEM <= 2 * RT, "two slots per thread");

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
    // scratch outputs of standalone reductions
    double red_out[MAXQ];
    double mm_out[2];       // min, max
};

}  // namespace hs
