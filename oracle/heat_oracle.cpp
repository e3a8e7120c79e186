// =============================================================================
// heat_oracle.cpp -- CPU restatement of the reference transient-heat hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity oracle for the B200
// library in mnhack8_b200/csrc. Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load it; the library never links,
// calls or falls back to it.
//
// It restates, in plain C++ (+OpenMP for the element loops), the single-rank
// semantics of the reference solver src/heat_solver_het.cu:
//   * grid / indexing / boundary             het.cu:155-167, 202-227
//   * reference matrices + closed-form check het.cu:661-708 (exit code 2)
//   * element apply `fast` (dense 8x8)       het.cu:340-349
//   * element apply `gauss`                  het.cu:242-257, 310-338
//   * operator: zero, element loop, [R flip], scatter, projection, ABFT D1
//                                            het.cu:352-378, 885-921
//   * Jacobi diagonal, source vector         het.cu:229-237, 381-422, 798-814
//   * build_rhs, PCG                         het.cu:963-971, 994-1039
//   * detectors D1/D2/D3, run_case, FI G/R   het.cu:940-953, 1107-1259
//   * --verify eigenmode, Gaussian IC        het.cu:556-584, 1293-1338
// plus the additions of the B200 library that have no reference counterpart:
//   * the `wht` element form: the same element matrix written through the
//     exact tensor-product structure of the Q1 cube element (Walsh-Hadamard
//     eigen-decomposition, 63 flops instead of 192);
//   * single-bit flips into the PCG vectors p, r, Ap at (step, iteration);
//   * user-set CG tolerance and Gaussian-IC width.
//
// Arithmetic is spelled out operation by operation (std::fma where the
// library uses __fma_rn; the file is compiled with -ffp-contract=off) and the
// node summation order and the reduction order follow the library's canonical
// definitions (below), so the library's deterministic ("colored") path must
// reproduce every value of this file bit for bit.
// =============================================================================
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- canonical reduction partitions (mirror the library's) --------------------
// Two fixed orders.  The APPLY order (the operator kernel's p.Ap and ABFT
// partials) follows the operator's slab tiles, described below.  The FLAT
// order (every other reduction: D2, E(t), plain dots)
// cuts the node index range into blocks of RT*KF consecutive nodes, thread t
// of block b accumulating the KF consecutive nodes b*RT*KF + t*KF + k,
// k = 0..KF-1, in order; blocks are combined like the apply order's partials.
//
// Slab tiles: the node grid is cut into tiles of CX planes (x) x R rows (y) x
// C columns (z), the last tile of each direction possibly short; tile
// t = (tx*NRB + rb)*NCB + cb starts at plane tx*CX, row rb*R, column cb*C.  A
// tile's RT threads own the positions j = l + k*RT (k = 0..SK-1) of a plane of
// (R+2) x (C+2) positions (one halo row / column on each side), position j at
// row rb*R - 1 + j/(C+2), column cb*C - 1 + j%(C+2); thread l accumulates the
// tile's own nodes among its positions, plane by plane in increasing x and
// positions in increasing k.  A block's RT values are combined by a 32-lane xor
// butterfly per warp then an 8-way xor butterfly over warps; the tile
// partials are combined by RT strided sequential sums followed by the same
// block tree.  (C, R, CX) is a fixed function of N, slab_layout below.
// The PCG vector update's dots (b.b, r.z, r.r) take the RUN order: the flat
// blocks' partials first summed in runs of consecutive blocks (ureduce).
const int RT = 256;
const int SK = 4;                 // positions per thread
const int SPOS = RT * SK;         // positions per tile plane, halo included
const int SLAB_SLOTS = 296;       // co-resident tiles the layout assumes
int g_KF = 2;                     // flat layout: consecutive nodes per thread
const long UPD_SLOTS = 740;       // runs of the update order: co-resident update CTAs (148 SMs x 5)

struct SlabLayout { int C, R, CX, NCB, NRB, NXB; long ntiles; };

// The library's tile shape: among C >= min(N+1, 30) with (R+2)(C+2) <= SPOS
// (R as large as that allows) and CX from the first waves of SLAB_SLOTS tiles,
// the one minimising waves x (CX+2) x ((R+2)(C+2) + 2(R+1)(C+1)); ties keep the
// smaller C, then fewer waves.
SlabLayout slab_layout(int N) {
    const long NN = N + 1;
    SlabLayout best{};
    long best_cost = -1;
    const long cmin = NN < 30 ? NN : 30;
    for (long C = cmin; C <= NN; ++C) {
        const long Cw = C + 2;
        const long Rmax = SPOS / Cw - 2;
        if (Rmax < 1) break;
        const long R = Rmax < NN ? Rmax : NN;
        const long NCB = (NN + C - 1) / C, NRB = (NN + R - 1) / R, tyz = NCB * NRB;
        const long work = Cw * (R + 2) + 2 * (C + 1) * (R + 1);
        const long w0 = (tyz + SLAB_SLOTS - 1) / SLAB_SLOTS;
        for (long w = w0; w < w0 + 4; ++w) {
            long nx = w * SLAB_SLOTS / tyz;
            if (nx < 1) continue;
            if (nx > NN) nx = NN;
            const long CX = (NN + nx - 1) / nx;
            const long NXB = (NN + CX - 1) / CX;
            const long waves = (tyz * NXB + SLAB_SLOTS - 1) / SLAB_SLOTS;
            const long cost = waves * (CX + 2) * work;
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
SlabLayout g_slab_override{};     // or_set_layout: a fixed tile shape (C > 0) instead of slab_layout(N)

inline double tree256(const double* v) {
    double ws[8];
    for (int w = 0; w < 8; ++w) {
        double a[32];
        for (int l = 0; l < 32; ++l) a[l] = v[w * 32 + l];
        for (int off = 16; off >= 1; off >>= 1) {
            double b[32];
            for (int l = 0; l < 32; ++l) b[l] = a[l] + a[l ^ off];
            std::memcpy(a, b, sizeof(a));
        }
        ws[w] = a[0];
    }
    for (int off = 4; off >= 1; off >>= 1) {
        double b[8];
        for (int l = 0; l < 8; ++l) b[l] = ws[l] + ws[l ^ off];
        std::memcpy(ws, b, sizeof(ws));
    }
    return ws[0];
}

inline uint64_t d2u(double x) { uint64_t u; std::memcpy(&u, &x, 8); return u; }
inline double u2d(uint64_t u) { double x; std::memcpy(&x, &u, 8); return x; }
inline double flip(double x, int bit) { return u2d(d2u(x) ^ (1ULL << bit)); }

// local node i of an element sits at offsets off[i] (het.cu:261-264)
const int OFF[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
// q-index (ox<<2 | oy<<1 | oz) of local node i, and back
const int Q_OF_LOCAL[8] = {0, 4, 6, 2, 1, 5, 7, 3};
const int LOCAL_OF_Q[8] = {0, 4, 3, 7, 1, 5, 2, 6};

// het.cu:242-257
void shape_func_grad(double xi, double eta, double zeta, double N[8], double dN[8][3]) {
    const int sgn[8][3] = {{-1,-1,-1},{1,-1,-1},{1,1,-1},{-1,1,-1},
                           {-1,-1,1},{1,-1,1},{1,1,1},{-1,1,1}};
    for (int i = 0; i < 8; ++i) {
        double sx = sgn[i][0], sy = sgn[i][1], sz = sgn[i][2];
        double a = 1 + sx * xi, b = 1 + sy * eta, c = 1 + sz * zeta;
        N[i] = 0.125 * a * b * c;
        dN[i][0] = 0.125 * sx * b * c;
        dN[i][1] = 0.125 * a * sy * c;
        dN[i][2] = 0.125 * a * b * sz;
    }
}

enum { FORM_DENSE = 0, FORM_GAUSS = 1, FORM_WHT = 2 };
enum { LV_NONE = 0, LV_G = 1, LV_R = 2, LV_H = 3, LV_P = 5, LV_RV = 6, LV_AP = 7 };

struct FI {
    int level = 0, step = -1, bit = 0, iter = 0;
    long target = 0;
};

struct Oracle {
    int N = 0, NN = 0;
    long Nn = 0, Ne = 0;
    double h = 0, dt = 0;
    int form = FORM_WHT, colored = 1, detect = 0, verify = 0, no_source = 0, ic_mode = 0;
    double ic_sigma = 0.1, src_sigma = 0.1;
    double kmin = 0, kmax = 0, rhocmin = 0, rhocmax = 0;
    std::vector<double> k, rhoc;
    double M[64], K[64];
    double detJ = 0, invJ = 0;
    double gN[8][8], gdx[8][8], gdy[8][8], gdz[8][8];   // Gauss tables [point][node]
    double cm[4], ck[4];                                  // wht eigen-constants / 8
    std::vector<double> diag, F, wM, wA;
    double norm_wM = 0, norm_wA = 0;
    double abft_step_max = 0;
    long abft_calls = 0;
    // FI state for the current step
    int armed_R = 0;       // level R armed (first matvec of the step)
    int vec_level = 0;     // 5/6/7 armed this step
    int vec_iter = 0;
    long vec_idx = 0;
    int fi_bit = 0;
    long fi_target_elem = -1;
    int matrix_ok = 1;
    double mat_err[5] = {0, 0, 0, 0, 0};
    std::vector<double> ye_buf;   // Ne*8, element outputs in q-order

    long nid(int ix, int iy, int iz) const { return ((long)ix * NN + iy) * NN + iz; }
    bool is_bnd(int ix, int iy, int iz) const {
        return ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N;
    }
    bool is_bnd_n(long n) const {
        int ix = (int)(n / ((long)NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
        return is_bnd(ix, iy, iz);
    }

    // ---- het.cu:661-708 ------------------------------------------------------
    void build_reference_matrices() {
        double Mh[64] = {0}, Kh[64] = {0};
        const double hx = h, hy = h, hz = h;
        const double dJ = hx * hy * hz / 8.0;
        const double iJ[3] = {2.0 / hx, 2.0 / hy, 2.0 / hz};
        const double gp = 1.0 / 1.7320508075688772;
        const double pts[2] = {-gp, gp};
        for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) for (int c = 0; c < 2; ++c) {
            double Nv[8], dN[8][3];
            shape_func_grad(pts[a], pts[b], pts[c], Nv, dN);
            for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) {
                Mh[i * 8 + j] += dJ * Nv[i] * Nv[j];
                Kh[i * 8 + j] += dJ * (iJ[0] * dN[i][0] * iJ[0] * dN[j][0]
                                     + iJ[1] * dN[i][1] * iJ[1] * dN[j][1]
                                     + iJ[2] * dN[i][2] * iJ[2] * dN[j][2]);
            }
        }
        const int sgn[8][3] = {{-1,-1,-1},{1,-1,-1},{1,1,-1},{-1,1,-1},
                               {-1,-1,1},{1,-1,1},{1,1,1},{-1,1,1}};
        const double V = hx * hy * hz;
        double errM = 0, sumM = 0, errKrow = 0, errKdiag = 0, errSym = 0;
        const double Kdiag = (hy * hz / hx + hx * hz / hy + hx * hy / hz) / 9.0;
        for (int i = 0; i < 8; ++i) {
            double rs = 0;
            for (int j = 0; j < 8; ++j) {
                int d = (sgn[i][0] != sgn[j][0]) + (sgn[i][1] != sgn[j][1]) + (sgn[i][2] != sgn[j][2]);
                double Mref = V / 216.0 * (double)(8 >> d);
                errM = std::fmax(errM, std::fabs(Mh[i * 8 + j] - Mref) / (V / 216.0 * 8));
                sumM += Mh[i * 8 + j];
                rs += Kh[i * 8 + j];
                errSym = std::fmax(errSym, std::fabs(Kh[i * 8 + j] - Kh[j * 8 + i]) + std::fabs(Mh[i * 8 + j] - Mh[j * 8 + i]));
            }
            errKrow = std::fmax(errKrow, std::fabs(rs) / Kdiag);
            errKdiag = std::fmax(errKdiag, std::fabs(Kh[i * 9] - Kdiag) / Kdiag);
        }
        double errSum = std::fabs(sumM - V) / V;
        matrix_ok = (errM < 1e-12 && errSum < 1e-12 && errKrow < 1e-12 && errKdiag < 1e-12 && errSym < 1e-12 * Kdiag);
        mat_err[0] = errM; mat_err[1] = errSum; mat_err[2] = errKrow; mat_err[3] = errKdiag; mat_err[4] = errSym;
        std::memcpy(M, Mh, sizeof(M));
        std::memcpy(K, Kh, sizeof(K));

        // Gauss tables for the `gauss` form (het.cu:313-328), point g = gi*4+gj*2+gk
        detJ = hx * hy * hz / 8.0;
        invJ = 2.0 / hx;
        for (int gi = 0; gi < 2; ++gi) for (int gj = 0; gj < 2; ++gj) for (int gk = 0; gk < 2; ++gk) {
            int g = gi * 4 + gj * 2 + gk;
            double Nv[8], dN[8][3];
            shape_func_grad(pts[gi], pts[gj], pts[gk], Nv, dN);
            for (int i = 0; i < 8; ++i) {
                gN[g][i] = Nv[i];
                gdx[g][i] = invJ * dN[i][0];
                gdy[g][i] = invJ * dN[i][1];
                gdz[g][i] = invJ * dN[i][2];
            }
        }
        // wht eigen-constants (tensor structure of the cube element, /8 folded)
        const double hs = h / 6.0, hb = h / 2.0, g2 = 2.0 / h;
        double mu[4] = {hb * hb * hb, hs * hb * hb, hs * hs * hb, hs * hs * hs};
        double ka[4] = {0.0, g2 * hb * hb, 2.0 * (g2 * hs * hb), 3.0 * (g2 * hs * hs)};
        for (int j = 0; j < 4; ++j) { cm[j] = mu[j] / 8.0; ck[j] = ka[j] / 8.0; }
    }

    // ---- element operator: xq, yq in q-order -------------------------------
    void elem_apply(long e, const double xq[8], double yq[8], double dt_eff) const {
        const double ke = k[e], re = rhoc[e];
        if (form == FORM_WHT) {
            double v[8];
            for (int q = 0; q < 8; ++q) v[q] = xq[q];
            for (int bit = 1; bit <= 4; bit <<= 1)
                for (int q = 0; q < 8; ++q) if (!(q & bit)) {
                    double u = v[q], w = v[q | bit];
                    v[q] = u + w; v[q | bit] = u - w;
                }
            const double dk = dt_eff * ke;
            double lam[4];
            lam[0] = re * cm[0];
            for (int j = 1; j < 4; ++j) lam[j] = std::fma(dk, ck[j], re * cm[j]);
            for (int q = 0; q < 8; ++q) v[q] = v[q] * lam[__builtin_popcount(q)];
            for (int bit = 1; bit <= 4; bit <<= 1)
                for (int q = 0; q < 8; ++q) if (!(q & bit)) {
                    double u = v[q], w = v[q | bit];
                    v[q] = u + w; v[q | bit] = u - w;
                }
            for (int q = 0; q < 8; ++q) yq[q] = v[q];
        } else if (form == FORM_DENSE) {
            double xl[8], yl[8];
            for (int i = 0; i < 8; ++i) xl[i] = xq[Q_OF_LOCAL[i]];
            const double dk = dt_eff * ke;
            for (int i = 0; i < 8; ++i) {
                double acc = 0.0;
                for (int j = 0; j < 8; ++j) {
                    double a = std::fma(re, M[i * 8 + j], dk * K[i * 8 + j]);
                    acc = std::fma(a, xl[j], acc);
                }
                yl[i] = acc;
            }
            for (int i = 0; i < 8; ++i) yq[Q_OF_LOCAL[i]] = yl[i];
        } else {  // gauss, het.cu:310-338
            double xl[8], yl[8];
            for (int i = 0; i < 8; ++i) { xl[i] = xq[Q_OF_LOCAL[i]]; yl[i] = 0.0; }
            for (int g = 0; g < 8; ++g) {
                for (int i = 0; i < 8; ++i) {
                    double Mx = 0.0, Kx = 0.0;
                    for (int j = 0; j < 8; ++j) {
                        double tm = (re * gN[g][i]) * gN[g][j];
                        Mx = std::fma(tm, xl[j], Mx);
                        double gg = std::fma(gdz[g][i], gdz[g][j], std::fma(gdy[g][i], gdy[g][j], gdx[g][i] * gdx[g][j]));
                        Kx = std::fma(ke * gg, xl[j], Kx);
                    }
                    yl[i] = std::fma(detJ, std::fma(dt_eff, Kx, Mx), yl[i]);
                }
            }
            for (int i = 0; i < 8; ++i) yq[Q_OF_LOCAL[i]] = yl[i];
        }
    }

    // all element outputs into ye_buf (q-order), with the level-R flip
    void compute_elements(const double* x, double dt_eff, bool fire_R) {
        ye_buf.resize((size_t)Ne * 8);
        #pragma omp parallel for schedule(static)
        for (long e = 0; e < Ne; ++e) {
            int ex = (int)(e / ((long)N * N)), ey = (int)((e / N) % N), ez = (int)(e % N);
            double xq[8];
            for (int q = 0; q < 8; ++q)
                xq[q] = x[nid(ex + ((q >> 2) & 1), ey + ((q >> 1) & 1), ez + (q & 1))];
            double* yq = &ye_buf[(size_t)e * 8];
            elem_apply(e, xq, yq, dt_eff);
            if (fire_R && e == fi_target_elem) yq[0] = flip(yq[0], fi_bit);
        }
    }

    // canonical node sum: from +0.0, the contribution of the element at whose
    // corner q the node sits, for q = 4, 7, 6, 5, 0, 3, 2, 1 (lower x layer
    // first, each layer's own-column element first), elements in the domain
    void gather_nodes(double* y) const {
        static const int order[8] = {4, 7, 6, 5, 0, 3, 2, 1};
        #pragma omp parallel for schedule(static)
        for (long n = 0; n < Nn; ++n) {
            int ix = (int)(n / ((long)NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
            double acc = 0.0;
            for (int s = 0; s < 8; ++s) {
                const int q = order[s];
                int ex = ix - ((q >> 2) & 1), ey = iy - ((q >> 1) & 1), ez = iz - (q & 1);
                if (ex < 0 || ey < 0 || ez < 0 || ex >= N || ey >= N || ez >= N) continue;
                acc = acc + ye_buf[((size_t)(((long)ex * N + ey) * N + ez)) * 8 + q];
            }
            y[n] = acc;
        }
    }

    // sequential element-order scatter (one admissible order of atomic mode)
    void scatter_atomic(double* y) const {
        for (long n = 0; n < Nn; ++n) y[n] = 0.0;
        for (long e = 0; e < Ne; ++e) {
            int ex = (int)(e / ((long)N * N)), ey = (int)((e / N) % N), ez = (int)(e % N);
            for (int i = 0; i < 8; ++i) {
                long g = nid(ex + OFF[i][0], ey + OFF[i][1], ez + OFF[i][2]);
                y[g] = y[g] + ye_buf[(size_t)e * 8 + Q_OF_LOCAL[i]];
            }
        }
    }

    // ---- canonical reduction ---------------------------------------------------
    template <class Term>
    double creduce(Term term) const {
        SlabLayout L = slab_layout(N);
        if (g_slab_override.C > 0) {
            L = g_slab_override;
            L.NCB = (NN + L.C - 1) / L.C; L.NRB = (NN + L.R - 1) / L.R; L.NXB = (NN + L.CX - 1) / L.CX;
            L.ntiles = (long)L.NCB * L.NRB * L.NXB;
        }
        const int Cw = L.C + 2, Rw = L.R + 2;
        std::vector<double> P(L.ntiles);
        #pragma omp parallel for schedule(static)
        for (long t = 0; t < L.ntiles; ++t) {
            const int cb = (int)(t % L.NCB), rb = (int)((t / L.NCB) % L.NRB), tx = (int)(t / ((long)L.NCB * L.NRB));
            const int y0 = rb * L.R, z0 = cb * L.C, xa = tx * L.CX, xb = std::min(xa + L.CX, NN) - 1;
            double v[RT];
            for (int l = 0; l < RT; ++l) {
                double acc = 0.0;
                for (int ix = xa; ix <= xb; ++ix)
                    for (int k = 0; k < SK; ++k) {
                        const int j = l + k * RT;
                        if (j >= Rw * Cw) continue;
                        const int lr = j / Cw, lc = j % Cw;
                        const int iy = y0 - 1 + lr, iz = z0 - 1 + lc;
                        if (lr < 1 || lr > L.R || lc < 1 || lc > L.C || iy > N || iz > N) continue;
                        acc = term(nid(ix, iy, iz), acc);
                    }
                v[l] = acc;
            }
            P[t] = tree256(v);
        }
        double v[RT];
        for (int l = 0; l < RT; ++l) {
            double acc = 0.0;
            for (size_t q = l; q < P.size(); q += RT) acc = acc + P[q];
            v[l] = acc;
        }
        return tree256(v);
    }
    // flat blocks' partials (one per block of RT*KF consecutive nodes)
    template <class Term>
    std::vector<double> fblocks(Term term) const {
        const long RB = (long)RT * g_KF;
        const long nb = (Nn + RB - 1) / RB;
        std::vector<double> P(nb);
        #pragma omp parallel for schedule(static)
        for (long b = 0; b < nb; ++b) {
            double v[RT];
            for (int l = 0; l < RT; ++l) {
                double acc = 0.0;
                for (int k = 0; k < g_KF; ++k) {
                    const long n = b * RB + (long)l * g_KF + k;
                    if (n >= Nn) break;
                    acc = term(n, acc);
                }
                v[l] = acc;
            }
            P[b] = tree256(v);
        }
        return P;
    }
    // partials combined: RT strided sequential sums, then the block tree
    static double combine(const std::vector<double>& P) {
        double v[RT];
        for (int l = 0; l < RT; ++l) {
            double acc = 0.0;
            for (size_t q = l; q < P.size(); q += RT) acc = acc + P[q];
            v[l] = acc;
        }
        return tree256(v);
    }
    template <class Term>
    double freduce(Term term) const { return combine(fblocks(term)); }
    // RUN order (the PCG vector update's r.r, r.z and b.b): the flat blocks
    // (RT*KF consecutive nodes) are dealt to G = min(blocks, UPD_SLOTS) runs,
    // run c taking blocks c, c+G, c+2G, ...; thread t of a run accumulates its
    // KF nodes of each of the run's blocks, block after block, in one sum from
    // +0.0; the run's RT sums go through the block tree, and the G run sums
    // are combined like partials.
    template <class Term>
    double ureduce(Term term) const {
        const long RB = (long)RT * g_KF;
        const long nb = (Nn + RB - 1) / RB;
        const long G = nb < UPD_SLOTS ? nb : UPD_SLOTS;
        std::vector<double> U(G);
        #pragma omp parallel for schedule(static)
        for (long c = 0; c < G; ++c) {
            double v[RT];
            for (int l = 0; l < RT; ++l) {
                double acc = 0.0;
                for (long b = c; b < nb; b += G)
                    for (int k = 0; k < g_KF; ++k) {
                        const long n = b * RB + (long)l * g_KF + k;
                        if (n >= Nn) break;
                        acc = term(n, acc);
                    }
                v[l] = acc;
            }
            U[c] = tree256(v);
        }
        return combine(U);
    }
    double dot(const double* a, const double* b) const {
        return freduce([&](long n, double acc) { return std::fma(a[n], b[n], acc); });
    }
    double udot(const double* a, const double* b) const {   // update order
        return ureduce([&](long n, double acc) { return std::fma(a[n], b[n], acc); });
    }
    double adot(const double* a, const double* b) const {   // apply order
        return creduce([&](long n, double acc) { return std::fma(a[n], b[n], acc); });
    }
    double one_int(long n) const { return is_bnd_n(n) ? 0.0 : 1.0; }

    // ---- operator (het.cu:885-921) ---------------------------------------------
    // apply y = (M + dt_eff K) x; returns the D1 relative checksum error
    // (or -1 if not evaluated).  fire_R: a pending level-R flip fires here.
    double apply(const double* x, double* y, double dt_eff, bool fire_R, bool project, bool d1) {
        compute_elements(x, dt_eff, fire_R);
        if (colored) gather_nodes(y); else scatter_atomic(y);
        if (project) {
            for (long n = 0; n < Nn; ++n) if (is_bnd_n(n)) y[n] = 0.0;
        }
        double rel = -1.0;
        if (detect && project && d1) {
            const double* w = (dt_eff == 0.0) ? wM.data() : wA.data();
            const double nw = (dt_eff == 0.0) ? norm_wM : norm_wA;
            double s = creduce([&](long n, double acc) { return std::fma(one_int(n), y[n], acc); });
            double c = adot(w, x);
            double nx = std::sqrt(adot(x, x));
            rel = std::fabs(s - c) / std::fma(nw, nx, 1e-300);
            if (!std::isfinite(rel)) rel = 1e300;
            abft_step_max = std::fmax(abft_step_max, rel);
            abft_calls++;
        }
        return rel;
    }

    // ---- setup (het.cu:756-816, 940-953) -------------------------------------
    void build_diag() {
        diag.assign(Nn, 0.0);
        std::vector<double> de((size_t)Ne * 8);
        for (long e = 0; e < Ne; ++e) {
            const double dk = dt * k[e];
            for (int i = 0; i < 8; ++i)
                de[(size_t)e * 8 + Q_OF_LOCAL[i]] = std::fma(rhoc[e], M[i * 9], dk * K[i * 9]);
        }
        std::swap(ye_buf, de);
        gather_nodes(diag.data());
        std::swap(ye_buf, de);
        for (long n = 0; n < Nn; ++n) if (is_bnd_n(n)) diag[n] = 1.0;
    }
    void build_source() {
        F.assign(Nn, 0.0);
        if (verify) return;
        if (no_source) {
            // the reference still builds F with the source on (no_source is set
            // after setup, het.cu:1444-1445) but never adds it to the RHS
        }
        const double gp = 1.0 / 1.7320508075688772;
        const double pts[2] = {-gp, gp};
        std::vector<double> fe((size_t)Ne * 8);
        #pragma omp parallel for schedule(static)
        for (long e = 0; e < Ne; ++e) {
            int ex = (int)(e / ((long)N * N)), ey = (int)((e / N) % N), ez = (int)(e % N);
            double x0 = (double)ex * h, y0 = (double)ey * h, z0 = (double)ez * h;
            double Fe[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int gi = 0; gi < 2; ++gi) for (int gj = 0; gj < 2; ++gj) for (int gk = 0; gk < 2; ++gk) {
                double xg = x0 + (pts[gi] + 1.0) * 0.5 * h;
                double yg = y0 + (pts[gj] + 1.0) * 0.5 * h;
                double zg = z0 + (pts[gk] + 1.0) * 0.5 * h;
                double dx = xg - 0.5, dy = yg - 0.5, dz = zg - 0.5;
                double r2 = dx * dx + dy * dy + dz * dz;
                double Q = 1000.0 * std::exp(-r2 / (2.0 * src_sigma * src_sigma));
                int g = gi * 4 + gj * 2 + gk;
                double dq = detJ * Q;
                for (int i = 0; i < 8; ++i) Fe[i] = std::fma(dq, gN[g][i], Fe[i]);
            }
            for (int i = 0; i < 8; ++i) fe[(size_t)e * 8 + Q_OF_LOCAL[i]] = Fe[i];
        }
        std::swap(ye_buf, fe);
        gather_nodes(F.data());
        std::swap(ye_buf, fe);
        for (long n = 0; n < Nn; ++n) if (is_bnd_n(n)) F[n] = 0.0;
    }
    void setup_detectors() {
        std::vector<double> ones(Nn);
        for (long n = 0; n < Nn; ++n) ones[n] = is_bnd_n(n) ? 0.0 : 1.0;
        wM.assign(Nn, 0.0); wA.assign(Nn, 0.0);
        int save = detect, save_col = colored; detect = 0; colored = 1;
        apply(ones.data(), wM.data(), 0.0, false, false, false);
        apply(ones.data(), wA.data(), dt, false, false, false);
        colored = save_col;
        norm_wM = std::sqrt(dot(wM.data(), wM.data()));
        norm_wA = std::sqrt(dot(wA.data(), wA.data()));
        detect = save;
    }

    // ---- build_rhs (het.cu:963-971) ---------------------------------------------
    void build_rhs(const double* T, double* b) {
        apply(T, b, 0.0, false, true, true);
        if (!verify && !no_source)
            for (long n = 0; n < Nn; ++n) b[n] = std::fma(dt, F[n], b[n]);
    }

    // ---- PCG (het.cu:994-1039) with the vector flips of the B200 library -------
    struct CgLog { std::vector<double> rel, alpha, beta; double rel0 = 0; };
    int pcg(const double* b, double* x, int max_iter, double tol, double* r, double* z,
            double* p, double* Ap, CgLog* log) {
        apply(x, Ap, dt, armed_R != 0, true, true);
        armed_R = 0;
        double bb = 0, rz = 0, rr = 0;
        for (long n = 0; n < Nn; ++n) { r[n] = std::fma(-1.0, Ap[n], b[n]); z[n] = r[n] / diag[n]; }
        bb = udot(b, b); rz = udot(r, z); rr = udot(r, r);
        double bnorm = std::sqrt(bb);
        if (bnorm < 1e-30) bnorm = 1.0;
        if (log) log->rel0 = std::sqrt(rr) / bnorm;
        double rho = rz, beta = 0.0;
        int it = 0;
        for (it = 0; it < max_iter; ++it) {
            for (long n = 0; n < Nn; ++n) p[n] = (it == 0) ? z[n] : std::fma(beta, p[n], z[n]);
            if (vec_level == LV_P && it == vec_iter) p[vec_idx] = flip(p[vec_idx], fi_bit);
            // the matvec and its checksum see the flipped Ap (level 7)
            compute_elements(p, dt, false);
            if (colored) gather_nodes(Ap); else scatter_atomic(Ap);
            for (long n = 0; n < Nn; ++n) if (is_bnd_n(n)) Ap[n] = 0.0;
            if (vec_level == LV_AP && it == vec_iter) Ap[vec_idx] = flip(Ap[vec_idx], fi_bit);
            if (detect) {
                double s = creduce([&](long n, double acc) { return std::fma(one_int(n), Ap[n], acc); });
                double c = adot(wA.data(), p);
                double nx = std::sqrt(adot(p, p));
                double rel = std::fabs(s - c) / std::fma(norm_wA, nx, 1e-300);
                if (!std::isfinite(rel)) rel = 1e300;
                abft_step_max = std::fmax(abft_step_max, rel);
                abft_calls++;
            }
            double pAp = adot(p, Ap);
            if (std::fabs(pAp) < 1e-30) break;
            double alpha = rho / pAp;
            for (long n = 0; n < Nn; ++n) {
                x[n] = std::fma(alpha, p[n], x[n]);
                r[n] = std::fma(-alpha, Ap[n], r[n]);
            }
            if (vec_level == LV_RV && it == vec_iter) r[vec_idx] = flip(r[vec_idx], fi_bit);
            for (long n = 0; n < Nn; ++n) z[n] = r[n] / diag[n];
            rr = udot(r, r); rz = udot(r, z);
            double rnorm = std::sqrt(rr);
            bool conv = (rnorm / bnorm < tol);
            beta = 0.0;
            if (!conv) { beta = rz / rho; rho = rz; }
            if (log) { log->rel.push_back(rnorm / bnorm); log->alpha.push_back(alpha); log->beta.push_back(beta); }
            if (conv) { it++; break; }
        }
        return it;
    }

    void gaussian_ic(double* T) const {
        const double den = 2.0 * ic_sigma * ic_sigma;
        for (long n = 0; n < Nn; ++n) {
            int ix = (int)(n / ((long)NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
            double x = (double)ix * h, y = (double)iy * h, z = (double)iz * h;
            double dx = x - 0.5, dy = y - 0.5, dz = z - 0.5;
            double r2 = dx * dx + dy * dy + dz * dz;
            T[n] = std::exp(-r2 / den);
            if (is_bnd(ix, iy, iz)) T[n] = 0.0;
        }
    }
    void exact_mode(double* v, double t, double alpha) const {
        const double pi = 3.14159265358979323846;
        double amp = std::exp(-3.0 * pi * pi * alpha * t);
        for (long n = 0; n < Nn; ++n) {
            int ix = (int)(n / ((long)NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
            double x = (double)ix * h, y = (double)iy * h, z = (double)iz * h;
            v[n] = amp * std::sin(pi * x) * std::sin(pi * y) * std::sin(pi * z);
            if (is_bnd(ix, iy, iz)) v[n] = 0.0;
        }
    }
};

}  // namespace

// =============================================================================
// C API (ctypes)
// =============================================================================
extern "C" {

struct or_step_out {
    int cg_iters;
    double d1, d2, tmin, tmax, E, spread;
    int snap;  // 1 if this step was a snapshot
};

// apply tile shape (cx planes, ty rows, tz columns; 0 = the per-N shape) and the
// flat order's nodes per thread kf
void or_set_layout(int cx, int ty, int tz, int kf) {
    g_slab_override = SlabLayout{};
    if (cx > 0 && ty > 0 && tz > 0) { g_slab_override.C = tz; g_slab_override.R = ty; g_slab_override.CX = cx; }
    g_KF = kf;
}
// the per-N tile shape: out[0..2] = cx, ty (rows), tz (columns); returns the tile count
long or_slab_layout(int N, int* out3) {
    const SlabLayout L = slab_layout(N);
    out3[0] = L.CX; out3[1] = L.R; out3[2] = L.C;
    return L.ntiles;
}

int or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

void* or_create(int N, double dt, int form, int colored, int detect, int verify, int no_source,
                int ic_mode, double ic_sigma, const double* k, const double* rhoc, int* status) {
    Oracle* o = new Oracle();
    o->N = N; o->NN = N + 1;
    o->Nn = (long)o->NN * o->NN * o->NN; o->Ne = (long)N * N * N;
    o->h = 1.0 / N; o->dt = dt;
    o->form = form; o->colored = colored; o->verify = verify; o->no_source = no_source;
    o->ic_mode = ic_mode; o->ic_sigma = ic_sigma;
    o->k.assign(k, k + o->Ne); o->rhoc.assign(rhoc, rhoc + o->Ne);
    o->kmin = o->kmax = k[0]; o->rhocmin = o->rhocmax = rhoc[0];
    for (long e = 0; e < o->Ne; ++e) {
        if (!(k[e] > 0) || !(rhoc[e] > 0)) { *status = 1; delete o; return nullptr; }
        o->kmin = std::fmin(o->kmin, k[e]); o->kmax = std::fmax(o->kmax, k[e]);
        o->rhocmin = std::fmin(o->rhocmin, rhoc[e]); o->rhocmax = std::fmax(o->rhocmax, rhoc[e]);
    }
    o->build_reference_matrices();
    if (!o->matrix_ok) { *status = 2; delete o; return nullptr; }
    o->build_diag();
    o->build_source();
    o->detect = 0;
    if (detect) { o->setup_detectors(); o->detect = 1; }
    *status = 0;
    return o;
}

void or_destroy(void* h) { delete (Oracle*)h; }

void or_get_vectors(void* h, double* diag, double* F, double* wM, double* wA, double* norms) {
    Oracle* o = (Oracle*)h;
    if (diag) std::memcpy(diag, o->diag.data(), o->Nn * 8);
    if (F) std::memcpy(F, o->F.data(), o->Nn * 8);
    if (wM && !o->wM.empty()) std::memcpy(wM, o->wM.data(), o->Nn * 8);
    if (wA && !o->wA.empty()) std::memcpy(wA, o->wA.data(), o->Nn * 8);
    if (norms) { norms[0] = o->norm_wM; norms[1] = o->norm_wA; }
}

void or_get_matrices(void* h, double* M, double* K, double* errs) {
    Oracle* o = (Oracle*)h;
    if (M) std::memcpy(M, o->M, sizeof(o->M));
    if (K) std::memcpy(K, o->K, sizeof(o->K));
    if (errs) std::memcpy(errs, o->mat_err, sizeof(o->mat_err));
}

double or_apply(void* h, const double* x, double* y, double dt_eff, int project, int d1,
                long fi_elem, int fi_bit) {
    Oracle* o = (Oracle*)h;
    o->fi_target_elem = fi_elem; o->fi_bit = fi_bit;
    double r = o->apply(x, y, dt_eff, fi_elem >= 0, project != 0, d1 != 0);
    o->fi_target_elem = -1;
    return r;
}

double or_dot(void* h, const double* a, const double* b) { return ((Oracle*)h)->dot(a, b); }
// the PCG update's order (RUN)
double or_udot(void* h, const double* a, const double* b) { return ((Oracle*)h)->udot(a, b); }

void or_build_rhs(void* h, const double* T, double* b) { ((Oracle*)h)->build_rhs(T, b); }

int or_pcg(void* h, const double* b, double* x, int max_iter, double tol, double* log_rel,
           double* log_alpha, double* log_beta, double* rel0) {
    Oracle* o = (Oracle*)h;
    std::vector<double> r(o->Nn), z(o->Nn), p(o->Nn), Ap(o->Nn);
    Oracle::CgLog lg;
    int it = o->pcg(b, x, max_iter, tol, r.data(), z.data(), p.data(), Ap.data(), &lg);
    for (size_t i = 0; i < lg.rel.size(); ++i) {
        if (log_rel) log_rel[i] = lg.rel[i];
        if (log_alpha) log_alpha[i] = lg.alpha[i];
        if (log_beta) log_beta[i] = lg.beta[i];
    }
    if (rel0) *rel0 = lg.rel0;
    return it;
}

// One full trajectory (het.cu:1107-1259). T (Nn) holds the final field on
// return. ref_snaps: n_snap*Nn snapshots of the reference run (or null);
// keep_snaps: output buffer for this run's snapshots (or null).
// d3_ref_tmin/tmax: the reference run's per-step range (or null).
int or_run_case(void* h, int n_steps, int snap_every, int max_iter, double tol,
                int fi_level, int fi_step, long fi_target, int fi_bit, int fi_iter,
                int reproject, double* T, const double* ref_snaps, double* keep_snaps,
                const double* d3_ref_tmin, const double* d3_ref_tmax,
                or_step_out* out, int* nonfinite) {
    Oracle* o = (Oracle*)h;
    const long Nn = o->Nn;
    std::vector<double> b(Nn), r(Nn), z(Nn), p(Nn), Ap(Nn);
    std::fill(T, T + Nn, 0.0);
    if (o->ic_mode == 1) o->gaussian_ic(T);
    *nonfinite = 0;
    int si = 0;
    o->abft_step_max = 0; o->abft_calls = 0;
    for (int step = 0; step < n_steps; ++step) {
        o->armed_R = 0; o->vec_level = 0;
        if (fi_level > 0 && step == fi_step) {
            if (fi_level == LV_G) {
                long idx = fi_target % Nn;
                T[idx] = flip(T[idx], fi_bit);
            } else if (fi_level == LV_R) {
                o->armed_R = 1; o->fi_target_elem = fi_target; o->fi_bit = fi_bit;
            } else {
                o->vec_level = fi_level; o->vec_iter = fi_iter; o->vec_idx = fi_target % Nn; o->fi_bit = fi_bit;
            }
        }
        o->build_rhs(T, b.data());
        int it = o->pcg(b.data(), T, max_iter, tol, r.data(), z.data(), p.data(), Ap.data(), nullptr);
        if (reproject) for (long n = 0; n < Nn; ++n) if (o->is_bnd_n(n)) T[n] = 0.0;
        o->armed_R = 0; o->vec_level = 0; o->fi_target_elem = -1;
        or_step_out& so = out[step];
        so.cg_iters = it;
        so.d1 = so.d2 = so.tmin = so.tmax = 0; so.E = -1; so.spread = 0; so.snap = 0;
        if (o->detect) {
            so.d1 = o->abft_step_max;
            o->apply(T, Ap.data(), o->dt, false, true, false);
            for (long n = 0; n < Nn; ++n) r[n] = std::fma(-1.0, Ap[n], b[n]);
            double bn = std::sqrt(o->dot(b.data(), b.data()));
            if (bn < 1e-300) bn = 1.0;
            so.d2 = std::sqrt(o->dot(r.data(), r.data())) / bn;
            double mn = 1e300, mx = -1e300;
            for (long n = 0; n < Nn; ++n) { mn = std::fmin(mn, T[n]); mx = std::fmax(mx, T[n]); }
            so.tmin = mn; so.tmax = mx;
            (void)d3_ref_tmin; (void)d3_ref_tmax;
            o->abft_step_max = 0; o->abft_calls = 0;
        }
        bool snap = (snap_every > 0 && step % snap_every == 0) || step == n_steps - 1;
        if (snap) {
            so.snap = 1;
            if (keep_snaps) std::memcpy(keep_snaps + (size_t)si * Nn, T, Nn * 8);
            if (ref_snaps) {
                const double* a = T;
                const double* bb = ref_snaps + (size_t)si * Nn;
                double num = o->freduce([&](long n, double acc) { double d = a[n] - bb[n]; return std::fma(d, d, acc); });
                double den = o->freduce([&](long n, double acc) { return std::fma(bb[n], bb[n], acc); });
                double dmax = 0.0;
                for (long n = 0; n < Nn; ++n) { double d = std::fabs(a[n] - bb[n]); if (d > dmax) dmax = d; }
                long cnt = 0;
                for (long n = 0; n < Nn; ++n) if (std::fabs(a[n] - bb[n]) > 1e-3 * dmax) ++cnt;
                so.spread = (dmax > 0) ? (double)cnt / (double)Nn : 0.0;
                if (den < 1e-300) den = 1.0;
                so.E = std::sqrt(num / den);
                if (!std::isfinite(so.E)) *nonfinite = 1;
            }
            ++si;
        }
    }
    return 0;
}

// --verify (het.cu:1293-1338): returns the relative L2 error; total CG iterations in *total_it
double or_verify(void* h, int n_steps, int max_iter, double tol, long* total_it) {
    Oracle* o = (Oracle*)h;
    const long Nn = o->Nn;
    std::vector<double> T(Nn), b(Nn), r(Nn), z(Nn), p(Nn), Ap(Nn);
    double alpha = o->kmin / o->rhocmin;
    o->exact_mode(T.data(), 0.0, alpha);
    long tot = 0;
    for (int step = 0; step < n_steps; ++step) {
        o->build_rhs(T.data(), b.data());
        tot += o->pcg(b.data(), T.data(), max_iter, tol, r.data(), z.data(), p.data(), Ap.data(), nullptr);
    }
    double t_end = n_steps * o->dt;
    o->exact_mode(r.data(), t_end, alpha);
    double en = std::sqrt(o->dot(r.data(), r.data()));
    for (long n = 0; n < Nn; ++n) r[n] = std::fma(-1.0, T[n], r[n]);
    double rel = std::sqrt(o->dot(r.data(), r.data())) / en;
    if (total_it) *total_it = tot;
    return rel;
}

void or_initial_condition(void* h, double* T) {
    Oracle* o = (Oracle*)h;
    std::fill(T, T + o->Nn, 0.0);
    if (o->ic_mode == 1) o->gaussian_ic(T);
}

}  // extern "C"
