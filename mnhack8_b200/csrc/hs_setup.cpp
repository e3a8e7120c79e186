// hs_setup.cpp -- host set-up arithmetic of libheat_b200 (compiled with
// -ffp-contract=off: every fused multiply-add below is an explicit std::fma).
#include "hs_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

namespace hs {

namespace {

// trilinear shape functions and reference gradients on [-1,1]^3 (het.cu:242-257)
void shape(double xi, double eta, double zeta, double Nv[8], double dN[8][3]) {
    static const int sgn[8][3] = {{-1,-1,-1},{1,-1,-1},{1,1,-1},{-1,1,-1},
                                  {-1,-1,1},{1,-1,1},{1,1,1},{-1,1,1}};
    for (int i = 0; i < 8; ++i) {
        const double sx = sgn[i][0], sy = sgn[i][1], sz = sgn[i][2];
        const double a = 1 + sx * xi, b = 1 + sy * eta, c = 1 + sz * zeta;
        Nv[i] = 0.125 * a * b * c;
        dN[i][0] = 0.125 * sx * b * c;
        dN[i][1] = 0.125 * a * sy * c;
        dN[i][2] = 0.125 * a * b * sz;
    }
}

const int kQofLocal[8] = {0, 4, 6, 2, 1, 5, 7, 3};

int hw_threads() {
    unsigned n = std::thread::hardware_concurrency();
    return n ? (int)std::min(n, 64u) : 4;
}

template <class F>
void parallel_for(long lo, long hi, F f) {
    const int nt = hw_threads();
    if (hi - lo < 4096 || nt <= 1) { f(lo, hi); return; }
    std::vector<std::thread> th;
    const long chunk = (hi - lo + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        long a = lo + t * chunk, b = std::min(hi, a + chunk);
        if (a >= b) break;
        th.emplace_back([=] { f(a, b); });
    }
    for (auto& x : th) x.join();
}

}  // namespace

RefMatrices build_reference_matrices(int N) {
    RefMatrices r;
    std::memset(&r, 0, sizeof(r));
    const double hx = 1.0 / N, hy = 1.0 / N, hz = 1.0 / N;
    const double detJ = hx * hy * hz / 8.0;
    const double iJ[3] = {2.0 / hx, 2.0 / hy, 2.0 / hz};
    const double gp = 1.0 / 1.7320508075688772;
    const double pts[2] = {-gp, gp};
    double Mh[64] = {0}, Kh[64] = {0};
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) for (int c = 0; c < 2; ++c) {
        double Nv[8], dN[8][3];
        shape(pts[a], pts[b], pts[c], Nv, dN);
        for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) {
            Mh[i * 8 + j] += detJ * Nv[i] * Nv[j];
            Kh[i * 8 + j] += detJ * (iJ[0] * dN[i][0] * iJ[0] * dN[j][0]
                                   + iJ[1] * dN[i][1] * iJ[1] * dN[j][1]
                                   + iJ[2] * dN[i][2] * iJ[2] * dN[j][2]);
        }
    }
    // closed forms: M = V/216 {8,4,2,1}[node distance], K row sums 0,
    // K diagonal (hy hz/hx + hx hz/hy + hx hy/hz)/9, both symmetric
    static const int sgn[8][3] = {{-1,-1,-1},{1,-1,-1},{1,1,-1},{-1,1,-1},
                                  {-1,-1,1},{1,-1,1},{1,1,1},{-1,1,1}};
    const double V = hx * hy * hz;
    double errM = 0, sumM = 0, errKrow = 0, errKdiag = 0, errSym = 0;
    const double Kdiag = (hy * hz / hx + hx * hz / hy + hx * hy / hz) / 9.0;
    for (int i = 0; i < 8; ++i) {
        double rs = 0;
        for (int j = 0; j < 8; ++j) {
            const int d = (sgn[i][0] != sgn[j][0]) + (sgn[i][1] != sgn[j][1]) + (sgn[i][2] != sgn[j][2]);
            const double Mref = V / 216.0 * (double)(8 >> d);
            errM = std::fmax(errM, std::fabs(Mh[i * 8 + j] - Mref) / (V / 216.0 * 8));
            sumM += Mh[i * 8 + j];
            rs += Kh[i * 8 + j];
            errSym = std::fmax(errSym, std::fabs(Kh[i * 8 + j] - Kh[j * 8 + i]) + std::fabs(Mh[i * 8 + j] - Mh[j * 8 + i]));
        }
        errKrow = std::fmax(errKrow, std::fabs(rs) / Kdiag);
        errKdiag = std::fmax(errKdiag, std::fabs(Kh[i * 9] - Kdiag) / Kdiag);
    }
    const double errSum = std::fabs(sumM - V) / V;
    r.ok = errM < 1e-12 && errSum < 1e-12 && errKrow < 1e-12 && errKdiag < 1e-12 && errSym < 1e-12 * Kdiag;
    r.err[0] = errM; r.err[1] = errSum; r.err[2] = errKrow; r.err[3] = errKdiag; r.err[4] = errSym;
    std::memcpy(r.M, Mh, sizeof(Mh));
    std::memcpy(r.K, Kh, sizeof(Kh));

    // gauss form tables (het.cu:313-328), point g = gi*4 + gj*2 + gk
    r.detJ = detJ;
    const double invJ = 2.0 / hx;
    for (int gi = 0; gi < 2; ++gi) for (int gj = 0; gj < 2; ++gj) for (int gk = 0; gk < 2; ++gk) {
        const int g = gi * 4 + gj * 2 + gk;
        double Nv[8], dN[8][3];
        shape(pts[gi], pts[gj], pts[gk], Nv, dN);
        for (int i = 0; i < 8; ++i) {
            r.gtab[g * 8 + i] = Nv[i];
            r.gtab[64 + g * 8 + i] = invJ * dN[i][0];
            r.gtab[128 + g * 8 + i] = invJ * dN[i][1];
            r.gtab[192 + g * 8 + i] = invJ * dN[i][2];
        }
    }
    // wht: eigenvalues of m = h/6 [2 1;1 2] are h/2, h/6; of k = 1/h [1 -1;-1 1]
    // are 0, 2/h.  Walsh index weight j (number of difference modes):
    // mass h^3 (1/6)^j (1/2)^(3-j), stiffness j (2/h) (h/6)^(j-1) (h/2)^(3-j).
    const double h = hx;
    const double hs = h / 6.0, hb = h / 2.0, g2 = 2.0 / h;
    const double mu[4] = {hb * hb * hb, hs * hb * hb, hs * hs * hb, hs * hs * hs};
    const double ka[4] = {0.0, g2 * hb * hb, 2.0 * (g2 * hs * hb), 3.0 * (g2 * hs * hs)};
    for (int j = 0; j < 4; ++j) { r.cm[j] = mu[j] / 8.0; r.ck[j] = ka[j] / 8.0; }
    return r;
}

// F_i = sum over elements (canonical node order: lower x-plane first, then
// (y, z) order) of int Q N_i, 2x2x2 Gauss (het.cu:381-407); boundary 0.
void build_source(int N, double src_sigma, std::vector<double>& F) {
    const long NN = N + 1, Nn = NN * NN * NN;
    F.assign(Nn, 0.0);
    const double h = 1.0 / N;
    const double detJ = h * h * h / 8.0;
    const double gp = 1.0 / 1.7320508075688772;
    const double pts[2] = {-gp, gp};
    double gN[8][8];
    for (int gi = 0; gi < 2; ++gi) for (int gj = 0; gj < 2; ++gj) for (int gk = 0; gk < 2; ++gk) {
        double Nv[8], dN[8][3];
        shape(pts[gi], pts[gj], pts[gk], Nv, dN);
        for (int i = 0; i < 8; ++i) gN[gi * 4 + gj * 2 + gk][i] = Nv[i];
    }
    auto elem_plane = [&](int ex, std::vector<double>& out) {   // out[(ey*N+ez)*8 + q]
        out.resize((size_t)N * N * 8);
        const double x0 = (double)ex * h;
        for (int ey = 0; ey < N; ++ey) for (int ez = 0; ez < N; ++ez) {
            const double y0 = (double)ey * h, z0 = (double)ez * h;
            double Fe[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int gi = 0; gi < 2; ++gi) for (int gj = 0; gj < 2; ++gj) for (int gk = 0; gk < 2; ++gk) {
                const double xg = x0 + (pts[gi] + 1.0) * 0.5 * h;
                const double yg = y0 + (pts[gj] + 1.0) * 0.5 * h;
                const double zg = z0 + (pts[gk] + 1.0) * 0.5 * h;
                const double dx = xg - 0.5, dy = yg - 0.5, dz = zg - 0.5;
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double Q = 1000.0 * std::exp(-r2 / (2.0 * src_sigma * src_sigma));
                const double dq = detJ * Q;
                const int g = gi * 4 + gj * 2 + gk;
                for (int i = 0; i < 8; ++i) Fe[i] = std::fma(dq, gN[g][i], Fe[i]);
            }
            double* o = &out[((size_t)ey * N + ez) * 8];
            for (int i = 0; i < 8; ++i) o[kQofLocal[i]] = Fe[i];
        }
    };
    // node planes 1..N-1 carry sources (x boundary planes are projected to 0)
    parallel_for(1, N, [&](long a, long b) {
        std::vector<double> lo, hi;
        elem_plane((int)a - 1, lo);
        for (long ix = a; ix < b; ++ix) {
            elem_plane((int)ix, hi);
            for (int iy = 1; iy < N; ++iy) for (int iz = 1; iz < N; ++iz) {
                // canonical node sum: element corners q = 4, 7, 6, 5, 0, 3, 2, 1
                static const int order[8] = {4, 7, 6, 5, 0, 3, 2, 1};
                double acc = 0.0;
                for (int s = 0; s < 8; ++s) {
                    const int q = order[s];
                    const std::vector<double>& pl = ((q >> 2) & 1) ? lo : hi;
                    const int ey = iy - ((q >> 1) & 1), ez = iz - (q & 1);
                    acc = acc + pl[((size_t)ey * N + ez) * 8 + q];
                }
                F[(ix * NN + iy) * NN + iz] = acc;
            }
            std::swap(lo, hi);
        }
    });
}

void gaussian_ic(int N, double sigma, double* T) {
    const long NN = N + 1, Nn = NN * NN * NN;
    const double h = 1.0 / N;
    const double den = 2.0 * sigma * sigma;
    parallel_for(0, Nn, [&](long a, long b) {
        for (long n = a; n < b; ++n) {
            const int ix = (int)(n / (NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
            const double x = (double)ix * h, y = (double)iy * h, z = (double)iz * h;
            const double dx = x - 0.5, dy = y - 0.5, dz = z - 0.5;
            const double r2 = dx * dx + dy * dy + dz * dz;
            T[n] = std::exp(-r2 / den);
            if (ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N) T[n] = 0.0;
        }
    });
}

void exact_mode(int N, double t, double alpha, double* v) {
    const long NN = N + 1, Nn = NN * NN * NN;
    const double h = 1.0 / N;
    const double pi = 3.14159265358979323846;
    const double amp = std::exp(-3.0 * pi * pi * alpha * t);
    parallel_for(0, Nn, [&](long a, long b) {
        for (long n = a; n < b; ++n) {
            const int ix = (int)(n / (NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
            const double x = (double)ix * h, y = (double)iy * h, z = (double)iz * h;
            v[n] = amp * std::sin(pi * x) * std::sin(pi * y) * std::sin(pi * z);
            if (ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N) v[n] = 0.0;
        }
    });
}

}  // namespace hs
