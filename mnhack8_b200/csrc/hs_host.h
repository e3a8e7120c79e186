// hs_host.h -- host-side set-up arithmetic shared by the library's translation units.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hs {

// Gauss-built reference matrices and their closed-form check
// (HeatOperator::build_reference_matrices, het.cu:661-708)
struct RefMatrices {
    double M[64], K[64];
    double gtab[256];        // gauss form: N, dNx, dNy, dNz at the 8 points
    double detJ;
    double cm[4], ck[4];     // wht eigen-constants / 8
    double err[5];           // M pattern, sum(M)-V, K rowsum, K diag, symmetry
    bool ok;
};
RefMatrices build_reference_matrices(int N);

// source vector F (het.cu:229-237, 381-407, 806-814) and initial conditions
// (het.cu:556-584), on the host so that the exp/sin values are the C
// library's, with the canonical node summation order of the operator.
void build_source(int N, double src_sigma, std::vector<double>& F);
void gaussian_ic(int N, double sigma, double* T);
void exact_mode(int N, double t, double alpha, double* v);

void set_error(const std::string& msg);

}  // namespace hs
