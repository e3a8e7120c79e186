// hs_cli.h -- twin-run records and summary (internal to libheat_b200).
#pragma once
#include <string>
#include <vector>

#include "../../include/heat_b200.h"

namespace hs {

struct RunRecords {
    std::vector<hs_step_record> steps;
    int nonfinite = 0;
    double solve_ms = 0;
};

struct DetSummary {
    int d1_first = -1, d2_first = -1, d3_first = -1;
    double d1_max = 0, d2_max = 0;
};

struct TwinSummary {
    std::vector<int> snap_steps;
    double Efl_max, Efl_final, Efa_max, Efa_int, Efa_final, thr, spread_at_max, spread_final;
    int step_max, iters_delta_max;
    const char* cls;
    DetSummary detA, detX;
    std::string by;
};

TwinSummary summarize(const RunRecords& A, const RunRecords& B, const RunRecords* F, int fi_level, double dt,
                      double thr_user, int detect);

}  // namespace hs
