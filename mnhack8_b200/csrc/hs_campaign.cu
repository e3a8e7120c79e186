// hs_campaign.cu -- seeded single-bit-flip campaign over one trajectory.
//
// The reference studies faults one process per flip (a clean twin and one
// faulted run of heat_solver_het per case, driven by its campaign scripts,
// het.cu:1506-1620).  Here one handle runs the clean trajectory once (kept
// as the reference, with its field at the start of every step), its clean
// twin once, and then every faulted trajectory resumed at its flip step from
// the kept clean field: the steps before a flip are bit-identical to the
// clean run in the deterministic (colored) mode, so only the steps from the
// flip on are recomputed.  Each faulted run is classified with the
// reference's twin-run rules (hs_classify).
//
// Included by hs_solver.cu (needs the handle's internals).
#include <random>

extern "C" hs_status hs_campaign(hs_solver* h, int n_steps, int snap_every, int n_flips, unsigned long long seed,
                                 int vec_mask, hs_step_record* clean_out, hs_flip_record* out) {
    if (!h || n_steps < 1 || n_flips < 0 || (n_flips > 0 && !out) || (vec_mask & 7) == 0 || (vec_mask & ~7)) {
        set_error("hs_campaign: bad arguments");
        return HS_ERR_ARG;
    }
    if (h->opt.scatter != HS_SCATTER_COLORED) {
        set_error("hs_campaign: needs the deterministic (colored) scatter to resume faulted runs mid-trajectory");
        return HS_ERR_ARG;
    }
    std::vector<int> levels;
    if (vec_mask & 1) levels.push_back(HS_FI_P);
    if (vec_mask & 2) levels.push_back(HS_FI_RV);
    if (vec_mask & 4) levels.push_back(HS_FI_AP);
    const long long Nn = h->Nn;

    // field at the start of every step of the clean run
    struct States {
        std::vector<double*> p;
        ~States() { for (double* q : p) if (q) cudaFree(q); }
    } states;
    states.p.assign(n_steps, nullptr);
    for (int s = 0; s < n_steps; ++s) HS_CUDA(cudaMalloc(&states.p[s], Nn * 8));

    std::vector<hs_step_record> A(n_steps), B(n_steps), F(n_steps);
    RunFrom keep;
    keep.keep_states = states.p.data();
    hs_status st = run_case_impl(h, n_steps, snap_every, nullptr, 0, 1, A.data(), nullptr, nullptr, keep);
    if (st != HS_OK) return st;
    int nfB = 0;
    st = run_case_impl(h, n_steps, snap_every, nullptr, 0, 0, B.data(), nullptr, &nfB, RunFrom{});
    if (st != HS_OK) return st;
    if (clean_out) std::copy(A.begin(), A.end(), clean_out);

    std::vector<long long> cum(n_steps + 1, 0);
    for (int s = 0; s < n_steps; ++s) cum[s + 1] = cum[s] + A[s].cg_iters;
    const long long total = cum[n_steps];
    if (n_flips > 0 && total <= 0) {
        set_error("hs_campaign: the clean run has no CG iterations to flip");
        return HS_ERR_STATE;
    }

    std::mt19937_64 rng(seed);
    for (int f = 0; f < n_flips; ++f) {
        // site: global iteration -> (step, iteration), vector, entry, bit
        const long long g = (long long)(rng() % (unsigned long long)total);
        const int step = (int)(std::upper_bound(cum.begin(), cum.end(), g) - cum.begin()) - 1;
        const int iter = (int)(g - cum[step]);
        const int level = levels[rng() % levels.size()];
        const long long idx = (long long)(rng() % (unsigned long long)Nn);
        const int bit = (int)(rng() % 64ULL);
        hs_fi_spec fi{};
        fi.level = level; fi.step = step; fi.target = idx; fi.bit = bit; fi.iter = iter; fi.rank = 0;
        // steps before the flip: the clean run, equal to the reference (E = 0)
        for (int s = 0; s < step; ++s) {
            F[s] = A[s];
            if (F[s].snap) { F[s].E = 0.0; F[s].spread = 0.0; }
        }
        int nf = 0;
        RunFrom from;
        from.s0 = step;
        from.T_start = states.p[step];
        st = run_case_impl(h, n_steps, snap_every, &fi, 0, 0, F.data(), nullptr, &nf, from);
        if (st != HS_OK) return st;
        hs_flip_record& r = out[f];
        std::memset(&r, 0, sizeof(r));
        r.step = step; r.iter = iter; r.level = level; r.bit = bit; r.idx = idx; r.nonfinite = nf;
        long long it = 0;
        for (int s = 0; s < n_steps; ++s) it += F[s].cg_iters;
        r.iters_total_delta = (int)(it - total);
        st = hs_classify(A.data(), B.data(), F.data(), n_steps, level, nf, h->opt.dt, 1e-13, h->opt.detect,
                         &r.summary);
        if (st != HS_OK) return st;
    }
    return HS_OK;
}
