// hs_cli.cpp -- the reference solver's command line on top of the C ABI:
// argv and usage (het.cu:1340-1350, 1380-1433), --verify, --diag-cg, the
// twin-run protocol with fault classification (het.cu:1506-1542) and the
// output files fi_trace_<tag>.csv, fi_summary_<tag>.csv, meta_<tag>.txt,
// T_final_<tag>_{clean,fault}_rank0.bin, verify.csv (het.cu:1544-1620,
// 1261-1269, 1326-1335).  The file formats are the reference's, column for
// column, so the reference's validation scripts read either binary.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/heat_b200.h"
#include "hs_cli.h"

namespace {

void usage(const char* prog) {
    fprintf(stderr,
            "usage: %s N t_final dt field_prefix [outdir]\n"
            "   [--fi LEVEL STEP TARGET BIT] [--fi-rank R] [--fi-iter K] [--snap S] [--tag NAME]\n"
            "   [--kernel gauss|fast|wht] [--scatter atomic|colored] [--thr X]\n"
            "   [--reproject-bc] [--detect] [--verify] [--no-source] [--ic zero|gaussian] [--dump-snaps]\n"
            "   [--ic-sigma S] [--rtol X] [--max-iter M] [--device D]\n"
            "   [--diag-cg FILE]   (one CG solve, logs iteration,rel_residual to FILE, then exits)\n"
            "  LEVEL: 1=G global memory, 2=R accumulator, 3=H halo staging buffer (needs >= 2 ranks),\n"
            "         5=p search direction, 6=r residual, 7=Ap operator output (at PCG iteration K)\n"
            "  BIT:   0-51 mantissa, 52-62 exponent, 63 sign\n",
            prog);
}

int exit_code(hs_status s) { return s == HS_ERR_MATRIX ? 2 : 1; }

void ensure_dir(const std::string& d) {
    if (d.empty()) return;
    struct stat sb;
    if (stat(d.c_str(), &sb) == 0) return;
    std::string cur;
    for (size_t i = 0; i < d.size(); ++i) {
        cur += d[i];
        if (d[i] == '/' || i + 1 == d.size()) mkdir(cur.c_str(), 0755);
    }
}

bool write_bin(const std::string& path, const std::vector<double>& v) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return false;
    fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
    return true;
}

const char* kname(int k) { return k == HS_KERNEL_GAUSS ? "gauss" : (k == HS_KERNEL_WHT ? "wht" : "fast"); }

}  // namespace

namespace hs {

// classification of one twin-run (het.cu:1521-1542) and the detector summary
TwinSummary summarize(const RunRecords& A, const RunRecords& B, const RunRecords* F, int fi_level, double dt,
                      double thr_user, int detect) {
    TwinSummary s{};
    const std::vector<hs_step_record>& rB = B.steps;
    std::vector<int> snap_steps;
    for (size_t i = 0; i < rB.size(); ++i) if (rB[i].snap) snap_steps.push_back((int)i);
    s.snap_steps = snap_steps;
    double Efl_max = 0, Efa_max = 0, Efa_int = 0, Efa_final = 0, Efl_final = 0, spread_at_max = 0, spread_final = 0;
    int step_max = -1, iters_delta_max = 0;
    for (size_t k = 0; k < snap_steps.size(); ++k) {
        const int st = snap_steps[k];
        Efl_max = std::fmax(Efl_max, rB[st].E);
        Efl_final = rB[st].E;
        if (fi_level > 0) {
            const double E = F->steps[st].E;
            if (std::isfinite(E) && E > Efa_max) { Efa_max = E; step_max = st; spread_at_max = F->steps[st].spread; }
            Efa_final = E;
            spread_final = F->steps[st].spread;
            const double w = (k + 1 < snap_steps.size()) ? (snap_steps[k + 1] - st) * dt : 0.0;
            if (std::isfinite(E)) Efa_int += E * w;
        }
    }
    if (fi_level > 0)
        for (size_t i = 0; i < F->steps.size(); ++i)
            iters_delta_max = std::max(iters_delta_max, F->steps[i].cg_iters - A.steps[i].cg_iters);
    const double thr = std::fmax(thr_user, 10.0 * Efl_max);
    const char* cls = "clean";
    if (fi_level > 0) {
        if (F->nonfinite) cls = "detected";
        else if (Efa_max <= thr) cls = "benign";
        else if (Efa_final <= thr) cls = "transient";
        else cls = "persistent";
    }
    s.Efl_max = Efl_max; s.Efl_final = Efl_final; s.Efa_max = Efa_max; s.step_max = step_max;
    s.Efa_int = Efa_int; s.Efa_final = Efa_final; s.thr = thr; s.iters_delta_max = iters_delta_max;
    s.cls = cls; s.spread_at_max = spread_at_max; s.spread_final = spread_final;
    // detectors (het.cu:1202-1234): D1 > 1e-10, D2 > 1e-6, D3 range vs cleanA
    auto det = [&](const RunRecords& X, bool vs_ref, DetSummary& d) {
        d = DetSummary{};
        for (size_t i = 0; i < X.steps.size(); ++i) {
            const hs_step_record& x = X.steps[i];
            bool d3 = !std::isfinite(x.tmin) || !std::isfinite(x.tmax);
            if (vs_ref && i < A.steps.size()) {
                const double ref_max = A.steps[i].tmax, ref_min = A.steps[i].tmin;
                const double margin = 1e-6 * std::fmax(std::fabs(ref_max), 1e-300) + 1e-12;
                if (x.tmax > ref_max + margin || x.tmin < ref_min - margin) d3 = true;
            }
            if (!(x.d1 <= 1e-10) && d.d1_first < 0) d.d1_first = (int)i;
            if (!(x.d2 <= 1e-6) && d.d2_first < 0) d.d2_first = (int)i;
            if (d3 && d.d3_first < 0) d.d3_first = (int)i;
            if (std::isfinite(x.d1)) d.d1_max = std::fmax(d.d1_max, x.d1); else d.d1_max = 1e300;
            if (std::isfinite(x.d2)) d.d2_max = std::fmax(d.d2_max, x.d2); else d.d2_max = 1e300;
        }
    };
    if (detect) {
        det(A, false, s.detA);
        if (fi_level > 0) det(*F, true, s.detX); else s.detX = s.detA;
        std::string by;
        if (s.detX.d1_first >= 0) by += "D1";
        if (s.detX.d2_first >= 0) by += (by.empty() ? "" : "+") + std::string("D2");
        if (s.detX.d3_first >= 0) by += (by.empty() ? "" : "+") + std::string("D3");
        if (by.empty()) by = "none";
        s.by = by;
    } else {
        s.by = "off";
    }
    return s;
}

}  // namespace hs

extern "C" hs_status hs_classify(const hs_step_record* A, const hs_step_record* B, const hs_step_record* F,
                                 int n_steps, int fi_level, int F_nonfinite, double dt, double thr_user, int detect,
                                 hs_twin_summary* out) {
    if (!A || !B || !out || n_steps < 0 || (fi_level > 0 && !F)) return HS_ERR_ARG;
    hs::RunRecords rA, rB, rF;
    rA.steps.assign(A, A + n_steps);
    rB.steps.assign(B, B + n_steps);
    if (F) { rF.steps.assign(F, F + n_steps); rF.nonfinite = F_nonfinite; }
    hs::TwinSummary s = hs::summarize(rA, rB, fi_level > 0 ? &rF : nullptr, fi_level, dt, thr_user, detect);
    std::memset(out, 0, sizeof(*out));
    out->E_floor_max = s.Efl_max; out->E_floor_final = s.Efl_final; out->E_fault_max = s.Efa_max;
    out->E_fault_int = s.Efa_int; out->E_fault_final = s.Efa_final; out->thr = s.thr;
    out->spread_at_max = s.spread_at_max; out->spread_final = s.spread_final;
    out->step_at_max = s.step_max; out->iters_delta_max = s.iters_delta_max;
    out->d1_first = s.detX.d1_first; out->d2_first = s.detX.d2_first; out->d3_first = s.detX.d3_first;
    out->d1_max = s.detX.d1_max; out->d2_max = s.detX.d2_max; out->d1_max_A = s.detA.d1_max; out->d2_max_A = s.detA.d2_max;
    snprintf(out->cls, sizeof(out->cls), "%s", s.cls);
    snprintf(out->detected_by, sizeof(out->detected_by), "%s", s.by.c_str());
    return HS_OK;
}

extern "C" int hs_cli_main(int argc, char** argv) {
    using namespace hs;
    const char* prog = argc > 0 ? argv[0] : "heat_solver_b200";
    if (argc < 5) { usage(prog); return 1; }
    const int N = atoi(argv[1]);
    const double t_final = atof(argv[2]);
    const double dt = atof(argv[3]);
    const char* field_prefix = argv[4];
    std::string outdir = "out", tag = "run", diag_cg_path;
    hs_fi_spec fi{};
    fi.step = -1;
    int snap_every = 5, verify_mode = 0, kernel = HS_KERNEL_FAST, colored = 0, reproject = 0, detect = 0;
    int no_source = 0, ic_mode = 0, dump_snaps = 0, max_iter = 500, device = 0;
    double thr_user = 1e-13, rtol = 1e-8, ic_sigma = 0.1;
    for (int i = 5; i < argc; ++i) {
        if (!strcmp(argv[i], "--fi") && i + 4 < argc) {
            fi.level = atoi(argv[++i]); fi.step = atoi(argv[++i]);
            fi.target = atoll(argv[++i]); fi.bit = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--fi-rank") && i + 1 < argc) { fi.rank = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--fi-iter") && i + 1 < argc) { fi.iter = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--snap") && i + 1 < argc) { snap_every = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--tag") && i + 1 < argc) { tag = argv[++i];
        } else if (!strcmp(argv[i], "--thr") && i + 1 < argc) { thr_user = atof(argv[++i]);
        } else if (!strcmp(argv[i], "--kernel") && i + 1 < argc) {
            const char* k = argv[++i];
            kernel = !strcmp(k, "gauss") ? HS_KERNEL_GAUSS : (!strcmp(k, "wht") ? HS_KERNEL_WHT : HS_KERNEL_FAST);
        } else if (!strcmp(argv[i], "--scatter") && i + 1 < argc) { colored = !strcmp(argv[++i], "colored");
        } else if (!strcmp(argv[i], "--reproject-bc")) { reproject = 1;
        } else if (!strcmp(argv[i], "--detect")) { detect = 1;
        } else if (!strcmp(argv[i], "--diag-cg") && i + 1 < argc) { diag_cg_path = argv[++i];
        } else if (!strcmp(argv[i], "--no-source")) { no_source = 1;
        } else if (!strcmp(argv[i], "--dump-snaps")) { dump_snaps = 1;
        } else if (!strcmp(argv[i], "--ic") && i + 1 < argc) { ic_mode = !strcmp(argv[++i], "gaussian");
        } else if (!strcmp(argv[i], "--ic-sigma") && i + 1 < argc) { ic_sigma = atof(argv[++i]);
        } else if (!strcmp(argv[i], "--rtol") && i + 1 < argc) { rtol = atof(argv[++i]);
        } else if (!strcmp(argv[i], "--max-iter") && i + 1 < argc) { max_iter = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--device") && i + 1 < argc) { device = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--verify")) { verify_mode = 1;
        } else if (!strcmp(argv[i], "--qrank") || !strcmp(argv[i], "--qblock")) {
            fprintf(stderr, "hybrid quantum coupling (--qrank/--qblock) is not part of this solver\n");
            return 1;
        } else if (argv[i][0] != '-') { outdir = argv[i];
        } else { fprintf(stderr, "unknown option %s\n", argv[i]); usage(prog); return 1; }
    }
    if (N < 1) { fprintf(stderr, "N must be >= 1\n"); return 1; }
    if (fi.level > 0 && (fi.rank < 0 || fi.rank >= 1)) { fprintf(stderr, "--fi-rank must be in [0,1)\n"); return 1; }
    if (fi.level == HS_FI_H) { fprintf(stderr, "level H needs >= 2 ranks and --fi-rank < nprocs-1\n"); return 1; }
    if (fi.level == 4) { fprintf(stderr, "level 4 (handoff transit) needs --qrank --qblock\n"); return 1; }
    if (fi.level > 0 && (fi.bit < 0 || fi.bit > 63)) { fprintf(stderr, "BIT must be in 0..63\n"); return 1; }
    if (fi.level > 0 && fi.level != HS_FI_G && fi.level != HS_FI_R && fi.level < HS_FI_P) {
        fprintf(stderr, "unknown fault level %d\n", fi.level);
        return 1;
    }
    if (fi.level > HS_FI_AP) { fprintf(stderr, "unknown fault level %d\n", fi.level); return 1; }
    if (fi.level > 0 && fi.target < 0) { fprintf(stderr, "TARGET must be >= 0\n"); return 1; }

    const int n_steps = (int)(t_final / dt + 0.5);
    const int nprocs = 1;
    printf("=== Assembly-Free FEM Heat Solver v2 (Backward Euler + Jacobi-PCG) ===\n");
    printf("Grid %d^3 (DOFs %ld)  ranks %d (1D x-decomp, %d cells/rank)\n", N, (long)(N + 1) * (N + 1) * (N + 1),
           nprocs, N / nprocs);
    printf("dt %.4e  t_final %.4e  steps %d  kernel %s  scatter %s  mode %s\n", dt, t_final, n_steps, kname(kernel),
           colored ? "colored" : "atomic", verify_mode ? "VERIFY" : "production");
    fflush(stdout);

    const long long ne = (long long)N * N * N;
    std::vector<double> k(ne), rhoc(ne);
    hs_status st = hs_load_fields(field_prefix, N, k.data(), rhoc.data());
    if (st != HS_OK) { fprintf(stderr, "%s\n", hs_last_error()); return exit_code(st); }
    hs_options opt;
    hs_default_options(&opt);
    opt.N = N; opt.dt = dt; opt.kernel = kernel; opt.scatter = colored ? HS_SCATTER_COLORED : HS_SCATTER_ATOMIC;
    opt.detect = detect; opt.verify = verify_mode; opt.no_source = no_source; opt.ic_mode = ic_mode;
    opt.ic_sigma = ic_sigma; opt.rtol = rtol; opt.max_iter = max_iter; opt.device = device;
    hs_solver* h = nullptr;
    st = hs_create(&opt, k.data(), rhoc.data(), &h);
    if (st != HS_OK) {
        if (st == HS_ERR_MATRIX) printf("%s\n", hs_last_error());
        fprintf(stderr, "%s\n", hs_last_error());
        return exit_code(st);
    }
    double fs[9];
    hs_field_stats(h, fs);
    printf("Reference matrices: M pattern %.1e, sum(M)-V %.1e, K rowsum %.1e, K diag %.1e, symmetry %.1e  -> OK\n",
           fs[4], fs[5], fs[6], fs[7], fs[8]);
    printf("Material: k in [%g, %g] (contrast %.3g), rho*c in [%g, %g]\n", fs[0], fs[1], fs[1] / fs[0], fs[2], fs[3]);
    fflush(stdout);
    ensure_dir(outdir);
    const char* kn = kname(kernel);
    const char* sn = colored ? "colored" : "atomic";
    int rc = 0;

    if (verify_mode) {
        double rel = 0, ms = 0;
        long long tot = 0;
        st = hs_verify(h, n_steps, &rel, &tot, &ms);
        if (st != HS_OK) { fprintf(stderr, "%s\n", hs_last_error()); hs_destroy(h); return exit_code(st); }
        const double t_end = n_steps * dt;
        const double alpha = fs[0] / fs[2];
        printf("VERIFY: N=%d dt=%.4e t_end=%.6e alpha=%g rel_L2_err=%.6e  (%s/%s, %.1f ms, %.1f CG it/step)\n", N, dt,
               t_end, alpha, rel, kn, sn, ms, (double)tot / n_steps);
        std::string p = outdir + "/verify.csv";
        FILE* vf = fopen(p.c_str(), "r");
        const int fresh = (vf == nullptr);
        if (vf) fclose(vf);
        vf = fopen(p.c_str(), "a");
        if (!vf) { fprintf(stderr, "cannot write %s\n", p.c_str()); hs_destroy(h); return 1; }
        if (fresh) fprintf(vf, "N,dt,t_end,nprocs,kernel,scatter,rel_L2_err,solve_ms,avg_cg_iters\n");
        fprintf(vf, "%d,%.6e,%.6e,%d,%s,%s,%.10e,%.3f,%.3f\n", N, dt, t_end, nprocs, kn, sn, rel, ms,
                (double)tot / n_steps);
        fclose(vf);
    } else if (!diag_cg_path.empty()) {
        std::vector<double> rel(max_iter + 1), al(max_iter + 1), be(max_iter + 1);
        double rel0 = 0;
        int it = 0;
        st = hs_diag_cg(h, max_iter, rtol, &rel0, rel.data(), al.data(), be.data(), max_iter + 1, &it);
        if (st != HS_OK) { fprintf(stderr, "%s\n", hs_last_error()); hs_destroy(h); return exit_code(st); }
        FILE* lf = fopen(diag_cg_path.c_str(), "w");
        if (!lf) { fprintf(stderr, "cannot write %s\n", diag_cg_path.c_str()); hs_destroy(h); return 1; }
        fprintf(lf, "iter,rel_residual,alpha,beta\n");
        fprintf(lf, "0,%.10e,,\n", rel0);
        for (int i = 0; i < it && i < max_iter; ++i) fprintf(lf, "%d,%.10e,%.10e,%.10e\n", i + 1, rel[i], al[i], be[i]);
        fclose(lf);
        printf("diag-cg: %d iterations to %g, contrast k_max/k_min=%.3g -> %s\n", it, rtol, fs[1] / fs[0],
               diag_cg_path.c_str());
    } else {
        if (dump_snaps) hs_set_dump(h, outdir.c_str(), tag.c_str());
        const long long Nn = hs_num_nodes(h);
        RunRecords A, B, F;
        std::vector<double> Tclean(Nn), Tfault(Nn);
        A.steps.resize(n_steps); B.steps.resize(n_steps); F.steps.resize(n_steps);
        hs_set_case_tag(h, "cleanA");
        st = hs_run_case(h, n_steps, snap_every, nullptr, reproject, 1, A.steps.data(), Tclean.data(), &A.nonfinite);
        if (st == HS_OK) {
            if (!write_bin(outdir + "/T_final_" + tag + "_clean_rank0.bin", Tclean)) {
                fprintf(stderr, "cannot write %s/T_final_%s_clean_rank0.bin\n", outdir.c_str(), tag.c_str());
                hs_destroy(h);
                return 1;
            }
            hs_set_case_tag(h, "cleanB");
            st = hs_run_case(h, n_steps, snap_every, nullptr, reproject, 0, B.steps.data(), nullptr, &B.nonfinite);
        }
        int on_bnd = -1;
        if (st == HS_OK && fi.level > 0) {
            on_bnd = hs_target_on_boundary(h, &fi);
            hs_set_case_tag(h, "fault");
            st = hs_run_case(h, n_steps, snap_every, &fi, reproject, 0, F.steps.data(), Tfault.data(), &F.nonfinite);
            if (st == HS_OK) write_bin(outdir + "/T_final_" + tag + "_fault_rank0.bin", Tfault);
        }
        if (st != HS_OK) { fprintf(stderr, "%s\n", hs_last_error()); hs_destroy(h); return exit_code(st); }
        for (auto* R : {&A, &B, &F}) {
            R->solve_ms = 0;
            for (auto& s : R->steps) R->solve_ms += s.solve_ms;
        }
        if (fi.level <= 0) F.solve_ms = 0;
        TwinSummary S = summarize(A, B, fi.level > 0 ? &F : nullptr, fi.level, dt, thr_user, detect);
        const RunRecords& rX = fi.level > 0 ? F : A;
        // fi_trace
        std::string tp = outdir + "/fi_trace_" + tag + ".csv";
        FILE* tf = fopen(tp.c_str(), "w");
        if (!tf) { fprintf(stderr, "cannot write %s\n", tp.c_str()); hs_destroy(h); return 1; }
        fprintf(tf, "step,t,E_noise_floor,E_fault,spread_F,cg_A,cg_B,cg_F,d1_abft_A,d1_abft_F,d2_resid_A,d2_resid_F,"
                    "d3_tmin_F,d3_tmax_F,hyb_block_err_A,hyb_block_err_F,hyb_d4_F\n");
        for (int s : S.snap_steps) {
            fprintf(tf, "%d,%.6e,%.10e,%.10e,%.4f,%d,%d,%d", s, s * dt, B.steps[s].E,
                    fi.level > 0 ? F.steps[s].E : 0.0, fi.level > 0 ? F.steps[s].spread : 0.0, A.steps[s].cg_iters,
                    B.steps[s].cg_iters, fi.level > 0 ? F.steps[s].cg_iters : -1);
            if (detect)
                fprintf(tf, ",%.3e,%.3e,%.3e,%.3e,%.6e,%.6e", A.steps[s].d1, rX.steps[s].d1, A.steps[s].d2,
                        rX.steps[s].d2, rX.steps[s].tmin, rX.steps[s].tmax);
            else
                fprintf(tf, ",,,,,,");
            fprintf(tf, ",,,\n");
        }
        fclose(tf);
        double meanA = 0;
        for (auto& s : A.steps) meanA += s.cg_iters;
        meanA /= std::max<size_t>(1, A.steps.size());
        std::string sp = outdir + "/fi_summary_" + tag + ".csv";
        FILE* sf = fopen(sp.c_str(), "w");
        if (!sf) { fprintf(stderr, "cannot write %s\n", sp.c_str()); hs_destroy(h); return 1; }
        fprintf(sf, "tag,N,dt,n_steps,nprocs,kernel,scatter,reproject_bc,kmin,kmax,rhocmin,rhocmax,"
                    "fi_level,fi_rank,fi_step,fi_target,fi_bit,target_on_boundary,"
                    "E_floor_max,E_floor_final,E_fault_max,step_at_max,E_fault_int,E_fault_final,"
                    "thr,iters_delta_max,mean_cg_iters_A,solve_ms_A,solve_ms_B,solve_ms_F,class,spread_at_max,spread_final,"
                    "detect,d1_first,d2_first,d3_first,d1_max_F,d2_max_F,d1_max_A,d2_max_A,detected_by,"
                    "hybrid,hyb_block_err_max_A,hyb_block_err_max_F,d4_first_F\n");
        fprintf(sf, "%s,%d,%.3e,%d,%d,%s,%s,%d,%g,%g,%g,%g,%d,%d,%d,%ld,%d,%d,"
                    "%.6e,%.6e,%.6e,%d,%.6e,%.6e,%.3e,%d,%.2f,%.3f,%.3f,%.3f,%s",
                tag.c_str(), N, dt, n_steps, nprocs, kn, sn, reproject, fs[0], fs[1], fs[2], fs[3], fi.level, fi.rank,
                fi.step, (long)fi.target, fi.bit, on_bnd, S.Efl_max, S.Efl_final, S.Efa_max, S.step_max, S.Efa_int,
                S.Efa_final, S.thr, S.iters_delta_max, meanA, A.solve_ms, B.solve_ms, F.solve_ms, S.cls);
        fprintf(sf, ",%.4f,%.4f", S.spread_at_max, S.spread_final);
        fprintf(sf, ",%d,%d,%d,%d,%.3e,%.3e,%.3e,%.3e,%s", detect, S.detX.d1_first, S.detX.d2_first, S.detX.d3_first,
                S.detX.d1_max, S.detX.d2_max, S.detA.d1_max, S.detA.d2_max, S.by.c_str());
        fprintf(sf, ",%d,%.3e,%.3e,%d\n", 0, 0.0, 0.0, -1);
        fclose(sf);
        if (detect)
            printf("detectors    D1 first %d (max %.2e)  D2 first %d (max %.2e)  D3 first %d  -> %s   [clean A: D1 %.2e D2 %.2e]\n",
                   S.detX.d1_first, S.detX.d1_max, S.detX.d2_first, S.detX.d2_max, S.detX.d3_first, S.by.c_str(),
                   S.detA.d1_max, S.detA.d2_max);
        printf("\n=== Done (%s) ===\n", tag.c_str());
        printf("solve wall A/B/F (ms): %.1f / %.1f / %.1f   mean CG iters A: %.2f\n", A.solve_ms, B.solve_ms,
               F.solve_ms, meanA);
        printf("noise floor  max %.3e  final %.3e\n", S.Efl_max, S.Efl_final);
        if (fi.level > 0)
            printf("fault        max %.3e @step %d  int %.3e  final %.3e  iters+%d  bnd %d  -> %s\n", S.Efa_max,
                   S.step_max, S.Efa_int, S.Efa_final, S.iters_delta_max, on_bnd, S.cls);
        std::string mp = outdir + "/meta_" + tag + ".txt";
        FILE* mf = fopen(mp.c_str(), "w");
        if (mf) {
            fprintf(mf, "N %d\nnprocs %d\ndt %g\nn_steps %d\nfield %s\nkernel %s\nscatter %s\n", N, nprocs, dt, n_steps,
                    field_prefix, kn, sn);
            fclose(mf);
        }
    }
    hs_destroy(h);
    return rc;
}
