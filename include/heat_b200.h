/* heat_b200.h -- C ABI of the B200 transient-heat PCG library (libheat_b200.so).
 *
 * One opaque solver handle per problem instance (grid, material field, time
 * step, operator options).  Every entry point returns an hs_status; nothing
 * aborts the process.  The CLI (hs_cli_main) maps the codes onto the exit
 * codes of the reference solver.
 *
 * The reference, src/heat_solver_het.cu, has no library API: its operator is
 * a C++ class (HeatOperator, het.cu:618-989) plus a free PCG function
 * (pcg_solve, het.cu:994-1039) driven by a CLI (main, het.cu:1355-1629).
 * Each declaration below names the reference code it replaces.
 *
 * Vector arguments marked "device" are device pointers to (N+1)^3 float64
 * node values in the reference's node order n = ix*(N+1)^2 + iy*(N+1) + iz
 * (het.cu:202-205).  Element fields are N^3 float64 in element order
 * e = ix*N^2 + iy*N + iz (het.cu:289-291, scripts/gen_field.py:5-6).
 *
 * Threading: a handle is used by one host thread at a time; handles are
 * independent and each owns its own CUDA stream.
 */
#ifndef HEAT_B200_H
#define HEAT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define HS_API_VERSION 2

typedef struct hs_solver hs_solver;

typedef enum hs_status {
    HS_OK = 0,
    HS_ERR_ARG = 1,      /* bad argument, bad field value; reference: MPI_Abort(.., 1) */
    HS_ERR_MATRIX = 2,   /* reference-matrix self-check failed; reference: MPI_Abort(.., 2), het.cu:705 */
    HS_ERR_IO = 3,       /* missing or short field file, unwritable output (exit code 1 in the CLI) */
    HS_ERR_CUDA = 4,     /* CUDA error or no device (exit code 1 in the CLI) */
    HS_ERR_STATE = 5     /* call not valid for this handle's options */
} hs_status;

/* element operator form (--kernel) */
enum {
    HS_KERNEL_FAST = 0,   /* rhoc*M^ + dt*k*K^ with the Gauss-built 8x8 matrices, het.cu:340-349 */
    HS_KERNEL_GAUSS = 1,  /* 2x2x2 Gauss integration per call, het.cu:310-338 */
    HS_KERNEL_WHT = 2     /* same element matrix through its exact tensor-product
                             (Walsh-Hadamard) structure; no reference counterpart */
};
/* scatter (--scatter) */
enum { HS_SCATTER_ATOMIC = 0, HS_SCATTER_COLORED = 1 };
/* fault-injection levels (--fi LEVEL ...) */
enum {
    HS_FI_NONE = 0,
    HS_FI_G = 1,   /* T[target % Nn] before the RHS of the step, het.cu:1130-1135 */
    HS_FI_R = 2,   /* ye[0] of element `target` in the step's first matvec, het.cu:369-374 */
    HS_FI_H = 3,   /* host halo buffer; needs >= 2 ranks, rejected here (het.cu:1419-1422) */
    HS_FI_P = 5,   /* PCG search direction p[target % Nn] at loop iteration `iter` (new) */
    HS_FI_RV = 6,  /* PCG residual r[target % Nn] after its update at iteration `iter` (new) */
    HS_FI_AP = 7   /* operator output Ap[target % Nn] at iteration `iter` (new) */
};

/* Solver options; hs_default_options fills the reference defaults
 * (het.cu:1385-1391: kernel fast, scatter atomic, tol 1e-8, 500 iterations). */
typedef struct hs_options {
    int N;              /* elements per axis on [0,1]^3 */
    double dt;          /* implicit-Euler step */
    int kernel;         /* HS_KERNEL_* */
    int scatter;        /* HS_SCATTER_* */
    int detect;         /* D1/D2/D3 detectors (--detect) */
    int verify;         /* eigenmode check mode: source off (--verify) */
    int no_source;      /* --no-source */
    int ic_mode;        /* 0 zero, 1 Gaussian bump (--ic) */
    double ic_sigma;    /* Gaussian IC width, reference 0.1 (het.cu:566) (--ic-sigma, new) */
    double rtol;        /* PCG relative tolerance, reference 1e-8 (het.cu:1162) (--rtol, new) */
    int max_iter;       /* PCG iteration cap, reference 500 */
    int device;         /* CUDA device ordinal */
} hs_options;

typedef struct hs_fi_spec {
    int level;          /* HS_FI_* */
    int step;           /* time step at which it fires */
    long long target;   /* node (G, P, RV, AP: taken modulo Nn) or element (R) index */
    int bit;            /* 0..63, XOR on the IEEE-754 word */
    int iter;           /* PCG loop iteration (P, RV, AP) */
    int rank;           /* --fi-rank; only 0 is valid on one device */
} hs_fi_spec;

/* per-step record of one trajectory (RunResult, het.cu:1082-1096) */
typedef struct hs_step_record {
    int cg_iters;
    int snap;           /* 1 if the step was a snapshot step */
    double d1, d2, tmin, tmax;   /* detectors (0 when detect is off) */
    double E, spread;   /* vs the reference trajectory at snapshot steps, else -1 / 0 */
    double solve_ms;    /* build_rhs + PCG (+ reprojection) device time of the step */
} hs_step_record;

/* canonical reduction orders of an N-element grid: the operator's slab tile
 * (planes cx, rows ty, columns tz; rt threads of bpt positions each, halo
 * included) and the flat order's nodes per thread kf */
typedef struct hs_layout_info { int cx, ty, tz, rt, bpt, kf; } hs_layout_info;

void        hs_default_options(hs_options* opt);
const char* hs_last_error(void);               /* message of the last failing call on this thread */
int         hs_api_version(void);
void        hs_get_layout(int N, hs_layout_info* out);
/* Gaussian initial condition of width sigma centred in the cube, the
 * reference's --ic gaussian with a sigma parameter (het.cu:556-568), into
 * T_host ((N+1)^3 doubles). */
hs_status   hs_gaussian_ic(int N, double sigma, double* T_host);

/* Read <prefix>_k.bin and <prefix>_rhoc.bin (N^3 float64 each) into host
 * buffers; rejects short files and non-positive/NaN values
 * (HeatOperator::load_fields, het.cu:711-753). */
hs_status hs_load_fields(const char* prefix, int N, double* k_out, double* rhoc_out);

/* Build the operator: reference matrices + self-check, Jacobi diagonal,
 * source vector, ABFT weights (HeatOperator::setup, het.cu:756-816, 940-953).
 * k/rhoc are host arrays of N^3 values. */
hs_status hs_create(const hs_options* opt, const double* k_host, const double* rhoc_host, hs_solver** out);
void      hs_destroy(hs_solver* s);
long long hs_num_nodes(const hs_solver* s);
/* kmin, kmax, rhocmin, rhocmax and the five reference-matrix check errors */
hs_status hs_field_stats(const hs_solver* s, double out9[9]);

/* y = (M + dt_eff K) x [+ Dirichlet projection] (apply_operator, het.cu:885-921).
 * allow_fi: a fault armed by hs_arm_fi (level R) fires in this call.
 * abft_rel (nullable): D1 relative checksum error when the handle has
 * detect on and project != 0, else -1. x, y: device, not overlapping
 * (HS_ERR_ARG otherwise). */
hs_status hs_apply(hs_solver* s, const double* x, double* y, double dt_eff, int allow_fi, int project,
                   double* abft_rel);
/* z = r / diag (apply_preconditioner, het.cu:957-960). device. */
hs_status hs_precond(hs_solver* s, const double* r, double* z);
/* b = M T + dt F (build_rhs, het.cu:963-971). device. */
hs_status hs_build_rhs(hs_solver* s, const double* T, double* b);
/* fixed-order dot product over all nodes (HeatOperator::dot, het.cu:973-987). device. */
hs_status hs_dot(hs_solver* s, const double* x, const double* y, double* out);
/* Jacobi-PCG from x (pcg_solve, het.cu:994-1039), device resident; *iters
 * as the reference returns it. b, x: device. */
hs_status hs_pcg(hs_solver* s, const double* b, double* x, int max_iter, double tol, int* iters);
/* arm a level-R or vector fault for the next hs_apply(allow_fi=1) / hs_pcg */
hs_status hs_arm_fi(hs_solver* s, const hs_fi_spec* fi);

/* One full trajectory from the initial condition (run_case, het.cu:1107-1259).
 * keep_reference != 0: this run is the reference (its snapshots are kept on
 * the device); otherwise E(t) and spread are measured against the kept
 * reference and D3 against its per-step range.  T_final_host (nullable, Nn
 * values) receives the final field.  out: n_steps records. */
hs_status hs_run_case(hs_solver* s, int n_steps, int snap_every, const hs_fi_spec* fi, int reproject,
                      int keep_reference, hs_step_record* out, double* T_final_host, int* nonfinite);

/* --verify (run_verify, het.cu:1293-1338): homogeneous field required. */
hs_status hs_verify(hs_solver* s, int n_steps, double* rel_err, long long* total_iters, double* ms);

/* End-to-end solve with host buffers: copies T0 in, runs n_steps implicit-
 * Euler steps (build_rhs + PCG), copies the field back. */
hs_status hs_solve_host(hs_solver* s, const double* T0_host, double* T_host, int n_steps, long long* total_iters,
                        double* device_ms);

/* Advance the device-resident field n_steps implicit-Euler steps (build_rhs +
 * PCG each, no host traffic); from_ic != 0 restarts from the initial
 * condition (kept on the device) first.  Device time and CG iterations.
 * hs_set_field / hs_get_field move the field (host buffers). */
hs_status hs_advance(hs_solver* s, int n_steps, int from_ic, long long* total_iters, double* device_ms);
hs_status hs_set_field(hs_solver* s, const double* T_host);
hs_status hs_get_field(hs_solver* s, double* T_host);

/* Per-launch device time of one kernel of the hot path, averaged over reps
 * launches with the L2 cache flushed before each (which: 0 the PCG operator
 * kernel p = z + beta p, Ap = A p with its p.Ap and checksum partials; 1 the
 * PCG vector update; 2 a plain projected apply y = A x).  Leaves the solver
 * state to be re-initialised by the next run. */
hs_status hs_time_kernel(hs_solver* s, int which, int reps, double* ms_per_launch);

/* --diag-cg (het.cu:1491-1504): one build_rhs + PCG from the initial
 * condition, logging the relative residual before the loop (rel0) and
 * rel/alpha/beta per iteration (up to cap entries). */
hs_status hs_diag_cg(hs_solver* s, int max_iter, double tol, double* rel0, double* rel, double* alpha, double* beta,
                     int cap, int* iters);

/* --dump-snaps (het.cu:1239-1245): write snap_<tag>_<case>_<step>_rank0.bin
 * into dir at every snapshot step of later hs_run_case calls (dir null: off). */
hs_status hs_set_dump(hs_solver* s, const char* dir, const char* tag);
hs_status hs_set_case_tag(hs_solver* s, const char* case_tag);

/* Is the fault target on the Dirichlet boundary? (target_on_boundary,
 * het.cu:1272-1290); 1, 0, or -1 without a fault. */
int hs_target_on_boundary(const hs_solver* s, const hs_fi_spec* fi);

/* Twin-run summary and fault class (het.cu:1506-1542, 1585-1595) from the
 * per-step records of cleanA, cleanB and the fault run (F null without a
 * fault).  Host-only arithmetic. */
typedef struct hs_twin_summary {
    double E_floor_max, E_floor_final, E_fault_max, E_fault_int, E_fault_final, thr;
    double spread_at_max, spread_final;
    int step_at_max, iters_delta_max;
    int d1_first, d2_first, d3_first, pad;
    double d1_max, d2_max, d1_max_A, d2_max_A;
    char cls[16];
    char detected_by[16];
} hs_twin_summary;
hs_status hs_classify(const hs_step_record* A, const hs_step_record* B, const hs_step_record* F, int n_steps,
                      int fi_level, int F_nonfinite, double dt, double thr_user, int detect, hs_twin_summary* out);

/* One flip of a fault-injection campaign and the twin-run outcome. */
typedef struct hs_flip_record {
    int step;                 /* time step of the flip */
    int iter;                 /* PCG iteration of the flip */
    int level;                /* HS_FI_P (p after formation), HS_FI_RV (r after its update), HS_FI_AP (Ap) */
    int bit;                  /* 0..63 */
    long long idx;            /* vector entry, 0..(N+1)^3-1 */
    int nonfinite;            /* the faulted run produced a non-finite field */
    int iters_total_delta;    /* faulted minus clean CG iterations over the trajectory */
    hs_twin_summary summary;  /* hs_classify(clean, clean twin, faulted) */
} hs_flip_record;

/* Seeded single-bit-flip campaign over one trajectory.  No counterpart in the
 * reference, which runs one twin-run process per flip (het.cu:1506-1620).
 * Runs the clean trajectory (kept as the reference, with its field at the
 * start of every step), its clean twin, then n_flips faulted trajectories,
 * each resumed at its flip step from the kept clean field (colored scatter
 * only).  Flip sites come from std::mt19937_64(seed), each draw the
 * generator's next output modulo its range, in this order: a global CG
 * iteration over the clean run's total (mapped to step and iteration), a
 * vector among the levels in vec_mask (bit 0 p, bit 1 r, bit 2 Ap), a node
 * entry, a bit in 0..63.  clean_out (nullable): the clean run's n_steps
 * records.  Device memory: n_steps extra fields. */
hs_status hs_campaign(hs_solver* s, int n_steps, int snap_every, int n_flips, unsigned long long seed, int vec_mask,
                      hs_step_record* clean_out, hs_flip_record* out);

/* ---- batched mixed-precision solves (no counterpart in the reference) ----
 * Many independent solves live in one handle and advance together, one
 * implicit-Euler step of every instance per hs_batch_step (one CUDA-graph
 * launch).  Each step solves (M + dt K) T = M T_old by defect correction:
 * FP64 residual r = b - A T with the ABFT checksum, an FP32 Jacobi-PCG solve
 * of A d = r (FP32 operator and preconditioner, FP64 dot products) to the
 * relative tolerance max(inner_tol, rtol ||b|| / (2 ||r||)), T += d in FP64
 * at the interior nodes (a correction whose inner solve went non-finite is
 * discarded and re-solved), until ||b - A T|| / ||b|| < rtol (the true
 * residual) or max_outer corrections.  Element form wht, deterministic
 * scatter, Dirichlet T = 0, no source.  Instances can be added and removed
 * between steps (continuous batching). */
typedef struct hs_batch hs_batch;
typedef struct hs_batch_options {
    double rtol;          /* outer tolerance on ||b - A T|| / ||b||, e.g. 1e-8 */
    double inner_tol;     /* FP32 inner PCG relative tolerance, e.g. 1e-4 */
    int max_outer;        /* corrections per step */
    int max_inner;        /* inner PCG iterations per correction */
    int detect;           /* ABFT checksum on every operator apply */
    int tile_planes;      /* operator tiles span min(N+1, tile_planes) planes; 0: a depth set by N
                             alone (the instance by itself fills the GPU, within 8..32 planes) */
    int device;
    int extrapolate;      /* start each step (after the first) from 2 T - T_prev instead of T */
} hs_batch_options;
typedef struct hs_batch_inst_info {
    int N, steps_done, steps_left, pad;
    long long inner_iters, outer_iters, applies32, applies64, tiles;
    int fault_fired;      /* an armed vector fault has fired */
    int stalls;           /* steps that ended at max_outer without reaching rtol */
    int inner_faults;     /* inner solves that went non-finite (correction discarded) */
    int pad2;
    double rel_residual;  /* last true relative residual */
    double d1_max64;      /* largest D1 of the FP64 applies */
    double d1_max32;      /* largest D1 of the FP32 applies (their noise floor when clean) */
} hs_batch_inst_info;
void      hs_batch_default_options(hs_batch_options* o);
hs_status hs_batch_create(const hs_batch_options* opt, hs_batch** out);
void      hs_batch_destroy(hs_batch* b);
/* k, rhoc: N^3 host arrays; T0: (N+1)^3 host field or null (zero); the
 * instance takes n_steps steps.  Sets *slot. */
hs_status hs_batch_add(hs_batch* b, int N, double dt, const double* k, const double* rhoc, const double* T0,
                       int n_steps, int* slot);
/* As hs_batch_add, with the instance's conductivity generated on the device:
 * a periodic Gaussian field of covariance exp(-r^2/L^2) (L in domain units),
 * standardised, k = exp(mu + sigma g), rho*c = rhoc.  The reference draws
 * these fields on the host with scripts/gen_field.py:29-61 (NumPy's random
 * stream and FFT); this generator has the same law but its own counter-based
 * random stream (see hs_field_lognormal), so the field is a fixed function of
 * (N, seed, L, mu, sigma) and is not the reference file bit for bit.
 * No host field crosses the bus; the generation runs on the add stream. */
hs_status hs_batch_add_lognormal(hs_batch* b, int N, double dt, double mu, double sigma, double L,
                                 unsigned long long seed, double rhoc, const double* T0, int n_steps, int* slot);
/* level-G fault: flip bit `bit` of T[idx % (N+1)^3] before the instance's step `step` */
hs_status hs_batch_arm_flip(hs_batch* b, int slot, int step, long long idx, int bit);
/* fault in an FP32 inner vector: level HS_FI_P (p after formation), HS_FI_RV
 * (r after its update) or HS_FI_AP (Ap after projection), entry idx, bit 0..31,
 * in step `step`, correction `outer` (1-based), inner iteration `iter` */
typedef struct hs_batch_fault { int level, step, outer, iter; long long idx; int bit, pad; } hs_batch_fault;
hs_status hs_batch_arm_fault(hs_batch* b, int slot, const hs_batch_fault* f);
hs_status hs_batch_remove(hs_batch* b, int slot);
/* one step of every instance with steps left; device time of the launch */
hs_status hs_batch_step(hs_batch* b, int* n_active, double* device_ms);
/* hs_batch_step in two halves, so that the host can admit instances while the
 * step runs: _begin launches the step of every instance with steps left and
 * returns at once; _end waits for it (*n_stepped instances, device time).
 * Between them hs_batch_add sets up new instances on a stream of its own (they
 * join at the next step), and hs_batch_remove frees an instance after the step
 * (its slot is reused only once the step has ended).  A second _begin before
 * _end is an error. */
hs_status hs_batch_step_begin(hs_batch* b, int* n_active);
hs_status hs_batch_step_end(hs_batch* b, int* n_stepped, double* device_ms);
hs_status hs_batch_info(hs_batch* b, int slot, hs_batch_inst_info* out);
hs_status hs_batch_get_field(hs_batch* b, int slot, double* T_host);

/* x.y over the (N+1)^3 nodes of an N-element grid without allocating any
 * device memory.  No counterpart in the reference.  For callers that cannot
 * call cudaMalloc (a host application that owns the device-memory budget, a
 * path that must not take the allocator's locks): the result equals hs_dot's
 * bit for bit (same fixed reduction order), but the per-block partial sums
 * live in a static device array of 131072 doubles (1 MiB, held by every GPU
 * that loads the library until exit).  The reduction stores two values per
 * block of 512 nodes, so the array serves 65536 blocks: N <= 321; larger
 * grids return HS_ERR_ARG before anything is launched.  x, y and out (one
 * double) are device pointers on the current device; the work is enqueued on
 * the default stream and *out is valid once that stream has completed.  The
 * first call on a device looks up the array's device address and should come
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race.  Do not call it on a device after cudaDeviceReset (the
 * cached address of the array is then stale). */
hs_status hs_dot_noalloc(int N, const double* x, const double* y, double* out);

/* A lognormal conductivity field of the reference generator's law
 * (scripts/gen_field.py:29-61: white noise filtered to the periodic
 * covariance exp(-r^2/L^2), standardised, k = exp(mu + sigma g)) generated on
 * the current device into k_dev and rhoc_dev (N^3 doubles each, device;
 * rhoc_dev is set to rhoc).  The filter is the real-space Gaussian kernel of
 * the reference's Fourier filter, applied as three periodic 1-D passes; the
 * noise is SplitMix64 of (seed, element) through Box-Muller.  Deterministic
 * for given arguments; synchronous on the default stream. */
hs_status hs_field_lognormal(int N, double mu, double sigma, double L, unsigned long long seed, double rhoc,
                             double* k_dev, double* rhoc_dev);

/* The reference solver's command line (het.cu:1340-1350, 1380-1433) with its
 * output files; returns the process exit code. */
int hs_cli_main(int argc, char** argv);

#ifdef __cplusplus
}
#endif
#endif /* HEAT_B200_H */
