// hs_solver.cu -- solver handle, operator calls, device-resident PCG under a
// CUDA graph with a conditional while node, trajectories (libheat_b200).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/heat_b200.h"
#include "hs_host.h"
#include "hs_kernels.cuh"

using namespace hs;

namespace hs {
static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
}  // namespace hs

#define HS_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess) {                                                          \
            hs::set_error(std::string("CUDA error: ") + cudaGetErrorString(_e) + " at " + \
                          __FILE__ + ":" + std::to_string(__LINE__));                    \
            return HS_ERR_CUDA;                                                           \
        }                                                                                 \
    } while (0)

namespace {

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr; n = count;
        return count ? cudaMalloc(&p, count * sizeof(T)) : cudaSuccess;
    }
    ~DevBuf() { if (p) cudaFree(p); }
};

// CUDA events released on every return path
struct Events {
    std::vector<cudaEvent_t> e;
    cudaError_t create(size_t n) {
        e.assign(n, nullptr);
        for (auto& v : e) {
            const cudaError_t r = cudaEventCreate(&v);
            if (r != cudaSuccess) { v = nullptr; return r; }
        }
        return cudaSuccess;
    }
    cudaEvent_t operator[](size_t i) const { return e[i]; }
    ~Events() { for (auto v : e) if (v) cudaEventDestroy(v); }
};

inline int grid_for(long long n, int threads, int cap = 148 * 16) {
    long long g = (n + threads - 1) / threads;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

struct hs_solver {
    hs_options opt{};
    int N = 0;
    long long Nn = 0, Ne = 0;
    Part part{};
    RefMatrices mats{};
    ElemConsts ec{};
    double kmin = 0, kmax = 0, rhocmin = 0, rhocmax = 0;
    cudaStream_t s = nullptr;

    DevBuf<double> rhoc, kc, gtab;
    DevBuf<double2> coef;               // (rho*c, k) per element, the operator kernel's layout
    DevBuf<double> diag, F, wM, wA;
    DevBuf<double> T, b, r, z, p0, p1, Ap;
    DevBuf<double> partials;            // operator tiles (and the standalone reductions)
    DevBuf<double> upart;               // PCG vector update: run sums (RUN order)
    int n_sm = 148;
    DevBuf<unsigned> ticket;
    DevBuf<DevState> st;
    DevBuf<double> red;                 // standalone reduction outputs
    DevBuf<unsigned long long> sp;      // spread: [gmax bits, count]
    DevBuf<double> logs;                // diag-cg log buffers (3 * cap)
    DevBuf<double> T0;                  // initial condition kept on the device (hs_advance)
    bool has_F = false;

    // PCG graphs built on first use: [0] step (RHS + PCG), [1] PCG only
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};

    // pending user-armed fault for hs_apply / hs_pcg
    hs_fi_spec pending{};
    bool pending_set = false;

    // reference trajectory (kept by a keep_reference run)
    std::vector<double*> ref_snaps;
    std::vector<double> ref_tmin, ref_tmax;
    int ref_nsteps = 0, ref_snap_every = -1;

    // --dump-snaps
    std::string dump_dir, dump_tag, case_tag;

    ~hs_solver() {
        for (int i = 0; i < 2; ++i) {
            if (gexec[i]) cudaGraphExecDestroy(gexec[i]);
            if (graph[i]) cudaGraphDestroy(graph[i]);
        }
        for (double* q : ref_snaps) cudaFree(q);
        if (s) cudaStreamDestroy(s);
    }
};

namespace {

hs_status sync_state_config(hs_solver* h, int max_iter, double tol) {
    DevState hs{};
    std::memset(&hs, 0, sizeof(hs));
    HS_CUDA(cudaMemcpyAsync(&hs, h->st.p, sizeof(DevState), cudaMemcpyDeviceToHost, h->s));
    HS_CUDA(cudaStreamSynchronize(h->s));
    hs.max_iter = max_iter;
    hs.tol = tol;
    HS_CUDA(cudaMemcpyAsync(h->st.p, &hs, sizeof(DevState), cudaMemcpyHostToDevice, h->s));
    HS_CUDA(cudaStreamSynchronize(h->s));
    return HS_OK;
}

int nblocks(const hs_solver* h) { return (int)h->part.nblk; }

// ---- operator launches -------------------------------------------------------------
template <int FORM>
bool set_smem_form() {
    return cudaFuncSetAttribute(k_apply_slab<FORM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSlabSmem) == cudaSuccess &&
           cudaFuncSetAttribute(k_apply_slab<FORM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSlabSmem) == cudaSuccess;
}
bool set_smem_attributes() {
    static bool done = false, ok = true;
    if (done) return ok;
    done = true;
    ok = set_smem_form<FORM_WHT>() && set_smem_form<FORM_FAST>() && set_smem_form<FORM_GAUSS>();
    return ok;
}

// Launch with programmatic stream serialization when pdl is set: the kernel's
// CTAs may be scheduled while the previous kernel in the stream finishes, and
// wait (pdl_wait) before reading what it wrote.  Used between the kernels of
// the PCG loop, where it hides the launch gap.
template <typename... KArgs, typename... Args>
void launch_k(bool pdl, void (*k)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, args...);
}

template <int FORM>
void launch_slab(hs_solver* h, const ApplyArgs& a, bool pdl) {
    const int g = (int)h->part.ntiles;
    if (a.role == ROLE_LOOP) launch_k(pdl, k_apply_slab<FORM, true>, g, ST, kSlabSmem, h->s, a);
    else k_apply_slab<FORM, false><<<g, ST, kSlabSmem, h->s>>>(a);
}
void launch_colored(hs_solver* h, const ApplyArgs& a, bool pdl) {
    switch (h->opt.kernel) {
        case HS_KERNEL_WHT: launch_slab<FORM_WHT>(h, a, pdl); break;
        case HS_KERNEL_GAUSS: launch_slab<FORM_GAUSS>(h, a, pdl); break;
        default: launch_slab<FORM_FAST>(h, a, pdl); break;
    }
}
void launch_nodes(hs_solver* h, const GenArgs& a) {
    const int g = grid_for(h->Nn, RT, 1 << 30);
    switch (h->opt.kernel) {
        case HS_KERNEL_WHT: k_apply_nodes<FORM_WHT><<<g, RT, 0, h->s>>>(a); break;
        case HS_KERNEL_GAUSS: k_apply_nodes<FORM_GAUSS><<<g, RT, 0, h->s>>>(a); break;
        default: k_apply_nodes<FORM_FAST><<<g, RT, 0, h->s>>>(a); break;
    }
}
void launch_atomic(hs_solver* h, const AtomArgs& a) {
    const int N = h->N;
    const int g = ((N + AB_X - 1) / AB_X) * ((N + AB_Y - 1) / AB_Y) * ((N + AB_Z - 1) / AB_Z);
    switch (h->opt.kernel) {
        case HS_KERNEL_WHT: k_apply_atomic<FORM_WHT><<<g, RT, 0, h->s>>>(a); break;
        case HS_KERNEL_GAUSS: k_apply_atomic<FORM_GAUSS><<<g, RT, 0, h->s>>>(a); break;
        default: k_apply_atomic<FORM_FAST><<<g, RT, 0, h->s>>>(a); break;
    }
}

// Projected operator application y = A x (or the LOOP form p = z + beta p,
// Ap = A p).  Colored: one fused kernel.  Atomic: zero, element scatter with
// atomics, then projection + partials on the canonical partition.
void apply_projected(hs_solver* h, int role, const double* x, double* y, double dt_eff, bool d1,
                     const double* w, const double* F, double dtF, bool pdl = false) {
    if (h->opt.scatter == HS_SCATTER_COLORED) {
        ApplyArgs a{};
        a.part = h->part;
        a.N = h->N; a.role = role; a.dt_eff = dt_eff;
        a.x = x; a.z = h->z.p; a.pbuf0 = h->p0.p; a.pbuf1 = h->p1.p;
        a.y = y; a.coef = h->coef.p; a.w = w; a.F = F; a.dtF = dtF;
        a.d1 = d1 ? 1 : 0;
        a.partials = h->partials.p; a.st = h->st.p; a.ec = h->ec;
        launch_colored(h, a, pdl);
        // the loop role's reductions are finished by the vector update (k_update)
        if (role != ROLE_LOOP && d1) {
            FinalApplyArgs fa{h->partials.p, h->part.nblk, h->st.p, role, 1};
            k_final_apply<<<1, RT, 0, h->s>>>(fa);
        }
        return;
    }
    if (role == ROLE_LOOP) {
        FormPArgs fp{h->Nn, h->z.p, h->p0.p, h->p1.p, h->st.p};
        k_form_p<<<grid_for(h->Nn, RT), RT, 0, h->s>>>(fp);
    }
    k_zero<<<grid_for(h->Nn, RT), RT, 0, h->s>>>(h->Nn, y);
    AtomArgs aa{};
    aa.N = h->N; aa.role = role; aa.dt_eff = dt_eff; aa.x = x; aa.pbuf0 = h->p0.p; aa.pbuf1 = h->p1.p;
    aa.y = y; aa.rhoc = h->rhoc.p; aa.kc = h->kc.p; aa.st = h->st.p; aa.ec = h->ec;
    launch_atomic(h, aa);
    FinishArgs f{};
    f.part = h->part;
    f.N = h->N; f.role = role; f.d1 = d1 ? 1 : 0; f.p = x; f.pbuf0 = h->p0.p; f.pbuf1 = h->p1.p;
    f.y = y; f.w = w; f.F = F; f.dtF = dtF;
    f.partials = h->partials.p; f.ticket = h->ticket.p; f.st = h->st.p;
    k_finish_atomic<<<nblocks(h), ST, 0, h->s>>>(f);
    if (role != ROLE_LOOP && d1) {
        FinalApplyArgs fa{h->partials.p, h->part.nblk, h->st.p, role, 1};
        k_final_apply<<<1, RT, 0, h->s>>>(fa);
    }
}

void launch_update(hs_solver* h, int role, bool use_cond, cudaGraphConditionalHandle cond = 0, bool pdl = false) {
    UpdateArgs u{};
    u.Nn = h->Nn; u.nflat = h->part.nflat; u.role = role; u.x = h->T.p; u.b = h->b.p; u.r = h->r.p; u.z = h->z.p; u.Ap = h->Ap.p;
    u.d = h->diag.p; u.pbuf0 = h->p0.p; u.pbuf1 = h->p1.p; u.partials = h->upart.p; u.ticket = h->ticket.p;
    u.st = h->st.p; u.cond = cond; u.use_cond = 0;
    u.d1 = h->opt.detect != 0; u.apart = h->partials.p; u.nblk = h->part.nblk;
    u.cond = cond; u.use_cond = use_cond ? 1 : 0;
    // one CTA per run of the RUN order (one resident wave on B200)
    launch_k(pdl, k_update, (int)std::min<long long>(h->part.nflat, UPD_SLOTS), RT, 0, h->s, u);
}

// the solution update the loop still owes (x += alpha p of an even last iteration)
void launch_update_finish(hs_solver* h) {
    k_update_finish<<<grid_for(h->Nn, RT), RT, 0, h->s>>>(h->Nn, h->T.p, h->p0.p, h->p1.p, h->st.p);
}

void launch_reduce(hs_solver* h, int kind, const double* a, const double* b, double* out) {
    RedArgs r{h->Nn, h->part.nflat, h->N, kind, a, b, h->partials.p, h->ticket.p, out};
    k_reduce<<<(int)h->part.nflat, RT, 0, h->s>>>(r);
    k_final_reduce<<<1, RT, 0, h->s>>>(h->partials.p, h->part.nflat, out);
}

// RHS + first matvec + PCG prologue (stream order on h->s)
void enqueue_pcg_prologue(hs_solver* h, bool with_rhs) {
    const bool det = h->opt.detect != 0;
    if (with_rhs) {
        const bool src = !h->opt.verify && !h->opt.no_source && h->has_F;
        apply_projected(h, ROLE_RHS, h->T.p, h->b.p, 0.0, det, h->wM.p, src ? h->F.p : nullptr, h->opt.dt);
    }
    apply_projected(h, ROLE_X0, h->T.p, h->Ap.p, h->opt.dt, det, h->wA.p, nullptr, 0.0);
    launch_update(h, UPD_PRE, false);
}

// HS_GRAPH=0 in the environment launches the PCG loop directly from the host
// (chunks of iterations, the device "done" flag read back between chunks)
// instead of through the graph's while node: profilers cannot attribute
// kernels that run inside a conditional graph node.
// HS_PDL=1 launches the PCG loop's kernels with programmatic dependent launch
// (the next kernel's CTAs are scheduled while the previous one drains).  Off
// by default: on B200 it measured no gain (N=128: 72.4 against 71.9 us per CG
// iteration; N=256: 447 against 441 us).
bool pdl_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("HS_PDL");
        v = (e && e[0] == '1') ? 1 : 0;
    }
    return v == 1;
}

bool graphs_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("HS_GRAPH");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

// build a graph: [rhs] + x0 matvec + prologue, then while(!done){ (K1; K2) x kLoopUnroll }.
// Four iterations per pass of the while body spread the node's relaunch over
// them (N=128: 70.6 -> 67.8 us per CG iteration); a solve that ends mid-pass
// launches at most three iterations' kernels that return at once.
constexpr int kLoopUnroll = 4;
hs_status build_graph(hs_solver* h, int which) {
    if (h->gexec[which] || !graphs_enabled()) return HS_OK;
    const bool with_rhs = which == 0;
    cudaGraph_t g;
    HS_CUDA(cudaGraphCreate(&g, 0));
    cudaGraph_t pre;
    HS_CUDA(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    enqueue_pcg_prologue(h, with_rhs);
    HS_CUDA(cudaStreamEndCapture(h->s, &pre));
    cudaGraphNode_t n_pre;
    HS_CUDA(cudaGraphAddChildGraphNode(&n_pre, g, nullptr, 0, pre));
    cudaGraphDestroy(pre);
    cudaGraphConditionalHandle cond;
    HS_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t n_loop;
    HS_CUDA(cudaGraphAddNode(&n_loop, g, &n_pre, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    HS_CUDA(cudaStreamBeginCaptureToGraph(h->s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const bool det = h->opt.detect != 0;
    // kLoopUnroll iterations per pass of the while body: every kernel returns at
    // once when the solve is done, and each final kernel sets the condition
    // (programmatic launches between the body's kernels; the body's first kernel follows none)
    const bool pdl = h->opt.scatter == HS_SCATTER_COLORED && pdl_enabled();
    for (int u = 0; u < kLoopUnroll; ++u) {
        apply_projected(h, ROLE_LOOP, nullptr, h->Ap.p, h->opt.dt, det, h->wA.p, nullptr, 0.0, pdl && u > 0);
        launch_update(h, UPD_LOOP, true, cond, pdl);
    }
    HS_CUDA(cudaStreamEndCapture(h->s, &body));
    // after the loop: the solution update still owed
    cudaGraph_t post;
    HS_CUDA(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    launch_update_finish(h);
    HS_CUDA(cudaStreamEndCapture(h->s, &post));
    cudaGraphNode_t n_post;
    HS_CUDA(cudaGraphAddChildGraphNode(&n_post, g, &n_loop, 1, post));
    cudaGraphDestroy(post);
    HS_CUDA(cudaGraphInstantiate(&h->gexec[which], g, 0));
    h->graph[which] = g;
    return HS_OK;
}

hs_status arm_step(hs_solver* h, const hs_fi_spec* fi, int step, bool allow_G) {
    StepCtl c{};
    if (fi && fi->level > 0 && fi->step == step) {
        if (fi->level == HS_FI_G) {
            if (allow_G) { c.flipG = 1; c.gidx = (long long)(fi->target % h->Nn); c.bit = fi->bit; }
        } else if (fi->level == HS_FI_R) {
            c.armR = 1; c.elem = fi->target; c.bit = fi->bit;
        } else if (fi->level >= HS_FI_P) {
            c.vec = fi->level; c.iter = fi->iter; c.idx = (long long)(fi->target % h->Nn); c.bit = fi->bit;
        }
    }
    k_step_begin<<<1, 1, 0, h->s>>>(h->st.p, c, h->T.p);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
}

hs_status validate_fi(const hs_solver* h, const hs_fi_spec* fi) {
    if (!fi || fi->level == 0) return HS_OK;
    if (fi->rank != 0) { set_error("--fi-rank must be in [0,1)"); return HS_ERR_ARG; }
    if (fi->level == HS_FI_H) { set_error("level H needs >= 2 ranks and --fi-rank < nprocs-1"); return HS_ERR_ARG; }
    if (fi->level == 4) { set_error("level 4 (handoff transit) needs --qrank --qblock"); return HS_ERR_ARG; }
    if (fi->level != HS_FI_G && fi->level != HS_FI_R && fi->level != HS_FI_P && fi->level != HS_FI_RV &&
        fi->level != HS_FI_AP) { set_error("unknown fault level"); return HS_ERR_ARG; }
    if (fi->bit < 0 || fi->bit > 63) { set_error("BIT must be in 0..63"); return HS_ERR_ARG; }
    if (fi->target < 0) { set_error("fault target must be >= 0"); return HS_ERR_ARG; }
    (void)h;
    return HS_OK;
}

}  // namespace

// =============================================================================
// C API
// =============================================================================
extern "C" {

int hs_api_version(void) { return HS_API_VERSION; }
const char* hs_last_error(void) { return hs::g_err.c_str(); }

void hs_get_layout(int N, hs_layout_info* out) {
    if (!out) return;
    const SlabLayout L = slab_layout(N);
    out->cx = L.CX; out->ty = L.R; out->tz = L.C; out->rt = RT; out->bpt = SK; out->kf = KF;
}

hs_status hs_gaussian_ic(int N, double sigma, double* T_host) {
    if (N < 1 || N > 1200 || !(sigma > 0) || !T_host) { set_error("hs_gaussian_ic: bad arguments"); return HS_ERR_ARG; }
    gaussian_ic(N, sigma, T_host);
    return HS_OK;
}

void hs_default_options(hs_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->N = 8; o->dt = 1e-3;
    o->kernel = HS_KERNEL_FAST; o->scatter = HS_SCATTER_ATOMIC;
    o->ic_sigma = 0.1; o->rtol = 1e-8; o->max_iter = 500; o->device = 0;
}

hs_status hs_load_fields(const char* prefix, int N, double* k_out, double* rhoc_out) {
    if (!prefix || N <= 0 || !k_out || !rhoc_out) { set_error("bad arguments"); return HS_ERR_ARG; }
    const long long ne = (long long)N * N * N;
    std::string fk = std::string(prefix) + "_k.bin", fr = std::string(prefix) + "_rhoc.bin";
    FILE* f1 = fopen(fk.c_str(), "rb");
    FILE* f2 = fopen(fr.c_str(), "rb");
    if (!f1 || !f2) {
        if (f1) fclose(f1);
        if (f2) fclose(f2);
        set_error("Cannot open " + fk + " / " + fr + " (run gen_field.py)");
        return HS_ERR_IO;
    }
    size_t a = fread(k_out, sizeof(double), (size_t)ne, f1);
    size_t b = fread(rhoc_out, sizeof(double), (size_t)ne, f2);
    fclose(f1); fclose(f2);
    if (a != (size_t)ne || b != (size_t)ne) {
        char msg[256];
        snprintf(msg, sizeof(msg), "Field file too small: expected %lld doubles for this rank "
                 "(grid mismatch? regenerate with gen_field.py --n %d)", ne, N);
        set_error(msg);
        return HS_ERR_IO;
    }
    for (long long i = 0; i < ne; ++i) {
        if (!(k_out[i] > 0) || !(rhoc_out[i] > 0)) {
            char msg[160];
            snprintf(msg, sizeof(msg), "rank 0: non-positive or NaN coefficient at element %lld", i);
            set_error(msg);
            return HS_ERR_ARG;
        }
    }
    return HS_OK;
}

hs_status hs_create(const hs_options* opt, const double* k_host, const double* rhoc_host, hs_solver** out) {
    if (!opt || !k_host || !rhoc_host || !out) { set_error("bad arguments"); return HS_ERR_ARG; }
    *out = nullptr;
    if (opt->N < 1 || opt->N > 1200) { set_error("N must be in [1, 1200]"); return HS_ERR_ARG; }
    if (!(opt->dt >= 0)) { set_error("dt must be >= 0"); return HS_ERR_ARG; }
    if (opt->kernel < 0 || opt->kernel > 2 || opt->scatter < 0 || opt->scatter > 1) {
        set_error("bad kernel/scatter option");
        return HS_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("No CUDA devices"); return HS_ERR_CUDA; }
    HS_CUDA(cudaSetDevice(opt->device % ndev));
    if (!set_smem_attributes()) { set_error("cannot raise the shared-memory limit of the operator kernel"); return HS_ERR_CUDA; }
    std::unique_ptr<hs_solver> h(new hs_solver());
    h->opt = *opt;
    const int N = opt->N;
    h->N = N;
    h->Nn = (long long)(N + 1) * (N + 1) * (N + 1);
    h->Ne = (long long)N * N * N;
    h->part = make_part(N);
    h->kmin = h->kmax = k_host[0];
    h->rhocmin = h->rhocmax = rhoc_host[0];
    for (long long e = 0; e < h->Ne; ++e) {
        if (!(k_host[e] > 0) || !(rhoc_host[e] > 0)) {
            char msg[160];
            snprintf(msg, sizeof(msg), "rank 0: non-positive or NaN coefficient at element %lld", e);
            set_error(msg);
            return HS_ERR_ARG;
        }
        h->kmin = std::fmin(h->kmin, k_host[e]); h->kmax = std::fmax(h->kmax, k_host[e]);
        h->rhocmin = std::fmin(h->rhocmin, rhoc_host[e]); h->rhocmax = std::fmax(h->rhocmax, rhoc_host[e]);
    }
    h->mats = build_reference_matrices(N);
    if (!h->mats.ok) {
        char msg[256];
        snprintf(msg, sizeof(msg), "Reference matrices: M pattern %.1e, sum(M)-V %.1e, K rowsum %.1e, K diag %.1e, "
                 "symmetry %.1e  -> FAIL", h->mats.err[0], h->mats.err[1], h->mats.err[2], h->mats.err[3], h->mats.err[4]);
        set_error(msg);
        return HS_ERR_MATRIX;
    }
    std::memcpy(h->ec.M, h->mats.M, sizeof(h->ec.M));
    std::memcpy(h->ec.K, h->mats.K, sizeof(h->ec.K));
    std::memcpy(h->ec.cm, h->mats.cm, sizeof(h->ec.cm));
    std::memcpy(h->ec.ck, h->mats.ck, sizeof(h->ec.ck));
    h->ec.detJ = h->mats.detJ;

    HS_CUDA(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    HS_CUDA(cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, dev));
    const size_t Nn = (size_t)h->Nn, Ne = (size_t)h->Ne;
    HS_CUDA(h->rhoc.alloc(Ne)); HS_CUDA(h->kc.alloc(Ne)); HS_CUDA(h->gtab.alloc(256)); HS_CUDA(h->coef.alloc(Ne));
    HS_CUDA(h->diag.alloc(Nn)); HS_CUDA(h->F.alloc(Nn));
    HS_CUDA(h->T.alloc(Nn)); HS_CUDA(h->b.alloc(Nn)); HS_CUDA(h->r.alloc(Nn)); HS_CUDA(h->z.alloc(Nn));
    HS_CUDA(h->p0.alloc(Nn)); HS_CUDA(h->p1.alloc(Nn)); HS_CUDA(h->Ap.alloc(Nn));
    HS_CUDA(h->partials.alloc((size_t)MAXQ * std::max(h->part.nblk, h->part.nflat) + 4096));
    HS_CUDA(h->upart.alloc((size_t)3 * h->part.nflat + 256));
    HS_CUDA(h->ticket.alloc(1)); HS_CUDA(h->st.alloc(1)); HS_CUDA(h->red.alloc(8)); HS_CUDA(h->sp.alloc(2));
    HS_CUDA(cudaMemsetAsync(h->ticket.p, 0, sizeof(unsigned), h->s));
    HS_CUDA(cudaMemsetAsync(h->st.p, 0, sizeof(DevState), h->s));
    for (DevBuf<double>* v : {&h->T, &h->b, &h->r, &h->z, &h->p0, &h->p1, &h->Ap})
        HS_CUDA(cudaMemsetAsync(v->p, 0, Nn * sizeof(double), h->s));
    HS_CUDA(cudaMemcpyAsync(h->rhoc.p, rhoc_host, Ne * 8, cudaMemcpyHostToDevice, h->s));
    HS_CUDA(cudaMemcpyAsync(h->kc.p, k_host, Ne * 8, cudaMemcpyHostToDevice, h->s));
    {
        std::vector<double2> ce((size_t)Ne);
        for (long long e = 0; e < Ne; ++e) ce[e] = make_double2(rhoc_host[e], k_host[e]);
        HS_CUDA(cudaMemcpyAsync(h->coef.p, ce.data(), Ne * 16, cudaMemcpyHostToDevice, h->s));
        HS_CUDA(cudaStreamSynchronize(h->s));
    }
    HS_CUDA(cudaMemcpyAsync(h->gtab.p, h->mats.gtab, 256 * 8, cudaMemcpyHostToDevice, h->s));
    h->ec.gtab = h->gtab.p;

    // Jacobi diagonal (het.cu:798-804)
    GenArgs ga{};
    ga.N = N; ga.kind = GEN_DIAG; ga.project = 1; ga.dt_eff = opt->dt; ga.y = h->diag.p;
    ga.rhoc = h->rhoc.p; ga.kc = h->kc.p; ga.ec = h->ec; ga.fi_elem = -1;
    launch_nodes(h.get(), ga);
    HS_CUDA(cudaGetLastError());
    // source (het.cu:806-814): built unless --verify; used unless --no-source
    HS_CUDA(cudaMemsetAsync(h->F.p, 0, Nn * 8, h->s));
    if (!opt->verify && !opt->no_source) {
        std::vector<double> F;
        build_source(N, 0.1, F);
        HS_CUDA(cudaMemcpyAsync(h->F.p, F.data(), Nn * 8, cudaMemcpyHostToDevice, h->s));
        HS_CUDA(cudaStreamSynchronize(h->s));
        h->has_F = true;
    }
    // ABFT weights (het.cu:940-953): w_M = M 1_int, w_A = A 1_int, unprojected
    if (opt->detect) {
        HS_CUDA(h->wM.alloc(Nn)); HS_CUDA(h->wA.alloc(Nn));
        // ones on the interior: r <- 1, boundary 0
        std::vector<double> ones(Nn);
        for (size_t n = 0; n < Nn; ++n) {
            const long long NN = N + 1;
            int ix = (int)(n / (NN * NN)), iy = (int)((n / NN) % NN), iz = (int)(n % NN);
            ones[n] = (ix == 0 || ix == N || iy == 0 || iy == N || iz == 0 || iz == N) ? 0.0 : 1.0;
        }
        HS_CUDA(cudaMemcpyAsync(h->r.p, ones.data(), Nn * 8, cudaMemcpyHostToDevice, h->s));
        GenArgs gw{};
        gw.N = N; gw.kind = GEN_APPLY; gw.project = 0; gw.x = h->r.p; gw.rhoc = h->rhoc.p; gw.kc = h->kc.p;
        gw.ec = h->ec; gw.fi_elem = -1;
        gw.dt_eff = 0.0; gw.y = h->wM.p;
        launch_nodes(h.get(), gw);
        gw.dt_eff = opt->dt; gw.y = h->wA.p;
        launch_nodes(h.get(), gw);
        launch_reduce(h.get(), RED_DOT, h->wM.p, h->wM.p, h->red.p);
        launch_reduce(h.get(), RED_DOT, h->wA.p, h->wA.p, h->red.p + 2);
        double nr[4];
        HS_CUDA(cudaMemcpyAsync(nr, h->red.p, 4 * 8, cudaMemcpyDeviceToHost, h->s));
        HS_CUDA(cudaStreamSynchronize(h->s));
        DevState hs{};
        HS_CUDA(cudaMemcpy(&hs, h->st.p, sizeof(hs), cudaMemcpyDeviceToHost));
        hs.norm_wM = std::sqrt(nr[0]);
        hs.norm_wA = std::sqrt(nr[2]);
        HS_CUDA(cudaMemcpy(h->st.p, &hs, sizeof(hs), cudaMemcpyHostToDevice));
        HS_CUDA(cudaMemsetAsync(h->r.p, 0, Nn * 8, h->s));
    }
    HS_CUDA(cudaStreamSynchronize(h->s));
    HS_CUDA(cudaGetLastError());
    hs_status st = sync_state_config(h.get(), opt->max_iter, opt->rtol);
    if (st != HS_OK) return st;
    *out = h.release();
    return HS_OK;
}

void hs_destroy(hs_solver* s) { delete s; }

long long hs_num_nodes(const hs_solver* s) { return s ? s->Nn : 0; }

hs_status hs_field_stats(const hs_solver* s, double out9[9]) {
    if (!s || !out9) return HS_ERR_ARG;
    out9[0] = s->kmin; out9[1] = s->kmax; out9[2] = s->rhocmin; out9[3] = s->rhocmax;
    for (int i = 0; i < 5; ++i) out9[4 + i] = s->mats.err[i];
    return HS_OK;
}

hs_status hs_arm_fi(hs_solver* s, const hs_fi_spec* fi) {
    if (!s) return HS_ERR_ARG;
    hs_status v = validate_fi(s, fi);
    if (v != HS_OK) return v;
    if (fi) { s->pending = *fi; s->pending_set = fi->level > 0; } else s->pending_set = false;
    return HS_OK;
}

hs_status hs_apply(hs_solver* s, const double* x, double* y, double dt_eff, int allow_fi, int project, double* abft_rel) {
    if (!s || !x || !y) { set_error("bad arguments"); return HS_ERR_ARG; }
    if (x < y + s->Nn && y < x + s->Nn) {
        // tiles read halo nodes of x that neighbouring tiles write in y
        set_error("hs_apply: x and y overlap (the operator is not applied in place)");
        return HS_ERR_ARG;
    }
    if (abft_rel) *abft_rel = -1.0;
    StepCtl c{};
    if (allow_fi && s->pending_set && s->pending.level == HS_FI_R) {
        c.armR = 1; c.elem = s->pending.target; c.bit = s->pending.bit;
        s->pending_set = false;
    }
    if (!project) {
        GenArgs g{};
        g.N = s->N; g.kind = GEN_APPLY; g.project = 0; g.dt_eff = dt_eff; g.x = x; g.y = y;
        g.rhoc = s->rhoc.p; g.kc = s->kc.p; g.ec = s->ec; g.fi_elem = c.armR ? c.elem : -1; g.fi_bit = c.bit;
        g.fire_r = c.armR;
        launch_nodes(s, g);
        HS_CUDA(cudaGetLastError());
        HS_CUDA(cudaStreamSynchronize(s->s));
        return HS_OK;
    }
    const bool d1 = s->opt.detect != 0;
    k_step_begin<<<1, 1, 0, s->s>>>(s->st.p, c, s->T.p);
    // dt_eff == 0 is the mass matrix: checksum against w_M (build_rhs), else w_A
    if (dt_eff == 0.0)
        apply_projected(s, ROLE_RHS, x, y, dt_eff, d1, s->wM.p, nullptr, 0.0);
    else
        apply_projected(s, ROLE_X0, x, y, dt_eff, d1, s->wA.p, nullptr, 0.0);
    k_step_end<<<1, 1, 0, s->s>>>(s->st.p, (int*)(s->red.p + 6), s->red.p + 7);
    HS_CUDA(cudaGetLastError());
    DevState hsx{};
    HS_CUDA(cudaMemcpyAsync(&hsx, s->st.p, sizeof(hsx), cudaMemcpyDeviceToHost, s->s));
    HS_CUDA(cudaStreamSynchronize(s->s));
    if (d1 && abft_rel) *abft_rel = hsx.d1_last;
    return HS_OK;
}

hs_status hs_precond(hs_solver* s, const double* r, double* z) {
    if (!s || !r || !z) return HS_ERR_ARG;
    k_jacobi<<<grid_for(s->Nn, RT), RT, 0, s->s>>>(s->Nn, r, s->diag.p, z);
    HS_CUDA(cudaGetLastError());
    HS_CUDA(cudaStreamSynchronize(s->s));
    return HS_OK;
}

hs_status hs_build_rhs(hs_solver* s, const double* T, double* b) {
    if (!s || !T || !b) return HS_ERR_ARG;
    const bool src = !s->opt.verify && !s->opt.no_source && s->has_F;
    const bool d1 = s->opt.detect != 0;
    k_step_begin<<<1, 1, 0, s->s>>>(s->st.p, StepCtl{}, s->T.p);
    apply_projected(s, ROLE_RHS, T, b, 0.0, d1, s->wM.p, src ? s->F.p : nullptr, s->opt.dt);
    HS_CUDA(cudaGetLastError());
    HS_CUDA(cudaStreamSynchronize(s->s));
    return HS_OK;
}

hs_status hs_dot(hs_solver* s, const double* x, const double* y, double* out) {
    if (!s || !x || !y || !out) return HS_ERR_ARG;
    launch_reduce(s, RED_DOT, x, y, s->red.p);
    HS_CUDA(cudaGetLastError());
    HS_CUDA(cudaMemcpyAsync(out, s->red.p, 8, cudaMemcpyDeviceToHost, s->s));
    HS_CUDA(cudaStreamSynchronize(s->s));
    return HS_OK;
}

}  // extern "C"

// ---- trajectories ------------------------------------------------------------------
namespace {

// one implicit-Euler step on h->T (PCG through the graph); per-step outputs
// written to device slots. Caller records events around it.
hs_status pcg_direct(hs_solver* h, bool with_rhs) {
    enqueue_pcg_prologue(h, with_rhs);
    const bool det = h->opt.detect != 0;
    DevState hsx{};
    for (int it = 0; it < (1 << 30); it += 16) {
        const bool pdl = h->opt.scatter == HS_SCATTER_COLORED && pdl_enabled();
        for (int k = 0; k < 16; ++k) {
            apply_projected(h, ROLE_LOOP, nullptr, h->Ap.p, h->opt.dt, det, h->wA.p, nullptr, 0.0, pdl && k > 0);
            launch_update(h, UPD_LOOP, false, 0, pdl);
        }
        HS_CUDA(cudaMemcpyAsync(&hsx, h->st.p, sizeof(hsx), cudaMemcpyDeviceToHost, h->s));
        HS_CUDA(cudaStreamSynchronize(h->s));
        if (hsx.done) break;
    }
    launch_update_finish(h);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
}

hs_status enqueue_step(hs_solver* h, const hs_fi_spec* fi, int step, int reproject, int* d_iters, double* d_d1,
                       cudaEvent_t e0, cudaEvent_t e1) {
    hs_status st = arm_step(h, fi, step, true);
    if (st != HS_OK) return st;
    if (e0) HS_CUDA(cudaEventRecord(e0, h->s));
    if (graphs_enabled()) {
        HS_CUDA(cudaGraphLaunch(h->gexec[0], h->s));
    } else {
        st = pcg_direct(h, true);
        if (st != HS_OK) return st;
    }
    if (reproject) k_set_boundary<<<grid_for(h->Nn, RT), RT, 0, h->s>>>(h->N, h->T.p, 0.0);
    if (e1) HS_CUDA(cudaEventRecord(e1, h->s));
    k_step_end<<<1, 1, 0, h->s>>>(h->st.p, d_iters, d_d1);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
}

}  // namespace

// where a trajectory starts (run_case_impl)
struct RunFrom {
    int s0 = 0;                            // first step computed
    const double* T_start = nullptr;       // device field at the start of step s0 (s0 > 0)
    double* const* keep_states = nullptr;  // optional: field at the start of every step
};
hs_status run_case_impl(hs_solver* h, int n_steps, int snap_every, const hs_fi_spec* fi, int reproject,
                        int keep_reference, hs_step_record* out, double* T_final_host, int* nonfinite,
                        const RunFrom& from);

extern "C" {

hs_status hs_pcg(hs_solver* s, const double* b, double* x, int max_iter, double tol, int* iters) {
    if (!s || !b || !x) return HS_ERR_ARG;
    hs_status st = sync_state_config(s, max_iter, tol);
    if (st != HS_OK) return st;
    st = build_graph(s, 1);
    if (st != HS_OK) return st;
    HS_CUDA(cudaMemcpyAsync(s->b.p, b, s->Nn * 8, cudaMemcpyDeviceToDevice, s->s));
    HS_CUDA(cudaMemcpyAsync(s->T.p, x, s->Nn * 8, cudaMemcpyDeviceToDevice, s->s));
    hs_fi_spec fi{};
    const hs_fi_spec* pf = nullptr;
    if (s->pending_set) { fi = s->pending; fi.step = 0; pf = &fi; s->pending_set = false; }
    st = arm_step(s, pf, 0, false);
    if (st != HS_OK) return st;
    if (graphs_enabled()) {
        HS_CUDA(cudaGraphLaunch(s->gexec[1], s->s));
    } else {
        st = pcg_direct(s, false);
        if (st != HS_OK) return st;
    }
    k_step_end<<<1, 1, 0, s->s>>>(s->st.p, (int*)(s->red.p + 6), s->red.p + 7);
    HS_CUDA(cudaGetLastError());
    HS_CUDA(cudaMemcpyAsync(x, s->T.p, s->Nn * 8, cudaMemcpyDeviceToDevice, s->s));
    DevState hsx{};
    HS_CUDA(cudaMemcpyAsync(&hsx, s->st.p, sizeof(hsx), cudaMemcpyDeviceToHost, s->s));
    HS_CUDA(cudaStreamSynchronize(s->s));
    if (iters) *iters = hsx.result;
    return sync_state_config(s, s->opt.max_iter, s->opt.rtol);
}

hs_status hs_run_case(hs_solver* h, int n_steps, int snap_every, const hs_fi_spec* fi, int reproject,
                      int keep_reference, hs_step_record* out, double* T_final_host, int* nonfinite) {
    return run_case_impl(h, n_steps, snap_every, fi, reproject, keep_reference, out, T_final_host, nonfinite,
                         RunFrom{});
}

}  // extern "C"

// One trajectory (run_case, het.cu:1107-1259).  from.s0 > 0 resumes at step
// s0 from the field from.T_start (records of earlier steps are left to the
// caller); from.keep_states, if set, receives the field at the start of every
// step (n_steps device buffers of (N+1)^3 doubles).
hs_status run_case_impl(hs_solver* h, int n_steps, int snap_every, const hs_fi_spec* fi, int reproject,
                        int keep_reference, hs_step_record* out, double* T_final_host, int* nonfinite,
                        const RunFrom& from) {
    if (!h || n_steps < 0 || !out) { set_error("bad arguments"); return HS_ERR_ARG; }
    if (from.s0 < 0 || from.s0 > n_steps || (from.s0 > 0 && (!from.T_start || keep_reference))) {
        set_error("bad resume step");
        return HS_ERR_ARG;
    }
    hs_status st = validate_fi(h, fi);
    if (st != HS_OK) return st;
    st = sync_state_config(h, h->opt.max_iter, h->opt.rtol);
    if (st != HS_OK) return st;
    st = build_graph(h, 0);
    if (st != HS_OK) return st;
    const long long Nn = h->Nn;
    const int s0 = from.s0;
    // initial condition (het.cu:1115-1116), or the resumed field
    if (s0 > 0) {
        HS_CUDA(cudaMemcpyAsync(h->T.p, from.T_start, Nn * 8, cudaMemcpyDeviceToDevice, h->s));
    } else if (h->opt.ic_mode == 1) {
        std::vector<double> T0(Nn);
        gaussian_ic(h->N, h->opt.ic_sigma, T0.data());
        HS_CUDA(cudaMemcpyAsync(h->T.p, T0.data(), Nn * 8, cudaMemcpyHostToDevice, h->s));
        HS_CUDA(cudaStreamSynchronize(h->s));
    } else {
        HS_CUDA(cudaMemsetAsync(h->T.p, 0, Nn * 8, h->s));
    }
    int n_snap = 0;
    for (int s = 0; s < n_steps; ++s)
        if ((snap_every > 0 && s % snap_every == 0) || s == n_steps - 1) ++n_snap;
    const bool compare = !keep_reference && h->ref_nsteps == n_steps && h->ref_snap_every == snap_every &&
                         (int)h->ref_snaps.size() == n_snap;
    if (keep_reference) {
        for (double* q : h->ref_snaps) cudaFree(q);
        h->ref_snaps.clear();
        for (int i = 0; i < n_snap; ++i) {
            double* q = nullptr;
            HS_CUDA(cudaMalloc(&q, Nn * 8));
            h->ref_snaps.push_back(q);
        }
        h->ref_nsteps = n_steps; h->ref_snap_every = snap_every;
    }
    // per-step device outputs
    DevBuf<int> d_it;
    DevBuf<double> d_rec;   // per step: d1, d2, tmin, tmax, E, spread
    HS_CUDA(d_it.alloc(std::max(n_steps, 1)));
    HS_CUDA(d_rec.alloc((size_t)std::max(n_steps, 1) * 8));
    HS_CUDA(cudaMemsetAsync(d_rec.p, 0, (size_t)std::max(n_steps, 1) * 8 * 8, h->s));
    Events ev;
    HS_CUDA(ev.create(2 * (size_t)n_steps));
    int si = 0;
    for (int step = 0; step < s0; ++step)
        if ((snap_every > 0 && step % snap_every == 0) || step == n_steps - 1) ++si;
    for (int step = s0; step < n_steps; ++step) {
        double* rec = d_rec.p + (size_t)step * 8;
        if (from.keep_states)
            HS_CUDA(cudaMemcpyAsync(from.keep_states[step], h->T.p, Nn * 8, cudaMemcpyDeviceToDevice, h->s));
        st = enqueue_step(h, fi, step, reproject, d_it.p + step, rec + 0, ev[2 * step], ev[2 * step + 1]);
        if (st != HS_OK) return st;
        if (h->opt.detect) {
            // D2: true residual with a fresh matvec (het.cu:1205-1210); D3 range (het.cu:1219)
            apply_projected(h, ROLE_PLAIN, h->T.p, h->z.p, h->opt.dt, false, nullptr, nullptr, 0.0);
            launch_reduce(h, RED_RESID, h->z.p, h->b.p, h->red.p);
            k_d2_finish<<<1, 1, 0, h->s>>>(h->red.p, rec + 1);
            const int gmm = std::min<long long>(148 * 8, (Nn + RT - 1) / RT);
            k_minmax<<<gmm, RT, 0, h->s>>>(h->N, h->T.p, h->partials.p, h->ticket.p, rec + 2);
        }
        const bool snap = (snap_every > 0 && step % snap_every == 0) || step == n_steps - 1;
        if (snap && !h->dump_dir.empty()) {
            std::vector<double> hv(Nn);
            HS_CUDA(cudaMemcpyAsync(hv.data(), h->T.p, Nn * 8, cudaMemcpyDeviceToHost, h->s));
            HS_CUDA(cudaStreamSynchronize(h->s));
            char pth[900];
            snprintf(pth, sizeof(pth), "%s/snap_%s_%s_%05d_rank0.bin", h->dump_dir.c_str(), h->dump_tag.c_str(),
                     h->case_tag.c_str(), step);
            FILE* f = fopen(pth, "wb");
            if (f) { fwrite(hv.data(), sizeof(double), hv.size(), f); fclose(f); }
        }
        if (snap) {
            if (keep_reference) {
                HS_CUDA(cudaMemcpyAsync(h->ref_snaps[si], h->T.p, Nn * 8, cudaMemcpyDeviceToDevice, h->s));
            } else if (compare) {
                const double* ref = h->ref_snaps[si];
                launch_reduce(h, RED_DIFF, h->T.p, ref, h->red.p);
                HS_CUDA(cudaMemsetAsync(h->sp.p, 0, 2 * sizeof(unsigned long long), h->s));
                const int g = grid_for(Nn, RT);
                k_absdiff_max<<<g, RT, 0, h->s>>>(Nn, h->T.p, ref, h->sp.p);
                k_absdiff_count<<<g, RT, 0, h->s>>>(Nn, h->T.p, ref, h->sp.p, 1e-3, h->sp.p + 1);
                k_e_finish<<<1, 1, 0, h->s>>>(h->red.p, h->sp.p, h->sp.p + 1, Nn, rec + 4, rec + 5);
            }
            ++si;
        }
        HS_CUDA(cudaGetLastError());
    }
    HS_CUDA(cudaStreamSynchronize(h->s));
    std::vector<int> it(std::max(n_steps, 1));
    std::vector<double> rec((size_t)std::max(n_steps, 1) * 8);
    HS_CUDA(cudaMemcpy(it.data(), d_it.p, n_steps * sizeof(int), cudaMemcpyDeviceToHost));
    HS_CUDA(cudaMemcpy(rec.data(), d_rec.p, (size_t)n_steps * 8 * 8, cudaMemcpyDeviceToHost));
    int nf = 0;
    si = 0;
    if (keep_reference) { h->ref_tmin.assign(n_steps, 0.0); h->ref_tmax.assign(n_steps, 0.0); }
    for (int step = s0; step < n_steps; ++step) {
        hs_step_record& o = out[step];
        const double* rr = &rec[(size_t)step * 8];
        o.cg_iters = it[step];
        o.d1 = h->opt.detect ? rr[0] : 0.0;
        o.d2 = h->opt.detect ? rr[1] : 0.0;
        o.tmin = h->opt.detect ? rr[2] : 0.0;
        o.tmax = h->opt.detect ? rr[3] : 0.0;
        const bool snap = (snap_every > 0 && step % snap_every == 0) || step == n_steps - 1;
        o.snap = snap ? 1 : 0;
        o.E = (snap && compare) ? rr[4] : -1.0;
        o.spread = (snap && compare) ? rr[5] : 0.0;
        if (snap && compare && !std::isfinite(o.E)) nf = 1;
        float ms = 0.f;
        HS_CUDA(cudaEventElapsedTime(&ms, ev[2 * step], ev[2 * step + 1]));
        o.solve_ms = ms;
        if (keep_reference) { h->ref_tmin[step] = o.tmin; h->ref_tmax[step] = o.tmax; }
    }
    if (nonfinite) *nonfinite = nf;
    if (T_final_host) HS_CUDA(cudaMemcpy(T_final_host, h->T.p, Nn * 8, cudaMemcpyDeviceToHost));
    return HS_OK;
}

extern "C" {

hs_status hs_verify(hs_solver* h, int n_steps, double* rel_err, long long* total_iters, double* ms) {
    if (!h) return HS_ERR_ARG;
    if (h->kmin != h->kmax || h->rhocmin != h->rhocmax) {
        char msg[256];
        snprintf(msg, sizeof(msg), "--verify needs a homogeneous field (k %g..%g, rhoc %g..%g)", h->kmin, h->kmax,
                 h->rhocmin, h->rhocmax);
        set_error(msg);
        return HS_ERR_ARG;
    }
    hs_status st = sync_state_config(h, h->opt.max_iter, h->opt.rtol);
    if (st != HS_OK) return st;
    st = build_graph(h, 0);
    if (st != HS_OK) return st;
    const double alpha = h->kmin / h->rhocmin;
    const long long Nn = h->Nn;
    std::vector<double> v(Nn);
    exact_mode(h->N, 0.0, alpha, v.data());
    HS_CUDA(cudaMemcpyAsync(h->T.p, v.data(), Nn * 8, cudaMemcpyHostToDevice, h->s));
    DevBuf<int> d_it;
    DevBuf<double> d_d1;
    HS_CUDA(d_it.alloc(std::max(n_steps, 1)));
    HS_CUDA(d_d1.alloc(std::max(n_steps, 1)));
    Events ev2;
    HS_CUDA(ev2.create(2));
    cudaEvent_t e0 = ev2[0], e1 = ev2[1];
    HS_CUDA(cudaEventRecord(e0, h->s));
    for (int step = 0; step < n_steps; ++step) {
        st = enqueue_step(h, nullptr, step, 0, d_it.p + step, d_d1.p + step, nullptr, nullptr);
        if (st != HS_OK) return st;
    }
    HS_CUDA(cudaEventRecord(e1, h->s));
    HS_CUDA(cudaEventSynchronize(e1));
    float fms = 0.f;
    HS_CUDA(cudaEventElapsedTime(&fms, e0, e1));
    std::vector<int> it(std::max(n_steps, 1));
    HS_CUDA(cudaMemcpy(it.data(), d_it.p, n_steps * sizeof(int), cudaMemcpyDeviceToHost));
    long long tot = 0;
    for (int i = 0; i < n_steps; ++i) tot += it[i];
    // error against exp(-3 pi^2 alpha t) sin sin sin (het.cu:1314-1320)
    exact_mode(h->N, n_steps * h->opt.dt, alpha, v.data());
    HS_CUDA(cudaMemcpyAsync(h->r.p, v.data(), Nn * 8, cudaMemcpyHostToDevice, h->s));
    launch_reduce(h, RED_DOT, h->r.p, h->r.p, h->red.p);
    launch_reduce(h, RED_RESID, h->T.p, h->r.p, h->red.p + 2);   // q0 = |r - T|^2
    double rv[4];
    HS_CUDA(cudaMemcpyAsync(rv, h->red.p, 32, cudaMemcpyDeviceToHost, h->s));
    HS_CUDA(cudaStreamSynchronize(h->s));
    const double en = std::sqrt(rv[0]);
    if (rel_err) *rel_err = std::sqrt(rv[2]) / en;
    if (total_iters) *total_iters = tot;
    if (ms) *ms = fms;
    return HS_OK;
}

hs_status hs_solve_host(hs_solver* h, const double* T0_host, double* T_host, int n_steps, long long* total_iters,
                        double* device_ms) {
    if (!h || !T0_host || !T_host || n_steps < 0) return HS_ERR_ARG;
    hs_status st = build_graph(h, 0);
    if (st != HS_OK) return st;
    const long long Nn = h->Nn;
    DevBuf<int> d_it;
    DevBuf<double> d_d1;
    HS_CUDA(d_it.alloc(std::max(n_steps, 1)));
    HS_CUDA(d_d1.alloc(std::max(n_steps, 1)));
    Events ev2;
    HS_CUDA(ev2.create(2));
    cudaEvent_t e0 = ev2[0], e1 = ev2[1];
    HS_CUDA(cudaEventRecord(e0, h->s));
    HS_CUDA(cudaMemcpyAsync(h->T.p, T0_host, Nn * 8, cudaMemcpyHostToDevice, h->s));
    for (int step = 0; step < n_steps; ++step) {
        st = enqueue_step(h, nullptr, step, 0, d_it.p + step, d_d1.p + step, nullptr, nullptr);
        if (st != HS_OK) return st;
    }
    HS_CUDA(cudaMemcpyAsync(T_host, h->T.p, Nn * 8, cudaMemcpyDeviceToHost, h->s));
    HS_CUDA(cudaEventRecord(e1, h->s));
    HS_CUDA(cudaEventSynchronize(e1));
    float fms = 0.f;
    HS_CUDA(cudaEventElapsedTime(&fms, e0, e1));
    std::vector<int> it(std::max(n_steps, 1));
    HS_CUDA(cudaMemcpy(it.data(), d_it.p, n_steps * sizeof(int), cudaMemcpyDeviceToHost));
    long long tot = 0;
    for (int i = 0; i < n_steps; ++i) tot += it[i];
    if (total_iters) *total_iters = tot;
    if (device_ms) *device_ms = fms;
    return HS_OK;
}

}  // extern "C"

extern "C" {

hs_status hs_set_dump(hs_solver* s, const char* dir, const char* tag) {
    if (!s) return HS_ERR_ARG;
    s->dump_dir = dir ? dir : "";
    s->dump_tag = tag ? tag : "";
    return HS_OK;
}

hs_status hs_set_case_tag(hs_solver* s, const char* case_tag) {
    if (!s) return HS_ERR_ARG;
    s->case_tag = case_tag ? case_tag : "";
    return HS_OK;
}

int hs_target_on_boundary(const hs_solver* s, const hs_fi_spec* fi) {
    if (!s || !fi || fi->level <= 0) return -1;
    const long long N = s->N, NN = N + 1;
    auto bnd = [&](long long ix, long long iy, long long iz, long long hi) {
        return (ix == 0 || ix == hi || iy == 0 || iy == hi || iz == 0 || iz == hi) ? 1 : 0;
    };
    if (fi->level == HS_FI_R) {   // node 0 of the element (het.cu:1278-1281)
        const long long e = fi->target % s->Ne;
        return bnd(e / (N * N), (e / N) % N, e % N, N);
    }
    const long long nd = fi->target % s->Nn;
    return bnd(nd / (NN * NN), (nd / NN) % NN, nd % NN, N);
}

hs_status hs_diag_cg(hs_solver* h, int max_iter, double tol, double* rel0, double* rel, double* alpha, double* beta,
                     int cap, int* iters) {
    if (!h || cap < 0) return HS_ERR_ARG;
    hs_status st = sync_state_config(h, max_iter, tol);
    if (st != HS_OK) return st;
    DevBuf<double> lg;
    HS_CUDA(lg.alloc((size_t)3 * std::max(cap, 1)));
    DevState hsx{};
    HS_CUDA(cudaMemcpy(&hsx, h->st.p, sizeof(hsx), cudaMemcpyDeviceToHost));
    hsx.log_rel = lg.p; hsx.log_alpha = lg.p + cap; hsx.log_beta = lg.p + 2 * cap; hsx.log_cap = cap;
    HS_CUDA(cudaMemcpy(h->st.p, &hsx, sizeof(hsx), cudaMemcpyHostToDevice));
    // one solve from the initial condition, no fault, no detector bookkeeping
    std::vector<double> T0(h->Nn, 0.0);
    if (h->opt.ic_mode == 1) gaussian_ic(h->N, h->opt.ic_sigma, T0.data());
    HS_CUDA(cudaMemcpyAsync(h->T.p, T0.data(), h->Nn * 8, cudaMemcpyHostToDevice, h->s));
    st = build_graph(h, 0);
    if (st != HS_OK) return st;
    DevBuf<int> d_it;
    DevBuf<double> d_d1;
    HS_CUDA(d_it.alloc(1)); HS_CUDA(d_d1.alloc(1));
    st = enqueue_step(h, nullptr, 0, 0, d_it.p, d_d1.p, nullptr, nullptr);
    if (st != HS_OK) return st;
    HS_CUDA(cudaStreamSynchronize(h->s));
    int it = 0;
    HS_CUDA(cudaMemcpy(&it, d_it.p, sizeof(int), cudaMemcpyDeviceToHost));
    HS_CUDA(cudaMemcpy(&hsx, h->st.p, sizeof(hsx), cudaMemcpyDeviceToHost));
    const int n = std::min(it, cap);
    if (rel && n) HS_CUDA(cudaMemcpy(rel, lg.p, n * 8, cudaMemcpyDeviceToHost));
    if (alpha && n) HS_CUDA(cudaMemcpy(alpha, lg.p + cap, n * 8, cudaMemcpyDeviceToHost));
    if (beta && n) HS_CUDA(cudaMemcpy(beta, lg.p + 2 * cap, n * 8, cudaMemcpyDeviceToHost));
    if (rel0) *rel0 = hsx.rel0;
    if (iters) *iters = it;
    hsx.log_rel = hsx.log_alpha = hsx.log_beta = nullptr; hsx.log_cap = 0;
    HS_CUDA(cudaMemcpy(h->st.p, &hsx, sizeof(hsx), cudaMemcpyHostToDevice));
    return sync_state_config(h, h->opt.max_iter, h->opt.rtol);
}

}  // extern "C"

extern "C" {

hs_status hs_set_field(hs_solver* h, const double* T_host) {
    if (!h || !T_host) return HS_ERR_ARG;
    HS_CUDA(cudaMemcpyAsync(h->T.p, T_host, h->Nn * 8, cudaMemcpyHostToDevice, h->s));
    HS_CUDA(cudaStreamSynchronize(h->s));
    return HS_OK;
}

hs_status hs_get_field(hs_solver* h, double* T_host) {
    if (!h || !T_host) return HS_ERR_ARG;
    HS_CUDA(cudaMemcpyAsync(T_host, h->T.p, h->Nn * 8, cudaMemcpyDeviceToHost, h->s));
    HS_CUDA(cudaStreamSynchronize(h->s));
    return HS_OK;
}

hs_status hs_advance(hs_solver* h, int n_steps, int from_ic, long long* total_iters, double* device_ms) {
    if (!h || n_steps < 0) return HS_ERR_ARG;
    hs_status st = build_graph(h, 0);
    if (st != HS_OK) return st;
    if (from_ic && !h->T0.p) {
        std::vector<double> v(h->Nn, 0.0);
        if (h->opt.ic_mode == 1) gaussian_ic(h->N, h->opt.ic_sigma, v.data());
        HS_CUDA(h->T0.alloc(h->Nn));
        HS_CUDA(cudaMemcpy(h->T0.p, v.data(), h->Nn * 8, cudaMemcpyHostToDevice));
    }
    DevBuf<int> d_it;
    DevBuf<double> d_d1;
    HS_CUDA(d_it.alloc(std::max(n_steps, 1)));
    HS_CUDA(d_d1.alloc(std::max(n_steps, 1)));
    Events ev2;
    HS_CUDA(ev2.create(2));
    cudaEvent_t e0 = ev2[0], e1 = ev2[1];
    HS_CUDA(cudaEventRecord(e0, h->s));
    if (from_ic) HS_CUDA(cudaMemcpyAsync(h->T.p, h->T0.p, h->Nn * 8, cudaMemcpyDeviceToDevice, h->s));
    for (int step = 0; step < n_steps; ++step) {
        st = enqueue_step(h, nullptr, step, 0, d_it.p + step, d_d1.p + step, nullptr, nullptr);
        if (st != HS_OK) return st;
    }
    HS_CUDA(cudaEventRecord(e1, h->s));
    HS_CUDA(cudaEventSynchronize(e1));
    float fms = 0.f;
    HS_CUDA(cudaEventElapsedTime(&fms, e0, e1));
    std::vector<int> it(std::max(n_steps, 1));
    HS_CUDA(cudaMemcpy(it.data(), d_it.p, n_steps * sizeof(int), cudaMemcpyDeviceToHost));
    long long tot = 0;
    for (int i = 0; i < n_steps; ++i) tot += it[i];
    if (total_iters) *total_iters = tot;
    if (device_ms) *device_ms = fms;
    return HS_OK;
}

hs_status hs_time_kernel(hs_solver* h, int which, int reps, double* ms_per_launch) {
    if (!h || reps < 1 || which < 0 || which > 2) return HS_ERR_ARG;
    // state for repeated launches: loop running at iteration 1, never converging
    DevState hsx{};
    HS_CUDA(cudaMemcpy(&hsx, h->st.p, sizeof(hsx), cudaMemcpyDeviceToHost));
    DevState saved = hsx;
    hsx.done = 0; hsx.broken = 0; hsx.iter = 1; hsx.beta = 0.5; hsx.rho = 1.0; hsx.alpha = 1e-3;
    hsx.bnorm = 1.0; hsx.tol = 0.0; hsx.max_iter = 1 << 30; hsx.fi_armR = 0; hsx.fi_vec = 0;
    hsx.log_rel = hsx.log_alpha = hsx.log_beta = nullptr; hsx.log_cap = 0;
    HS_CUDA(cudaMemcpy(h->st.p, &hsx, sizeof(hsx), cudaMemcpyHostToDevice));
    // nonzero, SPD-consistent inputs (p.Ap > 0): the positive diagonal
    for (double* v : {h->z.p, h->p0.p, h->p1.p, h->T.p, h->r.p})
        k_copy<<<grid_for(h->Nn, RT), RT, 0, h->s>>>(h->Nn, h->diag.p, v);
    // L2 scrub buffer (256 MiB > 126 MB L2), read before each timed launch
    DevBuf<double> flush;
    const size_t fl = (size_t)32 << 20;   // doubles
    HS_CUDA(flush.alloc(fl));
    HS_CUDA(cudaMemsetAsync(flush.p, 0, fl * 8, h->s));
    Events ev;
    HS_CUDA(ev.create(2 * (size_t)reps));
    const bool det = h->opt.detect != 0;
    // the update finishes the operator's reductions: give it one operator's partials
    if (which == 1) apply_projected(h, ROLE_LOOP, nullptr, h->Ap.p, h->opt.dt, det, h->wA.p, nullptr, 0.0);
    for (int r = 0; r < reps; ++r) {
        k_l2_scrub<<<148 * 8, 256, 0, h->s>>>(flush.p, (long long)fl, h->red.p + 5);
        HS_CUDA(cudaEventRecord(ev[2 * r], h->s));
        if (which == 0) {
            apply_projected(h, ROLE_LOOP, nullptr, h->Ap.p, h->opt.dt, det, h->wA.p, nullptr, 0.0);
        } else if (which == 1) {
            // keep the iteration counter (and so the p buffer) fixed at 1
            launch_update(h, UPD_LOOP, false);
        } else {
            apply_projected(h, ROLE_PLAIN, h->T.p, h->z.p, h->opt.dt, false, nullptr, nullptr, 0.0);
        }
        HS_CUDA(cudaEventRecord(ev[2 * r + 1], h->s));
        if (which == 1) {
            DevState* d = h->st.p;
            HS_CUDA(cudaMemcpyAsync(&d->iter, &hsx.iter, sizeof(int), cudaMemcpyHostToDevice, h->s));
        }
    }
    HS_CUDA(cudaStreamSynchronize(h->s));
    HS_CUDA(cudaGetLastError());
    double tot = 0;
    for (int r = 0; r < reps; ++r) {
        float ms = 0.f;
        HS_CUDA(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]));
        tot += ms;
    }
    saved.done = 1;
    HS_CUDA(cudaMemcpy(h->st.p, &saved, sizeof(saved), cudaMemcpyHostToDevice));
    if (ms_per_launch) *ms_per_launch = tot / reps;
    return HS_OK;
}

}  // extern "C"

// the allocation-free dot product shares this translation unit's kernels
#include "hs_noalloc.cu"
// the fault-injection campaign resumes trajectories through run_case_impl
#include "hs_campaign.cu"
// lognormal fields generated on the device (standalone and for batched instances)
#include "hs_field.cu"
// the batched mixed-precision solver reuses the slab partition and set-up kernels
#include "hs_batch.cu"
