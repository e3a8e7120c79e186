// hs_batch.cu -- batched mixed-precision transient-heat solver (libheat_b200).
//
// No counterpart in the reference, which runs one solve per MPI job.  Many
// independent solves (different N, dt, fields, step counts) live in slots of
// one handle and advance together: hs_batch_step runs one implicit-Euler step
// of every instance that has steps left, as one CUDA-graph launch:
//   b = M T (FP64 slab operator, ABFT checked);
//   start from T, or from 2 T - T_prev (extrapolate, from the second step);
//   r = b - A T (FP64 slab operator, ABFT checked), test ||r|| / ||b|| < rtol;
//   while not converged (bounded by max_outer):
//       FP32 Jacobi-PCG on A d = r to inner_tol (bounded by max_inner),
//       every launch covering the tiles of all instances still iterating;
//       T += d (FP64, interior nodes; discarded if the inner solve went
//       non-finite); r = b - A T; test.
// Instances are added and removed between steps (continuous batching): the
// host compacts their tile and block ranges into device maps that the graph
// reads, so the graph stays valid until the capacity has to grow.
//
// Included by hs_solver.cu.
#include "hs_batch_kernels.cuh"

namespace {

// tile shape of one batched instance, a function of N and planes alone so that
// an instance's arithmetic never depends on the rest of the batch.  planes == 0:
// an instance large enough to fill the GPU by itself with tiles of at least 8
// planes takes the single-instance slab layout (the FP64 operator's, whose
// cost model counts waves over SLAB_SLOTS); a smaller one takes C, R with the
// fewest positions loaded per node and the depth at which it would fill
// SLAB_SLOTS tiles, within 8..32.  planes > 0: those C, R and min(N+1, planes).
Part batch_part(int N, int planes) {
    const long long NN = N + 1;
    if (planes < 1 && slab_layout(N).CX >= 8) return make_part(N);
    long long bestC = NN, bestR = 1, best_cost = -1;
    const long long cmin = NN < 30 ? NN : 30;
    for (long long C = cmin; C <= NN; ++C) {
        const long long Cw = C + 2;
        const long long Rmax = SPOS / Cw - 2;
        if (Rmax < 1) break;
        const long long R = Rmax < NN ? Rmax : NN;
        const long long NCB = (NN + C - 1) / C, NRB = (NN + R - 1) / R;
        const long long cost = NCB * NRB * (Cw * (R + 2) + 2 * (C + 1) * (R + 1));
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; bestC = C; bestR = R; }
    }
    const long long tyz = ((NN + bestC - 1) / bestC) * ((NN + bestR - 1) / bestR);
    long long depth = planes;
    if (planes < 1) {
        depth = (NN * tyz + SLAB_SLOTS - 1) / SLAB_SLOTS;
        depth = depth < 8 ? 8 : (depth > 32 ? 32 : depth);
    }
    const long long CX = depth < NN ? depth : NN;
    Part p{};
    p.N = N; p.NN = (int)NN;
    p.C = (int)bestC; p.R = (int)bestR; p.CX = (int)CX;
    p.Cw = p.C + 2; p.Rw = p.R + 2;
    p.NCB = (int)((NN + bestC - 1) / bestC); p.NRB = (int)((NN + bestR - 1) / bestR); p.NXB = (int)((NN + CX - 1) / CX);
    p.ntiles = (long long)p.NCB * p.NRB * p.NXB; p.nblk = p.ntiles;
    p.Nn = NN * NN * NN;
    p.nflat = (p.Nn + (long long)RT * KF - 1) / ((long long)RT * KF);
    return p;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct hs_batch {
    hs_batch_options opt{};
    cudaStream_t s = nullptr;
    struct Slot {
        bool used = false;
        int N = 0;
        double dt = 0;
        int steps_left = 0, steps_done = 0;
        int flip_step = -1, flip_bit = 0;   // armed level-G flip (T[flip_idx] before step flip_step)
        long long flip_idx = 0;
        hs_batch_fault fault{};             // armed vector fault (level 5/6/7, FP32 inner vectors)
        Part part{};
        void* mem = nullptr;      // one allocation holding every buffer of the instance
        BInst desc{};
        bool in_step = false;     // part of the step in flight
        bool held = false;        // removed while a step was in flight: reusable after it ends
    };
    std::vector<Slot> slots;
    DevBuf<BInst> d_inst;
    DevBuf<BState> d_st;
    DevBuf<int> d_t2i, d_f2i;
    DevBuf<double> pa, pf;
    DevBuf<double> sq, spart;     // set-up reductions of hs_batch_add
    cudaMemPool_t pool = nullptr; // instance arenas: stream-ordered, kept reserved for reuse
    cudaStream_t s_add = nullptr; // set-up of added instances, overlapping a step in flight
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool inflight = false;        // hs_batch_step_begin without its hs_batch_step_end
    long long cap_tiles = 0, cap_flat = 0;
    bool dirty = true;            // maps / descriptors need an upload
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long long graph_tiles = -1, graph_flat = -1;
    ~hs_batch() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (Slot& sl : slots) if (sl.mem) cudaFreeAsync(sl.mem, s);
        if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
        if (s_add) { cudaStreamSynchronize(s_add); cudaStreamDestroy(s_add); }
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (pool) cudaMemPoolDestroy(pool);
    }
};

namespace {

void set_bsmem() {
    static bool done = false;
    if (done) return;
    done = true;
    cudaFuncSetAttribute(kb_apply<double, BK_RESID>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(BSlabSmem<double>));
    cudaFuncSetAttribute(kb_apply<double, BK_RHS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(BSlabSmem<double>));
    cudaFuncSetAttribute(kb_apply<float, BK_LOOP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(BSlabSmem<float>));
}

BatchArgs batch_args(hs_batch* b) {
    BatchArgs a{};
    a.inst = b->d_inst.p; a.tile2inst = b->d_t2i.p; a.flat2inst = b->d_f2i.p;
    a.n_inst = (int)b->slots.size();
    a.ntiles = b->cap_tiles; a.nflat = b->cap_flat;
    a.pa = b->pa.p; a.pf = b->pf.p;
    a.rtol = b->opt.rtol; a.inner_tol = b->opt.inner_tol;
    a.max_outer = b->opt.max_outer; a.max_inner = b->opt.max_inner;
    a.detect = b->opt.detect;
    a.extrapolate = b->opt.extrapolate;
    return a;
}

// compact the live instances' tile and block ranges; grow the capacity (and
// drop the graph) when they no longer fit; upload maps and descriptors
hs_status upload(hs_batch* b) {
    long long nt = 0, nf = 0;
    for (auto& sl : b->slots) if (sl.used) { nt += sl.part.ntiles; nf += sl.part.nflat; }
    if (nt > b->cap_tiles || nf > b->cap_flat || !b->d_t2i.p) {
        b->cap_tiles = std::max<long long>({nt, 2 * b->cap_tiles, 1024});
        b->cap_flat = std::max<long long>({nf, 2 * b->cap_flat, 1024});
        HS_CUDA(b->d_t2i.alloc(b->cap_tiles));
        HS_CUDA(b->d_f2i.alloc(b->cap_flat));
        // compensated partials: (hi, lo) per quantity
        HS_CUDA(b->pa.alloc((size_t)2 * MAXQ * b->cap_tiles));
        HS_CUDA(b->pf.alloc((size_t)2 * 4 * b->cap_flat));
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    }
    std::vector<int> t2i(b->cap_tiles, -1), f2i(b->cap_flat, -1);
    std::vector<BInst> desc(b->slots.size());
    long long t0 = 0, f0 = 0;
    for (size_t i = 0; i < b->slots.size(); ++i) {
        auto& sl = b->slots[i];
        BInst d = sl.desc;
        d.active = 0;
        if (sl.used) {
            d.tile0 = t0; d.flat0 = f0;
            for (long long t = 0; t < sl.part.ntiles; ++t) t2i[t0 + t] = (int)i;
            for (long long f = 0; f < sl.part.nflat; ++f) f2i[f0 + f] = (int)i;
            t0 += sl.part.ntiles; f0 += sl.part.nflat;
            d.active = sl.steps_left > 0 ? 1 : 0;
        }
        sl.desc.tile0 = d.tile0; sl.desc.flat0 = d.flat0;
        desc[i] = d;
    }
    HS_CUDA(cudaMemcpyAsync(b->d_t2i.p, t2i.data(), t2i.size() * sizeof(int), cudaMemcpyHostToDevice, b->s));
    HS_CUDA(cudaMemcpyAsync(b->d_f2i.p, f2i.data(), f2i.size() * sizeof(int), cudaMemcpyHostToDevice, b->s));
    HS_CUDA(cudaMemcpyAsync(b->d_inst.p, desc.data(), desc.size() * sizeof(BInst), cudaMemcpyHostToDevice, b->s));
    HS_CUDA(cudaStreamSynchronize(b->s));
    b->dirty = false;
    return HS_OK;
}

// outer-iteration tail: r = b - A T, test, start of the next inner solve
void enqueue_resid(hs_batch* b, const BatchArgs& a) {
    kb_apply<double, BK_RESID><<<(int)a.ntiles, ST, sizeof(BSlabSmem<double>), b->s>>>(a);
    kb_final_apply<BK_RESID><<<a.n_inst, RT, 0, b->s>>>(a);
    kb_resid<<<(int)a.nflat, RT, 0, b->s>>>(a);
    kb_outer_final<<<a.n_inst, RT, 0, b->s>>>(a);
}

hs_status build_batch_graph(hs_batch* b) {
    if (b->gexec) return HS_OK;
    const BatchArgs a = batch_args(b);
    cudaGraph_t g;
    HS_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle c_out, c_in;
    HS_CUDA(cudaGraphConditionalHandleCreate(&c_out, g, 0, cudaGraphCondAssignDefault));
    // prologue: step state, b = M T, first residual and test
    cudaGraph_t pre;
    HS_CUDA(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
    kb_step_begin<<<(a.n_inst + 127) / 128, 128, 0, b->s>>>(a);
    kb_apply<double, BK_RHS><<<(int)a.ntiles, ST, sizeof(BSlabSmem<double>), b->s>>>(a);
    kb_final_apply<BK_RHS><<<a.n_inst, RT, 0, b->s>>>(a);
    kb_extrapolate<<<(int)a.nflat, RT, 0, b->s>>>(a);
    enqueue_resid(b, a);
    kb_cond<0><<<1, 1024, 0, b->s>>>(a, c_out, nullptr);
    HS_CUDA(cudaStreamEndCapture(b->s, &pre));
    cudaGraphNode_t n_pre;
    HS_CUDA(cudaGraphAddChildGraphNode(&n_pre, g, nullptr, 0, pre));
    cudaGraphDestroy(pre);
    // outer loop
    cudaGraphNodeParams po{};
    po.type = cudaGraphNodeTypeConditional;
    po.conditional.handle = c_out;
    po.conditional.type = cudaGraphCondTypeWhile;
    po.conditional.size = 1;
    cudaGraphNode_t n_out;
    HS_CUDA(cudaGraphAddNode(&n_out, g, &n_pre, 1, &po));
    cudaGraph_t obody = po.conditional.phGraph_out[0];
    HS_CUDA(cudaGraphConditionalHandleCreate(&c_in, obody, 0, cudaGraphCondAssignDefault));
    cudaGraph_t ohead;
    HS_CUDA(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
    kb_cond<1><<<1, 1024, 0, b->s>>>(a, c_in, nullptr);
    HS_CUDA(cudaStreamEndCapture(b->s, &ohead));
    cudaGraphNode_t n_head;
    HS_CUDA(cudaGraphAddChildGraphNode(&n_head, obody, nullptr, 0, ohead));
    cudaGraphDestroy(ohead);
    cudaGraphNodeParams pi{};
    pi.type = cudaGraphNodeTypeConditional;
    pi.conditional.handle = c_in;
    pi.conditional.type = cudaGraphCondTypeWhile;
    pi.conditional.size = 1;
    cudaGraphNode_t n_in;
    HS_CUDA(cudaGraphAddNode(&n_in, obody, &n_head, 1, &pi));
    cudaGraph_t ibody = pi.conditional.phGraph_out[0];
    HS_CUDA(cudaStreamBeginCaptureToGraph(b->s, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    // four inner iterations per pass (an instance that is done skips them), one condition
    for (int u = 0; u < 4; ++u) {
        kb_apply<float, BK_LOOP><<<(int)a.ntiles, ST, sizeof(BSlabSmem<float>), b->s>>>(a);
        kb_final_apply<BK_LOOP><<<a.n_inst, RT, 0, b->s>>>(a);
        kb_update32<<<(int)a.nflat, RT, 0, b->s>>>(a);
        kb_final_update32<<<a.n_inst, RT, 0, b->s>>>(a);
    }
    kb_cond<1><<<1, 1024, 0, b->s>>>(a, c_in, nullptr);
    HS_CUDA(cudaStreamEndCapture(b->s, &ibody));
    cudaGraph_t otail;
    HS_CUDA(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
    kb_correct<<<(int)a.nflat, RT, 0, b->s>>>(a);
    kb_count_bad<<<(a.n_inst + 127) / 128, 128, 0, b->s>>>(a);
    enqueue_resid(b, a);
    kb_cond<0><<<1, 1024, 0, b->s>>>(a, c_out, nullptr);
    HS_CUDA(cudaStreamEndCapture(b->s, &otail));
    cudaGraphNode_t n_tail;
    HS_CUDA(cudaGraphAddChildGraphNode(&n_tail, obody, &n_in, 1, otail));
    cudaGraphDestroy(otail);
    HS_CUDA(cudaGraphInstantiate(&b->gexec, g, 0));
    b->graph = g;
    return HS_OK;
}

// One step as direct launches with the loop conditions read back by the host
// (HS_GRAPH=0: profilers cannot attribute kernels inside conditional nodes).
// Both loops stay bounded by max_outer / max_inner through the same flags.
hs_status step_direct(hs_batch* b) {
    const BatchArgs a = batch_args(b);
    DevBuf<int> flag;
    HS_CUDA(flag.alloc(2));
    int host_flag = 0;
    auto read = [&](int i) -> hs_status {
        HS_CUDA(cudaMemcpyAsync(&host_flag, flag.p + i, sizeof(int), cudaMemcpyDeviceToHost, b->s));
        HS_CUDA(cudaStreamSynchronize(b->s));
        return HS_OK;
    };
    kb_step_begin<<<(a.n_inst + 127) / 128, 128, 0, b->s>>>(a);
    kb_apply<double, BK_RHS><<<(int)a.ntiles, ST, sizeof(BSlabSmem<double>), b->s>>>(a);
    kb_final_apply<BK_RHS><<<a.n_inst, RT, 0, b->s>>>(a);
    kb_extrapolate<<<(int)a.nflat, RT, 0, b->s>>>(a);
    enqueue_resid(b, a);
    kb_cond<0><<<1, 1024, 0, b->s>>>(a, 0, flag.p);
    for (;;) {
        if (read(0) != HS_OK) return HS_ERR_CUDA;
        if (!host_flag) break;
        kb_cond<1><<<1, 1024, 0, b->s>>>(a, 0, flag.p + 1);
        for (;;) {
            if (read(1) != HS_OK) return HS_ERR_CUDA;
            if (!host_flag) break;
            kb_apply<float, BK_LOOP><<<(int)a.ntiles, ST, sizeof(BSlabSmem<float>), b->s>>>(a);
            kb_final_apply<BK_LOOP><<<a.n_inst, RT, 0, b->s>>>(a);
            kb_update32<<<(int)a.nflat, RT, 0, b->s>>>(a);
            kb_final_update32<<<a.n_inst, RT, 0, b->s>>>(a);
            kb_cond<1><<<1, 1024, 0, b->s>>>(a, 0, flag.p + 1);
        }
        kb_correct<<<(int)a.nflat, RT, 0, b->s>>>(a);
        kb_count_bad<<<(a.n_inst + 127) / 128, 128, 0, b->s>>>(a);
        enqueue_resid(b, a);
        kb_cond<0><<<1, 1024, 0, b->s>>>(a, 0, flag.p);
    }
    HS_CUDA(cudaGetLastError());
    return HS_OK;
}

}  // namespace

extern "C" {

void hs_batch_default_options(hs_batch_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->rtol = 1e-8; o->inner_tol = 1e-4; o->max_outer = 10; o->max_inner = 500;
    o->detect = 1; o->tile_planes = 0; o->device = 0; o->extrapolate = 1;
}

hs_status hs_batch_create(const hs_batch_options* opt, hs_batch** out) {
    if (!opt || !out) { set_error("bad arguments"); return HS_ERR_ARG; }
    *out = nullptr;
    if (!(opt->rtol > 0) || !(opt->inner_tol > 0) || opt->max_outer < 1 || opt->max_inner < 1 ||
        opt->tile_planes < 0) {
        set_error("hs_batch_create: rtol, inner_tol > 0; max_outer, max_inner >= 1; tile_planes >= 0");
        return HS_ERR_ARG;
    }
    HS_CUDA(cudaSetDevice(opt->device));
    auto b = std::make_unique<hs_batch>();
    b->opt = *opt;
    HS_CUDA(cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking));
    HS_CUDA(cudaStreamCreateWithFlags(&b->s_add, cudaStreamNonBlocking));
    HS_CUDA(cudaEventCreate(&b->ev0));
    HS_CUDA(cudaEventCreate(&b->ev1));
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = opt->device;
    HS_CUDA(cudaMemPoolCreate(&b->pool, &pp));
    uint64_t keep = UINT64_MAX;     // freed arenas stay with the pool for the next instances
    HS_CUDA(cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    int no = 0;                     // an add never waits on the step stream for a freed arena
    HS_CUDA(cudaMemPoolSetAttribute(b->pool, cudaMemPoolReuseAllowInternalDependencies, &no));
    set_bsmem();
    *out = b.release();
    return HS_OK;
}

void hs_batch_destroy(hs_batch* b) {
    if (!b) return;
    cudaSetDevice(b->opt.device);
    delete b;
}

}  // extern "C"

namespace {
// An instance from host coefficient arrays (k, rhoc) or, when gen is set, from
// a lognormal field generated on the device into the instance's arrays.
hs_status batch_add_impl(hs_batch* b, int N, double dt, const double* k, const double* rhoc, const FieldSpecDev* gen,
                         const double* T0, int n_steps, int* slot_out) {
    HS_CUDA(cudaSetDevice(b->opt.device));
    const long long NN = N + 1, Nn = NN * NN * NN, Ne = (long long)N * N * N;
    if (!gen)
        for (long long e = 0; e < Ne; ++e)
            if (!(k[e] > 0) || !(rhoc[e] > 0)) { set_error("hs_batch_add: non-positive coefficient"); return HS_ERR_ARG; }
    const RefMatrices mats = build_reference_matrices(N);
    if (!mats.ok) { set_error("reference-matrix self-check failed"); return HS_ERR_MATRIX; }
    // slot
    // A free slot is inactive in the descriptors of any step in flight (a slot
    // removed during that step is held until it ends), so its state may be
    // written on s_add while the step runs.  Growing the slot arrays replaces
    // what the step reads: it waits for the step first.
    int slot = -1;
    for (size_t i = 0; i < b->slots.size(); ++i)
        if (!b->slots[i].used && !b->slots[i].held) { slot = (int)i; break; }
    if (slot < 0) {
        HS_CUDA(cudaStreamSynchronize(b->s));
        slot = (int)b->slots.size();
        b->slots.emplace_back();
        // descriptor and state arrays follow the slot count (the graph reads n_inst)
        DevBuf<BInst> ni;
        DevBuf<BState> ns;
        HS_CUDA(ni.alloc(b->slots.size()));
        HS_CUDA(ns.alloc(b->slots.size()));
        HS_CUDA(cudaMemsetAsync(ns.p, 0, b->slots.size() * sizeof(BState), b->s));
        if (b->d_st.p)
            HS_CUDA(cudaMemcpyAsync(ns.p, b->d_st.p, (b->slots.size() - 1) * sizeof(BState), cudaMemcpyDeviceToDevice, b->s));
        HS_CUDA(cudaStreamSynchronize(b->s));
        std::swap(b->d_inst.p, ni.p); std::swap(b->d_inst.n, ni.n);
        std::swap(b->d_st.p, ns.p); std::swap(b->d_st.n, ns.n);
        for (size_t i = 0; i < b->slots.size(); ++i) b->slots[i].desc.st = b->d_st.p + i;
        if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    }
    hs_batch::Slot& sl = b->slots[slot];
    // one allocation: FP64 node vectors T b y r wA wM diag, coefficients, FP32 vectors
    const size_t v8 = align256(Nn * 8), v4 = align256(Nn * 4), e16 = align256(Ne * 16), e8 = align256(Ne * 8),
                 e8b = align256(Ne * 8);
    const size_t bytes = 8 * v8 + e16 + e8 + 2 * e8b + 7 * v4;
    void* mem = nullptr;
    cudaStream_t sa = b->s_add;
    HS_CUDA(cudaMallocFromPoolAsync(&mem, bytes, b->pool, sa));
    char* q = (char*)mem;
    auto take = [&](size_t n) { char* r = q; q += n; return r; };
    BInst d{};
    d.T = (double*)take(v8); d.b = (double*)take(v8); d.y64 = (double*)take(v8); d.r64 = (double*)take(v8);
    d.Tm1 = (double*)take(v8);
    double* wA = (double*)take(v8); double* wM = (double*)take(v8); double* diag = (double*)take(v8);
    d.coef64 = (const double2*)take(e16); d.coef32 = (const float2*)take(e8);
    double* rh = (double*)take(e8b); double* kk = (double*)take(e8b);
    d.dinv32 = (const float*)take(v4);
    d.r32 = (float*)take(v4); d.z32 = (float*)take(v4); d.p32a = (float*)take(v4); d.p32b = (float*)take(v4);
    d.Ap32 = (float*)take(v4); d.d32 = (float*)take(v4);
    d.wA = wA; d.wM = wM;
    d.dt = dt;
    for (int j = 0; j < 4; ++j) { d.cm[j] = mats.cm[j]; d.ck[j] = mats.ck[j]; d.cmf[j] = (float)mats.cm[j]; d.ckf[j] = (float)mats.ck[j]; }
    d.st = b->d_st.p + slot;
    // coefficients (interleaved on the device), initial field
    const int gn = (int)std::min<long long>((Nn + RT - 1) / RT, 1 << 30);
    const long long nflat = (Nn + (long long)RT * KF - 1) / ((long long)RT * KF);
    if (!b->sq.p) HS_CUDA(b->sq.alloc(4));
    if (b->spart.n < (size_t)(2 * nflat)) HS_CUDA(b->spart.alloc(2 * nflat));   // s_add is its only user
    if (gen) {
        // the field on the device (the partials and the two moments reuse the set-up scratch)
        HS_CUDA(enqueue_field_lognormal(*gen, kk, rh, b->spart.p, b->sq.p, sa));
    } else {
        HS_CUDA(cudaMemcpyAsync(rh, rhoc, Ne * 8, cudaMemcpyHostToDevice, sa));
        HS_CUDA(cudaMemcpyAsync(kk, k, Ne * 8, cudaMemcpyHostToDevice, sa));
    }
    if (T0) HS_CUDA(cudaMemcpyAsync(d.T, T0, Nn * 8, cudaMemcpyHostToDevice, sa));
    else HS_CUDA(cudaMemsetAsync(d.T, 0, Nn * 8, sa));
    k_pack_coef<<<grid_for(Ne, RT), RT, 0, sa>>>(Ne, rh, kk, (double2*)d.coef64, (float2*)d.coef32);
    // diagonal, ABFT weights and their norms (node-parallel operator, FP64)
    ElemConsts ec{};
    std::memcpy(ec.M, mats.M, sizeof(ec.M)); std::memcpy(ec.K, mats.K, sizeof(ec.K));
    std::memcpy(ec.cm, mats.cm, sizeof(ec.cm)); std::memcpy(ec.ck, mats.ck, sizeof(ec.ck));
    ec.detJ = mats.detJ;
    GenArgs ga{};
    ga.N = N; ga.kind = GEN_DIAG; ga.project = 1; ga.dt_eff = dt; ga.y = diag; ga.rhoc = rh; ga.kc = kk;
    ga.ec = ec; ga.fi_elem = -1;
    k_apply_nodes<FORM_WHT><<<gn, RT, 0, sa>>>(ga);
    k_recip32<<<gn, RT, 0, sa>>>(Nn, diag, (float*)d.dinv32);
    k_ones_interior<<<gn, RT, 0, sa>>>(N, d.r64);
    GenArgs gw = ga;
    gw.kind = GEN_APPLY; gw.project = 0; gw.x = d.r64;
    gw.dt_eff = 0.0; gw.y = wM;
    k_apply_nodes<FORM_WHT><<<gn, RT, 0, sa>>>(gw);
    gw.dt_eff = dt; gw.y = wA;
    k_apply_nodes<FORM_WHT><<<gn, RT, 0, sa>>>(gw);
    RedArgs r1{Nn, nflat, N, RED_DOT, wM, wM, b->spart.p, nullptr, nullptr};
    k_reduce<<<(int)nflat, RT, 0, sa>>>(r1);
    k_final_reduce<<<1, RT, 0, sa>>>(b->spart.p, nflat, b->sq.p);
    RedArgs r2{Nn, nflat, N, RED_DOT, wA, wA, b->spart.p, nullptr, nullptr};
    k_reduce<<<(int)nflat, RT, 0, sa>>>(r2);
    k_final_reduce<<<1, RT, 0, sa>>>(b->spart.p, nflat, b->sq.p + 2);
    kb_init_state<<<1, 1, 0, sa>>>(b->d_st.p + slot, b->sq.p);
    HS_CUDA(cudaGetLastError());
    // the caller's host arrays are free again once this returns
    HS_CUDA(cudaStreamSynchronize(sa));
    sl.used = true; sl.N = N; sl.dt = dt; sl.steps_left = n_steps; sl.steps_done = 0;
    sl.part = batch_part(N, b->opt.tile_planes);
    d.part = sl.part;
    sl.mem = mem;
    sl.desc = d;
    b->dirty = true;
    if (slot_out) *slot_out = slot;
    return HS_OK;
}
}  // namespace

extern "C" {

hs_status hs_batch_add(hs_batch* b, int N, double dt, const double* k, const double* rhoc, const double* T0,
                       int n_steps, int* slot_out) {
    if (!b || N < 1 || N > 1200 || !(dt > 0) || !k || !rhoc || n_steps < 0) {
        set_error("hs_batch_add: bad arguments");
        return HS_ERR_ARG;
    }
    return batch_add_impl(b, N, dt, k, rhoc, nullptr, T0, n_steps, slot_out);
}

hs_status hs_batch_add_lognormal(hs_batch* b, int N, double dt, double mu, double sigma, double L,
                                 unsigned long long seed, double rhoc, const double* T0, int n_steps, int* slot_out) {
    if (!b || N < 1 || N > 1200 || !(dt > 0) || !(sigma >= 0) || !(L > 0) || !(rhoc > 0) || n_steps < 0) {
        set_error("hs_batch_add_lognormal: bad arguments");
        return HS_ERR_ARG;
    }
    const FieldSpecDev f{N, mu, sigma, L, rhoc, seed};
    return batch_add_impl(b, N, dt, nullptr, nullptr, &f, T0, n_steps, slot_out);
}

hs_status hs_batch_arm_flip(hs_batch* b, int slot, int step, long long idx, int bit) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used || step < 0 || idx < 0 ||
        bit < 0 || bit > 63) {
        set_error("hs_batch_arm_flip: bad arguments");
        return HS_ERR_ARG;
    }
    auto& sl = b->slots[slot];
    sl.flip_step = step; sl.flip_idx = idx % sl.part.Nn; sl.flip_bit = bit;
    return HS_OK;
}

hs_status hs_batch_arm_fault(hs_batch* b, int slot, const hs_batch_fault* f) {
    if (!b || !f || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used || f->step < 0 ||
        f->outer < 1 || f->iter < 0 || f->idx < 0 || f->bit < 0 || f->bit > 31 ||
        (f->level != HS_FI_P && f->level != HS_FI_RV && f->level != HS_FI_AP)) {
        set_error("hs_batch_arm_fault: level 5/6/7, step >= 0, outer >= 1, iter >= 0, bit 0..31");
        return HS_ERR_ARG;
    }
    auto& sl = b->slots[slot];
    sl.fault = *f;
    sl.fault.idx = f->idx % sl.part.Nn;
    return HS_OK;
}

hs_status hs_batch_remove(hs_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) {
        set_error("hs_batch_remove: no such instance");
        return HS_ERR_ARG;
    }
    HS_CUDA(cudaSetDevice(b->opt.device));
    auto& sl = b->slots[slot];
    HS_CUDA(cudaFreeAsync(sl.mem, b->s));      // after every step already queued
    sl = hs_batch::Slot{};
    sl.held = b->inflight;
    sl.desc.st = b->d_st.p + slot;
    b->dirty = true;
    return HS_OK;
}

hs_status hs_batch_step_begin(hs_batch* b, int* n_active) {
    if (!b) { set_error("bad arguments"); return HS_ERR_ARG; }
    if (b->inflight) { set_error("hs_batch_step_begin: a step is already in flight"); return HS_ERR_ARG; }
    HS_CUDA(cudaSetDevice(b->opt.device));
    int act = 0;
    for (auto& sl : b->slots) {
        sl.in_step = sl.used && sl.steps_left > 0;
        act += sl.in_step ? 1 : 0;
    }
    if (n_active) *n_active = act;
    if (act == 0) return HS_OK;
    // activity follows the steps left: refresh the descriptors when it changes
    for (auto& sl : b->slots) if (sl.used && sl.desc.active != (sl.in_step ? 1 : 0)) b->dirty = true;
    if (b->dirty) {
        hs_status st = upload(b);
        if (st != HS_OK) return st;
        for (auto& sl : b->slots) sl.desc.active = sl.in_step ? 1 : 0;
    }
    const bool graph = graphs_enabled();
    hs_status st = graph ? build_batch_graph(b) : HS_OK;
    if (st != HS_OK) return st;
    // armed flips of this step (level G: one bit of the field before the step)
    for (auto& sl : b->slots) {
        if (!sl.in_step) continue;
        if (sl.flip_step == sl.steps_done) k_flip<<<1, 1, 0, b->s>>>(sl.desc.T, sl.flip_idx, sl.flip_bit);
        if (sl.fault.level && sl.fault.step == sl.steps_done)
            kb_arm<<<1, 1, 0, b->s>>>(sl.desc.st, sl.fault.level, sl.fault.outer, sl.fault.iter, sl.fault.idx,
                                      sl.fault.bit);
    }
    HS_CUDA(cudaEventRecord(b->ev0, b->s));
    if (graph) {
        HS_CUDA(cudaGraphLaunch(b->gexec, b->s));
    } else {
        st = step_direct(b);
        if (st != HS_OK) return st;
    }
    HS_CUDA(cudaEventRecord(b->ev1, b->s));
    b->inflight = true;
    return HS_OK;
}

hs_status hs_batch_step_end(hs_batch* b, int* n_stepped, double* device_ms) {
    if (!b) { set_error("bad arguments"); return HS_ERR_ARG; }
    if (n_stepped) *n_stepped = 0;
    if (device_ms) *device_ms = 0.0;
    if (!b->inflight) return HS_OK;            // nothing was launched
    HS_CUDA(cudaSetDevice(b->opt.device));
    b->inflight = false;
    HS_CUDA(cudaEventSynchronize(b->ev1));
    HS_CUDA(cudaGetLastError());
    int n = 0;
    for (auto& sl : b->slots) {
        sl.held = false;
        if (!sl.in_step) continue;
        if (sl.fault.level && sl.fault.step == sl.steps_done) kb_arm<<<1, 1, 0, b->s>>>(sl.desc.st, 0, 0, 0, 0, 0);
        --sl.steps_left; ++sl.steps_done; ++n;
        sl.in_step = false;
    }
    float ms = 0.f;
    HS_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    if (n_stepped) *n_stepped = n;
    if (device_ms) *device_ms = ms;
    return HS_OK;
}

hs_status hs_batch_step(hs_batch* b, int* n_active, double* device_ms) {
    if (device_ms) *device_ms = 0.0;
    hs_status st = hs_batch_step_begin(b, n_active);
    if (st != HS_OK) return st;
    return hs_batch_step_end(b, nullptr, device_ms);
}

hs_status hs_batch_info(hs_batch* b, int slot, hs_batch_inst_info* out) {
    if (!b || !out || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) {
        set_error("hs_batch_info: no such instance");
        return HS_ERR_ARG;
    }
    HS_CUDA(cudaSetDevice(b->opt.device));
    BState st{};
    HS_CUDA(cudaMemcpyAsync(&st, b->d_st.p + slot, sizeof(st), cudaMemcpyDeviceToHost, b->s));
    HS_CUDA(cudaStreamSynchronize(b->s));
    const auto& sl = b->slots[slot];
    std::memset(out, 0, sizeof(*out));
    out->N = sl.N; out->steps_done = sl.steps_done; out->steps_left = sl.steps_left;
    out->inner_iters = st.inner_total; out->outer_iters = st.outer_total;
    out->applies32 = st.applies32; out->applies64 = st.applies64;
    out->rel_residual = st.rel64; out->d1_max64 = st.d1_max64; out->d1_max32 = st.d1_max32;
    out->tiles = sl.part.ntiles;
    out->fault_fired = st.fi_fired; out->stalls = st.stalls; out->inner_faults = st.inner_faults;
    return HS_OK;
}

hs_status hs_batch_get_field(hs_batch* b, int slot, double* T_host) {
    if (!b || !T_host || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) {
        set_error("hs_batch_get_field: no such instance");
        return HS_ERR_ARG;
    }
    HS_CUDA(cudaSetDevice(b->opt.device));
    const auto& sl = b->slots[slot];
    HS_CUDA(cudaMemcpyAsync(T_host, sl.desc.T, sl.part.Nn * 8, cudaMemcpyDeviceToHost, b->s));
    HS_CUDA(cudaStreamSynchronize(b->s));
    return HS_OK;
}

}  // extern "C"
