// batch_host.cu -- scdat_batch: many independent scenarios (each a scdat_ctx with its own mesh,
// species and particles) advanced together.  One step is: zero the accumulators, three push
// passes each launched once over every (scenario, species) job, charge finalisation and
// right-hand side over every scenario, the mixed-form field solve with its refinement and
// PCG loops controlled on the device, then potentials, nodal field and tet records.  The step
// is captured once as a CUDA graph whose two loops are conditional WHILE nodes, so a step is
// one graph launch with no host round trip; scdat_batch_tuning chooses the launch shapes and
// scdat_batch_autotune times the candidates on the live batch.
#include "batch.cuh"
#include "ctx.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>

using namespace scdat;

namespace {

struct DeferBufs {
    DBuf<uint32_t> idx[2];
    DBuf<int> it[2];
    DBuf<double> rem[2], vs[2];
};

struct MapBufs {
    DBuf<int> ctx_of, first;
    BlockMap view{};
};

// Blocks per scenario in proportion to its share of `sizes` (at least one each).
int build_map(MapBufs& m, const std::vector<int64_t>& sizes, int target, cudaStream_t st)
{
    const int n = (int)sizes.size();
    double tot = 0.0;
    for (int64_t v : sizes) tot += (double)std::max<int64_t>(v, 1);
    std::vector<int> first((size_t)n + 1, 0), of;
    for (int k = 0; k < n; ++k) {
        int b = (int)std::floor((double)target * (double)std::max<int64_t>(sizes[k], 1) / tot + 0.5);
        b = std::max(1, std::min(b, target));
        first[k + 1] = first[k] + b;
        for (int i = 0; i < b; ++i) of.push_back(k);
    }
    if (m.ctx_of.upload(of.data(), of.size(), st) != cudaSuccess) return SCDAT_ERR_CUDA;
    if (m.first.upload(first.data(), first.size(), st) != cudaSuccess) return SCDAT_ERR_CUDA;
    m.view = BlockMap{m.ctx_of.p, m.first.p, first[n]};
    return SCDAT_OK;
}

}  // namespace

struct scdat_batch {
    std::string err;
    std::vector<scdat_ctx*> ctx;
    std::vector<std::pair<int, int>> job_of;  // push job -> (scenario, species)
    std::vector<std::unique_ptr<DeferBufs>> defer;
    DBuf<unsigned> dcount;
    DBuf<PushJob> pjobs;
    DBuf<FieldJob> fjobs;
    DBuf<int64_t> prefix;
    DBuf<unsigned> pass_ctr;  // work counters of the three push passes
    DBuf<PcgScalars> sco;
    DBuf<int> any;
    DBuf<unsigned long long> passes;  // [outer passes, inner double-iterations]
    int* any_host = nullptr;
    MapBufs nodes, rows, tets;
    scdat_batch_tuning tune{};
    int nsm = 148;
    cudaStream_t st = nullptr, st2 = nullptr, st3 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_ready = false;
    int64_t steps = 0;
    double last_step_ms = 0.0;

    // Drains the batch's streams before anything is released (work still in flight writes into
    // the contexts' buffers), then lets the contexts go.
    ~scdat_batch()
    {
        for (cudaStream_t s : {st, st2, st3})
            if (s) cudaStreamSynchronize(s);
        release_graph();
        if (any_host) cudaFreeHost(any_host);
        for (cudaStream_t s : {st, st2, st3})
            if (s) cudaStreamDestroy(s);
        for (scdat_ctx* c : ctx) --c->batch_refs;
    }
    void release_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        graph_ready = false;
    }
};

#define BCK(call)                                                          \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) {                                           \
            b->err = std::string(#call) + ": " + cudaGetErrorString(e_);  \
            return SCDAT_ERR_CUDA;                                         \
        }                                                                  \
    } while (0)

namespace {

// Job tables from the contexts' current buffers (particle arrays move when a context sorts).
int upload_jobs(scdat_batch* b)
{
    std::vector<PushJob> pj;
    std::vector<FieldJob> fj;
    for (size_t j = 0; j < b->job_of.size(); ++j) {
        scdat_ctx* c = b->ctx[b->job_of[j].first];
        const int s = b->job_of[j].second;
        const int64_t N = c->hm.N;
        PushJob J{};
        J.M = c->mv;
        J.P = store_of(c, s);
        J.S = species_dev(c, s);
        J.pp = push_params(c, true);
        J.A = ChargeAcc{c->acc_l0.p + s * N, nullptr, nullptr};  // batched contexts are all mixed: one word
        J.L = c->led.p;
        J.ke_acc = c->ke_acc.p;
        DeferBufs& d = *b->defer[j];
        const unsigned cap = (unsigned)d.idx[0].n;
        J.D1 = DeferList{b->dcount.p + 2 * j, cap, d.idx[0].p, d.it[0].p, d.rem[0].p, d.vs[0].p};
        J.D2 = DeferList{b->dcount.p + 2 * j + 1, cap, d.idx[1].p, d.it[1].p, d.rem[1].p, d.vs[1].p};
        pj.push_back(J);
    }
    for (size_t k = 0; k < b->ctx.size(); ++k) {
        scdat_ctx* c = b->ctx[k];
        FieldJob F{};
        F.A = c->pv;
        F.N = c->hm.N;
        F.T = c->hm.T;
        F.S = (int)c->species.size();
        F.l0 = c->acc_l0.p;
        F.l1 = nullptr;
        F.h = nullptr;
        F.ke_acc = c->ke_acc.p;
        F.vmax = c->vmax.p;
        F.led_active = &c->led.p->active;
        F.lsq_bad = &c->led.p->lsq_bad;
        F.uq = c->uq;
        F.rho = c->rho.p;
        F.totq = c->totq.p;
        F.phi = c->phi.p;
        F.sign = (double)c->prm.poisson_charge_sign;
        F.b = c->b.p;
        F.x = c->x.p;
        F.r = c->r.p;
        F.rf = c->rf.p;
        F.xf = c->xf.p;
        F.zf = c->zf.p;
        F.pf = c->pf.p;
        F.pnf = c->pnf.p;
        F.qf = c->qf.p;
        F.qq = reinterpret_cast<float*>(c->q.p);
        F.sc = c->sc.p;
        F.sco = b->sco.p + k;
        F.part = c->part.p;
        F.rtol = c->prm.pcg_rtol;
        F.max_iter = c->prm.pcg_max_iter;
        F.lsq_reg = 0.0;
        F.xyz = c->xyz.p;
        F.gptr = c->gptr.p;
        F.gcol = c->gcol.p;
        F.E = c->E.p;
        F.Ef = c->Ef.p;
        F.tet = c->tet.p;
        F.trec = c->trec.p;
        F.surf = c->surface ? c->surf.p : nullptr;
        F.led = c->led.p;
        F.dt = c->prm.dt;
        F.surf_node = c->surf_node.p;
        F.surf_mask = c->surf_mask.p;
        F.surf_n = (int64_t)c->surf_node.n;
        fj.push_back(F);
    }
    BCK(cudaMemcpyAsync(b->pjobs.p, pj.data(), sizeof(PushJob) * pj.size(), cudaMemcpyHostToDevice, b->st));
    BCK(cudaMemcpyAsync(b->fjobs.p, fj.data(), sizeof(FieldJob) * fj.size(), cudaMemcpyHostToDevice, b->st));
    return SCDAT_OK;
}

int build_maps(scdat_batch* b)
{
    std::vector<int64_t> nn, rr, tt;
    for (scdat_ctx* c : b->ctx) {
        nn.push_back(c->hm.N);
        rr.push_back(c->pv.R);
        tt.push_back(c->hm.T);
    }
    int rc = build_map(b->nodes, nn, b->nsm * b->tune.field_blocks_per_sm, b->st);
    if (!rc) rc = build_map(b->rows, rr, b->nsm * b->tune.field_blocks_per_sm, b->st);
    if (!rc) rc = build_map(b->tets, tt, b->nsm * b->tune.field_blocks_per_sm, b->st);
    if (rc) b->err = "block map upload failed";
    return rc;
}

// The step as launches on stream s.  With graph handles (cond_outer/cond_inner != 0) the
// loops are conditional nodes added by the caller; without them the host drives the loops.
void enqueue_front(scdat_batch* b, cudaStream_t s)
{
    const int nj = (int)b->job_of.size(), nc = (int)b->ctx.size();
    launch_batch_zero(b->fjobs.p, b->pjobs.p, nc, nj, b->nsm * 2, s);
    const int grid = b->nsm * b->tune.push_blocks_per_sm;
    for (int pass = 1; pass <= 3; ++pass) {
        launch_batch_prefix(b->pjobs.p, nj, pass, b->prefix.p, b->pass_ctr.p, s);
        launch_push_mixed_batch(b->pjobs.p, nj, b->prefix.p, b->pass_ctr.p, pass, grid, s);
    }
    launch_batch_surface(b->fjobs.p, nc, s);
    launch_batch_finalize_rhs(b->fjobs.p, b->nodes.view, b->rows.view, s);
    launch_batch_pcg_mixed_prologue(b->fjobs.p, b->rows.view, nc, s);
}

void enqueue_back(scdat_batch* b, cudaStream_t s)
{
    launch_batch_epilogue(b->fjobs.p, b->nodes.view, b->rows.view, b->tets.view, b->pjobs.p, (int)b->job_of.size(), s);
}

int read_any(scdat_batch* b)
{
    BCK(cudaMemcpyAsync(b->any_host, b->any.p, sizeof(int), cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    return *b->any_host;
}

// one step with host-driven loops (no graph)
int step_eager(scdat_batch* b)
{
    const int nc = (int)b->ctx.size();
    enqueue_front(b, b->st);
    for (int outer = 0; outer < 13; ++outer) {
        launch_batch_outer_begin(b->fjobs.p, b->rows.view, nc, 0ull, b->any.p, b->st);
        int a = read_any(b);
        if (a < 0) return SCDAT_ERR_CUDA;
        while (a) {
            for (int k = 0; k < 8; ++k) launch_batch_inner_iter2(b->fjobs.p, b->rows.view, nc, 0ull, b->any.p, b->passes.p, b->st);
            a = read_any(b);
            if (a < 0) return SCDAT_ERR_CUDA;
        }
        launch_batch_outer_end(b->fjobs.p, b->rows.view, nc, 0ull, b->any.p, b->passes.p, b->st);
        a = read_any(b);
        if (a < 0) return SCDAT_ERR_CUDA;
        if (!a) break;
    }
    enqueue_back(b, b->st);
    BCK(cudaGetLastError());
    return SCDAT_OK;
}

// Adds a WHILE conditional node after the current capture point of `s` and returns its body.
int add_while(scdat_batch* b, cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t* body)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    BCK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    BCK(cudaGraphAddNode(&node, g, deps, nd, &cp));
    *body = cp.conditional.phGraph_out[0];
    BCK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return SCDAT_OK;
}

int capture_graph(scdat_batch* b)
{
    b->release_graph();
    const int nc = (int)b->ctx.size();
    BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    enqueue_front(b, b->st);
    cudaStreamCaptureStatus cs;
    cudaGraph_t top = nullptr;
    BCK(cudaStreamGetCaptureInfo(b->st, &cs, nullptr, &top, nullptr, nullptr));
    cudaGraphConditionalHandle h_out;
    BCK(cudaGraphConditionalHandleCreate(&h_out, top, 1, cudaGraphCondAssignDefault));
    cudaGraph_t obody = nullptr;
    int rc = add_while(b, b->st, h_out, &obody);
    if (rc) return rc;
    {
        BCK(cudaStreamBeginCaptureToGraph(b->st2, obody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cudaGraphConditionalHandle h_in;
        BCK(cudaGraphConditionalHandleCreate(&h_in, obody, 1, cudaGraphCondAssignDefault));
        launch_batch_outer_begin(b->fjobs.p, b->rows.view, nc, (unsigned long long)h_in, nullptr, b->st2);
        cudaGraph_t ibody = nullptr;
        rc = add_while(b, b->st2, h_in, &ibody);
        if (rc) return rc;
        BCK(cudaStreamBeginCaptureToGraph(b->st3, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        launch_batch_inner_iter2(b->fjobs.p, b->rows.view, nc, (unsigned long long)h_in, nullptr, b->passes.p, b->st3);
        BCK(cudaStreamEndCapture(b->st3, &ibody));
        launch_batch_outer_end(b->fjobs.p, b->rows.view, nc, (unsigned long long)h_out, nullptr, b->passes.p, b->st2);
        BCK(cudaStreamEndCapture(b->st2, &obody));
    }
    enqueue_back(b, b->st);
    BCK(cudaStreamEndCapture(b->st, &b->graph));
    BCK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_ready = true;
    return SCDAT_OK;
}

int sync_contexts(scdat_batch* b)
{
    for (scdat_ctx* c : b->ctx) BCK(cudaStreamSynchronize(c->st));
    return SCDAT_OK;
}

// host-side bookkeeping after n steps: counters, solver statistics, re-sorting
int after_steps(scdat_batch* b, int n)
{
    BCK(cudaStreamSynchronize(b->st));
    std::vector<PcgScalars> o(b->ctx.size());
    BCK(cudaMemcpy(o.data(), b->sco.p, sizeof(PcgScalars) * o.size(), cudaMemcpyDeviceToHost));
    bool resorted = false;
    for (size_t k = 0; k < b->ctx.size(); ++k) {
        scdat_ctx* c = b->ctx[k];
        c->last_pcg_iter = o[k].iter;
        c->last_pcg_rel = std::sqrt(o[k].rr / (o[k].bb > 0.0 ? o[k].bb : 1.0));
        const int64_t before = c->steps;
        c->steps += n;
        c->sim_time += n * c->prm.dt;
        const int si = c->prm.sort_interval;
        if (si > 0 && c->steps / si != before / si) {
            for (int s = 0; s < (int)c->species.size(); ++s) {
                if (!species_sorts_now(c, s)) continue;
                int rc = do_sort(c, s);
                if (rc) {
                    b->err = c->err;
                    return rc;
                }
            }
            resorted = true;
        }
        int rc = check_flags(c);
        if (rc) {
            b->err = c->err;
            return rc;
        }
    }
    return resorted ? upload_jobs(b) : SCDAT_OK;
}

}  // namespace

extern "C" {

SCDAT_API void scdat_batch_default_tuning(scdat_batch_tuning* t)
{
    if (!t) return;
    t->push_blocks_per_sm = 4;
    t->field_blocks_per_sm = 8;
    t->use_graph = 1;
    t->pad = 0;
}

SCDAT_API int scdat_batch_create(int32_t n, scdat_ctx* const* ctxs, scdat_batch** out)
{
    if (!out) return SCDAT_ERR_ARG;
    *out = nullptr;
    if (n <= 0 || !ctxs) return SCDAT_ERR_ARG;
    scdat_batch* b = new scdat_batch();
    *out = b;  // on failure the caller reads scdat_batch_last_error and destroys it
    int njobs = 0;
    for (int k = 0; k < n; ++k) {
        scdat_ctx* c = ctxs[k];
        if (!c || !c->mixed || c->species.empty()) {
            b->err = "every scenario must be a mixed-precision context with species set";
            return SCDAT_ERR_STATE;
        }
        b->ctx.push_back(c);
        ++c->batch_refs;
        njobs += (int)c->species.size();
    }
    if (njobs > kMaxBatchJobs) {
        b->err = "more than 1024 (scenario, species) jobs in one batch";
        return SCDAT_ERR_CAPACITY;
    }
    scdat_batch_default_tuning(&b->tune);
    b->nsm = b->ctx[0]->nsm;
    BCK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    BCK(cudaStreamCreateWithFlags(&b->st2, cudaStreamNonBlocking));
    BCK(cudaStreamCreateWithFlags(&b->st3, cudaStreamNonBlocking));
    BCK(cudaMallocHost((void**)&b->any_host, sizeof(int)));
    for (int k = 0; k < n; ++k) {
        scdat_ctx* c = b->ctx[k];
        for (int s = 0; s < (int)c->species.size(); ++s) {
            b->job_of.emplace_back(k, s);
            auto d = std::make_unique<DeferBufs>();
            const size_t cap = (size_t)std::max<int64_t>(c->species[s].cap, 1) / 4 + 4096;
            for (int l = 0; l < 2; ++l) {
                BCK(d->idx[l].alloc(cap));
                BCK(d->it[l].alloc(cap));
                BCK(d->rem[l].alloc(cap));
                BCK(d->vs[l].alloc(cap));
            }
            b->defer.push_back(std::move(d));
        }
    }
    BCK(b->dcount.alloc(2 * (size_t)njobs));
    BCK(b->pjobs.alloc((size_t)njobs));
    BCK(b->fjobs.alloc((size_t)n));
    BCK(b->prefix.alloc((size_t)njobs + 1));
    BCK(b->pass_ctr.alloc(3));
    BCK(b->sco.alloc((size_t)n));
    BCK(cudaMemsetAsync(b->sco.p, 0, sizeof(PcgScalars) * n, b->st));
    BCK(b->any.alloc(1));
    BCK(b->passes.alloc(2));
    BCK(cudaMemsetAsync(b->passes.p, 0, 2 * sizeof(unsigned long long), b->st));
    int rc = sync_contexts(b);
    if (rc) return rc;
    // the inner-solve scalars start with their reduction tickets at zero
    for (scdat_ctx* c : b->ctx) BCK(cudaMemsetAsync(c->sc.p, 0, sizeof(PcgScalars), b->st));
    rc = upload_jobs(b);
    if (!rc) rc = build_maps(b);
    if (rc) return rc;
    BCK(cudaStreamSynchronize(b->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_batch_destroy(scdat_batch* b)
{
    delete b;
    return SCDAT_OK;
}

SCDAT_API const char* scdat_batch_last_error(const scdat_batch* b) { return b ? b->err.c_str() : "null batch"; }

SCDAT_API int scdat_batch_set_tuning(scdat_batch* b, const scdat_batch_tuning* t)
{
    if (!b || !t) return SCDAT_ERR_ARG;
    // each field block writes one reduction partial per scenario (grid_red slots); push launches
    // keep the same bound (8 blocks per SM, twice what is resident)
    const int push_max = b->ctx[0]->grid_push / b->nsm, field_max = b->ctx[0]->grid_red / b->nsm;
    if (t->push_blocks_per_sm < 1 || t->push_blocks_per_sm > push_max || t->field_blocks_per_sm < 1 ||
        t->field_blocks_per_sm > field_max) {
        b->err = "tuning out of range (push and field 1..8 blocks per SM)";
        return SCDAT_ERR_ARG;
    }
    const bool maps = t->field_blocks_per_sm != b->tune.field_blocks_per_sm;
    b->tune = *t;
    b->release_graph();
    if (maps) {
        int rc = build_maps(b);
        if (rc) return rc;
        BCK(cudaStreamSynchronize(b->st));
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_batch_get_tuning(const scdat_batch* b, scdat_batch_tuning* t)
{
    if (!b || !t) return SCDAT_ERR_ARG;
    *t = b->tune;
    return SCDAT_OK;
}

SCDAT_API int scdat_batch_step(scdat_batch* b, int32_t n_steps)
{
    if (!b) return SCDAT_ERR_ARG;
    if (n_steps < 0) {
        b->err = "negative step count";
        return SCDAT_ERR_ARG;
    }
    if (n_steps == 0) return SCDAT_OK;
    int rc = sync_contexts(b);
    if (!rc) rc = upload_jobs(b);
    if (rc) return rc;
    if (b->tune.use_graph && !b->graph_ready) {
        rc = capture_graph(b);
        if (rc) {
            cudaStreamCaptureStatus cs;
            if (cudaStreamIsCapturing(b->st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(b->st, &g);
                if (g) cudaGraphDestroy(g);
            }
            cudaGetLastError();
            return rc;
        }
    }
    // steps run in runs that end where some context re-sorts (host work between graph launches)
    int done = 0;
    while (done < n_steps) {
        int run = n_steps - done;
        for (scdat_ctx* c : b->ctx) {
            const int si = c->prm.sort_interval;
            if (si > 0) run = std::min<int64_t>(run, si - (c->steps % si));
        }
        StageEvents ev;
        BCK(cudaEventCreate(&ev.e0));
        BCK(cudaEventCreate(&ev.e1));
        BCK(cudaEventRecord(ev.e0, b->st));
        for (int k = 0; k < run; ++k) {
            if (b->tune.use_graph) {
                BCK(cudaGraphLaunch(b->exec, b->st));
            } else {
                rc = step_eager(b);
                if (rc) return rc;
            }
        }
        BCK(cudaEventRecord(ev.e1, b->st));
        BCK(cudaEventSynchronize(ev.e1));
        float ms = 0.f;
        BCK(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
        b->last_step_ms = ms / run;
        rc = after_steps(b, run);
        if (rc) return rc;
        done += run;
        b->steps += run;
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_batch_stream(const scdat_batch* b, void** stream)
{
    if (!b || !stream) return SCDAT_ERR_ARG;
    *stream = (void*)b->st;
    return SCDAT_OK;
}

// Kernels of this library launched by the steps so far: 16 per step plus 6 per refinement
// pass and 5 per inner double-iteration (the loop passes are counted on the device).
SCDAT_API int scdat_batch_kernel_launches(scdat_batch* b, int64_t* launches)
{
    if (!b || !launches) return SCDAT_ERR_ARG;
    unsigned long long p[2] = {0, 0};
    BCK(cudaMemcpy(p, b->passes.p, sizeof(p), cudaMemcpyDeviceToHost));
    *launches = 16 * b->steps + 6 * (int64_t)p[0] + 5 * (int64_t)p[1];
    return SCDAT_OK;
}

SCDAT_API int scdat_batch_last_step_ms(const scdat_batch* b, double* ms)
{
    if (!b || !ms) return SCDAT_ERR_ARG;
    *ms = b->last_step_ms;
    return SCDAT_OK;
}

// Tries each candidate launch shape for `steps_each` real steps of the batch and keeps the
// fastest (the steps advance the scenarios like any other steps).
SCDAT_API int scdat_batch_autotune(scdat_batch* b, int32_t steps_each, scdat_batch_tuning* chosen)
{
    if (!b || steps_each < 1) return SCDAT_ERR_ARG;
    const int push_c[] = {2, 4, 8};
    const int field_c[] = {4, 8};
    scdat_batch_tuning best = b->tune;
    double best_ms = 1e300;
    for (int fb : field_c)
        for (int pb : push_c) {
            scdat_batch_tuning t = b->tune;
            t.push_blocks_per_sm = pb;
            t.field_blocks_per_sm = fb;
            int rc = scdat_batch_set_tuning(b, &t);
            if (!rc) rc = scdat_batch_step(b, steps_each);
            if (rc) return rc;
            if (b->last_step_ms < best_ms) {
                best_ms = b->last_step_ms;
                best = t;
            }
        }
    int rc = scdat_batch_set_tuning(b, &best);
    if (rc) return rc;
    if (chosen) *chosen = best;
    return SCDAT_OK;
}

}  // extern "C"
