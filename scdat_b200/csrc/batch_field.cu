// batch_field.cu -- the field half of the batched step: charge finalisation, right-hand side,
// the mixed-form solve (FP32-SpMV PCG inside FP64 refinement) and the nodal field, each one
// launch over all scenarios.  Every block runs a single-scenario body (field_kern.cuh) on
// its scenario's arrays; the loop control of the solve is on the device (per-scenario
// convergence flags, and CUDA-graph conditional handles when the step is captured).
#include "batch.cuh"
#include "field_kern.cuh"

namespace scdat {

__device__ __forceinline__ int map_ctx(const BlockMap& m, Grid& g)
{
    const int k = m.ctx_of[blockIdx.x];
    g.b = blockIdx.x - m.first[k];
    g.n = m.first[k + 1] - m.first[k];
    return k;
}

__device__ __forceinline__ void set_cond(unsigned long long h, unsigned v)
{
    if (h) cudaGraphSetConditional((cudaGraphConditionalHandle)h, v);
}

// Zero the per-step accumulators of every scenario: charge limbs, per-block kinetic-energy
// partials, the active count and the defer-list counts.
__global__ void k_batch_zero(const FieldJob* __restrict__ jobs, const PushJob* __restrict__ pjobs, int npjobs)
{
    const FieldJob& J = jobs[blockIdx.y];
    const int64_t nl = (int64_t)J.S * J.N;
    unsigned long long* l0 = J.l0;
    unsigned long long* l1 = J.l1;
    unsigned long long* h = J.h;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nl; i += (int64_t)gridDim.x * blockDim.x) {
        l0[i] = 0ull;
        if (l1) {  // limb layout (the precision form uses l0 alone)
            l1[i] = 0ull;
            h[i] = 0ull;
        }
    }
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            J.ke_acc[0] = 0ull;
            J.ke_acc[1] = 0ull;
            *J.led_active = 0ull;
            J.totq[0] = 0ull;
            J.totq[1] = 0ull;
            *J.lsq_bad = 0ull;
        }
        for (int s = threadIdx.x; s < J.S; s += blockDim.x) {  // the null-collision speed bound
            J.vmax[2 * s] = J.vmax[2 * s + 1];
            J.vmax[2 * s + 1] = 0u;
        }
        if (blockIdx.y == 0)
            for (int j = threadIdx.x; j < npjobs; j += blockDim.x) {
                *pjobs[j].D1.count = 0u;
                *pjobs[j].D2.count = 0u;
            }
    }
}

// one block per scenario: its surface circuit's step (face charges -> potentials -> nodes)
__global__ void k_batch_surface(const FieldJob* __restrict__ jobs)
{
    const FieldJob& J = jobs[blockIdx.x];
    if (!J.surf) return;
    if (threadIdx.x < J.surf->n) surface_advance_face(J.surf, J.led, threadIdx.x, J.uq, J.dt);
    __syncthreads();
    for (int64_t i = threadIdx.x; i < J.surf_n; i += blockDim.x)
        if (J.surf_mask[i]) J.phi[J.surf_node[i]] = surface_node_potential(J.surf, J.surf_mask[i]);
}

__global__ void k_batch_finalize(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    k_finalize_rho_body(J.N, J.S, J.l0, J.l1, J.h, J.uq, J.rho, J.totq, J.totq + 1, g);
}

__global__ void k_batch_rhs(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    k_gather_rows_body(J.A, J.phi, J.x, g);
    k_rhs_body(J.A, J.rho, J.phi, J.sign, J.b, g);
}

// one thread per scenario: a fresh refinement loop
__global__ void k_batch_prologue(const FieldJob* __restrict__ jobs, int njobs)
{
    for (int k = threadIdx.x; k < njobs; k += blockDim.x) {
        PcgScalars* o = jobs[k].sco;
        o->iter = 0;
        o->outer = 0;  // outer iterations
        o->done = jobs[k].A.R > 0 ? 0 : 1;
        o->rtol = jobs[k].rtol;
        o->max_iter = jobs[k].max_iter;
    }
}

// FP64 residual r = b - A x and its norms into the outer scalars
__global__ void k_batch_residual(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    if (J.sco->done) return;
    k_residual64_body(J.A, J.b, J.x, J.r, J.rf, J.sco, J.part, g);
}

// One thread per scenario: converged, out of iterations or out of refinement passes ends the
// scenario's loop; otherwise start an FP32 solve of A e = r to the tolerance this pass needs.  Sets the inner loop's
// condition to "some scenario still solving" (run_pcg_mixed in capi.cu is the same loop
// driven from the host).
__global__ void k_batch_inner_setup(const FieldJob* __restrict__ jobs, int njobs, unsigned long long cond,
                                    int* any_out)
{
    int active = 0;
    for (int k = threadIdx.x; k < njobs; k += blockDim.x) {
        PcgScalars* o = jobs[k].sco;
        if (o->done) continue;
        const double bb = o->bb > 0.0 ? o->bb : 1.0;
        if (o->rr <= o->rtol * o->rtol * bb || o->iter >= o->max_iter || o->outer >= kMaxRefinePasses) {
            o->done = 1;
            continue;
        }
        PcgScalars* s = jobs[k].sc;
        s->rtol = inner_rtol(o->rr, bb, o->rtol);
        s->max_iter = max(1, o->max_iter - o->iter);
        s->abs_thr2 = 0.0;
        s->done = 0;
        s->iter = 0;
        active = 1;
    }
    active = __syncthreads_or(active);
    if (threadIdx.x == 0) {
        set_cond(cond, active ? 1u : 0u);
        if (any_out) *any_out = active;
    }
}

__global__ void k_batch_zero_xf(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    if (J.sco->done) return;
    k_zero_f32_body(J.A.R, J.xf, g);
}

__global__ void k_batch_inner_init(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    if (J.sco->done) return;
    k_pcg_init_body<float>(J.A, J.A.valf, J.rf, J.xf, J.qf, J.zf, J.sc, J.part, g);
}

template <int ODD>
__global__ void k_batch_spmv32(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    if (J.sco->done) return;
    if (ODD)
        k_pcg_spmv_body<float>(J.A, J.A.valf, J.zf, J.pnf, J.pf, J.qq, J.sc, J.part, g);
    else
        k_pcg_spmv_body<float>(J.A, J.A.valf, J.zf, J.pf, J.pnf, J.qq, J.sc, J.part, g);
}

template <int ODD>
__global__ void k_batch_update32(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    if (J.sco->done) return;
    k_pcg_update_body<float>(J.A, J.xf, ODD ? J.pf : J.pnf, J.qf, J.qq, J.zf, J.sc, J.part, g);
}

__global__ void k_batch_inner_check(const FieldJob* __restrict__ jobs, int njobs, unsigned long long cond,
                                    int* any_out, unsigned long long* passes)
{
    int active = 0;
    for (int k = threadIdx.x; k < njobs; k += blockDim.x)
        if (!jobs[k].sco->done && !jobs[k].sc->done) active = 1;
    active = __syncthreads_or(active);
    if (threadIdx.x == 0) {
        set_cond(cond, active ? 1u : 0u);
        if (any_out) *any_out = active;
        passes[1] += 1ull;
    }
}

__global__ void k_batch_add_correction(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    if (J.sco->done) return;
    k_add_correction_body(J.A.R, J.x, J.xf, g);
}

__global__ void k_batch_outer_end(const FieldJob* __restrict__ jobs, int njobs, unsigned long long cond, int* any_out,
                                  unsigned long long* passes)
{
    int active = 0;
    for (int k = threadIdx.x; k < njobs; k += blockDim.x) {
        PcgScalars* o = jobs[k].sco;
        if (o->done) continue;
        o->iter += jobs[k].sc->iter;
        o->outer += 1;
        active = 1;
    }
    active = __syncthreads_or(active);
    if (threadIdx.x == 0) {
        set_cond(cond, active ? 1u : 0u);
        if (any_out) *any_out = active;
        passes[0] += 1ull;
    }
}

__global__ void k_batch_scatter(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    k_scatter_rows_body(J.A, J.x, J.phi, g);
}

__global__ void k_batch_lsq(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    k_lsq_field_body(J.N, J.xyz, J.gptr, J.gcol, J.phi, J.lsq_reg, J.E, J.Ef, J.lsq_bad, g);
}

__global__ void k_batch_zero_if_flag(const FieldJob* __restrict__ jobs, BlockMap m)
{
    Grid g;
    const FieldJob& J = jobs[map_ctx(m, g)];
    k_zero_if_flag_body(3 * J.N, J.E, J.Ef, J.lsq_bad, g);
}

// the step counter that keys the MCC random streams
__global__ void k_batch_advance(PushJob* __restrict__ pjobs, int npjobs)
{
    for (int j = threadIdx.x; j < npjobs; j += blockDim.x) pjobs[j].pp.step += 1u;
}

// ---------------------------------------------------------------------------------------
void launch_batch_zero(const FieldJob* jobs, const PushJob* pjobs, int njobs, int npjobs, int grid, cudaStream_t st)
{
    k_batch_zero<<<dim3(grid, njobs), 256, 0, st>>>(jobs, pjobs, npjobs);
}

void launch_batch_surface(const FieldJob* jobs, int njobs, cudaStream_t st)
{
    k_batch_surface<<<njobs, 256, 0, st>>>(jobs);
}

void launch_batch_finalize_rhs(const FieldJob* jobs, const BlockMap& nodes, const BlockMap& rows, cudaStream_t st)
{
    k_batch_finalize<<<nodes.blocks, 256, 0, st>>>(jobs, nodes);
    k_batch_rhs<<<rows.blocks, 256, 0, st>>>(jobs, rows);
}

void launch_batch_pcg_mixed_prologue(const FieldJob* jobs, const BlockMap&, int njobs, cudaStream_t st)
{
    k_batch_prologue<<<1, 256, 0, st>>>(jobs, njobs);
}

void launch_batch_outer_begin(const FieldJob* jobs, const BlockMap& rows, int njobs, unsigned long long cond_inner,
                              int* any_out, cudaStream_t st)
{
    k_batch_residual<<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_inner_setup<<<1, 1024, 0, st>>>(jobs, njobs, cond_inner, any_out);
    k_batch_zero_xf<<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_inner_init<<<rows.blocks, 256, 0, st>>>(jobs, rows);
}

void launch_batch_inner_iter2(const FieldJob* jobs, const BlockMap& rows, int njobs, unsigned long long cond_inner,
                              int* any_out, unsigned long long* passes, cudaStream_t st)
{
    k_batch_spmv32<0><<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_update32<0><<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_spmv32<1><<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_update32<1><<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_inner_check<<<1, 1024, 0, st>>>(jobs, njobs, cond_inner, any_out, passes);
}

void launch_batch_outer_end(const FieldJob* jobs, const BlockMap& rows, int njobs, unsigned long long cond_outer,
                            int* any_out, unsigned long long* passes, cudaStream_t st)
{
    k_batch_add_correction<<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_outer_end<<<1, 1024, 0, st>>>(jobs, njobs, cond_outer, any_out, passes);
}

void launch_batch_epilogue(const FieldJob* jobs, const BlockMap& nodes, const BlockMap& rows, const BlockMap& tets,
                           PushJob* pjobs, int npjobs, cudaStream_t st)
{
    k_batch_scatter<<<rows.blocks, 256, 0, st>>>(jobs, rows);
    k_batch_lsq<<<nodes.blocks, 256, 0, st>>>(jobs, nodes);
    k_batch_zero_if_flag<<<nodes.blocks, 256, 0, st>>>(jobs, nodes);
    launch_batch_refresh_trec(jobs, tets, st);
    k_batch_advance<<<1, 256, 0, st>>>(pjobs, npjobs);
}

}  // namespace scdat
