// capi.cu -- the scdat_ctx object behind the C ABI in include/scdat_b200.h.
//
// Owns the device copies of the mesh, fields, per-species particle stores and the ledger,
// and sequences one PIC-MCC step on a CUDA stream:
//   clear charge -> push (gather/Boris/relocate/deposit/boundary/MCC) -> finalise charge
//   -> RHS -> PCG -> potentials -> nodal LSQ field
// which is the order of PICCycle::executeTimeStep (PICCycle.cpp:311-416) followed by the
// background MCC step of the reference driver (Main/main_PICcore.cpp:487-515).
#include "ctx.cuh"
#include "mg_setup.h"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace scdat {
void launch_push_f64(const MeshView& M, const ParticleStore& P, const SpeciesDev& S, const PushParams& pp,
                     const DeferList& D1, const DeferList& D2, ChargeAcc A, LedgerDev* L, unsigned long long* ke_acc,
                     unsigned* ctr, int grid, cudaStream_t st);
void launch_mcc_f64(const ParticleStore& P, const SpeciesDev& S, const PushParams& pp, LedgerDev* L, int grid,
                    cudaStream_t st);
void launch_push_mixed(const MeshView& M, const ParticleStore& P, const SortedSource& R, const SpeciesDev& S,
                       const PushParams& pp, const DeferList& D1, const DeferList& D2, ChargeAcc A, LedgerDev* L,
                       unsigned long long* ke_acc, unsigned* ctr, int grid, bool stay_first, cudaStream_t st);
void launch_mcc_mixed(const ParticleStore& P, const SpeciesDev& S, const PushParams& pp, LedgerDev* L, int grid,
                      cudaStream_t st);
void launch_refresh_erec(int64_t T, const int4* tet, const double* E, double* erec, cudaStream_t st);
void launch_refresh_trec(int64_t T, const int4* tet, const double* E, float* trec, cudaStream_t st);
void launch_to_mixed(const MeshView& M, int64_t n, const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz, const ParticleStore& P, cudaStream_t st);
void launch_from_mixed(const MeshView& M, int64_t n, const ParticleStore& P, double* x, double* y, double* z,
                       double* vx, double* vy, double* vz, cudaStream_t st);
void launch_seed_box(const int32_t* hex_ijk, int64_t ncell, int32_t ppc, int32_t S_total, int32_t s, double h,
                     double sigma, uint64_t seed, const ParticleStore& P, bool mixed, const MeshView& M,
                     cudaStream_t st);
void launch_seed_tets(const int32_t* tets, int64_t ntet, int32_t per_tet, int32_t S_total, int32_t s, double sigma,
                      const double drift[3], uint64_t seed, const ParticleStore& P, bool mixed, const MeshView& M,
                      cudaStream_t st);
void launch_layer_moments(const ParticleStore& P, int64_t n, bool mixed, const MeshView& M, double z0, double z1,
                          int n_layers, double* cnt, double* v2, cudaStream_t st);
void launch_sort_keys(int64_t n, const int32_t* tet, uint32_t inactive_key, uint32_t* keys, uint32_t* vals,
                      int64_t* active, cudaStream_t st);
template <typename T>
void launch_gather_store(int64_t n, const int64_t* active, const uint32_t* perm, const GatherArrays<T>& in,
                         const GatherArrays<T>& out, cudaStream_t st);
void launch_gather_mixed(int64_t n, const int64_t* active, const uint32_t* perm, const uint32_t* sorted_keys,
                         uint32_t nohint_key, const float4* in_mix, const uint32_t* in_id, float4* out_mix,
                         int32_t* out_tet, uint32_t* out_id, cudaStream_t st);
void launch_scatter_values(int64_t n, const int64_t* idx, const double* v, double* dst, cudaStream_t st);
void launch_rotate_vmax(int S, unsigned* v, cudaStream_t st);
}  // namespace scdat

using namespace scdat;


#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                          \
            return SCDAT_ERR_CUDA;                                                                  \
        }                                                                                           \
    } while (0)

#define ARG(cond, msg)                  \
    do {                                \
        if (!(cond)) {                  \
            ctx->err = msg;             \
            return SCDAT_ERR_ARG;       \
        }                               \
    } while (0)

namespace {

double pow2_ceil(double v)
{
    if (!(v > 0.0) || !std::isfinite(v)) return 1.0;
    int e;
    std::frexp(v, &e);  // v = f * 2^e, f in [0.5, 1)
    return std::ldexp(1.0, e);
}

}  // namespace

namespace scdat {

static ParticleStore store_view(scdat_ctx* ctx, int s)
{
    SpeciesState& S = ctx->species[s];
    ParticleStore P{};
    P.x = S.x.p; P.y = S.y.p; P.z = S.z.p;
    P.vx = S.vx.p; P.vy = S.vy.p; P.vz = S.vz.p;
    P.mix = S.mix.p;
    P.tet = S.tet.p;
    P.id = S.id.p;
    P.count = ctx->counts.p + s;
    return P;
}

// Apply a re-sort still pending on species s (mixed form): one gather of the store through the
// permutation, the tet of each kept particle being its sorted key.
int settle_store(scdat_ctx* ctx, int s)
{
    SpeciesState& S = ctx->species[s];
    if (!S.perm_pending) return SCDAT_OK;
    S.perm_pending = false;
    ++ctx->launches;
    launch_gather_mixed(S.n, ctx->counts.p + s, S.perm.p, S.skey.p, (uint32_t)ctx->hm.T, S.mix.p, S.id.p, S.mix2.p,
                        S.tet2.p, S.id2.p, ctx->st);
    S.mix.swap(S.mix2);
    S.tet.swap(S.tet2);
    S.id.swap(S.id2);
    CK(cudaGetLastError());
    return SCDAT_OK;
}

// The store of species s for any use other than the push (which reads a pending re-sort itself).
ParticleStore store_of(scdat_ctx* ctx, int s)
{
    settle_store(ctx, s);
    return store_view(ctx, s);
}

SpeciesDev species_dev(const scdat_ctx* ctx, int s)
{
    const SpeciesState& S = ctx->species[s];
    SpeciesDev d{};
    d.q = S.sp.charge;
    d.m = S.sp.mass;
    d.w = S.sp.weight;
    d.qm = S.sp.charge / S.sp.mass;
    int nseg = std::min(std::max(ctx->prm.deposit_segments, 1), 128);
    d.cw_seg = (S.sp.charge / (double)nseg) * S.sp.weight;
    d.electron_like = S.sp.electron_like;
    d.mcc_enabled = S.mcc.enabled;
    d.mcc_mode = S.mcc.mode;
    d.mcc_n = S.mcc.target_density;
    d.mcc_sigma = S.mcc.sigma_max;
    d.mcc_eref = S.mcc.e_ref_ev;
    d.mcc_alpha = S.mcc.alpha;
    d.mcc_eth = S.mcc.e_threshold_ev;
    d.vmax = ctx->vmax.p ? ctx->vmax.p + 2 * s : nullptr;
    return d;
}

PushParams push_params(const scdat_ctx* ctx, bool do_mcc)
{
    PushParams pp{};
    pp.dt = ctx->prm.dt;
    pp.floor_ratio = ctx->prm.adaptive_floor_ratio;
    pp.nseg = std::min(std::max(ctx->prm.deposit_segments, 1), 128);
    pp.dep_kernel = ctx->prm.deposit_kernel;
    for (int f = 0; f < 6; ++f) pp.face_bc[f] = ctx->prm.face_bc[f];
    for (int a = 0; a < 3; ++a) {
        bool per = (ctx->prm.face_bc[2 * a] == SCDAT_BC_PERIODIC || ctx->prm.face_bc[2 * a + 1] == SCDAT_BC_PERIODIC);
        double span = ctx->hg.bmax[a] - ctx->hg.bmin[a];
        // PeriodicBoundaryCondition maps every configured axis (x and y in the reference
        // drivers, Main/main_PICcore.cpp:435-448); an axis is periodic when one of its faces is.
        pp.period[a] = per ? span : 0.0;
    }
    pp.body_tally = ctx->prm.body_tally;
    pp.do_mcc = do_mcc ? 1 : 0;
    double sx = std::max(ctx->hg.bmax[0] - ctx->hg.bmin[0], 1e-12), sy = std::max(ctx->hg.bmax[1] - ctx->hg.bmin[1], 1e-12),
           sz = std::max(ctx->hg.bmax[2] - ctx->hg.bmin[2], 1e-12);
    double ms = std::max(sx, std::max(sy, sz));
    pp.otol = std::max(1.0e-10, 1.0e-8 * ms);           // PICCycle.cpp:1238
    pp.ntol = std::max(5.0 * pp.otol, 1.0e-9 * ms);      // PICCycle.cpp:1239
    pp.inv_uq = 1.0 / ctx->uq;
    pp.inv_ue = 1.0 / ctx->ue;
    pp.seed = ctx->prm.seed;
    pp.step = (uint32_t)ctx->steps;
    pp.deposit = 1;
    pp.patches = ctx->surface ? 1 : 0;
    pp.see_model = ctx->see_model;
    pp.see_dmax = ctx->see_dmax;
    pp.see_emax_ev = ctx->see_emax;
    pp.see_sims_n = ctx->see_sims_n;
    pp.see_sims_xm = ctx->see_sims_xm;
    for (int k = 0; k < 4; ++k) pp.see_katz[k] = ctx->see_katz[k];
    for (int a = 0; a < 3; ++a) {
        pp.blo[a] = ctx->body_lo[a];
        pp.bhi[a] = ctx->body_hi[a];
    }
    return pp;
}

int check_flags(scdat_ctx* ctx)
{
    unsigned long long f = 0;
    CK(cudaMemcpyAsync(&f, &ctx->led.p->flags, sizeof(f), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (f & kFlagBadTet) {
        ctx->err = "device flag: invalid tet index seen";
        return SCDAT_ERR_DEVICE_FLAG;
    }
    if (f & kFlagDeferOverflow) {
        ctx->err = "device flag: deferred-particle list overflow";
        return SCDAT_ERR_DEVICE_FLAG;
    }
    return SCDAT_OK;
}

// ---- the stages ----------------------------------------------------------------------
// Pass-1 form of species s for this push (mixed form).  A stay-first pass 1 pays off for a
// species of which few particles leave their tet or need more than one sub-step in a step
// (ions beside electrons of the same temperature); for the others its deferrals cost more than
// the walk code it drops.  Automatic choice: a stay-first probe on the first push and every
// kStayProbe-th, then stay-first while the last probe deferred under kStayMaxFrac of the
// species.  Both forms give bitwise the same result.
constexpr int kStayProbe = 32;
constexpr double kStayMaxFrac = 0.2;

bool stay_first_now(scdat_ctx* ctx, int s)
{
    SpeciesState& S = ctx->species[s];
    if (S.stay_pending) {  // the last stay-first push's deferral count has arrived
        S.stay_frac = S.stay_n > 0 ? (double)ctx->h_deferred[s] / (double)S.stay_n : 1.0;
        S.stay_pending = false;
    }
    bool stay;
    if (S.push_mode == SCDAT_PUSH_WALKING)
        stay = false;
    else if (S.push_mode == SCDAT_PUSH_STAY_FIRST)
        stay = true;
    else
        stay = S.stay_frac < 0.0 || S.pushes % kStayProbe == 0 || S.stay_frac < kStayMaxFrac;
    ++S.pushes;
    if (stay) S.stay_n = S.n;
    return stay;
}

int do_push(scdat_ctx* ctx, bool do_mcc)
{
    const int S = (int)ctx->species.size();
    if (S == 0) {
        ctx->err = "species not set";
        return SCDAT_ERR_STATE;
    }
    const int64_t N = ctx->hm.N;
    CK(cudaMemsetAsync(ctx->acc_l0.p, 0, sizeof(unsigned long long) * S * N, ctx->st));
    if (!ctx->mixed) {  // the precision form accumulates one word per node (fx_red_word)
        CK(cudaMemsetAsync(ctx->acc_l1.p, 0, sizeof(unsigned long long) * S * N, ctx->st));
        CK(cudaMemsetAsync(ctx->acc_h.p, 0, sizeof(unsigned long long) * S * N, ctx->st));
    }
    CK(cudaMemsetAsync(ctx->ke_acc.p, 0, 2 * sizeof(unsigned long long), ctx->st));
    CK(cudaMemsetAsync(&ctx->led.p->active, 0, sizeof(unsigned long long), ctx->st));
    ++ctx->launches;
    launch_rotate_vmax(S, ctx->vmax.p, ctx->st);
    PushParams pp = push_params(ctx, do_mcc);
    StageEvents ev;
    if (ctx->timing) {
        CK(cudaEventCreate(&ev.e0));
        CK(cudaEventCreate(&ev.e1));
        CK(cudaEventRecord(ev.e0, ctx->st));
    }
    for (int s = 0; s < S; ++s) {
        if (ctx->species[s].cap == 0) continue;
        ctx->push_particles += ctx->species[s].n;
        SpeciesState& Ss = ctx->species[s];
        ParticleStore P = store_view(ctx, s);
        SortedSource R{};
        if (Ss.perm_pending) {
            // pass 1 gathers the re-sorted store itself: it reads through the permutation and
            // writes the sorted order into the second buffers, which every pass then uses
            R = SortedSource{Ss.perm.p, Ss.skey.p, (uint32_t)ctx->hm.T, Ss.mix.p, Ss.id.p};
            P.mix = Ss.mix2.p;
            P.tet = Ss.tet2.p;
            P.id = Ss.id2.p;
        }
        SpeciesDev sd = species_dev(ctx, s);
        // defer-list counts [0, 1] and the three passes' work counters [2, 5)
        CK(cudaMemsetAsync(ctx->dcount.p, 0, 5 * sizeof(unsigned), ctx->st));
        DeferList d1{ctx->dcount.p, ctx->d1cap, ctx->d1idx.p, ctx->d1it.p, ctx->d1rem.p, ctx->d1vs.p};
        DeferList d2{ctx->dcount.p + 1, ctx->dcap, ctx->d2idx.p, ctx->d2it.p, ctx->d2rem.p, ctx->d2vs.p};
        ctx->launches += 3;
        ChargeAcc acc = ctx->mixed ? ChargeAcc{ctx->acc_l0.p + s * N, nullptr, nullptr}
                                   : ChargeAcc{ctx->acc_l0.p + s * N, ctx->acc_l1.p + s * N, ctx->acc_h.p + s * N};
        if (ctx->mixed) {
            const bool stay = stay_first_now(ctx, s);
            launch_push_mixed(ctx->mv, P, R, sd, pp, d1, d2, acc, ctx->led.p, ctx->ke_acc.p, ctx->dcount.p + 2,
                              ctx->grid_push, stay, ctx->st);
            if (Ss.perm_pending) {
                Ss.perm_pending = false;
                Ss.mix.swap(Ss.mix2);
                Ss.tet.swap(Ss.tet2);
                Ss.id.swap(Ss.id2);
            }
            if (stay) {
                // pass 1's deferred count, read by the next push's choice (the field solve in
                // between synchronises the stream)
                CK(cudaMemcpyAsync(ctx->h_deferred + s, ctx->dcount.p, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                   ctx->st));
                ctx->species[s].stay_pending = true;
            }
        } else
            launch_push_f64(ctx->mv, P, sd, pp, d1, d2, acc, ctx->led.p, ctx->ke_acc.p, ctx->dcount.p + 2,
                            ctx->grid_push, ctx->st);
    }
    CK(cudaGetLastError());
    if (ctx->timing) {
        CK(cudaEventRecord(ev.e1, ctx->st));
        ev.commit(ctx->ev_push);
        ctx->push_launches += 1;
    }
    CK(cudaMemsetAsync(ctx->totq.p, 0, sizeof(unsigned long long) * 2, ctx->st));
    ++ctx->launches;
    launch_finalize_rho(N, S, ctx->acc_l0.p, ctx->mixed ? nullptr : ctx->acc_l1.p, ctx->mixed ? nullptr : ctx->acc_h.p,
                        ctx->uq, ctx->rho.p, ctx->totq.p,
                        ctx->totq.p + 1, ctx->grid_nodes, ctx->st);
    CK(cudaGetLastError());
    return SCDAT_OK;
}

// copy the nodal field into the per-tet records the push kernels read
int refresh_tet_field(scdat_ctx* ctx)
{
    ++ctx->launches;
    if (ctx->mixed)
        launch_refresh_trec(ctx->hm.T, ctx->tet.p, ctx->E.p, ctx->trec.p, ctx->st);
    else
        launch_refresh_erec(ctx->hm.T, ctx->tet.p, ctx->E.p, ctx->erec.p, ctx->st);
    CK(cudaGetLastError());
    return SCDAT_OK;
}

int do_lsq(scdat_ctx* ctx, double reg)
{
    CK(cudaMemsetAsync(&ctx->led.p->lsq_bad, 0, sizeof(unsigned long long), ctx->st));
    ctx->launches += 2;
    launch_lsq(ctx->hm.N, ctx->xyz.p, ctx->gptr.p, ctx->gcol.p, ctx->phi.p, reg, ctx->E.p, ctx->Ef.p,
               &ctx->led.p->lsq_bad, ctx->grid_nodes, ctx->st);
    CK(cudaGetLastError());
    return refresh_tet_field(ctx);
}

int pcg_scalars_init(scdat_ctx* ctx, double rtol, int max_iter, double abs_thr2)
{
    PcgScalars h{};
    h.rtol = rtol;
    h.max_iter = max_iter;
    h.abs_thr2 = abs_thr2;
    CK(cudaMemcpyAsync(ctx->sc.p, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->st));
    return SCDAT_OK;
}

int read_scalars(scdat_ctx* ctx, PcgScalars& h)
{
    CK(cudaMemcpyAsync(&h, ctx->sc.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

// Multigrid-preconditioned CG on the Dirichlet-reduced system in V's precision, from x: b, x and
// the CG vectors r, z, p, q are R-vectors of the caller.  Blocks until the solve ends.
template <typename V>
int run_mgpcg(scdat_ctx* ctx, const V* b, V* x, V* r, V* z, V* p, V* q, double rtol, int max_iter, PcgScalars& h)
{
    const PoissonView& A = ctx->pv;
    int rc = pcg_scalars_init(ctx, rtol, max_iter, 0.0);
    if (rc) return rc;
    launch_mgpcg_init<V>(A, b, x, r, ctx->sc.p, ctx->part.p, ctx->grid_red, ctx->st);
    launch_vcycle<V>(ctx->mg_plan, r, z, ctx->sc.p, ctx->part.p, ctx->st);
    const int per_cycle = 7 * ((int)ctx->mg_plan.lv.size() - 1) + 1;
    ctx->launches += 1 + per_cycle;
    const int batch = 2;  // iterations queued between convergence reads (kernels after convergence return at once)
    for (int k = 0; k < max_iter; k += batch) {
        for (int j = 0; j < batch; ++j) {
            ctx->launches += 3 + per_cycle;
            launch_mgpcg_iter<V>(A, ctx->mg_plan, x, r, z, p, q, ctx->sc.p, ctx->part.p, ctx->grid_red, ctx->st);
        }
        CK(cudaGetLastError());
        rc = read_scalars(ctx, h);
        if (rc) return rc;
        if (h.done) break;
    }
    if (max_iter <= 0) return read_scalars(ctx, h);
    return SCDAT_OK;
}

int run_pcg64(scdat_ctx* ctx, const double* bvec, double* xvec, double rtol, int max_iter, int& iters,
              double& relres)
{
    const PoissonView& A = ctx->pv;
    if (ctx->precond == SCDAT_PRECOND_MULTIGRID) {
        PcgScalars h{};
        int rc = run_mgpcg<double>(ctx, bvec, xvec, ctx->r.p, ctx->z.p, ctx->p.p, ctx->q.p, rtol, max_iter, h);
        if (rc) return rc;
        iters = h.iter;
        relres = std::sqrt(h.rr / (h.bb > 0.0 ? h.bb : 1.0));
        return SCDAT_OK;
    }
    int rc = pcg_scalars_init(ctx, rtol, max_iter, 0.0);
    if (rc) return rc;
    ++ctx->launches;
    launch_pcg_init64(A, bvec, xvec, ctx->r.p, ctx->z.p, ctx->sc.p, ctx->part.p, ctx->grid_red, ctx->st);
    double* p = ctx->p.p;
    double* pn = ctx->pn.p;
    const int batch = 16;
    PcgScalars h{};
    for (int k = 0; k < max_iter; k += batch) {
        for (int j = 0; j < batch; ++j) {
            ctx->launches += 2;
            launch_pcg_iter64(A, xvec, ctx->r.p, ctx->z.p, p, pn, ctx->q.p, ctx->sc.p, ctx->part.p, ctx->grid_red,
                              ctx->st);
            std::swap(p, pn);
        }
        CK(cudaGetLastError());
        rc = read_scalars(ctx, h);
        if (rc) return rc;
        if (h.done) break;
    }
    if (max_iter <= 0) {
        rc = read_scalars(ctx, h);
        if (rc) return rc;
    }
    iters = h.iter;
    relres = std::sqrt(h.rr / (h.bb > 0.0 ? h.bb : 1.0));
    return SCDAT_OK;
}

// FP32-SpMV PCG inside an FP64 iterative-refinement loop (mixed form).
int run_pcg_mixed(scdat_ctx* ctx, double rtol, int max_iter, int& iters, double& relres)
{
    const PoissonView& A = ctx->pv;
    const int R = A.R;
    iters = 0;
    relres = 0.0;
    PcgScalars h{};
    // every pass ends with the FP64 residual of the corrected x, so relres always describes the
    // returned solution, also when the pass cap ends the loop
    for (int outer = 0;; ++outer) {
        ++ctx->launches;
        launch_residual64(A, ctx->b.p, ctx->x.p, ctx->r.p, ctx->rf.p, ctx->sc.p, ctx->part.p, ctx->grid_red, ctx->st);
        CK(cudaGetLastError());
        int rc = read_scalars(ctx, h);
        if (rc) return rc;
        double bb = h.bb > 0.0 ? h.bb : 1.0;
        relres = std::sqrt(h.rr / bb);
        if (h.rr <= rtol * rtol * bb || iters >= max_iter || outer == kMaxRefinePasses) break;
        // inner FP32 solve A e = r from e = 0, to the tolerance this pass needs
        ctx->launches += 1;
        launch_zero_f32(R, ctx->xf.p, ctx->grid_red, ctx->st);
        if (ctx->precond == SCDAT_PRECOND_MULTIGRID) {
            PcgScalars hi{};
            rc = run_mgpcg<float>(ctx, ctx->rf.p, ctx->xf.p, ctx->qf.p, ctx->zf.p, ctx->pf.p, ctx->pnf.p,
                                  inner_rtol(h.rr, bb, rtol), std::max(1, max_iter - iters), hi);
            if (rc) return rc;
            iters += hi.iter;
            ++ctx->launches;
            launch_add_correction(R, ctx->x.p, ctx->xf.p, ctx->grid_red, ctx->st);
            CK(cudaGetLastError());
            continue;
        }
        ctx->launches += 1;
        rc = pcg_scalars_init(ctx, inner_rtol(h.rr, bb, rtol), std::max(1, max_iter - iters), 0.0);
        if (rc) return rc;
        launch_pcg_init32(A, ctx->rf.p, ctx->xf.p, ctx->qf.p, ctx->zf.p, ctx->sc.p, ctx->part.p, ctx->grid_red,
                          ctx->st);
        // qf doubles as the inner residual vector; the direction buffers are pf/pnf, A*p goes to the
        // inner q buffer below
        float* p = ctx->pf.p;
        float* pn = ctx->pnf.p;
        float* rr = ctx->qf.p;
        float* qq = reinterpret_cast<float*>(ctx->q.p);  // FP64 q buffer is free during the inner solve
        const int batch = 16;
        PcgScalars hi{};
        for (int k = 0; k < max_iter; k += batch) {
            for (int j = 0; j < batch; ++j) {
                ctx->launches += 2;
                launch_pcg_iter32(A, ctx->xf.p, rr, ctx->zf.p, p, pn, qq, ctx->sc.p, ctx->part.p, ctx->grid_red,
                                  ctx->st);
                std::swap(p, pn);
            }
            CK(cudaGetLastError());
            rc = read_scalars(ctx, hi);
            if (rc) return rc;
            if (hi.done) break;
        }
        iters += hi.iter;
        ++ctx->launches;
        launch_add_correction(R, ctx->x.p, ctx->xf.p, ctx->grid_red, ctx->st);
        CK(cudaGetLastError());
    }
    return SCDAT_OK;
}

// Builds the lattice multigrid hierarchy of the context's mesh on the host and uploads it.
int setup_multigrid(scdat_ctx* ctx)
{
    HostMg hmg;
    std::string why = build_multigrid(ctx->hm, ctx->hps, hmg);
    if (!why.empty()) {
        ctx->err = "multigrid preconditioner unavailable: " + why;
        return SCDAT_ERR_ARG;
    }
    cudaStream_t st = ctx->st;
    const size_t vb = ctx->mixed ? sizeof(float) : sizeof(double);
    ctx->mgl.clear();
    MgPlan plan;
    plan.grid_max = ctx->grid_red;
    const int L = (int)hmg.lv.size();
    for (int l = 0; l < L; ++l) {
        const HostMgLevel& H = hmg.lv[l];
        auto D = std::make_unique<MgDevLevel>();
        MgLevelDev v{};
        v.R = H.R;
        v.omega = (float)H.omega;
        if (l == 0) {
            v.row_ptr = ctx->pv.row_ptr;
            v.col = ctx->pv.col;
            v.val = ctx->pv.val;
            v.valf = ctx->pv.valf;
            v.diag = ctx->pv.diag;
            v.diagf = ctx->pv.diagf;
            v.dinv = ctx->pv.dinv;
            v.dinvf = ctx->pv.dinvf;
        } else {
            std::vector<float> valf(H.val.begin(), H.val.end()), diagf(H.diag.begin(), H.diag.end());
            std::vector<double> dinv(H.R);
            std::vector<float> dinvf(H.R);
            for (int r = 0; r < H.R; ++r) {
                dinv[r] = 1.0 / H.diag[r];
                dinvf[r] = (float)dinv[r];
            }
            if (valf.empty()) valf.push_back(0.0f);
            std::vector<double> val = H.val;
            std::vector<int32_t> col = H.col;
            if (val.empty()) {
                val.push_back(0.0);
                col.push_back(0);
            }
            CK(D->row_ptr.upload(H.row_ptr.data(), H.row_ptr.size(), st));
            CK(D->col.upload(col.data(), col.size(), st));
            CK(D->val.upload(val.data(), val.size(), st));
            CK(D->valf.upload(valf.data(), valf.size(), st));
            CK(D->diag.upload(H.diag.data(), H.diag.size(), st));
            CK(D->diagf.upload(diagf.data(), diagf.size(), st));
            CK(D->dinv.upload(dinv.data(), dinv.size(), st));
            CK(D->dinvf.upload(dinvf.data(), dinvf.size(), st));
            CK(cudaStreamSynchronize(st));  // the host vectors above go out of scope
            v.row_ptr = D->row_ptr.p;
            v.col = D->col.p;
            v.val = D->val.p;
            v.valf = D->valf.p;
            v.diag = D->diag.p;
            v.diagf = D->diagf.p;
            v.dinv = D->dinv.p;
            v.dinvf = D->dinvf.p;
        }
        if (l + 1 < L) {
            CK(D->p_ptr.upload(H.p_ptr.data(), H.p_ptr.size(), st));
            CK(D->p_col.upload(H.p_col.data(), H.p_col.size(), st));
            CK(D->p_w.upload(H.p_w.data(), H.p_w.size(), st));
            CK(D->r_ptr.upload(H.r_ptr.data(), H.r_ptr.size(), st));
            CK(D->r_col.upload(H.r_col.data(), H.r_col.size(), st));
            CK(D->r_w.upload(H.r_w.data(), H.r_w.size(), st));
            v.p_ptr = D->p_ptr.p;
            v.p_col = D->p_col.p;
            v.p_w = D->p_w.p;
            v.r_ptr = D->r_ptr.p;
            v.r_col = D->r_col.p;
            v.r_w = D->r_w.p;
        }
        // work vectors, each padded to 256 bytes
        const size_t vbytes = ((size_t)std::max(H.R, 1) * vb + 255) & ~(size_t)255;
        CK(D->work.alloc(5 * vbytes));
        MgWork w{};
        unsigned char* base = D->work.p;
        w.b = base;
        w.xa = base + vbytes;
        w.xb = base + 2 * vbytes;
        w.res = base + 3 * vbytes;
        w.xo = base + 4 * vbytes;
        plan.lv.push_back(v);
        plan.w.push_back(w);
        ctx->mgl.push_back(std::move(D));
    }
    std::vector<float> cf(hmg.coarse_inv.begin(), hmg.coarse_inv.end());
    CK(ctx->mg_cinv.upload(hmg.coarse_inv.data(), hmg.coarse_inv.size(), st));
    CK(ctx->mg_cinvf.upload(cf.data(), cf.size(), st));
    CK(cudaStreamSynchronize(st));
    plan.cinv = ctx->mg_cinv.p;
    plan.cinvf = ctx->mg_cinvf.p;
    ctx->mg_plan = plan;
    return SCDAT_OK;
}

int do_solve_field(scdat_ctx* ctx)
{
    const PoissonView& A = ctx->pv;
    StageEvents ev;
    if (ctx->timing) {
        CK(cudaEventCreate(&ev.e0));
        CK(cudaEventCreate(&ev.e1));
        CK(cudaEventRecord(ev.e0, ctx->st));
    }
    if (A.R > 0) {
        ctx->launches += 3;
        launch_gather_rows(A, ctx->phi.p, ctx->x.p, ctx->grid_red, ctx->st);
        launch_rhs(A, ctx->rho.p, ctx->phi.p, (double)ctx->prm.poisson_charge_sign, ctx->b.p, ctx->grid_red, ctx->st);
        CK(cudaGetLastError());
        int it = 0;
        double rel = 0.0;
        int rc = ctx->mixed ? run_pcg_mixed(ctx, ctx->prm.pcg_rtol, ctx->prm.pcg_max_iter, it, rel)
                            : run_pcg64(ctx, ctx->b.p, ctx->x.p, ctx->prm.pcg_rtol, ctx->prm.pcg_max_iter, it, rel);
        if (rc) return rc;
        ctx->last_pcg_iter = it;
        ctx->last_pcg_rel = rel;
        launch_scatter_rows(A, ctx->x.p, ctx->phi.p, ctx->grid_red, ctx->st);
        CK(cudaGetLastError());
    }
    int rc = do_lsq(ctx, 0.0);
    if (ctx->timing) {
        CK(cudaEventRecord(ev.e1, ctx->st));
        ev.commit(ctx->ev_field);
        ctx->field_solves += 1;
    }
    return rc;
}

int harvest_timing(scdat_ctx* ctx)
{
    CK(cudaStreamSynchronize(ctx->st));
    for (auto& pr : ctx->ev_push) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        ctx->push_ms += ms;
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    ctx->ev_push.clear();
    for (auto& pr : ctx->ev_field) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        ctx->field_ms += ms;
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    ctx->ev_field.clear();
    for (auto& pr : ctx->ev_sort) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        ctx->sort_ms += ms;
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    ctx->ev_sort.clear();
    return SCDAT_OK;
}

// the surface circuit's step: face charges -> face potentials -> Dirichlet values of the
// body's surface nodes for the following field solve
int do_surface(scdat_ctx* ctx)
{
    if (!ctx->surface) return SCDAT_OK;
    ctx->launches += 2;
    launch_surface_advance(ctx->surf.p, ctx->led.p, ctx->uq, ctx->prm.dt, ctx->st);
    launch_surface_apply(ctx->surf.p, (int64_t)ctx->surf_node.n, ctx->surf_node.p, ctx->surf_mask.p, ctx->phi.p,
                         ctx->st);
    CK(cudaGetLastError());
    return SCDAT_OK;
}

}  // namespace scdat

bool species_sorts_now(const scdat_ctx* ctx, int s)
{
    const int si = ctx->species[s].sort_interval > 0 ? ctx->species[s].sort_interval : ctx->prm.sort_interval;
    return si > 0 && ctx->steps % si == 0;
}

namespace scdat {

int do_sort(scdat_ctx* ctx, int s)
{
    SpeciesState& S = ctx->species[s];
    const int64_t n = S.n;
    if (n == 0) return SCDAT_OK;
    int rc = settle_store(ctx, s);  // the keys are read from the store in its current order
    if (rc) return rc;
    const uint32_t inactive = (uint32_t)ctx->hm.T;  // keys: tet, T (no hint), T+1 (inactive)
    int bits = 1;
    while (((uint64_t)1 << bits) <= (uint64_t)inactive + 1) ++bits;
    StageEvents ev;
    if (ctx->timing) {
        CK(cudaEventCreate(&ev.e0));
        CK(cudaEventCreate(&ev.e1));
        CK(cudaEventRecord(ev.e0, ctx->st));
    }
    // the mixed form sorts into the species' own permutation and key buffers and leaves the
    // gather to the next pass 1 (or to settle_store)
    uint32_t* kout = ctx->mixed ? S.skey.p : ctx->kout.p;
    uint32_t* vout = ctx->mixed ? S.perm.p : ctx->vout.p;
    ctx->launches += ctx->mixed ? 1 : 2;  // keys (+ the FP64 form's gather); the radix sort itself is CUB's
    launch_sort_keys(n, S.tet.p, inactive, ctx->kin.p, ctx->vin.p, ctx->nact.p, ctx->st);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ctx->kin.p, kout, ctx->vin.p, vout, (int)n, 0, bits, ctx->st));
    if (tmp > ctx->cub_tmp.n) CK(ctx->cub_tmp.alloc(tmp));
    CK(cub::DeviceRadixSort::SortPairs(ctx->cub_tmp.p, tmp, ctx->kin.p, kout, ctx->vin.p, vout, (int)n, 0, bits,
                                       ctx->st));
    if (ctx->mixed) {
        S.perm_pending = true;
    } else {
        const uint32_t* perm = ctx->vout.p;
        if (ctx->scratchi.n < S.tet.n) CK(ctx->scratchi.alloc(S.tet.n));
        if (ctx->scratchu.n < S.id.n) CK(ctx->scratchu.alloc(S.id.n));
        DBuf<double>* da[6] = {&S.x, &S.y, &S.z, &S.vx, &S.vy, &S.vz};
        GatherArrays<double> in{}, out{};
        for (int a = 0; a < 6; ++a) {
            if (ctx->shadow64[a].n < da[a]->n) CK(ctx->shadow64[a].alloc(da[a]->n));
            in.v[a] = da[a]->p;
            out.v[a] = ctx->shadow64[a].p;
        }
        in.tet = S.tet.p; in.id = S.id.p;
        out.tet = ctx->scratchi.p; out.id = ctx->scratchu.p;
        launch_gather_store<double>(n, ctx->nact.p, perm, in, out, ctx->st);
        for (int a = 0; a < 6; ++a) da[a]->swap(ctx->shadow64[a]);
        S.tet.swap(ctx->scratchi);
        S.id.swap(ctx->scratchu);
    }
    CK(cudaGetLastError());
    if (ctx->timing) {
        CK(cudaEventRecord(ev.e1, ctx->st));
        ev.commit(ctx->ev_sort);
        ctx->sorts += 1;
    }
    int64_t act = 0;
    CK(cudaMemcpyAsync(&act, ctx->nact.p, sizeof(act), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    S.n = act;
    CK(cudaMemcpyAsync(ctx->counts.p + s, &S.n, sizeof(int64_t), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

}  // namespace scdat

// ======================================================================================
// C ABI
// ======================================================================================
namespace {
// reason of the calling thread's last failed scdat_create (its context is gone by then)
thread_local std::string t_create_err;
int create_ctx(const scdat_mesh_desc* mesh, const scdat_params* params, scdat_ctx* ctx);
}  // namespace

extern "C" {

SCDAT_API const char* scdat_version(void) { return "scdat_b200 0.1.0 (sm_100a)"; }

SCDAT_API void scdat_default_params(scdat_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->dt = 0.0;
    p->deposit_kernel = SCDAT_DEP_LINEAR;
    p->deposit_segments = 10;
    p->adaptive_floor_ratio = 0.001;
    p->precision = SCDAT_PREC_FP64;
    p->use_neighbor_lists = 1;
    for (int f = 0; f < 6; ++f) p->face_bc[f] = SCDAT_BC_NONE;
    p->body_tally = 1;
    p->poisson_charge_sign = -1;
    p->pcg_rtol = 1e-8;
    p->pcg_max_iter = 5000;
    p->sort_interval = 0;
    p->particle_capacity = 0;
    p->seed = 0x5CDA7B200ull;
}

SCDAT_API const char* scdat_last_error(const scdat_ctx* ctx)
{
    if (ctx) return ctx->err.c_str();
    return t_create_err.empty() ? "null context" : t_create_err.c_str();
}

SCDAT_API int scdat_create(const scdat_mesh_desc* mesh, const scdat_params* params, scdat_ctx** out)
{
    if (!mesh || !params || !out) {
        t_create_err = "scdat_create: null argument";
        return SCDAT_ERR_ARG;
    }
    *out = nullptr;
    auto holder = std::make_unique<scdat_ctx>();
    const int rc = create_ctx(mesh, params, holder.get());
    if (rc != SCDAT_OK) {
        // the context (its stream and buffers included) is freed here; its reason stays readable
        t_create_err = holder->err.empty() ? std::string("scdat_create failed") : holder->err;
        return rc;
    }
    t_create_err.clear();
    *out = holder.release();
    return SCDAT_OK;
}

}  // extern "C"

namespace {

// The body of scdat_create: fills ctx, or returns an error with ctx->err set.
int create_ctx(const scdat_mesh_desc* mesh, const scdat_params* params, scdat_ctx* ctx)
{
    ARG(mesh->n_nodes > 0 && mesh->n_tets > 0, "empty mesh");
    ARG(mesh->n_nodes < (int64_t)0x7fffffff && mesh->n_tets < (int64_t)0x7fffffff, "mesh too large for int32 indices");
    ARG(mesh->node_xyz && mesh->tet_nodes && mesh->node_dirichlet, "null mesh array");
    ARG(params->dt > 0.0 && std::isfinite(params->dt), "dt must be positive");
    ctx->prm = *params;
    ctx->mixed = params->precision == SCDAT_PREC_MIXED;
    HostMesh& m = ctx->hm;
    m.N = mesh->n_nodes;
    m.T = mesh->n_tets;
    m.xyz.assign(mesh->node_xyz, mesh->node_xyz + 3 * m.N);
    m.tet.assign(mesh->tet_nodes, mesh->tet_nodes + 4 * m.T);
    m.dirichlet.assign(mesh->node_dirichlet, mesh->node_dirichlet + m.N);
    if (mesh->tet_eps_rel) m.eps_rel.assign(mesh->tet_eps_rel, mesh->tet_eps_rel + m.T);
    for (int64_t i = 0; i < 4 * m.T; ++i) ARG(m.tet[i] >= 0 && m.tet[i] < m.N, "tet node index out of range");
    std::string e;
    if (mesh->tet_neighbors) {
        m.nbr.assign(mesh->tet_neighbors, mesh->tet_neighbors + 4 * m.T);
        for (int64_t i = 0; i < 4 * m.T; ++i) ARG(m.nbr[i] >= -1 && m.nbr[i] < m.T, "tet neighbour out of range");
    } else if (!(e = compute_face_neighbors(m, m.nbr)).empty()) {
        ctx->err = e;
        return SCDAT_ERR_ARG;
    }
    if (!(e = compute_geometry(m, ctx->hg)).empty() || !(e = build_locate_grid(m, ctx->hg, ctx->hgrid)).empty() ||
        !(e = build_node_graph(m, ctx->hgr)).empty() || !(e = assemble_poisson(m, ctx->hgr, ctx->hps)).empty()) {
        ctx->err = e;
        return SCDAT_ERR_ARG;
    }
    CK(cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, dev));
    ctx->grid_push = ctx->nsm * 8;
    ctx->grid_nodes = ctx->nsm * 8;
    ctx->grid_red = ctx->nsm * 8;
    cudaStream_t st = ctx->st;
    // mesh
    CK(ctx->xyz.upload(m.xyz.data(), m.xyz.size(), st));
    CK(ctx->geom.upload(ctx->hg.geom.data(), ctx->hg.geom.size(), st));
    CK(ctx->geomf.upload(ctx->hg.geomf.data(), ctx->hg.geomf.size(), st));
    CK(ctx->tet.upload(reinterpret_cast<const int4*>(m.tet.data()), (size_t)m.T, st));
    CK(ctx->nbr.upload(reinterpret_cast<const int4*>(m.nbr.data()), (size_t)m.T, st));
    CK(ctx->bin_start.upload(ctx->hgrid.bin_start.data(), ctx->hgrid.bin_start.size(), st));
    CK(ctx->bin_tets.upload(ctx->hgrid.bin_tets.data(), ctx->hgrid.bin_tets.size(), st));
    CK(ctx->gptr.upload(ctx->hgr.ptr.data(), ctx->hgr.ptr.size(), st));
    CK(ctx->gcol.upload(ctx->hgr.col.data(), ctx->hgr.col.size(), st));
    MeshView& mv = ctx->mv;
    mv.N = m.N;
    mv.T = m.T;
    mv.xyz = ctx->xyz.p;
    mv.tet = ctx->tet.p;
    mv.nbr = ctx->nbr.p;
    if (ctx->mixed) {
        // static words of the 256-byte tet records: J^-1, node ids, neighbours and the origin
        // shifts to them (E refreshed after each field solve)
        std::vector<float> rec((size_t)(64 * m.T), 0.0f);
        for (int64_t t = 0; t < m.T; ++t) {
            float* r = &rec[64 * t];
            for (int k = 0; k < 9; ++k) r[k] = ctx->hg.geomf[12 * t + k];
            for (int k = 0; k < 4; ++k) std::memcpy(&r[24 + k], &m.tet[4 * t + k], sizeof(int32_t));
            for (int k = 0; k < 4; ++k) std::memcpy(&r[28 + k], &m.nbr[4 * t + k], sizeof(int32_t));
            const int64_t o = m.tet[4 * t];
            for (int k = 0; k < 4; ++k) {
                const int32_t nb = m.nbr[4 * t + k];
                std::memcpy(&r[35 + 4 * k], &nb, sizeof(int32_t));  // the walk's (shift, neighbour) float4
                if (nb < 0) continue;
                const int64_t on = m.tet[4 * (int64_t)nb];
                for (int a = 0; a < 3; ++a) r[32 + 4 * k + a] = (float)(m.xyz[3 * o + a] - m.xyz[3 * on + a]);
            }
        }
        CK(ctx->trec.upload(rec.data(), rec.size(), st));
    } else {
        CK(ctx->erec.alloc((size_t)(12 * m.T)));
        CK(cudaMemsetAsync(ctx->erec.p, 0, sizeof(double) * 12 * m.T, st));
    }
    mv.geom = ctx->geom.p;
    mv.geomf = ctx->geomf.p;
    mv.trec = ctx->trec.p;
    mv.erec = ctx->erec.p;
    for (int a = 0; a < 3; ++a) {
        mv.gmin[a] = ctx->hgrid.gmin[a];
        mv.ginv[a] = ctx->hgrid.ginv[a];
        mv.gdim[a] = ctx->hgrid.gdim[a];
        mv.bmin[a] = ctx->hg.bmin[a];
        mv.bmax[a] = ctx->hg.bmax[a];
    }
    mv.gdelta = ctx->hgrid.gdelta;
    mv.bin_start = ctx->bin_start.p;
    mv.bin_tets = ctx->bin_tets.p;
    mv.use_nbr = params->use_neighbor_lists;
    // poisson
    HostPoisson& ps = ctx->hps;
    CK(ctx->row_node.upload(ps.row_node.data(), ps.row_node.size(), st));
    CK(ctx->cv.upload(ps.cv.data(), ps.cv.size(), st));
    CK(ctx->lift_ptr.upload(ps.lift_ptr.data(), ps.lift_ptr.size(), st));
    CK(ctx->lift_node.upload(ps.lift_node.data(), ps.lift_node.size(), st));
    CK(ctx->lift_val.upload(ps.lift_val.data(), ps.lift_val.size(), st));
    CK(ctx->row_ptr.upload(ps.row_ptr.data(), ps.row_ptr.size(), st));
    CK(ctx->col.upload(ps.col.data(), ps.col.size(), st));
    CK(ctx->val.upload(ps.val.data(), ps.val.size(), st));
    CK(ctx->valf.upload(ps.valf.data(), ps.valf.size(), st));
    CK(ctx->diag.upload(ps.diag.data(), ps.diag.size(), st));
    CK(ctx->dinv.upload(ps.dinv.data(), ps.dinv.size(), st));
    CK(ctx->diagf.upload(ps.diagf.data(), ps.diagf.size(), st));
    CK(ctx->dinvf.upload(ps.dinvf.data(), ps.dinvf.size(), st));
    PoissonView& pv = ctx->pv;
    pv.R = ps.R;
    pv.row_node = ctx->row_node.p;
    pv.cv = ctx->cv.p;
    pv.lift_ptr = ctx->lift_ptr.p;
    pv.lift_val = ctx->lift_val.p;
    pv.lift_node = ctx->lift_node.p;
    pv.row_ptr = ctx->row_ptr.p;
    pv.col = ctx->col.p;
    pv.val = ctx->val.p;
    pv.valf = ctx->valf.p;
    pv.diag = ctx->diag.p;
    pv.dinv = ctx->dinv.p;
    pv.diagf = ctx->diagf.p;
    pv.dinvf = ctx->dinvf.p;
    size_t R = (size_t)std::max(ps.R, 1);
    for (DBuf<double>* v : {&ctx->b, &ctx->x, &ctx->r, &ctx->z, &ctx->p, &ctx->pn, &ctx->q}) CK(v->alloc(R));
    for (DBuf<float>* v : {&ctx->xf, &ctx->rf, &ctx->zf, &ctx->pf, &ctx->pnf, &ctx->qf}) CK(v->alloc(R));
    CK(ctx->sc.alloc(1));
    CK(ctx->part.alloc((size_t)ctx->grid_red * 4));
    // fields
    CK(ctx->rho.alloc((size_t)m.N));
    CK(ctx->tmp_rho.alloc((size_t)m.N));
    CK(ctx->phi.alloc((size_t)m.N));
    CK(ctx->E.alloc((size_t)(3 * m.N)));
    CK(ctx->Ef.alloc((size_t)(3 * m.N)));
    CK(cudaMemsetAsync(ctx->rho.p, 0, sizeof(double) * m.N, st));
    CK(cudaMemsetAsync(ctx->phi.p, 0, sizeof(double) * m.N, st));
    CK(cudaMemsetAsync(ctx->E.p, 0, sizeof(double) * 3 * m.N, st));
    CK(cudaMemsetAsync(ctx->Ef.p, 0, sizeof(float) * 3 * m.N, st));
    CK(ctx->totq.alloc(2));
    CK(ctx->led.alloc(1));
    CK(cudaMemsetAsync(ctx->led.p, 0, sizeof(LedgerDev), st));
    CK(ctx->ke_acc.alloc(2));
    CK(cudaMemsetAsync(ctx->ke_acc.p, 0, 2 * sizeof(unsigned long long), ctx->st));
    CK(ctx->nact.alloc(1));
    CK(cudaStreamSynchronize(st));
    return SCDAT_OK;
}

}  // namespace

extern "C" {

SCDAT_API int scdat_destroy(scdat_ctx* ctx)
{
    if (!ctx) return SCDAT_ERR_ARG;
    if (ctx->batch_refs > 0) {
        ctx->err = "context is held by a batch: destroy the batch first";
        return SCDAT_ERR_STATE;
    }
    delete ctx;  // drains the stream, then releases events, stream and buffers
    return SCDAT_OK;
}

SCDAT_API int scdat_set_species(scdat_ctx* ctx, int32_t n_species, const scdat_species* sp)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(n_species > 0 && n_species <= 16 && sp, "need 1..16 species");
    ARG(ctx->species.empty(), "species are already set");
    ctx->species = std::vector<SpeciesState>((size_t)n_species);
    // fixed-point units: one macro-particle charge, and the energy of a 1 MeV macro-particle
    // (resolution 2^-64 of that, range 2^63 of it)
    double mq = 0.0, me = 0.0;
    for (int s = 0; s < n_species; ++s) {
        ARG(sp[s].mass > 0.0 && std::isfinite(sp[s].charge) && sp[s].weight > 0.0, "bad species entry");
        ctx->species[s].sp = sp[s];
        mq = std::max(mq, std::fabs(sp[s].charge * sp[s].weight));
        me = std::max(me, 1.602176634e-13 * std::max(1.0, sp[s].weight));
    }
    ctx->uq = pow2_ceil(mq);
    ctx->ue = pow2_ceil(me);
    const int64_t N = ctx->hm.N;
    CK(ctx->acc_l0.alloc((size_t)(n_species * N)));
    CK(ctx->acc_l1.alloc((size_t)(n_species * N)));
    CK(ctx->acc_h.alloc((size_t)(n_species * N)));
    CK(ctx->counts.alloc((size_t)n_species));
    CK(ctx->vmax.alloc(2 * (size_t)n_species));
    CK(cudaMemsetAsync(ctx->vmax.p, 0, 2 * sizeof(unsigned) * n_species, ctx->st));
    CK(cudaMallocHost((void**)&ctx->h_deferred, sizeof(unsigned) * n_species));
    std::memset(ctx->h_deferred, 0, sizeof(unsigned) * n_species);
    CK(cudaMemsetAsync(ctx->counts.p, 0, sizeof(int64_t) * n_species, ctx->st));
    CK(cudaMemsetAsync(ctx->acc_l0.p, 0, sizeof(unsigned long long) * n_species * N, ctx->st));
    CK(cudaMemsetAsync(ctx->acc_l1.p, 0, sizeof(unsigned long long) * n_species * N, ctx->st));
    CK(cudaMemsetAsync(ctx->acc_h.p, 0, sizeof(unsigned long long) * n_species * N, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

static int alloc_species(scdat_ctx* ctx, int s, int64_t n)
{
    SpeciesState& S = ctx->species[s];
    int64_t cap = std::max<int64_t>(n, 1);
    S.perm_pending = false;
    if (ctx->mixed) {
        CK(S.mix.alloc(2 * (size_t)cap));
        CK(S.mix2.alloc(2 * (size_t)cap));
        CK(S.tet2.alloc((size_t)cap));
        CK(S.id2.alloc((size_t)cap));
        CK(S.perm.alloc((size_t)cap));
        CK(S.skey.alloc((size_t)cap));
        for (DBuf<double>* a : {&S.x, &S.y, &S.z, &S.vx, &S.vy, &S.vz}) a->release();
    } else {
        for (DBuf<double>* a : {&S.x, &S.y, &S.z, &S.vx, &S.vy, &S.vz}) CK(a->alloc((size_t)cap));
        S.mix.release();
    }
    CK(S.tet.alloc((size_t)cap));
    CK(S.id.alloc((size_t)cap));
    S.cap = cap;
    S.n = n;
    CK(cudaMemcpyAsync(ctx->counts.p + s, &S.n, sizeof(int64_t), cudaMemcpyHostToDevice, ctx->st));
    // new particles: no maximum speed yet (the next push's MCC takes the direct draw)
    CK(cudaMemsetAsync(ctx->vmax.p + 2 * s, 0, 2 * sizeof(unsigned), ctx->st));
    // deferred lists of the multi-pass push: pass 1's list covers the largest species (a
    // stay-first pass 1 may defer every particle), pass 2's a quarter of it (a full list only
    // means the overflow finishes in pass 2)
    unsigned want1 = (unsigned)std::min<int64_t>(cap + 4096, 0x7fffffff);
    unsigned want = (unsigned)std::min<int64_t>(cap / 4 + 4096, 0x7fffffff);
    if (!ctx->dcount.p) CK(ctx->dcount.alloc(5));
    if (want1 > ctx->d1cap) {
        CK(ctx->d1idx.alloc(want1));
        CK(ctx->d1it.alloc(want1));
        CK(ctx->d1rem.alloc(want1));
        CK(ctx->d1vs.alloc(want1));
        ctx->d1cap = want1;
    }
    if (want > ctx->dcap) {
        CK(ctx->d2idx.alloc(want));
        CK(ctx->d2it.alloc(want));
        CK(ctx->d2rem.alloc(want));
        CK(ctx->d2vs.alloc(want));
        ctx->dcap = want;
    }
    // sort scratch and re-sort targets must cover the largest species (allocated here, not in
    // the first re-sort of a timed run)
    size_t need = (size_t)cap;
    if (ctx->kin.n < need) {
        CK(ctx->kin.alloc(need));
        CK(ctx->kout.alloc(need));
        CK(ctx->vin.alloc(need));
        CK(ctx->vout.alloc(need));
    }
    for (int a = 0; a < 6; ++a) {
        if (!ctx->mixed && ctx->shadow64[a].n < need) CK(ctx->shadow64[a].alloc(need));
    }
    if (ctx->scratchi.n < need) CK(ctx->scratchi.alloc(need));
    if (ctx->scratchu.n < need) CK(ctx->scratchu.alloc(need));
    int bits = 1;
    while (((uint64_t)1 << bits) <= (uint64_t)ctx->hm.T + 1) ++bits;
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ctx->kin.p, ctx->kout.p, ctx->vin.p, ctx->vout.p, (int)cap, 0,
                                       bits, ctx->st));
    if (tmp > ctx->cub_tmp.n) CK(ctx->cub_tmp.alloc(tmp));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_particles(scdat_ctx* ctx, int32_t species, int64_t n, const double* x, const double* v,
                                  const int32_t* tet_hint, const uint32_t* ids)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "bad species index");
    ARG(n >= 0 && (n == 0 || (x && v)), "bad particle arrays");
    ARG(n < (int64_t)0xffffffffLL, "too many particles for 32-bit ids");
    int rc = alloc_species(ctx, species, n);
    if (rc) return rc;
    if (n == 0) return SCDAT_OK;
    SpeciesState& S = ctx->species[species];
    std::vector<double> cx((size_t)n), cy((size_t)n), cz((size_t)n), wx((size_t)n), wy((size_t)n), wz((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        cx[i] = x[3 * i]; cy[i] = x[3 * i + 1]; cz[i] = x[3 * i + 2];
        wx[i] = v[3 * i]; wy[i] = v[3 * i + 1]; wz[i] = v[3 * i + 2];
    }
    std::vector<int32_t> t((size_t)n, kTetNoHint);
    if (tet_hint)
        for (int64_t i = 0; i < n; ++i) t[i] = (tet_hint[i] >= 0 && tet_hint[i] < ctx->hm.T) ? tet_hint[i] : kTetNoHint;
    std::vector<uint32_t> id((size_t)n);
    for (int64_t i = 0; i < n; ++i) id[i] = ids ? ids[i] : (uint32_t)i;
    CK(cudaMemcpyAsync(S.tet.p, t.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(S.id.p, id.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->st));
    if (!ctx->mixed) {
        CK(cudaMemcpyAsync(S.x.p, cx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(S.y.p, cy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(S.z.p, cz.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(S.vx.p, wx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(S.vy.p, wy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(S.vz.p, wz.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
    } else {
        DBuf<double> dx, dy, dz, dvx, dvy, dvz;
        CK(dx.upload(cx.data(), n, ctx->st));
        CK(dy.upload(cy.data(), n, ctx->st));
        CK(dz.upload(cz.data(), n, ctx->st));
        CK(dvx.upload(wx.data(), n, ctx->st));
        CK(dvy.upload(wy.data(), n, ctx->st));
        CK(dvz.upload(wz.data(), n, ctx->st));
        launch_to_mixed(ctx->mv, n, dx.p, dy.p, dz.p, dvx.p, dvy.p, dvz.p, store_of(ctx, species), ctx->st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_seed_tet_particles(scdat_ctx* ctx, int32_t species, int64_t n_tets, const int32_t* tets,
                                       int32_t n_per_tet, double temp_ev, const double* drift, uint64_t seed)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "bad species index");
    ARG(n_per_tet >= 0 && temp_ev >= 0.0, "bad count or temperature");
    ARG(tets ? n_tets >= 0 : n_tets == 0, "give the tet list and its length, or neither (all tets)");
    const int64_t nt = tets ? n_tets : ctx->hm.T;
    std::vector<int32_t> list;
    if (tets) {
        for (int64_t k = 0; k < n_tets; ++k) ARG(tets[k] >= 0 && tets[k] < ctx->hm.T, "tet index out of range");
        list.assign(tets, tets + n_tets);
    }
    const int64_t n = nt * n_per_tet;
    ARG(n < (int64_t)0xffffffffLL, "too many particles for 32-bit ids");
    int rc = alloc_species(ctx, species, n);
    if (rc) return rc;
    if (n == 0) return SCDAT_OK;
    DBuf<int32_t> dl;
    if (tets) CK(dl.upload(list.data(), list.size(), ctx->st));
    const double sigma = std::sqrt(temp_ev * 1.602176634e-19 / ctx->species[species].sp.mass);
    const double zero[3] = {0.0, 0.0, 0.0};
    launch_seed_tets(tets ? dl.p : nullptr, nt, n_per_tet, (int32_t)ctx->species.size(), species, sigma,
                     drift ? drift : zero, seed, store_of(ctx, species), ctx->mixed, ctx->mv, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

// ResultExporter / CSVExporter columnar layout (Tools/Output/src/CSVExporter.cpp:11-47): the
// parent directory created, a header "axis,series..." with the series in name order (a later
// series of an equal name replaces an earlier one, as std::map assignment does), then one row
// per axis value, %.8e.  err: the reason on failure.
static int write_columns_csv(const char* path, const char* axis, int64_t n_rows, const double* av, int32_t n_series,
                             const char* const* names, const double* const* values, std::string& err)
{
    std::map<std::string, const double*> series;
    for (int32_t s = 0; s < n_series; ++s) series[names[s]] = values[s];
    std::error_code ec;
    const std::filesystem::path p(path);
    std::filesystem::create_directories(p.parent_path().empty() ? std::filesystem::path(".") : p.parent_path(), ec);
    FILE* f = std::fopen(path, "w");
    if (!f) {
        err = std::string("Failed to open csv output: ") + path;
        return SCDAT_ERR_ARG;
    }
    std::fprintf(f, "%s", axis);
    for (auto& s : series) std::fprintf(f, ",%s", s.first.c_str());
    std::fprintf(f, "\n");
    for (int64_t r = 0; r < n_rows; ++r) {
        std::fprintf(f, "%.8e", av[r]);
        for (auto& s : series) std::fprintf(f, ",%.8e", s.second[r]);
        std::fprintf(f, "\n");
    }
    std::fclose(f);
    return SCDAT_OK;
}

static int write_columns(scdat_ctx* ctx, const char* path, const std::string& axis, const std::vector<double>& av,
                         const std::vector<std::pair<std::string, std::vector<double>>>& series)
{
    std::vector<const char*> names;
    std::vector<const double*> vals;
    for (auto& s : series) {
        names.push_back(s.first.c_str());
        vals.push_back(s.second.data());
    }
    return write_columns_csv(path, axis.c_str(), (int64_t)av.size(), av.data(), (int32_t)series.size(), names.data(),
                             vals.data(), ctx->err);
}

SCDAT_API int scdat_export_layer_profile_csv(scdat_ctx* ctx, const char* path, int32_t n_layers)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(path && n_layers > 0, "need a path and at least one layer");
    const int64_t N = ctx->hm.N;
    const double z0 = ctx->hg.bmin[2], z1 = ctx->hg.bmax[2];
    std::vector<double> phi((size_t)N), E(3 * (size_t)N);
    CK(cudaMemcpyAsync(phi.data(), ctx->phi.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(E.data(), ctx->E.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, ctx->st));
    // node layers by z
    std::vector<double> ps(n_layers, 0.0), es(n_layers, 0.0), nn(n_layers, 0.0);
    CK(cudaStreamSynchronize(ctx->st));
    for (int64_t i = 0; i < N; ++i) {
        const double z = ctx->hm.xyz[3 * i + 2];
        int l = (int)((z - z0) / (z1 - z0) * n_layers);
        l = std::min(std::max(l, 0), n_layers - 1);
        ps[l] += phi[i];
        es[l] += E[3 * i + 2];
        nn[l] += 1.0;
    }
    // particle moments per species and layer
    const double lv = (ctx->hg.bmax[0] - ctx->hg.bmin[0]) * (ctx->hg.bmax[1] - ctx->hg.bmin[1]) * (z1 - z0) / n_layers;
    std::vector<double> ne(n_layers, 0.0), ni(n_layers, 0.0), te(n_layers, 0.0);
    DBuf<double> cnt, v2;
    CK(cnt.alloc(n_layers));
    CK(v2.alloc(n_layers));
    for (int s = 0; s < (int)ctx->species.size(); ++s) {
        if (ctx->species[s].n == 0) continue;
        CK(cudaMemsetAsync(cnt.p, 0, sizeof(double) * n_layers, ctx->st));
        CK(cudaMemsetAsync(v2.p, 0, sizeof(double) * n_layers, ctx->st));
        launch_layer_moments(store_of(ctx, s), ctx->species[s].n, ctx->mixed, ctx->mv, z0, z1, n_layers, cnt.p, v2.p,
                             ctx->st);
        CK(cudaGetLastError());
        std::vector<double> c(n_layers), v(n_layers);
        CK(cudaMemcpyAsync(c.data(), cnt.p, sizeof(double) * n_layers, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(v.data(), v2.p, sizeof(double) * n_layers, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        const auto& sp = ctx->species[s].sp;
        for (int l = 0; l < n_layers; ++l) {
            const double dens = c[l] * sp.weight / lv;
            if (sp.electron_like) {
                ne[l] += dens;
                // 3/2 kT = 1/2 m <v^2> (the electrons' thermal plus drift energy), in eV
                if (c[l] > 0) te[l] = sp.mass * (v[l] / c[l]) / (3.0 * 1.602176634e-19);
            } else if (sp.charge > 0.0) {
                ni[l] += dens;
            }
        }
    }
    std::vector<double> zc(n_layers), pm(n_layers), em(n_layers);
    for (int l = 0; l < n_layers; ++l) {
        zc[l] = z0 + (l + 0.5) * (z1 - z0) / n_layers;
        pm[l] = nn[l] > 0 ? ps[l] / nn[l] : 0.0;
        em[l] = nn[l] > 0 ? es[l] / nn[l] : 0.0;
    }
    // series in name order, as the reference's std::map keeps them
    return write_columns(ctx, path, "z_m", zc,
                         {{"electric_field_z_v_per_m", em},
                          {"electron_density_m3", ne},
                          {"electron_temperature_ev", te},
                          {"ion_density_m3", ni},
                          {"potential_v", pm}});
}

SCDAT_API int scdat_export_nodes_csv(scdat_ctx* ctx, const char* path)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(path, "need a path");
    const int64_t N = ctx->hm.N;
    std::vector<double> rho((size_t)N), phi((size_t)N), E(3 * (size_t)N);
    int rc = scdat_get_fields(ctx, rho.data(), phi.data(), E.data());
    if (rc) return rc;
    std::vector<double> id((size_t)N), x((size_t)N), y((size_t)N), z((size_t)N), ex((size_t)N), ey((size_t)N),
        ez((size_t)N);
    for (int64_t i = 0; i < N; ++i) {
        id[i] = (double)i;
        x[i] = ctx->hm.xyz[3 * i];
        y[i] = ctx->hm.xyz[3 * i + 1];
        z[i] = ctx->hm.xyz[3 * i + 2];
        ex[i] = E[3 * i];
        ey[i] = E[3 * i + 1];
        ez[i] = E[3 * i + 2];
    }
    return write_columns(ctx, path, "node", id,
                         {{"charge_c", rho},
                          {"electric_field_x_v_per_m", ex},
                          {"electric_field_y_v_per_m", ey},
                          {"electric_field_z_v_per_m", ez},
                          {"potential_v", phi},
                          {"x_m", x},
                          {"y_m", y},
                          {"z_m", z}});
}

SCDAT_API int scdat_export_columns_csv(const char* path, const char* axis_name, int64_t n_rows, const double* axis,
                                       int32_t n_series, const char* const* names, const double* const* values)
{
    if (!path || !axis_name || n_rows < 0 || n_series < 0 || (n_rows > 0 && !axis) ||
        (n_series > 0 && (!names || !values)))
        return SCDAT_ERR_ARG;
    for (int32_t s = 0; s < n_series; ++s)
        if (!names[s] || (n_rows > 0 && !values[s])) return SCDAT_ERR_ARG;
    std::string err;
    return write_columns_csv(path, axis_name, n_rows, axis, n_series, names, values, err);
}

SCDAT_API int scdat_get_particle_count(scdat_ctx* ctx, int32_t species, int64_t* n)
{
    if (!ctx || !n) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "bad species index");
    *n = ctx->species[species].n;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_particles(scdat_ctx* ctx, int32_t species, int64_t capacity, double* x, double* v,
                                  int32_t* tet, uint8_t* status, uint32_t* ids, int64_t* n_out)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "bad species index");
    SpeciesState& S = ctx->species[species];
    const int64_t n = S.n;
    if (n_out) *n_out = n;
    ARG(capacity >= n, "capacity smaller than the particle count");
    if (n == 0) return SCDAT_OK;
    {
        int rc = settle_store(ctx, species);
        if (rc) return rc;
    }
    std::vector<double> cx((size_t)n), cy((size_t)n), cz((size_t)n), wx((size_t)n), wy((size_t)n), wz((size_t)n);
    std::vector<int32_t> t((size_t)n);
    std::vector<uint32_t> id((size_t)n);
    if (ctx->mixed) {
        DBuf<double> dx, dy, dz, dvx, dvy, dvz;
        for (DBuf<double>* a : {&dx, &dy, &dz, &dvx, &dvy, &dvz}) CK(a->alloc((size_t)n));
        launch_from_mixed(ctx->mv, n, store_of(ctx, species), dx.p, dy.p, dz.p, dvx.p, dvy.p, dvz.p, ctx->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(cx.data(), dx.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(cy.data(), dy.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(cz.data(), dz.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(wx.data(), dvx.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(wy.data(), dvy.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(wz.data(), dvz.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    } else {
        CK(cudaMemcpyAsync(cx.data(), S.x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(cy.data(), S.y.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(cz.data(), S.z.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(wx.data(), S.vx.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(wy.data(), S.vy.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(wz.data(), S.vz.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
    }
    CK(cudaMemcpyAsync(t.data(), S.tet.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(id.data(), S.id.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int64_t i = 0; i < n; ++i) {
        if (x) { x[3 * i] = cx[i]; x[3 * i + 1] = cy[i]; x[3 * i + 2] = cz[i]; }
        if (v) { v[3 * i] = wx[i]; v[3 * i + 1] = wy[i]; v[3 * i + 2] = wz[i]; }
        if (tet) tet[i] = t[i];
        if (status) status[i] = t[i] >= kTetNoHint ? SCDAT_ACTIVE : (t[i] == kTetAbsorbed ? SCDAT_ABSORBED : SCDAT_ESCAPED);
        if (ids) ids[i] = id[i];
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_kuhn_box_mesh(int32_t nx, int32_t ny, int32_t nz, double h, const int32_t* body_lo,
                                  const int32_t* body_hi, double bias, double wall, int64_t* n_nodes, int64_t* n_tets,
                                  double* node_xyz, int32_t* tet_nodes, uint8_t* node_dirichlet, double* node_phi,
                                  int32_t* hex_ijk, int64_t* n_cells)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || !(h > 0.0) || !n_nodes || !n_tets) return SCDAT_ERR_ARG;
    std::vector<double> xyz, phi;
    std::vector<int32_t> tet, hex;
    std::vector<uint8_t> dir;
    build_kuhn_box(nx, ny, nz, h, body_lo, body_hi, bias, wall, xyz, tet, dir, phi, hex);
    *n_nodes = (int64_t)dir.size();
    *n_tets = (int64_t)(tet.size() / 4);
    if (n_cells) *n_cells = (int64_t)(hex.size() / 3);
    if (node_xyz) std::memcpy(node_xyz, xyz.data(), sizeof(double) * xyz.size());
    if (tet_nodes) std::memcpy(tet_nodes, tet.data(), sizeof(int32_t) * tet.size());
    if (node_dirichlet) std::memcpy(node_dirichlet, dir.data(), dir.size());
    if (node_phi) std::memcpy(node_phi, phi.data(), sizeof(double) * phi.size());
    if (hex_ijk) std::memcpy(hex_ijk, hex.data(), sizeof(int32_t) * hex.size());
    return SCDAT_OK;
}

SCDAT_API int scdat_seed_box_particles(scdat_ctx* ctx, int32_t species, int32_t nx, int32_t ny, int32_t nz, double h,
                                       const int32_t* body_lo, const int32_t* body_hi, int32_t n_per_cell,
                                       double temp_ev, uint64_t seed)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "bad species index");
    ARG(n_per_cell > 0 && temp_ev >= 0.0, "bad seeding parameters");
    std::vector<double> xyz, phi;
    std::vector<int32_t> tet, hex;
    std::vector<uint8_t> dir;
    build_kuhn_box(nx, ny, nz, h, body_lo, body_hi, 0.0, 0.0, xyz, tet, dir, phi, hex);
    ARG((int64_t)(tet.size() / 4) == ctx->hm.T && (int64_t)dir.size() == ctx->hm.N,
        "mesh is not the Kuhn box of these dimensions");
    const int64_t ncell = (int64_t)(hex.size() / 3);
    const int64_t n = ncell * n_per_cell;
    ARG(n < (int64_t)0xffffffffLL, "too many particles for 32-bit ids");
    int rc = alloc_species(ctx, species, n);
    if (rc) return rc;
    DBuf<int32_t> dh;
    CK(dh.upload(hex.data(), hex.size(), ctx->st));
    const SpeciesState& S = ctx->species[species];
    double sigma = std::sqrt(temp_ev * 1.602176634e-19 / S.sp.mass);
    launch_seed_box(dh.p, ncell, n_per_cell, (int32_t)ctx->species.size(), species, h, sigma, seed,
                    store_of(ctx, species), ctx->mixed, ctx->mv, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_potential(scdat_ctx* ctx, const double* phi)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(phi, "null potential");
    CK(cudaMemcpyAsync(ctx->phi.p, phi, sizeof(double) * ctx->hm.N, cudaMemcpyHostToDevice, ctx->st));
    int rc = do_lsq(ctx, 1.0e-18);  // PICCycle's own LSQ regularisation (PICCycle.cpp:208)
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_node_potentials(scdat_ctx* ctx, int64_t n, const int64_t* nodes, const double* values)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(n >= 0 && (n == 0 || (nodes && values)), "bad node arrays");
    if (n == 0) return SCDAT_OK;
    for (int64_t i = 0; i < n; ++i) ARG(nodes[i] >= 0 && nodes[i] < ctx->hm.N, "node index out of range");
    // staging buffers kept by the context (grown on demand), so a per-step call allocates nothing
    if (ctx->stage_nodes.n < (size_t)n) CK(ctx->stage_nodes.alloc((size_t)n));
    if (ctx->stage_vals.n < (size_t)n) CK(ctx->stage_vals.alloc((size_t)n));
    CK(cudaMemcpyAsync(ctx->stage_nodes.p, nodes, sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->stage_vals.p, values, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
    launch_scatter_values(n, ctx->stage_nodes.p, ctx->stage_vals.p, ctx->phi.p, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_electric_field(scdat_ctx* ctx, const double* E)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(E, "null field");
    const int64_t n3 = 3 * ctx->hm.N;
    CK(cudaMemcpyAsync(ctx->E.p, E, sizeof(double) * n3, cudaMemcpyHostToDevice, ctx->st));
    std::vector<float> f((size_t)n3);
    for (int64_t i = 0; i < n3; ++i) f[i] = (float)E[i];
    CK(cudaMemcpyAsync(ctx->Ef.p, f.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, ctx->st));
    int rc = refresh_tet_field(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_charge_density(scdat_ctx* ctx, const double* rho)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(rho, "null charge density");
    CK(cudaMemcpyAsync(ctx->rho.p, rho, sizeof(double) * ctx->hm.N, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_dt(scdat_ctx* ctx, double dt)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(dt > 0.0 && std::isfinite(dt), "time step must be positive");
    ctx->prm.dt = dt;
    return SCDAT_OK;
}

SCDAT_API int scdat_set_seed(scdat_ctx* ctx, uint64_t seed)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ctx->prm.seed = seed;
    return SCDAT_OK;
}

SCDAT_API int scdat_set_surface_circuit(scdat_ctx* ctx, const scdat_surface_circuit* sc)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(sc, "null surface circuit");
    ARG(!ctx->species.empty(), "set the species first");
    for (int a = 0; a < 3; ++a) ARG(sc->body_hi[a] > sc->body_lo[a], "empty body box");
    const double ext[3] = {sc->body_hi[0] - sc->body_lo[0], sc->body_hi[1] - sc->body_lo[1],
                           sc->body_hi[2] - sc->body_lo[2]};
    SurfaceDev h{};
    h.n = 6;
    for (int f = 0; f < 6; ++f) {
        const int a = f / 2;
        const double area = sc->area[f] > 0.0 ? sc->area[f] : ext[(a + 1) % 3] * ext[(a + 2) % 3];
        ARG(sc->eps_r[f] >= 1.0 && sc->thickness[f] > 0.0, "each face needs eps_r >= 1 and a positive thickness");
        ARG(sc->shunt_s[f] >= 0.0 && std::isfinite(sc->didv[f]) && std::isfinite(sc->v0[f]), "bad face parameters");
        h.C[f] = 8.8541878128e-12 * sc->eps_r[f] * area / sc->thickness[f];
        h.G[f] = sc->shunt_s[f];
        h.didv[f] = sc->didv[f];
        h.V[f] = sc->v0[f];
    }
    // Dirichlet nodes on the body box's surface, with the faces each lies on
    const double tol = 1e-9 * std::max(ext[0], std::max(ext[1], ext[2]));
    std::vector<int32_t> nodes;
    std::vector<uint8_t> masks;
    for (int64_t i = 0; i < ctx->hm.N; ++i) {
        if (!ctx->hm.dirichlet[i]) continue;
        const double* p = &ctx->hm.xyz[3 * i];
        bool inside = true;
        for (int a = 0; a < 3; ++a) inside = inside && p[a] >= sc->body_lo[a] - tol && p[a] <= sc->body_hi[a] + tol;
        if (!inside) continue;
        unsigned m = 0;
        for (int f = 0; f < 6; ++f) {
            const int a = f / 2;
            const double plane = (f & 1) ? sc->body_hi[a] : sc->body_lo[a];
            if (std::fabs(p[a] - plane) <= tol) m |= 1u << f;
        }
        if (!m) continue;
        nodes.push_back((int32_t)i);
        masks.push_back((uint8_t)m);
    }
    ARG(!nodes.empty(), "no Dirichlet node lies on the body box");
    CK(ctx->surf.alloc(1));
    CK(cudaMemcpyAsync(ctx->surf.p, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->st));
    CK(ctx->surf_node.upload(nodes.data(), nodes.size(), ctx->st));
    CK(ctx->surf_mask.upload(masks.data(), masks.size(), ctx->st));
    CK(cudaMemsetAsync(ctx->led.p->patch_q, 0, sizeof(ctx->led.p->patch_q) + sizeof(ctx->led.p->patch_n), ctx->st));
    for (int a = 0; a < 3; ++a) {
        ctx->body_lo[a] = sc->body_lo[a];
        ctx->body_hi[a] = sc->body_hi[a];
    }
    ctx->surface = true;
    ctx->prm.body_tally = 1;
    launch_surface_apply(ctx->surf.p, (int64_t)nodes.size(), ctx->surf_node.p, ctx->surf_mask.p, ctx->phi.p, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

// The Sims yield's xm for exponent n, as legacySimsYield finds it (SurfaceMaterialModel.cpp:252-263):
// the first of 10000 grid points x in (0.5, 2.5] within 1e-3 of (1 - 1/n)(e^x - 1), else 2.5.
static double sims_xm(double n)
{
    double xm = 2.5;
    for (int i = 1; i < 10001; ++i) {
        const double x = 0.5 + (double)i * (2.5 - 0.5) / 10000.0;
        const double y = (1.0 - 1.0 / n) * (std::exp(x) - 1.0);
        if (std::fabs(x - y) <= 1.0e-3) {
            xm = x;
            break;
        }
    }
    return xm;
}

SCDAT_API int scdat_set_secondary_yield_params(scdat_ctx* ctx, double sims_exponent_n, const double* katz)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(std::isfinite(sims_exponent_n), "non-finite Sims exponent");
    if (katz)
        for (int k = 0; k < 4; ++k) ARG(std::isfinite(katz[k]), "non-finite Katz coefficient");
    ctx->see_sims_n = std::max(1.05, sims_exponent_n);
    ctx->see_sims_xm = sims_xm(ctx->see_sims_n);
    const double dflt[4] = {0.85, 0.35, 0.12, 1.05};
    for (int k = 0; k < 4; ++k) ctx->see_katz[k] = katz ? katz[k] : dflt[k];
    return SCDAT_OK;
}

SCDAT_API int scdat_set_secondary_emission(scdat_ctx* ctx, int32_t model, double delta_max, double e_max_ev)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(model >= 0 && model <= 4, "model: 0 off, 1 Sternglass, 2 Whipple, 3 Sims, 4 Katz");
    if (ctx->see_sims_xm == 0.0) ctx->see_sims_xm = sims_xm(ctx->see_sims_n);
    ARG(model == 0 || (delta_max >= 0.0 && e_max_ev > 0.0), "yield needs delta_max >= 0 and e_max > 0");
    ctx->see_model = model;
    ctx->see_dmax = delta_max;
    ctx->see_emax = e_max_ev;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_surface_state(scdat_ctx* ctx, double* V, double* Q, double* I, int64_t* counts)
{
    if (!ctx) return SCDAT_ERR_ARG;
    if (!ctx->surface) {
        ctx->err = "no surface circuit";
        return SCDAT_ERR_STATE;
    }
    SurfaceDev h{};
    LedgerDev l{};
    CK(cudaMemcpyAsync(&h, ctx->surf.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&l, ctx->led.p, sizeof(l), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int f = 0; f < 6; ++f) {
        if (V) V[f] = h.V[f];
        if (Q) Q[f] = h.Q[f];
        if (I) I[f] = h.I[f];
        if (counts) counts[f] = (int64_t)l.patch_n[f];
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_set_elastic_mcc(scdat_ctx* ctx, int32_t species, const scdat_elastic* proc)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "bad species index");
    ARG(proc && proc->target_density >= 0.0 && proc->sigma_max >= 0.0, "bad collision process");
    ARG(proc->mode >= 0 && proc->mode <= 2, "collision mode must be 0, 1 or 2");
    ctx->species[species].mcc = *proc;
    return SCDAT_OK;
}

SCDAT_API int scdat_push(scdat_ctx* ctx)
{
    if (!ctx) return SCDAT_ERR_ARG;
    int rc = do_push(ctx, false);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return check_flags(ctx);
}

SCDAT_API int scdat_solve_field(scdat_ctx* ctx)
{
    if (!ctx) return SCDAT_ERR_ARG;
    int rc = do_solve_field(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    if (!(ctx->last_pcg_rel <= ctx->prm.pcg_rtol)) {
        ctx->err = ctx->last_pcg_iter >= ctx->prm.pcg_max_iter
                       ? "field solve reached its iteration cap"
                       : "field solve stopped above its tolerance (refinement pass cap, CG breakdown or non-finite residual)";
        return SCDAT_ERR_NOT_CONVERGED;
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_collide(scdat_ctx* ctx)
{
    if (!ctx) return SCDAT_ERR_ARG;
    PushParams pp = push_params(ctx, true);
    for (int s = 0; s < (int)ctx->species.size(); ++s) {
        if (!ctx->species[s].mcc.enabled || ctx->species[s].cap == 0) continue;
        if (ctx->mixed)
            launch_mcc_mixed(store_of(ctx, s), species_dev(ctx, s), pp, ctx->led.p, ctx->grid_push, ctx->st);
        else
            launch_mcc_f64(store_of(ctx, s), species_dev(ctx, s), pp, ctx->led.p, ctx->grid_push, ctx->st);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_set_species_sort_interval(scdat_ctx* ctx, int32_t species, int32_t interval)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "species out of range");
    const int si = ctx->prm.sort_interval;
    ARG(interval == 0 || (interval > 0 && si > 0 && interval % si == 0),
        "species sort interval must be 0 or a positive multiple of params.sort_interval");
    ctx->species[species].sort_interval = interval;
    return SCDAT_OK;
}

SCDAT_API int scdat_set_species_push_mode(scdat_ctx* ctx, int32_t species, int32_t mode)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size(), "species out of range");
    ARG(mode == SCDAT_PUSH_AUTO || mode == SCDAT_PUSH_WALKING || mode == SCDAT_PUSH_STAY_FIRST, "unknown push mode");
    ctx->species[species].push_mode = mode;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_field_solver_levels(scdat_ctx* ctx, int32_t max_levels, int32_t* levels, int64_t* rows,
                                            int64_t* nnz, int64_t* transfer_nnz)
{
    if (!ctx || !levels) return SCDAT_ERR_ARG;
    ARG(max_levels >= 0, "negative level capacity");
    const bool mg = ctx->precond == SCDAT_PRECOND_MULTIGRID;
    const int L = mg ? (int)ctx->mg_plan.lv.size() : 1;
    *levels = L;
    for (int l = 0; l < std::min(L, (int)max_levels); ++l) {
        const int64_t r = mg ? ctx->mg_plan.lv[l].R : ctx->pv.R;
        int64_t z = 0, t = 0;
        if (l == 0)
            z = (int64_t)ctx->hps.col.size();
        else
            z = (int64_t)ctx->mgl[l]->col.n;
        if (mg && l + 1 < L) t = (int64_t)ctx->mgl[l]->p_col.n;
        if (mg && l + 1 == L) z = r * r;  // the coarsest level is solved by a dense inverse
        if (rows) rows[l] = r;
        if (nnz) nnz[l] = z;
        if (transfer_nnz) transfer_nnz[l] = t;
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_set_field_preconditioner(scdat_ctx* ctx, int32_t kind)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(kind == SCDAT_PRECOND_JACOBI || kind == SCDAT_PRECOND_MULTIGRID, "unknown preconditioner");
    if (kind == SCDAT_PRECOND_MULTIGRID && ctx->mgl.empty()) {
        int rc = setup_multigrid(ctx);
        if (rc) return rc;
    }
    ctx->precond = kind;
    return SCDAT_OK;
}

SCDAT_API int scdat_compact(scdat_ctx* ctx)
{
    if (!ctx) return SCDAT_ERR_ARG;
    for (int s = 0; s < (int)ctx->species.size(); ++s) {
        int rc = do_sort(ctx, s);
        if (rc) return rc;
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_step(scdat_ctx* ctx, int32_t n_steps)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(n_steps >= 0, "negative step count");
    for (int k = 0; k < n_steps; ++k) {
        int rc = do_push(ctx, true);
        if (rc) return rc;
        rc = do_surface(ctx);
        if (rc) return rc;
        rc = do_solve_field(ctx);
        if (rc) return rc;
        ctx->steps += 1;
        ctx->sim_time += ctx->prm.dt;
        if (ctx->prm.sort_interval > 0 && ctx->steps % ctx->prm.sort_interval == 0) {
            for (int s = 0; s < (int)ctx->species.size(); ++s) {
                if (!species_sorts_now(ctx, s)) continue;
                rc = do_sort(ctx, s);
                if (rc) return rc;
            }
        }
    }
    CK(cudaStreamSynchronize(ctx->st));
    return check_flags(ctx);
}

SCDAT_API int scdat_get_fields(scdat_ctx* ctx, double* rho, double* phi, double* E)
{
    if (!ctx) return SCDAT_ERR_ARG;
    const int64_t N = ctx->hm.N;
    if (rho) CK(cudaMemcpyAsync(rho, ctx->rho.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->st));
    if (phi) CK(cudaMemcpyAsync(phi, ctx->phi.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->st));
    if (E) CK(cudaMemcpyAsync(E, ctx->E.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_get_species_charge(scdat_ctx* ctx, int32_t species, double* rho_s)
{
    if (!ctx) return SCDAT_ERR_ARG;
    ARG(species >= 0 && species < (int)ctx->species.size() && rho_s, "bad species index");
    const int64_t N = ctx->hm.N;
    launch_species_rho(N, ctx->acc_l0.p + species * N, ctx->mixed ? nullptr : ctx->acc_l1.p + species * N,
                       ctx->mixed ? nullptr : ctx->acc_h.p + species * N,
                       ctx->uq, ctx->tmp_rho.p, ctx->grid_nodes, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rho_s, ctx->tmp_rho.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API int scdat_sample_with_derivative(scdat_ctx* const* c3, int64_t n_body, const int64_t* body_nodes,
                                           int32_t row, double v, double probe_delta_v, int32_t window_steps,
                                           double area_m2, scdat_current_sample* out)
{
    if (!c3 || !out || !c3[0] || !c3[1] || !c3[2]) return SCDAT_ERR_ARG;
    scdat_ctx* ctx = c3[1];
    ARG(n_body > 0 && body_nodes && window_steps > 0 && area_m2 > 0.0, "need surface nodes, a window and an area");
    ARG(row >= 0 && row <= 6, "ledger row out of range (0..5 faces, 6 body)");
    std::memset(out, 0, sizeof(*out));
    const double d = std::max(0.1, std::fabs(probe_delta_v));
    const double pot[3] = {v - d, v, v + d};
    double before[3][8], after[3][8];
    std::vector<double> vals((size_t)n_body);
    for (int k = 0; k < 3; ++k) {
        std::fill(vals.begin(), vals.end(), pot[k]);
        int rc = scdat_set_node_potentials(c3[k], n_body, body_nodes, vals.data());
        if (rc) return rc;
        double led[7 * 8];
        rc = scdat_get_ledger(c3[k], led);
        if (rc) return rc;
        std::memcpy(before[k], led + 8 * row, sizeof(before[k]));
    }
    const bool mixed = c3[0]->mixed && c3[1]->mixed && c3[2]->mixed;
    if (mixed) {
        scdat_batch* b = nullptr;
        int rc = scdat_batch_create(3, c3, &b);
        if (!rc) rc = scdat_batch_step(b, window_steps);
        if (rc) ctx->err = b ? scdat_batch_last_error(b) : "batch failed";
        scdat_batch_destroy(b);
        if (rc) return rc;
    } else {
        for (int k = 0; k < 3; ++k) {
            int rc = scdat_step(c3[k], window_steps);
            if (rc) return rc;
        }
    }
    double net[3];
    for (int k = 0; k < 3; ++k) {
        double led[7 * 8];
        int rc = scdat_get_ledger(c3[k], led);
        if (rc) return rc;
        std::memcpy(after[k], led + 8 * row, sizeof(after[k]));
        const double span = window_steps * c3[k]->prm.dt * area_m2;
        const double je = (after[k][0] - before[k][0]) / span, ji = (after[k][1] - before[k][1]) / span,
                     jm = -(after[k][2] - before[k][2]) / span;
        net[k] = je + ji + jm;
        if (k == 1) {
            out->electron_collection_a_per_m2 = je;
            out->ion_collection_a_per_m2 = ji;
            out->emitted_electron_a_per_m2 = jm;
        }
    }
    out->surface_potential_v = v;
    out->net_collection_a_per_m2 = net[1];
    out->current_derivative_a_per_m2_per_v = (net[2] - net[0]) / (2.0 * d);
    out->valid = 1;
    out->window_steps = window_steps;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_ledger(scdat_ctx* ctx, double* ledger)
{
    if (!ctx || !ledger) return SCDAT_ERR_ARG;
    LedgerDev h{};
    CK(cudaMemcpyAsync(&h, ctx->led.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int f = 0; f < 7; ++f) {
        double* r = ledger + 8 * f;
        r[0] = fx_to_double(h.row[f][0], (long long)h.row[f][1], ctx->uq);
        r[1] = fx_to_double(h.row[f][2], (long long)h.row[f][3], ctx->uq);
        r[2] = fx_to_double(h.emit_q[f][0], (long long)h.emit_q[f][1], ctx->uq);
        r[3] = fx_to_double(h.row[f][4], (long long)h.row[f][5], ctx->ue);
        r[4] = (double)h.row[f][6];
        r[5] = (double)h.row[f][7];
        r[6] = 0.0;
        r[7] = 0.0;
    }
    return SCDAT_OK;
}

SCDAT_API int scdat_reset_ledger(scdat_ctx* ctx)
{
    if (!ctx) return SCDAT_ERR_ARG;
    CK(cudaMemsetAsync(ctx->led.p->row, 0, sizeof(ctx->led.p->row), ctx->st));
    CK(cudaMemsetAsync(ctx->led.p->emit_q, 0, sizeof(ctx->led.p->emit_q), ctx->st));
    CK(cudaMemsetAsync(&ctx->led.p->surf_lo, 0, 2 * sizeof(unsigned long long), ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCDAT_OK;
}

SCDAT_API void* scdat_stream(scdat_ctx* ctx) { return ctx ? (void*)ctx->st : nullptr; }

SCDAT_API int scdat_set_timing(scdat_ctx* ctx, int32_t enable)
{
    if (!ctx) return SCDAT_ERR_ARG;
    int rc = harvest_timing(ctx);
    if (rc) return rc;
    ctx->timing = enable != 0;
    ctx->push_ms = ctx->field_ms = ctx->sort_ms = 0.0;
    ctx->push_launches = ctx->field_solves = ctx->push_particles = ctx->launches = ctx->sorts = 0;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_timing(scdat_ctx* ctx, double* push_ms, int64_t* push_launches, int64_t* push_particles,
                               double* field_ms, int64_t* field_solves, int64_t* kernel_launches)
{
    if (!ctx) return SCDAT_ERR_ARG;
    int rc = harvest_timing(ctx);
    if (rc) return rc;
    if (push_ms) *push_ms = ctx->push_ms;
    if (push_launches) *push_launches = ctx->push_launches;
    if (push_particles) *push_particles = ctx->push_particles;
    if (field_ms) *field_ms = ctx->field_ms;
    if (field_solves) *field_solves = ctx->field_solves;
    if (kernel_launches) *kernel_launches = ctx->launches;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_sort_timing(scdat_ctx* ctx, double* sort_ms, int64_t* sorts)
{
    if (!ctx) return SCDAT_ERR_ARG;
    int rc = harvest_timing(ctx);
    if (rc) return rc;
    if (sort_ms) *sort_ms = ctx->sort_ms;
    if (sorts) *sorts = ctx->sorts;
    return SCDAT_OK;
}

SCDAT_API int scdat_get_statistics(scdat_ctx* ctx, scdat_stats* st)
{
    if (!ctx || !st) return SCDAT_ERR_ARG;
    LedgerDev h{};
    unsigned long long ke[2] = {0, 0};
    unsigned long long tq[2] = {0, 0};
    CK(cudaMemcpyAsync(&h, ctx->led.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(ke, ctx->ke_acc.p, sizeof(ke), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(tq, ctx->totq.p, sizeof(tq), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::memset(st, 0, sizeof(*st));
    st->completed_steps = ctx->steps;
    st->simulation_time = ctx->sim_time;
    st->total_charge = fx_to_double(tq[0], (long long)tq[1], ctx->uq);
    st->total_energy = fx_to_double(ke[0], (long long)ke[1], kKeUnit);
    st->active_particles = (int64_t)h.active;
    int64_t stored = 0;
    for (auto& S : ctx->species) stored += S.n;
    st->stored_particles = stored;
    st->surface_deposited_charge = fx_to_double(h.surf_lo, (long long)h.surf_hi, ctx->uq);
    st->substeps = (int64_t)h.substeps;
    st->lost_events = (int64_t)h.lost_events;
    st->mcc_collisions = (int64_t)h.mcc_hits;
    st->last_pcg_iterations = ctx->last_pcg_iter;
    st->last_pcg_relres = ctx->last_pcg_rel;
    return SCDAT_OK;
}

}  // extern "C"
