// ctx.cuh -- the scdat_ctx object behind the C ABI (include/scdat_b200.h), shared by the
// single-context entry points (capi.cu) and the batched step (batch_host.cu).
#pragma once

#include "../../include/scdat_b200.h"
#include "common.cuh"
#include "field.cuh"
#include "mesh_setup.h"
#include "mg.cuh"
#include "push.cuh"
#include "surface.cuh"

#include <memory>
#include <string>
#include <utility>
#include <vector>

using namespace scdat;

struct scdat_ctx;
// true when species s re-sorts at the context's current step count (a multiple of the
// context's sort interval)
bool species_sorts_now(const scdat_ctx* ctx, int s);

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count)
    {
        release();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
    cudaError_t upload(const T* h, size_t count, cudaStream_t st)
    {
        cudaError_t e = alloc(count);
        if (e != cudaSuccess || count == 0) return e;
        return cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st);
    }
    void swap(DBuf& o)
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
};

struct SpeciesState {
    scdat_species sp{};
    scdat_elastic mcc{};
    int64_t cap = 0;
    int64_t n = 0;  // host view of the stored count (updated on set/compact)
    int sort_interval = 0;  // 0: the context's params.sort_interval
    // pass-1 form of the mixed push (scdat_set_species_push_mode) and the automatic choice's
    // state: pushes so far, the deferred fraction of the last stay-first push (-1: none yet),
    // the particle count of that push, and whether its count is still to be read
    int push_mode = 0;
    int64_t pushes = 0;
    double stay_frac = -1.0;
    int64_t stay_n = 0;
    bool stay_pending = false;
    DBuf<double> x, y, z, vx, vy, vz;
    DBuf<float4> mix;  // mixed form: two float4 per particle (see ParticleStore)
    DBuf<int32_t> tet;
    DBuf<uint32_t> id;
    // Mixed form: a re-sort leaves its permutation and sorted keys here and the next pass 1
    // reads the store through them, writing the sorted store into mix2/tet2/id2 (then swapped
    // in); anything else that needs the store first runs the gather (settle_store).
    DBuf<float4> mix2;
    DBuf<int32_t> tet2;
    DBuf<uint32_t> id2, perm, skey;
    bool perm_pending = false;
};

// The start and end events of one timed stage.  An early error return destroys them; commit()
// hands the recorded pair to a context's list, whose owner destroys it after reading it.
struct StageEvents {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    StageEvents() = default;
    StageEvents(const StageEvents&) = delete;
    StageEvents& operator=(const StageEvents&) = delete;
    ~StageEvents()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    void commit(std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& list)
    {
        list.emplace_back(e0, e1);
        e0 = e1 = nullptr;
    }
};

// One multigrid level on the device (level 0 shares the context's Poisson arrays and only
// holds its transfers and work vectors).
struct MgDevLevel {
    DBuf<int32_t> row_ptr, col, p_ptr, p_col, r_ptr, r_col;
    DBuf<double> val, diag, dinv;
    DBuf<float> valf, diagf, dinvf, p_w, r_w;
    DBuf<unsigned char> work;  // b, xa, xb, res, xo in the context's precision
};

struct scdat_ctx {
    std::string err;
    scdat_params prm{};
    bool mixed = false;
    HostMesh hm;
    HostGeometry hg;
    HostGrid hgrid;
    HostGraph hgr;
    HostPoisson hps;
    MeshView mv{};
    PoissonView pv{};
    // mesh
    DBuf<double> xyz, geom, erec;
    DBuf<float> geomf, trec;
    DBuf<int4> tet, nbr;
    DBuf<int32_t> bin_start, bin_tets, gptr, gcol;
    // poisson
    DBuf<int32_t> row_node, lift_ptr, lift_node, row_ptr, col;
    DBuf<double> cv, lift_val, val, diag, dinv;
    DBuf<float> valf, diagf, dinvf;
    DBuf<double> b, x, r, z, p, pn, q;
    DBuf<float> xf, rf, zf, pf, pnf, qf;
    DBuf<PcgScalars> sc;
    DBuf<double> part;
    // lattice multigrid preconditioner (scdat_set_field_preconditioner): per-level operators,
    // transfers and work vectors, the coarsest dense inverse, and the launch plan over them
    int precond = 0;
    std::vector<std::unique_ptr<MgDevLevel>> mgl;
    DBuf<double> mg_cinv;
    DBuf<float> mg_cinvf;
    MgPlan mg_plan;
    // fields
    DBuf<double> rho, phi, E, tmp_rho;
    DBuf<float> Ef;
    DBuf<unsigned long long> acc_l0, acc_l1, acc_h, totq;
    DBuf<unsigned> vmax;  // [2 per species]: maximum speed of the previous / current push (float bits)
    // particles
    std::vector<SpeciesState> species;
    DBuf<int64_t> counts;
    DBuf<LedgerDev> led;
    DBuf<unsigned long long> ke_acc;  // kinetic energy of the last push, fixed point (lo, hi)
    // sort scratch
    DBuf<uint32_t> kin, kout, vin, vout;
    DBuf<unsigned char> cub_tmp;
    DBuf<double> shadow64[6];  // re-sort targets, swapped with the store's arrays
    DBuf<int32_t> scratchi;
    DBuf<uint32_t> scratchu;
    DBuf<int64_t> nact;
    DBuf<int64_t> idx64;
    DBuf<int64_t> stage_nodes;  // scdat_set_node_potentials staging
    DBuf<double> stage_vals;
    // deferred-particle lists of the multi-pass push
    DBuf<unsigned> dcount;
    DBuf<uint32_t> d1idx, d2idx;
    DBuf<int> d1it, d2it;
    DBuf<double> d1rem, d2rem, d1vs, d2vs;
    unsigned dcap = 0, d1cap = 0;
    unsigned* h_deferred = nullptr;  // pinned: pass-1 deferred count of each species' last stay-first push
    // surface circuit of the body faces (scdat_set_surface_circuit)
    bool surface = false;
    int see_model = 0;
    double see_dmax = 0.0, see_emax = 300.0;
    double see_sims_n = 1.6, see_sims_xm = 0.0;  // xm set with the exponent
    double see_katz[4] = {0.85, 0.35, 0.12, 1.05};
    double body_lo[3] = {0, 0, 0}, body_hi[3] = {0, 0, 0};
    DBuf<SurfaceDev> surf;
    DBuf<int32_t> surf_node;
    DBuf<uint8_t> surf_mask;
    double uq = 1.0, ue = 1.0;
    int64_t steps = 0;
    double sim_time = 0.0;
    int last_pcg_iter = 0;
    double last_pcg_rel = 0.0;
    cudaStream_t st = nullptr;
    int nsm = 148;
    int grid_push = 148 * 8, grid_nodes = 148 * 4, grid_red = 148 * 8;
    // optional per-kernel timing (CUDA events around the launches on the context stream)
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_push, ev_field, ev_sort;
    double push_ms = 0.0, field_ms = 0.0, sort_ms = 0.0;
    int64_t sorts = 0;
    int64_t push_launches = 0, field_solves = 0;
    int64_t push_particles = 0;
    int64_t launches = 0;  // kernels of this library launched since scdat_set_timing
    // batches that hold this context (scdat_batch_create / scdat_batch_destroy); a batch's
    // captured graph and job tables point into the context's buffers, so scdat_destroy refuses
    // while it is non-zero
    int batch_refs = 0;

    // The context owns its stream and timing events, so a context that scdat_create abandons
    // on an error releases them too.  The stream is drained first; the device buffers are
    // freed after this body, by their own destructors.
    scdat_ctx() = default;
    scdat_ctx(const scdat_ctx&) = delete;
    scdat_ctx& operator=(const scdat_ctx&) = delete;
    ~scdat_ctx()
    {
        if (st) cudaStreamSynchronize(st);
        if (h_deferred) cudaFreeHost(h_deferred);
        for (auto* evs : {&ev_push, &ev_field, &ev_sort})
            for (auto& pr : *evs) {
                cudaEventDestroy(pr.first);
                cudaEventDestroy(pr.second);
            }
        if (st) cudaStreamDestroy(st);
    }
};

namespace scdat {
// helpers of capi.cu used by the batched step
ParticleStore store_of(scdat_ctx* ctx, int s);
int settle_store(scdat_ctx* ctx, int s);
SpeciesDev species_dev(const scdat_ctx* ctx, int s);
PushParams push_params(const scdat_ctx* ctx, bool do_mcc);
int check_flags(scdat_ctx* ctx);
int do_sort(scdat_ctx* ctx, int s);
int do_push(scdat_ctx* ctx, bool do_mcc);
int do_surface(scdat_ctx* ctx);
int do_solve_field(scdat_ctx* ctx);
int do_lsq(scdat_ctx* ctx, double reg);
int refresh_tet_field(scdat_ctx* ctx);
int run_pcg64(scdat_ctx* ctx, const double* bvec, double* xvec, double rtol, int max_iter, int& iters, double& relres);
}  // namespace scdat
