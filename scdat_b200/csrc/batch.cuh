// batch.cuh -- descriptors of the batched step: many independent scenarios (one scdat_ctx
// each, meshes of different sizes) advanced by single launches over all of them.
//
// Push: one job per (scenario, species); a launch walks a global index of 256-particle
// chunks in job order, each block taking chunks blockIdx.x, blockIdx.x + grid, ... so its
// sequence of jobs, and every fixed-order sum it feeds, is the same on every run.
// Field: one job per scenario; every scenario owns a contiguous range of the launch's blocks
// (sized to its share of the rows, nodes or tets), and each block runs the single-scenario
// kernel body on that scenario with its index inside the range.
#pragma once

#include "field.cuh"
#include "push.cuh"
#include "surface.cuh"

namespace scdat {

constexpr int kMaxBatchJobs = 1024;

struct PushJob {
    MeshView M;
    ParticleStore P;
    SpeciesDev S;
    PushParams pp;
    ChargeAcc A;
    LedgerDev* L;
    unsigned long long* ke_acc;  // kinetic energy of the push, exact fixed point (lo, hi)
    DeferList D1, D2;
};

struct FieldJob {
    PoissonView A;
    int64_t N, T;
    int S;
    // per-step accumulators
    unsigned long long *l0, *l1, *h;  // charge limbs [S*N]
    unsigned long long* ke_acc;       // kinetic energy of the push, exact fixed point (lo, hi)
    unsigned* vmax;                   // [2 per species] maximum speeds (SpeciesDev::vmax)
    unsigned long long* led_active;
    unsigned long long* lsq_bad;
    // charge finalisation
    double uq;
    double* rho;
    unsigned long long* totq;  // [2]
    // right-hand side and solution
    double* phi;
    double sign;
    double *b, *x, *r;
    float *rf, *xf, *zf, *pf, *pnf, *qf, *qq;
    PcgScalars* sc;   // inner (FP32) solve
    PcgScalars* sco;  // outer refinement loop
    double* part;
    double rtol;
    int max_iter;
    // nodal field and the tet records
    double lsq_reg;  // 0 after a solve (a runtime value, so the body compiles as in field.cu)
    const double* xyz;
    const int32_t* gptr;
    const int32_t* gcol;
    double* E;
    float* Ef;
    const int4* tet;
    float* trec;
    // surface circuit (surf == nullptr: none)
    SurfaceDev* surf;
    LedgerDev* led;
    double dt;
    const int32_t* surf_node;
    const uint8_t* surf_mask;
    int64_t surf_n;
};

// Block b of a field launch works on scenario ctx_of[b], as block b - first[ctx] of
// first[ctx + 1] - first[ctx].
struct BlockMap {
    const int* ctx_of;
    const int* first;
    int blocks;
};

// push (push_mixed.cu); chunk_prefix[j] = first 32-particle chunk of job j, computed on the
// device from the live counts by launch_batch_prefix, which also zeroes the pass's work counter
// ctr[pass - 1].
void launch_batch_prefix(const PushJob* jobs, int njobs, int pass, int64_t* chunk_prefix, unsigned* ctr,
                         cudaStream_t st);
void launch_push_mixed_batch(const PushJob* jobs, int njobs, const int64_t* chunk_prefix, unsigned* ctr, int pass,
                             int grid, cudaStream_t st);
void launch_batch_refresh_trec(const FieldJob* jobs, const BlockMap& tets, cudaStream_t st);

// field (batch_field.cu).  cond_* are CUDA-graph conditional handles (0 outside a graph);
// any_out (nullable) receives the same "some scenario still iterating" flag for a host loop.
void launch_batch_zero(const FieldJob* jobs, const PushJob* pjobs, int njobs, int npjobs, int grid, cudaStream_t st);
void launch_batch_surface(const FieldJob* jobs, int njobs, cudaStream_t st);
void launch_batch_finalize_rhs(const FieldJob* jobs, const BlockMap& nodes, const BlockMap& rows, cudaStream_t st);
void launch_batch_pcg_mixed_prologue(const FieldJob* jobs, const BlockMap& rows, int njobs, cudaStream_t st);
void launch_batch_outer_begin(const FieldJob* jobs, const BlockMap& rows, int njobs, unsigned long long cond_inner,
                              int* any_out, cudaStream_t st);
// passes[0] counts refinement passes, passes[1] inner double-iterations (launch accounting)
void launch_batch_inner_iter2(const FieldJob* jobs, const BlockMap& rows, int njobs, unsigned long long cond_inner,
                              int* any_out, unsigned long long* passes, cudaStream_t st);
void launch_batch_outer_end(const FieldJob* jobs, const BlockMap& rows, int njobs, unsigned long long cond_outer,
                            int* any_out, unsigned long long* passes, cudaStream_t st);
void launch_batch_epilogue(const FieldJob* jobs, const BlockMap& nodes, const BlockMap& rows, const BlockMap& tets,
                           PushJob* pjobs, int npjobs, cudaStream_t st);

}  // namespace scdat
