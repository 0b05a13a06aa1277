// mg.cuh -- device views and launchers of the lattice-multigrid preconditioned CG (mg.cu).
//
// One V-cycle per CG iteration as the preconditioner M ~ A^-1: on each level two damped-Jacobi
// sweeps (the first from zero), the residual restricted by P^T, the coarser level's cycle
// prolonged by P and added, two more sweeps; the coarsest level is one dense mat-vec with its
// inverse.  Pre- and post-smoothing mirror each other, so M is symmetric and CG applies.  All
// reductions are fixed-shape (last-block tails), so a solve gives the same bits on every run.
#pragma once

#include "field.cuh"

#include <vector>

namespace scdat {

struct MgLevelDev {
    int R;
    // operator: off-diagonal CSR + diagonal, FP64 and FP32 copies
    const int32_t* row_ptr;
    const int32_t* col;
    const double* val;
    const float* valf;
    const double* diag;
    const float* diagf;
    const double* dinv;
    const float* dinvf;
    float omega;
    // to the next coarser level (null on the coarsest)
    const int32_t* p_ptr;
    const int32_t* p_col;
    const float* p_w;
    const int32_t* r_ptr;
    const int32_t* r_col;
    const float* r_w;
};

// Per-level work vectors of one precision (level 0 takes its right-hand side and output from
// the CG): b (levels >= 1), two smoothing iterates, the residual, the level's output.
struct MgWork {
    void* b;
    void* xa;
    void* xb;
    void* res;
    void* xo;
};

struct MgPlan {
    std::vector<MgLevelDev> lv;
    std::vector<MgWork> w;
    const double* cinv = nullptr;  // dense inverse of the coarsest operator [Rc*Rc]
    const float* cinvf = nullptr;
    int grid_max = 0;              // blocks of 256 for the level-0 launches
};

// z = M r (level 0's right-hand side r, output z), with sc->rz = r.z computed by the last sweep.
template <typename V>
void launch_vcycle(const MgPlan& mg, const V* r, V* z, PcgScalars* sc, double* part, cudaStream_t st);

// The CG around it on level 0 (A = the Dirichlet-reduced Poisson matrix, in V's precision):
//   init:   r = b - A x; rr, bb; convergence threshold
//   dir:    p = z + beta p (beta = rz / rz_prev; p = z on the first iteration)
//   spmv:   q = A p; pq
//   update: x += alpha p; r -= alpha q; rr; iteration count and convergence test
// launch_mgpcg_iter queues dir, spmv, update and the next V-cycle.
template <typename V>
void launch_mgpcg_init(const PoissonView& A, const V* b, const V* x, V* r, PcgScalars* sc, double* part, int grid,
                       cudaStream_t st);
template <typename V>
void launch_mgpcg_iter(const PoissonView& A, const MgPlan& mg, V* x, V* r, V* z, V* p, V* q, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st);

}  // namespace scdat
