// field.cuh -- views and launchers of the field-solve kernels (field.cu).
#pragma once

#include "common.cuh"

namespace scdat {

// Dirichlet-reduced edge-Laplacian: one row per non-Dirichlet node (PoissonSolver.cpp:274-385
// after LinearSystem::applyDirichletBC, LinearSystem.cpp:37-58).
struct PoissonView {
    int R;
    const int32_t* row_node;  // [R] node of each row
    const double* cv;         // [R] nodal control volume sum_e V_e/4
    const int32_t* lift_ptr;  // [R+1] Dirichlet couplings of each row
    const double* lift_val;   // K_rd
    const int32_t* lift_node; // d
    const int32_t* row_ptr;   // [R+1] off-diagonal couplings to other rows
    const int32_t* col;       // row index
    const double* val;        // K_rr' (FP64)
    const float* valf;        // K_rr' (FP32, mixed form)
    const double* diag;       // K_rr
    const double* dinv;       // 1 / K_rr
    const float* diagf;       // K_rr (FP32, mixed form)
    const float* dinvf;       // 1 / K_rr (FP32, mixed form)
};

struct PcgScalars {
    double rz, rz_prev, pq, rr, bb, thr2, rtol, abs_thr2;
    int iter, done, max_iter, outer;  // outer: refinement passes (batched mixed solve)
    unsigned int ticket;
    unsigned int pad2[3];
};

// Relative tolerance of the next FP32 inner solve of the mixed refinement, from the FP64
// residual rr = |r|^2 against bb = |b|^2: enough for the corrected residual to clear the target
// rtol in this pass with a factor-4 margin, but no tighter than 1e-5 (what an FP32 Jacobi-PCG
// reliably reaches) and no looser than 1e-1.  The host-driven and the graph-driven loops both
// call it, so they take the same passes.
// Refinement passes of the mixed solve (FP32 inner solve + FP64 correction) before it stops;
// the FP64 residual of the last corrected x is still computed and reported.
constexpr int kMaxRefinePasses = 12;

__host__ __device__ inline double inner_rtol(double rr, double bb, double rtol)
{
    const double need = 0.25 * rtol * sqrt(bb / rr);
    return fmin(1e-1, fmax(1e-5, need));
}

void launch_finalize_rho(int64_t N, int S, const unsigned long long* l0, const unsigned long long* l1,
                         const unsigned long long* h, double unit, double* rho, unsigned long long* tlo,
                         unsigned long long* thi, int grid, cudaStream_t st);
void launch_species_rho(int64_t N, const unsigned long long* l0, const unsigned long long* l1,
                        const unsigned long long* h, double unit, double* out, int grid, cudaStream_t st);
void launch_rhs(const PoissonView& A, const double* rho, const double* phi, double sign, double* b, int grid,
                cudaStream_t st);
void launch_gather_rows(const PoissonView& A, const double* phi, double* x, int grid, cudaStream_t st);
void launch_scatter_rows(const PoissonView& A, const double* x, double* phi, int grid, cudaStream_t st);
void launch_lsq(int64_t N, const double* xyz, const int32_t* gptr, const int32_t* gcol, const double* phi, double reg,
                double* E, float* Ef, unsigned long long* flags, int grid, cudaStream_t st);
void launch_pcg_init64(const PoissonView& A, const double* b, const double* x, double* r, double* z, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st);
void launch_pcg_iter64(const PoissonView& A, double* x, double* r, double* z, double* p, double* pn, double* q,
                       PcgScalars* sc, double* part, int grid, cudaStream_t st);
void launch_pcg_init32(const PoissonView& A, const float* b, const float* x, float* r, float* z, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st);
void launch_pcg_iter32(const PoissonView& A, float* x, float* r, float* z, float* p, float* pn, float* q,
                       PcgScalars* sc, double* part, int grid, cudaStream_t st);
void launch_residual64(const PoissonView& A, const double* b, const double* x, double* r, float* rf, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st);
void launch_add_correction(int R, double* x, const float* e, int grid, cudaStream_t st);
void launch_zero_f32(int R, float* v, int grid, cudaStream_t st);

}  // namespace scdat
