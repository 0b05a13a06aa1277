// field.cu -- per-step field solve on the device.
//
//  k_finalize_rho   fixed-point node accumulators -> FP64 nodal charge, exact total charge
//  k_rhs            b_r = sign*rho*CV - sum_d K_rd phi_d on the Dirichlet-reduced rows
//                   (PoissonSolver.cpp:331-385, LinearSystem.cpp:37-58)
//  k_pcg_*          Jacobi-preconditioned CG (ConjugateGradientCommon.h:74-161 restated as
//                   two bandwidth kernels per iteration; the dot products use a fixed-order
//                   last-block reduction, so the solve is deterministic)
//  k_lsq_field      E_i = -LSQ gradient of phi over the node graph
//                   (PoissonSolver.cpp:474-529,749-787; PICCycle.cpp:129-220)
#include "field_kern.cuh"

namespace scdat {

__global__ void k_finalize_rho(int64_t N, int S, const unsigned long long* __restrict__ l0,
                               const unsigned long long* __restrict__ l1, const unsigned long long* __restrict__ h,
                               double unit, double* __restrict__ rho, unsigned long long* total_lo,
                               unsigned long long* total_hi)
{
    k_finalize_rho_body(N, S, l0, l1, h, unit, rho, total_lo, total_hi, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_species_rho(int64_t N, const unsigned long long* __restrict__ l0,
                              const unsigned long long* __restrict__ l1, const unsigned long long* __restrict__ h,
                              double unit, double* __restrict__ out)
{
    k_species_rho_body(N, l0, l1, h, unit, out, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_rhs(PoissonView A, const double* __restrict__ rho, const double* __restrict__ phi, double sign,
                      double* __restrict__ b)
{
    k_rhs_body(A, rho, phi, sign, b, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_gather_rows(PoissonView A, const double* __restrict__ phi, double* __restrict__ x)
{
    k_gather_rows_body(A, phi, x, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_scatter_rows(PoissonView A, const double* __restrict__ x, double* __restrict__ phi)
{
    k_scatter_rows_body(A, x, phi, Grid{blockIdx.x, gridDim.x});
}

template <typename V>
__global__ void k_pcg_init(PoissonView A, const V* __restrict__ val, const V* __restrict__ b, const V* __restrict__ x,
                           V* __restrict__ r, V* __restrict__ z, PcgScalars* sc, double* part)
{
    k_pcg_init_body(A, val, b, x, r, z, sc, part, Grid{blockIdx.x, gridDim.x});
}

template <typename V>
__global__ void k_pcg_spmv(PoissonView A, const V* __restrict__ val, const V* __restrict__ z, const V* __restrict__ p,
                           V* __restrict__ pn, V* __restrict__ q, PcgScalars* sc, double* part)
{
    k_pcg_spmv_body(A, val, z, p, pn, q, sc, part, Grid{blockIdx.x, gridDim.x});
}

template <typename V>
__global__ void k_pcg_update(PoissonView A, V* __restrict__ x, const V* __restrict__ pn, V* __restrict__ r,
                             const V* __restrict__ q, V* __restrict__ z, PcgScalars* sc, double* part)
{
    k_pcg_update_body(A, x, pn, r, q, z, sc, part, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_residual64(PoissonView A, const double* __restrict__ b, const double* __restrict__ x,
                             double* __restrict__ r, float* __restrict__ rf, PcgScalars* sc, double* part)
{
    k_residual64_body(A, b, x, r, rf, sc, part, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_add_correction(int R, double* __restrict__ x, const float* __restrict__ e)
{
    k_add_correction_body(R, x, e, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_zero_f32(int R, float* __restrict__ v)
{
    k_zero_f32_body(R, v, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_lsq_field(int64_t N, const double* __restrict__ xyz, const int32_t* __restrict__ gptr,
                            const int32_t* __restrict__ gcol, const double* __restrict__ phi, double reg,
                            double* __restrict__ E, float* __restrict__ Ef, unsigned long long* flags)
{
    k_lsq_field_body(N, xyz, gptr, gcol, phi, reg, E, Ef, flags, Grid{blockIdx.x, gridDim.x});
}

__global__ void k_zero_if_flag(int64_t n3, double* E, float* Ef, const unsigned long long* flags)
{
    k_zero_if_flag_body(n3, E, Ef, flags, Grid{blockIdx.x, gridDim.x});
}

// ---------------------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------------------
void launch_finalize_rho(int64_t N, int S, const unsigned long long* l0, const unsigned long long* l1,
                         const unsigned long long* h, double unit, double* rho, unsigned long long* tlo,
                         unsigned long long* thi, int grid, cudaStream_t st)
{
    k_finalize_rho<<<grid, 256, 0, st>>>(N, S, l0, l1, h, unit, rho, tlo, thi);
}

void launch_species_rho(int64_t N, const unsigned long long* l0, const unsigned long long* l1,
                        const unsigned long long* h, double unit, double* out, int grid, cudaStream_t st)
{
    k_species_rho<<<grid, 256, 0, st>>>(N, l0, l1, h, unit, out);
}

void launch_rhs(const PoissonView& A, const double* rho, const double* phi, double sign, double* b, int grid,
                cudaStream_t st)
{
    k_rhs<<<grid, 256, 0, st>>>(A, rho, phi, sign, b);
}

void launch_gather_rows(const PoissonView& A, const double* phi, double* x, int grid, cudaStream_t st)
{
    k_gather_rows<<<grid, 256, 0, st>>>(A, phi, x);
}

void launch_scatter_rows(const PoissonView& A, const double* x, double* phi, int grid, cudaStream_t st)
{
    k_scatter_rows<<<grid, 256, 0, st>>>(A, x, phi);
}

void launch_lsq(int64_t N, const double* xyz, const int32_t* gptr, const int32_t* gcol, const double* phi, double reg,
                double* E, float* Ef, unsigned long long* flags, int grid, cudaStream_t st)
{
    k_lsq_field<<<grid, 256, 0, st>>>(N, xyz, gptr, gcol, phi, reg, E, Ef, flags);
    k_zero_if_flag<<<grid, 256, 0, st>>>(3 * N, E, Ef, flags);
}

void launch_pcg_init64(const PoissonView& A, const double* b, const double* x, double* r, double* z, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st)
{
    k_pcg_init<double><<<grid, 256, 0, st>>>(A, A.val, b, x, r, z, sc, part);
}

void launch_pcg_iter64(const PoissonView& A, double* x, double* r, double* z, double* p, double* pn, double* q,
                       PcgScalars* sc, double* part, int grid, cudaStream_t st)
{
    k_pcg_spmv<double><<<grid, 256, 0, st>>>(A, A.val, z, p, pn, q, sc, part);
    k_pcg_update<double><<<grid, 256, 0, st>>>(A, x, pn, r, q, z, sc, part);
}

void launch_pcg_init32(const PoissonView& A, const float* b, const float* x, float* r, float* z, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st)
{
    k_pcg_init<float><<<grid, 256, 0, st>>>(A, A.valf, b, x, r, z, sc, part);
}

void launch_pcg_iter32(const PoissonView& A, float* x, float* r, float* z, float* p, float* pn, float* q,
                       PcgScalars* sc, double* part, int grid, cudaStream_t st)
{
    k_pcg_spmv<float><<<grid, 256, 0, st>>>(A, A.valf, z, p, pn, q, sc, part);
    k_pcg_update<float><<<grid, 256, 0, st>>>(A, x, pn, r, q, z, sc, part);
}

void launch_residual64(const PoissonView& A, const double* b, const double* x, double* r, float* rf, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st)
{
    k_residual64<<<grid, 256, 0, st>>>(A, b, x, r, rf, sc, part);
}

void launch_add_correction(int R, double* x, const float* e, int grid, cudaStream_t st)
{
    k_add_correction<<<grid, 256, 0, st>>>(R, x, e);
}

void launch_zero_f32(int R, float* v, int grid, cudaStream_t st)
{
    k_zero_f32<<<grid, 256, 0, st>>>(R, v);
}

}  // namespace scdat
