// pcg_csr.cu -- context-free Jacobi-preconditioned CG on a caller-assembled system held in
// device memory (the role of LinearSystem::solve(ITERATIVE),
// Tools/Solver/src/LinearSystem.cpp:84-87,258-327, with the Jacobi preconditioner of
// Tools/Solver/include/ConjugateGradientCommon.h:74-161).  Same kernels as the per-step
// field solve.
#include "../../include/scdat_b200.h"
#include "pcg_csr.cuh"

#include <cmath>
#include <cstring>

namespace scdat {

__global__ void k_reciprocal(int R, const double* __restrict__ d, double* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) out[i] = 1.0 / d[i];
}

// Device scratch of one solve: 6 R-vectors, the scalars and the reduction partials.
size_t pcg_scratch_bytes(int R, int grid)
{
    size_t v = (size_t)R * sizeof(double);
    v = (v + 255) & ~(size_t)255;
    return 6 * v + 256 + (((size_t)grid * 4 * sizeof(double) + 255) & ~(size_t)255);
}

PcgScratch pcg_scratch_carve(void* base, int R, int grid)
{
    size_t v = (((size_t)R * sizeof(double)) + 255) & ~(size_t)255;
    char* p = static_cast<char*>(base);
    PcgScratch s;
    s.dinv = reinterpret_cast<double*>(p); p += v;
    s.r = reinterpret_cast<double*>(p); p += v;
    s.z = reinterpret_cast<double*>(p); p += v;
    s.p = reinterpret_cast<double*>(p); p += v;
    s.pn = reinterpret_cast<double*>(p); p += v;
    s.q = reinterpret_cast<double*>(p); p += v;
    s.sc = reinterpret_cast<PcgScalars*>(p); p += 256;
    s.part = reinterpret_cast<double*>(p);
    (void)grid;
    return s;
}

// Runs the solve on `st` with the given scratch; blocks until done (host reads the
// convergence flag every 16 iterations).  Returns a cudaError_t.
cudaError_t pcg_csr_run(int R, const int32_t* row_ptr, const int32_t* col, const double* val, const double* diag,
                        const double* b, double* x, double rtol, int max_iter, cudaStream_t st, const PcgScratch& s,
                        int grid, int* iters, double* relres)
{
    PoissonView A{};
    A.R = R;
    A.row_ptr = row_ptr;
    A.col = col;
    A.val = val;
    A.diag = diag;
    A.dinv = s.dinv;
    k_reciprocal<<<grid, 256, 0, st>>>(R, diag, s.dinv);
    PcgScalars h{};
    h.rtol = rtol;
    h.max_iter = max_iter;
    cudaError_t e = cudaMemcpyAsync(s.sc, &h, sizeof(h), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    launch_pcg_init64(A, b, x, s.r, s.z, s.sc, s.part, grid, st);
    double* p = s.p;
    double* pn = s.pn;
    for (int k = 0; k < max_iter; k += 16) {
        for (int j = 0; j < 16; ++j) {
            launch_pcg_iter64(A, x, s.r, s.z, p, pn, s.q, s.sc, s.part, grid, st);
            double* t = p;
            p = pn;
            pn = t;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(&h, s.sc, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        if (h.done) break;
    }
    if ((e = cudaMemcpyAsync(&h, s.sc, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    if (iters) *iters = h.iter;
    if (relres) *relres = std::sqrt(h.rr / (h.bb > 0.0 ? h.bb : 1.0));
    return cudaGetLastError();
}

}  // namespace scdat

using namespace scdat;

extern "C" SCDAT_API int scdat_pcg_csr(int32_t R, const int32_t* row_ptr, const int32_t* col, const double* val,
                                       const double* diag, const double* b, double* x, double rtol, int32_t max_iter,
                                       void* stream, int32_t* iterations, double* relres)
{
    if (R < 0 || max_iter < 0 || !(rtol >= 0.0)) return SCDAT_ERR_ARG;
    if (R == 0) {
        if (iterations) *iterations = 0;
        if (relres) *relres = 0.0;
        return SCDAT_OK;
    }
    if (!row_ptr || !diag || !b || !x) return SCDAT_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = 148 * 4;
    void* base = nullptr;
    if (cudaMalloc(&base, pcg_scratch_bytes(R, grid)) != cudaSuccess) return SCDAT_ERR_CUDA;
    PcgScratch s = pcg_scratch_carve(base, R, grid);
    int it = 0;
    double rel = 0.0;
    cudaError_t e = pcg_csr_run(R, row_ptr, col, val, diag, b, x, rtol, max_iter, st, s, grid, &it, &rel);
    cudaFree(base);
    if (e != cudaSuccess) return SCDAT_ERR_CUDA;
    if (iterations) *iterations = it;
    if (relres) *relres = rel;
    // converged only when the residual test holds: an iteration cap, a CG breakdown (p.Ap <= 0,
    // e.g. an indefinite matrix) or a non-finite residual (a zero diagonal entry) all report
    // NOT_CONVERGED, as LinearSystem::conjugateGradient returns false on |pAp| < 1e-30
    // (LinearSystem.cpp:258-327)
    return (rel <= rtol) ? SCDAT_OK : SCDAT_ERR_NOT_CONVERGED;
}
