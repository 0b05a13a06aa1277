// pcg_noalloc.cu -- the CSR Jacobi-PCG for callers that cannot allocate device memory.
//
// Some callers may not call cudaMalloc at all: code running inside a host application that
// owns a fixed device-memory arena (and hands the library only pointers into it), or code
// that runs while the allocator is unavailable or forbidden, e.g. from inside a driver
// callback.  This entry point gives them the solve of scdat_pcg_csr with no allocation: its
// scratch (six vectors of at most kNoAllocMaxRows doubles, the scalars and the reduction
// partials) lives in one file-scope __device__ array that every GPU loading the library
// keeps until the process exits.
#include "../../include/scdat_b200.h"
#include "pcg_csr.cuh"

#include <mutex>

namespace {

constexpr int kNoAllocGrid = 148 * 4;
constexpr int kNoAllocMaxRows = 1 << 18;  // 262,144 rows: about 12.6 MB of scratch
constexpr size_t kVecBytes = (((size_t)kNoAllocMaxRows * sizeof(double)) + 255) & ~(size_t)255;
constexpr size_t kScratchBytes = 6 * kVecBytes + 256 + ((((size_t)kNoAllocGrid * 4 * sizeof(double)) + 255) & ~(size_t)255);

__device__ __align__(256) unsigned char g_pcg_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_pcg_scratch on the current device (the host-side name of the array is
// only a stand-in).  Looked up once per device, with that device current.
cudaError_t scratch_address(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_pcg_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

using namespace scdat;

extern "C" SCDAT_API int scdat_pcg_csr_noalloc(int32_t R, const int32_t* row_ptr, const int32_t* col,
                                               const double* val, const double* diag, const double* b, double* x,
                                               double rtol, int32_t max_iter, void* stream, int32_t* iterations,
                                               double* relres)
{
    if (R < 0 || max_iter < 0 || !(rtol >= 0.0)) return SCDAT_ERR_ARG;
    if (R > kNoAllocMaxRows) return SCDAT_ERR_CAPACITY;
    if (R == 0) {
        if (iterations) *iterations = 0;
        if (relres) *relres = 0.0;
        return SCDAT_OK;
    }
    if (!row_ptr || !diag || !b || !x) return SCDAT_ERR_ARG;
    void* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return SCDAT_ERR_CUDA;
    PcgScratch s = pcg_scratch_carve(base, R, kNoAllocGrid);
    int it = 0;
    double rel = 0.0;
    cudaError_t e = pcg_csr_run(R, row_ptr, col, val, diag, b, x, rtol, max_iter, static_cast<cudaStream_t>(stream),
                                s, kNoAllocGrid, &it, &rel);
    if (e != cudaSuccess) return SCDAT_ERR_CUDA;
    if (iterations) *iterations = it;
    if (relres) *relres = rel;
    // same status rule as scdat_pcg_csr: anything short of the residual test is NOT_CONVERGED
    return (rel <= rtol) ? SCDAT_OK : SCDAT_ERR_NOT_CONVERGED;
}
