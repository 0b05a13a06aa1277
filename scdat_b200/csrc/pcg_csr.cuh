// pcg_csr.cuh -- the shared driver of the context-free CSR Jacobi-PCG entry points.
#pragma once

#include "field.cuh"

namespace scdat {

struct PcgScratch {
    double *dinv, *r, *z, *p, *pn, *q;
    PcgScalars* sc;
    double* part;
};

size_t pcg_scratch_bytes(int R, int grid);
PcgScratch pcg_scratch_carve(void* base, int R, int grid);
cudaError_t pcg_csr_run(int R, const int32_t* row_ptr, const int32_t* col, const double* val, const double* diag,
                        const double* b, double* x, double rtol, int max_iter, cudaStream_t st, const PcgScratch& s,
                        int grid, int* iters, double* relres);

}  // namespace scdat
