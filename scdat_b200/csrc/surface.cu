// surface.cu -- device kernels of the surface circuit (see surface.cuh).
#include "surface.cuh"

#include <algorithm>

namespace scdat {

__global__ void k_surface_advance(SurfaceDev* S, LedgerDev* L, double unit, double dt)
{
    const int k = threadIdx.x;
    if (k < S->n) surface_advance_face(S, L, k, unit, dt);
}

// phi of each surface node = mean of the potentials of the faces in its mask (ascending order)
__global__ void k_surface_apply(const SurfaceDev* __restrict__ S, int64_t n, const int32_t* __restrict__ node,
                                const uint8_t* __restrict__ mask, double* __restrict__ phi)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (mask[i]) phi[node[i]] = surface_node_potential(S, mask[i]);
}

void launch_surface_advance(SurfaceDev* S, LedgerDev* L, double unit, double dt, cudaStream_t st)
{
    k_surface_advance<<<1, 32, 0, st>>>(S, L, unit, dt);
}

void launch_surface_apply(const SurfaceDev* S, int64_t n, const int32_t* node, const uint8_t* mask, double* phi,
                          cudaStream_t st)
{
    if (n <= 0) return;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 1184);
    k_surface_apply<<<grid, 256, 0, st>>>(S, n, node, mask, phi);
}

}  // namespace scdat
