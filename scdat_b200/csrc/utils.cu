// utils.cu -- auxiliary device kernels: re-sort keys and gathers, node scatters, and the
// seeded generator of box plasmas (uniform in each hex cell, Maxwellian velocities from
// Philox streams keyed by particle id, the same streams the CPU oracle uses).
#include "push.cuh"

namespace scdat {

// key = tet id for active particles, inactive_key for absorbed/escaped ones (sorted last,
// then dropped: ParticleContainer::removeInactiveParticles, ParticleManager.cpp:157-177).
__global__ void k_sort_keys(int64_t n, const int32_t* __restrict__ tet, uint32_t inactive_key, uint32_t* keys,
                            uint32_t* vals, unsigned long long* active)
{
    unsigned long long a = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int t = tet[i];
        bool act = t >= kTetNoHint;
        // an active particle without a hint sorts just before the inactive ones
        keys[i] = act ? (t >= 0 ? (uint32_t)t : inactive_key - 1u) : inactive_key;
        vals[i] = (uint32_t)i;
        a += act ? 1ull : 0ull;
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(active, a);
}

void launch_sort_keys(int64_t n, const int32_t* tet, uint32_t inactive_key, uint32_t* keys, uint32_t* vals,
                      int64_t* active, cudaStream_t st)
{
    cudaMemsetAsync(active, 0, sizeof(int64_t), st);
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    if (grid < 1) grid = 1;
    k_sort_keys<<<grid, 256, 0, st>>>(n, tet, inactive_key + 1u, keys, vals, reinterpret_cast<unsigned long long*>(active));
}

template <typename T>
__global__ void k_gather(int64_t n, const uint32_t* __restrict__ perm, const T* __restrict__ in, T* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[perm[i]];
}

template <typename T>
void launch_gather(int64_t n, const uint32_t* perm, const T* in, T* out, cudaStream_t st)
{
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    if (grid < 1) grid = 1;
    k_gather<T><<<grid, 256, 0, st>>>(n, perm, in, out);
}
template void launch_gather<double>(int64_t, const uint32_t*, const double*, double*, cudaStream_t);
template void launch_gather<float>(int64_t, const uint32_t*, const float*, float*, cudaStream_t);
template void launch_gather<int32_t>(int64_t, const uint32_t*, const int32_t*, int32_t*, cudaStream_t);
template void launch_gather<uint32_t>(int64_t, const uint32_t*, const uint32_t*, uint32_t*, cudaStream_t);

__global__ void k_scatter_values(int64_t n, const int64_t* __restrict__ idx, const double* __restrict__ v, double* dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[idx[i]] = v[i];
}

void launch_scatter_values(int64_t n, const int64_t* idx, const double* v, double* dst, cudaStream_t st)
{
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    if (grid < 1) grid = 1;
    k_scatter_values<<<grid, 256, 0, st>>>(n, idx, v, dst);
}

// Box-plasma seeding: particle k of species s in meshed hex c has id (c*S + s)*ppc + k.
// Position uniform in the hex from Philox purposes 0 and 1, velocity from Box-Muller on
// purposes 4 and 5; the tet is the Kuhn permutation that orders the local coordinates.
__global__ void k_seed_box(const int32_t* __restrict__ hex_ijk, int64_t ncell, int32_t ppc, int32_t S_total, int32_t s,
                           double h, double sigma, uint64_t seed, ParticleStore P, int mixed, MeshView M)
{
    const int64_t n = ncell * ppc;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = k / ppc, j = k % ppc;
        uint64_t id = ((uint64_t)c * S_total + s) * ppc + j;
        double u0, u1, u2, u3, g0, g1, g2, g3;
        uniform2(seed, id, 0u, 0u, u0, u1);
        uniform2(seed, id, 0u, 1u, u2, u3);
        uniform2(seed, id, 0u, 4u, g0, g1);
        uniform2(seed, id, 0u, 5u, g2, g3);
        double loc[3] = {u0, u1, u2};
        double x = ((double)hex_ijk[3 * c] + loc[0]) * h;
        double y = ((double)hex_ijk[3 * c + 1] + loc[1]) * h;
        double z = ((double)hex_ijk[3 * c + 2] + loc[2]) * h;
        // descending order of the local coordinates picks the Kuhn tet (stable on ties)
        int a = 0, b = 1, d = 2;
        if (loc[b] > loc[a]) { int t = a; a = b; b = t; }
        if (loc[d] > loc[b]) { int t = b; b = d; d = t; }
        if (loc[b] > loc[a]) { int t = a; a = b; b = t; }
        int perm = a == 0 ? (b == 1 ? 0 : 1) : (a == 1 ? (b == 0 ? 2 : 3) : (b == 0 ? 4 : 5));
        int tet = (int)(6 * c + perm);
        double r1 = sqrt(-2.0 * log(g0)), r2 = sqrt(-2.0 * log(g2));
        const double tp = 6.283185307179586476925286766559;
        double vx = sigma * r1 * cos(tp * g1), vy = sigma * r1 * sin(tp * g1), vz = sigma * r2 * cos(tp * g3);
        if (mixed) {
            int o = __ldg(&M.tet[tet].x);
            P.xf[k] = (float)(x - M.xyz[3 * o]);
            P.yf[k] = (float)(y - M.xyz[3 * o + 1]);
            P.zf[k] = (float)(z - M.xyz[3 * o + 2]);
            P.vxf[k] = (float)vx; P.vyf[k] = (float)vy; P.vzf[k] = (float)vz;
        } else {
            P.x[k] = x; P.y[k] = y; P.z[k] = z;
            P.vx[k] = vx; P.vy[k] = vy; P.vz[k] = vz;
        }
        P.tet[k] = tet;
        P.id[k] = (uint32_t)id;
    }
}

void launch_seed_box(const int32_t* hex_ijk, int64_t ncell, int32_t ppc, int32_t S_total, int32_t s, double h,
                     double sigma, uint64_t seed, const ParticleStore& P, bool mixed, const MeshView& M,
                     cudaStream_t st)
{
    k_seed_box<<<148 * 8, 256, 0, st>>>(hex_ijk, ncell, ppc, S_total, s, h, sigma, seed, P, mixed ? 1 : 0, M);
}

}  // namespace scdat
