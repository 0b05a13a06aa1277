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

// One pass of the re-sort permutation over a species' whole store: the six coordinate arrays,
// the tet ids and the particle ids move together, and only the active prefix (the particles the
// sort keeps) is written.
template <typename T>
__global__ void k_gather_store(const int64_t* __restrict__ active, const uint32_t* __restrict__ perm,
                               GatherArrays<T> in, GatherArrays<T> out)
{
    const int64_t n = *active;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t j = __ldg(perm + i);
        T v[6];
#pragma unroll
        for (int a = 0; a < 6; ++a) v[a] = __ldg(in.v[a] + j);
        const int32_t t = __ldg(in.tet + j);
        const uint32_t id = __ldg(in.id + j);
#pragma unroll
        for (int a = 0; a < 6; ++a) out.v[a][i] = v[a];
        out.tet[i] = t;
        out.id[i] = id;
    }
}

template <typename T>
void launch_gather_store(int64_t n, const int64_t* active, const uint32_t* perm, const GatherArrays<T>& in,
                         const GatherArrays<T>& out, cudaStream_t st)
{
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    if (grid < 1) grid = 1;
    k_gather_store<T><<<grid, 256, 0, st>>>(active, perm, in, out);
}
// The same for the mixed form's 32-byte records (one sector each) and ids; the tet of a kept
// particle is its sorted key (read in order, not gathered): the tet id, or nohint_key for a
// particle without a hint.
__global__ void k_gather_mixed(const int64_t* __restrict__ active, const uint32_t* __restrict__ perm,
                               const uint32_t* __restrict__ sorted_keys, uint32_t nohint_key,
                               const float4* __restrict__ in_mix, const uint32_t* __restrict__ in_id,
                               float4* __restrict__ out_mix, int32_t* __restrict__ out_tet,
                               uint32_t* __restrict__ out_id)
{
    const int64_t n = *active;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t j = __ldg(perm + i);
        const float4 a = __ldg(in_mix + 2 * (int64_t)j), b = __ldg(in_mix + 2 * (int64_t)j + 1);
        const uint32_t key = __ldg(sorted_keys + i);
        const int32_t t = key < nohint_key ? (int32_t)key : kTetNoHint;
        const uint32_t id = __ldg(in_id + j);
        out_mix[2 * i] = a;
        out_mix[2 * i + 1] = b;
        out_tet[i] = t;
        out_id[i] = id;
    }
}

void launch_gather_mixed(int64_t n, const int64_t* active, const uint32_t* perm, const uint32_t* sorted_keys,
                         uint32_t nohint_key, const float4* in_mix, const uint32_t* in_id, float4* out_mix,
                         int32_t* out_tet, uint32_t* out_id, cudaStream_t st)
{
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    if (grid < 1) grid = 1;
    k_gather_mixed<<<grid, 256, 0, st>>>(active, perm, sorted_keys, nohint_key, in_mix, in_id, out_mix, out_tet,
                                         out_id);
}

template void launch_gather_store<double>(int64_t, const int64_t*, const uint32_t*, const GatherArrays<double>&,
                                          const GatherArrays<double>&, cudaStream_t);

__global__ void k_scatter_values(int64_t n, const int64_t* __restrict__ idx, const double* __restrict__ v, double* dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[idx[i]] = v[i];
}

// Start of a push: each species' maximum speed of the previous push becomes the one the
// null-collision MCC uses ([2s] <- [2s+1]), and the current slot starts from zero.
__global__ void k_rotate_vmax(int S, unsigned* v)
{
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
        v[2 * s] = v[2 * s + 1];
        v[2 * s + 1] = 0u;
    }
}

void launch_rotate_vmax(int S, unsigned* v, cudaStream_t st) { k_rotate_vmax<<<1, 32, 0, st>>>(S, v); }

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
            mix_store(P, k, (float)(x - M.xyz[3 * o]), (float)(y - M.xyz[3 * o + 1]), (float)(z - M.xyz[3 * o + 2]),
                      (float)vx, (float)vy, (float)vz);
        } else {
            P.x[k] = x; P.y[k] = y; P.z[k] = z;
            P.vx[k] = vx; P.vy[k] = vy; P.vz[k] = vz;
        }
        P.tet[k] = tet;
        P.id[k] = (uint32_t)id;
    }
}

// ParticleSource sampling on a tet mesh: n_per_tet particles in each listed tet (all tets when
// tets == nullptr), positions uniform in the tet from Dirichlet(1,1,1,1) barycentric weights
// w_k = e_k / sum e, e_k = -log(max(1e-12, u_k)) (samplePointInTetra,
// Toolkit/Surface Charging/src/PicMccSurfaceCurrentSampler.cpp:270-287), velocities a drifting
// Maxwellian by Box-Muller; draws from Philox(seed) keyed by id = (tet_index * S + s) * n_per_tet + k.
__global__ void k_seed_tets(const int32_t* __restrict__ tets, int64_t ntet, int32_t per_tet, int32_t S_total, int32_t s,
                            double sigma, double dx, double dy, double dz, uint64_t seed, ParticleStore P, int mixed,
                            MeshView M)
{
    const int64_t n = ntet * per_tet;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = k / per_tet, j = k % per_tet;
        const int tet = tets ? tets[c] : (int)c;
        const uint64_t id = ((uint64_t)c * S_total + s) * per_tet + j;
        double u[4], g[4];
        uniform2(seed, id, 0u, 0u, u[0], u[1]);
        uniform2(seed, id, 0u, 1u, u[2], u[3]);
        uniform2(seed, id, 0u, 4u, g[0], g[1]);
        uniform2(seed, id, 0u, 5u, g[2], g[3]);
        double e[4], es = 0.0;
        for (int q = 0; q < 4; ++q) {
            e[q] = -log(fmax(1.0e-12, u[q]));
            es += e[q];
        }
        const int4 tn = M.tet[tet];
        const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
        double x = 0.0, y = 0.0, z = 0.0;
        for (int q = 0; q < 4; ++q) {
            const double w = e[q] / es;
            x += w * M.xyz[3 * nd[q]];
            y += w * M.xyz[3 * nd[q] + 1];
            z += w * M.xyz[3 * nd[q] + 2];
        }
        const double r1 = sqrt(-2.0 * log(g[0])), r2 = sqrt(-2.0 * log(g[2]));
        const double tp = 6.283185307179586476925286766559;
        const double vx = dx + sigma * r1 * cos(tp * g[1]), vy = dy + sigma * r1 * sin(tp * g[1]),
                     vz = dz + sigma * r2 * cos(tp * g[3]);
        if (mixed) {
            mix_store(P, k, (float)(x - M.xyz[3 * nd[0]]), (float)(y - M.xyz[3 * nd[0] + 1]),
                      (float)(z - M.xyz[3 * nd[0] + 2]), (float)vx, (float)vy, (float)vz);
        } else {
            P.x[k] = x; P.y[k] = y; P.z[k] = z;
            P.vx[k] = vx; P.vy[k] = vy; P.vz[k] = vz;
        }
        P.tet[k] = tet;
        P.id[k] = (uint32_t)id;
    }
}

void launch_seed_tets(const int32_t* tets, int64_t ntet, int32_t per_tet, int32_t S_total, int32_t s, double sigma,
                      const double drift[3], uint64_t seed, const ParticleStore& P, bool mixed, const MeshView& M,
                      cudaStream_t st)
{
    k_seed_tets<<<148 * 8, 256, 0, st>>>(tets, ntet, per_tet, S_total, s, sigma, drift[0], drift[1], drift[2], seed, P,
                                         mixed ? 1 : 0, M);
}

// Per-layer particle moments for the z-layer profile: weight and weight * v^2 of one species
// in n_layers equal slabs of [z0, z1] (double atomics: output only).
__global__ void k_layer_moments(ParticleStore P, int64_t n, int mixed, MeshView M, double z0, double z1, int n_layers,
                                double* __restrict__ cnt, double* __restrict__ v2)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int t = P.tet[i];
        if (t < 0) continue;
        double z, vx, vy, vz;
        if (mixed) {
            float rx, ry, rz, ux, uy, uz;
            mix_load(P, i, rx, ry, rz, ux, uy, uz);
            z = M.xyz[3 * __ldg(&M.tet[t].x) + 2] + (double)rz;
            vx = ux; vy = uy; vz = uz;
        } else {
            z = P.z[i];
            vx = P.vx[i]; vy = P.vy[i]; vz = P.vz[i];
        }
        int l = (int)((z - z0) / (z1 - z0) * n_layers);
        l = l < 0 ? 0 : (l >= n_layers ? n_layers - 1 : l);
        atomicAdd(cnt + l, 1.0);
        atomicAdd(v2 + l, vx * vx + vy * vy + vz * vz);
    }
}

void launch_layer_moments(const ParticleStore& P, int64_t n, bool mixed, const MeshView& M, double z0, double z1,
                          int n_layers, double* cnt, double* v2, cudaStream_t st)
{
    k_layer_moments<<<148 * 4, 256, 0, st>>>(P, n, mixed ? 1 : 0, M, z0, z1, n_layers, cnt, v2);
}

void launch_seed_box(const int32_t* hex_ijk, int64_t ncell, int32_t ppc, int32_t S_total, int32_t s, double h,
                     double sigma, uint64_t seed, const ParticleStore& P, bool mixed, const MeshView& M,
                     cudaStream_t st)
{
    k_seed_box<<<148 * 8, 256, 0, st>>>(hex_ijk, ncell, ppc, S_total, s, h, sigma, seed, P, mixed ? 1 : 0, M);
}

}  // namespace scdat
