// push_mixed.cu -- the precision form of the particle step.
//
// Particles store FP32 positions relative to the origin node (local vertex 0) of their tet
// and FP32 velocities (28 bytes with the tet id, against 52 in FP64).  Gather, adaptive
// sub-step, Boris and the in-tet test run in FP32 on the FP32 inverse Jacobians and FP32
// nodal E; a move into a face neighbour is re-based in FP32 from the FP64 node difference;
// anything farther (walk, grid lookup, boundary events) reconstructs the FP64 absolute
// position and uses the FP64 locate.  Deposit weights are FP32 barycentrics promoted to
// FP64 before the exact fixed-point accumulation.  The step structure is the reference's
// CrossTetrahedron::integrateTrajectory (PICParticleAlgorithms.cpp:536-740).
#include "push.cuh"

namespace scdat {

__device__ __forceinline__ bool inside_f(const float l[4])
{
    const float e = 1e-8f;
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) ok = ok && (l[i] >= -e) && (l[i] <= 1.0f + e);
    return ok;
}

struct GeomF {
    float j[9];
};

__device__ __forceinline__ GeomF load_geomf(const MeshView& M, int t)
{
    const float4* g = reinterpret_cast<const float4*>(M.geomf + 12 * (int64_t)t);
    float4 a = __ldg(g), b = __ldg(g + 1);
    float c = __ldg(M.geomf + 12 * (int64_t)t + 8);
    GeomF G;
    G.j[0] = a.x; G.j[1] = a.y; G.j[2] = a.z; G.j[3] = a.w;
    G.j[4] = b.x; G.j[5] = b.y; G.j[6] = b.z; G.j[7] = b.w; G.j[8] = c;
    return G;
}

__device__ __forceinline__ void baryf(const GeomF& G, float rx, float ry, float rz, float l[4])
{
    l[1] = G.j[0] * rx + G.j[1] * ry + G.j[2] * rz;
    l[2] = G.j[3] * rx + G.j[4] * ry + G.j[5] * rz;
    l[3] = G.j[6] * rx + G.j[7] * ry + G.j[8] * rz;
    l[0] = 1.0f - l[1] - l[2] - l[3];
}

__device__ __forceinline__ double3 origin(const MeshView& M, int t)
{
    int o = __ldg(&M.tet[t].x);
    return make_double3(__ldg(M.xyz + 3 * o), __ldg(M.xyz + 3 * o + 1), __ldg(M.xyz + 3 * o + 2));
}

__device__ __forceinline__ void dep_point_f(Fx128 acc[4], bool& any, const float l[4], double cw, double inv_uq)
{
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        Fx128 f = fx_from_double((cw * (double)l[i]) * inv_uq);
        fx_add(acc[i], f);
    }
    any = true;
}

// Relocate the FP32 offset r (relative to origin of `cur`): neighbour list first in FP32,
// then the FP64 walk / grid lookup.  Returns the new tet or -1; r and the carried start
// offset s are re-based to the new origin.
__device__ __forceinline__ int relocate_f(const MeshView& M, int cur, float& rx, float& ry, float& rz, float& sx,
                                          float& sy, float& sz)
{
    const double3 oc = origin(M, cur);
    if (M.use_nbr) {
        int4 nb = __ldg(M.nbr + cur);
        int cand[4] = {nb.x, nb.y, nb.z, nb.w};
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            int t = cand[f];
            if (t < 0) continue;
            double3 on = origin(M, t);
            float dx = (float)(oc.x - on.x), dy = (float)(oc.y - on.y), dz = (float)(oc.z - on.z);
            float qx = rx + dx, qy = ry + dy, qz = rz + dz;
            float l[4];
            baryf(load_geomf(M, t), qx, qy, qz, l);
            if (inside_f(l)) {
                rx = qx; ry = qy; rz = qz;
                sx += dx; sy += dy; sz += dz;
                return t;
            }
        }
    }
    double px = oc.x + (double)rx, py = oc.y + (double)ry, pz = oc.z + (double)rz;
    int t = locate_far(M, px, py, pz, cur);
    if (t < 0) return -1;
    double3 on = origin(M, t);
    float dx = (float)(oc.x - on.x), dy = (float)(oc.y - on.y), dz = (float)(oc.z - on.z);
    rx = (float)(px - on.x); ry = (float)(py - on.y); rz = (float)(pz - on.z);
    sx += dx; sy += dy; sz += dz;
    return t;
}

__global__ void __launch_bounds__(256) k_push_mixed(MeshView M, ParticleStore P, SpeciesDev S, PushParams pp,
                                                    const float* __restrict__ Ef, unsigned long long* rlo,
                                                    unsigned long long* rhi, LedgerDev* L, double* ke_part)
{
    const int64_t n = *P.count;
    double ke_sum = 0.0;
    unsigned long long nsub = 0, nlost = 0, nhit = 0, nact = 0;
    const float qm = (float)S.qm;
    const float dtf = (float)pp.dt;
    const float floor_ratio = (float)pp.floor_ratio;
    const int nseg = pp.nseg;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int cur = P.tet[i];
        if (cur <= kTetAbsorbed) continue;
        float rx = P.xf[i], ry = P.yf[i], rz = P.zf[i];
        float vx = P.vxf[i], vy = P.vyf[i], vz = P.vzf[i];
        const float vstart = sqrtf(vx * vx + vy * vy + vz * vz);
        bool lost = false;
        if (cur < 0) {
            // no hint: the offset is absolute (set when the particle was placed outside the mesh)
            double px = rx, py = ry, pz = rz;
            int t = locate_far(M, px, py, pz, -1);
            if (t < 0) {
                lost = true;
            } else {
                double3 o = origin(M, t);
                rx = (float)(px - o.x); ry = (float)(py - o.y); rz = (float)(pz - o.z);
                cur = t;
            }
        }
        if (!lost) {
            float remaining = dtf;
            int it = 0;
            while (remaining > 1e-20f && it < kMaxSubsteps) {
                ++it;
                GeomF G = load_geomf(M, cur);
                int4 tn = __ldg(M.tet + cur);
                float l[4];
                baryf(G, rx, ry, rz, l);
                float Ex = 0.f, Ey = 0.f, Ez = 0.f;
                if (inside_f(l)) {
                    int nd[4] = {tn.x, tn.y, tn.z, tn.w};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float* e = Ef + 3 * (int64_t)nd[k];
                        Ex = fmaf(__ldg(e), l[k], Ex);
                        Ey = fmaf(__ldg(e + 1), l[k], Ey);
                        Ez = fmaf(__ldg(e + 2), l[k], Ez);
                    }
                }
                float adt = remaining;
                float Em = sqrtf(Ex * Ex + Ey * Ey + Ez * Ez);
                if (Em > 1e-10f) {
                    float acc = Em * fabsf(qm);
                    if (acc > 1e-10f && vstart > 1.0f) adt = fminf(adt, 0.1f * vstart / acc);
                }
                adt = fmaxf(adt, remaining * floor_ratio);
                adt = fminf(adt, remaining);
                float sx = rx, sy = ry, sz = rz;
                if (fabsf(qm) > 1e-20f) {
                    float f = qm * (0.5f * adt);
                    vx = fmaf(2.0f * f, Ex, vx);
                    vy = fmaf(2.0f * f, Ey, vy);
                    vz = fmaf(2.0f * f, Ez, vz);
                }
                rx = fmaf(vx, adt, rx);
                ry = fmaf(vy, adt, ry);
                rz = fmaf(vz, adt, rz);
                baryf(G, rx, ry, rz, l);
                if (!inside_f(l)) {
                    int nt = relocate_f(M, cur, rx, ry, rz, sx, sy, sz);
                    if (nt < 0) {
                        lost = true;
                        break;
                    }
                    cur = nt;
                    G = load_geomf(M, cur);
                    tn = __ldg(M.tet + cur);
                }
                // deposit along start -> end in the post-move tet
                Fx128 acc[4] = {{0ull, 0ll}, {0ull, 0ll}, {0ull, 0ll}, {0ull, 0ll}};
                bool any = false;
                float tx = rx - sx, ty = ry - sy, tz = rz - sz;
                if (sqrtf(tx * tx + ty * ty + tz * tz) < 1e-15f) {
                    float q0[4];
                    baryf(G, sx, sy, sz, q0);
                    if (inside_f(q0)) dep_point_f(acc, any, q0, S.q * S.w, pp.inv_uq);
                } else if (pp.dep_kernel == 0) {
                    float q0[4];
                    baryf(G, rx, ry, rz, q0);
                    if (inside_f(q0)) dep_point_f(acc, any, q0, S.q * S.w, pp.inv_uq);
                } else {
                    float ls[4], dl[4];
                    baryf(G, sx, sy, sz, ls);
                    dl[1] = G.j[0] * tx + G.j[1] * ty + G.j[2] * tz;
                    dl[2] = G.j[3] * tx + G.j[4] * ty + G.j[5] * tz;
                    dl[3] = G.j[6] * tx + G.j[7] * ty + G.j[8] * tz;
                    dl[0] = -dl[1] - dl[2] - dl[3];
                    if (pp.dep_kernel == 2) {
                        const float gn[3] = {-0.7745966692414834f, 0.0f, 0.7745966692414834f};
                        const double gw[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
                        for (int sg = 0; sg < nseg; ++sg) {
                            float tc = ((float)sg + 0.5f) / (float)nseg, th = 0.5f / (float)nseg;
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                float tau = tc + th * gn[q];
                                float lq[4] = {ls[0] + tau * dl[0], ls[1] + tau * dl[1], ls[2] + tau * dl[2],
                                               ls[3] + tau * dl[3]};
                                if (inside_f(lq)) dep_point_f(acc, any, lq, (S.q * gw[q] / (double)nseg) * S.w, pp.inv_uq);
                            }
                        }
                    } else {
                        for (int sg = 0; sg < nseg; ++sg) {
                            float tau = ((float)sg + 0.5f) / (float)nseg;
                            float lq[4] = {ls[0] + tau * dl[0], ls[1] + tau * dl[1], ls[2] + tau * dl[2],
                                           ls[3] + tau * dl[3]};
                            if (inside_f(lq)) dep_point_f(acc, any, lq, S.cw_seg, pp.inv_uq);
                        }
                    }
                }
                if (any && pp.deposit) {
                    fx_atomic_add(rlo + tn.x, rhi + tn.x, acc[0]);
                    fx_atomic_add(rlo + tn.y, rhi + tn.y, acc[1]);
                    fx_atomic_add(rlo + tn.z, rhi + tn.z, acc[2]);
                    fx_atomic_add(rlo + tn.w, rhi + tn.w, acc[3]);
                }
                remaining -= adt;
                ++nsub;
            }
            if (it >= kMaxSubsteps) lost = true;
        }
        double dvx = vx, dvy = vy, dvz = vz;
        const double ke = 0.5 * S.m * (dvx * dvx + dvy * dvy + dvz * dvz);
        int tet_out = cur;
        if (lost) {
            ++nlost;
            // absolute position in FP64 for the boundary events
            double px, py, pz;
            if (cur >= 0) {
                double3 o = origin(M, cur);
                px = o.x + (double)rx; py = o.y + (double)ry; pz = o.z + (double)rz;
            } else {
                px = rx; py = ry; pz = rz;
                cur = 0;
            }
            tet_out = resolve_lost(M, S, pp, L, px, py, pz, ke, cur);
            if (tet_out >= 0) {
                double3 o = origin(M, tet_out);
                rx = (float)(px - o.x); ry = (float)(py - o.y); rz = (float)(pz - o.z);
            } else {
                // inactive particles keep an absolute FP32 position for read-back
                rx = (float)px; ry = (float)py; rz = (float)pz;
            }
        }
        ke_sum += ke;
        if (tet_out >= 0) {
            ++nact;
            if (pp.do_mcc && S.mcc_enabled && mcc_elastic(S, pp, P.id[i], dvx, dvy, dvz)) {
                ++nhit;
                vx = (float)dvx; vy = (float)dvy; vz = (float)dvz;
            }
        }
        P.xf[i] = rx; P.yf[i] = ry; P.zf[i] = rz;
        P.vxf[i] = vx; P.vyf[i] = vy; P.vzf[i] = vz;
        P.tet[i] = tet_out;
    }
    __shared__ double sk[256];
    __shared__ unsigned long long sc[4][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        nsub += __shfl_down_sync(0xffffffffu, nsub, o);
        nlost += __shfl_down_sync(0xffffffffu, nlost, o);
        nhit += __shfl_down_sync(0xffffffffu, nhit, o);
        nact += __shfl_down_sync(0xffffffffu, nact, o);
    }
    if (lane == 0) {
        sc[0][warp] = nsub; sc[1][warp] = nlost; sc[2][warp] = nhit; sc[3][warp] = nact;
    }
    sk[threadIdx.x] = ke_sum;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sk[threadIdx.x] += sk[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ke_part[blockIdx.x] += sk[0];
        unsigned long long a = 0, b = 0, c = 0, d = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += sc[0][w]; b += sc[1][w]; c += sc[2][w]; d += sc[3][w];
        }
        if (a) atomicAdd(&L->substeps, a);
        if (b) atomicAdd(&L->lost_events, b);
        if (c) atomicAdd(&L->mcc_hits, c);
        if (d) atomicAdd(&L->active, d);
    }
}

__global__ void k_mcc_mixed(ParticleStore P, SpeciesDev S, PushParams pp, LedgerDev* L)
{
    const int64_t n = *P.count;
    unsigned long long nhit = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (P.tet[i] <= kTetAbsorbed) continue;
        double vx = P.vxf[i], vy = P.vyf[i], vz = P.vzf[i];
        if (mcc_elastic(S, pp, P.id[i], vx, vy, vz)) {
            P.vxf[i] = (float)vx; P.vyf[i] = (float)vy; P.vzf[i] = (float)vz;
            ++nhit;
        }
    }
    if (nhit) atomicAdd(&L->mcc_hits, nhit);
}

// FP64 absolute state -> tet-relative FP32 store (locating every particle from its hint).
__global__ void k_to_mixed(MeshView M, int64_t n, const double* x, const double* y, const double* z, const double* vx,
                           const double* vy, const double* vz, ParticleStore P)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int t = locate(M, x[i], y[i], z[i], P.tet[i]);
        if (t >= 0) {
            double3 o = origin(M, t);
            P.xf[i] = (float)(x[i] - o.x); P.yf[i] = (float)(y[i] - o.y); P.zf[i] = (float)(z[i] - o.z);
        } else {
            P.xf[i] = (float)x[i]; P.yf[i] = (float)y[i]; P.zf[i] = (float)z[i];
        }
        P.tet[i] = t >= 0 ? t : kTetNoHint;
        P.vxf[i] = (float)vx[i]; P.vyf[i] = (float)vy[i]; P.vzf[i] = (float)vz[i];
    }
}

__global__ void k_from_mixed(MeshView M, int64_t n, ParticleStore P, double* x, double* y, double* z, double* vx,
                             double* vy, double* vz)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int t = P.tet[i];
        double ox = 0.0, oy = 0.0, oz = 0.0;
        if (t >= 0) {
            double3 o = origin(M, t);
            ox = o.x; oy = o.y; oz = o.z;
        }
        x[i] = ox + (double)P.xf[i]; y[i] = oy + (double)P.yf[i]; z[i] = oz + (double)P.zf[i];
        vx[i] = P.vxf[i]; vy[i] = P.vyf[i]; vz[i] = P.vzf[i];
    }
}

void launch_push_mixed(const MeshView& M, const ParticleStore& P, const SpeciesDev& S, const PushParams& pp,
                       const float* Ef, unsigned long long* rlo, unsigned long long* rhi, LedgerDev* L,
                       double* ke_part, int grid, cudaStream_t st)
{
    k_push_mixed<<<grid, 256, 0, st>>>(M, P, S, pp, Ef, rlo, rhi, L, ke_part);
}

void launch_mcc_mixed(const ParticleStore& P, const SpeciesDev& S, const PushParams& pp, LedgerDev* L, int grid,
                      cudaStream_t st)
{
    k_mcc_mixed<<<grid, 256, 0, st>>>(P, S, pp, L);
}

void launch_to_mixed(const MeshView& M, int64_t n, const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz, const ParticleStore& P, cudaStream_t st)
{
    k_to_mixed<<<148 * 4, 256, 0, st>>>(M, n, x, y, z, vx, vy, vz, P);
}

void launch_from_mixed(const MeshView& M, int64_t n, const ParticleStore& P, double* x, double* y, double* z,
                       double* vx, double* vy, double* vz, cudaStream_t st)
{
    k_from_mixed<<<148 * 4, 256, 0, st>>>(M, n, P, x, y, z, vx, vy, vz);
}

}  // namespace scdat
