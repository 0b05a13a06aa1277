// push_f64.cu -- the plain FP64 particle step: one thread per particle runs
// CrossTetrahedron::integrateTrajectory (PICParticleAlgorithms.cpp:536-740) with the
// adaptive sub-step (:750-801), Boris with B = 0 (:803-851), relocation (:853-891) and the
// per-sub-step trajectory deposit (:371-433), then the runtime boundary events
// (PICCycle.cpp:1221-1379) and, when enabled, the elastic background MCC.
//
// Charge goes into per-species 128-bit fixed-point node accumulators: the 10 sample points
// of a sub-step are summed exactly in registers, then each of the tet's 4 nodes takes one
// 64-bit atomic (plus one on carry), so the deposit is exact and order independent.
#include "push.cuh"

namespace scdat {

struct DepositAcc {
    Fx128 n[4];
    bool any;
};

__device__ __forceinline__ void dep_point(DepositAcc& acc, const double lam[4], double cw, double inv_uq)
{
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        Fx128 f = fx_from_double((cw * lam[i]) * inv_uq);
        fx_add(acc.n[i], f);
    }
    acc.any = true;
}

// ChargeDepositor::depositChargeAlongTrajectory into the post-move tet t
// (PICParticleAlgorithms.cpp:371-433); each sample point counts only when it lies in t.
__device__ __forceinline__ void deposit_traj(const MeshView& M, const SpeciesDev& S, const PushParams& pp, int t,
                                             double sx, double sy, double sz, double ex, double ey, double ez,
                                             unsigned long long* rlo, unsigned long long* rhi)
{
    DepositAcc acc;
#pragma unroll
    for (int i = 0; i < 4; ++i) acc.n[i] = Fx128{0ull, 0ll};
    acc.any = false;
    double tx = ex - sx, ty = ey - sy, tz = ez - sz;
    double lam[4];
    const double qw = S.q * S.w;
    if (sqrt(tx * tx + ty * ty + tz * tz) < 1e-15) {
        if (bary64(M, t, sx, sy, sz, lam)) dep_point(acc, lam, qw, pp.inv_uq);
    } else if (pp.dep_kernel == 0) {  // NearestPoint
        if (bary64(M, t, ex, ey, ez, lam)) dep_point(acc, lam, qw, pp.inv_uq);
    } else {
        // barycentrics are affine along the segment: lam(s + tau*tr) = lam_s + tau*dlam
        const double* g = M.geom + 12 * (int64_t)t;
        double ls[4], dl[4];
        bary64(M, t, sx, sy, sz, ls);
        dl[1] = __ldg(g + 0) * tx + __ldg(g + 1) * ty + __ldg(g + 2) * tz;
        dl[2] = __ldg(g + 3) * tx + __ldg(g + 4) * ty + __ldg(g + 5) * tz;
        dl[3] = __ldg(g + 6) * tx + __ldg(g + 7) * ty + __ldg(g + 8) * tz;
        dl[0] = -dl[1] - dl[2] - dl[3];
        const int nseg = pp.nseg;
        if (pp.dep_kernel == 2) {  // QuadratureGauss3
            const double gn[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};
            const double gw[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
            for (int sg = 0; sg < nseg; ++sg) {
                double t0 = (double)sg / (double)nseg, t1 = (double)(sg + 1) / (double)nseg;
                double tc = 0.5 * (t0 + t1), th = 0.5 * (t1 - t0);
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    double tau = tc + th * gn[q];
                    double l[4] = {ls[0] + tau * dl[0], ls[1] + tau * dl[1], ls[2] + tau * dl[2], ls[3] + tau * dl[3]};
                    if (bary_inside(l)) dep_point(acc, l, (S.q * gw[q] / (double)nseg) * S.w, pp.inv_uq);
                }
            }
        } else {  // LinearSegmentCloud
            for (int sg = 0; sg < nseg; ++sg) {
                double tau = ((double)sg + 0.5) / (double)nseg;
                double l[4] = {ls[0] + tau * dl[0], ls[1] + tau * dl[1], ls[2] + tau * dl[2], ls[3] + tau * dl[3]};
                if (bary_inside(l)) dep_point(acc, l, S.cw_seg, pp.inv_uq);
            }
        }
    }
    if (!acc.any) return;
    int4 tn = __ldg(M.tet + t);
    fx_atomic_add(rlo + tn.x, rhi + tn.x, acc.n[0]);
    fx_atomic_add(rlo + tn.y, rhi + tn.y, acc.n[1]);
    fx_atomic_add(rlo + tn.z, rhi + tn.z, acc.n[2]);
    fx_atomic_add(rlo + tn.w, rhi + tn.w, acc.n[3]);
}

__device__ __forceinline__ void gather_e(const MeshView& M, const double* __restrict__ E, int t, double px, double py,
                                         double pz, double& Ex, double& Ey, double& Ez)
{
    double lam[4];
    Ex = Ey = Ez = 0.0;
    if (!bary64(M, t, px, py, pz, lam)) return;  // interpolateVectorField returns 0 outside
    int4 tn = __ldg(M.tet + t);
    int nd[4] = {tn.x, tn.y, tn.z, tn.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double* e = E + 3 * (int64_t)nd[i];
        Ex = Ex + __ldg(e) * lam[i];
        Ey = Ey + __ldg(e + 1) * lam[i];
        Ez = Ez + __ldg(e + 2) * lam[i];
    }
}

__global__ void __launch_bounds__(256) k_push_f64(MeshView M, ParticleStore P, SpeciesDev S, PushParams pp,
                                                  const double* __restrict__ E, unsigned long long* rlo,
                                                  unsigned long long* rhi, LedgerDev* L, double* ke_part)
{
    const int64_t n = *P.count;
    double ke_sum = 0.0;
    unsigned long long nsub = 0, nlost = 0, nhit = 0, nact = 0;
    const double qm = S.qm;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int t0 = P.tet[i];
        if (t0 <= kTetAbsorbed) continue;
        double px = P.x[i], py = P.y[i], pz = P.z[i];
        double vx = P.vx[i], vy = P.vy[i], vz = P.vz[i];
        const double vstart = sqrt(vx * vx + vy * vy + vz * vz);
        int cur = locate(M, px, py, pz, t0);
        bool lost = false;
        int tet_out;
        if (cur < 0) {
            lost = true;
            cur = 0;  // result.final_element stays 0 (PICParticleAlgorithms.cpp:543,577)
        } else {
            double remaining = pp.dt;
            int it = 0;
            while (remaining > kMinTimeStep && it < kMaxSubsteps) {
                ++it;
                double Ex, Ey, Ez;
                gather_e(M, E, cur, px, py, pz, Ex, Ey, Ez);
                // CrossTetrahedron::adaptiveTimeStep with |B| = 0
                double adt = remaining;
                double Em = sqrt(Ex * Ex + Ey * Ey + Ez * Ez);
                if (Em > 1e-10) {
                    double acc = Em * fabs(qm);
                    if (acc > 1e-10 && vstart > 1.0) adt = fmin(adt, 0.1 * vstart / acc);
                }
                adt = fmax(adt, remaining * pp.floor_ratio);
                adt = fmin(adt, remaining);
                const double sx = px, sy = py, sz = pz;
                if (fabs(qm) > 1e-20) {
                    double f = qm * (0.5 * adt);
                    vx = vx + Ex * f; vy = vy + Ey * f; vz = vz + Ez * f;
                    vx = vx + Ex * f; vy = vy + Ey * f; vz = vz + Ez * f;
                }
                px = px + vx * adt;
                py = py + vy * adt;
                pz = pz + vz * adt;
                double lam[4];
                if (!bary64(M, cur, px, py, pz, lam)) {
                    int nt = locate(M, px, py, pz, cur);
                    if (nt < 0) {
                        lost = true;
                        break;
                    }
                    cur = nt;
                }
                if (pp.deposit) deposit_traj(M, S, pp, cur, sx, sy, sz, px, py, pz, rlo, rhi);
                remaining -= adt;
                ++nsub;
            }
            if (it >= kMaxSubsteps) lost = true;
        }
        tet_out = cur;
        const double ke = 0.5 * S.m * (vx * vx + vy * vy + vz * vz);
        if (lost) {
            ++nlost;
            tet_out = resolve_lost(M, S, pp, L, px, py, pz, ke, cur);
        }
        ke_sum += ke;  // updateStatistics counts every stored particle (PICCycle.cpp:941-966)
        if (tet_out >= 0) {
            ++nact;
            if (pp.do_mcc && S.mcc_enabled && mcc_elastic(S, pp, P.id[i], vx, vy, vz)) ++nhit;
        }
        P.x[i] = px; P.y[i] = py; P.z[i] = pz;
        P.vx[i] = vx; P.vy[i] = vy; P.vz[i] = vz;
        P.tet[i] = tet_out;
    }
    // block reduction of the statistics (fixed order -> deterministic)
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

// Standalone MCC pass (executeBackgroundMccStep, CollisionPicAdapter.cpp:338-434).
__global__ void k_mcc_f64(ParticleStore P, SpeciesDev S, PushParams pp, LedgerDev* L)
{
    const int64_t n = *P.count;
    unsigned long long nhit = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (P.tet[i] <= kTetAbsorbed) continue;
        double vx = P.vx[i], vy = P.vy[i], vz = P.vz[i];
        if (mcc_elastic(S, pp, P.id[i], vx, vy, vz)) {
            P.vx[i] = vx; P.vy[i] = vy; P.vz[i] = vz;
            ++nhit;
        }
    }
    if (nhit) atomicAdd(&L->mcc_hits, nhit);
}

void launch_push_f64(const MeshView& M, const ParticleStore& P, const SpeciesDev& S, const PushParams& pp,
                     const double* E, unsigned long long* rlo, unsigned long long* rhi, LedgerDev* L, double* ke_part,
                     int grid, cudaStream_t st)
{
    k_push_f64<<<grid, 256, 0, st>>>(M, P, S, pp, E, rlo, rhi, L, ke_part);
}

void launch_mcc_f64(const ParticleStore& P, const SpeciesDev& S, const PushParams& pp, LedgerDev* L, int grid,
                    cudaStream_t st)
{
    k_mcc_f64<<<grid, 256, 0, st>>>(P, S, pp, L);
}

}  // namespace scdat
