// push_f64.cu -- the plain FP64 particle step: one thread per particle runs
// CrossTetrahedron::integrateTrajectory (PICParticleAlgorithms.cpp:536-740) with the
// adaptive sub-step (:750-801), Boris with B = 0 (:803-851), relocation (:853-891) and the
// per-sub-step trajectory deposit (:371-433), then the runtime boundary events
// (PICCycle.cpp:1221-1379) and, when enabled, the elastic background MCC.
//
// Charge goes into per-species 128-bit fixed-point node accumulators staged per warp in
// shared memory, so the deposit is exact and independent of thread order.  The nodal E of
// each tet's 4 nodes is kept per tet (refreshed after every field solve), so the gather is
// one load beside the tet's geometry.  Sub-steps run in passes (see push_mixed.cu) to keep
// warps converged.
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
static __device__ __noinline__ void deposit_traj(const MeshView& M, const SpeciesDev& S, const PushParams& pp, int t,
                                                 double sx, double sy, double sz, double ex, double ey, double ez,
                                                 ChargeAcc A)
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
        const double* g = M.geom + 16 * (int64_t)t;
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
    int4 tn = rec_nodes(M, t);
    fx_red(A, tn.x, acc.n[0]);
    fx_red(A, tn.y, acc.n[1]);
    fx_red(A, tn.z, acc.n[2]);
    fx_red(A, tn.w, acc.n[3]);
}

struct FlightD {
    double px, py, pz, vx, vy, vz;
    double rem, vstart;
    int cur, it;
};

// Run sub-steps until the step's time is used up, the particle is lost, or `cap` sub-steps
// ran in this call.
__device__ __forceinline__ int advance_d(const MeshView& M, const SpeciesDev& S, const PushParams& pp, FlightD& f,
                                         int cap, ChargeAcc A,
                                         unsigned& nsub)
{
    const double qm = S.qm;
    const double qw = S.q * S.w;
    double lam[4];
    bool in = bary64(M, f.cur, f.px, f.py, f.pz, lam);  // reused as the next gather's weights
    int k = 0;
    while (f.rem > kMinTimeStep && f.it < kMaxSubsteps) {
        if (k == cap) return kCapped;
        ++k;
        ++f.it;
        double Ex = 0.0, Ey = 0.0, Ez = 0.0;
        if (in) {
            const double* e = M.erec + 12 * (int64_t)f.cur;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                Ex = Ex + __ldg(e + 3 * q) * lam[q];
                Ey = Ey + __ldg(e + 3 * q + 1) * lam[q];
                Ez = Ez + __ldg(e + 3 * q + 2) * lam[q];
            }
        }
        // CrossTetrahedron::adaptiveTimeStep with |B| = 0
        double adt = f.rem;
        double Em = sqrt(Ex * Ex + Ey * Ey + Ez * Ez);
        if (Em > 1e-10) {
            double acc = Em * fabs(qm);
            if (acc > 1e-10 && f.vstart > 1.0) adt = fmin(adt, 0.1 * f.vstart / acc);
        }
        adt = fmax(adt, f.rem * pp.floor_ratio);
        adt = fmin(adt, f.rem);
        const double sx = f.px, sy = f.py, sz = f.pz;
        if (fabs(qm) > 1e-20) {
            double h = qm * (0.5 * adt);
            f.vx = f.vx + Ex * h; f.vy = f.vy + Ey * h; f.vz = f.vz + Ez * h;
            f.vx = f.vx + Ex * h; f.vy = f.vy + Ey * h; f.vz = f.vz + Ez * h;
        }
        f.px = f.px + f.vx * adt;
        f.py = f.py + f.vy * adt;
        f.pz = f.pz + f.vz * adt;
        double le[4];
        if (bary64(M, f.cur, f.px, f.py, f.pz, le)) {
            if (pp.deposit) {
                if (in) {
                    // the segment stayed in the tet: the symmetric sample points sum to
                    // q*w*lambda(midpoint) for the segment-cloud and Gauss-3 kernels
                    double tx = f.px - sx, ty = f.py - sy, tz = f.pz - sz;
                    bool tiny = sqrt(tx * tx + ty * ty + tz * tz) < 1e-15;
                    int4 tn = rec_nodes(M, f.cur);
                    int nd[4] = {tn.x, tn.y, tn.z, tn.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        double lk = tiny ? lam[q] : (pp.dep_kernel == 0 ? le[q] : 0.5 * (lam[q] + le[q]));
                        fx_red(A, nd[q], fx_from_double((qw * lk) * pp.inv_uq));
                    }
                } else {
                    deposit_traj(M, S, pp, f.cur, sx, sy, sz, f.px, f.py, f.pz, A);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) lam[q] = le[q];
            in = true;
        } else {
            int nt = locate(M, f.px, f.py, f.pz, f.cur);
            if (nt < 0) return kLost;
            f.cur = nt;
            if (pp.deposit) deposit_traj(M, S, pp, nt, sx, sy, sz, f.px, f.py, f.pz, A);
            in = bary64(M, nt, f.px, f.py, f.pz, lam);
        }
        f.rem -= adt;
        ++nsub;
    }
    return f.it >= kMaxSubsteps ? kLost : kDone;
}

__device__ __forceinline__ void finish_d(const MeshView& M, const ParticleStore& P, const SpeciesDev& S,
                                         const PushParams& pp, LedgerDev* L, int64_t i, FlightD& f, int st,
                                         PushStats& c)
{
    const double ke = 0.5 * S.m * (f.vx * f.vx + f.vy * f.vy + f.vz * f.vz);
    int tet_out = f.cur;
    if (st == kLost) {
        c.ev |= kEvLost;
        tet_out = resolve_lost(M, S, pp, L, f.px, f.py, f.pz, ke, f.cur);
    }
    c.ke += ke;  // updateStatistics counts every stored particle (PICCycle.cpp:941-966)
    if (tet_out >= 0) {
        c.ev |= kEvActive;
        if (S.mcc_mode == 2) c.v2 = fmaxf(c.v2, (float)(f.vx * f.vx + f.vy * f.vy + f.vz * f.vz));  // the null-collision speed bound
        if (pp.do_mcc && S.mcc_enabled && mcc_elastic(S, pp, P.id[i], f.vx, f.vy, f.vz)) c.ev |= kEvHit;
    }
    P.x[i] = f.px; P.y[i] = f.py; P.z[i] = f.pz;
    P.vx[i] = f.vx; P.vy[i] = f.vy; P.vz[i] = f.vz;
    P.tet[i] = tet_out;
}

__device__ __forceinline__ void defer_store_d(const ParticleStore& P, const DeferList& D, unsigned slot, int64_t i,
                                              const FlightD& f)
{
    D.idx[slot] = (uint32_t)i;
    D.it[slot] = f.it;
    D.rem[slot] = f.rem;
    D.vstart[slot] = f.vstart;
    P.x[i] = f.px; P.y[i] = f.py; P.z[i] = f.pz;
    P.vx[i] = f.vx; P.vy[i] = f.vy; P.vz[i] = f.vz;
    P.tet[i] = f.cur;
}

// Pass 1: every stored particle, at most kCap1 sub-steps.
__global__ void __launch_bounds__(256) k_push_f64(const __grid_constant__ MeshView M, ParticleStore P,
    const __grid_constant__ SpeciesDev S, const __grid_constant__ PushParams pp,
                                                  DeferList D, ChargeAcc A,
                                                  LedgerDev* L, unsigned long long* ke_acc, unsigned* ctr)
{
    const int64_t n = *P.count;
    PushStats c{0.0, 0u, 0u};
    const int lane = threadIdx.x & 31;
    warp_stats_begin();
    for (;;) {
        // runs of kRun chunks, as in the mixed form
        const int64_t b0 = (int64_t)next_chunk(ctr) * (32 * kRun);
        if (b0 >= n) break;
        for (int64_t base = b0; base < b0 + 32 * kRun && base < n; base += 32) {
            const int64_t i = base + lane;
            int st = -1;
            FlightD f;
            if (i < n) {
                int t0 = P.tet[i];
                f.vx = P.vx[i]; f.vy = P.vy[i]; f.vz = P.vz[i];
                if (t0 <= kTetAbsorbed) {
                    // updateStatistics sums every particle the container still holds (PICCycle.cpp:941-966)
                    c.ke += 0.5 * S.m * (f.vx * f.vx + f.vy * f.vy + f.vz * f.vz);
                } else {
                    f.px = P.x[i]; f.py = P.y[i]; f.pz = P.z[i];
                    f.vstart = sqrt(f.vx * f.vx + f.vy * f.vy + f.vz * f.vz);
                    f.rem = pp.dt;
                    f.it = 0;
                    f.cur = locate(M, f.px, f.py, f.pz, t0);
                    if (f.cur < 0) {
                        f.cur = 0;  // result.final_element stays 0 (PICParticleAlgorithms.cpp:543,577)
                        st = kLost;
                    } else {
                        st = advance_d(M, S, pp, f, kCap1, A, c.nsub);
                    }
                }
            }
            unsigned slot = warp_append(st == kCapped, D.count);
            if (st == kCapped && slot < D.cap) {
                defer_store_d(P, D, slot, i, f);
            } else if (st >= 0) {
                if (st == kCapped) st = advance_d(M, S, pp, f, 0x7fffffff, A, c.nsub);
                finish_d(M, P, S, pp, L, i, f, st, c);
            }
            warp_chunk_end(c);
        }
    }
    warp_stats_flush(L, ke_acc, S.vmax);
}

// Passes 2 and 3 over a deferred list (see k_push_mixed_more).
__global__ void __launch_bounds__(256) k_push_f64_more(const __grid_constant__ MeshView M, ParticleStore P,
    const __grid_constant__ SpeciesDev S, const __grid_constant__ PushParams pp,
                                                       DeferList Din, DeferList Dout, int cap, ChargeAcc A, LedgerDev* L,
                                                       unsigned long long* ke_acc, unsigned* ctr)
{
    const int64_t n = (int64_t)min(*Din.count, Din.cap);
    PushStats c{0.0, 0u, 0u};
    const int lane = threadIdx.x & 31;
    const bool chain = Dout.count != nullptr;
    warp_stats_begin();
    for (;;) {
        const int64_t base = (int64_t)next_chunk(ctr) * 32;
        if (base >= n) break;
        const int64_t e = base + lane;
        int st = -1;
        FlightD f;
        int64_t i = 0;
        if (e < n) {
            i = Din.idx[e];
            f.cur = P.tet[i];
            f.px = P.x[i]; f.py = P.y[i]; f.pz = P.z[i];
            f.vx = P.vx[i]; f.vy = P.vy[i]; f.vz = P.vz[i];
            f.it = Din.it[e];
            f.rem = Din.rem[e];
            f.vstart = Din.vstart[e];
            st = advance_d(M, S, pp, f, chain ? cap : 0x7fffffff, A, c.nsub);
        }
        unsigned slot = chain ? warp_append(st == kCapped, Dout.count) : 0xffffffffu;
        if (st == kCapped && chain && slot < Dout.cap) {
            defer_store_d(P, Dout, slot, i, f);
        } else if (st >= 0) {
            if (st == kCapped) st = advance_d(M, S, pp, f, 0x7fffffff, A, c.nsub);
            finish_d(M, P, S, pp, L, i, f, st, c);
        }
        warp_chunk_end(c);
    }
    warp_stats_flush(L, ke_acc, S.vmax);
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

// Per-tet copy of the nodal E of its 4 nodes.
__global__ void k_refresh_erec(int64_t T, const int4* __restrict__ tet, const double* __restrict__ E, double* erec)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        int4 tn = tet[t];
        int nd[4] = {tn.x, tn.y, tn.z, tn.w};
        double* r = erec + 12 * t;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            r[3 * q] = E[3 * (int64_t)nd[q]];
            r[3 * q + 1] = E[3 * (int64_t)nd[q] + 1];
            r[3 * q + 2] = E[3 * (int64_t)nd[q] + 2];
        }
    }
}

void launch_push_f64(const MeshView& M, const ParticleStore& P, const SpeciesDev& S, const PushParams& pp,
                     const DeferList& D1, const DeferList& D2, ChargeAcc A, LedgerDev* L, unsigned long long* ke_acc,
                     unsigned* ctr, int grid, cudaStream_t st)
{
    k_push_f64<<<grid, 256, 0, st>>>(M, P, S, pp, D1, A, L, ke_acc, ctr);
    k_push_f64_more<<<grid, 256, 0, st>>>(M, P, S, pp, D1, D2, kCap2, A, L, ke_acc, ctr + 1);
    DeferList none{};
    k_push_f64_more<<<grid, 256, 0, st>>>(M, P, S, pp, D2, none, 0, A, L, ke_acc, ctr + 2);
}

void launch_mcc_f64(const ParticleStore& P, const SpeciesDev& S, const PushParams& pp, LedgerDev* L, int grid,
                    cudaStream_t st)
{
    k_mcc_f64<<<grid, 256, 0, st>>>(P, S, pp, L);
}

void launch_refresh_erec(int64_t T, const int4* tet, const double* E, double* erec, cudaStream_t st)
{
    k_refresh_erec<<<148 * 8, 256, 0, st>>>(T, tet, E, erec);
}

}  // namespace scdat
