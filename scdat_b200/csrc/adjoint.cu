// adjoint.cu -- reverse mode of the FP64 step over a window of steps, for gradients of a
// linear functional of the final potential and surface-circuit state with respect to the
// body bias, the electron temperature and the secondary-yield peak.
//
// The derivative is the pathwise one: the forward run's discrete structure is held fixed --
// the tet of every sub-step, which expression the adaptive sub-step took (remaining time,
// 0.1 v/a, or the floor), which deposit sample points fell in the post-move tet, which
// particles were collected by which face.  Within that structure every map is smooth and
// differentiated exactly:
//   gather        E(x) = sum_i lambda_i(x) E_i          (lambda affine in x per tet)
//   sub-step      dt = rem | 0.1 |v0| / (|qm| |E|) | floor * rem, v1 = v + qm dt E,
//                 x1 = x + v1 dt, rem1 = rem - dt       (CrossTetrahedron::integrateTrajectory,
//                 PICParticleAlgorithms.cpp:536-851, as push_f64.cu runs it)
//   deposit       q w lambda(midpoint) in the tet, or q w / nseg sum_j lambda(p_j) over the
//                 sample points in the post-move tet (ChargeDepositor, :371-433)
//   field         b = sign rho CV - K_rd phi_d, K phi = b (SPD), E = -LSQ gradient of phi
//                 (PoissonSolver.cpp:274-385,474-529): the adjoint is one solve with K and the
//                 transposed LSQ map
//   surface       the implicit node update of the surface circuit and the Sternglass /
//                 Whipple yields of the collected electrons (surface.cuh)
// A finite-difference check of the same window with frozen random streams agrees with it as
// long as the perturbation flips none of those discrete choices.
//
// Particle states are checkpointed every `checkpoint` steps on the forward pass; the reverse
// pass recomputes each segment from its checkpoint (the step is deterministic), then runs the
// per-particle adjoint kernel, which replays its particle's sub-steps into a local tape and
// reverses them.
#include "ctx.cuh"
#include "field_kern.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace scdat {


enum AdjFlag : unsigned long long {
    kAdjTapeFull = 1ull << 0,  // a particle needed more sub-steps than the tape holds
    kAdjMismatch = 1ull << 1,  // the replay did not reproduce the forward end state
};

struct SubTape {
    double x0[3];  // position at the sub-step's start
    double v1[3];  // velocity after the two half kicks
    double E[3];   // gathered field
    double adt;
    int cur;       // tet of the gather
    int in;        // the gather found the point in `cur`
    int branch;    // 0: dt = rem, 1: dt = 0.1 |v0| / (|qm| |E|), 2: dt = floor * rem
    int dep;       // 0 none, 1 in-tet midpoint (tiny: start point), 2 sample points in dtet
    int tiny;
    int dtet;
    unsigned mask; // sample points of dep 2 inside dtet
};

// gradient of barycentric i of tet t (lambda_{1..3} = J^-1 (x - o), lambda_0 = 1 - sum)
__device__ __forceinline__ void bary_grad(const MeshView& M, int t, double G[4][3])
{
    const double* g = M.geom + 16 * (int64_t)t;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) G[r + 1][c] = __ldg(g + 3 * r + c);
#pragma unroll
    for (int c = 0; c < 3; ++c) G[0][c] = -(G[1][c] + G[2][c] + G[3][c]);
}

// The sub-step engine: one sub-step of CrossTetrahedron::integrateTrajectory exactly as
// advance_d runs it (same operations in the same order), recording into T when given.
struct Flight {
    double p[3], v[3];
    double rem, vstart;
    int cur, it;
    bool in;
    double lam[4];
};

enum { kGo = 0, kEnd = 1, kOut = 2 };

__device__ int substep(const MeshView& M, const SpeciesDev& S, const PushParams& pp, Flight& f, SubTape* T)
{
    if (!(f.rem > kMinTimeStep && f.it < kMaxSubsteps)) return kEnd;
    const double qm = S.qm;
    ++f.it;
    double Ex = 0.0, Ey = 0.0, Ez = 0.0;
    if (f.in) {
        const double* e = M.erec + 12 * (int64_t)f.cur;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            Ex = Ex + __ldg(e + 3 * q) * f.lam[q];
            Ey = Ey + __ldg(e + 3 * q + 1) * f.lam[q];
            Ez = Ez + __ldg(e + 3 * q + 2) * f.lam[q];
        }
    }
    double adt = f.rem;
    int branch = 0;
    double Em = sqrt(Ex * Ex + Ey * Ey + Ez * Ez);
    if (Em > 1e-10) {
        double acc = Em * fabs(qm);
        if (acc > 1e-10 && f.vstart > 1.0) {
            const double a1 = 0.1 * f.vstart / acc;
            if (a1 < adt) {
                adt = a1;
                branch = 1;
            }
        }
    }
    const double fl = f.rem * pp.floor_ratio;
    if (fl > adt) {
        adt = fl;
        branch = 2;
    }
    if (f.rem < adt) {
        adt = f.rem;
        branch = 0;
    }
    const double sx = f.p[0], sy = f.p[1], sz = f.p[2];
    if (T) {
        T->x0[0] = sx; T->x0[1] = sy; T->x0[2] = sz;
        T->E[0] = Ex; T->E[1] = Ey; T->E[2] = Ez;
        T->adt = adt;
        T->cur = f.cur;
        T->in = f.in ? 1 : 0;
        T->branch = branch;
        T->dep = 0;
        T->tiny = 0;
        T->dtet = f.cur;
        T->mask = 0u;
    }
    if (fabs(qm) > 1e-20) {
        double h = qm * (0.5 * adt);
        f.v[0] = f.v[0] + Ex * h; f.v[1] = f.v[1] + Ey * h; f.v[2] = f.v[2] + Ez * h;
        f.v[0] = f.v[0] + Ex * h; f.v[1] = f.v[1] + Ey * h; f.v[2] = f.v[2] + Ez * h;
    }
    if (T) {
        T->v1[0] = f.v[0]; T->v1[1] = f.v[1]; T->v1[2] = f.v[2];
    }
    f.p[0] = f.p[0] + f.v[0] * adt;
    f.p[1] = f.p[1] + f.v[1] * adt;
    f.p[2] = f.p[2] + f.v[2] * adt;
    const double tx = f.p[0] - sx, ty = f.p[1] - sy, tz = f.p[2] - sz;
    const bool tiny = sqrt(tx * tx + ty * ty + tz * tz) < 1e-15;
    double le[4];
    int dep = 0, dtet = f.cur;
    if (bary64(M, f.cur, f.p[0], f.p[1], f.p[2], le)) {
        if (pp.deposit) dep = f.in ? 1 : 2;
#pragma unroll
        for (int q = 0; q < 4; ++q) f.lam[q] = le[q];
        f.in = true;
    } else {
        int nt = locate(M, f.p[0], f.p[1], f.p[2], f.cur);
        if (nt < 0) return kOut;
        f.cur = nt;
        if (pp.deposit) {
            dep = 2;
            dtet = nt;
        }
        f.in = bary64(M, nt, f.p[0], f.p[1], f.p[2], f.lam);
    }
    if (T) {
        T->dep = dep;
        T->dtet = dtet;
        T->tiny = tiny ? 1 : 0;
        if (dep == 2) {
            double ls[4];
            bary64(M, dtet, sx, sy, sz, ls);
            double G[4][3];
            bary_grad(M, dtet, G);
            // the same arithmetic as deposit_traj in push_f64.cu, so the inside tests agree
            double dl[4];
#pragma unroll
            for (int q = 1; q < 4; ++q) dl[q] = G[q][0] * tx + G[q][1] * ty + G[q][2] * tz;
            dl[0] = -dl[1] - dl[2] - dl[3];
            if (tiny || pp.dep_kernel == 0) {
                double l0[4];
                const bool ok = tiny ? bary64(M, dtet, sx, sy, sz, l0) : bary64(M, dtet, f.p[0], f.p[1], f.p[2], l0);
                T->mask = ok ? 1u : 0u;
            } else {
                for (int sg = 0; sg < pp.nseg; ++sg) {
                    double tau = ((double)sg + 0.5) / (double)pp.nseg;
                    double l[4] = {ls[0] + tau * dl[0], ls[1] + tau * dl[1], ls[2] + tau * dl[2], ls[3] + tau * dl[3]};
                    if (bary_inside(l)) T->mask |= 1u << sg;
                }
            }
        }
    }
    f.rem -= adt;
    return kGo;
}

struct AdjPushArgs {
    // particle state at the step's start and end (the forward run's)
    const double *x0, *y0, *z0, *vx0, *vy0, *vz0;
    const int32_t* tet0;
    const double *x1, *y1, *z1, *vx1, *vy1, *vz1;
    const int32_t* tet1;
    int64_t n;
    // adjoints of the particle state: in = at the step's end, out = at its start
    double *lx, *ly, *lz, *lvx, *lvy, *lvz;
    const double* lrho;        // adjoint of the step's deposited nodal charge [N]
    double* lE;                // adjoint of the nodal field the step gathered [3N], accumulated
    const double* ldq;         // adjoint of each face's collected charge this step [6]
    double* emitted;           // secondary charge per face this step [6], accumulated
    unsigned long long* flags;
};

// yield and its derivative in E (eV): Sternglass exactly, d/dE 7.4 dmax r exp(-2 sqrt r) =
// 7.4 dmax exp(-2 sqrt r) (1 - sqrt r) / Emax; the Whipple form by a central difference
__device__ __forceinline__ double see_yield_dE(const PushParams& pp, double e_ev, double& dy)
{
    const double y = see_yield(pp, e_ev);
    if (pp.see_model == 1) {
        const double r = e_ev / pp.see_emax_ev, sr = sqrt(r);
        dy = 7.4 * pp.see_dmax * exp(-2.0 * sr) * (1.0 - sr) / pp.see_emax_ev;
    } else {
        const double h = 1e-6 * fmax(e_ev, 1e-3);
        dy = (see_yield(pp, e_ev + h) - see_yield(pp, e_ev - h)) / (2.0 * h);
    }
    return y;
}

constexpr int kChunk = 32;   // dense tape: sub-steps replayed at a time on the reverse pass
constexpr int kSparse = 64;  // resume points every kChunk sub-steps: up to 2048 sub-steps a step

__global__ void __launch_bounds__(128) k_adj_push_f64(MeshView M, SpeciesDev S, PushParams pp, AdjPushArgs a)
{
    const double qw = S.q * S.w, qm = S.qm;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int t0 = a.tet0[i];
        if (t0 <= kTetAbsorbed) continue;  // inactive before the step: no dependence
        Flight f;
        f.p[0] = a.x0[i]; f.p[1] = a.y0[i]; f.p[2] = a.z0[i];
        f.v[0] = a.vx0[i]; f.v[1] = a.vy0[i]; f.v[2] = a.vz0[i];
        f.vstart = sqrt(f.v[0] * f.v[0] + f.v[1] * f.v[1] + f.v[2] * f.v[2]);
        f.rem = pp.dt;
        f.it = 0;
        f.cur = locate(M, f.p[0], f.p[1], f.p[2], t0);
        bool lost = f.cur < 0;
        int ns = 0;
        Flight ck[kSparse];
        bool overflow = false;
        if (!lost) {
            f.in = bary64(M, f.cur, f.p[0], f.p[1], f.p[2], f.lam);
            // forward: count the sub-steps, keeping a resume point at every chunk start
            for (;;) {
                if (ns % kChunk == 0) {
                    if (ns / kChunk == kSparse) {
                        overflow = true;
                        break;
                    }
                    ck[ns / kChunk] = f;
                }
                const int r = substep(M, S, pp, f, nullptr);
                if (r == kEnd) break;
                ++ns;
                if (r == kOut) {
                    lost = true;
                    break;
                }
            }
        }
        if (overflow) {
            atomicOr(a.flags, (unsigned long long)kAdjTapeFull);
            a.lx[i] = a.ly[i] = a.lz[i] = a.lvx[i] = a.lvy[i] = a.lvz[i] = 0.0;
            continue;
        }
        const int t1 = a.tet1[i];
        double lx[3] = {a.lx[i], a.ly[i], a.lz[i]}, lv[3] = {a.lvx[i], a.lvy[i], a.lvz[i]};
        if (t1 >= 0) {
            // active at the end: the replay must land where the forward run did (periodic
            // wraps shift the position by a constant)
            const double dv = fabs(f.v[0] - a.vx1[i]) + fabs(f.v[1] - a.vy1[i]) + fabs(f.v[2] - a.vz1[i]);
            if (dv > 1e-9 * (fabs(a.vx1[i]) + fabs(a.vy1[i]) + fabs(a.vz1[i]) + 1.0))
                atomicOr(a.flags, (unsigned long long)kAdjMismatch);
        } else {
            // left the domain this step (or earlier): only a body collection carries on, through
            // the charge its secondaries leave on the face
            lx[0] = lx[1] = lx[2] = 0.0;
            lv[0] = lv[1] = lv[2] = 0.0;
            if (t1 == kTetEscaped && lost && pp.patches && S.electron_like && pp.see_model) {
                const double px = a.x1[i], py = a.y1[i], pz = a.z1[i];
                const bool inside = px >= M.bmin[0] - pp.otol && px <= M.bmax[0] + pp.otol && py >= M.bmin[1] - pp.otol &&
                                    py <= M.bmax[1] + pp.otol && pz >= M.bmin[2] - pp.otol && pz <= M.bmax[2] + pp.otol;
                if (inside) {
                    const double d[6] = {fabs(px - pp.blo[0]), fabs(pp.bhi[0] - px), fabs(py - pp.blo[1]),
                                         fabs(pp.bhi[1] - py), fabs(pz - pp.blo[2]), fabs(pp.bhi[2] - pz)};
                    int k = 0;
                    for (int q = 1; q < 6; ++q)
                        if (d[q] < d[k]) k = q;
                    const double vx = a.vx1[i], vy = a.vy1[i], vz = a.vz1[i];
                    const double e_ev = 0.5 * S.m * (vx * vx + vy * vy + vz * vz) / kElementaryCharge;
                    double dy;
                    const double y = see_yield_dE(pp, e_ev, dy);
                    atomicAdd(&a.emitted[k], y * fabs(S.q) * S.w);
                    // d(emitted)/dv = dy/dE * m v / e * |q| w
                    const double c = a.ldq[k] * dy * fabs(S.q) * S.w * S.m / kElementaryCharge;
                    lv[0] = c * vx;
                    lv[1] = c * vy;
                    lv[2] = c * vz;
                }
            }
        }
        double lrem = 0.0, lvs = 0.0;
        SubTape tape[kChunk];
        for (int chunk = (ns - 1) / kChunk; ns > 0 && chunk >= 0; --chunk) {
            // replay this chunk into the dense tape
            Flight g = ck[chunk];
            const int first = chunk * kChunk, cnt = min(kChunk, ns - first);
            for (int k = 0; k < cnt; ++k) substep(M, S, pp, g, &tape[k]);
            for (int s = cnt - 1; s >= 0; --s) {
                const SubTape& T = tape[s];
                const double adt = T.adt;
                // deposit of this sub-step
                double ax0[3] = {0, 0, 0};
                if (T.dep) {
                    const int dt = T.dep == 1 ? T.cur : T.dtet;
                    double G[4][3];
                    bary_grad(M, dt, G);
                    const int4 tn = rec_nodes(M, dt);
                    const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
                    double c0 = 0.0, c1 = 0.0;  // weight of grad lambda on x0 and on x1
                    if (T.dep == 1 || T.mask) {
                        if (T.tiny) {
                            c0 = qw;
                        } else if (pp.dep_kernel == 0) {
                            c1 = qw;
                        } else if (T.dep == 1) {
                            c0 = 0.5 * qw;
                            c1 = 0.5 * qw;
                        } else {
                            for (int sg = 0; sg < pp.nseg; ++sg)
                                if ((T.mask >> sg) & 1u) {
                                    const double tau = ((double)sg + 0.5) / (double)pp.nseg;
                                    c0 += S.cw_seg * (1.0 - tau);
                                    c1 += S.cw_seg * tau;
                                }
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const double r = a.lrho[nd[q]];
                        for (int c = 0; c < 3; ++c) {
                            ax0[c] += r * c0 * G[q][c];
                            lx[c] += r * c1 * G[q][c];
                        }
                    }
                }
                // x1 = x0 + v1 dt, v1 = v0 + qm dt E, rem1 = rem0 - dt
                double lv1[3], lE[3];
                for (int c = 0; c < 3; ++c) lv1[c] = lv[c] + adt * lx[c];
                double ladt = -lrem;
                for (int c = 0; c < 3; ++c) ladt += T.v1[c] * lx[c];
                if (fabs(qm) > 1e-20) {
                    for (int c = 0; c < 3; ++c) {
                        lE[c] = qm * adt * lv1[c];
                        ladt += qm * T.E[c] * lv1[c];
                    }
                } else {
                    lE[0] = lE[1] = lE[2] = 0.0;
                }
                double lrem0 = lrem;
                if (T.branch == 0) {
                    lrem0 += ladt;
                } else if (T.branch == 2) {
                    lrem0 += ladt * pp.floor_ratio;
                } else {
                    // dt = 0.1 |v0| / (|qm| |E|)
                    const double E2 = T.E[0] * T.E[0] + T.E[1] * T.E[1] + T.E[2] * T.E[2];
                    lvs += ladt * adt / f.vstart;
                    for (int c = 0; c < 3; ++c) lE[c] -= ladt * adt * T.E[c] / E2;
                }
                // gather
                double lx0[3] = {lx[0], lx[1], lx[2]};
                if (T.in) {
                    double G[4][3], lam[4];
                    bary_grad(M, T.cur, G);
                    bary64(M, T.cur, T.x0[0], T.x0[1], T.x0[2], lam);
                    const int4 tn = rec_nodes(M, T.cur);
                    const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
                    const double* e = M.erec + 12 * (int64_t)T.cur;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        atomicAdd(a.lE + 3 * nd[q], lam[q] * lE[0]);
                        atomicAdd(a.lE + 3 * nd[q] + 1, lam[q] * lE[1]);
                        atomicAdd(a.lE + 3 * nd[q] + 2, lam[q] * lE[2]);
                        const double w =
                            lE[0] * __ldg(e + 3 * q) + lE[1] * __ldg(e + 3 * q + 1) + lE[2] * __ldg(e + 3 * q + 2);
                        for (int c = 0; c < 3; ++c) lx0[c] += w * G[q][c];
                    }
                }
                for (int c = 0; c < 3; ++c) {
                    lx[c] = lx0[c] + ax0[c];
                    lv[c] = lv1[c];
                }
                lrem = lrem0;
            }
        }
        // |v0| of the step start feeds every sub-step of branch 1
        if (f.vstart > 0.0) {
            lv[0] += lvs * a.vx0[i] / f.vstart;
            lv[1] += lvs * a.vy0[i] / f.vstart;
            lv[2] += lvs * a.vz0[i] / f.vstart;
        }
        a.lx[i] = lx[0]; a.ly[i] = lx[1]; a.lz[i] = lx[2];
        a.lvx[i] = lv[0]; a.lvy[i] = lv[1]; a.lvz[i] = lv[2];
    }
}

// E_i = -M_i^-1 sum_j d_ij (phi_j - phi_i): with y = -M_i^-1 lE_i,
// lphi_j += d_ij . y and lphi_i -= sum_j d_ij . y (the forward's own neighbour set and pivoting)
__global__ void k_adj_lsq(int64_t N, const double* __restrict__ xyz, const int32_t* __restrict__ gptr,
                          const int32_t* __restrict__ gcol, double reg, const double* __restrict__ lE, double* lphi,
                          const unsigned long long* lsq_bad)
{
    if ((*lsq_bad) & (1ull << 8)) return;  // the forward zeroed the whole field
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double l0 = lE[3 * i], l1 = lE[3 * i + 1], l2 = lE[3 * i + 2];
        if (l0 == 0.0 && l1 == 0.0 && l2 == 0.0) continue;
        double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
        int cnt = 0;
        for (int e = gptr[i]; e < gptr[i + 1]; ++e) {
            const int j = gcol[e];
            const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
            if (dx * dx + dy * dy + dz * dz <= 1e-24) continue;
            M[0][0] += dx * dx; M[0][1] += dx * dy; M[0][2] += dx * dz;
            M[1][0] += dy * dx; M[1][1] += dy * dy; M[1][2] += dy * dz;
            M[2][0] += dz * dx; M[2][1] += dz * dy; M[2][2] += dz * dz;
            ++cnt;
        }
        if (!cnt) continue;
        M[0][0] += reg; M[1][1] += reg; M[2][2] += reg;
        double rhs[3] = {-l0, -l1, -l2}, y[3] = {0, 0, 0};
        if (!solve3(M, rhs, y)) continue;
        double self = 0.0;
        for (int e = gptr[i]; e < gptr[i + 1]; ++e) {
            const int j = gcol[e];
            const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
            if (dx * dx + dy * dy + dz * dz <= 1e-24) continue;
            const double c = dx * y[0] + dy * y[1] + dz * y[2];
            atomicAdd(lphi + j, c);
            self -= c;
        }
        atomicAdd(lphi + i, self);
    }
}

// interior rows: rhs of the adjoint solve; Dirichlet nodes keep their adjoint
__global__ void k_adj_rows(PoissonView A, const double* __restrict__ lphi, double* __restrict__ brow)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.R; r += gridDim.x * blockDim.x)
        brow[r] = lphi[A.row_node[r]];
}

// lrho_n = sign CV_r mu_r on interior nodes; lphi_d -= K_rd mu_r on the Dirichlet couplings
__global__ void k_adj_split(PoissonView A, const double* __restrict__ mu, double sign, double* __restrict__ lrho,
                            double* lphid)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.R; r += gridDim.x * blockDim.x) {
        lrho[A.row_node[r]] = sign * A.cv[r] * mu[r];
        for (int e = A.lift_ptr[r]; e < A.lift_ptr[r + 1]; ++e) atomicAdd(lphid + A.lift_node[e], -A.lift_val[e] * mu[r]);
    }
}

}  // namespace scdat

// ======================================================================================
// Window driver
// ======================================================================================
namespace {

struct Snap {  // the state a segment is recomputed from
    std::vector<std::unique_ptr<DBuf<double>>> d;
    std::vector<std::unique_ptr<DBuf<int32_t>>> t;
    DBuf<double> phi;
    DBuf<SurfaceDev> surf;
    DBuf<LedgerDev> led;
    int64_t steps = 0;
    double sim_time = 0.0;
};

int snap_save(scdat_ctx* ctx, Snap& s)
{
    s.d.clear();
    s.t.clear();
    for (auto& S : ctx->species) {
        for (DBuf<double>* a : {&S.x, &S.y, &S.z, &S.vx, &S.vy, &S.vz}) {
            s.d.push_back(std::make_unique<DBuf<double>>());
            if (s.d.back()->alloc(std::max<size_t>(a->n, 1)) != cudaSuccess) return SCDAT_ERR_CUDA;
            if (a->n) cudaMemcpyAsync(s.d.back()->p, a->p, sizeof(double) * a->n, cudaMemcpyDeviceToDevice, ctx->st);
        }
        s.t.push_back(std::make_unique<DBuf<int32_t>>());
        if (s.t.back()->alloc(std::max<size_t>(S.tet.n, 1)) != cudaSuccess) return SCDAT_ERR_CUDA;
        if (S.tet.n) cudaMemcpyAsync(s.t.back()->p, S.tet.p, sizeof(int32_t) * S.tet.n, cudaMemcpyDeviceToDevice, ctx->st);
    }
    if (s.phi.alloc(ctx->hm.N) != cudaSuccess || s.led.alloc(1) != cudaSuccess) return SCDAT_ERR_CUDA;
    cudaMemcpyAsync(s.phi.p, ctx->phi.p, sizeof(double) * ctx->hm.N, cudaMemcpyDeviceToDevice, ctx->st);
    cudaMemcpyAsync(s.led.p, ctx->led.p, sizeof(LedgerDev), cudaMemcpyDeviceToDevice, ctx->st);
    if (ctx->surface) {
        if (s.surf.alloc(1) != cudaSuccess) return SCDAT_ERR_CUDA;
        cudaMemcpyAsync(s.surf.p, ctx->surf.p, sizeof(SurfaceDev), cudaMemcpyDeviceToDevice, ctx->st);
    }
    s.steps = ctx->steps;
    s.sim_time = ctx->sim_time;
    return cudaGetLastError() == cudaSuccess ? SCDAT_OK : SCDAT_ERR_CUDA;
}

int snap_load(scdat_ctx* ctx, const Snap& s)
{
    size_t k = 0;
    for (size_t sp = 0; sp < ctx->species.size(); ++sp) {
        auto& S = ctx->species[sp];
        for (DBuf<double>* a : {&S.x, &S.y, &S.z, &S.vx, &S.vy, &S.vz}) {
            if (a->n) cudaMemcpyAsync(a->p, s.d[k]->p, sizeof(double) * a->n, cudaMemcpyDeviceToDevice, ctx->st);
            ++k;
        }
        if (S.tet.n) cudaMemcpyAsync(S.tet.p, s.t[sp]->p, sizeof(int32_t) * S.tet.n, cudaMemcpyDeviceToDevice, ctx->st);
    }
    cudaMemcpyAsync(ctx->phi.p, s.phi.p, sizeof(double) * ctx->hm.N, cudaMemcpyDeviceToDevice, ctx->st);
    cudaMemcpyAsync(ctx->led.p, s.led.p, sizeof(LedgerDev), cudaMemcpyDeviceToDevice, ctx->st);
    if (ctx->surface) cudaMemcpyAsync(ctx->surf.p, s.surf.p, sizeof(SurfaceDev), cudaMemcpyDeviceToDevice, ctx->st);
    ctx->steps = s.steps;
    ctx->sim_time = s.sim_time;
    return cudaGetLastError() == cudaSuccess ? SCDAT_OK : SCDAT_ERR_CUDA;
}

// one forward step exactly as scdat_step runs it (the window keeps the particle order: no sort)
int fwd_step(scdat_ctx* ctx)
{
    int rc = do_push(ctx, true);
    if (!rc) rc = do_surface(ctx);
    if (!rc) rc = do_solve_field(ctx);
    if (rc) return rc;
    ctx->steps += 1;
    ctx->sim_time += ctx->prm.dt;
    return SCDAT_OK;
}

}  // namespace

#define ACK(call)                                                          \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) {                                           \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return SCDAT_ERR_CUDA;                                         \
        }                                                                  \
    } while (0)

extern "C" {

SCDAT_API int scdat_adjoint_window(scdat_ctx* ctx, const scdat_adjoint_request* rq, scdat_adjoint_result* res)
{
    if (!ctx || !rq || !res) return SCDAT_ERR_ARG;
    std::memset(res, 0, sizeof(*res));
    auto fail = [&](const char* m) {
        ctx->err = m;
        return SCDAT_ERR_ARG;
    };
    if (ctx->mixed) return fail("the adjoint window runs the FP64 form");
    if (ctx->species.empty()) return fail("species not set");
    if (rq->steps <= 0) return fail("the window needs at least one step");
    if (ctx->prm.deposit_kernel == SCDAT_DEP_GAUSS3) return fail("the adjoint covers the segment-cloud and nearest-point deposits");
    for (auto& S : ctx->species)
        if (S.mcc.enabled) return fail("switch the MCC off inside an adjoint window");
    const int steps = rq->steps, C = rq->checkpoint > 0 ? rq->checkpoint : 10;
    const int64_t N = ctx->hm.N;
    const int nsp = (int)ctx->species.size();
    const PoissonView& A = ctx->pv;
    const int sort_saved = ctx->prm.sort_interval;
    ctx->prm.sort_interval = 0;
    cudaStream_t st = ctx->st;

    // ---- forward with checkpoints
    const int nck = (steps + C - 1) / C;
    std::vector<Snap> ck((size_t)nck);
    int rc = SCDAT_OK;
    for (int t = 0; t < steps && !rc; ++t) {
        if (t % C == 0) rc = snap_save(ctx, ck[t / C]);
        if (!rc) rc = fwd_step(ctx);
    }
    Snap fin;
    if (!rc) rc = snap_save(ctx, fin);
    if (rc) {
        ctx->prm.sort_interval = sort_saved;
        return rc;
    }
    // objective J = g_phi . phi_T + g_V . V_T + g_Q . Q_T
    std::vector<double> phiT((size_t)N), gphi((size_t)N, 0.0);
    ACK(cudaMemcpyAsync(phiT.data(), ctx->phi.p, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
    SurfaceDev sh{};
    if (ctx->surface) ACK(cudaMemcpyAsync(&sh, ctx->surf.p, sizeof(sh), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    if (rq->g_phi) std::memcpy(gphi.data(), rq->g_phi, sizeof(double) * N);
    double J = 0.0;
    for (int64_t n = 0; n < N; ++n) J += gphi[n] * phiT[n];
    for (int f = 0; f < 6 && ctx->surface; ++f) J += rq->g_V[f] * sh.V[f] + rq->g_Q[f] * sh.Q[f];
    res->J = J;

    // ---- adjoint buffers
    DBuf<double> lphi, lphid, lrho, lE, brow, mu, emit, ldq;
    DBuf<unsigned long long> aflags;
    ACK(lphi.alloc(N));
    ACK(lphid.alloc(N));
    ACK(lrho.alloc(N));
    ACK(lE.alloc(3 * N));
    ACK(brow.alloc(std::max(A.R, 1)));
    ACK(mu.alloc(std::max(A.R, 1)));
    ACK(emit.alloc(6));
    ACK(ldq.alloc(6));
    ACK(aflags.alloc(1));
    ACK(cudaMemsetAsync(aflags.p, 0, sizeof(unsigned long long), st));
    ACK(cudaMemsetAsync(lE.p, 0, sizeof(double) * 3 * N, st));
    std::vector<std::unique_ptr<DBuf<double>>> lpart;  // 6 arrays per species
    for (auto& S : ctx->species)
        for (int c = 0; c < 6; ++c) {
            lpart.push_back(std::make_unique<DBuf<double>>());
            ACK(lpart.back()->alloc(std::max<size_t>(S.x.n, 1)));
            ACK(cudaMemsetAsync(lpart.back()->p, 0, sizeof(double) * std::max<size_t>(S.x.n, 1), st));
        }
    // body (bias) nodes and the surface nodes' face masks
    std::vector<int64_t> bias_nodes(rq->bias_nodes, rq->bias_nodes + std::max<int64_t>(rq->n_bias_nodes, 0));
    std::vector<int32_t> snode;
    std::vector<uint8_t> smask;
    if (ctx->surface) {
        snode.resize(ctx->surf_node.n);
        smask.resize(ctx->surf_mask.n);
        ACK(cudaMemcpy(snode.data(), ctx->surf_node.p, sizeof(int32_t) * snode.size(), cudaMemcpyDeviceToHost));
        ACK(cudaMemcpy(smask.data(), ctx->surf_mask.p, sizeof(uint8_t) * smask.size(), cudaMemcpyDeviceToHost));
    }
    double lV[6] = {0, 0, 0, 0, 0, 0}, lbias = 0.0, ldelta = 0.0;
    for (int f = 0; f < 6; ++f) lV[f] = ctx->surface ? rq->g_V[f] : 0.0;
    const int grid = ctx->grid_nodes, gr = ctx->grid_red;
    const double sign = (double)ctx->prm.poisson_charge_sign;

    // field adjoint of one solve: lphi (all nodes, host-seeded with `seed`) + LSQ^T lE ->
    // lrho (interior) and the Dirichlet adjoint, folded into the bias and the face potentials
    auto field_adjoint = [&](const std::vector<double>* seed) -> int {
        if (seed) ACK(cudaMemcpyAsync(lphi.p, seed->data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
        else ACK(cudaMemsetAsync(lphi.p, 0, sizeof(double) * N, st));
        k_adj_lsq<<<grid, 256, 0, st>>>(N, ctx->xyz.p, ctx->gptr.p, ctx->gcol.p, 0.0, lE.p, lphi.p, &ctx->led.p->lsq_bad);
        ACK(cudaGetLastError());
        ACK(cudaMemsetAsync(lrho.p, 0, sizeof(double) * N, st));
        ACK(cudaMemcpyAsync(lphid.p, lphi.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        if (A.R > 0) {
            k_adj_rows<<<gr, 256, 0, st>>>(A, lphi.p, brow.p);
            ACK(cudaMemsetAsync(mu.p, 0, sizeof(double) * A.R, st));
            int it = 0;
            double rel = 0.0;
            int r = run_pcg64(ctx, brow.p, mu.p, 1e-14, std::max(20000, 4 * A.R), it, rel);
            if (r) return r;
            k_adj_split<<<gr, 256, 0, st>>>(A, mu.p, sign, lrho.p, lphid.p);
            ACK(cudaGetLastError());
        }
        std::vector<double> h((size_t)N);
        ACK(cudaMemcpyAsync(h.data(), lphid.p, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
        ACK(cudaStreamSynchronize(st));
        if (ctx->surface) {
            for (size_t k = 0; k < snode.size(); ++k) {
                int c = 0;
                for (int f = 0; f < 6; ++f) c += (smask[k] >> f) & 1;
                for (int f = 0; f < 6; ++f)
                    if ((smask[k] >> f) & 1) lV[f] += h[snode[k]] / c;
            }
        } else {
            for (int64_t n : bias_nodes) lbias += h[(size_t)n];
        }
        ACK(cudaMemsetAsync(lE.p, 0, sizeof(double) * 3 * N, st));
        return SCDAT_OK;
    };

    // ---- reverse, one segment at a time
    const double dt = ctx->prm.dt;
    rc = field_adjoint(&gphi);  // the solve that produced phi_T
    for (int seg = nck - 1; seg >= 0 && !rc; --seg) {
        const int t_begin = seg * C, t_end = std::min(steps, t_begin + C);
        // recompute the segment, keeping each step's starting state
        std::vector<Snap> s((size_t)(t_end - t_begin + 1));
        rc = snap_load(ctx, ck[seg]);
        if (!rc) rc = do_lsq(ctx, 0.0);  // the field of the restored potential (a solve's)
        for (int t = t_begin; t < t_end && !rc; ++t) {
            rc = snap_save(ctx, s[t - t_begin]);
            if (!rc) rc = fwd_step(ctx);
        }
        if (!rc) rc = snap_save(ctx, s[t_end - t_begin]);
        for (int t = t_end - 1; t >= t_begin && !rc; --t) {
            const Snap& a0 = s[t - t_begin];
            const Snap& a1 = s[t - t_begin + 1];
            // surface circuit of step t: V_{t+1} = ((C/dt - dI/dV) V_t + dq/dt) / (C/dt + G - dI/dV)
            double ldq_h[6] = {0, 0, 0, 0, 0, 0};
            if (ctx->surface) {
                for (int f = 0; f < 6; ++f) {
                    const double cdt = sh.C[f] / dt, den = cdt + sh.G[f] - sh.didv[f];
                    ldq_h[f] = (den > 0.0 ? lV[f] / (den * dt) : 0.0) + rq->g_Q[f];
                    if (den > 0.0) lV[f] *= (cdt - sh.didv[f]) / den;
                }
            }
            ACK(cudaMemcpyAsync(ldq.p, ldq_h, sizeof(ldq_h), cudaMemcpyHostToDevice, st));
            ACK(cudaMemsetAsync(emit.p, 0, 6 * sizeof(double), st));
            // the field the step gathered: phi_t -> E_t -> tet records
            ACK(cudaMemcpyAsync(ctx->phi.p, a0.phi.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
            rc = do_lsq(ctx, 0.0);
            if (rc) break;
            PushParams pp = push_params(ctx, false);
            pp.step = (uint32_t)(a0.steps);
            for (int sp = 0; sp < nsp && !rc; ++sp) {
                auto& S = ctx->species[sp];
                if (S.x.n == 0) continue;
                AdjPushArgs aa{};
                aa.x0 = a0.d[6 * sp]->p; aa.y0 = a0.d[6 * sp + 1]->p; aa.z0 = a0.d[6 * sp + 2]->p;
                aa.vx0 = a0.d[6 * sp + 3]->p; aa.vy0 = a0.d[6 * sp + 4]->p; aa.vz0 = a0.d[6 * sp + 5]->p;
                aa.tet0 = a0.t[sp]->p;
                aa.x1 = a1.d[6 * sp]->p; aa.y1 = a1.d[6 * sp + 1]->p; aa.z1 = a1.d[6 * sp + 2]->p;
                aa.vx1 = a1.d[6 * sp + 3]->p; aa.vy1 = a1.d[6 * sp + 4]->p; aa.vz1 = a1.d[6 * sp + 5]->p;
                aa.tet1 = a1.t[sp]->p;
                aa.n = S.n;
                aa.lx = lpart[6 * sp]->p; aa.ly = lpart[6 * sp + 1]->p; aa.lz = lpart[6 * sp + 2]->p;
                aa.lvx = lpart[6 * sp + 3]->p; aa.lvy = lpart[6 * sp + 4]->p; aa.lvz = lpart[6 * sp + 5]->p;
                aa.lrho = lrho.p;
                aa.lE = lE.p;
                aa.ldq = ldq.p;
                aa.emitted = emit.p;
                aa.flags = aflags.p;
                k_adj_push_f64<<<ctx->grid_push, 128, 0, st>>>(ctx->mv, species_dev(ctx, sp), pp, aa);
                ACK(cudaGetLastError());
            }
            if (rc) break;
            if (ctx->surface && ctx->see_model && ctx->see_dmax > 0.0) {
                double em[6];
                ACK(cudaMemcpyAsync(em, emit.p, sizeof(em), cudaMemcpyDeviceToHost, st));
                ACK(cudaStreamSynchronize(st));
                for (int f = 0; f < 6; ++f) ldelta += ldq_h[f] * em[f] / ctx->see_dmax;
            }
            // the solve that produced phi_t (the window's initial solve when t == 0)
            rc = field_adjoint(nullptr);
        }
    }
    // electron temperature: v_e(0) scales with sqrt(Te) (seeded Maxwellian, frozen draws)
    double lte = 0.0;
    if (!rc && rq->te_ev > 0.0) {
        for (int sp = 0; sp < nsp && !rc; ++sp) {
            if (!ctx->species[sp].sp.electron_like) continue;
            const size_t n = (size_t)ctx->species[sp].n;
            if (!n) continue;
            std::vector<double> v(3 * n), l(3 * n);
            for (int c = 0; c < 3; ++c) {
                ACK(cudaMemcpy(v.data() + c * n, ck[0].d[6 * sp + 3 + c]->p, sizeof(double) * n, cudaMemcpyDeviceToHost));
                ACK(cudaMemcpy(l.data() + c * n, lpart[6 * sp + 3 + c]->p, sizeof(double) * n, cudaMemcpyDeviceToHost));
            }
            for (size_t k = 0; k < 3 * n; ++k) lte += l[k] * v[k];
        }
        lte /= 2.0 * rq->te_ev;
    }
    unsigned long long fl = 0;
    if (!rc) {
        ACK(cudaMemcpy(&fl, aflags.p, sizeof(fl), cudaMemcpyDeviceToHost));
        rc = snap_load(ctx, fin);
        if (!rc) rc = do_lsq(ctx, 0.0);
        ACK(cudaStreamSynchronize(st));
    }
    ctx->prm.sort_interval = sort_saved;
    if (rc) return rc;
    if (ctx->surface)
        for (int f = 0; f < 6; ++f) lbias += lV[f];  // the faces start at the bias
    res->dJ_dbias = lbias;
    res->dJ_dte = lte;
    res->dJ_ddelta_max = ldelta;
    res->flags = (int64_t)fl;
    if (fl) {
        ctx->err = (fl & kAdjTapeFull) ? "a particle needed more than 2048 sub-steps in one step"
                                       : "the adjoint replay did not reproduce the forward run";
        return SCDAT_ERR_DEVICE_FLAG;
    }
    return SCDAT_OK;
}

}  // extern "C"
