// push.cuh -- device functions of the particle path: barycentric containment, locate,
// boundary events, MCC.  Shared by the FP64 and the mixed-precision push kernels.
#pragma once

#include "common.cuh"

namespace scdat {

struct ParticleStore {
    // FP64 form: absolute positions.  Mixed form: one 32-byte record per particle, two float4:
    // (x, y, z, vx) with the position as a float offset from the origin node of the particle's
    // tet, then (vy, vz, unused, unused) -- one sector per particle for the push's loads and
    // stores and for the re-sort's gather.
    double *x, *y, *z, *vx, *vy, *vz;
    float4* mix;
    int32_t* tet;
    uint32_t* id;
    const int64_t* count;  // device-resident particle count of this species
};

// A re-sort whose gather the mixed form's pass 1 does itself: particle i of the sorted order is
// record perm[i] of the old arrays (mix, id) and its tet is the sorted key (a key of nohint_key
// or above: no hint); pass 1 writes it to position i of its ParticleStore.  perm == nullptr:
// nothing pending, pass 1 reads the store in place.
struct SortedSource {
    const uint32_t* perm;
    const uint32_t* keys;
    uint32_t nohint_key;
    const float4* mix;
    const uint32_t* id;
};

__device__ __forceinline__ void mix_load(const ParticleStore& P, int64_t i, float& x, float& y, float& z, float& vx,
                                         float& vy, float& vz)
{
    const float4 a = P.mix[2 * i], b = P.mix[2 * i + 1];
    x = a.x; y = a.y; z = a.z; vx = a.w;
    vy = b.x; vz = b.y;
}

__device__ __forceinline__ void mix_store(const ParticleStore& P, int64_t i, float x, float y, float z, float vx,
                                          float vy, float vz)
{
    P.mix[2 * i] = make_float4(x, y, z, vx);
    P.mix[2 * i + 1] = make_float4(vy, vz, 0.0f, 0.0f);
}

__device__ __forceinline__ bool bary_inside(const double lam[4])
{
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) ok = ok && (lam[i] >= -kBaryEps) && (lam[i] <= 1.0 + kBaryEps);
    return ok;  // false for NaN (degenerate tets store NaN geometry)
}

// Barycentric coordinates of p in tet t from the precomputed inverse Jacobian
// (equivalent, up to rounding, to the signed-volume ratios of
// FieldInterpolator::isPointInTetrahedron, PICParticleAlgorithms.cpp:247-296).
__device__ __forceinline__ bool bary64(const MeshView& M, int t, double px, double py, double pz, double lam[4])
{
    const double2* g2 = reinterpret_cast<const double2*>(M.geom + 16 * (int64_t)t);
    double2 a = __ldg(g2 + 0), b = __ldg(g2 + 1), c = __ldg(g2 + 2), d = __ldg(g2 + 3), e = __ldg(g2 + 4),
            f = __ldg(g2 + 5);
    double dx = px - e.y, dy = py - f.x, dz = pz - f.y;
    lam[1] = a.x * dx + a.y * dy + b.x * dz;
    lam[2] = b.y * dx + c.x * dy + c.y * dz;
    lam[3] = d.x * dx + d.y * dy + e.x * dz;
    lam[0] = 1.0 - lam[1] - lam[2] - lam[3];
    return bary_inside(lam);
}

// Lowest-id tet containing p among the grid candidates (exactly the result of the
// reference's linear scan, PICParticleAlgorithms.cpp:882-888), or -1.
static __device__ __noinline__ int grid_lookup(const MeshView& M, double px, double py, double pz)
{
    double p[3] = {px, py, pz};
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double l = (p[a] - M.gdelta - M.gmin[a]) * M.ginv[a];
        double h = (p[a] + M.gdelta - M.gmin[a]) * M.ginv[a];
        if (!(h >= 0.0) || !(l < (double)M.gdim[a])) return -1;  // outside the grid (or NaN)
        lo[a] = l < 0.0 ? 0 : (int)l;
        hi[a] = h >= (double)M.gdim[a] ? M.gdim[a] - 1 : (int)h;
    }
    int best = 0x7fffffff;
    double lam[4];
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                int b = i + M.gdim[0] * (j + M.gdim[1] * k);
                int s = __ldg(M.bin_start + b), e = __ldg(M.bin_start + b + 1);
                for (int q = s; q < e; ++q) {
                    int t = __ldg(M.bin_tets + q);
                    if (t >= best) break;
                    if (bary64(M, t, px, py, pz, lam)) {
                        best = t;
                        break;
                    }
                }
            }
    return best == 0x7fffffff ? -1 : best;
}

__device__ __forceinline__ int4 rec_nbr(const MeshView& M, int t)
{
    return __ldg(reinterpret_cast<const int4*>(M.geom + 16 * (int64_t)t + 12));
}

__device__ __forceinline__ int4 rec_nodes(const MeshView& M, int t)
{
    return __ldg(reinterpret_cast<const int4*>(M.geom + 16 * (int64_t)t + 14));
}

// Straight walk from `start` across the most violated face (lam holds start's barycentrics).
// Returns the tet reached that contains p, or -1 at a boundary face, a degenerate tet or the
// step cap.  *unique is set when every barycentric clears 1e-6: no other tet can then hold
// the point within the 1e-8 containment tolerance, so the reference's search order
// (hint, neighbour list, lowest id) cannot pick a different tet.
__device__ __forceinline__ int walk64(const MeshView& M, double px, double py, double pz, int start, double lam[4],
                                      bool* unique)
{
    int t = start;
    for (int k = 0; k < kWalkSteps; ++k) {
        double mn = fmin(fmin(lam[0], lam[1]), fmin(lam[2], lam[3]));
        if (!(mn == mn)) return -1;  // NaN: degenerate tet
        if (bary_inside(lam)) {
            *unique = mn >= 1e-6;
            return t;
        }
        int f = 0;
        double lm = lam[0];
        if (lam[1] < lm) { lm = lam[1]; f = 1; }
        if (lam[2] < lm) { lm = lam[2]; f = 2; }
        if (lam[3] < lm) f = 3;
        int4 nb = rec_nbr(M, t);
        int nt = f == 0 ? nb.x : (f == 1 ? nb.y : (f == 2 ? nb.z : nb.w));
        if (nt < 0) return -1;
        t = nt;
        bary64(M, t, px, py, pz, lam);
    }
    return -1;
}

// Without a usable hint: walk from `start` when given, else (or when the walk cannot decide)
// the exact grid lookup of the lowest containing id.
static __device__ __noinline__ int locate_far(const MeshView& M, double px, double py, double pz, int start)
{
    if (start >= 0) {
        double lam[4];
        bary64(M, start, px, py, pz, lam);
        bool uniq = false;
        int t = walk64(M, px, py, pz, start, lam, &uniq);
        if (t >= 0 && uniq) return t;
    }
    return grid_lookup(M, px, py, pz);
}

// CrossTetrahedron::locateParticle (PICParticleAlgorithms.cpp:853-891): the hint if it holds
// the point; otherwise the unique holder found by the walk; only for points within the
// tolerance band of several tets, the reference order itself (neighbour list, then the
// lowest id over all tets, which the grid lookup reproduces).
static __device__ __noinline__ int locate_slow(const MeshView& M, double px, double py, double pz, int hint,
                                               double lam[4])
{
    bool uniq = false;
    int t = walk64(M, px, py, pz, hint, lam, &uniq);
    if (t >= 0 && uniq) return t;
    if (M.use_nbr) {
        int4 nb = rec_nbr(M, hint);
        double l2[4];
        if (nb.x >= 0 && bary64(M, nb.x, px, py, pz, l2)) return nb.x;
        if (nb.y >= 0 && bary64(M, nb.y, px, py, pz, l2)) return nb.y;
        if (nb.z >= 0 && bary64(M, nb.z, px, py, pz, l2)) return nb.z;
        if (nb.w >= 0 && bary64(M, nb.w, px, py, pz, l2)) return nb.w;
    }
    return grid_lookup(M, px, py, pz);
}

__device__ __forceinline__ int locate(const MeshView& M, double px, double py, double pz, int hint)
{
    double lam[4];
    if (hint >= 0) {
        if (bary64(M, hint, px, py, pz, lam)) return hint;
        return locate_slow(M, px, py, pz, hint, lam);
    }
    return grid_lookup(M, px, py, pz);
}

// PICCycle::detectBoundaryFace, PICCycle.cpp:1074-1133.
__device__ inline int detect_face(const MeshView& M, double px, double py, double pz, double otol, bool near,
                                  double ntol)
{
    if (px < M.bmin[0] - otol) return 0;
    if (px > M.bmax[0] + otol) return 1;
    if (py < M.bmin[1] - otol) return 2;
    if (py > M.bmax[1] + otol) return 3;
    if (pz < M.bmin[2] - otol) return 4;
    if (pz > M.bmax[2] + otol) return 5;
    if (!near) return -1;
    double d[6] = {fabs(px - M.bmin[0]), fabs(px - M.bmax[0]), fabs(py - M.bmin[1]),
                   fabs(py - M.bmax[1]), fabs(pz - M.bmin[2]), fabs(pz - M.bmax[2])};
    int best = -1;
    double bd = 1.79769313486231570815e+308;
#pragma unroll
    for (int f = 0; f < 6; ++f)
        if (d[f] <= ntol && d[f] < bd) {
            best = f;
            bd = d[f];
        }
    return best;
}

__device__ inline void ledger_tally(LedgerDev* L, int row, const SpeciesDev& S, const PushParams& pp, double ke,
                                    bool surface)
{
    double qw = S.q * S.w;
    double en = ke * fmax(1.0, S.w);
    Fx128 fq = fx_from_double(qw * pp.inv_uq);
    Fx128 fe = fx_from_double(en * pp.inv_ue);
    fx_atomic_add(&L->row[row][4], &L->row[row][5], fe);
    if (S.electron_like) {
        fx_atomic_add(&L->row[row][0], &L->row[row][1], fq);
        atomicAdd(&L->row[row][6], 1ull);
    } else if (S.q > 0.0) {
        fx_atomic_add(&L->row[row][2], &L->row[row][3], fq);
        atomicAdd(&L->row[row][7], 1ull);
    }
    if (surface) fx_atomic_add(&L->surf_lo, &L->surf_hi, fq);
}

constexpr double kElementaryCharge = 1.602176634e-19;

// Secondary-electron yield at incident energy e_ev.  Sternglass's universal curve
// delta = 7.4 dmax (E/Emax) exp(-2 sqrt(E/Emax)) (peak dmax at Emax); or the reference's
// Whipple form, legacyWhippleYield (Tools/Material/src/SurfaceMaterialModel.cpp:231-244).
__device__ inline double see_yield(const PushParams& pp, double e_ev)
{
    if (!(e_ev > 0.0) || !(pp.see_dmax > 0.0)) return 0.0;
    if (pp.see_model == 1) {
        const double r = e_ev / pp.see_emax_ev;
        return 7.4 * pp.see_dmax * r * exp(-2.0 * sqrt(r));
    }
    if (pp.see_model == 3) {  // legacySimsYield (SurfaceMaterialModel.cpp:246-273)
        if (e_ev <= 10.0) return 0.0;
        const double ep = fmax(1.0, pp.see_emax_ev), n = pp.see_sims_n, xm = pp.see_sims_xm;
        const double x = xm * pow(e_ev / ep, n);
        if (x <= 1.0e-12 || fabs(1.0 - exp(-xm)) < 1.0e-12) return 0.0;
        return pp.see_dmax / (1.0 - exp(-xm)) * pow(ep / e_ev, n - 1.0) * 2.0 * (x + exp(-x) - 1.0) / x;
    }
    if (pp.see_model == 4) {  // legacyKatzYield (SurfaceMaterialModel.cpp:275-302)
        if (e_ev <= 1.0e-9) return 0.0;
        const double ep = fmax(1.0, pp.see_emax_ev);
        const double ek = e_ev * 1.0e-3, pk = ep * 1.0e-3;
        const double* k = pp.see_katz;
        const double range = k[0] * pow(ek, k[1]) + k[2] * pow(ek, k[3]);
        const double peak_range = k[0] * pow(pk, k[1]) + k[2] * pow(pk, k[3]);
        if (range <= 1.0e-12 || peak_range <= 1.0e-12) return 0.0;
        const double att = exp(-pow(range / peak_range - 1.0, 2.0));
        const double roll = 1.0 / (1.0 + pow(e_ev / fmax(1.0, 3.0 * ep), 0.7));
        return pp.see_dmax * att * (0.55 + 0.45 * roll);
    }
    const double ep = fmax(1.0, pp.see_emax_ev);
    const double q = 2.28 * pow(e_ev / ep, 1.35);
    if (q <= 1.0e-12) return 0.0;
    return 2.228 * (q - 1.0 + exp(-q)) / q * pp.see_dmax * pow(ep / e_ev, 0.35);
}

// PICCycle::applyRuntimeBoundaryCondition + processRuntimeBoundaryEvents for one lost
// particle (PICCycle.cpp:1221-1379).  Updates position (periodic wrap) and returns the new
// tet code (>= 0 active, kTetAbsorbed, kTetEscaped).
static __device__ __noinline__ int resolve_lost(const MeshView& M, const SpeciesDev& S, const PushParams& pp, LedgerDev* L, double& px,
                            double& py, double& pz, double ke, int hint)
{
    int resolved = -1;
    int status = 0;  // 0 active, 1 absorbed, 2 escaped
    bool ok = false, done = false;
    for (int pass = 0; pass < 6 && !done; ++pass) {
        int f = detect_face(M, px, py, pz, pp.otol, pass == 0, pp.ntol);
        if (f < 0) {
            resolved = locate(M, px, py, pz, hint);
            ok = resolved >= 0;
            done = true;
            break;
        }
        int bc = pp.face_bc[f];
        if (bc == 0) {
            ok = false;
            done = true;
            break;
        }
        if (bc == 1) {
            status = 1;
            ledger_tally(L, f, S, pp, ke, true);
            ok = true;
            done = true;
            break;
        }
        // periodic: PeriodicBoundaryCondition::mapPeriodicPosition (BoundaryConditions.cpp:93-140)
        double c[3] = {px, py, pz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double Lp = pp.period[a];
            if (Lp <= 1e-12) continue;
            c[a] = fmod(c[a], Lp);
            if (c[a] < 0.0) c[a] += Lp;
        }
        px = c[0]; py = c[1]; pz = c[2];
        int h2 = locate(M, px, py, pz, hint);
        hint = h2;
        if (h2 >= 0) resolved = h2;
    }
    if (!done) {
        resolved = locate(M, px, py, pz, hint);
        ok = resolved >= 0;
    }
    if (!ok) status = 2;
    if (status == 0 && resolved < 0) status = 2;
    if (status == 2 && pp.body_tally) {
        if (detect_face(M, px, py, pz, pp.otol, false, 0.0) < 0) {
            ledger_tally(L, 6, S, pp, ke, false);
            if (pp.patches) {
                // the face of the body box nearest to where the particle left the mesh
                const double d[6] = {fabs(px - pp.blo[0]), fabs(pp.bhi[0] - px), fabs(py - pp.blo[1]),
                                     fabs(pp.bhi[1] - py), fabs(pz - pp.blo[2]), fabs(pp.bhi[2] - pz)};
                int k = 0;
                double dk = d[0];
#pragma unroll
                for (int f = 1; f < 6; ++f)
                    if (d[f] < dk) {
                        dk = d[f];
                        k = f;
                    }
                fx_atomic_add(&L->patch_q[k][0], &L->patch_q[k][1], fx_from_double(S.q * S.w * pp.inv_uq));
                atomicAdd(&L->patch_n[k], 1ull);
                // secondaries leave the face: it gains delta |q| w, the ledger records their charge
                if (pp.see_model && S.electron_like) {
                    const double emitted = see_yield(pp, ke / kElementaryCharge) * fabs(S.q) * S.w;
                    if (emitted > 0.0) {
                        fx_atomic_add(&L->patch_q[k][0], &L->patch_q[k][1], fx_from_double(emitted * pp.inv_uq));
                        fx_atomic_add(&L->emit_q[6][0], &L->emit_q[6][1], fx_from_double(-emitted * pp.inv_uq));
                    }
                }
            }
        }
    }
    if (status == 1) return kTetAbsorbed;
    if (status == 2) return kTetEscaped;
    return resolved;
}

// ElasticCollisionCrossSection::calculateCrossSection, CollisonTypes.cpp:60-78.
__device__ inline double sigma_elastic(const SpeciesDev& S, double e_ev)
{
    if (!(e_ev >= S.mcc_eth)) return 0.0;
    double eref = S.mcc_eref > 1e-6 ? S.mcc_eref : 1e-6;
    double s = S.mcc_alpha == 0.0 ? S.mcc_sigma : S.mcc_sigma * pow(eref / e_ev, S.mcc_alpha);
    s = fmin(s, S.mcc_sigma);
    return s > 0.0 ? s : 0.0;
}

// MonteCarloCollisionHandler::processCollisions for one elastic process
// (CollisionAlgorithm.cpp:500-538, 189-210) with Philox streams (seed; id, step, 2|3).
// mode 0: the reference's two draws against p = nu dt; mode 1: one draw against
// 1 - exp(-nu dt); mode 2: null collision (below).
__device__ inline bool mcc_elastic(const SpeciesDev& S, const PushParams& pp, uint32_t pid, double& vx, double& vy,
                                   double& vz)
{
    const double qe = 1.602176634e-19;
    const double v2 = vx * vx + vy * vy + vz * vz;
    bool hit;
    double speed;
    if (S.mcc_mode == 2) {
        // null collision: with nu_max = n sigma_max vmax (sigma <= sigma_max and speed <= vmax
        // for every particle on this path), select with P = 1 - exp(-nu_max dt) by the cheap
        // selection draw, then collide with probability nu / nu_max on the Philox stream.  A
        // particle faster than vmax (and every particle before the first push has set vmax)
        // takes the direct draw of mode 1.
        const double vm = S.vmax ? (double)__uint_as_float(__ldg(S.vmax)) : 0.0;
        double u0, u1;
        if (vm > 0.0 && v2 <= vm * vm) {
            const double numax = S.mcc_n * S.mcc_sigma * vm;
            const double xmax = numax * pp.dt;
            const double us = select_uniform(pp.seed, pid, pp.step);
            // 1 - exp(-x) <= x, and the computed value exceeds x by at most 2^-52
            if (us >= xmax + 1e-15 || !(us < 1.0 - exp(-xmax))) return false;
            speed = sqrt(v2);
            const double nu = S.mcc_n * sigma_elastic(S, 0.5 * S.m * speed * speed / qe) * speed;
            uniform2(pp.seed, pid, pp.step, 2u, u0, u1);
            hit = u0 * numax < nu;
        } else {
            speed = sqrt(v2);
            const double nu = S.mcc_n * sigma_elastic(S, 0.5 * S.m * speed * speed / qe) * speed;
            uniform2(pp.seed, pid, pp.step, 2u, u0, u1);
            const double x = nu * pp.dt;
            hit = !(u0 >= x + 1e-15) && u0 < 1.0 - exp(-x);
        }
    } else {
        speed = sqrt(v2);
        const double nu = S.mcc_n * sigma_elastic(S, 0.5 * S.m * speed * speed / qe) * speed;
        double u0, u1;
        uniform2(pp.seed, pid, pp.step, 2u, u0, u1);
        if (S.mcc_mode == 0) {
            const double p = fmin(fmax(nu * pp.dt, 0.0), 1.0);
            hit = (u0 < p) && !(u1 >= p);
        } else {
            // p = 1 - exp(-x) <= x, and the computed p exceeds x by at most 2^-52 (exp within one
            // ulp near 1, the subtraction exact), so u0 >= x + 1e-15 already decides "no hit"
            // without the exponential; otherwise p is evaluated as before
            const double x = nu * pp.dt;
            hit = (u0 >= x + 1e-15) ? false : (u0 < 1.0 - exp(-x));
        }
    }
    if (!hit) return false;
    double w0, w1;
    uniform2(pp.seed, pid, pp.step, 3u, w0, w1);
    const double theta = acos(-1.0 + 2.0 * w0);
    const double phi = 6.283185307179586476925286766559 * w1;
    const double st = sin(theta);
    vx = speed * st * cos(phi);
    vy = speed * st * sin(phi);
    vz = speed * cos(theta);
    return true;
}

}  // namespace scdat

namespace scdat {

// Particles that still have time left after a pass: index, sub-steps used, remaining time
// and the step-start speed (adaptiveTimeStep keeps using it, PICParticleAlgorithms.cpp:762).
struct DeferList {
    unsigned* count;
    unsigned cap;
    uint32_t* idx;
    int* it;
    double* rem;
    double* vstart;
};

enum { kDone = 0, kCapped = 1, kLost = 2 };

// Per-lane push statistics of the current 32-particle chunk (one particle per lane): its
// kinetic energy, its sub-steps and its events (kEvLost | kEvActive | kEvHit).
// warp_chunk_end folds them into the warp's totals in shared memory (kinetic energy as exact
// fixed point), so the lanes carry only a few registers and the sums do not depend on which
// warp took which chunk.
struct PushStats {
    double ke;
    unsigned nsub, ev;
    float v2;  // largest squared speed of the chunk's particles still active after their push
};
enum : unsigned { kEvLost = 1u, kEvActive = 2u, kEvHit = 4u };

// Kinetic energy accumulates as 128-bit fixed point with a unit of 2^-60 J: a 1 eV particle is
// resolved to 1e-19 of itself and the sum can reach 8 J.
constexpr double kKeInvUnit = 1152921504606846976.0;  // 2^60
constexpr double kKeUnit = 8.673617379884035e-19;     // 2^-60

// the warp's totals for the kernel: kinetic energy; sub-steps, lost, MCC hits, active
struct WarpStats {
    Fx128 ke;
    unsigned long long n[4];
    unsigned v2max;  // float bits of the largest squared speed (non-negative floats order as integers)
};

__device__ __forceinline__ WarpStats& warp_slot()
{
    __shared__ WarpStats slot[32];
    return slot[threadIdx.x >> 5];
}

// start of a push kernel; every lane calls it
__device__ __forceinline__ void warp_stats_begin()
{
    if ((threadIdx.x & 31) == 0) warp_slot() = WarpStats{Fx128{0ull, 0ll}, {0ull, 0ull, 0ull, 0ull}, 0u};
    __syncwarp();
}

// end of a chunk; every lane calls it: energies as fixed point summed exactly, counts by
// warp reductions and ballots
__device__ __forceinline__ void warp_chunk_end(PushStats& c)
{
    const Fx128 v = fx_from_double(c.ke * kKeInvUnit);
    unsigned long long lo = v.lo;
    long long hi = v.hi;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long lo2 = __shfl_down_sync(0xffffffffu, lo, o);
        const long long hi2 = __shfl_down_sync(0xffffffffu, hi, o);
        const unsigned long long s = lo + lo2;
        hi += hi2 + (s < lo ? 1 : 0);
        lo = s;
    }
    const unsigned sub = __reduce_add_sync(0xffffffffu, c.nsub);
    const unsigned lost = __popc(__ballot_sync(0xffffffffu, c.ev & kEvLost));
    const unsigned hit = __popc(__ballot_sync(0xffffffffu, c.ev & kEvHit));
    const unsigned act = __popc(__ballot_sync(0xffffffffu, c.ev & kEvActive));
    const unsigned v2 = __reduce_max_sync(0xffffffffu, __float_as_uint(c.v2));
    if ((threadIdx.x & 31) == 0) {
        WarpStats& w = warp_slot();
        fx_add(w.ke, Fx128{lo, hi});
        w.n[0] += sub;
        w.n[1] += lost;
        w.n[2] += hit;
        w.n[3] += act;
        w.v2max = max(w.v2max, v2);
    }
    c = PushStats{0.0, 0u, 0u, 0.0f};
}

// Flush the warp's totals into a ledger and its kinetic-energy accumulator (lo, hi words);
// every lane calls it, after warp_chunk_end.  Integer sums only, so the totals do not depend
// on the schedule.
// vmax: the species' maximum-speed slots (SpeciesDev::vmax, may be null); the current push's
// slot [1] is raised to the warp's largest speed.
__device__ __forceinline__ void warp_stats_flush(LedgerDev* L, unsigned long long* ke_acc, unsigned* vmax = nullptr)
{
    if ((threadIdx.x & 31) == 0) {
        WarpStats& w = warp_slot();
        if (w.n[0]) atomicAdd(&L->substeps, w.n[0]);
        if (w.n[1]) atomicAdd(&L->lost_events, w.n[1]);
        if (w.n[2]) atomicAdd(&L->mcc_hits, w.n[2]);
        if (w.n[3]) atomicAdd(&L->active, w.n[3]);
        fx_atomic_add(ke_acc, ke_acc + 1, w.ke);
        if (vmax && w.v2max) atomicMax(vmax + 1, __float_as_uint(sqrtf(__uint_as_float(w.v2max))));
        w = WarpStats{Fx128{0ull, 0ll}, {0ull, 0ull, 0ull, 0ull}, 0u};
    }
    __syncwarp();
}

// Pass 1 hands out runs of kRun consecutive 32-particle chunks: a warp's next chunk then lies
// in the tets of its previous one (particles are sorted by tet), so the records it needs are
// still in L1, and the work counter sees one atomic per 256 particles.
constexpr int kRun = 8;

// next chunk (or run) of a launch's work counter (the same value in every lane)
__device__ __forceinline__ unsigned next_chunk(unsigned* ctr)
{
    unsigned g = 0;
    if ((threadIdx.x & 31) == 0) g = atomicAdd(ctr, 1u);
    return __shfl_sync(0xffffffffu, g, 0);
}

// warp-aggregated append to a deferred list; every lane of the warp calls it
__device__ __forceinline__ unsigned warp_append(bool want, unsigned* cnt)
{
    const int lane = threadIdx.x & 31;
    unsigned m = __ballot_sync(0xffffffffu, want);
    unsigned base = 0;
    if (m) {
        int leader = __ffs(m) - 1;
        if (lane == leader) base = atomicAdd(cnt, (unsigned)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    return base + (unsigned)__popc(m & ((1u << lane) - 1u));
}

constexpr int kCap1 = 1;   // sub-steps every particle gets in pass 1 (1, 2, 4: 45.6, 46.1, 47.0 ms at 128^3)
constexpr int kCap2 = 16;  // further sub-steps in pass 2; pass 3 runs to the end

}  // namespace scdat
