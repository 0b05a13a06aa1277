// push_mixed.cu -- the precision form of the particle step.
//
// Particles store FP32 positions relative to the origin node (local vertex 0) of their tet
// and FP32 velocities (a 32-byte record, plus the tet and particle ids).  Every tet has one
// 256-byte record: in its first line the FP32 inverse Jacobian, the nodal E of its 4 nodes as
// E0 and three differences (refreshed after every field solve), its node ids and neighbours,
// so a sub-step inside the tet reads one cache line; in its second, per face the FP32 origin
// shift to the neighbour with the neighbour's id, which the walk reads.  Gather, adaptive
// sub-step, Boris and the in-tet test run in FP32; a move into a face neighbour is re-based in
// FP32 by the stored shift; a walk that meets a boundary face or runs long reconstructs the
// FP64 absolute position and uses the FP64 locate.  Deposit weights are FP32 barycentrics
// promoted to FP64 before the exact fixed-point accumulation (one 64-bit word per node,
// fx_red_word).
//
// Sub-steps run in passes so that warps stay converged: pass 1 gives every particle at most
// kCap1 sub-steps and appends the unfinished ones to a list; pass 2 gives those up to kCap2
// more; pass 3 finishes the rest.  The step structure is the reference's
// CrossTetrahedron::integrateTrajectory (PICParticleAlgorithms.cpp:536-740).
#include "batch.cuh"
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

// record layout (64 words): [0..8] J^-1, [9..11] E0, [12..20] E1-E0, E2-E0, E3-E0,
// [21..23] unused, [24..27] node ids, [28..31] face neighbours | [32..47] per face f the origin
// minus the neighbour's origin (FP32) and the neighbour id, one float4 each (the walk reads one
// 16-byte load per step for both), [48..63] unused

__device__ __forceinline__ int4 node_ids(const MeshView& M, int t)
{
    return __ldg(reinterpret_cast<const int4*>(M.trec + 64 * (int64_t)t) + 6);
}

// Rewrite words 9..20 of record t (E0 and the three differences) from the nodal field, keeping
// J^-1 and the node ids that share those 16-byte lines.  Four lanes share a record, lane q
// writing its float4 2 + q, so a warp writes 8 records' 64 contiguous bytes each.
__device__ __forceinline__ void refresh_trec_part(int64_t t, int q, const int4* __restrict__ tet,
                                                  const double* __restrict__ E, float* trec)
{
    const int4 tn = __ldg(tet + t);
    const double* e0 = E + 3 * (int64_t)tn.x;
    float4* r4 = reinterpret_cast<float4*>(trec + 64 * t) + 2 + q;
    const double a0 = __ldg(e0), a1 = __ldg(e0 + 1), a2 = __ldg(e0 + 2);
    if (q == 0) {
        const float j8 = r4->x;
        *r4 = make_float4(j8, (float)a0, (float)a1, (float)a2);
    } else if (q == 1) {
        const double* e1 = E + 3 * (int64_t)tn.y;
        const double* e2 = E + 3 * (int64_t)tn.z;
        *r4 = make_float4((float)(__ldg(e1) - a0), (float)(__ldg(e1 + 1) - a1), (float)(__ldg(e1 + 2) - a2),
                          (float)(__ldg(e2) - a0));
    } else if (q == 2) {
        const double* e2 = E + 3 * (int64_t)tn.z;
        const double* e3 = E + 3 * (int64_t)tn.w;
        *r4 = make_float4((float)(__ldg(e2 + 1) - a1), (float)(__ldg(e2 + 2) - a2), (float)(__ldg(e3) - a0),
                          (float)(__ldg(e3 + 1) - a1));
    } else {
        const double* e3 = E + 3 * (int64_t)tn.w;
        const float4 old = *r4;
        *r4 = make_float4((float)(__ldg(e3 + 2) - a2), old.y, old.z, old.w);
    }
}

__device__ __forceinline__ void baryj(const float* j, float rx, float ry, float rz, float l[4])
{
    l[1] = j[0] * rx + j[1] * ry + j[2] * rz;
    l[2] = j[3] * rx + j[4] * ry + j[5] * rz;
    l[3] = j[6] * rx + j[7] * ry + j[8] * rz;
    l[0] = 1.0f - l[1] - l[2] - l[3];
}

__device__ __forceinline__ void load_j(const MeshView& M, int t, float j[9])
{
    const float4* g = reinterpret_cast<const float4*>(M.trec + 64 * (int64_t)t);
    float4 a = __ldg(g), b = __ldg(g + 1);
    j[0] = a.x; j[1] = a.y; j[2] = a.z; j[3] = a.w; j[4] = b.x; j[5] = b.y; j[6] = b.z; j[7] = b.w;
    j[8] = __ldg(M.trec + 64 * (int64_t)t + 8);
}

__device__ __forceinline__ double3 origin(const MeshView& M, int t)
{
    int o = __ldg(&M.tet[t].x);
    return make_double3(__ldg(M.xyz + 3 * o), __ldg(M.xyz + 3 * o + 1), __ldg(M.xyz + 3 * o + 2));
}

// Result of a relocation: the new tet (or -1), the offset r and the carried start offset s
// re-based to its origin.  Returned by value so that the caller's flight state stays in
// registers across the out-of-line call.
struct Reloc {
    int t;
    float rx, ry, rz, sx, sy, sz;
};

// Relocate the FP32 offset r (relative to the origin of `cur`) by a straight walk across the
// most violated face, re-basing r (and the carried start offset s) with each neighbour's
// stored origin shift; a walk that meets a boundary face or runs long falls back to the FP64
// locate on the absolute position.
static __device__ __noinline__ Reloc relocate_f(const MeshView& M, int cur, float rx, float ry, float rz, float sx,
                                                float sy, float sz)
{
    int t = cur;
    float qx = rx, qy = ry, qz = rz, ox = 0.f, oy = 0.f, oz = 0.f;
    float l[4], j[9];
    load_j(M, t, j);
    baryj(j, qx, qy, qz, l);
    for (int k = 0; k < kWalkSteps; ++k) {
        // the most violated face (lowest barycentric, the first on ties), without indexing l
        int f = 0;
        float lm = l[0];
        if (l[1] < lm) { lm = l[1]; f = 1; }
        if (l[2] < lm) { lm = l[2]; f = 2; }
        if (l[3] < lm) f = 3;
        const float4 sh = __ldg(reinterpret_cast<const float4*>(M.trec + 64 * (int64_t)t) + 8 + f);
        const int nt = __float_as_int(sh.w);
        if (nt < 0) break;
        const float dx = sh.x, dy = sh.y, dz = sh.z;
        qx += dx; qy += dy; qz += dz;
        ox += dx; oy += dy; oz += dz;
        t = nt;
        load_j(M, t, j);
        baryj(j, qx, qy, qz, l);
        if (inside_f(l)) return Reloc{t, qx, qy, qz, sx + ox, sy + oy, sz + oz};
        if (!(l[0] == l[0])) break;
    }
    const double3 oc = origin(M, cur);
    double px = oc.x + (double)rx, py = oc.y + (double)ry, pz = oc.z + (double)rz;
    int tt = locate_far(M, px, py, pz, cur);
    if (tt < 0) return Reloc{-1, rx, ry, rz, sx, sy, sz};
    double3 on = origin(M, tt);
    float dx = (float)(oc.x - on.x), dy = (float)(oc.y - on.y), dz = (float)(oc.z - on.z);
    return Reloc{tt, (float)(px - on.x), (float)(py - on.y), (float)(pz - on.z), sx + dx, sy + dy, sz + dz};
}

// Deposit along start -> end (both FP32 offsets from the origin of t) into t, whose inverse
// Jacobian the caller holds in j: the sample points that lie in t (the sub-step changed tet),
// summed in FP32 per node, then converted once to fixed point.
__device__ __forceinline__ void deposit_traj_f(const MeshView& M, const SpeciesDev& S, const PushParams& pp, int t,
                                               const float j[9], float sx, float sy, float sz, float rx, float ry,
                                               float rz, ChargeAcc A)
{
    float sum[4] = {0.f, 0.f, 0.f, 0.f};
    double cw = S.cw_seg;
    bool any = false;
    const int nseg = pp.nseg;
    float tx = rx - sx, ty = ry - sy, tz = rz - sz;
    if (sqrtf(tx * tx + ty * ty + tz * tz) < 1e-15f || pp.dep_kernel == 0) {
        float q0[4];
        if (pp.dep_kernel == 0 && !(sqrtf(tx * tx + ty * ty + tz * tz) < 1e-15f)) baryj(j, rx, ry, rz, q0);
        else baryj(j, sx, sy, sz, q0);
        if (inside_f(q0)) {
            for (int q = 0; q < 4; ++q) sum[q] = q0[q];
            any = true;
        }
        cw = S.q * S.w;
    } else {
        float ls[4], dl[4];
        baryj(j, sx, sy, sz, ls);
        dl[1] = j[0] * tx + j[1] * ty + j[2] * tz;
        dl[2] = j[3] * tx + j[4] * ty + j[5] * tz;
        dl[3] = j[6] * tx + j[7] * ty + j[8] * tz;
        dl[0] = -dl[1] - dl[2] - dl[3];
        if (pp.dep_kernel == 2) {
            const float gn[3] = {-0.7745966692414834f, 0.0f, 0.7745966692414834f};
            const float gw[3] = {5.0f / 18.0f, 8.0f / 18.0f, 5.0f / 18.0f};
            for (int sg = 0; sg < nseg; ++sg) {
                float tc = ((float)sg + 0.5f) / (float)nseg, th = 0.5f / (float)nseg;
                for (int q = 0; q < 3; ++q) {
                    float tau = tc + th * gn[q];
                    float lq[4] = {ls[0] + tau * dl[0], ls[1] + tau * dl[1], ls[2] + tau * dl[2], ls[3] + tau * dl[3]};
                    if (inside_f(lq)) {
                        for (int k = 0; k < 4; ++k) sum[k] = fmaf(gw[q], lq[k], sum[k]);
                        any = true;
                    }
                }
            }
        } else {
            // The segment cloud's points tau_k = (k + 1/2) / nseg lie on a line, and
            // lambda_i(tau) = ls_i + tau dl_i is affine, so the points inside the tet (every
            // lambda_i in [-1e-8, 1 + 1e-8]) are those with tau in one interval [lo, hi]: their
            // count n and the sum of their lambdas, n ls + (sum of their tau) dl, follow in closed
            // form instead of point by point.
            const float e = 1e-8f;
            float lo = 0.0f, hi = 1.0f;
            bool empty = false;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (dl[i] != 0.0f) {
                    const float inv = 1.0f / dl[i];
                    const float a = (-e - ls[i]) * inv, b = (1.0f + e - ls[i]) * inv;
                    lo = fmaxf(lo, fminf(a, b));
                    hi = fminf(hi, fmaxf(a, b));
                } else if (!(ls[i] >= -e && ls[i] <= 1.0f + e)) {
                    empty = true;
                }
            }
            const int ka = max(0, (int)ceilf(lo * (float)nseg - 0.5f));
            const int kb = min(nseg - 1, (int)floorf(hi * (float)nseg - 0.5f));
            if (!empty && kb >= ka) {
                const float n = (float)(kb - ka + 1);
                const float st = 0.5f * n * (float)(ka + kb + 1) / (float)nseg;
#pragma unroll
                for (int k = 0; k < 4; ++k) sum[k] = n * ls[k] + st * dl[k];
                any = true;
            }
        }
    }
    if (!any) return;
    const int4 nd4 = node_ids(M, t);
    const int nd[4] = {nd4.x, nd4.y, nd4.z, nd4.w};
    for (int k = 0; k < 4; ++k) {
        int node = nd[k];
        fx_red_word(A, node, (cw * (double)sum[k]) * pp.inv_uq);
    }
}

struct FlightF {
    float rx, ry, rz, vx, vy, vz;
    float rem, vstart;
    int cur, it;
};

// Run sub-steps until the step's time is used up, the particle is lost, or `cap` sub-steps
// ran in this call.
__device__ __forceinline__ int advance_f(const MeshView& M, const SpeciesDev& S, const PushParams& pp, FlightF& f,
                                         int cap, ChargeAcc A,
                                         unsigned& nsub)
{
    const float qm = (float)S.qm;
    const float floor_ratio = (float)pp.floor_ratio;
    const double qw = S.q * S.w;
    // only J^-1 stays in registers; E0, the E differences and the node ids are read from the
    // record (already in L1) where they are used
    const float4* rec = reinterpret_cast<const float4*>(M.trec + 64 * (int64_t)f.cur);
    float J[9];
    load_j(M, f.cur, J);
    float l[4];
    baryj(J, f.rx, f.ry, f.rz, l);
    bool in = inside_f(l);
    int k = 0;
    while (f.rem > 1e-20f && f.it < kMaxSubsteps) {
        if (k == cap) return kCapped;
        ++k;
        ++f.it;
        float Ex = 0.f, Ey = 0.f, Ez = 0.f;
        if (in) {  // E = E0 + sum_i lambda_i (E_i - E0), i = 1..3
            const float4 c = __ldg(rec + 2), d = __ldg(rec + 3), e = __ldg(rec + 4), g = __ldg(rec + 5);
            Ex = fmaf(l[1], d.x, fmaf(l[2], d.w, fmaf(l[3], e.z, c.y)));
            Ey = fmaf(l[1], d.y, fmaf(l[2], e.x, fmaf(l[3], e.w, c.z)));
            Ez = fmaf(l[1], d.z, fmaf(l[2], e.y, fmaf(l[3], g.x, c.w)));
        }
        float adt = f.rem;
        float Em = sqrtf(Ex * Ex + Ey * Ey + Ez * Ez);
        if (Em > 1e-10f) {
            float acc = Em * fabsf(qm);
            if (acc > 1e-10f && f.vstart > 1.0f) adt = fminf(adt, 0.1f * f.vstart / acc);
        }
        adt = fmaxf(adt, f.rem * floor_ratio);
        adt = fminf(adt, f.rem);
        float sx = f.rx, sy = f.ry, sz = f.rz;
        if (fabsf(qm) > 1e-20f) {
            float h = 2.0f * (qm * (0.5f * adt));
            f.vx = fmaf(h, Ex, f.vx);
            f.vy = fmaf(h, Ey, f.vy);
            f.vz = fmaf(h, Ez, f.vz);
        }
        f.rx = fmaf(f.vx, adt, f.rx);
        f.ry = fmaf(f.vy, adt, f.ry);
        f.rz = fmaf(f.vz, adt, f.rz);
        float le[4];
        baryj(J, f.rx, f.ry, f.rz, le);
        if (inside_f(le)) {
            if (pp.deposit) {
                if (in) {
                    float tx = f.rx - sx, ty = f.ry - sy, tz = f.rz - sz;
                    bool tiny = sqrtf(tx * tx + ty * ty + tz * tz) < 1e-15f;
                    const int4 nd4 = __ldg(reinterpret_cast<const int4*>(rec) + 6);
                    const int nd[4] = {nd4.x, nd4.y, nd4.z, nd4.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        float lk = tiny ? l[q] : (pp.dep_kernel == 0 ? le[q] : 0.5f * (l[q] + le[q]));
                        fx_red_word(A, nd[q], (qw * (double)lk) * pp.inv_uq);
                    }
                } else {
                    deposit_traj_f(M, S, pp, f.cur, J, sx, sy, sz, f.rx, f.ry, f.rz, A);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) l[q] = le[q];
            in = true;
        } else {
            const Reloc rl = relocate_f(M, f.cur, f.rx, f.ry, f.rz, sx, sy, sz);
            const int nt = rl.t;
            if (nt < 0) return kLost;
            f.rx = rl.rx; f.ry = rl.ry; f.rz = rl.rz;
            sx = rl.sx; sy = rl.sy; sz = rl.sz;
            f.cur = nt;
            rec = reinterpret_cast<const float4*>(M.trec + 64 * (int64_t)nt);
            load_j(M, nt, J);
            if (pp.deposit) deposit_traj_f(M, S, pp, nt, J, sx, sy, sz, f.rx, f.ry, f.rz, A);
            baryj(J, f.rx, f.ry, f.rz, l);
            in = inside_f(l);
        }
        f.rem -= adt;
        ++nsub;
    }
    return f.it >= kMaxSubsteps ? kLost : kDone;
}

// End of a particle's step: boundary events for a lost particle, the statistics, the fused
// MCC, and the store.
__device__ __forceinline__ void finish_f(const MeshView& M, const ParticleStore& P, const SpeciesDev& S,
                                         const PushParams& pp, LedgerDev* L, int64_t i, FlightF& f, int st,
                                         PushStats& c)
{
    double dvx = f.vx, dvy = f.vy, dvz = f.vz;
    const double ke = 0.5 * S.m * (dvx * dvx + dvy * dvy + dvz * dvz);
    int tet_out = f.cur;
    if (st == kLost) {
        c.ev |= kEvLost;
        double px, py, pz;
        int hint = f.cur;
        if (f.cur >= 0) {
            double3 o = origin(M, f.cur);
            px = o.x + (double)f.rx; py = o.y + (double)f.ry; pz = o.z + (double)f.rz;
        } else {
            px = f.rx; py = f.ry; pz = f.rz;
            hint = 0;
        }
        tet_out = resolve_lost(M, S, pp, L, px, py, pz, ke, hint);
        if (tet_out >= 0) {
            double3 o = origin(M, tet_out);
            f.rx = (float)(px - o.x); f.ry = (float)(py - o.y); f.rz = (float)(pz - o.z);
        } else {
            // inactive particles keep an absolute FP32 position for read-back
            f.rx = (float)px; f.ry = (float)py; f.rz = (float)pz;
        }
    }
    c.ke += ke;
    if (tet_out >= 0) {
        c.ev |= kEvActive;
        if (S.mcc_mode == 2) c.v2 = fmaxf(c.v2, (float)(dvx * dvx + dvy * dvy + dvz * dvz));  // the null-collision speed bound
        if (pp.do_mcc && S.mcc_enabled && mcc_elastic(S, pp, P.id[i], dvx, dvy, dvz)) {
            c.ev |= kEvHit;
            f.vx = (float)dvx; f.vy = (float)dvy; f.vz = (float)dvz;
        }
    }
    mix_store(P, i, f.rx, f.ry, f.rz, f.vx, f.vy, f.vz);
    P.tet[i] = tet_out;
}

__device__ __forceinline__ void defer_store_f(const ParticleStore& P, const DeferList& D, unsigned slot, int64_t i,
                                              const FlightF& f)
{
    D.idx[slot] = (uint32_t)i;
    D.it[slot] = f.it;
    D.rem[slot] = f.rem;
    D.vstart[slot] = f.vstart;
    mix_store(P, i, f.rx, f.ry, f.rz, f.vx, f.vy, f.vz);
    P.tet[i] = f.cur;
}

// Pass 1's load of particle i: from the store in place, or through a pending re-sort (R), whose
// particle id it copies into the store at once (the fused MCC reads it there).  Every particle
// a re-sort keeps is active, and pass 1 writes each of them back (finished or deferred).
__device__ __forceinline__ void load_first(const ParticleStore& P, const SortedSource& R, int64_t i, FlightF& f)
{
    if (R.perm) {
        const uint32_t j = __ldg(R.perm + i);
        const uint32_t key = __ldg(R.keys + i);
        f.cur = key < R.nohint_key ? (int)key : kTetNoHint;
        const float4 a = __ldg(R.mix + 2 * (int64_t)j), b = __ldg(R.mix + 2 * (int64_t)j + 1);
        f.rx = a.x; f.ry = a.y; f.rz = a.z; f.vx = a.w;
        f.vy = b.x; f.vz = b.y;
        P.id[i] = __ldg(R.id + j);
    } else {
        f.cur = P.tet[i];
        mix_load(P, i, f.rx, f.ry, f.rz, f.vx, f.vy, f.vz);
    }
}

// Pass 1 for the 32 particles [base, base + 32) of one warp: at most kCap1 sub-steps, the
// unfinished ones appended to D.
__device__ __forceinline__ void push1_warp(const MeshView& M, const ParticleStore& P, const SortedSource& R,
                                           const SpeciesDev& S, const PushParams& pp, const DeferList& D, ChargeAcc A,
                                           LedgerDev* L, int64_t base, int64_t n, PushStats& c)
{
    const int64_t i = base + (threadIdx.x & 31);
    int st = -1;
    FlightF f;
    if (i < n) {
        load_first(P, R, i, f);
        if (f.cur <= kTetAbsorbed) {
            // updateStatistics sums every particle the container still holds (PICCycle.cpp:941-966)
            double ux = f.vx, uy = f.vy, uz = f.vz;
            c.ke += 0.5 * S.m * (ux * ux + uy * uy + uz * uz);
        } else {
            f.vstart = sqrtf(f.vx * f.vx + f.vy * f.vy + f.vz * f.vz);
            f.rem = (float)pp.dt;
            f.it = 0;
            st = kDone;
            if (f.cur < 0) {
                // no hint: the stored offset is an absolute position
                double px = f.rx, py = f.ry, pz = f.rz;
                int t = locate_far(M, px, py, pz, -1);
                if (t < 0) {
                    st = kLost;
                } else {
                    double3 o = origin(M, t);
                    f.rx = (float)(px - o.x); f.ry = (float)(py - o.y); f.rz = (float)(pz - o.z);
                    f.cur = t;
                }
            }
            if (st != kLost) st = advance_f(M, S, pp, f, kCap1, A, c.nsub);
        }
    }
    unsigned slot = warp_append(st == kCapped, D.count);
    if (st == kCapped && slot < D.cap) {
        defer_store_f(P, D, slot, i, f);
    } else if (st >= 0) {
        if (st == kCapped) st = advance_f(M, S, pp, f, 0x7fffffff, A, c.nsub);
        finish_f(M, P, S, pp, L, i, f, st, c);
    }
    warp_chunk_end(c);
}

// Pass 1's one sub-step for a species that rarely leaves its tet, with no walk code: the
// sub-step is computed exactly as advance_f computes it and committed (deposit, position,
// velocity, time) only when the particle ends inside its tet.  A particle that would leave
// its tet, or whose start point is outside it, keeps its state untouched and goes to the
// walking passes, which then run the same sub-step with the same arithmetic; so the result is
// bitwise the walking pass 1's.  kDone: step finished; kCapped: continue in pass 2.
__device__ __forceinline__ int advance_stay_f(const MeshView& M, const SpeciesDev& S, const PushParams& pp,
                                              FlightF& f, ChargeAcc A, unsigned& nsub)
{
    if (!(f.rem > 1e-20f && f.it < kMaxSubsteps)) return f.it >= kMaxSubsteps ? kLost : kDone;
    const float qm = (float)S.qm;
    const float4* rec = reinterpret_cast<const float4*>(M.trec + 64 * (int64_t)f.cur);
    float l[4];
    {
        float J[9];
        load_j(M, f.cur, J);
        baryj(J, f.rx, f.ry, f.rz, l);
    }
    if (!inside_f(l)) return kCapped;
    const float4 c = __ldg(rec + 2), d = __ldg(rec + 3), e = __ldg(rec + 4), g = __ldg(rec + 5);
    const float Ex = fmaf(l[1], d.x, fmaf(l[2], d.w, fmaf(l[3], e.z, c.y)));
    const float Ey = fmaf(l[1], d.y, fmaf(l[2], e.x, fmaf(l[3], e.w, c.z)));
    const float Ez = fmaf(l[1], d.z, fmaf(l[2], e.y, fmaf(l[3], g.x, c.w)));
    float adt = f.rem;
    const float Em = sqrtf(Ex * Ex + Ey * Ey + Ez * Ez);
    if (Em > 1e-10f) {
        const float acc = Em * fabsf(qm);
        if (acc > 1e-10f && f.vstart > 1.0f) adt = fminf(adt, 0.1f * f.vstart / acc);
    }
    adt = fmaxf(adt, f.rem * (float)pp.floor_ratio);
    adt = fminf(adt, f.rem);
    float vx = f.vx, vy = f.vy, vz = f.vz;
    if (fabsf(qm) > 1e-20f) {
        const float h = 2.0f * (qm * (0.5f * adt));
        vx = fmaf(h, Ex, vx);
        vy = fmaf(h, Ey, vy);
        vz = fmaf(h, Ez, vz);
    }
    const float rx = fmaf(vx, adt, f.rx), ry = fmaf(vy, adt, f.ry), rz = fmaf(vz, adt, f.rz);
    float le[4];
    {
        float J[9];
        load_j(M, f.cur, J);
        baryj(J, rx, ry, rz, le);
    }
    if (!inside_f(le)) return kCapped;
    ++f.it;
    if (pp.deposit) {
        const double qw = S.q * S.w;
        const float tx = rx - f.rx, ty = ry - f.ry, tz = rz - f.rz;
        const bool tiny = sqrtf(tx * tx + ty * ty + tz * tz) < 1e-15f;
        const int4 nd4 = __ldg(reinterpret_cast<const int4*>(rec) + 6);
        const int nd[4] = {nd4.x, nd4.y, nd4.z, nd4.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float lk = tiny ? l[q] : (pp.dep_kernel == 0 ? le[q] : 0.5f * (l[q] + le[q]));
            fx_red_word(A, nd[q], (qw * (double)lk) * pp.inv_uq);
        }
    }
    f.rx = rx; f.ry = ry; f.rz = rz;
    f.vx = vx; f.vy = vy; f.vz = vz;
    f.rem -= adt;
    ++nsub;
    return (f.rem > 1e-20f && f.it < kMaxSubsteps) ? kCapped : (f.it >= kMaxSubsteps ? kLost : kDone);
}

// Stay-first pass 1 for the 32 particles [base, base + 32): one sub-step for those that stay in
// their tet; everything else (leaving the tet, more time left, no location hint) goes to D,
// whose capacity covers the whole species, so nothing overflows.
__device__ __forceinline__ void push1_stay_warp(const MeshView& M, const ParticleStore& P, const SortedSource& R,
                                                const SpeciesDev& S, const PushParams& pp, const DeferList& D,
                                                ChargeAcc A, LedgerDev* L, int64_t base, int64_t n, PushStats& c)
{
    const int64_t i = base + (threadIdx.x & 31);
    int st = -1;
    FlightF f;
    if (i < n) {
        load_first(P, R, i, f);
        if (f.cur <= kTetAbsorbed) {
            double ux = f.vx, uy = f.vy, uz = f.vz;
            c.ke += 0.5 * S.m * (ux * ux + uy * uy + uz * uz);
        } else {
            f.vstart = sqrtf(f.vx * f.vx + f.vy * f.vy + f.vz * f.vz);
            f.rem = (float)pp.dt;
            f.it = 0;
            st = f.cur < 0 ? kCapped : advance_stay_f(M, S, pp, f, A, c.nsub);
        }
    }
    const unsigned slot = warp_append(st == kCapped, D.count);
    if (st == kCapped) {
        if (slot < D.cap) {
            defer_store_f(P, D, slot, i, f);
        } else {
            // the step fails with this flag; the particle is stored as it stands
            atomicOr(&L->flags, (unsigned long long)kFlagDeferOverflow);
            mix_store(P, i, f.rx, f.ry, f.rz, f.vx, f.vy, f.vz);
            P.tet[i] = f.cur;
        }
    } else if (st >= 0) {
        finish_f(M, P, S, pp, L, i, f, st, c);
    }
    warp_chunk_end(c);
}

// Passes 2 and 3 for entries [base, base + 32) of list Din (up to `cap` sub-steps, then
// append to Dout; with Dout.count == nullptr the particles run to the end).
__device__ __forceinline__ void push_more_warp(const MeshView& M, const ParticleStore& P, const SpeciesDev& S,
                                               const PushParams& pp, const DeferList& Din, const DeferList& Dout,
                                               int cap, ChargeAcc A, LedgerDev* L, int64_t base, int64_t n,
                                               PushStats& c)
{
    const bool chain = Dout.count != nullptr;
    const int64_t e = base + (threadIdx.x & 31);
    int st = -1;
    FlightF f;
    int64_t i = 0;
    if (e < n) {
        i = Din.idx[e];
        f.cur = P.tet[i];
        mix_load(P, i, f.rx, f.ry, f.rz, f.vx, f.vy, f.vz);
        f.it = Din.it[e];
        f.rem = (float)Din.rem[e];
        f.vstart = (float)Din.vstart[e];
        st = kDone;
        if (f.cur < 0) {
            // no location hint (only a stay-first pass 1 defers these): locate the absolute position
            const double px = f.rx, py = f.ry, pz = f.rz;
            const int t = locate_far(M, px, py, pz, -1);
            if (t < 0) {
                st = kLost;
            } else {
                const double3 o = origin(M, t);
                f.rx = (float)(px - o.x); f.ry = (float)(py - o.y); f.rz = (float)(pz - o.z);
                f.cur = t;
            }
        }
        if (st != kLost) st = advance_f(M, S, pp, f, chain ? cap : 0x7fffffff, A, c.nsub);
    }
    unsigned slot = chain ? warp_append(st == kCapped, Dout.count) : 0xffffffffu;
    if (st == kCapped && chain && slot < Dout.cap) {
        defer_store_f(P, Dout, slot, i, f);
    } else if (st >= 0) {
        if (st == kCapped) st = advance_f(M, S, pp, f, 0x7fffffff, A, c.nsub);
        finish_f(M, P, S, pp, L, i, f, st, c);
    }
    warp_chunk_end(c);
}

// Pass 1: every stored particle.  Warps take runs of kRun 32-particle chunks from the launch's
// work counter until none are left, so no warp idles while another still has work.
// 5 blocks of 256 per SM (48 registers): with the record's vector loads and the folded re-sort
// gather, the fewer spills now pay more than the sixth block's warps (push per step at 128^3:
// 5 blocks 35.97 ms, 6 blocks 36.92, 4 blocks 40.2; the walk inlined: 36.11 at 6 blocks,
// 37.56 at 5).
__global__ void __launch_bounds__(256, 5) k_push_mixed(const __grid_constant__ MeshView M, ParticleStore P,
                                                    const __grid_constant__ SortedSource R,
                                                    const __grid_constant__ SpeciesDev S,
                                                    const __grid_constant__ PushParams pp, DeferList D, ChargeAcc A,
                                                    LedgerDev* L, unsigned long long* ke_acc, unsigned* ctr)
{
    const int64_t n = *P.count;
    PushStats c{0.0, 0u, 0u};
    warp_stats_begin();
    for (;;) {
        const int64_t b0 = (int64_t)next_chunk(ctr) * (32 * kRun);
        if (b0 >= n) break;
        for (int64_t base = b0; base < b0 + 32 * kRun && base < n; base += 32)
            push1_warp(M, P, R, S, pp, D, A, L, base, n, c);
    }
    warp_stats_flush(L, ke_acc, S.vmax);
}

// Stay-first pass 1 (same work distribution as k_push_mixed); no walk code, so at 4 blocks of
// 256 per SM it fits in 62 registers without spilling.  Its launch is bound by L1 wavefronts
// (scattered record loads, one atomic per lane and node), so the spills of a denser launch cost
// more than its extra warps gain: 4 blocks 37.66 ms of push per step at 128^3, 5 blocks
// 38.5, 6 blocks (40 registers, 200 bytes of spill stores) 38.83.
__global__ void __launch_bounds__(256, 4) k_push_mixed_stay(const __grid_constant__ MeshView M, ParticleStore P,
                                                         const __grid_constant__ SortedSource R,
                                                         const __grid_constant__ SpeciesDev S,
                                                         const __grid_constant__ PushParams pp, DeferList D,
                                                         ChargeAcc A, LedgerDev* L, unsigned long long* ke_acc,
                                                         unsigned* ctr)
{
    const int64_t n = *P.count;
    PushStats c{0.0, 0u, 0u};
    warp_stats_begin();
    for (;;) {
        const int64_t b0 = (int64_t)next_chunk(ctr) * (32 * kRun);
        if (b0 >= n) break;
        for (int64_t base = b0; base < b0 + 32 * kRun && base < n; base += 32)
            push1_stay_warp(M, P, R, S, pp, D, A, L, base, n, c);
    }
    warp_stats_flush(L, ke_acc, S.vmax);
}

// Passes 2 and 3, 4 blocks of 256 per SM (64 registers; push per step at 128^3: 4 blocks 36.32
// ms, 3 blocks 36.46, 5 blocks 36.55).
__global__ void __launch_bounds__(256, 4) k_push_mixed_more(const __grid_constant__ MeshView M, ParticleStore P,
                                                         const __grid_constant__ SpeciesDev S,
                                                         const __grid_constant__ PushParams pp, DeferList Din,
                                                         DeferList Dout, int cap, ChargeAcc A, LedgerDev* L,
                                                         unsigned long long* ke_acc, unsigned* ctr)
{
    const int64_t n = (int64_t)min(*Din.count, Din.cap);
    PushStats c{0.0, 0u, 0u};
    warp_stats_begin();
    for (;;) {
        const int64_t base = (int64_t)next_chunk(ctr) * 32;
        if (base >= n) break;
        push_more_warp(M, P, S, pp, Din, Dout, cap, A, L, base, n, c);
    }
    warp_stats_flush(L, ke_acc, S.vmax);
}

// ---- batched step: all (scenario, species) jobs in one launch per pass -----------------
__global__ void k_batch_prefix(const PushJob* __restrict__ jobs, int njobs, int pass, int64_t* __restrict__ pre,
                               unsigned* __restrict__ ctr)
{
    __shared__ int64_t cnt[kMaxBatchJobs];
    for (int j = threadIdx.x; j < njobs; j += blockDim.x) {
        const PushJob& J = jobs[j];
        int64_t n;
        if (pass == 1)
            n = *J.P.count;
        else if (pass == 2)
            n = min((int64_t)*J.D1.count, (int64_t)J.D1.cap);
        else
            n = min((int64_t)*J.D2.count, (int64_t)J.D2.cap);
        const int64_t unit = pass == 1 ? 32 * kRun : 32;  // particles per counter value
        cnt[j] = (n + unit - 1) / unit;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t a = 0;
        for (int j = 0; j < njobs; ++j) {
            pre[j] = a;
            a += cnt[j];
        }
        pre[njobs] = a;
        ctr[pass - 1] = 0u;
    }
}

// Pass `pass` (1, 2 or 3) of every job.  Warps take units g of the global index from the pass's
// work counter (pass 1: runs of kRun 32-particle chunks; passes 2 and 3: single chunks); unit g
// belongs to the job j with pre[j] <= g < pre[j + 1], and a warp flushes its statistics into a
// job's ledger when it moves on to another job.
template <int PASS>
__global__ void __launch_bounds__(256, 4) k_push_mixed_batch(const PushJob* __restrict__ jobs, int njobs,
                                                          const int64_t* __restrict__ pre, unsigned* __restrict__ ctr)
{
    __shared__ int64_t spre[kMaxBatchJobs + 1];
    for (int j = threadIdx.x; j <= njobs; j += blockDim.x) spre[j] = pre[j];
    __syncthreads();
    const int64_t total = spre[njobs];
    PushStats c{0.0, 0u, 0u};
    warp_stats_begin();
    int cur = -1;
    for (;;) {
        const int64_t g = (int64_t)next_chunk(ctr + PASS - 1);
        if (g >= total) break;
        int lo = 0, hi = njobs;  // spre[lo] <= g < spre[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (spre[mid] <= g)
                lo = mid;
            else
                hi = mid;
        }
        if (lo != cur) {
            if (cur >= 0) warp_stats_flush(jobs[cur].L, jobs[cur].ke_acc, jobs[cur].S.vmax);
            cur = lo;
        }
        const PushJob& J = jobs[cur];
        if (PASS == 1) {
            const int64_t n = *J.P.count, b0 = (g - spre[cur]) * (32 * kRun);
            for (int64_t base = b0; base < b0 + 32 * kRun && base < n; base += 32)
                push1_warp(J.M, J.P, SortedSource{}, J.S, J.pp, J.D1, J.A, J.L, base, n, c);
            continue;
        }
        const int64_t base = (g - spre[cur]) * 32;
        if (PASS == 2) {
            const int64_t n = min((int64_t)*J.D1.count, (int64_t)J.D1.cap);
            push_more_warp(J.M, J.P, J.S, J.pp, J.D1, J.D2, kCap2, J.A, J.L, base, n, c);
        } else {
            const int64_t n = min((int64_t)*J.D2.count, (int64_t)J.D2.cap);
            push_more_warp(J.M, J.P, J.S, J.pp, J.D2, DeferList{}, 0, J.A, J.L, base, n, c);
        }
    }
    if (cur >= 0) warp_stats_flush(jobs[cur].L, jobs[cur].ke_acc, jobs[cur].S.vmax);
}

// nodal E -> tet records of every scenario (tets block map)
__global__ void k_batch_refresh_trec(const FieldJob* __restrict__ jobs, BlockMap m)
{
    const int k = m.ctx_of[blockIdx.x];
    const unsigned lb = blockIdx.x - m.first[k], nb = m.first[k + 1] - m.first[k];
    const FieldJob& J = jobs[k];
    for (int64_t g = lb * (int64_t)blockDim.x + threadIdx.x; g < 4 * J.T; g += (int64_t)nb * blockDim.x)
        refresh_trec_part(g >> 2, (int)(g & 3), J.tet, J.E, J.trec);
}

__global__ void k_mcc_mixed(ParticleStore P, SpeciesDev S, PushParams pp, LedgerDev* L)
{
    const int64_t n = *P.count;
    unsigned long long nhit = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (P.tet[i] <= kTetAbsorbed) continue;
        float rx, ry, rz, ux, uy, uz;
        mix_load(P, i, rx, ry, rz, ux, uy, uz);
        double vx = ux, vy = uy, vz = uz;
        if (mcc_elastic(S, pp, P.id[i], vx, vy, vz)) {
            mix_store(P, i, rx, ry, rz, (float)vx, (float)vy, (float)vz);
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
            mix_store(P, i, (float)(x[i] - o.x), (float)(y[i] - o.y), (float)(z[i] - o.z), (float)vx[i], (float)vy[i],
                      (float)vz[i]);
        } else {
            mix_store(P, i, (float)x[i], (float)y[i], (float)z[i], (float)vx[i], (float)vy[i], (float)vz[i]);
        }
        P.tet[i] = t >= 0 ? t : kTetNoHint;
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
        float rx, ry, rz, ux, uy, uz;
        mix_load(P, i, rx, ry, rz, ux, uy, uz);
        x[i] = ox + (double)rx; y[i] = oy + (double)ry; z[i] = oz + (double)rz;
        vx[i] = ux; vy[i] = uy; vz[i] = uz;
    }
}

// Refresh the nodal-E words of every tet record from the FP64 nodal field.
__global__ void k_refresh_trec(int64_t T, const int4* __restrict__ tet, const double* __restrict__ E, float* trec)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < 4 * T; g += (int64_t)gridDim.x * blockDim.x)
        refresh_trec_part(g >> 2, (int)(g & 3), tet, E, trec);
}

void launch_push_mixed(const MeshView& M, const ParticleStore& P, const SortedSource& R, const SpeciesDev& S,
                       const PushParams& pp, const DeferList& D1, const DeferList& D2, ChargeAcc A, LedgerDev* L,
                       unsigned long long* ke_acc, unsigned* ctr, int grid, bool stay_first, cudaStream_t st)
{
    if (stay_first)
        k_push_mixed_stay<<<grid, 256, 0, st>>>(M, P, R, S, pp, D1, A, L, ke_acc, ctr);
    else
        k_push_mixed<<<grid, 256, 0, st>>>(M, P, R, S, pp, D1, A, L, ke_acc, ctr);
    k_push_mixed_more<<<grid, 256, 0, st>>>(M, P, S, pp, D1, D2, kCap2, A, L, ke_acc, ctr + 1);
    DeferList none{};
    k_push_mixed_more<<<grid, 256, 0, st>>>(M, P, S, pp, D2, none, 0, A, L, ke_acc, ctr + 2);
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

void launch_batch_prefix(const PushJob* jobs, int njobs, int pass, int64_t* chunk_prefix, unsigned* ctr,
                         cudaStream_t st)
{
    k_batch_prefix<<<1, 1024, 0, st>>>(jobs, njobs, pass, chunk_prefix, ctr);
}

void launch_push_mixed_batch(const PushJob* jobs, int njobs, const int64_t* chunk_prefix, unsigned* ctr, int pass,
                             int grid, cudaStream_t st)
{
    if (pass == 1)
        k_push_mixed_batch<1><<<grid, 256, 0, st>>>(jobs, njobs, chunk_prefix, ctr);
    else if (pass == 2)
        k_push_mixed_batch<2><<<grid, 256, 0, st>>>(jobs, njobs, chunk_prefix, ctr);
    else
        k_push_mixed_batch<3><<<grid, 256, 0, st>>>(jobs, njobs, chunk_prefix, ctr);
}

void launch_batch_refresh_trec(const FieldJob* jobs, const BlockMap& tets, cudaStream_t st)
{
    k_batch_refresh_trec<<<tets.blocks, 256, 0, st>>>(jobs, tets);
}

void launch_refresh_trec(int64_t T, const int4* tet, const double* E, float* trec, cudaStream_t st)
{
    k_refresh_trec<<<148 * 8, 256, 0, st>>>(T, tet, E, trec);
}

}  // namespace scdat
