/*
 * scdat_oracle.c -- CPU restatement of the SCDAT PIC-MCC step (TEST INFRASTRUCTURE).
 *
 * This file is the parity oracle for the B200 kernels.  It restates, in plain C99,
 * the reference's algorithm for one PIC-MCC step on a tetrahedral mesh:
 *   gather + adaptive Boris + relocation + trajectory deposit
 *       Tools/Particle/src/PICParticleAlgorithms.cpp:107-296, 325-448, 536-939
 *   runtime boundary events and the 6-face surface ledger
 *       Tools/PICcore/src/PICCycle.cpp:1074-1379, Tools/Boundary/src/BoundaryConditions.cpp:55-140,347-392
 *   edge-weight Poisson assembly, Dirichlet elimination and the nodal LSQ field
 *       Tools/FieldSolver/src/PoissonSolver.cpp:18-37,274-385,474-529,749-787
 *       Tools/Solver/src/LinearSystem.cpp:37-58
 *   background MCC (elastic, reference two-draw form)
 *       Tools/Interactions/Collisions/src/CollisionAlgorithm.cpp:70-76,108-125,189-210,500-538,700-704
 *       Tools/Interactions/Collisions/src/CollisonTypes.cpp:60-78
 *
 * Only the test-suite, the smoke check and the CPU-baseline leg of the benchmark load
 * this code, and only as the checker.  The product path never calls it.
 *
 * Parity pin: the restatement is checked against the reference classes themselves,
 * compiled from the reference sources by oracle/Makefile into oracle/_ref/, on small
 * meshes (see tests/test_oracle_vs_reference.py and the fixtures in tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written from the paper.  */
/* ------------------------------------------------------------------------- */
ORC_API void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Two uniforms in (0,1) with 53-bit resolution from one Philox block. */
static void orc_uniform2(uint64_t seed, uint64_t id, uint32_t step, uint32_t purpose, double u[2])
{
    uint32_t ctr[4] = {(uint32_t)id, (uint32_t)(id >> 32), step, purpose};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    for (int k = 0; k < 2; ++k) {
        uint64_t m = ((uint64_t)o[2 * k] << 21) ^ (uint64_t)(o[2 * k + 1] >> 11);
        m &= ((uint64_t)1 << 53) - 1;
        u[k] = ((double)m + 0.5) * (1.0 / 9007199254740992.0);
    }
}

ORC_API void orc_uniforms(uint64_t seed, uint64_t id, uint32_t step, uint32_t purpose, double* u2)
{
    orc_uniform2(seed, id, step, purpose, u2);
}

/* ------------------------------------------------------------------------- */
/* Geometry                                                                    */
/* ------------------------------------------------------------------------- */
typedef struct {
    double x, y, z;
} v3;

static inline v3 v3sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline double v3dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 v3cross(v3 a, v3 b)
{
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline double v3mag(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 node_pos(const double* xyz, int64_t n) { v3 r = {xyz[3 * n], xyz[3 * n + 1], xyz[3 * n + 2]}; return r; }

/* Signed volume x6, PICParticleAlgorithms.cpp:261-268 (v1.dot(v2.cross(v3))). */
static inline double sv6(v3 a, v3 b, v3 c, v3 d)
{
    return v3dot(v3sub(b, a), v3cross(v3sub(c, a), v3sub(d, a)));
}

/* FieldInterpolator::isPointInTetrahedron, volume branch, PICParticleAlgorithms.cpp:247-296.
 * Returns 1 when every barycentric lies in [-1e-8, 1+1e-8]. */
static int orc_bary(const double* xyz, const int32_t* tet4, int64_t t, v3 p, double lam[4])
{
    const int32_t* tn = tet4 + 4 * t;
    v3 a = node_pos(xyz, tn[0]), b = node_pos(xyz, tn[1]), c = node_pos(xyz, tn[2]), d = node_pos(xyz, tn[3]);
    double V6 = sv6(a, b, c, d);
    if (fabs(V6) < 1e-15) return 0;
    lam[0] = sv6(p, b, c, d) / V6;
    lam[1] = sv6(a, p, c, d) / V6;
    lam[2] = sv6(a, b, p, d) / V6;
    lam[3] = sv6(a, b, c, p) / V6;
    const double eps = 1e-8;
    for (int i = 0; i < 4; ++i)
        if (lam[i] < -eps || lam[i] > 1.0 + eps) return 0;
    return 1;
}

ORC_API int orc_barycentric(const double* xyz, const int32_t* tet4, int64_t t, const double* p, double* lam)
{
    v3 q = {p[0], p[1], p[2]};
    return orc_bary(xyz, tet4, t, q, lam);
}

/* Scan accelerator for the linear scan below (an exact stand-in, not a different rule).
 * Uniform bins over the mesh's bounding box; each bin lists, in ascending id order, every tet
 * whose bounding box -- widened by 1e-6 of its diagonal, far more than the 1e-8 barycentric
 * tolerance lets a containing point lie outside the tet -- overlaps the bin.  Every tet that
 * contains a point p is therefore listed in p's bin, so the first containing tet of that
 * list is the lowest-id containing tet, which is what the linear scan returns.  A point
 * outside every widened box is in no tet.  Bin indices of boxes and points come from the same
 * monotone expression, so a point on a bin face finds the tets listed for its bin.  Used only
 * while orc_grid_use() has selected a grid built for the same tet array. */
typedef struct {
    const int32_t* tet4;
    int64_t T;
    double lo[3], hi[3], inv[3];
    int n[3];
    int64_t* start; /* [bins+1] */
    int32_t* ids;
} orc_grid;

static const orc_grid* g_locate_grid = NULL;

static int grid_axis_bin(const orc_grid* g, int a, double x)
{
    int b = (int)floor((x - g->lo[a]) * g->inv[a]);
    return b < 0 ? 0 : (b >= g->n[a] ? g->n[a] - 1 : b);
}

static void tet_box(const double* xyz, const int32_t* tn, double lo[3], double hi[3])
{
    for (int a = 0; a < 3; ++a) {
        lo[a] = hi[a] = xyz[3 * tn[0] + a];
        for (int k = 1; k < 4; ++k) {
            double v = xyz[3 * tn[k] + a];
            if (v < lo[a]) lo[a] = v;
            if (v > hi[a]) hi[a] = v;
        }
    }
    double d = sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                    (hi[2] - lo[2]) * (hi[2] - lo[2]));
    for (int a = 0; a < 3; ++a) {
        lo[a] -= 1e-6 * d;
        hi[a] += 1e-6 * d;
    }
}

ORC_API void* orc_grid_create(const double* xyz, const int32_t* tet4, int64_t T)
{
    if (T <= 0) return NULL;
    orc_grid* g = (orc_grid*)calloc(1, sizeof(orc_grid));
    g->tet4 = tet4;
    g->T = T;
    for (int64_t t = 0; t < T; ++t) {
        double lo[3], hi[3];
        tet_box(xyz, tet4 + 4 * t, lo, hi);
        for (int a = 0; a < 3; ++a) {
            if (t == 0 || lo[a] < g->lo[a]) g->lo[a] = lo[a];
            if (t == 0 || hi[a] > g->hi[a]) g->hi[a] = hi[a];
        }
    }
    /* about two tets per bin */
    double ext[3], vol = 1.0;
    for (int a = 0; a < 3; ++a) {
        ext[a] = g->hi[a] - g->lo[a];
        if (ext[a] <= 0.0) ext[a] = 1.0;
        vol *= ext[a];
    }
    double cell = cbrt(vol / ((double)T / 2.0 + 1.0));
    int64_t bins = 1;
    for (int a = 0; a < 3; ++a) {
        int n = (int)ceil(ext[a] / cell);
        g->n[a] = n < 1 ? 1 : (n > 1024 ? 1024 : n);
        g->inv[a] = (double)g->n[a] / ext[a];
        bins *= g->n[a];
    }
    g->start = (int64_t*)calloc((size_t)bins + 1, sizeof(int64_t));
    for (int pass = 0; pass < 2; ++pass) {
        int64_t* fill = NULL;
        if (pass == 1) {
            for (int64_t b = 0; b < bins; ++b) g->start[b + 1] += g->start[b];
            g->ids = (int32_t*)malloc(sizeof(int32_t) * (size_t)(g->start[bins] > 0 ? g->start[bins] : 1));
            fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)bins);
            memcpy(fill, g->start, sizeof(int64_t) * (size_t)bins);
        }
        for (int64_t t = 0; t < T; ++t) { /* ascending t: each bin's list is sorted */
            double lo[3], hi[3];
            tet_box(xyz, tet4 + 4 * t, lo, hi);
            int b0[3], b1[3];
            for (int a = 0; a < 3; ++a) {
                b0[a] = grid_axis_bin(g, a, lo[a]);
                b1[a] = grid_axis_bin(g, a, hi[a]);
            }
            for (int k = b0[2]; k <= b1[2]; ++k)
                for (int j = b0[1]; j <= b1[1]; ++j)
                    for (int i = b0[0]; i <= b1[0]; ++i) {
                        int64_t b = i + (int64_t)g->n[0] * (j + (int64_t)g->n[1] * k);
                        if (pass == 0)
                            g->start[b + 1] += 1;
                        else
                            g->ids[fill[b]++] = (int32_t)t;
                    }
        }
        free(fill);
    }
    return g;
}

ORC_API void orc_grid_destroy(void* h)
{
    orc_grid* g = (orc_grid*)h;
    if (!g) return;
    if (g_locate_grid == g) g_locate_grid = NULL;
    free(g->start);
    free(g->ids);
    free(g);
}

/* Select the grid the scan uses (NULL: the plain linear scan). */
ORC_API void orc_grid_use(void* h) { g_locate_grid = (const orc_grid*)h; }

/* The lowest-id tet containing p: the linear scan of locateParticle, or its exact stand-in. */
static int64_t orc_scan(const double* xyz, const int32_t* tet4, int64_t T, v3 p)
{
    double lam[4];
    const orc_grid* g = g_locate_grid;
    if (g && g->tet4 == tet4 && g->T == T) {
        const double c[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; ++a)
            if (!(c[a] >= g->lo[a] && c[a] <= g->hi[a])) return -1;
        int64_t b = grid_axis_bin(g, 0, c[0]) +
                    (int64_t)g->n[0] * (grid_axis_bin(g, 1, c[1]) + (int64_t)g->n[1] * grid_axis_bin(g, 2, c[2]));
        for (int64_t e = g->start[b]; e < g->start[b + 1]; ++e)
            if (orc_bary(xyz, tet4, g->ids[e], p, lam)) return g->ids[e];
        return -1;
    }
    for (int64_t t = 0; t < T; ++t)
        if (orc_bary(xyz, tet4, t, p, lam)) return t;
    return -1;
}

/* CrossTetrahedron::locateParticle, PICParticleAlgorithms.cpp:853-891: the hint, then the
 * hint's neighbour list in order (nbr4 row, -1 entries skipped; nbr4 == NULL means the
 * lists are empty, as the reference ships), then the lowest-id tet of a linear scan. */
static int64_t orc_locate(const double* xyz, const int32_t* tet4, const int32_t* nbr4, int64_t T,
                          v3 p, int64_t hint)
{
    double lam[4];
    if (hint >= 0 && hint < T) {
        if (orc_bary(xyz, tet4, hint, p, lam)) return hint;
        if (nbr4) {
            for (int f = 0; f < 4; ++f) {
                int32_t nb = nbr4[4 * hint + f];
                if (nb >= 0 && orc_bary(xyz, tet4, nb, p, lam)) return nb;
            }
        }
    }
    return orc_scan(xyz, tet4, T, p);
}

ORC_API int64_t orc_locate_point(const double* xyz, const int32_t* tet4, const int32_t* nbr4, int64_t T,
                                 const double* p, int64_t hint)
{
    v3 q = {p[0], p[1], p[2]};
    return orc_locate(xyz, tet4, nbr4, T, q, hint);
}

/* ------------------------------------------------------------------------- */
/* Push: gather + adaptive Boris + relocation + deposit                        */
/* ------------------------------------------------------------------------- */
enum { ORC_ACTIVE = 0, ORC_ABSORBED = 1, ORC_ESCAPED = 2 };
/* TrajectoryChargeDepositionKernel numbering, PICParticleAlgorithms.h:32-37 */
enum { ORC_DEP_NEAREST = 0, ORC_DEP_LINEAR = 1, ORC_DEP_GAUSS3 = 2 };

typedef struct {
    double dt;
    double floor_ratio;   /* PIC_ADAPTIVE_FLOOR_RATIO, default 0.001 (PICParticleAlgorithms.cpp:788-797) */
    int32_t nseg;         /* trajectory deposition segments (PICCycle.h:55) */
    int32_t dep_kernel;   /* ORC_DEP_* */
    int32_t deposit;      /* 0: no charge deposit */
    int32_t pad;
} orc_push_params;

typedef struct {
    int64_t substeps;     /* CrossTetrahedron::Statistics::total_crossings */
    int64_t lost;         /* particles whose trajectory ended lost */
    int64_t max_iter_hit; /* particles that hit the 100000 sub-step cap */
    int64_t pad;
} orc_push_stats;

/* FieldInterpolator::interpolateVectorField, PICParticleAlgorithms.cpp:150-181. */
static v3 orc_gather(const double* xyz, const int32_t* tet4, int64_t t, v3 p, const double* Fn)
{
    v3 r = {0, 0, 0};
    double lam[4];
    if (!orc_bary(xyz, tet4, t, p, lam)) return r;
    for (int i = 0; i < 4; ++i) {
        int64_t n = tet4[4 * t + i];
        r.x = r.x + Fn[3 * n] * lam[i];
        r.y = r.y + Fn[3 * n + 1] * lam[i];
        r.z = r.z + Fn[3 * n + 2] * lam[i];
    }
    return r;
}

/* ChargeDepositor::depositCharge, PICParticleAlgorithms.cpp:325-369. */
static void orc_deposit_point(const double* xyz, const int32_t* tet4, int64_t t, v3 p, double charge,
                              double weight, double* rho)
{
    double lam[4];
    if (!orc_bary(xyz, tet4, t, p, lam)) return;
    for (int i = 0; i < 4; ++i) rho[tet4[4 * t + i]] += (charge * weight) * lam[i];
}

/* ChargeDepositor::depositChargeAlongTrajectory, PICParticleAlgorithms.cpp:371-433. */
static void orc_deposit_traj(const double* xyz, const int32_t* tet4, int64_t t, v3 s, v3 e, double charge,
                             double weight, const orc_push_params* pp, double* rho)
{
    v3 tr = v3sub(e, s);
    if (v3mag(tr) < 1e-15) {
        orc_deposit_point(xyz, tet4, t, s, charge, weight, rho);
        return;
    }
    if (pp->dep_kernel == ORC_DEP_NEAREST) {
        orc_deposit_point(xyz, tet4, t, e, charge, weight, rho);
        return;
    }
    int nseg = pp->nseg < 1 ? 1 : (pp->nseg > 128 ? 128 : pp->nseg);
    if (pp->dep_kernel == ORC_DEP_GAUSS3) {
        const double gn[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};
        const double gw[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
        for (int sgi = 0; sgi < nseg; ++sgi) {
            double t0 = (double)sgi / (double)nseg, t1 = (double)(sgi + 1) / (double)nseg;
            double tc = 0.5 * (t0 + t1), th = 0.5 * (t1 - t0);
            for (int q = 0; q < 3; ++q) {
                double tt = tc + th * gn[q];
                v3 sp = {s.x + tr.x * tt, s.y + tr.y * tt, s.z + tr.z * tt};
                orc_deposit_point(xyz, tet4, t, sp, charge * gw[q] / (double)nseg, weight, rho);
            }
        }
        return;
    }
    double cps = charge / (double)nseg;
    for (int sgi = 0; sgi < nseg; ++sgi) {
        double tt = ((double)sgi + 0.5) / (double)nseg;
        v3 sp = {s.x + tr.x * tt, s.y + tr.y * tt, s.z + tr.z * tt};
        orc_deposit_point(xyz, tet4, t, sp, cps, weight, rho);
    }
}

/* CrossTetrahedron::adaptiveTimeStep, PICParticleAlgorithms.cpp:750-801 (B == 0 on this path). */
static double orc_adaptive_dt(double qm, double vmag_start, v3 E, double dt_max, double floor_ratio)
{
    double dt = dt_max;
    double Em = v3mag(E);
    if (Em > 1e-10) {
        double acc = Em * fabs(qm);
        if (acc > 1e-10 && vmag_start > 1.0) {
            double dtv = 0.1 * vmag_start / acc;
            dt = dt < dtv ? dt : dtv;
        }
    }
    double fl = dt_max * floor_ratio;
    dt = dt > fl ? dt : fl;
    dt = dt < dt_max ? dt : dt_max;
    return dt;
}

/* CrossTetrahedron::borisIntegration with |B| == 0, PICParticleAlgorithms.cpp:803-851. */
static v3 orc_boris_e(v3 v, v3 E, double qm, double dt)
{
    double hdt = 0.5 * dt;
    double f = qm * hdt;
    v3 vm = {v.x + E.x * f, v.y + E.y * f, v.z + E.z * f};
    v3 vp = {vm.x + E.x * f, vm.y + E.y * f, vm.z + E.z * f};
    return vp;
}

ORC_API void orc_boris(const double* v, const double* E, double qm, double dt, double* out)
{
    v3 vv = {v[0], v[1], v[2]}, EE = {E[0], E[1], E[2]};
    v3 r = orc_boris_e(vv, EE, qm, dt);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

/*
 * CrossTetrahedron::integrateTrajectory, PICParticleAlgorithms.cpp:536-740, for every
 * active particle.  x, v: [P*3] in/out.  tet: [P] in = hint (-1 none), out = final tet.
 * lost: [P] out (1 when the trajectory ended lost).  rho accumulates nodal charge [C].
 * Species tables q, m, w are indexed by species[P].
 */
ORC_API int orc_push(int64_t N, const double* xyz, int64_t T, const int32_t* tet4, const int32_t* nbr4,
                     const double* Enode, int64_t P, double* x, double* v, const int32_t* species,
                     int32_t* tet, const uint8_t* status, uint8_t* lost, const double* sq, const double* sm,
                     const double* sw, const orc_push_params* pp, double* rho, orc_push_stats* st)
{
    (void)N;
    for (int64_t ip = 0; ip < P; ++ip) {
        lost[ip] = 0;
        if (status[ip] != ORC_ACTIVE) continue;
        int s = species[ip];
        double q = sq[s], m = sm[s], w = sw[s];
        double qm = q / m;
        v3 pos = {x[3 * ip], x[3 * ip + 1], x[3 * ip + 2]};
        v3 vel = {v[3 * ip], v[3 * ip + 1], v[3 * ip + 2]};
        const double vstart = v3mag(vel); /* particle->getVelocity() stays at the step-start value */
        int64_t cur = orc_locate(xyz, tet4, nbr4, T, pos, tet[ip]);
        if (cur < 0) {
            lost[ip] = 1;
            tet[ip] = 0; /* result.final_element = 0 when the start is outside (:543,:577) */
            st->lost++;
            continue;
        }
        double remaining = pp->dt;
        int it = 0;
        int is_lost = 0;
        double lam[4];
        while (remaining > 1e-20 && it < 100000) {
            it++;
            v3 E = orc_gather(xyz, tet4, cur, pos, Enode);
            double adt = orc_adaptive_dt(qm, vstart, E, remaining, pp->floor_ratio);
            v3 start = pos;
            if (fabs(qm) > 1e-20) vel = orc_boris_e(vel, E, qm, adt);
            pos.x = pos.x + vel.x * adt;
            pos.y = pos.y + vel.y * adt;
            pos.z = pos.z + vel.z * adt;
            if (!orc_bary(xyz, tet4, cur, pos, lam)) {
                /* dichotomyBoundaryIntersection (:893-939) only gates the branch: the start
                 * point is always inside `cur`, so the relocation below always runs. */
                int64_t nt = orc_locate(xyz, tet4, nbr4, T, pos, cur);
                if (nt >= 0) {
                    cur = nt;
                } else {
                    is_lost = 1;
                    break;
                }
            }
            if (pp->deposit) orc_deposit_traj(xyz, tet4, cur, start, pos, q, w, pp, rho);
            remaining -= adt;
            st->substeps++;
        }
        if (it >= 100000) {
            is_lost = 1;
            st->max_iter_hit++;
        }
        if (is_lost) st->lost++;
        x[3 * ip] = pos.x; x[3 * ip + 1] = pos.y; x[3 * ip + 2] = pos.z;
        v[3 * ip] = vel.x; v[3 * ip + 1] = vel.y; v[3 * ip + 2] = vel.z;
        tet[ip] = (int32_t)cur;
        lost[ip] = (uint8_t)is_lost;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Runtime boundary events and the surface ledger                              */
/* ------------------------------------------------------------------------- */
enum { ORC_BC_NONE = 0, ORC_BC_ABSORB = 1, ORC_BC_PERIODIC = 2 };

/* Ledger row layout (7 rows: XMin..ZMax, then the interior body), PICCycle.h:153-163:
 * [0] absorbed_electron_charge_c [1] absorbed_ion_charge_c [2] emitted_electron_charge_c
 * [3] incident_energy_j [4] absorbed_electron_particles [5] absorbed_ion_particles
 * [6] emitted_electron_particles [7] unused */
#define ORC_LEDGER_W 8

typedef struct {
    double bmin[3], bmax[3];  /* domain bounds, PICCycle.cpp:1039-1066 */
    int32_t face_bc[6];       /* ORC_BC_* per face */
    double period[3];         /* periodic length per axis (0 = not periodic), BoundaryConditions.cpp:93-140 */
    int32_t body_tally;       /* 1: tally particles lost to an interior hole in ledger row 6 */
    int32_t pad;
} orc_bc_params;

static int orc_detect_face(const orc_bc_params* b, v3 p, double otol, int near, double ntol)
{
    if (p.x < b->bmin[0] - otol) return 0;
    if (p.x > b->bmax[0] + otol) return 1;
    if (p.y < b->bmin[1] - otol) return 2;
    if (p.y > b->bmax[1] + otol) return 3;
    if (p.z < b->bmin[2] - otol) return 4;
    if (p.z > b->bmax[2] + otol) return 5;
    if (!near) return -1;
    int best = -1;
    double bd = 1.79769313486231570815e+308;
    double d[6] = {fabs(p.x - b->bmin[0]), fabs(p.x - b->bmax[0]), fabs(p.y - b->bmin[1]),
                   fabs(p.y - b->bmax[1]), fabs(p.z - b->bmin[2]), fabs(p.z - b->bmax[2])};
    for (int f = 0; f < 6; ++f)
        if (d[f] <= ntol && d[f] < bd) { best = f; bd = d[f]; }
    return best;
}

static int orc_is_electron_like(double q) { return q < 0.0; }
static int orc_is_ion_like(double q) { return q > 0.0; }

/*
 * PICCycle::processRuntimeBoundaryEvents / applyRuntimeBoundaryCondition /
 * recordSurfaceBoundaryInteraction, PICCycle.cpp:1221-1379, for every particle with lost[i].
 * status updated in place; tet updated to the resolved element; ledger [7*8] accumulated;
 * surface_charge accumulates q*w of absorbed particles (PICCycle.cpp:1271).
 */
ORC_API int orc_boundary(int64_t T, const double* xyz, const int32_t* tet4, const int32_t* nbr4, int64_t P,
                         double* x, const double* v, const int32_t* species, int32_t* tet, uint8_t* status,
                         const uint8_t* lost, const double* sq, const double* sm, const double* sw,
                         const orc_bc_params* b, double* ledger, double* surface_charge)
{
    double sx = fmax(b->bmax[0] - b->bmin[0], 1e-12), sy = fmax(b->bmax[1] - b->bmin[1], 1e-12),
           sz = fmax(b->bmax[2] - b->bmin[2], 1e-12);
    double ms = fmax(sx, fmax(sy, sz));
    double otol = fmax(1e-10, 1e-8 * ms);
    double ntol = fmax(5.0 * otol, 1e-9 * ms);
    for (int64_t ip = 0; ip < P; ++ip) {
        if (!lost[ip]) continue;
        if (status[ip] != ORC_ACTIVE) continue;
        int s = species[ip];
        double q = sq[s], m = sm[s], w = sw[s];
        v3 pos = {x[3 * ip], x[3 * ip + 1], x[3 * ip + 2]};
        v3 vel = {v[3 * ip], v[3 * ip + 1], v[3 * ip + 2]};
        double ke = 0.5 * m * (vel.x * vel.x + vel.y * vel.y + vel.z * vel.z);
        int64_t hint = tet[ip];
        int64_t resolved = -1;
        int ok = 0, done = 0;
        for (int pass = 0; pass < 6 && !done; ++pass) {
            if (status[ip] != ORC_ACTIVE) { ok = 1; done = 1; break; }
            int f = orc_detect_face(b, pos, otol, pass == 0, ntol);
            if (f < 0) {
                resolved = orc_locate(xyz, tet4, nbr4, T, pos, hint);
                ok = resolved >= 0;
                done = 1;
                break;
            }
            int bc = b->face_bc[f];
            if (bc == ORC_BC_NONE) { ok = 0; done = 1; break; }
            if (bc == ORC_BC_ABSORB) {
                status[ip] = ORC_ABSORBED;
            } else if (bc == ORC_BC_PERIODIC) {
                double c[3] = {pos.x, pos.y, pos.z};
                for (int a = 0; a < 3; ++a) {
                    double L = b->period[a];
                    if (L <= 1e-12) continue;
                    c[a] = fmod(c[a], L);
                    if (c[a] < 0.0) c[a] += L;
                }
                pos.x = c[0]; pos.y = c[1]; pos.z = c[2];
            }
            double* row = ledger + ORC_LEDGER_W * f;
            if (status[ip] == ORC_ABSORBED) {
                row[3] += ke * fmax(1.0, w);
                if (orc_is_electron_like(q)) { row[0] += q * w; row[4] += 1.0; }
                else if (orc_is_ion_like(q)) { row[1] += q * w; row[5] += 1.0; }
                *surface_charge += q * w;
                ok = 1; done = 1;
                break;
            }
            int64_t h2 = orc_locate(xyz, tet4, nbr4, T, pos, hint);
            hint = h2;
            if (h2 >= 0) resolved = h2;
        }
        if (!done) {
            if (status[ip] == ORC_ACTIVE) {
                resolved = orc_locate(xyz, tet4, nbr4, T, pos, hint);
                ok = resolved >= 0;
            } else {
                ok = 1;
            }
        }
        if (!ok) status[ip] = ORC_ESCAPED;
        if (status[ip] == ORC_ACTIVE) {
            if (resolved >= 0) tet[ip] = (int32_t)resolved;
            else status[ip] = ORC_ESCAPED;
        }
        if (status[ip] == ORC_ESCAPED && b->body_tally) {
            /* New capability (no reference counterpart): a particle lost inside the domain
             * bounds went into an interior hole (the conducting body); tally it there. */
            if (orc_detect_face(b, pos, otol, 0, 0.0) < 0) {
                double* row = ledger + ORC_LEDGER_W * 6;
                row[3] += ke * fmax(1.0, w);
                if (orc_is_electron_like(q)) { row[0] += q * w; row[4] += 1.0; }
                else if (orc_is_ion_like(q)) { row[1] += q * w; row[5] += 1.0; }
            }
        }
        x[3 * ip] = pos.x; x[3 * ip + 1] = pos.y; x[3 * ip + 2] = pos.z;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Poisson: edge-weight Laplacian, Dirichlet elimination, CG, nodal LSQ field  */
/* ------------------------------------------------------------------------- */
static const double ORC_EPS0 = 8.8541878128e-12; /* PoissonSolver.cpp:18 */

/* elementMeasure, PoissonSolver.cpp:31-38 with TetrahedronElement::getVolume, MeshAlgorithms.cpp:29-54 */
static double orc_tet_measure(const double* xyz, const int32_t* tn)
{
    v3 a = node_pos(xyz, tn[0]), b = node_pos(xyz, tn[1]), c = node_pos(xyz, tn[2]), d = node_pos(xyz, tn[3]);
    double ax = b.x - a.x, ay = b.y - a.y, az = b.z - a.z;
    double bx = c.x - a.x, by = c.y - a.y, bz = c.z - a.z;
    double cx = d.x - a.x, cy = d.y - a.y, cz = d.z - a.z;
    double det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
    double vol = fabs(det) / 6.0;
    return fmax(fabs(vol), 1e-12);
}

static int cmp64(const void* a, const void* b)
{
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

/*
 * Assemble the node graph in CSR (row i: sorted neighbour ids, diagonal excluded) and the
 * edge weights K_ij = -sum_e eps*(V_e/6)/d_ij^2 (PoissonSolver.cpp:274-329), the diagonal
 * K_ii = -sum_j K_ij, and the nodal control volume CV_i = sum_e V_e/4 (:331-359).
 * eps_tet[T] is the permittivity of each tet in F/m (NULL = vacuum).
 * Two-pass API: call with colind == NULL to get nnz in *nnz_out (rowptr filled), then again.
 */
ORC_API int orc_assemble(int64_t N, const double* xyz, int64_t T, const int32_t* tet4, const double* eps_tet,
                         int64_t* rowptr, int32_t* colind, double* offw, double* diag, double* cv,
                         int64_t* nnz_out)
{
    /* neighbour sets via a dense bitmap-free approach: collect (i,j) pairs, sort, unique */
    int64_t npairs = 12 * T;
    int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * (size_t)(npairs > 0 ? npairs : 1));
    int64_t k = 0;
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* tn = tet4 + 4 * t;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                if (i != j) keys[k++] = (int64_t)tn[i] * N + tn[j];
    }
    qsort(keys, (size_t)k, sizeof(int64_t), cmp64);
    int64_t u = 0;
    for (int64_t i = 0; i < k; ++i)
        if (u == 0 || keys[i] != keys[u - 1]) keys[u++] = keys[i];
    for (int64_t i = 0; i <= N; ++i) rowptr[i] = 0;
    for (int64_t i = 0; i < u; ++i) rowptr[keys[i] / N + 1]++;
    for (int64_t i = 0; i < N; ++i) rowptr[i + 1] += rowptr[i];
    *nnz_out = u;
    if (!colind) { free(keys); return 0; }
    for (int64_t i = 0; i < u; ++i) { colind[i] = (int32_t)(keys[i] % N); offw[i] = 0.0; }
    free(keys);
    for (int64_t i = 0; i < N; ++i) { diag[i] = 0.0; cv[i] = 0.0; }
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* tn = tet4 + 4 * t;
        double meas = orc_tet_measure(xyz, tn);
        double epsv = eps_tet ? eps_tet[t] : ORC_EPS0;
        double es = meas / 6.0;
        for (int i = 0; i < 4; ++i) {
            cv[tn[i]] += meas / 4.0;
            for (int j = i + 1; j < 4; ++j) {
                v3 pi = node_pos(xyz, tn[i]), pj = node_pos(xyz, tn[j]);
                double d = fmax(v3mag(v3sub(pi, pj)), 1e-12);
                double wgt = epsv * es / (d * d);
                diag[tn[i]] += wgt;
                diag[tn[j]] += wgt;
                /* find j in row i and i in row j */
                for (int64_t e = rowptr[tn[i]]; e < rowptr[tn[i] + 1]; ++e)
                    if (colind[e] == tn[j]) { offw[e] -= wgt; break; }
                for (int64_t e = rowptr[tn[j]]; e < rowptr[tn[j] + 1]; ++e)
                    if (colind[e] == tn[i]) { offw[e] -= wgt; break; }
            }
        }
    }
    return 0;
}


/*
 * Solve the Dirichlet-eliminated system (LinearSystem.cpp:37-58): for interior rows
 *   sum_{j interior} K_ij phi_j = -rho_i*CV_i - sum_{d Dirichlet} K_id phi_d,
 * Dirichlet rows keep phi.  charge_sign = -1 reproduces PoissonSolver.cpp:356 (b = -rho*V/4);
 * rho_scale multiplies rho before use (1 = reference units).  Jacobi-preconditioned CG from
 * the phi passed in, until ||r|| <= rtol*||b_interior|| or max_iter.  Returns iterations.
 */
ORC_API int orc_poisson_cg(int64_t N, const int64_t* rowptr, const int32_t* colind, const double* offw,
                           const double* diag, const double* cv, const uint8_t* dirichlet, const double* rho,
                           double charge_sign, double* phi, double rtol, int max_iter, double* final_rel)
{
    double* b = (double*)calloc((size_t)N, sizeof(double));
    double* r = (double*)calloc((size_t)N, sizeof(double));
    double* z = (double*)calloc((size_t)N, sizeof(double));
    double* p = (double*)calloc((size_t)N, sizeof(double));
    double* Ap = (double*)calloc((size_t)N, sizeof(double));
    double bn = 0.0;
    for (int64_t i = 0; i < N; ++i) {
        if (dirichlet[i]) continue;
        double bi = charge_sign * rho[i] * cv[i];
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
            if (dirichlet[colind[e]]) bi -= offw[e] * phi[colind[e]];
        b[i] = bi;
        bn += bi * bi;
    }
    bn = sqrt(bn);
    /* r = b - A phi */
    double rn = 0.0;
    for (int64_t i = 0; i < N; ++i) {
        if (dirichlet[i]) continue;
        double s = diag[i] * phi[i];
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
            if (!dirichlet[colind[e]]) s += offw[e] * phi[colind[e]];
        r[i] = b[i] - s;
        rn += r[i] * r[i];
    }
    rn = sqrt(rn);
    double thr = rtol * (bn > 0 ? bn : 1.0);
    int it = 0;
    if (rn > thr) {
        double rz = 0.0;
        for (int64_t i = 0; i < N; ++i) {
            if (dirichlet[i]) continue;
            z[i] = r[i] / diag[i];
            p[i] = z[i];
            rz += r[i] * z[i];
        }
        for (it = 1; it <= max_iter; ++it) {
            double pAp = 0.0;
            for (int64_t i = 0; i < N; ++i) {
                if (dirichlet[i]) continue;
                double s = diag[i] * p[i];
                for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
                    if (!dirichlet[colind[e]]) s += offw[e] * p[colind[e]];
                Ap[i] = s;
                pAp += p[i] * s;
            }
            if (pAp == 0.0) break;
            double alpha = rz / pAp;
            rn = 0.0;
            double rz2 = 0.0;
            for (int64_t i = 0; i < N; ++i) {
                if (dirichlet[i]) continue;
                phi[i] += alpha * p[i];
                r[i] -= alpha * Ap[i];
                z[i] = r[i] / diag[i];
                rn += r[i] * r[i];
                rz2 += r[i] * z[i];
            }
            rn = sqrt(rn);
            if (rn <= thr) break;
            double beta = rz2 / rz;
            rz = rz2;
            for (int64_t i = 0; i < N; ++i) {
                if (dirichlet[i]) continue;
                p[i] = z[i] + beta * p[i];
            }
        }
        if (it > max_iter) it = max_iter;
    }
    if (final_rel) *final_rel = rn / (bn > 0 ? bn : 1.0);
    free(b); free(r); free(z); free(p); free(Ap);
    return it;
}

/* solve3x3 with partial pivoting, PoissonSolver.cpp:124-172 */
static int orc_solve3(double M[3][3], double rhs[3], double sol[3])
{
    for (int piv = 0; piv < 3; ++piv) {
        int best = piv;
        for (int row = piv + 1; row < 3; ++row)
            if (fabs(M[row][piv]) > fabs(M[best][piv])) best = row;
        if (fabs(M[best][piv]) < 1.0e-18) return 0;
        if (best != piv) {
            for (int c = 0; c < 3; ++c) { double t = M[best][c]; M[best][c] = M[piv][c]; M[piv][c] = t; }
            double t = rhs[best]; rhs[best] = rhs[piv]; rhs[piv] = t;
        }
        for (int row = piv + 1; row < 3; ++row) {
            double f = M[row][piv] / M[piv][piv];
            for (int c = piv; c < 3; ++c) M[row][c] -= f * M[piv][c];
            rhs[row] -= f * rhs[piv];
        }
    }
    for (int row = 2; row >= 0; --row) {
        double s = rhs[row];
        for (int c = row + 1; c < 3; ++c) s -= M[row][c] * sol[c];
        sol[row] = s / M[row][row];
    }
    return 1;
}

/*
 * PoissonSolver::computeElectricFieldGradient + computeLeastSquaresGradient,
 * PoissonSolver.cpp:474-529, 749-787: E_i = -argmin sum_j (g.d_ij - dphi_ij)^2 over the
 * node graph.  reg adds to the normal-matrix diagonal (0 here; PICCycle.cpp:208 uses 1e-18).
 */
ORC_API int orc_lsq_efield(int64_t N, const double* xyz, const int64_t* rowptr, const int32_t* colind,
                           const double* phi, double reg, double* E)
{
    for (int64_t i = 0; i < N; ++i) {
        double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, rhs[3] = {0, 0, 0}, sol[3] = {0, 0, 0};
        int cnt = 0;
        v3 pi = node_pos(xyz, i);
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            int64_t j = colind[e];
            v3 d = v3sub(node_pos(xyz, j), pi);
            if (d.x * d.x + d.y * d.y + d.z * d.z <= 1e-24) continue;
            double dp = phi[j] - phi[i];
            M[0][0] += d.x * d.x; M[0][1] += d.x * d.y; M[0][2] += d.x * d.z;
            M[1][0] += d.y * d.x; M[1][1] += d.y * d.y; M[1][2] += d.y * d.z;
            M[2][0] += d.z * d.x; M[2][1] += d.z * d.y; M[2][2] += d.z * d.z;
            rhs[0] += d.x * dp; rhs[1] += d.y * dp; rhs[2] += d.z * dp;
            cnt++;
        }
        E[3 * i] = E[3 * i + 1] = E[3 * i + 2] = 0.0;
        if (!cnt) continue;
        M[0][0] += reg; M[1][1] += reg; M[2][2] += reg;
        if (!orc_solve3(M, rhs, sol)) continue;
        E[3 * i] = -sol[0]; E[3 * i + 1] = -sol[1]; E[3 * i + 2] = -sol[2];
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Background MCC                                                              */
/* ------------------------------------------------------------------------- */
static const double ORC_QE = 1.602176634e-19; /* Constants.h:46 */

/* One elastic process per species row: target density n, sigma_max, E_ref, alpha
 * (ElasticCollisionCrossSection, CollisonTypes.cpp:60-78).  mode 0 = reference two-draw
 * form (CollisionAlgorithm.cpp:525-531 then :195-200, effective probability p^2);
 * mode 1 = one draw against 1-exp(-nu*dt).  Streams: Philox(seed; id, step, purpose 2). */
typedef struct {
    double n_target, sigma_max, e_ref, alpha, e_threshold;
    int32_t enabled;
    int32_t pad;
} orc_elastic;

static double orc_sigma_elastic(const orc_elastic* pr, double e_ev)
{
    if (!(e_ev >= pr->e_threshold)) return 0.0;
    double eref = pr->e_ref > 1e-6 ? pr->e_ref : 1e-6;
    double s = pr->sigma_max * pow(eref / e_ev, pr->alpha);
    s = s < pr->sigma_max ? s : pr->sigma_max;
    return s > 0.0 ? s : 0.0;
}

/* splitmix64's output mix (Steele, Lea and Flood, OOPSLA 2014) and the null-collision
 * selection draw for (seed; id, step), as the device computes them. */
static uint64_t orc_mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return z;
}

static double orc_select_uniform(uint64_t seed, uint32_t id, uint32_t step)
{
    const uint64_t key = ((uint64_t)step << 32) | (uint64_t)id;
    const uint64_t z = orc_mix64(orc_mix64(seed ^ 0x5CDA7B2005CDA7B2ull) + key * 0x9E3779B97F4A7C15ull);
    return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

/* vmax (mode 2): per species, the largest speed of the previous push (0: none yet). */
ORC_API int64_t orc_mcc(int64_t P, double* v, const int32_t* species, const uint8_t* status, const int64_t* pid,
                        const double* sm, const orc_elastic* proc, double dt, uint64_t seed, uint32_t step,
                        int mode, const double* vmax)
{
    int64_t hits = 0;
    const double two_pi = 2.0 * 3.14159265358979323846;
    for (int64_t ip = 0; ip < P; ++ip) {
        if (status[ip] != ORC_ACTIVE) continue;
        const orc_elastic* pr = proc + species[ip];
        if (!pr->enabled) continue;
        double m = sm[species[ip]];
        v3 vel = {v[3 * ip], v[3 * ip + 1], v[3 * ip + 2]};
        const double v2 = vel.x * vel.x + vel.y * vel.y + vel.z * vel.z;
        double speed = sqrt(v2);
        double e_ev = 0.5 * m * speed * speed / ORC_QE;
        double nu = pr->n_target * orc_sigma_elastic(pr, e_ev) * speed;
        double u[2], u2[2];
        const double vm = (mode == 2 && vmax) ? vmax[species[ip]] : 0.0;
        int hit;
        if (mode == 2 && vm > 0.0 && v2 <= vm * vm) {
            /* null collision: selection with 1 - exp(-nu_max dt), then nu / nu_max */
            const double numax = pr->n_target * pr->sigma_max * vm;
            const double xmax = numax * dt;
            const double us = orc_select_uniform(seed, (uint32_t)pid[ip], step);
            if (us >= xmax + 1e-15 || !(us < 1.0 - exp(-xmax))) continue;
            orc_uniform2(seed, (uint64_t)pid[ip], step, 2u, u);
            hit = u[0] * numax < nu;
        } else if (mode == 2) {
            orc_uniform2(seed, (uint64_t)pid[ip], step, 2u, u);
            const double x = nu * dt;
            hit = !(u[0] >= x + 1e-15) && u[0] < 1.0 - exp(-x);
        } else if (mode == 0) {
            orc_uniform2(seed, (uint64_t)pid[ip], step, 2u, u);
            double p = nu * dt;
            p = p < 0.0 ? 0.0 : (p > 1.0 ? 1.0 : p);
            hit = (u[0] < p) && !(u[1] >= p);
        } else {
            orc_uniform2(seed, (uint64_t)pid[ip], step, 2u, u);
            double p = 1.0 - exp(-nu * dt);
            hit = u[0] < p;
        }
        if (!hit) continue;
        hits++;
        orc_uniform2(seed, (uint64_t)pid[ip], step, 3u, u2);
        double theta = acos(-1.0 + 2.0 * u2[0]);
        double phi = two_pi * u2[1];
        double st = sin(theta);
        v[3 * ip] = speed * st * cos(phi);
        v[3 * ip + 1] = speed * st * sin(phi);
        v[3 * ip + 2] = speed * cos(theta);
    }
    return hits;
}
