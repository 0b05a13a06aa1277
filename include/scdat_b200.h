/*
 * scdat_b200.h -- C ABI of the B200 PIC-MCC step and its per-step Poisson solve.
 *
 * Plain pointers and sizes only; every call returns SCDAT_OK (0) or a negative
 * scdat_status, and scdat_last_error() gives a one-line reason.  No exception crosses
 * the ABI.  Host arrays are read or written synchronously unless the name says "async".
 *
 * Each entry point cites the reference interface it replaces (paths inside the SCDAT
 * tree).  The reference keeps this state in PICCycle (Tools/PICcore/include/PICCycle.h),
 * its helpers CrossTetrahedron / FieldInterpolator / ChargeDepositor
 * (Tools/Particle/include/PICParticleAlgorithms.h), PoissonSolver
 * (Tools/FieldSolver/include/PoissonSolver.h) and the background MCC handler
 * (Tools/Interactions/Collisions/include/CollisionAlgorithm.h, CollisionPicAdapter.h).
 */
#ifndef SCDAT_B200_H
#define SCDAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCDAT_API __attribute__((visibility("default")))

typedef enum {
    SCDAT_OK = 0,
    SCDAT_ERR_ARG = -1,        /* bad argument (null pointer, out-of-range index, size)   */
    SCDAT_ERR_CUDA = -2,       /* a CUDA call failed; scdat_last_error() has the message   */
    SCDAT_ERR_STATE = -3,      /* call out of order (e.g. step before species are set)      */
    SCDAT_ERR_CAPACITY = -4,   /* particle capacity exceeded                                */
    SCDAT_ERR_NOT_CONVERGED = -5, /* field solve hit its iteration cap (result kept)       */
    SCDAT_ERR_DEVICE_FLAG = -6 /* a kernel reported an error through the device flag word   */
} scdat_status;

typedef enum { SCDAT_PREC_FP64 = 0, SCDAT_PREC_MIXED = 1 } scdat_precision;

/* Preconditioner of the field solve's CG (scdat_set_field_preconditioner). */
typedef enum { SCDAT_PRECOND_JACOBI = 0, SCDAT_PRECOND_MULTIGRID = 1 } scdat_preconditioner;

/* TrajectoryChargeDepositionKernel, Tools/Particle/include/PICParticleAlgorithms.h:32-37 */
typedef enum { SCDAT_DEP_NEAREST = 0, SCDAT_DEP_LINEAR = 1, SCDAT_DEP_GAUSS3 = 2 } scdat_deposit_kernel;

/* Particle boundary condition per box face, PICCycle::setBoundaryCondition
 * (PICCycle.h:68) with AbsorbingBoundaryCondition(1.0) / PeriodicBoundaryCondition
 * (Tools/Boundary/include/BoundaryConditions.h). */
typedef enum { SCDAT_BC_NONE = 0, SCDAT_BC_ABSORB = 1, SCDAT_BC_PERIODIC = 2 } scdat_face_bc;

/* Particle status as stored on the device (ParticleStatus ACTIVE/ABSORBED/ESCAPED,
 * Tools/Particle/include/ParticleDefinitions.h:161-176). */
typedef enum { SCDAT_ACTIVE = 0, SCDAT_ABSORBED = 1, SCDAT_ESCAPED = 2 } scdat_particle_status;

/* Mesh: nodes and 4-node tets, as VolMesh::addNode/addElement build them
 * (Tools/Mesh/include/MeshParsing.h:152-155).  tet_neighbors (nullable) is the per-tet
 * neighbour list Element::addNeighbor fills (MeshAlgorithms.h:193): the tet across the face
 * opposite local vertex f, -1 on the boundary.  When NULL the library derives it.
 * node_dirichlet marks Mesh::BoundaryType::DIRICHLET nodes.  tet_eps_rel (nullable): relative
 * permittivity per tet (PoissonSolver.cpp:21-29,655-662; NULL = vacuum everywhere). */
typedef struct {
    int64_t n_nodes;
    int64_t n_tets;
    const double* node_xyz;        /* [n_nodes*3] */
    const int32_t* tet_nodes;      /* [n_tets*4] */
    const int32_t* tet_neighbors;  /* [n_tets*4] or NULL */
    const uint8_t* node_dirichlet; /* [n_nodes] 1 = Dirichlet */
    const double* tet_eps_rel;     /* [n_tets] or NULL */
} scdat_mesh_desc;

/* PICCycle::Parameters (PICCycle.h:46-58) plus the device-side choices. */
typedef struct {
    double dt;                    /* time_step [s] */
    int32_t deposit_kernel;       /* scdat_deposit_kernel, default LINEAR */
    int32_t deposit_segments;     /* trajectory_charge_deposition_segments, default 10 */
    double adaptive_floor_ratio;  /* PIC_ADAPTIVE_FLOOR_RATIO, default 0.001 */
    int32_t precision;            /* scdat_precision */
    int32_t use_neighbor_lists;   /* 1: locate tries the hint's neighbour list first */
    int32_t face_bc[6];           /* scdat_face_bc per XMin,XMax,YMin,YMax,ZMin,ZMax */
    int32_t body_tally;           /* 1: particles lost into an interior hole go to ledger row 6 */
    int32_t poisson_charge_sign;  /* -1: b = -rho*V/4 as PoissonSolver.cpp:356; +1: physical */
    double pcg_rtol;              /* relative residual target of the field solve */
    int32_t pcg_max_iter;         /* iteration cap per solve */
    int32_t sort_interval;        /* re-sort particles by tet every N steps (0 = never) */
    int64_t particle_capacity;    /* total device particle slots over all species */
    uint64_t seed;                /* Philox key for MCC */
} scdat_params;

/* One species: charge [C], mass [kg], macro weight, and whether it is electron-like for the
 * ledger (PICCycle.cpp:52-85). */
typedef struct {
    double charge;
    double mass;
    double weight;
    int32_t electron_like;
    int32_t pad;
} scdat_species;

/* Elastic background collision for one species: ElasticCollisionCrossSection
 * (Tools/Interactions/Collisions/src/CollisonTypes.cpp:60-78) against a neutral background.
 * mode 0: the reference two-draw test (CollisionAlgorithm.cpp:525-531 then :195-200);
 * mode 1: one draw against 1-exp(-nu*dt);
 * mode 2: null collision: with nu_max = n * sigma_max * vmax, where vmax is the species'
 * largest speed at the end of the previous push, every particle no faster than vmax is
 * selected with probability 1-exp(-nu_max*dt) by a cheap counter-based draw and then collides
 * with probability nu/nu_max; faster particles (and all of them before the first push) take
 * mode 1's draw.  The collision law is mode 1's to first order in nu*dt, and most particles
 * skip the Philox draws. */
typedef struct {
    double target_density;  /* m^-3 */
    double sigma_max;       /* m^2 */
    double e_ref_ev;        /* reference_energy */
    double alpha;           /* power_index (0 = constant cross-section) */
    double e_threshold_ev;
    int32_t enabled;
    int32_t mode;
} scdat_elastic;

/* PICCycle::CycleStatistics (PICCycle.h:135-144) plus device counters. */
typedef struct {
    int64_t completed_steps;
    double simulation_time;
    double total_charge;             /* computeTotalCharge, PICParticleAlgorithms.cpp:440-448 */
    double total_energy;             /* updateStatistics, PICCycle.cpp:941-966 */
    int64_t active_particles;        /* active particles after the step */
    int64_t stored_particles;        /* particles held (active + not yet compacted) */
    double surface_deposited_charge; /* PICCycle.cpp:1271 */
    int64_t substeps;                /* CrossTetrahedron::Statistics::total_crossings */
    int64_t lost_events;
    int64_t mcc_collisions;
    int32_t last_pcg_iterations;
    int32_t pad;
    double last_pcg_relres;
} scdat_stats;

typedef struct scdat_ctx scdat_ctx;

/* Defaults for scdat_params (dt must still be set). */
SCDAT_API void scdat_default_params(scdat_params* p);

/* PICCycle::setMesh + initialize (PICCycle.h:64-75, PICCycle.cpp:227-309) and the
 * PoissonSolver assembly (PoissonSolver.cpp:251-385): uploads the mesh, precomputes tet
 * geometry, the locate grid, the node graph and the Dirichlet-reduced matrix. */
SCDAT_API int scdat_create(const scdat_mesh_desc* mesh, const scdat_params* params, scdat_ctx** out);
SCDAT_API int scdat_destroy(scdat_ctx* ctx);
/* One-line reason of the context's last failed call.  With ctx NULL: the reason of the calling
 * thread's last failed scdat_create (whose context no longer exists), or "null context". */
SCDAT_API const char* scdat_last_error(const scdat_ctx* ctx);

/* ParticleManager species (ParticleFactory::createElectron/createIon,
 * Tools/Particle/src/ParticleDefinitions.cpp:374-392).  Call once before particles. */
SCDAT_API int scdat_set_species(scdat_ctx* ctx, int32_t n_species, const scdat_species* sp);

/* ParticleContainer::addParticles (ParticleManager.h:77) for one species.  tet_hint
 * (nullable) seeds PICCycle::addParticleLocation (PICCycle.h:71); ids (nullable) key the
 * MCC random streams (default: running index).  Replaces the species' particles. */
SCDAT_API int scdat_set_particles(scdat_ctx* ctx, int32_t species, int64_t n, const double* x, const double* v,
                                  const int32_t* tet_hint, const uint32_t* ids);

/* Device-side seeding of a Kuhn box built by scdat_kuhn_box_mesh with the same dimensions:
 * n_per_cell particles of the species in every meshed hex cell, uniform positions and a
 * Maxwellian of temperature temp_ev, from Philox(seed) keyed by the particle id
 * (cell*n_species + species)*n_per_cell + k.  Replaces the species' particles. */
SCDAT_API int scdat_seed_box_particles(scdat_ctx* ctx, int32_t species, int32_t nx, int32_t ny, int32_t nz,
                                       double h, const int32_t* body_lo, const int32_t* body_hi,
                                       int32_t n_per_cell, double temp_ev, uint64_t seed);

/* Builds the 6-tet Kuhn box the benchmark configurations use (the reference box mesher makes
 * a non-conforming 5-tet split, Tools/Mesh/src/MeshParsing.cpp:1209-1260, so this replaces it
 * for those inputs): nx*ny*nz hex cells of edge h from the origin, node id
 * i + (nx+1)*(j + (ny+1)*k), hex cells x-fastest minus the half-open body index range
 * [body_lo, body_hi) (both NULL: no body), 6 tets per cell.  Outer-face nodes are Dirichlet
 * at `wall`, body nodes at `bias`.  Call with NULL output arrays to get the sizes. */
SCDAT_API int scdat_kuhn_box_mesh(int32_t nx, int32_t ny, int32_t nz, double h, const int32_t* body_lo,
                                  const int32_t* body_hi, double bias, double wall, int64_t* n_nodes, int64_t* n_tets,
                                  double* node_xyz, int32_t* tet_nodes, uint8_t* node_dirichlet, double* node_phi,
                                  int32_t* hex_ijk, int64_t* n_cells);

/* ParticleSource-style injection on any tet mesh: n_per_tet particles of the species in each
 * of the n_tets listed tets (tets == NULL and n_tets == 0: every tet), positions uniform in the
 * tet from Dirichlet(1,1,1,1) weights e_k / sum e, e_k = -log(max(1e-12, u_k)) as
 * samplePointInTetra (Toolkit/Surface Charging/src/PicMccSurfaceCurrentSampler.cpp:270-287),
 * velocities a Maxwellian of temp_ev plus drift[3] (nullable); Philox(seed) keyed by the id
 * (tet_index * n_species + species) * n_per_tet + k.  Replaces the species' particles. */
SCDAT_API int scdat_seed_tet_particles(scdat_ctx* ctx, int32_t species, int64_t n_tets, const int32_t* tets,
                                       int32_t n_per_tet, double temp_ev, const double* drift, uint64_t seed);

/* Result files in the reference's columnar CSV layout (ResultExporter / CSVExporter,
 * Tools/Output/src/CSVExporter.cpp:11-47: header "axis,series..." with the series in name order,
 * one row per axis value, %.8e).  The layer profile is the PIC-MCC driver's output
 * (Main/main_PICcore.cpp:312-334): n_layers equal z slabs with the mean potential and E_z of
 * their nodes, electron and ion densities and the electron temperature (m <v^2> / 3e). */
SCDAT_API int scdat_export_layer_profile_csv(scdat_ctx* ctx, const char* path, int32_t n_layers);
/* Every node: position, potential, charge and field. */
SCDAT_API int scdat_export_nodes_csv(scdat_ctx* ctx, const char* path);
/* CSVExporter::exportDataSet (Tools/Output/src/CSVExporter.cpp:11-47) on a columnar data set:
 * n_rows axis values and n_series named series of n_rows values each, written in series-name
 * order (the reference's std::map), the parent directory created first.  Host code only: needs
 * no context and no GPU; the two exports above write through it. */
SCDAT_API int scdat_export_columns_csv(const char* path, const char* axis_name, int64_t n_rows, const double* axis,
                                       int32_t n_series, const char* const* names, const double* const* values);

/* ParticleContainer iteration (ParticleManager.h:113-126): copy one species back. */
SCDAT_API int scdat_get_particle_count(scdat_ctx* ctx, int32_t species, int64_t* n);
SCDAT_API int scdat_get_particles(scdat_ctx* ctx, int32_t species, int64_t capacity, double* x, double* v,
                                  int32_t* tet, uint8_t* status, uint32_t* ids, int64_t* n_out);

/* PICCycle::setPotential (PICCycle.h:105-120): node potentials (Dirichlet values included)
 * and the nodal LSQ field recomputed with the 1e-18 regularisation (PICCycle.cpp:180-220). */
SCDAT_API int scdat_set_potential(scdat_ctx* ctx, const double* phi);
/* PICCycle::setNodePotential (PICCycle.h:122-133) for a batch of nodes. */
SCDAT_API int scdat_set_node_potentials(scdat_ctx* ctx, int64_t n, const int64_t* nodes, const double* values);
/* FieldInterpolator::setElectricField (PICParticleAlgorithms.h:92): freeze a nodal E. */
SCDAT_API int scdat_set_electric_field(scdat_ctx* ctx, const double* E);

/* PoissonSolver::setChargeDensity (Tools/FieldSolver/include/PoissonSolver.h:41-43): nodal
 * charge [C] for the next scdat_solve_field.  The next scdat_push or scdat_step replaces it
 * with the deposited charge. */
SCDAT_API int scdat_set_charge_density(scdat_ctx* ctx, const double* rho);
/* PICCycle::setTimeStep (PICCycle.h:92-98). */
SCDAT_API int scdat_set_dt(scdat_ctx* ctx, double dt);
/* MonteCarloCollisionHandler(seed) (CollisionAlgorithm.h:176): the Philox key of the MCC
 * streams from the next step on. */
SCDAT_API int scdat_set_seed(scdat_ctx* ctx, uint64_t seed);

/* Surface circuit of the body (the surface-charging caller's dielectric faces, no PICCycle
 * counterpart): each face XMin..ZMax of the body box [body_lo, body_hi] is a circuit node with
 * capacitance eps0*eps_r*A/d (Toolkit/Surface Charging/src/DensePlasmaSurfaceCharging.cpp:6544-6552;
 * A = the face's area when area[f] is 0), a shunt conductance to ground and a linearised plasma
 * current.  Each scdat_step collects the charge of the particles lost into the body per face,
 * advances the face potentials with the implicit node update of
 * SurfaceCircuitCoupling::advanceImplicit (Tools/Coupling/src/SurfaceCircuitCoupling.cpp:953-966)
 * in FP64, and gives the body's surface nodes the mean potential of their faces before the field
 * solve.  Turns on body_tally. */
typedef struct {
    double body_lo[3], body_hi[3];
    double eps_r[6];       /* relative permittivity of each face's dielectric */
    double thickness[6];   /* m */
    double area[6];        /* m^2; 0 = from the box */
    double v0[6];          /* initial potential, V */
    double shunt_s[6];     /* conductance to ground, S (0 = floating) */
    double didv[6];        /* plasma current linearisation dI/dV, A/V (0 = plain charge integration) */
} scdat_surface_circuit;
SCDAT_API int scdat_set_surface_circuit(scdat_ctx* ctx, const scdat_surface_circuit* sc);
/* Secondary emission of electrons collected by the body (needs the surface circuit):
 * model 1 is Sternglass's universal yield 7.4 dmax (E/Emax) exp(-2 sqrt(E/Emax)); models 2, 3
 * and 4 the reference's legacy yields as evaluateLegacySecondaryElectronYield computes them
 * (Tools/Material/src/SurfaceMaterialModel.cpp:619-637): 2 legacyWhippleYield (:231-244),
 * 3 legacySimsYield (:246-273), 4 legacyKatzYield (:275-302); 0 off.
 * The emitted charge delta |q| w of each collected electron returns to its face as current and
 * is recorded in ledger row 6 as emitted electron charge (no secondary macro-particles are
 * created). */
SCDAT_API int scdat_set_secondary_emission(scdat_ctx* ctx, int32_t model, double delta_max, double e_max_ev);
/* The shape parameters of the legacy yields: the Sims exponent n (the reference's default 1.6;
 * values below 1.05 act as 1.05, as in the reference) and the Katz range coefficients
 * {r1, n1, r2, n2} (NULL: the reference's defaults {0.85, 0.35, 0.12, 1.05}, the material
 * scalars katz_r1, katz_n1, katz_r2, katz_n2). */
SCDAT_API int scdat_set_secondary_yield_params(scdat_ctx* ctx, double sims_exponent_n, const double* katz);
/* Face potentials [6], collected charge [6], last-step current [6] and the number of particles
 * collected so far [6]; any pointer may be NULL. */
SCDAT_API int scdat_get_surface_state(scdat_ctx* ctx, double* V, double* Q, double* I, int64_t* counts);

/* MonteCarloCollisionHandler::addCollisionProcess (CollisionAlgorithm.h:176-226) for one
 * species; executed once per step after the push, like executeBackgroundMccStep
 * (CollisionPicAdapter.cpp:338-434). */
SCDAT_API int scdat_set_elastic_mcc(scdat_ctx* ctx, int32_t species, const scdat_elastic* proc);

/* PICCycle::executeTimeStep (PICCycle.cpp:311-416) followed by the background MCC step and
 * removal of inactive particles, n_steps times, all on the device. */
SCDAT_API int scdat_step(scdat_ctx* ctx, int32_t n_steps);

/* Stages, for parity tests and callers that drive the cycle themselves:
 *   scdat_push          -- ChargeDepositor::clearChargeDensity + pushParticles + boundary events
 *                          (PICCycle.cpp:331, 466-629, 1331-1379) with the current field
 *   scdat_solve_field   -- solvePoissonEquation + updateElectricField (PICCycle.cpp:645-894)
 *   scdat_collide       -- executeBackgroundMccStep (CollisionPicAdapter.cpp:338-434)
 *   scdat_compact       -- ParticleContainer::removeInactiveParticles (ParticleManager.cpp:157-177) */
SCDAT_API int scdat_push(scdat_ctx* ctx);
SCDAT_API int scdat_solve_field(scdat_ctx* ctx);
SCDAT_API int scdat_collide(scdat_ctx* ctx);
SCDAT_API int scdat_compact(scdat_ctx* ctx);

/* Re-sort one species only every `interval` steps instead of every params.sort_interval steps
 * (no reference counterpart: the reference does not sort).  A species that crosses few tets
 * per step (ions beside electrons of the same temperature move ~43x slower) stays ordered for
 * many steps, so sorting it at the electrons' rate costs time and buys nothing.  interval must
 * be a positive multiple of params.sort_interval, or 0 to follow it. */
SCDAT_API int scdat_set_species_sort_interval(scdat_ctx* ctx, int32_t species, int32_t interval);

/* Pass-1 form of one species' push in the precision form (no reference counterpart; the
 * reference pushes particle by particle).  WALKING: pass 1 gives every particle one sub-step
 * with the full relocation walk.  STAY_FIRST: pass 1 carries no walk code and completes only
 * sub-steps that end in the particle's own tet; the others go to the walking passes, which
 * redo that sub-step with the same arithmetic, so both forms give bitwise the same result.
 * STAY_FIRST is faster for a species that rarely leaves its tet (ions beside electrons of the
 * same temperature).  AUTO (default) probes STAY_FIRST every 32 pushes and keeps it while it
 * defers under a fifth of the species.  The plain FP64 form ignores the setting. */
typedef enum { SCDAT_PUSH_AUTO = 0, SCDAT_PUSH_WALKING = 1, SCDAT_PUSH_STAY_FIRST = 2 } scdat_push_mode;
SCDAT_API int scdat_set_species_push_mode(scdat_ctx* ctx, int32_t species, int32_t mode);

/* Preconditioner of the field solve (the reference's CG is Jacobi-preconditioned,
 * Tools/Solver/include/ConjugateGradientCommon.h:74-161, which stays the default).
 * SCDAT_PRECOND_MULTIGRID builds, on the first call, a lattice multigrid hierarchy for meshes
 * whose nodes lie on a regular lattice (e.g. scdat_kuhn_box_mesh): trilinear prolongation,
 * Galerkin coarse operators P^T A P, damped-Jacobi smoothing (two sweeps before and after), a
 * dense inverse on the coarsest level (at most 1024 rows), one V-cycle per CG iteration.  It
 * preconditions the FP64 CG of the plain form and the FP32 inner CG of the precision form;
 * the convergence test (||r|| <= rtol ||b||, in FP64 for the precision form) is unchanged, so
 * only the iteration count differs.  Returns SCDAT_ERR_ARG (scdat_last_error says why) when
 * the mesh has no such hierarchy.  The batched step keeps Jacobi-PCG. */
SCDAT_API int scdat_set_field_preconditioner(scdat_ctx* ctx, int32_t kind);
/* Sizes of the field solver's levels (for bandwidth accounting): *levels (1 for Jacobi), and
 * for each of the first max_levels: rows, off-diagonal nonzeros of the operator (the dense
 * coarsest level reports rows^2) and nonzeros of the prolongation to the next level (0 on the
 * last).  Any output array may be NULL. */
SCDAT_API int scdat_get_field_solver_levels(scdat_ctx* ctx, int32_t max_levels, int32_t* levels, int64_t* rows,
                                            int64_t* nnz, int64_t* transfer_nnz);

/* PICCycle::getChargeDensity/getPotential/getElectricField (PICCycle.h:79-90); any pointer
 * may be NULL.  rho is nodal charge [C]; E is [n_nodes*3]. */
SCDAT_API int scdat_get_fields(scdat_ctx* ctx, double* rho, double* phi, double* E);
/* Per-species nodal charge of the last deposit (no reference counterpart: the reference only
 * keeps the sum). */
SCDAT_API int scdat_get_species_charge(scdat_ctx* ctx, int32_t species, double* rho_s);
/* PICCycle::getSurfaceCurrentLedger (PICCycle.h:175-178): 7 rows (XMin..ZMax, interior body)
 * x 8 columns: absorbed e charge, absorbed ion charge, emitted e charge, incident energy,
 * absorbed e count, absorbed ion count, emitted e count, 0.  Cumulative since create/reset. */
SCDAT_API int scdat_get_ledger(scdat_ctx* ctx, double* ledger);
SCDAT_API int scdat_reset_ledger(scdat_ctx* ctx);
/* PICCycle::getStatistics (PICCycle.h:165-168). */
SCDAT_API int scdat_get_statistics(scdat_ctx* ctx, scdat_stats* st);

/* ---- Batched scenarios (no reference counterpart: the reference runs one PICCycle at a
 * time) ----
 * A batch advances many independent contexts (each with its own mesh, species, particles and
 * potentials, all created with SCDAT_PREC_MIXED) together: every push pass is one launch over
 * all (scenario, species) pairs, the field solve one launch per kernel over all scenarios with
 * per-scenario convergence, and the whole step is captured once as a CUDA graph whose solver
 * loops are conditional nodes.  The contexts stay valid for every query (scdat_get_*); step
 * them only through the batch while it exists. */
typedef struct scdat_batch scdat_batch;
typedef struct {
    int32_t push_blocks_per_sm;   /* grid of the push launches, in blocks of 256 per SM (default 4) */
    int32_t field_blocks_per_sm;  /* blocks per SM shared among the scenarios in the field launches (8) */
    int32_t use_graph;            /* 1: one CUDA-graph launch per step; 0: host-driven loops */
    int32_t pad;
} scdat_batch_tuning;

SCDAT_API void scdat_batch_default_tuning(scdat_batch_tuning* t);
/* On failure *out still holds the batch so that scdat_batch_last_error can be read; destroy it. */
SCDAT_API int scdat_batch_create(int32_t n, scdat_ctx* const* ctxs, scdat_batch** out);
SCDAT_API int scdat_batch_destroy(scdat_batch* b);
SCDAT_API const char* scdat_batch_last_error(const scdat_batch* b);
SCDAT_API int scdat_batch_step(scdat_batch* b, int32_t n_steps);
SCDAT_API int scdat_batch_set_tuning(scdat_batch* b, const scdat_batch_tuning* t);
SCDAT_API int scdat_batch_get_tuning(const scdat_batch* b, scdat_batch_tuning* t);
/* Times each candidate launch shape on steps_each real steps and keeps the fastest. */
SCDAT_API int scdat_batch_autotune(scdat_batch* b, int32_t steps_each, scdat_batch_tuning* chosen);
/* Device time per step of the last run of steps (CUDA events on the batch stream). */
SCDAT_API int scdat_batch_last_step_ms(const scdat_batch* b, double* ms);
/* The CUDA stream the batch steps on (a cudaStream_t). */
SCDAT_API int scdat_batch_stream(const scdat_batch* b, void** stream);
/* Kernels of this library the batch's steps have launched so far. */
SCDAT_API int scdat_batch_kernel_launches(scdat_batch* b, int64_t* launches);

/* PicMccSurfaceCurrentSampler::sampleWithDerivative (Toolkit/Surface Charging/src/
 * PicMccSurfaceCurrentSampler.cpp:641-670): three contexts holding the same scenario (mesh,
 * species, particles, seed) run window_steps steps with the surface nodes held at V - d, V and
 * V + d, d = max(0.1, |probe_delta_v|) as in the reference, as one batch when all three are
 * mixed-precision (one at a time otherwise).  The collected charge is that of ledger row
 * `ledger_row`: 0..5 a domain face XMin..ZMax (the reference samples its plate's ZMin face,
 * PicMccSurfaceCurrentSampler.cpp:587-588), 6 the body box.  Returns the centre window's
 * collection current densities (charge per second per area into the surface: electrons
 * negative, ions positive, secondaries leaving positive) and the central difference of the net
 * density over 2d. */
typedef struct {
    double surface_potential_v;
    double electron_collection_a_per_m2;
    double ion_collection_a_per_m2;
    double emitted_electron_a_per_m2;
    double net_collection_a_per_m2;
    double current_derivative_a_per_m2_per_v;
    int32_t valid;
    int32_t window_steps;
} scdat_current_sample;
SCDAT_API int scdat_sample_with_derivative(scdat_ctx* const* ctx3, int64_t n_surface, const int64_t* surface_nodes,
                                           int32_t ledger_row, double surface_potential_v, double probe_delta_v,
                                           int32_t window_steps, double area_m2, scdat_current_sample* out);

/* ---- Adjoint window (no reference counterpart) ----
 * Runs `steps` FP64 steps from the current state (which must follow a scdat_solve_field; MCC
 * off, segment-cloud or nearest-point deposit) with states checkpointed every `checkpoint`
 * steps, then the hand-written reverse pass, and returns
 *     J = g_phi . phi_T + g_V . V_T + g_Q . Q_T
 * (final potential; surface-circuit face potentials and collected charge) with its pathwise
 * derivatives in the body bias (the Dirichlet value of bias_nodes, or the faces' initial
 * potential when the surface circuit is on), the electron temperature the particles were
 * seeded at (velocities scale with sqrt(Te)) and the secondary-yield peak.  The discrete
 * choices of the forward run (tets, sub-step expressions, deposit points inside the post-move
 * tet, collections) are held fixed, so a finite difference with frozen random streams agrees
 * while it flips none of them.  The context ends at step T, as after scdat_step(steps). */
typedef struct {
    int32_t steps;
    int32_t checkpoint;          /* default 10 */
    const double* g_phi;         /* [n_nodes] or NULL */
    double g_V[6];
    double g_Q[6];
    const int64_t* bias_nodes;   /* nodes held at the bias (no surface circuit) */
    int64_t n_bias_nodes;
    double te_ev;                /* electron temperature of the seeded velocities (0: skip dJ/dTe) */
} scdat_adjoint_request;
typedef struct {
    double J;
    double dJ_dbias;
    double dJ_dte;
    double dJ_ddelta_max;
    int64_t flags;  /* 1: a particle's sub-steps overflowed the replay tape, 2: replay mismatch */
} scdat_adjoint_result;
SCDAT_API int scdat_adjoint_window(scdat_ctx* ctx, const scdat_adjoint_request* rq, scdat_adjoint_result* res);

/* The CUDA stream every call of this context runs on (a cudaStream_t), for callers that
 * order their own work or events against the library.  No reference counterpart. */
SCDAT_API void* scdat_stream(scdat_ctx* ctx);

/* Per-stage device timing with CUDA events on the context stream (no reference counterpart;
 * the reference keeps wall-clock stage shares under PIC_PROFILE_CYCLE, PICCycle.cpp:316-408).
 * scdat_set_timing(1) clears the counters and starts recording; scdat_get_timing returns the
 * summed device milliseconds of the particle push launches (all species of a step count as
 * one launch) and of the field solves since then, and how many kernels of this library were
 * launched. */
SCDAT_API int scdat_set_timing(scdat_ctx* ctx, int32_t enable);
SCDAT_API int scdat_get_timing(scdat_ctx* ctx, double* push_ms, int64_t* push_launches, int64_t* push_particles,
                               double* field_ms, int64_t* field_solves, int64_t* kernel_launches);
/* The same for the re-sorts by tet (key build, radix sort, gather of the store) since
 * scdat_set_timing(1): summed device milliseconds and the number of species sorted. */
SCDAT_API int scdat_get_sort_timing(scdat_ctx* ctx, double* sort_ms, int64_t* sorts);

/* LinearSystem::solve(ITERATIVE) (Tools/Solver/src/LinearSystem.cpp:84-87,258-327) without a
 * context: Jacobi-preconditioned CG on a caller-assembled SPD system whose arrays all live in
 * device memory.  Row r holds its off-diagonal entries in col/val[row_ptr[r]..row_ptr[r+1]) and
 * its diagonal in diag[r]; x is the start vector on entry and the solution on return; the
 * solve stops when ||r|| <= rtol*||b|| or after max_iter iterations (SCDAT_ERR_NOT_CONVERGED,
 * x kept).  stream is a cudaStream_t (NULL: the default stream); the call blocks until the
 * solve ends.  Scratch device memory (6 vectors of R doubles) is allocated and freed inside. */
SCDAT_API int scdat_pcg_csr(int32_t R, const int32_t* row_ptr, const int32_t* col, const double* val,
                            const double* diag, const double* b, double* x, double rtol, int32_t max_iter,
                            void* stream, int32_t* iterations, double* relres);

/* scdat_pcg_csr for callers that cannot allocate device memory (no counterpart in the
 * reference).  Some callers may not call cudaMalloc at all -- a host application that owns a
 * fixed device-memory arena and hands the library only pointers into it, or code running
 * where the allocator is unavailable -- so this call allocates nothing: its scratch lives in
 * one static device array of 12.6 MB that every GPU loading the library keeps until exit.
 * Limit: R <= 262144 rows; larger systems return SCDAT_ERR_CAPACITY before any GPU work.
 * The first call on each device looks up the array's device address (cudaGetSymbolAddress,
 * with that device current); make that first call before any stream capture.  All calls
 * share the one array, so calls that overlap on the GPU (other streams, other threads) race:
 * serialise them.  The looked-up address is kept for the life of the process: do not reset the
 * device (cudaDeviceReset) or otherwise recreate its primary context after the first call.
 * Arguments, results and blocking behaviour are those of scdat_pcg_csr. */
SCDAT_API int scdat_pcg_csr_noalloc(int32_t R, const int32_t* row_ptr, const int32_t* col, const double* val,
                                    const double* diag, const double* b, double* x, double rtol, int32_t max_iter,
                                    void* stream, int32_t* iterations, double* relres);

/* Library version string. */
SCDAT_API const char* scdat_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SCDAT_B200_H */
