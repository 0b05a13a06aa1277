// ref_harness.cpp -- extern "C" driver of the reference SCDAT classes (TEST INFRASTRUCTURE).
//
// Compiled by oracle/Makefile together with the reference's own sources (read in place
// from the reference tree) into oracle/_ref/libscdat_ref.so.  It builds identical mesh and
// particle state from flat arrays and runs the reference code paths:
//   CrossTetrahedron::crossTetrahedron          Tools/Particle/include/PICParticleAlgorithms.h:216-219
//   PoissonSolver::solve(DIRECT)                Tools/FieldSolver/include/PoissonSolver.h:26-67
//   PICCycle::setPotential (nodal LSQ field)    Tools/PICcore/include/PICCycle.h:105-120
//   PICCycle::executeTimeStep                   Tools/PICcore/src/PICCycle.cpp:311-416
//   Collision::executeBackgroundMccStep         Tools/Interactions/Collisions/include/CollisionPicAdapter.h:64-75
//   SurfaceCircuitCoupling::advanceImplicit     Tools/Coupling/src/SurfaceCircuitCoupling.cpp:866-1126
//   evaluateLegacySecondaryElectronYield        Tools/Material/src/SurfaceMaterialModel.cpp:620-636
//   PicMccSurfaceCurrentSampler::sampleWithDerivative
//                                               Toolkit/Surface Charging/src/PicMccSurfaceCurrentSampler.cpp:641-670
//   CSVExporter::exportDataSet                  Tools/Output/src/CSVExporter.cpp:11-47
// Only the parity tests and the CPU reference arm of the benchmark load it.
#include "PICcore/include/PICCycle.h"
#include "Mesh/include/MeshParsing.h"
#include "Particle/include/ParticleManager.h"
#include "Interactions/Collisions/include/CollisionPicAdapter.h"
#include "Coupling/include/SurfaceCircuitCoupling.h"
#include "Material/include/MaterialProperty.h"
#include "Material/include/SurfaceMaterialModel.h"
#include "PicMccSurfaceCurrentSampler.h"
#include "Output/include/CSVExporter.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#ifdef USE_OPENMP
#include <omp.h>
#endif
#include <cstring>
#include <memory>
#include <vector>

using SCDAT::Geometry::Point3D;
using SCDAT::Geometry::Vector3D;
namespace SM = SCDAT::Mesh;
namespace SP = SCDAT::Particle;

namespace {

struct RefMesh {
    std::shared_ptr<SM::VolMesh> mesh;
    std::vector<uint8_t> dirichlet;
};

SP::Particle make_particle(std::size_t id, int kind, const double* x, const double* v, double w)
{
    Point3D p(x[0], x[1], x[2]);
    Vector3D u(v[0], v[1], v[2]);
    if (kind == 0) return SP::ParticleFactory::createElectron(id, p, u, w);
    return SP::ParticleFactory::createIon(id, p, u, 1, 1, w);
}

}  // namespace

extern "C" {

// Mesh from flat arrays.  nbr4 (nullable): per-tet neighbour list added through the
// public Element::addNeighbor in row order, -1 skipped.  node_bc: 1 = Dirichlet.
void* ref_mesh_create(int64_t N, const double* xyz, int64_t T, const int32_t* tet4, const int32_t* nbr4,
                      const uint8_t* node_bc)
{
    auto* rm = new RefMesh();
    rm->mesh = std::make_shared<SM::VolMesh>();
    for (int64_t i = 0; i < N; ++i) rm->mesh->addNode(Point3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
    for (int64_t t = 0; t < T; ++t) {
        std::vector<std::size_t> ids = {(std::size_t)tet4[4 * t], (std::size_t)tet4[4 * t + 1],
                                        (std::size_t)tet4[4 * t + 2], (std::size_t)tet4[4 * t + 3]};
        rm->mesh->addElement(SM::ElementType::TETRAHEDRON, ids);
    }
    const auto& els = rm->mesh->getElements();
    if (nbr4) {
        for (int64_t t = 0; t < T; ++t)
            for (int f = 0; f < 4; ++f)
                if (nbr4[4 * t + f] >= 0) els[t]->addNeighbor(els[nbr4[4 * t + f]]);
    }
    rm->dirichlet.assign(node_bc, node_bc + N);
    const auto& nodes = rm->mesh->getNodes();
    for (int64_t i = 0; i < N; ++i)
        nodes[i]->setBoundaryType(node_bc[i] ? SM::BoundaryType::DIRICHLET : SM::BoundaryType::INTERIOR);
    return rm;
}

void ref_mesh_destroy(void* h) { delete static_cast<RefMesh*>(h); }

// CrossTetrahedron over every particle with a frozen nodal E field.  kind[p]: 0 electron,
// 1 H+ ion.  tet: in = hint (-1 none), out = final element.  rho accumulates.
int ref_push(void* h, const double* Enode, int64_t P, double* x, double* v, const int32_t* kind, const double* w,
             int32_t* tet, uint8_t* lost, double dt, int nseg, int kernel, double* rho, int64_t* substeps)
{
    auto* rm = static_cast<RefMesh*>(h);
    const auto& nodes = rm->mesh->getNodes();
    const auto& els = rm->mesh->getElements();
    const std::size_t N = nodes.size();
    std::vector<Vector3D> E(N), B(N, Vector3D(0, 0, 0));
    for (std::size_t i = 0; i < N; ++i) E[i] = Vector3D(Enode[3 * i], Enode[3 * i + 1], Enode[3 * i + 2]);
    auto interp = std::make_shared<SP::FieldInterpolator>();
    interp->setMesh(nodes, els);
    interp->setElectricField(E);
    interp->setMagneticField(B);
    auto dep = std::make_shared<SP::ChargeDepositor>();
    dep->setMesh(nodes, els);
    dep->setTrajectoryDepositionScheme(static_cast<SP::TrajectoryChargeDepositionKernel>(kernel),
                                       static_cast<std::size_t>(nseg));
    SP::CrossTetrahedron ct;
    ct.setMesh(nodes, els);
    ct.setFieldInterpolator(interp);
    ct.setChargeDepositor(dep);
    std::vector<double> rhov(rho, rho + N);
    for (int64_t i = 0; i < P; ++i) {
        SP::Particle p = make_particle((std::size_t)i + 1, kind[i], x + 3 * i, v + 3 * i, w[i]);
        SP::ElementId hint = tet[i] < 0 ? static_cast<SP::ElementId>(-1) : (SP::ElementId)tet[i];
        auto r = ct.crossTetrahedron(&p, dt, rhov, true, hint);
        x[3 * i] = r.final_position.x(); x[3 * i + 1] = r.final_position.y(); x[3 * i + 2] = r.final_position.z();
        v[3 * i] = r.final_velocity.x(); v[3 * i + 1] = r.final_velocity.y(); v[3 * i + 2] = r.final_velocity.z();
        tet[i] = (int32_t)r.final_element;
        lost[i] = r.lost_particle ? 1 : 0;
    }
    std::memcpy(rho, rhov.data(), sizeof(double) * N);
    if (substeps) *substeps = ct.getStatistics().total_crossings;
    return 0;
}

// The reference particle path over all host threads, structured like the reference's own
// OpenMP branch of PICCycle::pushParticles (PICCycle.cpp:483-563): dynamic schedule over
// particles, thread-local charge buffers reduced at the end.  Returns wall seconds.
double ref_push_parallel(void* h, const double* Enode, int64_t P, double* x, double* v, const int32_t* kind,
                         const double* w, int32_t* tet, uint8_t* lost, double dt, int nseg, int kernel, double* rho,
                         int* threads_used)
{
    auto* rm = static_cast<RefMesh*>(h);
    const auto& nodes = rm->mesh->getNodes();
    const auto& els = rm->mesh->getElements();
    const std::size_t N = nodes.size();
    std::vector<Vector3D> E(N), B(N, Vector3D(0, 0, 0));
    for (std::size_t i = 0; i < N; ++i) E[i] = Vector3D(Enode[3 * i], Enode[3 * i + 1], Enode[3 * i + 2]);
    auto interp = std::make_shared<SP::FieldInterpolator>();
    interp->setMesh(nodes, els);
    interp->setElectricField(E);
    interp->setMagneticField(B);
    auto dep = std::make_shared<SP::ChargeDepositor>();
    dep->setMesh(nodes, els);
    dep->setTrajectoryDepositionScheme(static_cast<SP::TrajectoryChargeDepositionKernel>(kernel),
                                       static_cast<std::size_t>(nseg));
    SP::CrossTetrahedron ct;
    ct.setMesh(nodes, els);
    ct.setFieldInterpolator(interp);
    ct.setChargeDepositor(dep);
    std::vector<SP::Particle> parts;
    parts.reserve(P);
    for (int64_t i = 0; i < P; ++i) parts.push_back(make_particle((std::size_t)i + 1, kind[i], x + 3 * i, v + 3 * i, w[i]));
    int nt = 1;
#ifdef USE_OPENMP
    nt = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> trho(nt, std::vector<double>(N, 0.0));
    auto t0 = std::chrono::steady_clock::now();
#ifdef USE_OPENMP
#pragma omp parallel for schedule(dynamic, 1000)
#endif
    for (int64_t i = 0; i < P; ++i) {
        int tid = 0;
#ifdef USE_OPENMP
        tid = omp_get_thread_num();
#endif
        SP::ElementId hint = tet[i] < 0 ? static_cast<SP::ElementId>(-1) : (SP::ElementId)tet[i];
        auto r = ct.crossTetrahedron(&parts[i], dt, trho[tid], true, hint);
        x[3 * i] = r.final_position.x(); x[3 * i + 1] = r.final_position.y(); x[3 * i + 2] = r.final_position.z();
        v[3 * i] = r.final_velocity.x(); v[3 * i + 1] = r.final_velocity.y(); v[3 * i + 2] = r.final_velocity.z();
        tet[i] = (int32_t)r.final_element;
        lost[i] = r.lost_particle ? 1 : 0;
    }
    for (std::size_t n = 0; n < N; ++n)
        for (int t = 0; t < nt; ++t) rho[n] += trho[t][n];
    auto t1 = std::chrono::steady_clock::now();
    if (threads_used) *threads_used = nt;
    return std::chrono::duration<double>(t1 - t0).count();
}

// A fresh PoissonSolver: Dirichlet nodes take phi[i], nodal charge rho; DIRECT solve.
// phi out = node potentials, E out = node fields (PoissonSolver.cpp:387-401,452-529).
int ref_poisson(void* h, const double* rho, double* phi, double* E)
{
    auto* rm = static_cast<RefMesh*>(h);
    const auto& nodes = rm->mesh->getNodes();
    SCDAT::FieldSolver::PoissonSolver solver(rm->mesh);
    for (std::size_t i = 0; i < nodes.size(); ++i) {
        solver.setChargeDensity(nodes[i]->getId(), rho[i]);
        if (rm->dirichlet[i])
            solver.addBoundaryCondition(nodes[i]->getId(),
                                        std::make_shared<SCDAT::FieldSolver::BoundaryCondition>(
                                            SCDAT::FieldSolver::BoundaryConditionType::DIRICHLET, phi[i]));
    }
    if (!solver.solve(SCDAT::Solver::SolverType::DIRECT)) return 1;
    for (std::size_t i = 0; i < nodes.size(); ++i) {
        phi[i] = nodes[i]->getPotential();
        const auto& e = nodes[i]->getElectricField();
        E[3 * i] = e.x(); E[3 * i + 1] = e.y(); E[3 * i + 2] = e.z();
    }
    return 0;
}

}  // extern "C"

namespace {

// Constant elastic background collisions for both species (one process per species, as the
// PIC-MCC driver configures them), run after every executeTimeStep.
struct MccCfg {
    double n_target, sigma;
    unsigned seed;
    int64_t* hits;  // the handler's collision count (first-draw hits) over the run
};

int cycle_run(void* h, int64_t P, double* x, double* v, const int32_t* kind, const double* w, const int32_t* hint,
              int nsteps, double dt, const int32_t* face_bc, const double* phi0, int64_t* P_out, int64_t* id_out,
              int32_t* status_out, double* rho_out, double* phi_out, double* E_out, double* ledger_out,
              double* stats_out, double* seconds_out, const MccCfg* mcc)
{
    auto* rm = static_cast<RefMesh*>(h);
    const auto& nodes = rm->mesh->getNodes();
    const std::size_t N = nodes.size();
    auto pm = std::make_shared<SP::ParticleManager>((std::size_t)P + 16);
    std::vector<std::size_t> ids(P);
    for (int64_t i = 0; i < P; ++i) {
        Point3D p(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        Vector3D u(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        ids[i] = kind[i] == 0 ? pm->createElectron(p, u, w[i]) : pm->createIon(p, u, 1, 1, w[i]);
    }
    SCDAT::PICcore::PICCycle::Parameters prm;
    prm.time_step = dt;
    prm.max_iterations = 1 << 30;
    prm.verbose = false;
    SCDAT::PICcore::PICCycle cycle(prm);
    cycle.setMesh(nodes, rm->mesh->getElements());
    cycle.setParticleManager(pm);
    cycle.setPoissonSolver(std::make_shared<SCDAT::FieldSolver::PoissonSolver>(rm->mesh));
    using BF = SCDAT::PICcore::PICCycle::BoundaryFace;
    const Point3D lo = rm->mesh->getBoundingBoxMin(), hi = rm->mesh->getBoundingBoxMax();
    auto periodic = std::make_shared<SP::PeriodicBoundaryCondition>(
        std::vector<Vector3D>{Vector3D(hi.x() - lo.x(), 0, 0), Vector3D(0, hi.y() - lo.y(), 0)});
    for (int f = 0; f < 6; ++f) {
        if (face_bc[f] == 1) cycle.setBoundaryCondition((BF)f, std::make_shared<SP::AbsorbingBoundaryCondition>(1.0));
        else if (face_bc[f] == 2) cycle.setBoundaryCondition((BF)f, periodic);
    }
    if (!cycle.initialize()) return 1;
    std::vector<double> phi(phi0, phi0 + N);
    cycle.setPotential(phi);
    for (int64_t i = 0; i < P; ++i)
        if (hint[i] >= 0) cycle.addParticleLocation(pm->getParticle(ids[i]), (SP::ElementId)hint[i]);
    using namespace SCDAT::Collision;
    std::unique_ptr<MonteCarloCollisionHandler> handler;
    BackgroundMccRuntimeConfig mcc_cfg;  // keeps the configured processes (no re-initialisation)
    double volume = 1.0;
    if (mcc) {
        handler = std::make_unique<MonteCarloCollisionHandler>(mcc->seed);
        handler->clearCollisionProcesses();
        CollisionParameters cp;
        cp.energy_threshold = 0.0;
        cp.cross_section_max = mcc->sigma;
        cp.additional_params["reference_energy"] = 1.0;
        cp.additional_params["power_index"] = 0.0;  // constant cross-section
        handler->addCollisionProcess("elastic_electron", CollisionProcessFactory::createElasticProcess(
                                                             ParticleSpecies::ELECTRON, ParticleSpecies::NEUTRAL,
                                                             mcc->n_target, cp));
        handler->addCollisionProcess("elastic_ion", CollisionProcessFactory::createElasticProcess(
                                                        ParticleSpecies::ION, ParticleSpecies::NEUTRAL,
                                                        mcc->n_target, cp));
        volume = (hi.x() - lo.x()) * (hi.y() - lo.y()) * (hi.z() - lo.z());
    }
    auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < nsteps; ++s) {
        cycle.setPoissonSolver(std::make_shared<SCDAT::FieldSolver::PoissonSolver>(rm->mesh));
        if (!cycle.executeTimeStep()) return 2;
        if (mcc) executeBackgroundMccStep(pm->getContainer(), *handler, dt, volume, mcc_cfg);
    }
    if (mcc && mcc->hits) *mcc->hits = (int64_t)handler->getStatistics().total_collisions;
    auto t1 = std::chrono::steady_clock::now();
    if (seconds_out) *seconds_out = std::chrono::duration<double>(t1 - t0).count();
    auto& cont = pm->getContainer();
    int64_t k = 0;
    for (auto& p : cont) {
        const auto pos = p.getPosition();
        const auto vel = p.getVelocity();
        x[3 * k] = pos.x(); x[3 * k + 1] = pos.y(); x[3 * k + 2] = pos.z();
        v[3 * k] = vel.x(); v[3 * k + 1] = vel.y(); v[3 * k + 2] = vel.z();
        id_out[k] = (int64_t)p.getId();
        status_out[k] = (int32_t)p.getStatus();
        ++k;
    }
    *P_out = k;
    const auto& rho = cycle.getChargeDensity();
    const auto& ph = cycle.getPotential();
    const auto& E = cycle.getElectricField();
    for (std::size_t i = 0; i < N; ++i) {
        rho_out[i] = rho[i];
        phi_out[i] = ph[i];
        E_out[3 * i] = E[i].x(); E_out[3 * i + 1] = E[i].y(); E_out[3 * i + 2] = E[i].z();
    }
    const auto& led = cycle.getSurfaceCurrentLedger();
    for (int f = 0; f < 6; ++f) {
        double* r = ledger_out + 8 * f;
        r[0] = led[f].absorbed_electron_charge_c;
        r[1] = led[f].absorbed_ion_charge_c;
        r[2] = led[f].emitted_electron_charge_c;
        r[3] = led[f].incident_energy_j;
        r[4] = (double)led[f].absorbed_electron_particles;
        r[5] = (double)led[f].absorbed_ion_particles;
        r[6] = (double)led[f].emitted_electron_particles;
        r[7] = 0.0;
    }
    const auto& st = cycle.getStatistics();
    stats_out[0] = st.completed_steps;
    stats_out[1] = st.total_charge;
    stats_out[2] = st.total_energy;
    stats_out[3] = st.active_particles;
    stats_out[4] = st.surface_deposited_charge;
    return 0;
}

}  // namespace

extern "C" {

// Run nsteps of PICCycle::executeTimeStep (fresh PoissonSolver per step so the system is
// re-assembled, see PoissonSolver.cpp:387-392).  face_bc[6]: 0 none, 1 absorbing(1.0),
// 2 periodic over the x and y box lengths.  Particles come back in container order with their
// ids (1-based insertion order).
int ref_cycle_run(void* h, int64_t P, double* x, double* v, const int32_t* kind, const double* w,
                  const int32_t* hint, int nsteps, double dt, const int32_t* face_bc, const double* phi0,
                  int64_t* P_out, int64_t* id_out, int32_t* status_out, double* rho_out, double* phi_out,
                  double* E_out, double* ledger_out, double* stats_out, double* seconds_out)
{
    return cycle_run(h, P, x, v, kind, w, hint, nsteps, dt, face_bc, phi0, P_out, id_out, status_out, rho_out,
                     phi_out, E_out, ledger_out, stats_out, seconds_out, nullptr);
}

// The same run with Collision::executeBackgroundMccStep (CollisionPicAdapter.cpp:338-434) after
// every step: a constant elastic cross-section sigma against neutrals of density n_target for
// both species, the handler seeded with `seed`.  The container drops inactive particles after
// each MCC step, so only active particles come back.  *hits: the handler's collision count.
int ref_cycle_mcc_run(void* h, int64_t P, double* x, double* v, const int32_t* kind, const double* w,
                      const int32_t* hint, int nsteps, double dt, const int32_t* face_bc, const double* phi0,
                      double n_target, double sigma, unsigned seed, int64_t* P_out, int64_t* id_out,
                      int32_t* status_out, double* rho_out, double* phi_out, double* E_out, double* ledger_out,
                      double* stats_out, int64_t* hits)
{
    const MccCfg cfg{n_target, sigma, seed, hits};
    return cycle_run(h, P, x, v, kind, w, hint, nsteps, dt, face_bc, phi0, P_out, id_out, status_out, rho_out,
                     phi_out, E_out, ledger_out, stats_out, nullptr, &cfg);
}

// PICCycle::setPotential -> updateElectricField (LSQ with 1e-18 regularisation).
int ref_lsq_field(void* h, const double* phi, double* E)
{
    auto* rm = static_cast<RefMesh*>(h);
    const auto& nodes = rm->mesh->getNodes();
    const std::size_t N = nodes.size();
    auto pm = std::make_shared<SP::ParticleManager>(16);
    SCDAT::PICcore::PICCycle cycle;
    cycle.setMesh(nodes, rm->mesh->getElements());
    cycle.setParticleManager(pm);
    cycle.setPoissonSolver(std::make_shared<SCDAT::FieldSolver::PoissonSolver>(rm->mesh));
    if (!cycle.initialize()) return 1;
    cycle.setPotential(std::vector<double>(phi, phi + N));
    const auto& e = cycle.getElectricField();
    for (std::size_t i = 0; i < N; ++i) { E[3 * i] = e[i].x(); E[3 * i + 1] = e[i].y(); E[3 * i + 2] = e[i].z(); }
    return 0;
}

// Background MCC with one constant elastic process per species (sigma, n_target), run
// `repeats` times on copies of the same P particles.  Returns the handler's collision count
// (first-draw hits, CollisionAlgorithm.cpp:527-531) and, in *scattered, how many particles
// actually changed velocity (second draw passed too, :195-200).
int64_t ref_mcc_count(int64_t P, const double* v, int kind, double w, double sigma, double n_target, double dt,
                      unsigned seed, int repeats, int64_t* scattered)
{
    int64_t changed = 0;
    using namespace SCDAT::Collision;
    MonteCarloCollisionHandler handler(seed);
    handler.clearCollisionProcesses();
    CollisionParameters prm;
    prm.energy_threshold = 0.0;
    prm.cross_section_max = sigma;
    prm.additional_params["reference_energy"] = 1.0;
    prm.additional_params["power_index"] = 0.0;
    handler.addCollisionProcess(
        "elastic", CollisionProcessFactory::createElasticProcess(kind == 0 ? ParticleSpecies::ELECTRON : ParticleSpecies::ION,
                                                                 ParticleSpecies::NEUTRAL, n_target, prm));
    int64_t total = 0;
    for (int r = 0; r < repeats; ++r) {
        std::vector<ParticleObject> ps;
        ps.reserve(P);
        double z[3] = {0, 0, 0};
        for (int64_t i = 0; i < P; ++i) ps.push_back(make_particle((std::size_t)i + 1, kind, z, v + 3 * i, w));
        handler.processCollisions(ps, dt);
        for (int64_t i = 0; i < P; ++i) {
            const auto u = ps[i].getVelocity();
            if (u.x() != v[3 * i] || u.y() != v[3 * i + 1] || u.z() != v[3 * i + 2]) ++changed;
        }
    }
    total = (int64_t)handler.getStatistics().total_collisions;
    if (scattered) *scattered = changed;
    return total;
}

// One implicit advance of n independent circuit nodes (capacitance C, shunt conductance G to
// ground, potential V0, linearised plasma current I and dI/dV) by the reference's
// SurfaceCircuitCoupling; the new potentials go to V.
int ref_circuit_advance(int n, const double* C, const double* G, const double* V0, const double* I,
                        const double* dIdV, double dt, double* V)
{
    SCDAT::Coupling::SurfaceCircuitCoupling circuit;
    SCDAT::Coupling::SurfaceCircuitLinearization lin;
    for (int k = 0; k < n; ++k) {
        SCDAT::Coupling::SurfaceCircuitNode node;
        node.potential_v = V0[k];
        node.capacitance_f = C[k];
        node.shunt_conductance_s = G[k];
        circuit.addNode(node);
        lin.plasma_current_a.push_back(I[k]);
        lin.plasma_didv_a_per_v.push_back(dIdV[k]);
    }
    const auto r = circuit.advanceImplicit(dt, lin);
    if (!r.converged || (int)r.node_potentials_v.size() != n) return 1;
    for (int k = 0; k < n; ++k) V[k] = r.node_potentials_v[k];
    return 0;
}

// The reference's Whipple secondary-electron yield of a material with the given peak yield and
// peak energy, at each incident energy.
void ref_whipple_yield(double peak_yield, double peak_energy_ev, int n, const double* e_ev, double* out)
{
    SCDAT::Material::MaterialProperty mat;
    mat.setSecondaryElectronYield(peak_yield);
    mat.setScalarProperty("secondary_yield_peak_energy_ev", peak_energy_ev);
    for (int k = 0; k < n; ++k)
        out[k] = SCDAT::Material::evaluateLegacySecondaryElectronYield(
            mat, SCDAT::Material::LegacySecondaryYieldModel::Whipple, e_ev[k]);
}

// evaluateLegacySecondaryElectronYield for model 0 Whipple, 1 Sims (exponent sims_n), 2 Katz
// (range coefficients katz4 = r1, n1, r2, n2 as material scalars; NULL: the material defaults).
void ref_legacy_yield(int model, double peak_yield, double peak_energy_ev, double sims_n, const double* katz4, int n,
                      const double* e_ev, double* out)
{
    SCDAT::Material::MaterialProperty mat;
    mat.setSecondaryElectronYield(peak_yield);
    mat.setScalarProperty("secondary_yield_peak_energy_ev", peak_energy_ev);
    if (katz4) {
        mat.setScalarProperty("katz_r1", katz4[0]);
        mat.setScalarProperty("katz_n1", katz4[1]);
        mat.setScalarProperty("katz_r2", katz4[2]);
        mat.setScalarProperty("katz_n2", katz4[3]);
    }
    const auto m = model == 0 ? SCDAT::Material::LegacySecondaryYieldModel::Whipple
                   : model == 1 ? SCDAT::Material::LegacySecondaryYieldModel::Sims
                                : SCDAT::Material::LegacySecondaryYieldModel::Katz;
    for (int k = 0; k < n; ++k) out[k] = SCDAT::Material::evaluateLegacySecondaryElectronYield(mat, m, e_ev[k], sims_n);
}

// Collision::parseCollisionCrossSectionSetId: -1 for an unknown name, else the set's index.
int ref_parse_cross_section_set(const char* text)
{
    const auto id = SCDAT::Collision::parseCollisionCrossSectionSetId(text ? text : "");
    return id ? (int)*id : -1;
}

// Collision::estimateCollisionBackgroundDensities over n particles (type code, charge, weight,
// active flag) in `volume`, with the floors (neutral, ion, electron); out = the same three.
void ref_estimate_densities(int64_t n, const int32_t* type, const double* charge, const double* weight,
                            const uint8_t* active, double volume, const double* floor3, double* out3)
{
    SP::ParticleContainer box((std::size_t)std::max<int64_t>(n, 1));
    for (int64_t i = 0; i < n; ++i) {
        SP::Particle p((std::size_t)i + 1, (SP::ParticleType)type[i], Point3D(0, 0, 0), Vector3D(0, 0, 0), 1.0,
                       charge[i], weight[i]);
        if (!active[i]) p.setStatus(SP::ParticleStatus::ABSORBED);
        box.addParticle(p);
    }
    SCDAT::Collision::CollisionBackgroundDensities fl{};
    fl.neutral_density_m3 = floor3[0];
    fl.ion_density_m3 = floor3[1];
    fl.electron_density_m3 = floor3[2];
    const auto d = SCDAT::Collision::estimateCollisionBackgroundDensities(box, volume, fl);
    out3[0] = d.neutral_density_m3;
    out3[1] = d.ion_density_m3;
    out3[2] = d.electron_density_m3;
}

// The sampler's plate mesh for a sampler with no linked boundary faces: the options that
// createSamplingMesh derives from its config (PicMccSurfaceCurrentSampler.cpp:195-245: length and
// width from the area and aspect ratio, the gap as thickness, one cell across, max(4, z_layers)
// layers) through the reference's own GeometryMeshGenerator.  counts = {nodes, tets}; returns 1
// when a capacity is too small.
int ref_sampler_mesh(double area_m2, double aspect, double gap_m, int z_layers, int64_t cap_nodes, double* xyz,
                     int64_t cap_tets, int32_t* tet4, int64_t* counts)
{
    SM::GeometryDimensions dims;
    dims.shape = SM::GeometryShape::PLATE;
    const double ar = std::clamp(aspect, 0.25, 4.0);
    const double a = std::max(1.0e-12, area_m2);
    dims.length = std::sqrt(a * ar);
    dims.width = std::sqrt(a / ar);
    dims.thickness = std::max(1.0e-6, gap_m);
    SM::MeshGenerationOptions opt;
    opt.nx = 1;
    opt.ny = std::max<std::size_t>(1, (std::size_t)std::ceil(1.0 / std::max(0.5, ar)));
    opt.nz = std::max<std::size_t>(4, (std::size_t)std::max(0, z_layers));
    opt.tetrahedralize = true;
    auto mesh = SM::GeometryMeshGenerator::generateFromDimensions(dims, opt);
    if (!mesh) return 2;
    const auto& nodes = mesh->getNodes();
    const auto& els = mesh->getElements();
    counts[0] = (int64_t)nodes.size();
    counts[1] = (int64_t)els.size();
    if (counts[0] > cap_nodes || counts[1] > cap_tets) return 1;
    for (std::size_t i = 0; i < nodes.size(); ++i) {
        const auto p = nodes[i]->getPosition();
        xyz[3 * i] = p.x(); xyz[3 * i + 1] = p.y(); xyz[3 * i + 2] = p.z();
    }
    for (std::size_t e = 0; e < els.size(); ++e) {
        const auto& en = els[e]->getNodes();
        if (en.size() != 4) return 3;
        for (int k = 0; k < 4; ++k) tet4[4 * e + k] = (int32_t)en[k]->getId();
    }
    return 0;
}

// PicMccSurfaceCurrentSampler::sampleWithDerivative on a config with the given plate, plasma
// (electron and ion densities and temperatures, ion mass), particles per element, window,
// seed and potentials.  out = {electron, ion, emitted, net collection current densities,
// d(net)/dV, valid, deposition segments, the seed the sampler used}.
int ref_sampler_sample(double area_m2, double gap_m, int z_layers, int ppe, int window_steps, unsigned seed,
                       double ne, double ni, double te_ev, double ti_ev, double ion_amu, double surface_v,
                       double reference_v, double probe_dv, int enable_mcc, double* out)
{
    SCDAT::Toolkit::SurfaceCharging::PicMccSurfaceSamplerConfig c;
    c.surface_area_m2 = area_m2;
    c.gap_distance_m = gap_m;
    c.z_layers = (std::size_t)std::max(0, z_layers);
    c.particles_per_element = (std::size_t)std::max(1, ppe);
    c.window_steps = (std::size_t)std::max(1, window_steps);
    c.seed = seed;
    c.plasma.electron_density_m3 = ne;
    c.plasma.ion_density_m3 = ni;
    c.plasma.electron_temperature_ev = te_ev;
    c.plasma.ion_temperature_ev = ti_ev;
    c.plasma.ion_mass_amu = ion_amu;
    c.surface_potential_v = surface_v;
    c.plasma_reference_potential_v = reference_v;
    c.enable_mcc = enable_mcc != 0;
    SCDAT::Toolkit::SurfaceCharging::PicMccSurfaceCurrentSampler sampler;
    const auto r = sampler.sampleWithDerivative(c, probe_dv);
    out[0] = r.electron_collection_current_density_a_per_m2;
    out[1] = r.ion_collection_current_density_a_per_m2;
    out[2] = r.emitted_electron_current_density_a_per_m2;
    out[3] = r.net_collection_current_density_a_per_m2;
    out[4] = r.current_derivative_a_per_m2_per_v;
    out[5] = r.valid ? 1.0 : 0.0;
    out[6] = (double)r.deposition_segments;
    out[7] = (double)r.seed_used;
    return r.valid ? 0 : 1;
}

// CSVExporter::exportDataSet of a columnar data set (axis values and named series of n rows
// each); 0 on success.
int ref_csv_export(const char* path, const char* axis_name, int64_t n, const double* axis, int m,
                   const char* const* names, const double* const* values)
{
    SCDAT::Output::ColumnarDataSet ds;
    ds.axis_name = axis_name;
    ds.axis_values.assign(axis, axis + n);
    for (int s = 0; s < m; ++s) ds.scalar_series[names[s]] = std::vector<double>(values[s], values[s] + n);
    SCDAT::Output::CSVExporter ex;
    return ex.exportDataSet(path, ds).isSuccess() ? 0 : 1;
}

}  // extern "C"
