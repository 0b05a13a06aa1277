// The reference's own known-answer tests for the PIC path, re-hosted on the C++20 host layer
// (scdat_b200/host/scdat_host.hpp), plus a parity mode that runs a cycle through PICCycle
// for the Python side to compare with the oracle.
//
//   test_host_layer                    run the re-hosted tests; exit 1 on any failure
//   test_host_layer parity IN OUT      run the cycle described in IN, write the results to OUT
//
// Re-hosted from (paths inside the SCDAT tree):
//   Tools/PICcore/test/PICCycleBoundary_test.cpp:121-221   (4 tests)
//   Tools/FieldSolver/test/PoissonSolver_test.cpp:48-117
//   Tools/PICcore/test/PICcoreCollisionRuntime_test.cpp:9-42
// The reference meshes its 1x1x6 plate with its own box mesher; here it is the 6-tet Kuhn
// box of the same dimensions.
#include "scdat_host.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

int g_failures = 0;
int g_test_failures = 0;

#define EXPECT_TRUE(c)                                                                \
    do {                                                                              \
        if (!(c)) {                                                                   \
            std::printf("    expectation failed at line %d: %s\n", __LINE__, #c);     \
            ++g_failures;                                                             \
        }                                                                             \
    } while (0)
#define EXPECT_FALSE(c) EXPECT_TRUE(!(c))
#define EXPECT_LT(a, b) EXPECT_TRUE((a) < (b))
#define EXPECT_GT(a, b) EXPECT_TRUE((a) > (b))
#define EXPECT_LE(a, b) EXPECT_TRUE((a) <= (b))
#define EXPECT_GE(a, b) EXPECT_TRUE((a) >= (b))
#define EXPECT_EQ(a, b) EXPECT_TRUE((a) == (b))
#define EXPECT_NEAR(a, b, tol) EXPECT_TRUE(std::fabs((a) - (b)) <= (tol))
#define ASSERT_TRUE(c)                                                                \
    do {                                                                              \
        if (!(c)) {                                                                   \
            std::printf("    assertion failed at line %d: %s\n", __LINE__, #c);       \
            ++g_failures;                                                             \
            return;                                                                   \
        }                                                                             \
    } while (0)

using SCDAT::FieldSolver::BoundaryCondition;
using SCDAT::FieldSolver::BoundaryConditionType;
using SCDAT::FieldSolver::PoissonSolver;
using SCDAT::Geometry::Point3D;
using SCDAT::Geometry::Vector3D;
using SCDAT::Mesh::BoundaryType;
using SCDAT::Mesh::VolMesh;
using SCDAT::Particle::AbsorbingBoundaryCondition;
using SCDAT::Particle::ParticleManager;
using SCDAT::Particle::PeriodicBoundaryCondition;
using SCDAT::PICcore::PICCycle;
using SCDAT::Solver::SolverType;

std::shared_ptr<VolMesh> createPlateMesh(double lx, double ly, double lz)
{
    auto mesh = std::shared_ptr<VolMesh>(VolMesh::createKuhnBox(1, 1, 6, lx, ly, lz));
    return mesh;
}

// PICCycleBoundary_test.cpp:32-64: z faces Dirichlet, the rest interior
std::shared_ptr<VolMesh> createBoundaryTestMesh()
{
    auto mesh = createPlateMesh(1.0, 1.0, 1.0);
    const double z_min = mesh->getBoundingBoxMin().z();
    const double z_max = mesh->getBoundingBoxMax().z();
    for (const auto& node : mesh->getNodes()) {
        const double z = node->getPosition().z();
        node->setBoundaryType((std::fabs(z - z_min) < 1e-12 || std::fabs(z - z_max) < 1e-12) ? BoundaryType::DIRICHLET
                                                                                             : BoundaryType::INTERIOR);
    }
    return mesh;
}

// PICCycleBoundary_test.cpp:66-100
PICCycle createConfiguredCycle(const std::shared_ptr<VolMesh>& mesh, const std::shared_ptr<ParticleManager>& pm)
{
    auto poisson_solver = std::make_shared<PoissonSolver>(mesh);
    PICCycle::Parameters params;
    params.time_step = 1.0e-9;
    params.max_iterations = 4;
    params.statistics_frequency = 1;
    PICCycle cycle(params);
    cycle.setMesh(mesh->getNodes(), mesh->getElements());
    cycle.setParticleManager(pm);
    cycle.setPoissonSolver(poisson_solver);
    const Point3D lo = mesh->getBoundingBoxMin(), hi = mesh->getBoundingBoxMax();
    auto periodic = std::make_shared<PeriodicBoundaryCondition>(
        std::vector<Vector3D>{Vector3D(hi.x() - lo.x(), 0.0, 0.0), Vector3D(0.0, hi.y() - lo.y(), 0.0)});
    cycle.setBoundaryCondition(PICCycle::BoundaryFace::XMin, periodic);
    cycle.setBoundaryCondition(PICCycle::BoundaryFace::XMax, periodic);
    cycle.setBoundaryCondition(PICCycle::BoundaryFace::YMin, periodic);
    cycle.setBoundaryCondition(PICCycle::BoundaryFace::YMax, periodic);
    cycle.setBoundaryCondition(PICCycle::BoundaryFace::ZMin, std::make_shared<AbsorbingBoundaryCondition>(1.0));
    cycle.setBoundaryCondition(PICCycle::BoundaryFace::ZMax, std::make_shared<AbsorbingBoundaryCondition>(1.0));
    EXPECT_TRUE(cycle.initialize());
    cycle.setPotential(std::vector<double>(mesh->getNodeCount(), 0.0));
    return cycle;
}

std::size_t findElementWithLargestCoordinate(const VolMesh& mesh, int axis)
{
    std::size_t best = 0;
    double best_value = -1e300;
    for (std::size_t i = 0; i < mesh.getElementCount(); ++i) {
        const auto c = mesh.getElement(i)->getCentroid();
        const double v = axis == 0 ? c.x() : (axis == 1 ? c.y() : c.z());
        if (v > best_value) {
            best_value = v;
            best = i;
        }
    }
    return best;
}

void PeriodicBoundaryKeepsParticleActiveInsideDomain()
{
    auto mesh = createBoundaryTestMesh();
    auto pm = std::make_shared<ParticleManager>();
    PICCycle cycle = createConfiguredCycle(mesh, pm);
    const Point3D start = mesh->getElement(findElementWithLargestCoordinate(*mesh, 0))->getCentroid();
    const auto id = pm->createElectron(start, Vector3D(2.0e9, 0.0, 0.0), 1.0);
    ASSERT_TRUE(cycle.executeTimeStep());
    const auto* p = pm->getParticle(id);
    ASSERT_TRUE(p != nullptr);
    EXPECT_TRUE(p->isActive());
    EXPECT_GE(p->getPosition().x(), mesh->getBoundingBoxMin().x() - 1.0e-9);
    EXPECT_LE(p->getPosition().x(), mesh->getBoundingBoxMax().x() + 1.0e-9);
}

void AbsorbingBoundaryMarksParticleInactiveAndAccumulatesCharge()
{
    auto mesh = createBoundaryTestMesh();
    auto pm = std::make_shared<ParticleManager>();
    PICCycle cycle = createConfiguredCycle(mesh, pm);
    const Point3D start = mesh->getElement(findElementWithLargestCoordinate(*mesh, 2))->getCentroid();
    const auto id = pm->createElectron(start, Vector3D(0.0, 0.0, 2.0e9), 1.0);
    ASSERT_TRUE(cycle.executeTimeStep());
    const auto* p = pm->getParticle(id);
    ASSERT_TRUE(p != nullptr);
    EXPECT_FALSE(p->isActive());
    EXPECT_LT(cycle.getStatistics().surface_deposited_charge, 0.0);
    const auto& ledger = cycle.getSurfaceCurrentLedger();
    EXPECT_LT(ledger[(std::size_t)PICCycle::BoundaryFace::ZMax].absorbed_electron_charge_c, 0.0);
    EXPECT_EQ(ledger[(std::size_t)PICCycle::BoundaryFace::ZMax].absorbed_electron_particles, 1u);
}

void ManualPotentialProfileReconstructsElectricField()
{
    auto mesh = createBoundaryTestMesh();
    auto pm = std::make_shared<ParticleManager>();
    PICCycle cycle = createConfiguredCycle(mesh, pm);
    std::vector<double> potential(mesh->getNodeCount(), 0.0);
    for (const auto& node : mesh->getNodes()) potential[node->getId()] = 12.0 * node->getPosition().z();
    cycle.setPotential(potential);
    const auto& E = cycle.getElectricField();
    ASSERT_TRUE(E.size() == mesh->getNodeCount());
    double mean_ez = 0.0;
    for (const auto& f : E) {
        EXPECT_TRUE(std::isfinite(f.x()) && std::isfinite(f.y()) && std::isfinite(f.z()));
        mean_ez += f.z();
    }
    mean_ez /= (double)E.size();
    EXPECT_LT(mean_ez, -1.0);
    // a linear potential is reproduced exactly by the nodal least-squares gradient
    for (const auto& f : E) EXPECT_NEAR(f.z(), -12.0, 1e-9);
}

void LegacyFallbackDoesNotRecoverFarEscapes()
{
    auto mesh = createBoundaryTestMesh();
    auto pm = std::make_shared<ParticleManager>();
    PICCycle cycle = createConfiguredCycle(mesh, pm);
    cycle.clearBoundaryConditions();
    const Point3D start = mesh->getElement(findElementWithLargestCoordinate(*mesh, 2))->getCentroid();
    const auto id = pm->createElectron(start, Vector3D(0.0, 0.0, 5.0e12), 1.0);
    ASSERT_TRUE(cycle.executeTimeStep());
    const auto* p = pm->getParticle(id);
    ASSERT_TRUE(p != nullptr);
    EXPECT_FALSE(p->isActive());
    EXPECT_NEAR(cycle.getStatistics().surface_deposited_charge, 0.0, 1.0e-20);
}

// PoissonSolver_test.cpp:48-117
void SolvesFiniteDirichletProfileOnPlateMesh()
{
    auto mesh = createPlateMesh(0.01, 0.01, 0.02);
    ASSERT_TRUE(mesh->validate());
    const double z_min = mesh->getBoundingBoxMin().z(), z_max = mesh->getBoundingBoxMax().z();
    PoissonSolver solver(mesh);
    for (const auto& node : mesh->getNodes()) {
        const double z = node->getPosition().z();
        if (std::fabs(z - z_min) < 1e-12) {
            node->setBoundaryType(BoundaryType::DIRICHLET);
            solver.addBoundaryCondition(node->getId(),
                                        std::make_shared<BoundaryCondition>(BoundaryConditionType::DIRICHLET, 10.0));
        } else if (std::fabs(z - z_max) < 1e-12) {
            node->setBoundaryType(BoundaryType::DIRICHLET);
            solver.addBoundaryCondition(node->getId(),
                                        std::make_shared<BoundaryCondition>(BoundaryConditionType::DIRICHLET, 0.0));
        } else {
            node->setBoundaryType(BoundaryType::INTERIOR);
        }
    }
    ASSERT_TRUE(solver.solve(SolverType::DIRECT));
    bool found_interior = false;
    double max_field = 0.0;
    for (const auto& node : mesh->getNodes()) {
        const double phi = node->getPotential(), z = node->getPosition().z();
        EXPECT_TRUE(std::isfinite(phi));
        if (std::fabs(z - z_min) < 1e-12) {
            EXPECT_NEAR(phi, 10.0, 1e-8);
        } else if (std::fabs(z - z_max) < 1e-12) {
            EXPECT_NEAR(phi, 0.0, 1e-8);
        } else {
            found_interior = true;
            EXPECT_GE(phi, -1e-8);
            EXPECT_LE(phi, 10.0 + 1e-8);
        }
        const auto e = solver.getElectricField(node->getId());
        EXPECT_TRUE(std::isfinite(e.x()) && std::isfinite(e.y()) && std::isfinite(e.z()));
        max_field = std::max(max_field, e.magnitude());
    }
    EXPECT_TRUE(found_interior);
    EXPECT_GT(max_field, 0.0);
    EXPECT_GE(solver.getTotalEnergy(), 0.0);
    EXPECT_GE(solver.getMaxPotential(), solver.getMinPotential());
}

// PICcoreCollisionRuntime_test.cpp:9-42
void SharedCollisionRuntimeSupportsToolkitCrossSectionSets()
{
    SCDAT::Particle::ParticleManager particle_manager;
    SCDAT::Collision::MonteCarloCollisionHandler handler(12345);
    SCDAT::Collision::BackgroundMccRuntimeConfig cfg;
    cfg.floor_densities.neutral_density_m3 = 2.4e20;
    cfg.floor_densities.ion_density_m3 = 1.4e14;
    cfg.floor_densities.electron_density_m3 = 1.4e14;
    cfg.cross_section_set_id = SCDAT::Collision::CollisionCrossSectionSetId::SurfacePicV1;
    cfg.reinitialize_configuration = true;
    const auto r = SCDAT::Collision::executeBackgroundMccStep(particle_manager.getContainer(), handler, 1.0e-10, 1.0e-6, cfg);
    EXPECT_EQ(r.active_particles, 0u);
    EXPECT_EQ(r.effective_neutral_density_m3, cfg.floor_densities.neutral_density_m3);
    EXPECT_EQ(r.effective_ion_density_m3, cfg.floor_densities.ion_density_m3);
    EXPECT_EQ(r.effective_electron_density_m3, cfg.floor_densities.electron_density_m3);
    const auto s = SCDAT::Collision::parseCollisionCrossSectionSetId("surface_pic_v1");
    ASSERT_TRUE(s.has_value());
    EXPECT_TRUE(*s == SCDAT::Collision::CollisionCrossSectionSetId::SurfacePicV1);
    const auto a = SCDAT::Collision::parseCollisionCrossSectionSetId("vacuum_arc_pic_v1");
    ASSERT_TRUE(a.has_value());
    EXPECT_TRUE(*a == SCDAT::Collision::CollisionCrossSectionSetId::VacuumArcPicV1);
}

// Elastic MCC through the host layer: speeds are kept and the collision count is reported.
void ElasticBackgroundStepKeepsSpeeds()
{
    auto mesh = std::shared_ptr<VolMesh>(VolMesh::createKuhnBox(3, 3, 3, 0.15, 0.15, 0.15));
    for (const auto& n : mesh->getNodes()) {
        const auto& p = n->getPosition();
        const bool outer = p.x() < 1e-12 || p.y() < 1e-12 || p.z() < 1e-12 || p.x() > 0.15 - 1e-12 ||
                           p.y() > 0.15 - 1e-12 || p.z() > 0.15 - 1e-12;
        n->setBoundaryType(outer ? BoundaryType::DIRICHLET : BoundaryType::INTERIOR);
    }
    auto pm = std::make_shared<ParticleManager>();
    PICCycle::Parameters prm;
    prm.time_step = 1e-12;
    PICCycle cycle(prm);
    cycle.setMesh(mesh->getNodes(), mesh->getElements());
    cycle.setParticleManager(pm);
    cycle.setPoissonSolver(std::make_shared<PoissonSolver>(mesh));
    ASSERT_TRUE(cycle.initialize());
    std::vector<SCDAT::Particle::ParticleId> ids;
    for (int i = 0; i < 64; ++i)
        ids.push_back(pm->createElectron(Point3D(0.05 + 0.0007 * i, 0.07, 0.08), Vector3D(1e5, 2e5, -3e4), 1.0));
    ASSERT_TRUE(cycle.executeTimeStep());
    SCDAT::Collision::MonteCarloCollisionHandler handler(7);
    SCDAT::Collision::ElasticProcess e;
    e.projectile = SCDAT::Particle::ParticleType::ELECTRON;
    e.target_density_m3 = 1e30;  // nu*dt >> 1: every particle scatters
    e.sigma_max_m2 = 1e-19;
    handler.addElasticProcess(e);
    SCDAT::Collision::BackgroundMccRuntimeConfig cfg;
    std::vector<double> speed_before;
    for (auto id : ids) speed_before.push_back(pm->getParticle(id)->getVelocity().magnitude());
    const auto r = SCDAT::Collision::executeBackgroundMccStep(pm->getContainer(), handler, 1e-12, 1.0, cfg);
    EXPECT_EQ(r.active_particles, ids.size());
    EXPECT_EQ(r.collision_events, ids.size());
    for (std::size_t i = 0; i < ids.size(); ++i) {
        const auto* p = pm->getParticle(ids[i]);
        ASSERT_TRUE(p != nullptr);
        EXPECT_NEAR(p->getVelocity().magnitude(), speed_before[i], 1e-9 * speed_before[i]);
    }
    // a handler with a named cross-section set refuses to run processes the device lacks
    bool threw = false;
    cfg.reinitialize_configuration = true;
    try {
        SCDAT::Collision::executeBackgroundMccStep(pm->getContainer(), handler, 1e-12, 1.0, cfg);
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    EXPECT_TRUE(threw);
}

// ---- parity mode ---------------------------------------------------------------------
// IN (little-endian): int32 nx, ny, nz, nsteps, face_bc[6]; float64 h, dt; int64 n_particles;
// per node float64 phi0 (outer nodes Dirichlet); per particle int32 kind (0 electron, 1 H+),
// float64 x[3], v[3], weight.
// OUT: per particle float64 x[3], v[3], status; per node float64 rho, phi; float64 ledger[6][7];
// float64 surface charge.
template <typename T> T rd(std::ifstream& f)
{
    T v;
    f.read(reinterpret_cast<char*>(&v), sizeof(T));
    if (!f) throw std::runtime_error("short input");
    return v;
}
template <typename T> void wr(std::ofstream& f, T v) { f.write(reinterpret_cast<const char*>(&v), sizeof(T)); }

int parity(const char* in_path, const char* out_path)
{
    std::ifstream in(in_path, std::ios::binary);
    const int nx = rd<int32_t>(in), ny = rd<int32_t>(in), nz = rd<int32_t>(in), nsteps = rd<int32_t>(in);
    int face[6];
    for (int& f : face) f = rd<int32_t>(in);
    const double h = rd<double>(in), dt = rd<double>(in);
    const int64_t np = rd<int64_t>(in);
    auto mesh = std::shared_ptr<VolMesh>(VolMesh::createKuhnBox(nx, ny, nz, nx * h, ny * h, nz * h));
    const auto lo = mesh->getBoundingBoxMin(), hi = mesh->getBoundingBoxMax();
    std::vector<double> phi0(mesh->getNodeCount());
    for (auto& v : phi0) v = rd<double>(in);
    for (const auto& n : mesh->getNodes()) {
        const auto& p = n->getPosition();
        const bool outer = std::fabs(p.x() - lo.x()) < 1e-12 || std::fabs(p.y() - lo.y()) < 1e-12 ||
                           std::fabs(p.z() - lo.z()) < 1e-12 || std::fabs(p.x() - hi.x()) < 1e-12 ||
                           std::fabs(p.y() - hi.y()) < 1e-12 || std::fabs(p.z() - hi.z()) < 1e-12;
        n->setBoundaryType(outer ? BoundaryType::DIRICHLET : BoundaryType::INTERIOR);
        n->setPotential(phi0[n->getId()]);
    }
    auto pm = std::make_shared<ParticleManager>();
    PICCycle::Parameters prm;
    prm.time_step = dt;
    PICCycle cycle(prm);
    PICCycle::DeviceOptions opt;
    opt.pcg_rtol = 1e-15;
    cycle.setDeviceOptions(opt);
    cycle.setMesh(mesh->getNodes(), mesh->getElements());
    cycle.setParticleManager(pm);
    cycle.setPoissonSolver(std::make_shared<PoissonSolver>(mesh));
    std::vector<double> periods{hi.x() - lo.x(), hi.y() - lo.y(), hi.z() - lo.z()};
    for (int f = 0; f < 6; ++f) {
        const int a = f / 2;
        if (face[f] == 1) cycle.setBoundaryCondition((PICCycle::BoundaryFace)f, std::make_shared<AbsorbingBoundaryCondition>(1.0));
        if (face[f] == 2)
            cycle.setBoundaryCondition((PICCycle::BoundaryFace)f, std::make_shared<PeriodicBoundaryCondition>(std::vector<Vector3D>{
                                                                      Vector3D(a == 0 ? periods[0] : 0.0, a == 1 ? periods[1] : 0.0,
                                                                               a == 2 ? periods[2] : 0.0)}));
    }
    if (!cycle.initialize()) {
        std::printf("initialize failed: %s\n", cycle.lastError().c_str());
        return 2;
    }
    std::vector<SCDAT::Particle::ParticleId> ids;
    for (int64_t i = 0; i < np; ++i) {
        const int kind = rd<int32_t>(in);
        double x[3], v[3];
        for (double& c : x) c = rd<double>(in);
        for (double& c : v) c = rd<double>(in);
        const double w = rd<double>(in);
        ids.push_back(kind == 0 ? pm->createElectron(Point3D(x[0], x[1], x[2]), Vector3D(v[0], v[1], v[2]), w)
                                : pm->createIon(Point3D(x[0], x[1], x[2]), Vector3D(v[0], v[1], v[2]), 1, 1, w));
    }
    for (int s = 0; s < nsteps; ++s)
        if (!cycle.executeTimeStep()) {
            std::printf("step failed: %s\n", cycle.lastError().c_str());
            return 3;
        }
    std::ofstream out(out_path, std::ios::binary);
    const auto& cont = std::as_const(*pm).getContainer();
    for (auto id : ids) {
        const auto* p = cont.getParticle(id);
        wr(out, p->getPosition().x());
        wr(out, p->getPosition().y());
        wr(out, p->getPosition().z());
        wr(out, p->getVelocity().x());
        wr(out, p->getVelocity().y());
        wr(out, p->getVelocity().z());
        wr(out, (double)(p->isActive() ? 0 : (p->getStatus() == SCDAT::Particle::ParticleStatus::ABSORBED ? 1 : 2)));
    }
    for (double r : cycle.getChargeDensity()) wr(out, r);
    for (double r : cycle.getPotential()) wr(out, r);
    for (const auto& e : cycle.getSurfaceCurrentLedger()) {
        wr(out, e.absorbed_electron_charge_c);
        wr(out, e.absorbed_ion_charge_c);
        wr(out, e.emitted_electron_charge_c);
        wr(out, e.incident_energy_j);
        wr(out, (double)e.absorbed_electron_particles);
        wr(out, (double)e.absorbed_ion_particles);
        wr(out, (double)e.emitted_electron_particles);
    }
    wr(out, cycle.getStatistics().surface_deposited_charge);
    return out ? 0 : 4;
}

}  // namespace

// Host-side collision helpers on inputs from the test (no GPU): "parse <name>" prints the set
// index (-1: unknown); "densities <in> <out>" reads n, then n x (type, charge, weight, active),
// the volume and the three floors, and writes the three densities.
int collision_helpers(int argc, char** argv)
{
    if (argc == 3 && std::strcmp(argv[1], "parse") == 0) {
        const auto id = SCDAT::Collision::parseCollisionCrossSectionSetId(argv[2]);
        std::printf("%d\n", id ? (int)*id : -1);
        return 0;
    }
    std::ifstream in(argv[2], std::ios::binary);
    int64_t n = 0;
    in.read(reinterpret_cast<char*>(&n), sizeof(n));
    SCDAT::Particle::ParticleContainer box;
    for (int64_t i = 0; i < n; ++i) {
        double rec[4];
        in.read(reinterpret_cast<char*>(rec), sizeof(rec));
        SCDAT::Particle::Particle p((SCDAT::Particle::ParticleId)(i + 1), (SCDAT::Particle::ParticleType)(int)rec[0],
                                    SCDAT::Geometry::Point3D(0, 0, 0), SCDAT::Geometry::Vector3D(0, 0, 0), 1.0, rec[1],
                                    rec[2]);
        if (rec[3] == 0.0) p.setStatus(SCDAT::Particle::ParticleStatus::ABSORBED);
        box.addParticle(p);
    }
    double vf[4];
    in.read(reinterpret_cast<char*>(vf), sizeof(vf));
    if (!in) return 2;
    SCDAT::Collision::CollisionBackgroundDensities fl{};
    fl.neutral_density_m3 = vf[1];
    fl.ion_density_m3 = vf[2];
    fl.electron_density_m3 = vf[3];
    const auto d = SCDAT::Collision::estimateCollisionBackgroundDensities(box, vf[0], fl);
    std::ofstream out(argv[3], std::ios::binary);
    const double o[3] = {d.neutral_density_m3, d.ion_density_m3, d.electron_density_m3};
    out.write(reinterpret_cast<const char*>(o), sizeof(o));
    return out ? 0 : 3;
}

int main(int argc, char** argv)
{
    if ((argc == 3 && std::strcmp(argv[1], "parse") == 0) || (argc == 4 && std::strcmp(argv[1], "densities") == 0))
        return collision_helpers(argc, argv);
    if (argc == 4 && std::strcmp(argv[1], "parity") == 0) {
        try {
            return parity(argv[2], argv[3]);
        } catch (const std::exception& e) {
            std::printf("parity run failed: %s\n", e.what());
            return 5;
        }
    }
    const std::vector<std::pair<const char*, std::function<void()>>> tests = {
        {"PICCycleBoundaryTest.PeriodicBoundaryKeepsParticleActiveInsideDomain", PeriodicBoundaryKeepsParticleActiveInsideDomain},
        {"PICCycleBoundaryTest.AbsorbingBoundaryMarksParticleInactiveAndAccumulatesCharge",
         AbsorbingBoundaryMarksParticleInactiveAndAccumulatesCharge},
        {"PICCycleBoundaryTest.ManualPotentialProfileReconstructsElectricField", ManualPotentialProfileReconstructsElectricField},
        {"PICCycleBoundaryTest.LegacyFallbackDoesNotRecoverFarEscapes", LegacyFallbackDoesNotRecoverFarEscapes},
        {"PoissonSolverTest.SolvesFiniteDirichletProfileOnPlateMesh", SolvesFiniteDirichletProfileOnPlateMesh},
        {"PICcoreCollisionRuntimeTest.SharedCollisionRuntimeSupportsToolkitCrossSectionSets",
         SharedCollisionRuntimeSupportsToolkitCrossSectionSets},
        {"HostLayer.ElasticBackgroundStepKeepsSpeeds", ElasticBackgroundStepKeepsSpeeds},
    };
    for (const auto& [name, fn] : tests) {
        const int before = g_failures;
        try {
            fn();
        } catch (const std::exception& e) {
            std::printf("    exception: %s\n", e.what());
            ++g_failures;
        }
        const bool ok = g_failures == before;
        if (!ok) ++g_test_failures;
        std::printf("[%s] %s\n", ok ? "  OK  " : " FAIL ", name);
    }
    std::printf("%d test(s) failed\n", g_test_failures);
    return g_test_failures ? 1 : 0;
}
