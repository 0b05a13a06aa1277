// scdat_host.cpp -- the C++20 host layer: the reference's PIC-path classes driving the
// device through the C ABI.  No numerical step of the path runs here; see scdat_host.hpp.
#include "scdat_host.hpp"

#include <cmath>

#include <cctype>

#include "scdat_b200.h"

#include <algorithm>
#include <chrono>
#include <limits>
#include <stdexcept>
#include <utility>

namespace SCDAT {

// ==========================================================================================
// Mesh
// ==========================================================================================
namespace Mesh {

TetrahedronElement::TetrahedronElement(ElementId id, std::vector<NodePtr> nodes) : id_(id), nodes_(std::move(nodes))
{
    if (nodes_.size() != 4) throw std::invalid_argument("a tetrahedron needs 4 nodes");
    for (const auto& n : nodes_)
        if (!n) throw std::invalid_argument("null node in tetrahedron");
}

// |det[b-a, c-a, d-a]| / 6 (TetrahedronElement::getVolume, MeshAlgorithms.cpp:29-54)
double TetrahedronElement::getVolume() const
{
    const auto& a = nodes_[0]->getPosition();
    const Utils::Vector3D u = nodes_[1]->getPosition() - a, v = nodes_[2]->getPosition() - a,
                          w = nodes_[3]->getPosition() - a;
    const double det = u.x() * (v.y() * w.z() - v.z() * w.y()) - u.y() * (v.x() * w.z() - v.z() * w.x()) +
                       u.z() * (v.x() * w.y() - v.y() * w.x());
    return std::fabs(det) / 6.0;
}

Utils::Point3D TetrahedronElement::getCentroid() const
{
    double x = 0.0, y = 0.0, z = 0.0;
    for (const auto& n : nodes_) {
        x += n->getPosition().x();
        y += n->getPosition().y();
        z += n->getPosition().z();
    }
    return {0.25 * x, 0.25 * y, 0.25 * z};
}

NodeId VolMesh::addNode(const Utils::Point3D& position)
{
    const NodeId id = nodes_.size();
    nodes_.push_back(std::make_shared<Node>(id, position));
    return id;
}

ElementId VolMesh::addElement(const std::array<NodeId, 4>& ids)
{
    std::vector<NodePtr> nn;
    for (NodeId i : ids) {
        if (i >= nodes_.size()) throw std::out_of_range("element references a missing node");
        nn.push_back(nodes_[i]);
    }
    const ElementId id = elements_.size();
    elements_.push_back(std::make_shared<TetrahedronElement>(id, std::move(nn)));
    return id;
}

Utils::Point3D VolMesh::getBoundingBoxMin() const
{
    if (nodes_.empty()) return {};
    double x = std::numeric_limits<double>::max(), y = x, z = x;
    for (const auto& n : nodes_) {
        x = std::min(x, n->getPosition().x());
        y = std::min(y, n->getPosition().y());
        z = std::min(z, n->getPosition().z());
    }
    return {x, y, z};
}

Utils::Point3D VolMesh::getBoundingBoxMax() const
{
    if (nodes_.empty()) return {};
    double x = std::numeric_limits<double>::lowest(), y = x, z = x;
    for (const auto& n : nodes_) {
        x = std::max(x, n->getPosition().x());
        y = std::max(y, n->getPosition().y());
        z = std::max(z, n->getPosition().z());
    }
    return {x, y, z};
}

bool VolMesh::validate() const
{
    if (nodes_.empty() || elements_.empty()) return false;
    for (std::size_t i = 0; i < nodes_.size(); ++i)
        if (!nodes_[i] || nodes_[i]->getId() != i) return false;
    for (const auto& e : elements_)
        if (!e || !(e->getVolume() > 0.0)) return false;
    return true;
}

std::unique_ptr<VolMesh> VolMesh::createKuhnBox(int nx, int ny, int nz, double lx, double ly, double lz)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || !(lx > 0.0) || !(ly > 0.0) || !(lz > 0.0))
        throw std::invalid_argument("box needs positive cell counts and lengths");
    int64_t nn = 0, nt = 0, nc = 0;
    if (scdat_kuhn_box_mesh(nx, ny, nz, 1.0, nullptr, nullptr, 0.0, 0.0, &nn, &nt, nullptr, nullptr, nullptr, nullptr,
                            nullptr, &nc) != SCDAT_OK)
        throw std::invalid_argument("box mesher rejected the dimensions");
    std::vector<double> xyz((size_t)nn * 3), phi((size_t)nn);
    std::vector<int32_t> tet((size_t)nt * 4), hex((size_t)nc * 3);
    std::vector<uint8_t> dir((size_t)nn);
    if (scdat_kuhn_box_mesh(nx, ny, nz, 1.0, nullptr, nullptr, 0.0, 0.0, &nn, &nt, xyz.data(), tet.data(), dir.data(),
                            phi.data(), hex.data(), &nc) != SCDAT_OK)
        throw std::invalid_argument("box mesher failed");
    auto mesh = std::make_unique<VolMesh>();
    const double sx = lx / nx, sy = ly / ny, sz = lz / nz;
    for (int64_t i = 0; i < nn; ++i) mesh->addNode({xyz[3 * i] * sx, xyz[3 * i + 1] * sy, xyz[3 * i + 2] * sz});
    for (int64_t t = 0; t < nt; ++t)
        mesh->addElement({(NodeId)tet[4 * t], (NodeId)tet[4 * t + 1], (NodeId)tet[4 * t + 2], (NodeId)tet[4 * t + 3]});
    return mesh;
}

}  // namespace Mesh

// ==========================================================================================
// Particles
// ==========================================================================================
namespace Particle {

Particle::Particle(ParticleId id, ParticleType type, const Geometry::Point3D& position,
                   const Geometry::Vector3D& velocity, double mass, double charge, double weight)
    : id_(id), type_(type), position_(position), velocity_(velocity), mass_(mass), charge_(charge), weight_(weight)
{
}

ParticleContainer::ParticleContainer(std::size_t initial_capacity) { particles_.reserve(initial_capacity); }

void ParticleContainer::sync() const
{
    if (mirror_) mirror_->pull();
}

void ParticleContainer::rebuildIndex()
{
    index_.clear();
    for (std::size_t i = 0; i < particles_.size(); ++i) index_[particles_[i].getId()] = i;
}

void ParticleContainer::addParticle(const Particle& particle)
{
    sync();
    index_[particle.getId()] = particles_.size();
    particles_.push_back(particle);
    touch();
}

void ParticleContainer::addParticles(const std::vector<Particle>& particles)
{
    sync();
    for (const auto& p : particles) {
        index_[p.getId()] = particles_.size();
        particles_.push_back(p);
    }
    touch();
}

bool ParticleContainer::removeParticle(ParticleId id)
{
    sync();
    auto it = index_.find(id);
    if (it == index_.end()) return false;
    particles_.erase(particles_.begin() + (std::ptrdiff_t)it->second);
    rebuildIndex();
    touch();
    return true;
}

ParticlePtr ParticleContainer::getParticle(ParticleId id)
{
    sync();
    auto it = index_.find(id);
    if (it == index_.end()) return nullptr;
    touch();  // the caller may write through the pointer
    return &particles_[it->second];
}

const Particle* ParticleContainer::getParticle(ParticleId id) const
{
    sync();
    auto it = index_.find(id);
    return it == index_.end() ? nullptr : &particles_[it->second];
}

// ParticleContainer::removeInactiveParticles (ParticleManager.cpp:157-177)
std::size_t ParticleContainer::removeInactiveParticles()
{
    sync();
    const std::size_t before = particles_.size();
    particles_.erase(std::remove_if(particles_.begin(), particles_.end(), [](const Particle& p) { return !p.isActive(); }),
                     particles_.end());
    const std::size_t removed = before - particles_.size();
    if (removed) {
        rebuildIndex();
        touch();
        if (mirror_) mirror_->compact();
    }
    return removed;
}

std::vector<ParticlePtr> ParticleContainer::getParticlesByType(ParticleType type)
{
    sync();
    touch();
    std::vector<ParticlePtr> out;
    for (auto& p : particles_)
        if (p.getType() == type) out.push_back(&p);
    return out;
}

std::size_t ParticleContainer::size() const
{
    sync();
    return particles_.size();
}

std::size_t ParticleContainer::getActiveCount() const
{
    sync();
    return (std::size_t)std::count_if(particles_.begin(), particles_.end(), [](const Particle& p) { return p.isActive(); });
}

void ParticleContainer::clear()
{
    particles_.clear();
    index_.clear();
    touch();
}

std::vector<Particle>::iterator ParticleContainer::begin()
{
    sync();
    touch();
    return particles_.begin();
}
std::vector<Particle>::iterator ParticleContainer::end() { return particles_.end(); }
std::vector<Particle>::const_iterator ParticleContainer::begin() const
{
    sync();
    return particles_.begin();
}
std::vector<Particle>::const_iterator ParticleContainer::end() const { return particles_.end(); }

ParticleManager::ParticleManager(std::size_t max_particles)
    : max_particles_(max_particles), container_(std::make_unique<ParticleContainer>(std::min<std::size_t>(max_particles, 10000)))
{
}

// ParticleFactory::createElectron (ParticleDefinitions.cpp:374-380)
ParticleId ParticleManager::createElectron(const Geometry::Point3D& position, const Geometry::Vector3D& velocity,
                                           double weight)
{
    if (container_->size() >= max_particles_) throw std::length_error("particle manager is full");
    const ParticleId id = next_id_++;
    container_->addParticle(Particle(id, ParticleType::ELECTRON, position, velocity, Constants::kElectronMass,
                                     -Constants::kElementaryCharge, weight));
    return id;
}

// ParticleFactory::createIon (ParticleDefinitions.cpp:382-392): mass_number proton masses,
// charge_number elementary charges.
ParticleId ParticleManager::createIon(const Geometry::Point3D& position, const Geometry::Vector3D& velocity,
                                      int mass_number, int charge_number, double weight)
{
    if (mass_number <= 0) throw std::invalid_argument("ion mass number must be positive");
    if (container_->size() >= max_particles_) throw std::length_error("particle manager is full");
    const ParticleId id = next_id_++;
    container_->addParticle(Particle(id, ParticleType::ION, position, velocity, mass_number * Constants::kProtonMass,
                                     charge_number * Constants::kElementaryCharge, weight));
    return id;
}

AbsorbingBoundaryCondition::AbsorbingBoundaryCondition(double p) : p_(p)
{
    if (!(p >= 0.0 && p <= 1.0)) throw std::invalid_argument("absorption probability must be in [0,1]");
}

PeriodicBoundaryCondition::PeriodicBoundaryCondition(const std::vector<Geometry::Vector3D>& period_vectors)
    : periods_(period_vectors)
{
    if (periods_.empty() || periods_.size() > 3) throw std::invalid_argument("1 to 3 period vectors");
}

}  // namespace Particle

// ==========================================================================================
// Shared helpers
// ==========================================================================================
namespace {

struct MeshArrays {
    std::vector<double> xyz;
    std::vector<int32_t> tet;
    std::vector<uint8_t> dirichlet;
    std::vector<double> cv;  // nodal control volume sum_e V_e/4
    double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
};

// Node and element ids must equal their index (VolMesh numbering).
std::string flatten_mesh(const std::vector<Mesh::NodePtr>& nodes, const std::vector<Mesh::ElementPtr>& elements,
                         MeshArrays& m)
{
    const std::size_t N = nodes.size(), T = elements.size();
    if (N == 0 || T == 0) return "empty mesh";
    if (N > (std::size_t)std::numeric_limits<int32_t>::max()) return "too many nodes";
    m.xyz.assign(3 * N, 0.0);
    m.dirichlet.assign(N, 0);
    m.cv.assign(N, 0.0);
    for (int a = 0; a < 3; ++a) {
        m.bmin[a] = std::numeric_limits<double>::max();
        m.bmax[a] = std::numeric_limits<double>::lowest();
    }
    for (std::size_t i = 0; i < N; ++i) {
        if (!nodes[i] || nodes[i]->getId() != i) return "node ids must equal their index";
        const auto& p = nodes[i]->getPosition();
        const double c[3] = {p.x(), p.y(), p.z()};
        for (int a = 0; a < 3; ++a) {
            m.xyz[3 * i + a] = c[a];
            m.bmin[a] = std::min(m.bmin[a], c[a]);
            m.bmax[a] = std::max(m.bmax[a], c[a]);
        }
        m.dirichlet[i] = nodes[i]->getBoundaryType() == Mesh::BoundaryType::DIRICHLET ? 1 : 0;
    }
    m.tet.assign(4 * T, 0);
    for (std::size_t t = 0; t < T; ++t) {
        if (!elements[t] || elements[t]->getNodes().size() != 4) return "elements must be 4-node tetrahedra";
        const double v = elements[t]->getVolume();
        for (int k = 0; k < 4; ++k) {
            const auto id = elements[t]->getNodes()[k]->getId();
            if (id >= N || nodes[id] != elements[t]->getNodes()[k]) return "element node not in the node list";
            m.tet[4 * t + k] = (int32_t)id;
            m.cv[id] += 0.25 * v;
        }
    }
    return "";
}

// with no context, the reason of this thread's last failed scdat_create
const char* err_of(scdat_ctx* ctx) { return scdat_last_error(ctx); }

}  // namespace

// ==========================================================================================
// PoissonSolver
// ==========================================================================================
namespace FieldSolver {

struct PoissonSolver::Impl {
    scdat_ctx* ctx = nullptr;
    MeshArrays mesh;
    std::vector<uint8_t> built_dirichlet;
    double built_rtol = 0.0;
    ~Impl()
    {
        if (ctx) scdat_destroy(ctx);
    }
};

PoissonSolver::PoissonSolver(Mesh::VolMeshPtr mesh) : mesh_(std::move(mesh)), impl_(std::make_unique<Impl>()) {}
PoissonSolver::~PoissonSolver() = default;

void PoissonSolver::initialize() { assembleSystem(); }

void PoissonSolver::setMesh(Mesh::VolMeshPtr mesh)
{
    mesh_ = std::move(mesh);
    impl_ = std::make_unique<Impl>();
}

void PoissonSolver::addBoundaryCondition(Mesh::NodeId node_id, BoundaryConditionPtr bc)
{
    if (bc) bcs_[node_id] = std::move(bc);
}
void PoissonSolver::clearBoundaryConditions() { bcs_.clear(); }
void PoissonSolver::setChargeDensity(Mesh::NodeId node_id, double density) { rho_[node_id] = density; }
void PoissonSolver::setChargeDensity(const std::unordered_map<Mesh::NodeId, double>& d)
{
    for (const auto& kv : d) rho_[kv.first] = kv.second;
}
void PoissonSolver::clearChargeDensities() { rho_.clear(); }

// PoissonSolver::assembleSystem (PoissonSolver.cpp:274-385): the device context assembles
// the Dirichlet-reduced system of this mesh and these Dirichlet nodes.
void PoissonSolver::assembleSystem()
{
    error_.clear();
    if (!mesh_) {
        error_ = "no mesh";
        return;
    }
    Impl& I = *impl_;
    std::string e = flatten_mesh(mesh_->getNodes(), mesh_->getElements(), I.mesh);
    if (!e.empty()) {
        error_ = e;
        return;
    }
    for (const auto& kv : bcs_)
        if (kv.first < I.mesh.dirichlet.size() && kv.second->getType() == BoundaryConditionType::DIRICHLET)
            I.mesh.dirichlet[kv.first] = 1;
    if (I.ctx && I.built_dirichlet == I.mesh.dirichlet && I.built_rtol == rtol_) return;
    if (I.ctx) {
        scdat_destroy(I.ctx);
        I.ctx = nullptr;
    }
    scdat_mesh_desc d{};
    d.n_nodes = (int64_t)mesh_->getNodeCount();
    d.n_tets = (int64_t)mesh_->getElementCount();
    d.node_xyz = I.mesh.xyz.data();
    d.tet_nodes = I.mesh.tet.data();
    d.node_dirichlet = I.mesh.dirichlet.data();
    scdat_params p;
    scdat_default_params(&p);
    p.dt = 1.0;
    p.precision = SCDAT_PREC_FP64;
    p.pcg_rtol = rtol_;
    p.pcg_max_iter = std::max<int>(1000, 4 * (int)d.n_nodes);
    p.poisson_charge_sign = -1;
    p.particle_capacity = 1;
    if (scdat_create(&d, &p, &I.ctx) != SCDAT_OK) {
        error_ = std::string("device setup failed: ") + err_of(I.ctx);
        if (I.ctx) scdat_destroy(I.ctx);
        I.ctx = nullptr;
        return;
    }
    I.built_dirichlet = I.mesh.dirichlet;
    I.built_rtol = rtol_;
}

bool PoissonSolver::solve(Solver::SolverType)
{
    assembleSystem();
    Impl& I = *impl_;
    if (!I.ctx) return false;
    const std::size_t N = mesh_->getNodeCount();
    // Dirichlet values: the boundary condition's value, else the node's potential.
    std::vector<double> phi(N, 0.0), rho(N, 0.0);
    std::vector<int64_t> ids(N);
    for (std::size_t i = 0; i < N; ++i) {
        ids[i] = (int64_t)i;
        if (I.mesh.dirichlet[i]) {
            auto it = bcs_.find(i);
            phi[i] = (it != bcs_.end()) ? it->second->getValue() : mesh_->getNodes()[i]->getPotential();
        }
    }
    for (const auto& kv : rho_)
        if (kv.first < N) rho[kv.first] = kv.second;
    int rc = scdat_set_node_potentials(I.ctx, (int64_t)N, ids.data(), phi.data());
    if (rc == SCDAT_OK) rc = scdat_set_charge_density(I.ctx, rho.data());
    if (rc == SCDAT_OK) rc = scdat_solve_field(I.ctx);
    if (rc != SCDAT_OK) {
        error_ = err_of(I.ctx);
        return false;
    }
    std::vector<double> E(3 * N);
    phi_.assign(N, 0.0);
    if (scdat_get_fields(I.ctx, nullptr, phi_.data(), E.data()) != SCDAT_OK) {
        error_ = err_of(I.ctx);
        return false;
    }
    field_.resize(N);
    // updateNodePotentials / updateNodeElectricFields (PoissonSolver.cpp:440-529)
    for (std::size_t i = 0; i < N; ++i) {
        field_[i] = Utils::Vector3D(E[3 * i], E[3 * i + 1], E[3 * i + 2]);
        mesh_->getNodes()[i]->setPotential(phi_[i]);
        mesh_->getNodes()[i]->setElectricField(field_[i]);
    }
    return true;
}

double PoissonSolver::getPotential(Mesh::NodeId node_id) const { return node_id < phi_.size() ? phi_[node_id] : 0.0; }

Utils::Vector3D PoissonSolver::getElectricField(Mesh::NodeId node_id) const
{
    return node_id < field_.size() ? field_[node_id] : Utils::Vector3D();
}

// 0.5 eps0 |E_i|^2 times the nodal control volume (PoissonSolver.cpp:531-560)
double PoissonSolver::getTotalEnergy() const
{
    constexpr double eps0 = 8.8541878128e-12;
    double s = 0.0;
    for (std::size_t i = 0; i < field_.size() && i < impl_->mesh.cv.size(); ++i)
        s += 0.5 * eps0 * field_[i].magnitudeSquared() * impl_->mesh.cv[i];
    return s;
}

double PoissonSolver::getMaxPotential() const
{
    return phi_.empty() ? 0.0 : *std::max_element(phi_.begin(), phi_.end());
}
double PoissonSolver::getMinPotential() const
{
    return phi_.empty() ? 0.0 : *std::min_element(phi_.begin(), phi_.end());
}
Utils::Vector3D PoissonSolver::getMaxElectricField() const
{
    Utils::Vector3D best;
    for (const auto& e : field_)
        if (e.magnitudeSquared() > best.magnitudeSquared()) best = e;
    return best;
}

}  // namespace FieldSolver

// ==========================================================================================
// PICCycle
// ==========================================================================================
namespace PICcore {

using Particle::ParticleStatus;
using Particle::ParticleType;

namespace {
struct SpeciesKey {
    double charge, mass, weight;
    bool electron_like;
    bool operator==(const SpeciesKey& o) const
    {
        return charge == o.charge && mass == o.mass && weight == o.weight && electron_like == o.electron_like;
    }
};
constexpr int kMaxSpecies = 16;
}  // namespace

struct PICCycle::Impl final : Particle::DeviceMirror {
    Parameters params;
    DeviceOptions opts;
    std::vector<Mesh::NodePtr> nodes;
    std::vector<Mesh::ElementPtr> elements;
    std::shared_ptr<ParticleManager> pm;
    std::shared_ptr<PoissonSolver> solver;
    std::array<BoundaryConditionPtr, 6> bc{};
    std::array<SurfaceBoundaryMetadata, 6> meta{};
    std::unordered_map<Particle::ParticleId, ElementId> location;

    MeshArrays mesh;
    scdat_ctx* ctx = nullptr;
    bool initialized = false;
    std::vector<SpeciesKey> species;
    std::uint64_t uploaded_version = 0;
    bool device_ahead = false;
    int steps_since_compact = 0;
    std::string error;

    // host copies of the device results
    mutable bool fields_stale = true;
    mutable std::vector<double> rho, phi;
    mutable std::vector<Utils::Vector3D> E;
    CycleStatistics stats;
    std::array<SurfaceCurrentLedgerEntry, 6> ledger{};
    // tallies folded in from earlier device contexts (a new species set needs a new context)
    std::array<double, 6 * 8> ledger_base{};
    double surface_base = 0.0, surface_taken = 0.0;
    int64_t steps_base = 0;
    double time_base = 0.0;
    double wall_total = 0.0;

    ~Impl() override { release(); }

    void release()
    {
        if (pm && pm->getContainer().deviceMirror() == this) {
            pull();
            pm->getContainer().setDeviceMirror(nullptr);
        }
        if (ctx) scdat_destroy(ctx);
        ctx = nullptr;
    }

    bool fail(const std::string& why)
    {
        error = why;
        return false;
    }

    bool create_context()
    {
        scdat_mesh_desc d{};
        d.n_nodes = (int64_t)nodes.size();
        d.n_tets = (int64_t)elements.size();
        d.node_xyz = mesh.xyz.data();
        d.tet_nodes = mesh.tet.data();
        d.node_dirichlet = mesh.dirichlet.data();
        scdat_params p;
        scdat_default_params(&p);
        p.dt = params.time_step;
        p.deposit_kernel = (int)params.trajectory_charge_deposition_kernel == 0   ? SCDAT_DEP_NEAREST
                           : (int)params.trajectory_charge_deposition_kernel == 2 ? SCDAT_DEP_GAUSS3
                                                                                  : SCDAT_DEP_LINEAR;
        p.deposit_segments = (int)std::max<std::size_t>(1, params.trajectory_charge_deposition_segments);
        p.precision = opts.mixed_precision ? SCDAT_PREC_MIXED : SCDAT_PREC_FP64;
        p.pcg_rtol = opts.pcg_rtol;
        p.pcg_max_iter = opts.pcg_max_iter;
        p.poisson_charge_sign = opts.poisson_charge_sign;
        p.body_tally = opts.body_tally ? 1 : 0;
        p.sort_interval = 0;  // compaction is driven from here, after the host has the statuses
        for (int f = 0; f < 6; ++f) {
            p.face_bc[f] = SCDAT_BC_NONE;
            if (std::dynamic_pointer_cast<Particle::AbsorbingBoundaryCondition>(bc[f])) p.face_bc[f] = SCDAT_BC_ABSORB;
            if (std::dynamic_pointer_cast<Particle::PeriodicBoundaryCondition>(bc[f])) p.face_bc[f] = SCDAT_BC_PERIODIC;
        }
        std::size_t n = pm ? pm->getContainer().deviceWriteAccess().size() : 0;
        p.particle_capacity = (int64_t)std::max<std::size_t>(n + n / 4 + 1024, 4096);
        if (scdat_create(&d, &p, &ctx) != SCDAT_OK) {
            std::string why = std::string("device setup failed: ") + err_of(ctx);
            if (ctx) scdat_destroy(ctx);
            ctx = nullptr;
            return fail(why);
        }
        return true;
    }

    std::string check_boundaries() const
    {
        for (int f = 0; f < 6; ++f) {
            if (!bc[f]) continue;
            if (auto a = std::dynamic_pointer_cast<Particle::AbsorbingBoundaryCondition>(bc[f])) {
                if (a->getAbsorptionProbability() != 1.0)
                    return "only full absorption (probability 1) runs on the device";
                continue;
            }
            if (auto pb = std::dynamic_pointer_cast<Particle::PeriodicBoundaryCondition>(bc[f])) {
                const int axis = f / 2;
                bool ok = false;
                for (const auto& v : pb->getPeriodVectors()) {
                    const double c[3] = {v.x(), v.y(), v.z()};
                    const double L = mesh.bmax[axis] - mesh.bmin[axis];
                    if (std::fabs(c[axis] - L) <= 1e-9 * std::max(1.0, L) &&
                        std::fabs(c[(axis + 1) % 3]) + std::fabs(c[(axis + 2) % 3]) == 0.0)
                        ok = true;
                }
                if (!ok) return "a periodic face needs a period vector equal to the box length on its axis";
                continue;
            }
            return "unsupported particle boundary condition type";
        }
        return "";
    }

    // ---- DeviceMirror ----------------------------------------------------------------
    void pull() override
    {
        if (!device_ahead || !ctx || !pm) return;
        device_ahead = false;
        auto& parts = pm->getContainer().deviceWriteAccess();
        for (int s = 0; s < (int)species.size(); ++s) {
            int64_t n = 0;
            if (scdat_get_particle_count(ctx, s, &n) != SCDAT_OK || n == 0) continue;
            std::vector<double> x((size_t)n * 3), v((size_t)n * 3);
            std::vector<int32_t> tet((size_t)n);
            std::vector<uint8_t> st((size_t)n);
            std::vector<uint32_t> ids((size_t)n);
            int64_t got = 0;
            if (scdat_get_particles(ctx, s, n, x.data(), v.data(), tet.data(), st.data(), ids.data(), &got) != SCDAT_OK)
                continue;
            for (int64_t i = 0; i < got; ++i) {
                if (ids[i] >= parts.size()) continue;
                auto& p = parts[ids[i]];
                p.setPosition({x[3 * i], x[3 * i + 1], x[3 * i + 2]});
                p.setVelocity({v[3 * i], v[3 * i + 1], v[3 * i + 2]});
                p.setStatus(st[i] == SCDAT_ACTIVE     ? ParticleStatus::ACTIVE
                            : st[i] == SCDAT_ABSORBED ? ParticleStatus::ABSORBED
                                                      : ParticleStatus::ESCAPED);
                if (tet[i] >= 0) location[p.getId()] = (ElementId)tet[i];
            }
        }
    }

    void compact() override
    {
        if (!ctx) return;
        pull();
        scdat_compact(ctx);
        steps_since_compact = 0;
        // device ids index the container as uploaded; the host removal re-indexes it, so the
        // next step uploads again (the container's version moved)
    }

    bool collide(const std::vector<Collision::ElasticProcess>& procs, std::uint64_t seed, double dt,
                 std::size_t& collisions, std::string& why) override
    {
        collisions = 0;
        if (!ensure_uploaded()) {
            why = error;
            return false;
        }
        if (!ctx) return true;
        const bool same_dt = dt == params.time_step;
        if (!same_dt) {
            why = "the device MCC step uses the cycle's time step";
            return false;
        }
        scdat_set_seed(ctx, seed);
        for (int s = 0; s < (int)species.size(); ++s) {
            scdat_elastic e{};
            for (const auto& pr : procs) {
                const bool electron = pr.projectile == ParticleType::ELECTRON;
                if (electron != species[s].electron_like) continue;
                e.target_density = pr.target_density_m3;
                e.sigma_max = pr.sigma_max_m2;
                e.e_ref_ev = pr.reference_energy_ev;
                e.alpha = pr.power_index;
                e.e_threshold_ev = pr.threshold_ev;
                e.enabled = 1;
                e.mode = 0;
            }
            if (scdat_set_elastic_mcc(ctx, s, &e) != SCDAT_OK) {
                why = err_of(ctx);
                return false;
            }
        }
        scdat_stats before{}, after{};
        scdat_get_statistics(ctx, &before);
        if (scdat_collide(ctx) != SCDAT_OK) {
            why = err_of(ctx);
            return false;
        }
        scdat_get_statistics(ctx, &after);
        collisions = (std::size_t)(after.mcc_collisions - before.mcc_collisions);
        // PICCycle steps do not collide on their own: switch the processes off again
        for (int s = 0; s < (int)species.size(); ++s) {
            scdat_elastic off{};
            scdat_set_elastic_mcc(ctx, s, &off);
        }
        device_ahead = true;
        return true;
    }

    // ---- host -> device -------------------------------------------------------------
    bool ensure_uploaded()
    {
        if (!pm) return fail("no particle manager");
        auto& cont = pm->getContainer();
        if (cont.deviceMirror() != this) cont.setDeviceMirror(this);
        if (uploaded_version == cont.version()) return true;
        pull();
        auto& parts = cont.deviceWriteAccess();
        // species = distinct (charge, mass, weight) of the active particles
        std::vector<SpeciesKey> want = species;
        std::vector<int> of(parts.size(), -1);
        for (std::size_t i = 0; i < parts.size(); ++i) {
            const auto& p = parts[i];
            if (!p.isActive()) continue;
            SpeciesKey k{p.getCharge(), p.getMass(), p.getWeight(), p.getType() == ParticleType::ELECTRON};
            auto it = std::find(want.begin(), want.end(), k);
            if (it == want.end()) {
                if ((int)want.size() == kMaxSpecies) return fail("more than 16 distinct (charge, mass, weight) species");
                want.push_back(k);
                it = want.end() - 1;
            }
            of[i] = (int)(it - want.begin());
        }
        if (want.empty()) {  // nothing was ever uploaded and nothing is active
            uploaded_version = cont.version();
            return true;
        }
        if (want.size() != species.size()) {
            if (!species.empty()) {
                // a new species set needs a fresh context: keep its tallies and potential
                fold_tallies();
                std::vector<double> keep_phi((size_t)nodes.size());
                scdat_get_fields(ctx, nullptr, keep_phi.data(), nullptr);
                scdat_destroy(ctx);
                ctx = nullptr;
                if (!create_context()) return false;
                if (scdat_set_potential(ctx, keep_phi.data()) != SCDAT_OK) return fail(err_of(ctx));
            }
            std::vector<scdat_species> sp(want.size());
            for (std::size_t s = 0; s < want.size(); ++s) {
                sp[s].charge = want[s].charge;
                sp[s].mass = want[s].mass;
                sp[s].weight = want[s].weight;
                sp[s].electron_like = want[s].electron_like ? 1 : 0;
            }
            if (scdat_set_species(ctx, (int32_t)sp.size(), sp.data()) != SCDAT_OK) return fail(err_of(ctx));
            species = want;
        }
        for (int s = 0; s < (int)species.size(); ++s) {
            std::vector<double> x, v;
            std::vector<int32_t> hint;
            std::vector<uint32_t> ids;
            for (std::size_t i = 0; i < parts.size(); ++i) {
                if (of[i] != s) continue;
                const auto& p = parts[i];
                x.insert(x.end(), {p.getPosition().x(), p.getPosition().y(), p.getPosition().z()});
                v.insert(v.end(), {p.getVelocity().x(), p.getVelocity().y(), p.getVelocity().z()});
                auto it = location.find(p.getId());
                hint.push_back(it == location.end() ? -1 : (int32_t)it->second);
                ids.push_back((uint32_t)i);
            }
            if (scdat_set_particles(ctx, s, (int64_t)ids.size(), x.data(), v.data(), hint.data(), ids.data()) !=
                SCDAT_OK)
                return fail(err_of(ctx));
        }
        uploaded_version = cont.version();
        return true;
    }

    void fold_tallies()
    {
        if (!ctx) return;
        std::array<double, 7 * 8> L{};
        scdat_get_ledger(ctx, L.data());
        for (int i = 0; i < 6 * 8; ++i) ledger_base[i] += L[i];
        scdat_stats s{};
        scdat_get_statistics(ctx, &s);
        surface_base += s.surface_deposited_charge;
        steps_base += s.completed_steps;
        time_base += s.simulation_time;
    }

    void refresh_tallies()
    {
        std::array<double, 7 * 8> L{};
        if (ctx) scdat_get_ledger(ctx, L.data());
        for (int f = 0; f < 6; ++f) {
            const double* r = L.data() + 8 * f;
            const double* b = ledger_base.data() + 8 * f;
            auto& e = ledger[f];
            e.metadata = meta[f];
            e.absorbed_electron_charge_c = r[0] + b[0];
            e.absorbed_ion_charge_c = r[1] + b[1];
            e.emitted_electron_charge_c = r[2] + b[2];
            e.incident_energy_j = r[3] + b[3];
            e.absorbed_electron_particles = (std::size_t)(r[4] + b[4]);
            e.absorbed_ion_particles = (std::size_t)(r[5] + b[5]);
            e.emitted_electron_particles = (std::size_t)(r[6] + b[6]);
        }
        scdat_stats s{};
        if (ctx) scdat_get_statistics(ctx, &s);
        stats.completed_steps = (int)(s.completed_steps + steps_base);
        stats.simulation_time = s.simulation_time + time_base;
        stats.total_charge = s.total_charge;
        stats.total_energy = s.total_energy;
        stats.active_particles = (int)s.active_particles;
        stats.surface_deposited_charge = s.surface_deposited_charge + surface_base - surface_taken;
        stats.average_step_time = stats.completed_steps ? wall_total / stats.completed_steps : 0.0;
    }

    void fetch_fields() const
    {
        if (!fields_stale || !ctx) return;
        const std::size_t N = nodes.size();
        rho.assign(N, 0.0);
        phi.assign(N, 0.0);
        std::vector<double> e(3 * N, 0.0);
        scdat_get_fields(ctx, rho.data(), phi.data(), e.data());
        E.resize(N);
        for (std::size_t i = 0; i < N; ++i) E[i] = Utils::Vector3D(e[3 * i], e[3 * i + 1], e[3 * i + 2]);
        fields_stale = false;
    }
};

PICCycle::PICCycle() : impl_(std::make_unique<Impl>()) {}
PICCycle::PICCycle(const Parameters& params) : impl_(std::make_unique<Impl>()) { impl_->params = params; }
PICCycle::~PICCycle() = default;
PICCycle::PICCycle(PICCycle&&) noexcept = default;
PICCycle& PICCycle::operator=(PICCycle&&) noexcept = default;

void PICCycle::setMesh(const std::vector<Mesh::NodePtr>& nodes, const std::vector<Mesh::ElementPtr>& elements)
{
    impl_->nodes = nodes;
    impl_->elements = elements;
    impl_->initialized = false;
}
void PICCycle::setParticleManager(std::shared_ptr<ParticleManager> pm)
{
    if (impl_->pm && impl_->pm->getContainer().deviceMirror() == impl_.get()) {
        impl_->pull();
        impl_->pm->getContainer().setDeviceMirror(nullptr);
    }
    impl_->pm = std::move(pm);
    impl_->uploaded_version = 0;
}
void PICCycle::setPoissonSolver(std::shared_ptr<PoissonSolver> solver) { impl_->solver = std::move(solver); }
void PICCycle::setBoundaryCondition(BoundaryFace face, BoundaryConditionPtr condition)
{
    impl_->bc[(int)face] = std::move(condition);
    impl_->initialized = false;
}
void PICCycle::clearBoundaryConditions()
{
    impl_->bc = {};
    impl_->initialized = false;
}

void PICCycle::addParticleLocation(ParticlePtr particle, ElementId element_id)
{
    if (particle) impl_->location[particle->getId()] = element_id;
}
void PICCycle::updateParticleLocation(ParticlePtr particle, ElementId element_id)
{
    addParticleLocation(particle, element_id);
}
ElementId PICCycle::findParticleElement(ParticlePtr particle) const
{
    if (!particle) return static_cast<ElementId>(-1);
    impl_->pull();
    auto it = impl_->location.find(particle->getId());
    return it == impl_->location.end() ? static_cast<ElementId>(-1) : it->second;
}

// PICCycle::initialize (PICCycle.cpp:255-309): the device context takes the mesh, the face
// conditions and the Dirichlet node set; particles are mirrored at the first step.
bool PICCycle::initialize()
{
    Impl& I = *impl_;
    if (I.nodes.empty() || I.elements.empty() || !I.pm || !I.solver)
        return I.fail("PICCycle initialization failed: missing required components");
    if (I.initialized && I.ctx) return true;
    std::string e = flatten_mesh(I.nodes, I.elements, I.mesh);
    if (!e.empty()) return I.fail(e);
    e = I.check_boundaries();
    if (!e.empty()) return I.fail(e);
    if (I.ctx) {
        I.fold_tallies();
        scdat_destroy(I.ctx);
        I.ctx = nullptr;
    }
    I.species.clear();
    I.uploaded_version = 0;
    if (!I.create_context()) return false;
    // potential from the nodes (Dirichlet values included)
    std::vector<double> phi(I.nodes.size());
    for (std::size_t i = 0; i < phi.size(); ++i) phi[i] = I.nodes[i]->getPotential();
    if (scdat_set_potential(I.ctx, phi.data()) != SCDAT_OK) return I.fail(err_of(I.ctx));
    I.fields_stale = true;
    I.initialized = true;
    I.refresh_tallies();
    return true;
}

// PICCycle::executeTimeStep (PICCycle.cpp:311-416) on the device.  Returns true after a
// completed step (the reference's convergence check never ends the loop).
bool PICCycle::executeTimeStep()
{
    Impl& I = *impl_;
    if (!I.initialized && !initialize()) return false;
    if (!I.ensure_uploaded()) return false;
    const auto t0 = std::chrono::steady_clock::now();
    if (!I.species.empty()) {
        if (scdat_step(I.ctx, 1) != SCDAT_OK) return I.fail(err_of(I.ctx));
        I.device_ahead = true;
    } else {
        // no particles: the field solve still runs on the (empty) charge
        if (scdat_push(I.ctx) != SCDAT_OK || scdat_solve_field(I.ctx) != SCDAT_OK) return I.fail(err_of(I.ctx));
        I.steps_base += 1;
        I.time_base += I.params.time_step;
    }
    I.wall_total += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    I.fields_stale = true;
    if (I.opts.compact_interval > 0 && ++I.steps_since_compact >= I.opts.compact_interval) I.compact();
    I.refresh_tallies();
    return true;
}

bool PICCycle::executeSimulation(double total_time)
{
    if (!initialize()) return false;
    const int total_steps = static_cast<int>(total_time / impl_->params.time_step);
    for (int step = 0; step < total_steps; ++step) {
        if (!executeTimeStep()) return false;
        if (impl_->stats.completed_steps >= impl_->params.max_iterations) break;
    }
    return true;
}

const std::vector<double>& PICCycle::getChargeDensity() const
{
    impl_->fetch_fields();
    return impl_->rho;
}
const std::vector<double>& PICCycle::getPotential() const
{
    impl_->fetch_fields();
    return impl_->phi;
}
const std::vector<Utils::Vector3D>& PICCycle::getElectricField() const
{
    impl_->fetch_fields();
    return impl_->E;
}

void PICCycle::setTimeStep(double dt)
{
    if (!(dt > 0.0)) return;
    impl_->params.time_step = dt;
    if (impl_->ctx) scdat_set_dt(impl_->ctx, dt);
}
double PICCycle::getTimeStep() const { return impl_->params.time_step; }

// PICCycle::setPotential (PICCycle.h:105-120): node potentials, then the field by LSQ.
void PICCycle::setPotential(const std::vector<double>& potential)
{
    Impl& I = *impl_;
    if (I.nodes.size() == potential.size())
        for (std::size_t i = 0; i < I.nodes.size(); ++i)
            if (I.nodes[i]) I.nodes[i]->setPotential(potential[i]);
    if (I.ctx && potential.size() == I.nodes.size()) {
        if (scdat_set_potential(I.ctx, potential.data()) != SCDAT_OK) I.error = err_of(I.ctx);
        I.fields_stale = true;
    }
}

void PICCycle::setNodePotential(std::size_t node_id, double value)
{
    Impl& I = *impl_;
    if (node_id >= I.nodes.size()) return;
    I.nodes[node_id]->setPotential(value);
    if (I.ctx) {
        const int64_t id = (int64_t)node_id;
        if (scdat_set_node_potentials(I.ctx, 1, &id, &value) != SCDAT_OK) I.error = err_of(I.ctx);
        I.fields_stale = true;
    }
}

const PICCycle::CycleStatistics& PICCycle::getStatistics() const { return impl_->stats; }
void PICCycle::setBoundaryMetadata(BoundaryFace face, const SurfaceBoundaryMetadata& metadata)
{
    impl_->meta[(int)face] = metadata;
    impl_->ledger[(int)face].metadata = metadata;
}
const std::array<PICCycle::SurfaceCurrentLedgerEntry, 6>& PICCycle::getSurfaceCurrentLedger() const
{
    return impl_->ledger;
}
double PICCycle::getAndResetSurfaceCharge()
{
    const double q = impl_->stats.surface_deposited_charge;
    impl_->surface_taken += q;
    impl_->stats.surface_deposited_charge = 0.0;
    return q;
}

void PICCycle::setDeviceOptions(const DeviceOptions& options)
{
    impl_->opts = options;
    impl_->initialized = false;
}
const std::string& PICCycle::lastError() const { return impl_->error; }

}  // namespace PICcore

// ==========================================================================================
// Background MCC
// ==========================================================================================
namespace Collision {

MonteCarloCollisionHandler::MonteCarloCollisionHandler(std::uint64_t seed) : seed_(seed) {}

void MonteCarloCollisionHandler::addElasticProcess(const ElasticProcess& p)
{
    if (!(p.sigma_max_m2 >= 0.0) || !(p.target_density_m3 >= 0.0))
        throw std::invalid_argument("elastic process needs non-negative density and cross-section");
    elastic_.push_back(p);
}

void MonteCarloCollisionHandler::clearProcesses()
{
    elastic_.clear();
    unsupported_.clear();
}

// estimateCollisionBackgroundDensities (CollisionPicAdapter.cpp:212-261): the floors (a
// non-finite or negative floor counts as 0, sanitizeDensity at :58-65), raised by the weight
// densities of the container's active particles by class: electron-like (ELECTRON, or any
// negative charge), ion-like (PROTON, ION, or any positive charge) and neutral (the rest), as
// isElectronLike / isIonLike (:23-56) classify the types this layer knows.
namespace {
double sanitize_density(double d) { return std::isfinite(d) ? std::max(0.0, d) : 0.0; }

std::string lower_case(std::string t)
{
    std::transform(t.begin(), t.end(), t.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return t;
}
}  // namespace

CollisionBackgroundDensities estimateCollisionBackgroundDensities(const Particle::ParticleContainer& container,
                                                                  double volume_m3,
                                                                  const CollisionBackgroundDensities& floor)
{
    CollisionBackgroundDensities d{};
    d.neutral_density_m3 = sanitize_density(floor.neutral_density_m3);
    d.ion_density_m3 = sanitize_density(floor.ion_density_m3);
    d.electron_density_m3 = sanitize_density(floor.electron_density_m3);
    if (!(volume_m3 > 0.0) || !std::isfinite(volume_m3)) return d;
    double ne = 0.0, ni = 0.0, nn = 0.0;
    for (const auto& p : container) {
        if (!p.isActive()) continue;
        const double w = std::max(0.0, p.getWeight());
        const auto t = p.getType();
        if (t == Particle::ParticleType::ELECTRON || p.getCharge() < 0.0)
            ne += w;
        else if (t == Particle::ParticleType::PROTON || t == Particle::ParticleType::ION || p.getCharge() > 0.0)
            ni += w;
        else
            nn += w;
    }
    const double inv = 1.0 / volume_m3;
    d.electron_density_m3 = std::max(d.electron_density_m3, ne * inv);
    d.ion_density_m3 = std::max(d.ion_density_m3, ni * inv);
    d.neutral_density_m3 = std::max(d.neutral_density_m3, nn * inv);
    return d;
}

// parseCollisionCrossSectionSetId (CollisionPicAdapter.cpp:263-282): case-insensitive, with the
// reference's aliases of each set.
std::optional<CollisionCrossSectionSetId> parseCollisionCrossSectionSetId(const std::string& text)
{
    const std::string n = lower_case(text);
    if (n == "background_mcc_v1" || n == "backgroundmccv1" || n == "default" || n == "background")
        return CollisionCrossSectionSetId::BackgroundMccV1;
    if (n == "surface_pic_v1" || n == "surfacepicv1" || n == "surface_pic" || n == "surfacepic")
        return CollisionCrossSectionSetId::SurfacePicV1;
    if (n == "vacuum_arc_pic_v1" || n == "vacuumarcpicv1" || n == "arcpic_background_v1" || n == "arcpic")
        return CollisionCrossSectionSetId::VacuumArcPicV1;
    return std::nullopt;
}

std::string toString(CollisionCrossSectionSetId id)
{
    switch (id) {
    case CollisionCrossSectionSetId::SurfacePicV1: return "surface_pic_v1";
    case CollisionCrossSectionSetId::VacuumArcPicV1: return "vacuum_arc_pic_v1";
    default: return "background_mcc_v1";
    }
}

// The reference's named sets (CollisionPicAdapter.cpp:298-323) hold ionisation, excitation and
// charge-exchange processes beside elastic scattering.  The device path implements elastic
// scattering only, so a configured set is recorded as unsupported and refuses to run on
// particles.
void initializeConfiguredCollisionHandler(MonteCarloCollisionHandler& handler, CollisionCrossSectionSetId set_id,
                                          double, double, double)
{
    handler.clearProcesses();
    handler.markUnsupported("cross-section set " + toString(set_id));
}

CollisionStepResult executeBackgroundMccStep(Particle::ParticleContainer& container,
                                             MonteCarloCollisionHandler& handler, double dt, double volume_m3,
                                             const BackgroundMccRuntimeConfig& cfg)
{
    CollisionStepResult result{};
    if (!(dt > 0.0) || !std::isfinite(dt) || !(volume_m3 > 0.0) || !std::isfinite(volume_m3)) return result;
    const auto d = estimateCollisionBackgroundDensities(container, volume_m3, cfg.floor_densities);
    result.effective_neutral_density_m3 = d.neutral_density_m3;
    result.effective_ion_density_m3 = d.ion_density_m3;
    result.effective_electron_density_m3 = d.electron_density_m3;
    if (cfg.reinitialize_configuration)
        initializeConfiguredCollisionHandler(handler, cfg.cross_section_set_id, d.neutral_density_m3,
                                             d.ion_density_m3, d.electron_density_m3);
    result.active_particles = container.getActiveCount();
    if (result.active_particles == 0) return result;
    if (!handler.unsupportedProcesses().empty())
        throw std::invalid_argument("collision process not implemented on the device path: " +
                                    handler.unsupportedProcesses().front());
    Particle::DeviceMirror* mirror = container.deviceMirror();
    if (!mirror) throw std::invalid_argument("the container is not mirrored on the device (attach it to a PICCycle)");
    std::size_t events = 0;
    std::string why;
    if (!mirror->collide(handler.elasticProcesses(), handler.seed(), dt, events, why))
        throw std::runtime_error("device MCC step failed: " + why);
    auto& st = handler.mutableStatistics();
    st.total_collisions += (long long)events;
    st.collision_counts["elastic"] += (int)events;
    result.collision_events = events;
    container.removeInactiveParticles();
    return result;
}

CollisionStepResult executeBackgroundMccStep(Particle::ParticleContainer& container,
                                             MonteCarloCollisionHandler& handler, double dt, double volume_m3,
                                             const CollisionBackgroundDensities& floor_densities,
                                             bool reinitialize_configuration)
{
    BackgroundMccRuntimeConfig cfg;
    cfg.floor_densities = floor_densities;
    cfg.reinitialize_configuration = reinitialize_configuration;
    return executeBackgroundMccStep(container, handler, dt, volume_m3, cfg);
}

}  // namespace Collision
}  // namespace SCDAT
