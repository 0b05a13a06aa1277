// scdat_host.hpp -- C++20 host layer over the scdat_b200 C ABI that keeps the class
// interfaces of SCDAT's PIC path, so callers written against Tools/PICcore, Tools/Particle,
// Tools/FieldSolver and Tools/Interactions recompile against this header unchanged for the
// members they use on that path.
//
// Mirrored interfaces (reference paths inside the SCDAT tree):
//   SCDAT::PICcore::PICCycle                  Tools/PICcore/include/PICCycle.h:29-185
//   SCDAT::FieldSolver::PoissonSolver         Tools/FieldSolver/include/PoissonSolver.h:26-67
//   SCDAT::Particle::ParticleManager          Tools/Particle/include/ParticleManager.h:821-900
//   SCDAT::Particle::ParticleContainer        Tools/Particle/include/ParticleManager.h:55-146
//   SCDAT::Particle::Particle                 Tools/Particle/include/ParticleDefinitions.h:315-
//   SCDAT::Particle::{Absorbing,Periodic}BoundaryCondition
//                                             Tools/Boundary/include/BoundaryConditions.h:188-392
//   SCDAT::Mesh::{Node,TetrahedronElement,VolMesh}
//                                             Tools/Mesh/include/MeshAlgorithms.h:68-290,
//                                             Tools/Mesh/include/MeshParsing.h:152-155
//   SCDAT::Collision::{MonteCarloCollisionHandler, executeBackgroundMccStep, ...}
//                                             Tools/Interactions/Collisions/include/CollisionPicAdapter.h:20-110
//
// Every numerical step runs on the GPU through the C ABI (include/scdat_b200.h).  The host
// layer only keeps the reference's object model: it mirrors the ParticleContainer into the
// device store when the host copy changed, runs the step on the device, and copies particle
// state, fields and tallies back so that the reference's accessors see them.  Errors follow
// the reference: bool returns for the cycle and solver, std::invalid_argument for bad
// construction arguments, and a one-line reason from lastError().
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

namespace SCDAT {

// ------------------------------------------------------------------------------------------
// Geometry (Tools/Geometry/include/Point3D.h, Vector3D.h)
// ------------------------------------------------------------------------------------------
namespace Geometry {

class Vector3D {
  public:
    constexpr Vector3D() = default;
    constexpr Vector3D(double x, double y, double z) : x_(x), y_(y), z_(z) {}
    constexpr double x() const { return x_; }
    constexpr double y() const { return y_; }
    constexpr double z() const { return z_; }
    double magnitude() const { return std::sqrt(magnitudeSquared()); }
    constexpr double magnitudeSquared() const { return x_ * x_ + y_ * y_ + z_ * z_; }
    constexpr double dot(const Vector3D& o) const { return x_ * o.x_ + y_ * o.y_ + z_ * o.z_; }
    constexpr Vector3D operator+(const Vector3D& o) const { return {x_ + o.x_, y_ + o.y_, z_ + o.z_}; }
    constexpr Vector3D operator-(const Vector3D& o) const { return {x_ - o.x_, y_ - o.y_, z_ - o.z_}; }
    constexpr Vector3D operator*(double s) const { return {x_ * s, y_ * s, z_ * s}; }

  private:
    double x_ = 0.0, y_ = 0.0, z_ = 0.0;
};

class Point3D {
  public:
    constexpr Point3D() = default;
    constexpr Point3D(double x, double y, double z) : x_(x), y_(y), z_(z) {}
    constexpr double x() const { return x_; }
    constexpr double y() const { return y_; }
    constexpr double z() const { return z_; }
    constexpr Point3D operator+(const Vector3D& v) const { return {x_ + v.x(), y_ + v.y(), z_ + v.z()}; }
    constexpr Vector3D operator-(const Point3D& o) const { return {x_ - o.x_, y_ - o.y_, z_ - o.z_}; }

  private:
    double x_ = 0.0, y_ = 0.0, z_ = 0.0;
};

}  // namespace Geometry

namespace Utils {
using Geometry::Point3D;
using Geometry::Vector3D;
}  // namespace Utils

// ------------------------------------------------------------------------------------------
// Mesh (Tools/Mesh/include/MeshAlgorithms.h:31-35,68-290; MeshParsing.h:152-155)
// ------------------------------------------------------------------------------------------
namespace Mesh {

using NodeId = std::size_t;
using ElementId = std::size_t;
using MaterialId = std::size_t;

enum class BoundaryType { INTERIOR = 0, DIRICHLET = 1, NEUMANN = 2, PERIODIC = 3 };

class Node {
  public:
    Node(NodeId id, const Utils::Point3D& position) : id_(id), position_(position) {}
    NodeId getId() const { return id_; }
    const Utils::Point3D& getPosition() const { return position_; }
    BoundaryType getBoundaryType() const { return boundary_type_; }
    void setBoundaryType(BoundaryType type) { boundary_type_ = type; }
    double getPotential() const { return potential_; }
    void setPotential(double potential) { potential_ = potential; }
    const Utils::Vector3D& getElectricField() const { return electric_field_; }
    void setElectricField(const Utils::Vector3D& field) { electric_field_ = field; }
    double getChargeDensity() const { return charge_density_; }
    void setChargeDensity(double density) { charge_density_ = density; }

  private:
    NodeId id_;
    Utils::Point3D position_;
    BoundaryType boundary_type_ = BoundaryType::INTERIOR;
    double potential_ = 0.0;
    Utils::Vector3D electric_field_{};
    double charge_density_ = 0.0;
};
using NodePtr = std::shared_ptr<Node>;

// A 4-node linear tetrahedron (TetrahedronElement, MeshAlgorithms.h:236-250).
class TetrahedronElement {
  public:
    TetrahedronElement(ElementId id, std::vector<NodePtr> nodes);
    ElementId getId() const { return id_; }
    const std::vector<NodePtr>& getNodes() const { return nodes_; }
    MaterialId getMaterialId() const { return material_id_; }
    void setMaterialId(MaterialId material_id) { material_id_ = material_id; }
    double getVolume() const;
    Utils::Point3D getCentroid() const;

  private:
    ElementId id_;
    std::vector<NodePtr> nodes_;
    MaterialId material_id_ = 0;
};
using Element = TetrahedronElement;
using ElementPtr = std::shared_ptr<TetrahedronElement>;

// VolMesh (MeshParsing.h:140-200): node and element lists with ids equal to their index.
class VolMesh {
  public:
    NodeId addNode(const Utils::Point3D& position);
    ElementId addElement(const std::array<NodeId, 4>& node_ids);  // throws std::out_of_range
    const std::vector<NodePtr>& getNodes() const { return nodes_; }
    const std::vector<ElementPtr>& getElements() const { return elements_; }
    std::size_t getNodeCount() const { return nodes_.size(); }
    std::size_t getElementCount() const { return elements_.size(); }
    NodePtr getNode(NodeId id) const { return id < nodes_.size() ? nodes_[id] : nullptr; }
    ElementPtr getElement(ElementId id) const { return id < elements_.size() ? elements_[id] : nullptr; }
    Utils::Point3D getBoundingBoxMin() const;
    Utils::Point3D getBoundingBoxMax() const;
    // Every element has positive volume and valid node ids.
    bool validate() const;

    // nx*ny*nz hexes over [0,lx]x[0,ly]x[0,lz], 6 conforming tets each (the Kuhn split the
    // device mesher scdat_kuhn_box_mesh builds), node ids i + (nx+1)*(j + (ny+1)*k).
    static std::unique_ptr<VolMesh> createKuhnBox(int nx, int ny, int nz, double lx, double ly, double lz);

  private:
    std::vector<NodePtr> nodes_;
    std::vector<ElementPtr> elements_;
};
using VolMeshPtr = std::shared_ptr<VolMesh>;

}  // namespace Mesh

// ------------------------------------------------------------------------------------------
// Particles (Tools/Particle/include/ParticleDefinitions.h:70-306, ParticleManager.h:55-900)
// ------------------------------------------------------------------------------------------
namespace Particle {

using ParticleId = std::uint64_t;
using ElementId = Mesh::ElementId;

enum class ParticleType : std::uint8_t { UNKNOWN = 0, ELECTRON = 1, PROTON = 20, ION = 52 };

enum class ParticleStatus : std::uint8_t {
    UNINITIALIZED = 0,
    CREATED = 1,
    ACTIVE = 10,
    ABSORBED = 20,
    ESCAPED = 21,
};

enum class TrajectoryChargeDepositionKernel { NearestPoint, LinearSegmentCloud, QuadratureGauss3 };

class DeviceMirror;  // the device copy of a container (defined after Collision)

namespace Constants {
inline constexpr double kElementaryCharge = 1.602176634e-19;
inline constexpr double kElectronMass = 9.1093837015e-31;
inline constexpr double kProtonMass = 1.67262192369e-27;
}  // namespace Constants

class Particle {
  public:
    Particle() = default;
    Particle(ParticleId id, ParticleType type, const Geometry::Point3D& position, const Geometry::Vector3D& velocity,
             double mass, double charge, double weight);
    ParticleId getId() const { return id_; }
    ParticleType getType() const { return type_; }
    const Geometry::Point3D& getPosition() const { return position_; }
    const Geometry::Vector3D& getVelocity() const { return velocity_; }
    void setPosition(const Geometry::Point3D& p) { position_ = p; }
    void setVelocity(const Geometry::Vector3D& v) { velocity_ = v; }
    double getMass() const { return mass_; }
    double getCharge() const { return charge_; }
    double getWeight() const { return weight_; }
    void setWeight(double w) { weight_ = w; }
    ParticleStatus getStatus() const { return status_; }
    void setStatus(ParticleStatus s) { status_ = s; }
    bool isActive() const { return status_ == ParticleStatus::ACTIVE; }
    // 0.5 m |v|^2 [J] (the reference's kinetic energy of one physical particle)
    double getKineticEnergy() const { return 0.5 * mass_ * velocity_.magnitudeSquared(); }

  private:
    ParticleId id_ = 0;
    ParticleType type_ = ParticleType::UNKNOWN;
    Geometry::Point3D position_{};
    Geometry::Vector3D velocity_{};
    double mass_ = 0.0, charge_ = 0.0, weight_ = 1.0;
    ParticleStatus status_ = ParticleStatus::ACTIVE;
};
using ParticlePtr = Particle*;

// std::vector<Particle> plus an id index.  Every non-const access counts as a host-side
// change, so the next device step re-uploads the container (the reference hands out raw
// pointers into this vector, so writes through them cannot be seen otherwise).
class ParticleContainer {
  public:
    explicit ParticleContainer(std::size_t initial_capacity = 10000);
    void addParticle(const Particle& particle);
    void addParticles(const std::vector<Particle>& particles);
    bool removeParticle(ParticleId id);
    ParticlePtr getParticle(ParticleId id);
    const Particle* getParticle(ParticleId id) const;
    std::size_t removeInactiveParticles();
    std::vector<ParticlePtr> getParticlesByType(ParticleType type);
    std::size_t size() const;
    bool empty() const { return size() == 0; }
    std::size_t getActiveCount() const;
    void reserve(std::size_t capacity) { particles_.reserve(capacity); }
    void clear();
    std::vector<Particle>::iterator begin();
    std::vector<Particle>::iterator end();
    std::vector<Particle>::const_iterator begin() const;
    std::vector<Particle>::const_iterator end() const;

    // Host-layer plumbing (no reference counterpart): a version bumped by every change,
    // and the device mirror a PICCycle attaches, which brings device state back before a read.
    std::uint64_t version() const { return version_; }
    void setDeviceMirror(DeviceMirror* mirror) { mirror_ = mirror; }
    DeviceMirror* deviceMirror() const { return mirror_; }
    // Writes device results without counting as a host change.
    std::vector<Particle>& deviceWriteAccess() { return particles_; }
    void rebuildIndex();

  private:
    void sync() const;
    void touch() { ++version_; }
    std::vector<Particle> particles_;
    std::unordered_map<ParticleId, std::size_t> index_;
    std::uint64_t version_ = 1;
    DeviceMirror* mirror_ = nullptr;
};

class ParticleManager {
  public:
    explicit ParticleManager(std::size_t max_particles = 1000000);
    ParticleId createElectron(const Geometry::Point3D& position, const Geometry::Vector3D& velocity,
                              double weight = 1.0);
    ParticleId createIon(const Geometry::Point3D& position, const Geometry::Vector3D& velocity, int mass_number,
                         int charge_number, double weight = 1.0);
    ParticlePtr getParticle(ParticleId id) { return container_->getParticle(id); }
    const Particle* getParticle(ParticleId id) const { return std::as_const(*container_).getParticle(id); }
    std::vector<ParticlePtr> getParticlesByType(ParticleType type) { return container_->getParticlesByType(type); }
    std::size_t removeInactiveParticles() { return container_->removeInactiveParticles(); }
    const ParticleContainer& getContainer() const { return *container_; }
    ParticleContainer& getContainer() { return *container_; }

  private:
    std::size_t max_particles_;
    ParticleId next_id_ = 0;
    std::unique_ptr<ParticleContainer> container_;
};

// Particle boundary conditions a PICCycle face accepts (BoundaryConditions.h:188-392).
class BoundaryConditionBase {
  public:
    virtual ~BoundaryConditionBase() = default;
};
using BoundaryConditionPtr = std::shared_ptr<BoundaryConditionBase>;

class AbsorbingBoundaryCondition : public BoundaryConditionBase {
  public:
    // absorption_probability in [0,1]; the device path implements full absorption (1.0, the
    // value the reference's callers use), and PICCycle::initialize rejects other values.
    explicit AbsorbingBoundaryCondition(double absorption_probability = 1.0);
    double getAbsorptionProbability() const { return p_; }

  private:
    double p_;
};

class PeriodicBoundaryCondition : public BoundaryConditionBase {
  public:
    // Up to 3 period vectors, each along one box axis with the length of the box on that axis.
    explicit PeriodicBoundaryCondition(const std::vector<Geometry::Vector3D>& period_vectors);
    const std::vector<Geometry::Vector3D>& getPeriodVectors() const { return periods_; }

  private:
    std::vector<Geometry::Vector3D> periods_;
};

}  // namespace Particle

// ------------------------------------------------------------------------------------------
// Field solver (Tools/FieldSolver/include/PoissonSolver.h:26-67, BoundaryCondition.h)
// ------------------------------------------------------------------------------------------
namespace Solver {
enum class SolverType { DIRECT, ITERATIVE, CONJUGATE_GRADIENT, GMRES };
}

namespace FieldSolver {

enum class BoundaryConditionType { DIRICHLET, NEUMANN };

class BoundaryCondition {
  public:
    BoundaryCondition(BoundaryConditionType type, double value) : type_(type), value_(value) {}
    BoundaryConditionType getType() const { return type_; }
    double getValue() const { return value_; }

  private:
    BoundaryConditionType type_;
    double value_;
};
using BoundaryConditionPtr = std::shared_ptr<BoundaryCondition>;

// FEM Poisson solve on the device: assembly (PoissonSolver.cpp:274-385), Dirichlet
// elimination (LinearSystem.cpp:37-58), Jacobi-PCG, nodal LSQ field
// (PoissonSolver.cpp:474-529,749-787).  Every SolverType runs the same PCG to
// setTolerance() (default 1e-12 relative); the result matches the reference's direct solve
// to that tolerance.
class PoissonSolver {
  public:
    explicit PoissonSolver(Mesh::VolMeshPtr mesh);
    virtual ~PoissonSolver();
    PoissonSolver(const PoissonSolver&) = delete;
    PoissonSolver& operator=(const PoissonSolver&) = delete;

    void initialize();
    void setMesh(Mesh::VolMeshPtr mesh);
    void addBoundaryCondition(Mesh::NodeId node_id, BoundaryConditionPtr bc);
    void clearBoundaryConditions();
    void setChargeDensity(Mesh::NodeId node_id, double density);
    void setChargeDensity(const std::unordered_map<Mesh::NodeId, double>& densities);
    void clearChargeDensities();
    void assembleSystem();
    bool solve(Solver::SolverType solver_type = Solver::SolverType::DIRECT);

    double getPotential(Mesh::NodeId node_id) const;
    Utils::Vector3D getElectricField(Mesh::NodeId node_id) const;
    double getTotalEnergy() const;
    double getMaxPotential() const;
    double getMinPotential() const;
    Utils::Vector3D getMaxElectricField() const;

    // Device-side options (no reference counterpart).
    void setTolerance(double rtol) { rtol_ = rtol; }
    const std::string& lastError() const { return error_; }

  private:
    struct Impl;
    Mesh::VolMeshPtr mesh_;
    std::unordered_map<Mesh::NodeId, BoundaryConditionPtr> bcs_;
    std::unordered_map<Mesh::NodeId, double> rho_;
    std::vector<double> phi_;
    std::vector<Utils::Vector3D> field_;
    double rtol_ = 1.0e-12;
    std::string error_;
    std::unique_ptr<Impl> impl_;
};

}  // namespace FieldSolver

// ------------------------------------------------------------------------------------------
// The PIC cycle (Tools/PICcore/include/PICCycle.h:29-185)
// ------------------------------------------------------------------------------------------
namespace PICcore {

using ::SCDAT::FieldSolver::PoissonSolver;
using ::SCDAT::Particle::BoundaryConditionPtr;
using ::SCDAT::Particle::ElementId;
using ::SCDAT::Particle::ParticleManager;
using ::SCDAT::Particle::ParticlePtr;
using ::SCDAT::Particle::TrajectoryChargeDepositionKernel;

class PICCycle {
  public:
    enum class BoundaryFace { XMin = 0, XMax = 1, YMin = 2, YMax = 3, ZMin = 4, ZMax = 5 };

    struct Parameters {
        double time_step = 1e-12;
        int max_iterations = 1000;
        double convergence_tolerance = 1e-6;
        bool adaptive_time_step = false;
        bool charge_conservation = true;
        int statistics_frequency = 10;
        bool verbose = false;
        std::size_t trajectory_charge_deposition_segments = 10;
        TrajectoryChargeDepositionKernel trajectory_charge_deposition_kernel =
            TrajectoryChargeDepositionKernel::LinearSegmentCloud;
    };

    // Device-side choices (no reference counterpart); defaults give the FP64 form with the
    // reference's numerics.
    struct DeviceOptions {
        bool mixed_precision = false;   // FP32 cell-relative push + FP32-SpMV PCG under FP64 refinement
        double pcg_rtol = 1.0e-12;      // relative residual of the per-step field solve
        int pcg_max_iter = 20000;
        int compact_interval = 4;       // drop inactive particles from the device store every N steps
        int poisson_charge_sign = -1;   // b = -rho*V/4 as PoissonSolver.cpp:356
        bool body_tally = false;        // tally particles lost into interior holes (ledger row 6)
    };

    struct CycleStatistics {
        int completed_steps = 0;
        double simulation_time = 0.0;
        double total_charge = 0.0;
        double total_energy = 0.0;
        int active_particles = 0;
        double average_step_time = 0.0;
        double surface_deposited_charge = 0.0;
    };

    struct SurfaceBoundaryMetadata {
        int surface_id = -1;
        int material_id = -1;
        int circuit_node_id = -1;
    };

    struct SurfaceCurrentLedgerEntry {
        SurfaceBoundaryMetadata metadata;
        double absorbed_electron_charge_c = 0.0;
        double absorbed_ion_charge_c = 0.0;
        double emitted_electron_charge_c = 0.0;
        double incident_energy_j = 0.0;
        std::size_t absorbed_electron_particles = 0;
        std::size_t absorbed_ion_particles = 0;
        std::size_t emitted_electron_particles = 0;
    };

    PICCycle();
    explicit PICCycle(const Parameters& params);
    ~PICCycle();
    PICCycle(PICCycle&&) noexcept;
    PICCycle& operator=(PICCycle&&) noexcept;

    void setMesh(const std::vector<Mesh::NodePtr>& nodes, const std::vector<Mesh::ElementPtr>& elements);
    void setParticleManager(std::shared_ptr<ParticleManager> particle_manager);
    void setPoissonSolver(std::shared_ptr<PoissonSolver> poisson_solver);
    void setBoundaryCondition(BoundaryFace face, BoundaryConditionPtr condition);
    void clearBoundaryConditions();

    void addParticleLocation(ParticlePtr particle, ElementId element_id);
    void updateParticleLocation(ParticlePtr particle, ElementId new_element_id);
    ElementId findParticleElement(ParticlePtr particle) const;

    bool initialize();
    bool executeTimeStep();
    bool executeSimulation(double total_time);

    const std::vector<double>& getChargeDensity() const;
    const std::vector<double>& getPotential() const;
    const std::vector<Utils::Vector3D>& getElectricField() const;

    void setTimeStep(double dt);
    double getTimeStep() const;
    void setPotential(const std::vector<double>& potential);
    void setNodePotential(std::size_t node_id, double value);

    const CycleStatistics& getStatistics() const;
    void setBoundaryMetadata(BoundaryFace face, const SurfaceBoundaryMetadata& metadata);
    const std::array<SurfaceCurrentLedgerEntry, 6>& getSurfaceCurrentLedger() const;
    double getAndResetSurfaceCharge();

    void setDeviceOptions(const DeviceOptions& options);
    const std::string& lastError() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace PICcore

// ------------------------------------------------------------------------------------------
// Background MCC (Tools/Interactions/Collisions/include/CollisionPicAdapter.h:20-110)
// ------------------------------------------------------------------------------------------
namespace Collision {

struct CollisionBackgroundDensities {
    double neutral_density_m3 = 0.0;
    double ion_density_m3 = 0.0;
    double electron_density_m3 = 0.0;
};

enum class CollisionCrossSectionSetId { BackgroundMccV1, SurfacePicV1, VacuumArcPicV1 };

struct BackgroundMccRuntimeConfig {
    CollisionBackgroundDensities floor_densities;
    CollisionCrossSectionSetId cross_section_set_id = CollisionCrossSectionSetId::BackgroundMccV1;
    bool reinitialize_configuration = false;
};

struct CollisionStepResult {
    std::size_t active_particles = 0;
    std::size_t collision_events = 0;
    std::size_t generated_particles = 0;
    std::size_t ionization_events = 0;
    std::size_t excitation_events = 0;
    std::size_t charge_exchange_events = 0;
    double effective_neutral_density_m3 = 0.0;
    double effective_ion_density_m3 = 0.0;
    double effective_electron_density_m3 = 0.0;
};

// ElasticCollisionCrossSection (CollisonTypes.cpp:60-78): sigma(E) = sigma_max (E_ref/E)^alpha
// capped at sigma_max; alpha = 0 is the constant cross-section.
struct ElasticProcess {
    Particle::ParticleType projectile = Particle::ParticleType::ELECTRON;
    double target_density_m3 = 0.0;
    double sigma_max_m2 = 0.0;
    double reference_energy_ev = 1.0;
    double power_index = 0.0;
    double threshold_ev = 0.0;
};

// MonteCarloCollisionHandler (CollisionAlgorithm.h:176-226).  The device path executes the
// elastic process with the reference's two-draw acceptance (CollisionAlgorithm.cpp:525-531
// then :195-200); a handler configured with any other process type refuses to run on a
// non-empty container (std::invalid_argument) rather than skipping it.
class MonteCarloCollisionHandler {
  public:
    explicit MonteCarloCollisionHandler(std::uint64_t seed = 12345);
    void addElasticProcess(const ElasticProcess& process);
    void clearProcesses();
    const std::vector<ElasticProcess>& elasticProcesses() const { return elastic_; }
    // Names of configured processes the device path does not implement.
    const std::vector<std::string>& unsupportedProcesses() const { return unsupported_; }
    void markUnsupported(std::string name) { unsupported_.push_back(std::move(name)); }
    std::uint64_t seed() const { return seed_; }

    struct Statistics {
        long long total_collisions = 0;
        long long particles_created = 0;
        std::unordered_map<std::string, int> collision_counts;
    };
    const Statistics& getStatistics() const { return stats_; }
    Statistics& mutableStatistics() { return stats_; }

  private:
    std::uint64_t seed_;
    std::vector<ElasticProcess> elastic_;
    std::vector<std::string> unsupported_;
    Statistics stats_;
};

CollisionBackgroundDensities estimateCollisionBackgroundDensities(const Particle::ParticleContainer& container,
                                                                  double volume_m3,
                                                                  const CollisionBackgroundDensities& floor_densities);
std::optional<CollisionCrossSectionSetId> parseCollisionCrossSectionSetId(const std::string& text);
std::string toString(CollisionCrossSectionSetId set_id);
void initializeConfiguredCollisionHandler(MonteCarloCollisionHandler& handler, CollisionCrossSectionSetId set_id,
                                          double neutral_density_m3, double ion_density_m3,
                                          double electron_density_m3);

// One background MCC step over the active particles of a container that a PICCycle mirrors
// on the device (CollisionPicAdapter.cpp:338-434).  Inactive particles are removed afterwards,
// as the reference does.
CollisionStepResult executeBackgroundMccStep(Particle::ParticleContainer& container,
                                             MonteCarloCollisionHandler& handler, double dt, double volume_m3,
                                             const BackgroundMccRuntimeConfig& runtime_config);
CollisionStepResult executeBackgroundMccStep(Particle::ParticleContainer& container,
                                             MonteCarloCollisionHandler& handler, double dt, double volume_m3,
                                             const CollisionBackgroundDensities& floor_densities,
                                             bool reinitialize_configuration);

}  // namespace Collision

namespace Particle {
// What a PICCycle exposes to the container it mirrors (no reference counterpart).
class DeviceMirror {
  public:
    virtual ~DeviceMirror() = default;
    // Copy device particle state into the container if the device is ahead.
    virtual void pull() = 0;
    // One device MCC pass over the mirrored particles with these elastic processes; returns
    // false with a reason when the device cannot run it.
    virtual bool collide(const std::vector<Collision::ElasticProcess>& processes, std::uint64_t seed, double dt,
                         std::size_t& collisions, std::string& error) = 0;
    // Drop inactive particles on the device as well.
    virtual void compact() = 0;
};
}  // namespace Particle
}  // namespace SCDAT
