// ParticleModules.h -- the hot-path modules with the reference's class names,
// fields and public methods, each backed by the sm_100a C ABI (pk_hot.h):
//   NeighborQuery       Framework/Topology/NeighborQuery.h:12-95
//   SummationDensity    Dynamics/ParticleSystem/SummationDensity.h:14-67
//   DensityPBD          Dynamics/ParticleSystem/DensityPBD.h:17-88
//   ParticleIntegrator  Dynamics/ParticleSystem/ParticleIntegrator.h:7-54
//   ElasticityModule    Dynamics/ParticleSystem/ElasticityModule.h:18-107
//   BoundaryConstraint  Dynamics/ParticleSystem/BoundaryConstraint.h (box SDF)
// and the models/nodes that wire them (PositionBasedFluidModel.cpp:41-101,
// Peridynamics.cpp:29-80, ParticleFluid, ParticleElasticBody.cpp:15-98,
// StaticBoundary.cpp:45-94).
#pragma once
#include "Node.h"

namespace PhysIKA {

template <typename TDataType>
class NeighborQuery : public ComputeModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;

    NeighborQuery();
    NeighborQuery(Real s, Coord lo, Coord hi);
    ~NeighborQuery() override = default;

    void compute() override;
    void setBoundingBox(Coord lowerBound, Coord upperBound);
    void queryParticleNeighbors(NeighborList<int>& nbr, DeviceArray<Coord>& pos, Real radius);
    void setNeighborSizeLimit(int num) { m_maxNum = num; }

    DEF_EMPTY_IN_VAR(Radius, Real, "Search radius");
    DEF_EMPTY_IN_ARRAY(Position, Coord, DeviceType::GPU, "Particle position");
    DEF_EMPTY_OUT_NEIGHBOR_LIST(Neighborhood, int, "Neighboring particles' ids");

protected:
    bool initializeImpl() override;

private:
    void query(NeighborList<int>& nbr, DeviceArray<Coord>& pos, Real h);
    int m_maxNum = 0;
    Coord m_lowBound, m_highBound;
};

template <typename TDataType>
class SummationDensity : public ComputeModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    SummationDensity();
    void compute() override;
    void update() { compute(); }

    DEF_EMPTY_VAR(RestDensity, Real, "Rest density");
    DEF_EMPTY_VAR(SamplingDistance, Real, "Sampling distance");
    DEF_EMPTY_VAR(SmoothingLength, Real, "Smoothing length");
    DEF_EMPTY_IN_ARRAY(Position, Coord, DeviceType::GPU, "Particle position");
    DEF_EMPTY_IN_NEIGHBOR_LIST(NeighborIndex, int, "Neighboring particles");
    DEF_EMPTY_OUT_ARRAY(Density, Real, DeviceType::GPU, "Particle density");
};

template <typename TDataType>
class DensityPBD : public ConstraintModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;

    DensityPBD();
    ~DensityPBD() override = default;

    bool constrain() override;
    // Runs one Jacobi sweep on the given list (the reference's takeOneIteration).
    void takeOneIteration();
    void updateVelocity();

    DEF_EMPTY_VAR(IterationNumber, int, "Iteration number of the PBD solver");
    DEF_EMPTY_VAR(RestDensity, Real, "Reference density");
    DEF_EMPTY_VAR(SamplingDistance, Real, "");
    DEF_EMPTY_VAR(SmoothingLength, Real, "");
    DEF_EMPTY_IN_ARRAY(Position, Coord, DeviceType::GPU, "Input particle position");
    DEF_EMPTY_IN_ARRAY(Velocity, Coord, DeviceType::GPU, "Input particle velocity");
    DEF_EMPTY_IN_NEIGHBOR_LIST(NeighborIndex, int, "Neighboring particles' ids");
    DEF_EMPTY_OUT_ARRAY(Position, Coord, DeviceType::GPU, "Output particle position");
    DEF_EMPTY_OUT_ARRAY(Velocity, Coord, DeviceType::GPU, "Output particle velocity");
    DEF_EMPTY_OUT_ARRAY(Density, Real, DeviceType::GPU, "Final particle density");

private:
    pk_pbd_params params(int iterations);
    DeviceArray<Coord> m_position_old;  // scratch velocity of takeOneIteration
    DeviceArray<Coord> m_x_old;         // positions at the start of constrain()
};

template <typename TDataType>
class ParticleIntegrator : public NumericalIntegrator {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    ParticleIntegrator() = default;
    void begin() override;
    void end() override {}
    bool integrate() override;
    bool updateVelocity();
    bool updatePosition();

    DEF_EMPTY_IN_ARRAY(Position, Coord, DeviceType::GPU, "Position");
    DEF_EMPTY_IN_ARRAY(Velocity, Coord, DeviceType::GPU, "Velocity");
    DEF_EMPTY_IN_ARRAY(ForceDensity, Coord, DeviceType::GPU, "Force density");

protected:
    bool initializeImpl() override { return true; }

private:
    DeviceArray<Coord> m_prePosition, m_preVelocity;
};

template <typename TDataType>
class ElasticityModule : public ConstraintModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;

    ElasticityModule();
    ~ElasticityModule() override = default;

    bool constrain() override;
    virtual void solveElasticity();
    void setMu(Real mu) { m_mu.setValue(mu); }
    void setLambda(Real lambda) { m_lambda.setValue(lambda); }
    void setIterationNumber(int num) { m_iterNum.setValue(num); }
    int getIterationNumber() { return m_iterNum.getValue(); }
    void resetRestShape();
    // Stretch-break threshold (no reference counterpart; 0 = never break).
    void setBreakStretch(Real s) { m_breakStretch = s; }

    DEF_EMPTY_IN_VAR(Horizon, Real, "");
    DEF_EMPTY_IN_ARRAY(Position, Coord, DeviceType::GPU, "Particle position");
    DEF_EMPTY_IN_ARRAY(Velocity, Coord, DeviceType::GPU, "Particle velocity");
    DEF_EMPTY_IN_NEIGHBOR_LIST(Neighborhood, int, "Neighboring particles' ids");

protected:
    bool initializeImpl() override;
    // ElasticityModule.cu:390-421: K^-1 of the current rest shape, one
    // projection iteration against the positions saved by beginSolve(), and
    // v += (x - x_old)/dt.  beginSolve() is the Function1Pt::copy of
    // m_position_old at the top of solveElasticity.
    void beginSolve();
    void computeInverseK();
    virtual void enforceElasticity();
    void updateVelocity();
    // Subclasses set m_bulkCoefs here (the reference initialises it to 1).
    virtual void computeMaterialStiffness();
    pk_pd_params stepParams();

    VarField<Real> m_mu{Real(0.05)};
    VarField<Real> m_lambda{Real(0.1)};
    DeviceArray<Real> m_bulkCoefs;

private:
    VarField<int> m_iterNum{10};
    Real m_breakStretch = 0;
};

// ElastoplasticityModule (Dynamics/ParticleSystem/ElastoplasticityModule.h:18-80):
// projective peridynamics with a one-iteration DensityPBD after each
// projection, then plasticity on the rest shape (rotation, Drucker-Prager
// yielding, reconstruction).
template <typename TDataType>
class ElastoplasticityModule : public ElasticityModule<TDataType> {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;

    ElastoplasticityModule();
    ~ElastoplasticityModule() override = default;

    bool constrain() override;
    void solveElasticity() override;
    virtual void applyPlasticity();
    void applyYielding();
    void rotateRestShape();
    void reconstructRestShape();

    void setCohesion(Real c) { m_c.setValue(c); }
    void setFrictionAngle(Real phi) { m_phi.setValue(phi / 180); }  // stored as the reference stores it
    void enableFullyReconstruction() { m_reconstuct_all_neighborhood.setValue(true); }
    void disableFullyReconstruction() { m_reconstuct_all_neighborhood.setValue(false); }
    void enableIncompressibility() { m_incompressible.setValue(true); }
    void disableIncompressibility() { m_incompressible.setValue(false); }

protected:
    bool initializeImpl() override;
    Real computeA();
    Real computeB();
    pk_plastic_params plasticParams();

private:
    VarField<Real> m_c{Real(0.001)};
    VarField<Real> m_phi{Real(60.0 / 180.0)};
    VarField<bool> m_reconstuct_all_neighborhood{false};
    VarField<bool> m_incompressible{true};
    std::shared_ptr<DensityPBD<TDataType>> m_pbdModule;
};

// FractureModule (Dynamics/ParticleSystem/FractureModule.h:8-20): the same
// solve; particles past the yield limit lose their bulk stiffness.
template <typename TDataType>
class FractureModule : public ElastoplasticityModule<TDataType> {
public:
    FractureModule();
    void applyPlasticity() override;
};

// ImplicitViscosity (Dynamics/ParticleSystem/ImplicitViscosity.h:9-46): the
// member fields and setters of the reference; constrain() is pk_viscosity.
template <typename TDataType>
class ImplicitViscosity : public ConstraintModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    ImplicitViscosity();
    bool constrain() override;
    void setIterationNumber(int n) { m_maxInteration = n; }
    void setViscosity(Real mu) { m_viscosity.setValue(mu); }

    VarField<Real> m_viscosity{Real(0.05), "viscosity", "The viscosity of the fluid!", FieldType::Param, nullptr};
    VarField<Real> m_smoothingLength{Real(0.011), "smoothing_length", "The smoothing length in SPH!",
                                     FieldType::Param, nullptr};
    DeviceArrayField<Coord> m_position{0, "position", "Storing the particle positions!", FieldType::In, nullptr};
    DeviceArrayField<Coord> m_velocity{0, "velocity", "Storing the particle velocities!", FieldType::In, nullptr};
    NeighborField<int> m_neighborhood{"neighborhood", "Storing neighboring particles' ids!", FieldType::In,
                                      nullptr, 0, 0};

private:
    int m_maxInteration = 5;
};

// BoundaryConstraint with a box SDF (BoundaryConstraint.cu:108-117).
template <typename TDataType>
class BoundaryConstraint : public ConstraintModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    BoundaryConstraint() = default;
    using ConstraintModule::constrain;
    bool constrain(DeviceArray<Coord>& position, DeviceArray<Coord>& velocity, Real dt);
    void setCube(Coord lo, Coord hi, Real distance, bool inverted);
    Real m_normal_friction = 0.95f;
    Real m_tangent_friction = 0.0f;

private:
    bool m_set = false;
    Coord m_lo, m_hi;
    Real m_distance = 0.005f;
    bool m_inverted = true;
};

// PositionBasedFluidModel::step (PositionBasedFluidModel.cpp:83-101): begin,
// NeighborQuery, integrate, DensityPBD, ImplicitViscosity (viscosity 1 as the
// reference sets it, PositionBasedFluidModel.cpp:69-70; setViscosity(0) leaves
// it out), end.
template <typename TDataType>
class PositionBasedFluidModel : public NumericalModel {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    PositionBasedFluidModel();
    void step(float dt) override;
    void setNeighborSizeLimit(int cap) { m_cap = cap; }
    void setIterationNumber(int it) { m_iterations = it; }
    void setSamplingDistance(Real d) { m_samplingDistance = d; }
    void setViscosity(Real mu) { m_viscosity = mu; }

    VarField<Real> m_smoothingLength{Real(0.006)};
    DeviceArrayField<Coord> m_position{0, "position", "", FieldType::In, nullptr};
    DeviceArrayField<Coord> m_velocity{0, "velocity", "", FieldType::In, nullptr};
    DeviceArrayField<Coord> m_forceDensity{0, "force_density", "", FieldType::In, nullptr};

    std::shared_ptr<NeighborQuery<TDataType>> m_nbrQuery;
    std::shared_ptr<DensityPBD<TDataType>> m_pbdModule;
    std::shared_ptr<ParticleIntegrator<TDataType>> m_integrator;
    std::shared_ptr<ImplicitViscosity<TDataType>> m_visModule;

protected:
    bool initializeImpl() override;

private:
    Real m_viscosity = Real(1);
    int m_cap = 0;
    int m_iterations = 3;
    Real m_samplingDistance = Real(0.005);
};

// A particle node holding the current state (ParticleSystem.h currentPosition/...).
template <typename TDataType>
class ParticleSystem : public Node {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    explicit ParticleSystem(std::string name = "default") : Node(std::move(name)) {}
    void setParticles(const std::vector<Coord>& pos, const std::vector<Coord>& vel);
    void getParticles(std::vector<Coord>& pos, std::vector<Coord>& vel);
    // ParticleSystem::loadParticles (ParticleSystem.cpp:34-97), in ParticleIO.cpp:
    // an OBJ file's vertices, a ball or a box lattice, at rest.
    void loadParticles(std::string filename);
    void loadParticles(Coord center, Real r, Real distance);
    void loadParticles(Coord lo, Coord hi, Real distance);

    DEF_EMPTY_CURRENT_ARRAY(Position, Coord, DeviceType::GPU, "Particle position");
    DEF_EMPTY_CURRENT_ARRAY(Velocity, Coord, DeviceType::GPU, "Particle velocity");
    DEF_EMPTY_CURRENT_ARRAY(Force, Coord, DeviceType::GPU, "Force on each particle");
};

// ParticleFluid: a particle system stepped by PositionBasedFluidModel.
template <typename TDataType>
class ParticleFluid : public ParticleSystem<TDataType> {
public:
    typedef typename TDataType::Real Real;
    explicit ParticleFluid(std::string name = "fluid");
    bool initialize() override;
    void advance(float dt) override;
    std::shared_ptr<PositionBasedFluidModel<TDataType>> getModel() { return m_model_pbf; }

private:
    std::shared_ptr<PositionBasedFluidModel<TDataType>> m_model_pbf;
};

// ParticleElasticBody (ParticleElasticBody.cpp:15-98).
template <typename TDataType>
class ParticleElasticBody : public ParticleSystem<TDataType> {
public:
    typedef typename TDataType::Real Real;
    explicit ParticleElasticBody(std::string name = "elastic");
    bool initialize() override;
    void advance(float dt) override;
    std::shared_ptr<ElasticityModule<TDataType>> getElasticitySolver();
    void setElasticitySolver(std::shared_ptr<ElasticityModule<TDataType>> solver);
    VarField<Real>* varHorizon() { return &m_horizon; }

private:
    VarField<Real> m_horizon{Real(0.0085)};
};

// ParticleElastoplasticBody (ParticleElastoplasticBody.cpp:20-91): integrate,
// query, solveElasticity, query again, applyPlasticity, ImplicitViscosity.
template <typename TDataType>
class ParticleElastoplasticBody : public ParticleSystem<TDataType> {
public:
    typedef typename TDataType::Real Real;
    explicit ParticleElastoplasticBody(std::string name = "default");
    bool initialize() override;
    void advance(float dt) override;
    void setElastoplasticitySolver(std::shared_ptr<ElastoplasticityModule<TDataType>> solver);
    std::shared_ptr<ElastoplasticityModule<TDataType>> getElastoplasticitySolver();
    VarField<Real>* varHorizon() { return &m_horizon; }

private:
    VarField<Real> m_horizon{Real(0.0085)};
    std::shared_ptr<ParticleIntegrator<TDataType>> m_integrator;
    std::shared_ptr<NeighborQuery<TDataType>> m_nbrQuery;
    std::shared_ptr<DensityPBD<TDataType>> m_pbdModule;
    std::shared_ptr<ImplicitViscosity<TDataType>> m_visModule;
};

// StaticBoundary::advance (StaticBoundary.cpp:45-59): constrain every
// particle system with every obstacle, before they advance.
template <typename TDataType>
class StaticBoundary : public Node {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;
    explicit StaticBoundary(std::string name = "boundary") : Node(std::move(name)) {}
    void loadCube(Coord lo, Coord hi, Real distance = 0.005f, bool bOutBoundary = false);
    void addParticleSystem(std::shared_ptr<ParticleSystem<TDataType>> p) { m_systems.push_back(p); }
    void advance(float dt) override;

private:
    std::vector<std::shared_ptr<BoundaryConstraint<TDataType>>> m_obstacles;
    std::vector<std::shared_ptr<ParticleSystem<TDataType>>> m_systems;
};

}  // namespace PhysIKA
