// ParticleModules.cpp -- module bodies: every compute goes through the C ABI.
#include "ParticleModules.h"

#include <cmath>

#include <map>

namespace PhysIKA {

void pkCheck(int status, pk_ctx* ctx, const char* where)
{
    if (status == PK_OK) return;
    std::string msg = std::string(where) + ": " + (ctx ? pk_last_error(ctx) : "no context") +
                      " (status " + std::to_string(status) + ")";
    Log::sendMessage(Log::Error, msg);
    throw std::runtime_error(msg);
}

namespace {
pk_ctx* newContext()
{
    int dev = 0;
    cudaGetDevice(&dev);
    pk_ctx* c = nullptr;
    pkCheck(pk_ctx_create(&c, dev), nullptr, "pk_ctx_create");
    return c;
}

// One context per module instance that owns scratch, created on first use.
struct OwnedContext {
    pk_ctx* c = nullptr;
    ~OwnedContext()
    {
        if (c) pk_ctx_destroy(c);
    }
    pk_ctx* get()
    {
        if (!c) c = newContext();
        return c;
    }
};
std::map<const void*, OwnedContext>& registry()
{
    static std::map<const void*, OwnedContext> r;
    return r;
}
pk_ctx* contextOf(const void* owner) { return registry()[owner].get(); }

template <typename T>
float* F(DeviceArray<T>& a) { return reinterpret_cast<float*>(a.getDataPtr()); }
}  // namespace

pk_ctx* hotContext() { return contextOf(nullptr); }

// ================================================================ NeighborQuery

template <typename TDataType>
NeighborQuery<TDataType>::NeighborQuery()
{
    // NeighborQuery.cu:46-63: bounds from the scene graph, radius 0.011.
    Vector3f lo = SceneGraph::getInstance().getLowerBound();
    Vector3f hi = SceneGraph::getInstance().getUpperBound();
    m_lowBound = Coord(lo[0], lo[1], lo[2]);
    m_highBound = Coord(hi[0], hi[1], hi[2]);
    this->inRadius()->setValue(Real(0.011));
}

template <typename TDataType>
NeighborQuery<TDataType>::NeighborQuery(Real s, Coord lo, Coord hi)
{
    this->inRadius()->setValue(s);
    m_lowBound = lo;
    m_highBound = hi;
}

template <typename TDataType>
void NeighborQuery<TDataType>::setBoundingBox(Coord lowerBound, Coord upperBound)
{
    m_lowBound = lowerBound;
    m_highBound = upperBound;
}

template <typename TDataType>
bool NeighborQuery<TDataType>::initializeImpl()
{
    // NeighborQuery.cu:107-149
    if (!this->inPosition()->isEmpty() && this->outNeighborhood()->isEmpty())
        this->outNeighborhood()->setElementCount((int)this->inPosition()->getElementCount(), m_maxNum);
    if (this->inPosition()->isEmpty() || this->inRadius()->isEmpty()) {
        std::printf("Exception: NeighborQuery's fields are not fully initialized!\n");
        return false;
    }
    compute();
    return true;
}

template <typename TDataType>
void NeighborQuery<TDataType>::query(NeighborList<int>& nbr, DeviceArray<Coord>& pos, Real h)
{
    pk_ctx* c = contextOf(this);
    const int n = pos.size();
    pk_nq_params p;
    p.radius = h;
    for (int a = 0; a < 3; ++a) {
        p.lo[a] = m_lowBound[a];
        p.hi[a] = m_highBound[a];
    }
    p.cap = nbr.getNeighborLimit();
    p.max_neighbors = 0;
    if (nbr.isLimited()) {
        pkCheck(pk_nq_build(c, F(pos), n, &p, nbr.getIndex().getDataPtr(), nbr.getElements().getDataPtr(),
                            (long long)nbr.getElements().size(), nullptr, 0),
                c, "NeighborQuery::compute");
    } else {
        // one build into the list's current elements (the reference reads the
        // total back and resizes, NeighborQuery.cu:463-472); only a list that
        // outgrew them is built again at its new size
        long long total = 0;
        const long long have = (long long)nbr.getElements().size();
        int rc = pk_nq_build(c, F(pos), n, &p, nbr.getIndex().getDataPtr(), have > 0 ? nbr.getElements().getDataPtr() : nullptr,
                             have, &total, 0);
        if (rc == PK_ERR_CAPACITY || (rc == PK_OK && have == 0 && total > 0)) {
            nbr.getElements().resize((int)(total + total / 8));
            rc = pk_nq_build(c, F(pos), n, &p, nbr.getIndex().getDataPtr(), nbr.getElements().getDataPtr(),
                             (long long)nbr.getElements().size(), &total, 0);
        }
        pkCheck(rc, c, "NeighborQuery::compute");
        nbr.setTotal(total);
    }
    nbr.setProducer(c);
}

template <typename TDataType>
void NeighborQuery<TDataType>::compute()
{
    // NeighborQuery.cu:152-176
    if (this->inPosition()->isEmpty()) return;
    int p_num = (int)this->inPosition()->getElementCount();
    if ((int)this->outNeighborhood()->getElementCount() != p_num)
        this->outNeighborhood()->setElementCount(p_num);
    query(this->outNeighborhood()->getValue(), this->inPosition()->getValue(), this->inRadius()->getValue());
}

template <typename TDataType>
void NeighborQuery<TDataType>::queryParticleNeighbors(NeighborList<int>& nbr, DeviceArray<Coord>& pos,
                                                      Real radius)
{
    query(nbr, pos, radius);
}

// ============================================================ SummationDensity

template <typename TDataType>
SummationDensity<TDataType>::SummationDensity()
{
    this->varRestDensity()->setValue(Real(1000));
    this->varSmoothingLength()->setValue(Real(0.011));
    this->varSamplingDistance()->setValue(Real(0.005));
}

template <typename TDataType>
void SummationDensity<TDataType>::compute()
{
    int p_num = (int)this->inPosition()->getElementCount();
    int n_num = (int)this->inNeighborIndex()->getElementCount();
    if (p_num != n_num) {
        Log::sendMessage(Log::Error, "The input array sizes of DensitySummation are not compatible!");
        return;
    }
    if ((int)this->outDensity()->getElementCount() != p_num) this->outDensity()->setElementCount(p_num);
    auto& nbr = this->inNeighborIndex()->getValue();
    pk_pbd_params p{this->varSmoothingLength()->getValue(), this->varSamplingDistance()->getValue(),
                    this->varRestDensity()->getValue(), 0, 1.0f};
    pk_ctx* c = contextOf(this);
    pkCheck(pk_summation_density(c, F(this->inPosition()->getValue()), p_num, nbr.getIndex().getDataPtr(),
                                 nbr.getElements().getDataPtr(), nbr.getNeighborLimit(), nbr.total(), &p,
                                 this->outDensity()->getValue().getDataPtr(), 0),
            c, "SummationDensity::compute");
}

// ================================================================== DensityPBD

template <typename TDataType>
DensityPBD<TDataType>::DensityPBD()
{
    // DensityPBD.cu:240-260
    this->varIterationNumber()->setValue(3);
    this->varSamplingDistance()->setValue(Real(0.005));
    this->varSmoothingLength()->setValue(Real(0.011));
    this->varRestDensity()->setValue(Real(1000));
}

template <typename TDataType>
pk_pbd_params DensityPBD<TDataType>::params(int iterations)
{
    return pk_pbd_params{this->varSmoothingLength()->getValue(), this->varSamplingDistance()->getValue(),
                         this->varRestDensity()->getValue(), iterations, this->getParent()->getDt()};
}

template <typename TDataType>
bool DensityPBD<TDataType>::constrain()
{
    // DensityPBD.cu:271-302: the whole constrain (x_old copy, iterations,
    // velocity update) is one pk_pbd_solve.
    int num = (int)this->inPosition()->getElementCount();
    if ((int)this->outDensity()->getElementCount() != num) this->outDensity()->setElementCount(num);
    auto& nbr = this->inNeighborIndex()->getValue();
    pk_ctx* c = nbr.producer() ? nbr.producer() : contextOf(this);
    pk_pbd_params p = params(this->varIterationNumber()->getValue());
    if (m_x_old.size() != num) m_x_old.resize(num);
    Function1Pt::copy(m_x_old, this->inPosition()->getValue());
    pkCheck(pk_pbd_solve(c, F(this->inPosition()->getValue()), F(this->inVelocity()->getValue()), num,
                         nbr.getIndex().getDataPtr(), nbr.getElements().getDataPtr(), nbr.getNeighborLimit(),
                         nbr.total(), &p, this->outDensity()->getValue().getDataPtr(), 0),
            c, "DensityPBD::constrain");
    return true;
}

template <typename TDataType>
void DensityPBD<TDataType>::takeOneIteration()
{
    // One sweep on x only: the velocity the solve derives is discarded.
    int num = (int)this->inPosition()->getElementCount();
    if (m_position_old.size() != num) m_position_old.resize(num);
    m_position_old.reset();
    auto& nbr = this->inNeighborIndex()->getValue();
    pk_ctx* c = nbr.producer() ? nbr.producer() : contextOf(this);
    if ((int)this->outDensity()->getElementCount() != num) this->outDensity()->setElementCount(num);
    pk_pbd_params p = params(1);
    pkCheck(pk_pbd_solve(c, F(this->inPosition()->getValue()), F(m_position_old), num,
                         nbr.getIndex().getDataPtr(), nbr.getElements().getDataPtr(), nbr.getNeighborLimit(),
                         nbr.total(), &p, this->outDensity()->getValue().getDataPtr(), 0),
            c, "DensityPBD::takeOneIteration");
}

template <typename TDataType>
void DensityPBD<TDataType>::updateVelocity()
{
    // DP_UpdateVelocity (DensityPBD.cu:367-392): v += (x - x_old)/dt with the
    // positions saved by the last constrain().  constrain() already applies it.
    int num = (int)this->inPosition()->getElementCount();
    if (m_x_old.size() != num) {
        Log::sendMessage(Log::Error, "DensityPBD::updateVelocity before constrain()");
        return;
    }
    pk_ctx* c = contextOf(this);
    pkCheck(pk_update_velocity(c, F(this->inVelocity()->getValue()), F(this->inPosition()->getValue()),
                               F(m_x_old), num, this->getParent()->getDt(), 0),
            c, "DensityPBD::updateVelocity");
}

// ========================================================== ParticleIntegrator

template <typename TDataType>
void ParticleIntegrator<TDataType>::begin()
{
    // ParticleIntegrator.cu:19-34
    if (this->inPosition()->isEmpty()) return;
    int num = (int)this->inPosition()->getElementCount();
    m_prePosition.resize(num);
    m_preVelocity.resize(num);
    Function1Pt::copy(m_prePosition, this->inPosition()->getValue());
    Function1Pt::copy(m_preVelocity, this->inVelocity()->getValue());
    if (!this->inForceDensity()->isEmpty()) this->inForceDensity()->getValue().reset();
}

template <typename TDataType>
bool ParticleIntegrator<TDataType>::updateVelocity()
{
    Vector3f g = SceneGraph::getInstance().getGravity();
    float gv[3] = {g[0], g[1], g[2]};
    int n = (int)this->inPosition()->getElementCount();
    float* f = this->inForceDensity()->isEmpty() ? nullptr : F(this->inForceDensity()->getValue());
    pk_ctx* c = hotContext();
    pkCheck(pk_integrate(c, nullptr, F(this->inVelocity()->getValue()), f, n, gv, this->getParent()->getDt(), 0),
            c, "ParticleIntegrator::updateVelocity");
    return true;
}

template <typename TDataType>
bool ParticleIntegrator<TDataType>::updatePosition()
{
    int n = (int)this->inPosition()->getElementCount();
    pk_ctx* c = hotContext();
    pkCheck(pk_advect(c, F(this->inPosition()->getValue()), F(this->inVelocity()->getValue()), n,
                      this->getParent()->getDt(), 0),
            c, "ParticleIntegrator::updatePosition");
    return true;
}

template <typename TDataType>
bool ParticleIntegrator<TDataType>::integrate()
{
    // ParticleIntegrator.cu:128-138: both updates in one kernel
    if (this->inPosition()->isEmpty()) return true;
    Vector3f g = SceneGraph::getInstance().getGravity();
    float gv[3] = {g[0], g[1], g[2]};
    int n = (int)this->inPosition()->getElementCount();
    float* f = this->inForceDensity()->isEmpty() ? nullptr : F(this->inForceDensity()->getValue());
    pk_ctx* c = hotContext();
    pkCheck(pk_integrate(c, F(this->inPosition()->getValue()), F(this->inVelocity()->getValue()), f, n, gv,
                         this->getParent()->getDt(), 0),
            c, "ParticleIntegrator::integrate");
    return true;
}

// ============================================================ ElasticityModule

template <typename TDataType>
ElasticityModule<TDataType>::ElasticityModule()
{
    // ElasticityModule.cu:308-329
    this->inHorizon()->setValue(Real(0.0125));
}

template <typename TDataType>
bool ElasticityModule<TDataType>::initializeImpl()
{
    // ElasticityModule.cu:519-546
    if (this->inHorizon()->isEmpty() || this->inPosition()->isEmpty() || this->inVelocity()->isEmpty() ||
        this->inNeighborhood()->isEmpty()) {
        std::printf("Exception: ElasticityModule's fields are not fully initialized!\n");
        return false;
    }
    int num = (int)this->inPosition()->getElementCount();
    m_bulkCoefs.resize(num);
    resetRestShape();
    this->computeMaterialStiffness();
    return true;
}

template <typename TDataType>
void ElasticityModule<TDataType>::resetRestShape()
{
    auto& nbr = this->inNeighborhood()->getValue();
    pk_ctx* c = contextOf(this);
    pkCheck(pk_pd_init(c, F(this->inPosition()->getValue()), (int)this->inPosition()->getElementCount(),
                       nbr.getIndex().getDataPtr(), nbr.getElements().getDataPtr(), nbr.getNeighborLimit(),
                       nbr.total(), this->inHorizon()->getValue(), 0),
            c, "ElasticityModule::resetRestShape");
}

template <typename TDataType>
void ElasticityModule<TDataType>::computeMaterialStiffness()
{
    // EM_InitBulkStiffness (ElasticityModule.cu:371-387): every particle 1.
    // The context starts at 1 already; subclasses that fill m_bulkCoefs
    // push it with pk_pd_set_bulk here.
    std::vector<Real> ones((size_t)m_bulkCoefs.size(), Real(1));
    if (!ones.empty())
        cudaMemcpy(m_bulkCoefs.getDataPtr(), ones.data(), sizeof(Real) * ones.size(), cudaMemcpyHostToDevice);
    pk_ctx* c = contextOf(this);
    pkCheck(pk_pd_set_bulk(c, m_bulkCoefs.getDataPtr(), m_bulkCoefs.size(), 0), c,
            "ElasticityModule::computeMaterialStiffness");
}

template <typename TDataType>
pk_pd_params ElasticityModule<TDataType>::stepParams()
{
    return pk_pd_params{this->inHorizon()->getValue(), m_mu.getValue(), m_lambda.getValue(), 1,
                        this->getParent()->getDt(), 0};
}

template <typename TDataType>
void ElasticityModule<TDataType>::beginSolve()
{
    pk_ctx* c = contextOf(this);
    pk_pd_params p = stepParams();
    pkCheck(pk_pd_begin(c, F(this->inPosition()->getValue()), (int)this->inPosition()->getElementCount(), &p, 0),
            c, "ElasticityModule::solveElasticity");
}

template <typename TDataType>
void ElasticityModule<TDataType>::computeInverseK()
{
    pk_ctx* c = contextOf(this);
    pkCheck(pk_pd_compute_inverse_k(c, this->inHorizon()->getValue(), 0), c, "ElasticityModule::computeInverseK");
}

template <typename TDataType>
void ElasticityModule<TDataType>::enforceElasticity()
{
    // EM_EnforceElasticity + K_UpdatePosition (ElasticityModule.cu:123-292)
    pk_ctx* c = contextOf(this);
    pk_pd_params p = stepParams();
    pkCheck(pk_pd_enforce(c, F(this->inPosition()->getValue()), (int)this->inPosition()->getElementCount(), &p, 0),
            c, "ElasticityModule::enforceElasticity");
}

template <typename TDataType>
void ElasticityModule<TDataType>::updateVelocity()
{
    // K_UpdateVelocity (ElasticityModule.cu:295-306)
    pk_ctx* c = contextOf(this);
    pkCheck(pk_pd_update_velocity(c, F(this->inPosition()->getValue()), F(this->inVelocity()->getValue()),
                                  (int)this->inPosition()->getElementCount(), this->getParent()->getDt(), 0),
            c, "ElasticityModule::updateVelocity");
}

template <typename TDataType>
void ElasticityModule<TDataType>::solveElasticity()
{
    // ElasticityModule.cu:404-421
    pk_ctx* c = contextOf(this);
    pk_pd_params p{this->inHorizon()->getValue(), m_mu.getValue(), m_lambda.getValue(), m_iterNum.getValue(),
                   this->getParent()->getDt(), m_breakStretch};
    pkCheck(pk_pd_solve(c, F(this->inPosition()->getValue()), F(this->inVelocity()->getValue()),
                        (int)this->inPosition()->getElementCount(), &p, 0),
            c, "ElasticityModule::solveElasticity");
}

template <typename TDataType>
bool ElasticityModule<TDataType>::constrain()
{
    this->solveElasticity();
    return true;
}

// ====================================================== ElastoplasticityModule

template <typename TDataType>
ElastoplasticityModule<TDataType>::ElastoplasticityModule()
{
    // ElastoplasticityModule.cu:13-25 (m_c 0.001, m_phi 60/180, no full
    // reconstruction, incompressible)
}

template <typename TDataType>
typename TDataType::Real ElastoplasticityModule<TDataType>::computeA()
{
    const Real phi = m_phi.getValue();
    return Real(6.0) * m_c.getValue() * std::cos(phi) / (3.0f + std::sin(phi)) / std::sqrt(3.0f);
}

template <typename TDataType>
typename TDataType::Real ElastoplasticityModule<TDataType>::computeB()
{
    const Real phi = m_phi.getValue();
    return Real(2.0f) * std::sin(phi) / (3.0f + std::sin(phi)) / std::sqrt(3.0f);
}

template <typename TDataType>
pk_plastic_params ElastoplasticityModule<TDataType>::plasticParams()
{
    return pk_plastic_params{this->inHorizon()->getValue(), this->m_mu.getValue(), this->m_lambda.getValue(),
                             computeA(), computeB()};
}

template <typename TDataType>
bool ElastoplasticityModule<TDataType>::initializeImpl()
{
    // ElastoplasticityModule.cu:659-683: the inner DensityPBD on the body's
    // horizon, positions, velocities and neighbour list
    m_pbdModule = std::make_shared<DensityPBD<TDataType>>();
    this->inHorizon()->connect(m_pbdModule->varSmoothingLength());
    this->inPosition()->connect(m_pbdModule->inPosition());
    this->inVelocity()->connect(m_pbdModule->inVelocity());
    this->inNeighborhood()->connect(m_pbdModule->inNeighborIndex());
    m_pbdModule->setParent(this->getParent());
    m_pbdModule->initialize();
    return ElasticityModule<TDataType>::initializeImpl();
}

template <typename TDataType>
void ElastoplasticityModule<TDataType>::solveElasticity()
{
    // ElastoplasticityModule.cu:240-262
    this->beginSolve();
    this->computeInverseK();
    m_pbdModule->varIterationNumber()->setValue(1);
    const int total = this->getIterationNumber();
    for (int iter = 0; iter < total; ++iter) {
        this->enforceElasticity();
        if (m_incompressible.getValue()) m_pbdModule->constrain();
    }
    this->updateVelocity();
}

template <typename TDataType>
void ElastoplasticityModule<TDataType>::rotateRestShape()
{
    pk_ctx* c = contextOf(this);
    pkCheck(pk_pd_rotate_rest_shape(c, F(this->inPosition()->getValue()), (int)this->inPosition()->getElementCount(),
                                    this->inHorizon()->getValue(), 0),
            c, "ElastoplasticityModule::rotateRestShape");
}

template <typename TDataType>
void ElastoplasticityModule<TDataType>::applyYielding()
{
    pk_ctx* c = contextOf(this);
    pk_plastic_params p = plasticParams();
    pkCheck(pk_pd_apply_yielding(c, F(this->inPosition()->getValue()), (int)this->inPosition()->getElementCount(),
                                 &p, 0),
            c, "ElastoplasticityModule::applyYielding");
}

template <typename TDataType>
void ElastoplasticityModule<TDataType>::reconstructRestShape()
{
    auto& nbr = this->inNeighborhood()->getValue();
    pk_ctx* c = contextOf(this);
    pkCheck(pk_pd_reconstruct_rest_shape(c, F(this->inPosition()->getValue()),
                                         (int)this->inPosition()->getElementCount(), nbr.getIndex().getDataPtr(),
                                         nbr.getElements().getDataPtr(), nbr.getNeighborLimit(), nbr.total(),
                                         this->inHorizon()->getValue(),
                                         m_reconstuct_all_neighborhood.getValue() ? 1 : 0, 0),
            c, "ElastoplasticityModule::reconstructRestShape");
}

template <typename TDataType>
void ElastoplasticityModule<TDataType>::applyPlasticity()
{
    // ElastoplasticityModule.cu:264-271
    this->rotateRestShape();
    this->computeMaterialStiffness();
    this->applyYielding();
    this->reconstructRestShape();
}

template <typename TDataType>
bool ElastoplasticityModule<TDataType>::constrain()
{
    this->solveElasticity();
    this->applyPlasticity();
    return true;
}

template <typename TDataType>
FractureModule<TDataType>::FractureModule()
{
    // FractureModule.cu:7-13
    this->setCohesion(typename TDataType::Real(0.001));
    this->setIterationNumber(10);
}

template <typename TDataType>
void FractureModule<TDataType>::applyPlasticity()
{
    // FractureModule.cu:107-128; the context's stiffness is copied back into m_bulkCoefs
    pk_ctx* c = contextOf(this);
    pk_plastic_params p = this->plasticParams();
    pkCheck(pk_pd_fracture(c, F(this->inPosition()->getValue()), (int)this->inPosition()->getElementCount(), &p, 0),
            c, "FractureModule::applyPlasticity");
    if (this->m_bulkCoefs.size() > 0)
        pkCheck(pk_pd_get_bulk(c, this->m_bulkCoefs.getDataPtr(), 0), c, "FractureModule::applyPlasticity");
}

// =========================================================== ImplicitViscosity

template <typename TDataType>
ImplicitViscosity<TDataType>::ImplicitViscosity()
{
}

template <typename TDataType>
bool ImplicitViscosity<TDataType>::constrain()
{
    // ImplicitViscosity.cu:98-128
    int num = (int)m_position.getElementCount();
    if (num <= 0) return true;
    auto& nbr = m_neighborhood.getValue();
    pk_ctx* c = contextOf(this);
    pkCheck(pk_viscosity(c, F(m_position.getValue()), F(m_velocity.getValue()), num, nbr.getIndex().getDataPtr(),
                         nbr.getElements().getDataPtr(), nbr.getNeighborLimit(), nbr.total(),
                         m_viscosity.getValue(), m_smoothingLength.getValue(), m_maxInteration,
                         this->getParent()->getDt(), 0),
            c, "ImplicitViscosity::constrain");
    return true;
}

// ========================================================== BoundaryConstraint

template <typename TDataType>
void BoundaryConstraint<TDataType>::setCube(Coord lo, Coord hi, Real distance, bool inverted)
{
    m_lo = lo;
    m_hi = hi;
    m_distance = distance;
    m_inverted = inverted;
    float l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
    pk_ctx* c = contextOf(this);
    pkCheck(pk_boundary_set_box(c, l, h, distance, inverted ? 1 : 0, 0), c, "BoundaryConstraint::setCube");
    m_set = true;
}

template <typename TDataType>
bool BoundaryConstraint<TDataType>::constrain(DeviceArray<Coord>& position, DeviceArray<Coord>& velocity,
                                              Real dt)
{
    if (!m_set) return false;
    pk_ctx* c = contextOf(this);
    pkCheck(pk_boundary_constrain(c, F(position), F(velocity), position.size(), m_normal_friction,
                                  m_tangent_friction, dt, 0),
            c, "BoundaryConstraint::constrain");
    return true;
}

// ===================================================== PositionBasedFluidModel

template <typename TDataType>
PositionBasedFluidModel<TDataType>::PositionBasedFluidModel()
{
}

template <typename TDataType>
bool PositionBasedFluidModel<TDataType>::initializeImpl()
{
    // PositionBasedFluidModel.cpp:41-80 (the viscosity module is not part of
    // this hot path and is not created)
    Node* parent = this->getParent();
    m_nbrQuery = parent->template addComputeModule<NeighborQuery<TDataType>>("neighborhood");
    m_smoothingLength.connect(m_nbrQuery->inRadius());
    m_position.connect(m_nbrQuery->inPosition());
    m_nbrQuery->setNeighborSizeLimit(m_cap);
    if (!m_nbrQuery->initialize()) return false;

    m_pbdModule = parent->template addConstraintModule<DensityPBD<TDataType>>("density_constraint");
    m_smoothingLength.connect(m_pbdModule->varSmoothingLength());
    m_pbdModule->varIterationNumber()->setValue(m_iterations);
    m_pbdModule->varSamplingDistance()->setValue(m_samplingDistance);
    m_position.connect(m_pbdModule->inPosition());
    m_velocity.connect(m_pbdModule->inVelocity());
    m_nbrQuery->outNeighborhood()->connect(m_pbdModule->inNeighborIndex());
    m_pbdModule->initialize();

    m_integrator = parent->template setNumericalIntegrator<ParticleIntegrator<TDataType>>("integrator");
    m_position.connect(m_integrator->inPosition());
    m_velocity.connect(m_integrator->inVelocity());
    m_forceDensity.connect(m_integrator->inForceDensity());
    m_integrator->initialize();

    if (m_viscosity > Real(0)) {
        m_visModule = parent->template addConstraintModule<ImplicitViscosity<TDataType>>("viscosity");
        m_visModule->setViscosity(m_viscosity);
        m_smoothingLength.connect(&m_visModule->m_smoothingLength);
        m_position.connect(&m_visModule->m_position);
        m_velocity.connect(&m_visModule->m_velocity);
        m_nbrQuery->outNeighborhood()->connect(&m_visModule->m_neighborhood);
        m_visModule->initialize();
    }
    return true;
}

template <typename TDataType>
void PositionBasedFluidModel<TDataType>::step(float dt)
{
    // PositionBasedFluidModel.cpp:83-101
    (void)dt;
    m_integrator->begin();
    m_nbrQuery->compute();
    m_integrator->integrate();
    m_pbdModule->constrain();
    if (m_visModule) m_visModule->constrain();
    m_integrator->end();
}

// ================================================================ nodes

template <typename TDataType>
void ParticleSystem<TDataType>::setParticles(const std::vector<Coord>& pos, const std::vector<Coord>& vel)
{
    int n = (int)pos.size();
    this->currentPosition()->setElementCount(n);
    this->currentVelocity()->setElementCount(n);
    this->currentForce()->setElementCount(n);
    if (n == 0) return;
    cudaMemcpy(this->currentPosition()->getValue().getDataPtr(), pos.data(), sizeof(Coord) * n,
               cudaMemcpyHostToDevice);
    cudaMemcpy(this->currentVelocity()->getValue().getDataPtr(), vel.data(), sizeof(Coord) * n,
               cudaMemcpyHostToDevice);
}

template <typename TDataType>
void ParticleSystem<TDataType>::getParticles(std::vector<Coord>& pos, std::vector<Coord>& vel)
{
    int n = (int)this->currentPosition()->getElementCount();
    pos.resize(n);
    vel.resize(n);
    if (n == 0) return;
    cudaMemcpy(pos.data(), this->currentPosition()->getValue().getDataPtr(), sizeof(Coord) * n,
               cudaMemcpyDeviceToHost);
    cudaMemcpy(vel.data(), this->currentVelocity()->getValue().getDataPtr(), sizeof(Coord) * n,
               cudaMemcpyDeviceToHost);
}

template <typename TDataType>
ParticleFluid<TDataType>::ParticleFluid(std::string name) : ParticleSystem<TDataType>(std::move(name))
{
    m_model_pbf = this->template setNumericalModel<PositionBasedFluidModel<TDataType>>("pbd");
}

template <typename TDataType>
bool ParticleFluid<TDataType>::initialize()
{
    this->currentPosition()->connect(&m_model_pbf->m_position);
    this->currentVelocity()->connect(&m_model_pbf->m_velocity);
    this->currentForce()->connect(&m_model_pbf->m_forceDensity);
    return m_model_pbf->initialize();
}

template <typename TDataType>
void ParticleFluid<TDataType>::advance(float dt)
{
    m_model_pbf->step(dt);
}

template <typename TDataType>
ParticleElasticBody<TDataType>::ParticleElasticBody(std::string name)
    : ParticleSystem<TDataType>(std::move(name))
{
    // ParticleElasticBody.cpp:15-42
    auto integrator = this->template setNumericalIntegrator<ParticleIntegrator<TDataType>>("integrator");
    this->currentPosition()->connect(integrator->inPosition());
    this->currentVelocity()->connect(integrator->inVelocity());
    this->currentForce()->connect(integrator->inForceDensity());

    auto nbrQuery = this->template addComputeModule<NeighborQuery<TDataType>>("neighborhood");
    m_horizon.connect(nbrQuery->inRadius());
    this->currentPosition()->connect(nbrQuery->inPosition());

    auto elasticity = this->template addConstraintModule<ElasticityModule<TDataType>>("elasticity");
    m_horizon.connect(elasticity->inHorizon());
    this->currentPosition()->connect(elasticity->inPosition());
    this->currentVelocity()->connect(elasticity->inVelocity());
    nbrQuery->outNeighborhood()->connect(elasticity->inNeighborhood());
}

template <typename TDataType>
bool ParticleElasticBody<TDataType>::initialize()
{
    // ParticleSystem::initialize -> module initialisation in pipeline order
    auto integrator = this->template getModule<ParticleIntegrator<TDataType>>("integrator");
    auto nbrQuery = this->template getModule<NeighborQuery<TDataType>>("neighborhood");
    auto elasticity = this->template getModule<ElasticityModule<TDataType>>("elasticity");
    return integrator->initialize() && nbrQuery->initialize() && (elasticity == nullptr || elasticity->initialize());
}

template <typename TDataType>
void ParticleElasticBody<TDataType>::advance(float dt)
{
    // ParticleElasticBody.cpp:84-98: the neighbour list stays frozen
    (void)dt;
    auto integrator = this->template getModule<ParticleIntegrator<TDataType>>("integrator");
    auto module = this->template getModule<ElasticityModule<TDataType>>("elasticity");
    integrator->begin();
    integrator->integrate();
    if (module != nullptr) module->constrain();
    integrator->end();
}

template <typename TDataType>
std::shared_ptr<ElasticityModule<TDataType>> ParticleElasticBody<TDataType>::getElasticitySolver()
{
    return this->template getModule<ElasticityModule<TDataType>>("elasticity");
}

template <typename TDataType>
void ParticleElasticBody<TDataType>::setElasticitySolver(std::shared_ptr<ElasticityModule<TDataType>> solver)
{
    // ParticleElasticBody.cpp:123-137
    auto nbrQuery = this->template getModule<NeighborQuery<TDataType>>("neighborhood");
    auto module = this->template getModule<ElasticityModule<TDataType>>("elasticity");
    this->currentPosition()->connect(solver->inPosition());
    this->currentVelocity()->connect(solver->inVelocity());
    nbrQuery->outNeighborhood()->connect(solver->inNeighborhood());
    m_horizon.connect(solver->inHorizon());
    if (module) this->deleteModule(module);
    solver->setName("elasticity");
    this->addConstraintModule(solver);
}

// =================================================== ParticleElastoplasticBody

template <typename TDataType>
ParticleElastoplasticBody<TDataType>::ParticleElastoplasticBody(std::string name)
    : ParticleSystem<TDataType>(std::move(name))
{
    // ParticleElastoplasticBody.cpp:20-63 (surface mesh and its mapping left out)
    m_integrator = this->template setNumericalIntegrator<ParticleIntegrator<TDataType>>("integrator");
    this->currentPosition()->connect(m_integrator->inPosition());
    this->currentVelocity()->connect(m_integrator->inVelocity());
    this->currentForce()->connect(m_integrator->inForceDensity());

    m_nbrQuery = this->template addComputeModule<NeighborQuery<TDataType>>("neighborhood");
    m_horizon.connect(m_nbrQuery->inRadius());
    this->currentPosition()->connect(m_nbrQuery->inPosition());

    auto plasticity = this->template addConstraintModule<ElastoplasticityModule<TDataType>>("elastoplasticity");
    this->currentPosition()->connect(plasticity->inPosition());
    this->currentVelocity()->connect(plasticity->inVelocity());
    m_nbrQuery->outNeighborhood()->connect(plasticity->inNeighborhood());
    m_horizon.connect(plasticity->inHorizon());

    m_pbdModule = this->template addConstraintModule<DensityPBD<TDataType>>("pbd");
    m_horizon.connect(m_pbdModule->varSmoothingLength());
    this->currentPosition()->connect(m_pbdModule->inPosition());
    this->currentVelocity()->connect(m_pbdModule->inVelocity());
    m_nbrQuery->outNeighborhood()->connect(m_pbdModule->inNeighborIndex());

    m_visModule = this->template addConstraintModule<ImplicitViscosity<TDataType>>("viscosity");
    m_visModule->setViscosity(Real(1));
    m_horizon.connect(&m_visModule->m_smoothingLength);
    this->currentPosition()->connect(&m_visModule->m_position);
    this->currentVelocity()->connect(&m_visModule->m_velocity);
    m_nbrQuery->outNeighborhood()->connect(&m_visModule->m_neighborhood);
}

template <typename TDataType>
std::shared_ptr<ElastoplasticityModule<TDataType>> ParticleElastoplasticBody<TDataType>::getElastoplasticitySolver()
{
    return this->template getModule<ElastoplasticityModule<TDataType>>("elastoplasticity");
}

template <typename TDataType>
void ParticleElastoplasticBody<TDataType>::setElastoplasticitySolver(
    std::shared_ptr<ElastoplasticityModule<TDataType>> solver)
{
    // ParticleElastoplasticBody.cpp:135-150
    auto module = getElastoplasticitySolver();
    if (module) this->deleteModule(module);
    this->currentPosition()->connect(solver->inPosition());
    this->currentVelocity()->connect(solver->inVelocity());
    m_nbrQuery->outNeighborhood()->connect(solver->inNeighborhood());
    m_horizon.connect(solver->inHorizon());
    solver->setName("elastoplasticity");
    this->addConstraintModule(solver);
}

template <typename TDataType>
bool ParticleElastoplasticBody<TDataType>::initialize()
{
    // ParticleElastoplasticBody.cpp:106-112: the list first, then the modules
    if (!m_nbrQuery->initialize()) return false;
    m_nbrQuery->compute();
    auto plasticity = getElastoplasticitySolver();
    return m_integrator->initialize() && plasticity->initialize() && m_pbdModule->initialize() &&
           m_visModule->initialize();
}

template <typename TDataType>
void ParticleElastoplasticBody<TDataType>::advance(float dt)
{
    // ParticleElastoplasticBody.cpp:73-91
    (void)dt;
    auto module = getElastoplasticitySolver();
    m_integrator->begin();
    m_integrator->integrate();
    m_nbrQuery->compute();
    module->solveElasticity();
    m_nbrQuery->compute();
    module->applyPlasticity();
    m_visModule->constrain();
    m_integrator->end();
}

template <typename TDataType>
void StaticBoundary<TDataType>::loadCube(Coord lo, Coord hi, Real distance, bool bOutBoundary)
{
    auto boundary = std::make_shared<BoundaryConstraint<TDataType>>();
    boundary->setCube(lo, hi, distance, bOutBoundary);
    m_obstacles.push_back(boundary);
}

template <typename TDataType>
void StaticBoundary<TDataType>::advance(float dt)
{
    for (auto& ob : m_obstacles)
        for (auto& ps : m_systems)
            ob->constrain(ps->currentPosition()->getValue(), ps->currentVelocity()->getValue(), dt);
}

template class NeighborQuery<DataType3f>;
template class SummationDensity<DataType3f>;
template class DensityPBD<DataType3f>;
template class ParticleIntegrator<DataType3f>;
template class ElasticityModule<DataType3f>;
template class ImplicitViscosity<DataType3f>;
template class ElastoplasticityModule<DataType3f>;
template class FractureModule<DataType3f>;
template class ParticleElastoplasticBody<DataType3f>;
template class BoundaryConstraint<DataType3f>;
template class PositionBasedFluidModel<DataType3f>;
template class ParticleSystem<DataType3f>;
template class ParticleFluid<DataType3f>;
template class ParticleElasticBody<DataType3f>;
template class StaticBoundary<DataType3f>;

}  // namespace PhysIKA
