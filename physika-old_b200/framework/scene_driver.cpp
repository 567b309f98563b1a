// scene_driver.cpp -- headless scenes built from the Framework mirror, the way
// the reference's examples build them (Examples/App_SingleFluid: a ParticleFluid
// inside a StaticBoundary cube; App_Elasticity: a ParticleElasticBody), minus
// the GUI.  Exposed as C functions so a host application or a test can run a
// scene through the reference-named modules without writing C++.
#include <cstdio>
#include <exception>
#include <memory>
#include <vector>

#include "ParticleIO.h"
#include "ParticleModules.h"

using namespace PhysIKA;

namespace {
std::vector<Vector3f> to_coords(const float* a, int n)
{
    std::vector<Vector3f> v((size_t)n);
    for (int i = 0; i < n; ++i) v[(size_t)i] = Vector3f(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
    return v;
}
void from_coords(const std::vector<Vector3f>& v, float* a)
{
    for (size_t i = 0; i < v.size(); ++i)
        for (int c = 0; c < 3; ++c) a[3 * i + c] = v[i][c];
}
}  // namespace

extern "C" {

// A dam-break frame loop: SceneGraph bounds = [lo, hi], gravity (0, -9.8, 0);
// a ParticleFluid (PositionBasedFluidModel: NeighborQuery with `cap`, radius,
// DensityPBD with `iterations` and sampling distance `spacing`, ImplicitViscosity
// with `viscosity` (the reference's model uses 1; 0 leaves it out)) of n particles,
// and, when `boundary` is non-zero, a StaticBoundary cube [lo, hi] (SDF spacing
// sdf_spacing, particles kept inside) advanced before the fluid every frame
// (StaticBoundary.cpp:45-59).  x, v, x_out, v_out are host arrays of 3n
// floats.  Returns 0, or non-zero after printing the error.
__attribute__((visibility("default"))) int pkf_fluid_run(const float* x, const float* v, int n, const float lo[3],
                                                         const float hi[3], float spacing, float radius, int cap,
                                                         int iterations, float dt, float sdf_spacing, int boundary,
                                                         float viscosity, int steps, float* x_out, float* v_out)
{
    try {
        SceneGraph& scene = SceneGraph::getInstance();
        scene.setLowerBound(Vector3f(lo[0], lo[1], lo[2]));
        scene.setUpperBound(Vector3f(hi[0], hi[1], hi[2]));
        scene.setGravity(Vector3f(0.0f, -9.8f, 0.0f));
        auto fluid = std::make_shared<ParticleFluid<DataType3f>>("fluid");
        fluid->setDt(dt);
        auto model = fluid->getModel();
        model->m_smoothingLength.setValue(radius);
        model->setNeighborSizeLimit(cap);
        model->setIterationNumber(iterations);
        model->setSamplingDistance(spacing);
        model->setViscosity(viscosity);
        fluid->setParticles(to_coords(x, n), to_coords(v, n));
        StaticBoundary<DataType3f> walls("boundary");
        if (boundary) {
            walls.loadCube(Vector3f(lo[0], lo[1], lo[2]), Vector3f(hi[0], hi[1], hi[2]), sdf_spacing, true);
            walls.addParticleSystem(fluid);
        }
        if (!fluid->initialize()) return 1;
        for (int s = 0; s < steps; ++s) {
            if (boundary) walls.advance(dt);
            fluid->advance(dt);
        }
        std::vector<Vector3f> pos, vel;
        fluid->getParticles(pos, vel);
        from_coords(pos, x_out);
        from_coords(vel, v_out);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "pkf_fluid_run: %s\n", e.what());
        return 2;
    }
}

// The dam-break loop of pkf_fluid_run on particles loaded from an OBJ file
// (ParticleSystem::loadParticles(filename)), at rest, with a ParticleWriter
// attached to the fluid's positions: after every `write_every`-th frame it
// writes <out_path><prefix><index>.txt (color mapping 0).  Returns the number
// of particles, or a negative value after printing the error.
__attribute__((visibility("default"))) int pkf_fluid_obj_run(const char* obj_path, const float lo[3],
                                                             const float hi[3], float spacing, float radius,
                                                             int cap, int iterations, float dt, float sdf_spacing,
                                                             int boundary, float viscosity, int steps,
                                                             const char* out_path, const char* prefix,
                                                             int write_every)
{
    try {
        SceneGraph& scene = SceneGraph::getInstance();
        scene.setLowerBound(Vector3f(lo[0], lo[1], lo[2]));
        scene.setUpperBound(Vector3f(hi[0], hi[1], hi[2]));
        scene.setGravity(Vector3f(0.0f, -9.8f, 0.0f));
        auto fluid = std::make_shared<ParticleFluid<DataType3f>>("fluid");
        fluid->setDt(dt);
        auto model = fluid->getModel();
        model->m_smoothingLength.setValue(radius);
        model->setNeighborSizeLimit(cap);
        model->setIterationNumber(iterations);
        model->setSamplingDistance(spacing);
        model->setViscosity(viscosity);
        fluid->loadParticles(std::string(obj_path));
        const int n = (int)fluid->currentPosition()->getElementCount();
        StaticBoundary<DataType3f> walls("boundary");
        if (boundary) {
            walls.loadCube(Vector3f(lo[0], lo[1], lo[2]), Vector3f(hi[0], hi[1], hi[2]), sdf_spacing, true);
            walls.addParticleSystem(fluid);
        }
        ParticleWriter<DataType3f> writer;
        writer.setOutputPath(out_path ? out_path : "");
        writer.setNamePrefix(prefix ? prefix : "test_");
        fluid->currentPosition()->connect(&writer.m_position);
        writer.m_color_mapping.setElementCount(n);
        if (!fluid->initialize()) return -1;
        for (int s = 0; s < steps; ++s) {
            if (boundary) walls.advance(dt);
            fluid->advance(dt);
            if (write_every > 0 && (s + 1) % write_every == 0 && !writer.execute()) return -3;
        }
        return n;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "pkf_fluid_obj_run: %s\n", e.what());
        return -2;
    }
}

// An elastic body: ParticleElasticBody (ParticleElasticBody.cpp:15-98) with the
// given horizon and neighbour cap, bulk stiffness 1 (the reference's
// computeMaterialStiffness), gravity (0, -9.8, 0), `steps` frames of
// integrate + ElasticityModule::constrain.  Host arrays as pkf_fluid_run.
__attribute__((visibility("default"))) int pkf_elastic_run(const float* x, const float* v, int n, const float lo[3],
                                                           const float hi[3], float horizon, int cap, float dt,
                                                           int steps, float* x_out, float* v_out)
{
    try {
        SceneGraph& scene = SceneGraph::getInstance();
        scene.setLowerBound(Vector3f(lo[0], lo[1], lo[2]));
        scene.setUpperBound(Vector3f(hi[0], hi[1], hi[2]));
        scene.setGravity(Vector3f(0.0f, -9.8f, 0.0f));
        auto body = std::make_shared<ParticleElasticBody<DataType3f>>("bar");
        body->setDt(dt);
        body->varHorizon()->setValue(horizon);
        body->getModule<NeighborQuery<DataType3f>>("neighborhood")->setNeighborSizeLimit(cap);
        body->setParticles(to_coords(x, n), to_coords(v, n));
        if (!body->initialize()) return 1;
        for (int s = 0; s < steps; ++s) body->advance(dt);
        std::vector<Vector3f> pos, vel;
        body->getParticles(pos, vel);
        from_coords(pos, x_out);
        from_coords(vel, v_out);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "pkf_elastic_run: %s\n", e.what());
        return 2;
    }
}

// An elastoplastic body: ParticleElastoplasticBody (ParticleElastoplasticBody.cpp:20-91)
// with the given horizon, gravity (0, -9.8, 0) and `steps` frames; its solver
// is an ElastoplasticityModule with cohesion c and friction angle phi (degrees,
// setFrictionAngle), or a FractureModule when `fracture` is non-zero, and
// enableFullyReconstruction when `reconstruct_all` is.  Host arrays as
// pkf_fluid_run.
__attribute__((visibility("default"))) int pkf_elastoplastic_run(const float* x, const float* v, int n,
                                                                 const float lo[3], const float hi[3], float horizon,
                                                                 float dt, int fracture, float cohesion,
                                                                 float friction_deg, int reconstruct_all, int steps,
                                                                 float* x_out, float* v_out)
{
    try {
        SceneGraph& scene = SceneGraph::getInstance();
        scene.setLowerBound(Vector3f(lo[0], lo[1], lo[2]));
        scene.setUpperBound(Vector3f(hi[0], hi[1], hi[2]));
        scene.setGravity(Vector3f(0.0f, -9.8f, 0.0f));
        auto body = std::make_shared<ParticleElastoplasticBody<DataType3f>>("plastic");
        body->setDt(dt);
        body->varHorizon()->setValue(horizon);
        std::shared_ptr<ElastoplasticityModule<DataType3f>> solver;
        if (fracture)
            solver = std::make_shared<FractureModule<DataType3f>>();
        else
            solver = std::make_shared<ElastoplasticityModule<DataType3f>>();
        solver->setCohesion(cohesion);
        solver->setFrictionAngle(friction_deg);
        if (reconstruct_all) solver->enableFullyReconstruction();
        body->setElastoplasticitySolver(solver);
        body->setParticles(to_coords(x, n), to_coords(v, n));
        if (!body->initialize()) return 1;
        for (int s = 0; s < steps; ++s) body->advance(dt);
        std::vector<Vector3f> pos, vel;
        body->getParticles(pos, vel);
        from_coords(pos, x_out);
        from_coords(vel, v_out);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "pkf_elastoplastic_run: %s\n", e.what());
        return 2;
    }
}

// Independent fluid scenes stepped the way the reference steps them: every
// scene its own frame, each frame its own launches (one pk_pbf_step per scene
// per frame, issued from this host loop).  x, v: device arrays of all scenes'
// particles concatenated; offsets: host array of nscenes + 1 particle offsets.
// The baseline against which pk_pbf_step_batched (one frame for all scenes)
// is measured.  Returns the first non-zero pk status, else 0.
__attribute__((visibility("default"))) int pkf_pbf_frames_per_scene(pk_ctx* ctx, float* x, float* v,
                                                                    const int* offsets, int nscenes,
                                                                    const pk_pbf_params* p, int frames,
                                                                    pk_stream stream)
{
    if (!ctx || !x || !v || !offsets || nscenes < 1 || !p || frames < 0) return PK_ERR_ARG;
    for (int f = 0; f < frames; ++f)
        for (int s = 0; s < nscenes; ++s) {
            const int a = offsets[s], n = offsets[s + 1] - a;
            const int rc = pk_pbf_step(ctx, x + 3LL * a, v + 3LL * a, n, p, nullptr, stream);
            if (rc != PK_OK) return rc;
        }
    return PK_OK;
}

}  // extern "C"
