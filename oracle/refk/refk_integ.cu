// TEST INFRASTRUCTURE ONLY (golden-fixture driver): ParticleIntegrator's kernels.
#include "prelude.h"
#include "Dynamics/ParticleSystem/ParticleIntegrator.cu"
#include "refk.h"

namespace refk {
using namespace PhysIKA;

void integrate(DArr<Coord>& pos, DArr<Coord>& vel, DArr<Coord>& force, Coord g, Real dt)
{
    force.reset();
    cuExecute(pos.size(), K_UpdateVelocity, vel, force, g, dt);
    cuExecute(pos.size(), K_UpdatePosition, pos, vel, dt);
    cuSafeCall(cudaDeviceSynchronize());
}
}  // namespace refk
