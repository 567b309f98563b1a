// TEST INFRASTRUCTURE ONLY (golden-fixture driver): DensityPBD's kernels.
#include "prelude.h"
#include "Dynamics/ParticleSystem/DensityPBD.cu"
#include "refk.h"

namespace refk {
using namespace PhysIKA;

void pbd_iteration(DArr<Coord>& pos, DArr<Coord>& vel, NList<int>& nbr, DArr<Real>& rho,
                   DArr<Real>& lambda, DArr<Coord>& dpos, Real h, Real dt, Real mass)
{
    SpikyKernel<Real> kern;
    const int num = pos.size();
    dpos.reset();
    summation_density(rho, pos, nbr, h, mass);
    cuExecute(num, K_ComputeLambdas, lambda, rho, pos, nbr, kern, h);
    cuExecute(num, K_ComputeDisplacement, dpos, lambda, pos, nbr, kern, h, dt);
    cuExecute(num, K_UpdatePosition, pos, vel, dpos, dt);
    cuSafeCall(cudaDeviceSynchronize());
}

void pbd_update_velocity(DArr<Coord>& vel, DArr<Coord>& pos_old, DArr<Coord>& pos, Real dt)
{
    cuExecute(pos.size(), DP_UpdateVelocity, vel, pos_old, pos, dt);
    cuSafeCall(cudaDeviceSynchronize());
}
}  // namespace refk
