// TEST INFRASTRUCTURE ONLY (golden-fixture driver): SummationDensity's kernel.
#include "prelude.h"
#include "Dynamics/ParticleSystem/SummationDensity.cu"
#include "refk.h"

namespace refk {
using namespace PhysIKA;

void summation_density(DArr<Real>& rho, DArr<Coord>& pos, NList<int>& nbr, Real h, Real mass)
{
    cuExecute(rho.size(), K_ComputeDensity, rho, pos, nbr, h, mass);
    cuSafeCall(cudaDeviceSynchronize());
}

Real density_factor(Real d, Real H, Real rho_0, Real* mass)
{
    // The loop of SummationDensity::calculateScalingFactor, in the same float
    // arithmetic, on the reference's SpikyKernel.
    Real V = d * d * d;
    SpikyKernel<Real> kern;
    Real total_weight(0);
    int half_res = H / d + 1;
    for (int i = -half_res; i <= half_res; i++)
        for (int j = -half_res; j <= half_res; j++)
            for (int k = -half_res; k <= half_res; k++) {
                Real x = i * d, y = j * d, z = k * d;
                Real r = sqrt(x * x + y * y + z * z);
                total_weight += V * kern.Weight(r, H);
            }
    *mass = rho_0 * V;
    return 1.0 / total_weight;
}
}  // namespace refk
