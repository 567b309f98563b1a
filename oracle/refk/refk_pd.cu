// TEST INFRASTRUCTURE ONLY (golden-fixture driver): ElasticityModule's kernels.
#include "prelude.h"
#include "Dynamics/ParticleSystem/ElasticityModule.cu"
#include "refk.h"

namespace refk {
using namespace PhysIKA;

void pd_rest_shape(NList<NPair>& shape, NList<int>& nbr, DArr<Coord>& pos)
{
    // resetRestShape: same index array and layout as the query's list.
    const int num = pos.size();
    shape.getIndex().resize(nbr.getIndex().size());
    if (nbr.isLimited())
        shape.setNeighborLimit(nbr.getNeighborLimit());
    else
        shape.getElements().resize(nbr.getElements().size());
    cuSafeCall(cudaMemcpy(shape.getIndex().getDataPtr(), nbr.getIndex().getDataPtr(),
                          sizeof(int) * nbr.getIndex().size(), cudaMemcpyDeviceToDevice));
    uint pDims = cudaGridSize(num, BLOCK_SIZE);
    K_UpdateRestShape<<<pDims, BLOCK_SIZE>>>(shape, nbr, pos);
    cuSafeCall(cudaDeviceSynchronize());
}

void pd_inverse_k(DArr<Matrix>& invK, NList<NPair>& shape, Real horizon)
{
    uint pDims = cudaGridSize(invK.size(), BLOCK_SIZE);
    EM_PrecomputeShape<Real, Coord, Matrix, NPair><<<pDims, BLOCK_SIZE>>>(invK, shape, horizon);
    cuSafeCall(cudaDeviceSynchronize());
}

void pd_enforce(DArr<Coord>& pos, DArr<Coord>& pos_old, DArr<Coord>& disp, DArr<Real>& weights,
                DArr<Real>& bulk, DArr<Matrix>& invK, NList<NPair>& shape, Real horizon, Real mu,
                Real lambda)
{
    uint pDims = cudaGridSize(pos.size(), BLOCK_SIZE);
    disp.reset();
    weights.reset();
    EM_EnforceElasticity<<<pDims, BLOCK_SIZE>>>(disp, weights, bulk, invK, pos, shape, horizon, mu, lambda);
    cuSafeCall(cudaDeviceSynchronize());
    K_UpdatePosition<<<pDims, BLOCK_SIZE>>>(pos, pos_old, disp, weights);
    cuSafeCall(cudaDeviceSynchronize());
}

void pd_update_velocity(DArr<Coord>& vel, DArr<Coord>& pos_old, DArr<Coord>& pos, Real dt)
{
    uint pDims = cudaGridSize(pos.size(), BLOCK_SIZE);
    K_UpdateVelocity<<<pDims, BLOCK_SIZE>>>(vel, pos_old, pos, dt);
    cuSafeCall(cudaDeviceSynchronize());
}
}  // namespace refk
