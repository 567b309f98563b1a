// TEST INFRASTRUCTURE ONLY (golden-fixture driver): NeighborQuery's kernels.
#include "prelude.h"
#include "Framework/Topology/NeighborQuery.cu"
#include "refk.h"

namespace refk {
using namespace PhysIKA;

int neighbor_query(DArr<Coord>& pos, Real h, Coord lo, Coord hi, int cap, NList<int>& nbr)
{
    const int num = pos.size();
    GridHash<DT> hash;
    hash.setSpace(h, lo, hi);
    grid_construct(hash, pos);
    const uint pDims = cudaGridSize(num, BLOCK_SIZE);
    int total = 0;
    if (cap > 0) {
        nbr.resize(num, cap);
        int* ids = nullptr;
        Real* distance = nullptr;
        cuSafeCall(cudaMalloc((void**)&ids, (size_t)num * sizeof(int) * cap));
        cuSafeCall(cudaMalloc((void**)&distance, (size_t)num * sizeof(Real) * cap));
        K_ComputeNeighborFixed<<<pDims, BLOCK_SIZE>>>(nbr, pos, pos, hash, h, ids, distance);
        cuSafeCall(cudaDeviceSynchronize());
        cuSafeCall(cudaFree(ids));
        cuSafeCall(cudaFree(distance));
        total = num * cap;
    } else {
        nbr.resize(num);
        DeviceArray<int>& nbrNum = nbr.getIndex();
        K_CalNeighborSize<<<pDims, BLOCK_SIZE>>>(nbrNum, pos, pos, hash, h);
        cuSafeCall(cudaDeviceSynchronize());
        Reduction<int> reduce;
        Scan scan;
        total = reduce.accumulate(nbrNum.getDataPtr(), nbrNum.size());
        checked_count_and_scan(nbrNum.getDataPtr(), num, total, "dynamic list");
        std::vector<int> counts = download_ints(nbrNum.getDataPtr(), num);
        scan.exclusive(nbrNum, true);
        cuSafeCall(cudaDeviceSynchronize());
        checked_offsets(nbrNum.getDataPtr(), counts, "dynamic list");
        if (total > 0) {
            nbr.getElements().resize(total);
            K_GetNeighborElements<<<pDims, BLOCK_SIZE>>>(nbr, pos, pos, hash, h);
            cuSafeCall(cudaDeviceSynchronize());
        }
    }
    hash.release();
    return total;
}
}  // namespace refk
