// TEST INFRASTRUCTURE ONLY (golden-fixture driver): the reference's grid hash,
// Framework/Topology/GridHash.cu, compiled where it lies. Its explicit
// instantiation provides GridHash<DataType3f>::setSpace/clear/release.
#include <vector>
#include "prelude.h"
#include "Framework/Topology/GridHash.cu"
#include "refk.h"

namespace refk {
using namespace PhysIKA;

void checked_count_and_scan(int* d_counts, int num, int reduced, const char* what)
{
    // The reference sizes its id array by Reduction<int>::accumulate and places
    // each id at the exclusive scan of the counts. Its warp stage
    // (Reduction.cu:53-63) is volatile warp-synchronous code without
    // __syncwarp; before any kernel writes at those positions, the driver
    // checks the reduced sum and (after the caller's scan) the offsets against
    // a host computation, and stops on a mismatch instead of writing out of
    // bounds.
    std::vector<int> h(num);
    cuSafeCall(cudaMemcpy(h.data(), d_counts, sizeof(int) * num, cudaMemcpyDeviceToHost));
    long long s = 0;
    for (int v : h) s += v;
    if (s != reduced) {
        fprintf(stderr, "pkref_driver: %s: reduced sum %d differs from the host sum %lld\n", what, reduced, s);
        exit(4);
    }
}

void checked_offsets(int* d_offsets, const std::vector<int>& counts, const char* what)
{
    std::vector<int> h(counts.size());
    cuSafeCall(cudaMemcpy(h.data(), d_offsets, sizeof(int) * h.size(), cudaMemcpyDeviceToHost));
    long long s = 0;
    for (size_t k = 0; k < h.size(); k++) {
        if (h[k] != s) {
            fprintf(stderr, "pkref_driver: %s: scan offset %zu is %d, expected %lld\n", what, k, h[k], s);
            exit(4);
        }
        s += counts[k];
    }
}

std::vector<int> download_ints(int* d, int num)
{
    std::vector<int> h(num);
    cuSafeCall(cudaMemcpy(h.data(), d, sizeof(int) * num, cudaMemcpyDeviceToHost));
    return h;
}

void grid_construct(GridHash<DT>& hash, DArr<Coord>& pos)
{
    // GridHash::construct (GridHash.cu:297-323), the same launches in the same
    // order, with the checks above between them.
    hash.clear();
    dim3 pDims = int(ceil(pos.size() / BLOCK_SIZE + 0.5f));
    K_CalculateParticleNumber<<<pDims, BLOCK_SIZE>>>(hash, pos);
    cuSafeCall(cudaDeviceSynchronize());
    hash.particle_num = hash.m_reduce->accumulate(hash.index, hash.num);
    checked_count_and_scan(hash.index, hash.num, hash.particle_num, "grid hash");
    std::vector<int> counts = download_ints(hash.index, hash.num);
    if (hash.m_scan == nullptr) hash.m_scan = new Scan();
    hash.m_scan->exclusive(hash.index, hash.num);
    cuSafeCall(cudaDeviceSynchronize());
    checked_offsets(hash.index, counts, "grid hash");
    if (hash.ids != nullptr) cuSafeCall(cudaFree(hash.ids));
    cuSafeCall(cudaMalloc((void**)&hash.ids, hash.particle_num * sizeof(int)));
    K_ConstructHashTable<<<pDims, BLOCK_SIZE>>>(hash, pos);
    cuSafeCall(cudaDeviceSynchronize());
}
}  // namespace refk
