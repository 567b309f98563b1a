// pk_pd_common.cuh -- bond-list access and kernel functions shared by the
// peridynamics kernels (ElasticityModule, Dynamics/ParticleSystem/ElasticityModule.cu).
#pragma once
#include "pk_internal.cuh"

namespace pk {

// NeighborList::getNeighborSize / getElement (NeighborList.h:27-59) on the
// frozen rest shape (fixed layout: cap > 0; CSR: cap == 0).
__device__ __forceinline__ int pd_size(const int* index, int cap, long long total, int n, int i)
{
    if (cap > 0) return index[i];
    if (i >= n - 1) return (int)(total - index[i]);
    return index[i + 1] - index[i];
}
__device__ __forceinline__ long long pd_at(const int* index, int cap, int i, int k)
{
    return cap > 0 ? (long long)cap * i + k : (long long)index[i] + k;
}

// CorrectedKernel / SmoothKernel (Kernel.h:68-75,99-142), float.
__device__ __forceinline__ float smooth_w(float r, float h)
{
    float q = r / h;
    return q > 1.0f ? 0.0f : (1.0f - q * q);
}
__device__ __forceinline__ float corr_w(float r, float h)
{
    float q = r / h;
    return q * q * q * smooth_w(r, h);
}
__device__ __forceinline__ float corr_wrr(float r, float h)
{
    float q = r / h;
    return q * smooth_w(r, h) / (h * h);
}

}  // namespace pk
