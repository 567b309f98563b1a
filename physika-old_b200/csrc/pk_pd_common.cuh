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

// Eight lanes of one warp per particle (lane `sub` takes bonds sub, sub + 8,
// ...); the idle lanes of the last group mirror particle n - 1 and write
// nothing.  sum8 combines a group's partial sums with xor shuffles in a fixed
// order.
struct Lane8 {
    int i, sub;
    bool valid;
};
__device__ __forceinline__ Lane8 lane8_of(int n)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    Lane8 L;
    L.i = (int)(gid >> 3);
    L.sub = (int)(gid & 7);
    L.valid = L.i < n;
    if (!L.valid) L.i = n - 1;
    return L;
}
__device__ __forceinline__ float sum8(float v)
{
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
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

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations in double.
// After four sweeps an off-diagonal element too small to change either
// diagonal element it couples (|a_pp| + 100 |a_pq| == |a_pp|, likewise a_qq)
// is set to zero instead of rotated (the threshold rule of Numerical Recipes'
// jacobi, Press et al.), so the sweeps end once the matrix is diagonal to
// double precision instead of running on rounding noise.
__device__ inline void jacobi3(double A[3][3], double Q[3][3], double w[3])
{
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) Q[p][q] = (p == q) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
        if (off < 1e-300) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                double apq = A[p][q];
                const double g = 100.0 * fabs(apq);
                if (sweep > 3 && fabs(A[p][p]) + g == fabs(A[p][p]) && fabs(A[q][q]) + g == fabs(A[q][q])) {
                    A[p][q] = A[q][p] = 0.0;
                    continue;
                }
                if (fabs(apq) < 1e-300) continue;
                double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < 3; ++r) {
                    double arp = A[r][p], arq = A[r][q];
                    A[r][p] = c * arp - s * arq;
                    A[r][q] = s * arp + c * arq;
                }
                for (int r = 0; r < 3; ++r) {
                    double apr = A[p][r], aqr = A[q][r];
                    A[p][r] = c * apr - s * aqr;
                    A[q][r] = s * apr + c * aqr;
                }
                for (int r = 0; r < 3; ++r) {
                    double qrp = Q[r][p], qrq = Q[r][q];
                    Q[r][p] = c * qrp - s * qrq;
                    Q[r][q] = s * qrp + c * qrq;
                }
            }
    }
    for (int p = 0; p < 3; ++p) w[p] = A[p][p];
}

}  // namespace pk
