// pk_fixed.cu -- FixedPoints (Dynamics/ParticleSystem/FixedPoints.cu:110-169).
//
// The reference keeps a dense flag array and a dense array of target
// positions (updateContext) and launches one thread per particle
// (K_DoFixPoints :126-140).  Here the pins are a sparse list (ids, targets),
// one thread per pin: x[id] = target, v[id] = 0 as in the reference, or the
// given velocity for a kinematically moved pin (a pulled end).
#include "pk_kernels.cuh"

namespace pk {

__global__ void __launch_bounds__(256)
    k_fix_points(float* __restrict__ x, float* __restrict__ v, int n, const int* __restrict__ ids,
                 const float* __restrict__ target, const float* __restrict__ vel, int count,
                 int* __restrict__ err)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int i = ids[k];
    if (i < 0 || i >= n) {
        atomicOr(err, kErrBadIndex);
        return;
    }
    x[3 * i] = target[3 * k];
    x[3 * i + 1] = target[3 * k + 1];
    x[3 * i + 2] = target[3 * k + 2];
    v[3 * i] = vel ? vel[3 * k] : 0.0f;
    v[3 * i + 1] = vel ? vel[3 * k + 1] : 0.0f;
    v[3 * i + 2] = vel ? vel[3 * k + 2] : 0.0f;
}

// K_DoPlaneConstrain (FixedPoints.cu:150-162): tmp = dir . (x - origin);
// x -= tmp * dir where tmp < 0.  The dot product and the update use the fused
// forms nvcc gives glm's dot and `x - s*d` (the same contraction the golden
// vectors show for Vector3f::norm).
__global__ void __launch_bounds__(256)
    k_plane(float* __restrict__ x, int n, float ox, float oy, float oz, float dx, float dy, float dz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
    const float ex = __fsub_rn(px, ox), ey = __fsub_rn(py, oy), ez = __fsub_rn(pz, oz);
    const float tmp = __fmaf_rn(dz, ez, __fmaf_rn(dx, ex, __fmul_rn(dy, ey)));
    if (tmp < 0.0f) {
        x[3 * i] = __fmaf_rn(-tmp, dx, px);
        x[3 * i + 1] = __fmaf_rn(-tmp, dy, py);
        x[3 * i + 2] = __fmaf_rn(-tmp, dz, pz);
    }
}

int fix_points(float* x, float* v, int n, const int* ids, const float* target, const float* vel, int count,
               int* err, cudaStream_t st)
{
    if (count <= 0) return 0;
    k_fix_points<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(x, v, n, ids, target, vel, count, err);
    return 1;
}

int plane_constrain(float* x, int n, const float origin[3], const float dir[3], cudaStream_t st)
{
    if (n <= 0) return 0;
    k_plane<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, origin[0], origin[1], origin[2], dir[0], dir[1],
                                                         dir[2]);
    return 1;
}

}  // namespace pk
