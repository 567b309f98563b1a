// pk_boundary.cuh -- box SDF boundary (BoundaryConstraint + DistanceField3D).
//
// The SDF grid is built on the host once per box (pk_boundary_set_box) and
// sampled here.  Interior particles farther than two grid cells from every
// wall of an inverted box skip the 8-tap lookup: all 8 nodes around them are
// then positive, so the interpolated distance is positive and the reference
// would leave them untouched as well.
#pragma once
#include <curand_kernel.h>

#include "pk_internal.cuh"

namespace pk {

struct SdfView {
    const float* data;
    float left[3];
    float inv_h[3];  // (float)(1.0 / m_h) as in DistanceField3D.h:116
    float box_lo[3], box_hi[3];
    float margin;    // 2 * max cell size: early-out distance
    int nx, ny, nz;
    int inverted;
};

__device__ __forceinline__ float lerp_rn(float a, float b, float t)
{
    // (1 - t) * a + t * b (DistanceField3D.h:81-83), each operation rounded.
    return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, t), a), __fmul_rn(t, b));
}

// DistanceField3D::getDistance (DistanceField3D.h:113-170).
__device__ inline void sdf_distance(const SdfView& s, float px, float py, float pz, float& d,
                                    float3& nrm)
{
    float fx = __fmul_rn(__fsub_rn(px, s.left[0]), s.inv_h[0]);
    float fy = __fmul_rn(__fsub_rn(py, s.left[1]), s.inv_h[1]);
    float fz = __fmul_rn(__fsub_rn(pz, s.left[2]), s.inv_h[2]);
    int i = (int)floorf(fx), j = (int)floorf(fy), k = (int)floorf(fz);
    if (i < 0 || i >= s.nx - 1 || j < 0 || j >= s.ny - 1 || k < 0 || k >= s.nz - 1) {
        d = s.inverted ? -100000.0f : 100000.0f;
        nrm = make_float3(0.f, 0.f, 0.f);
        return;
    }
    float al = __fsub_rn(fx, (float)i), be = __fsub_rn(fy, (float)j), ga = __fsub_rn(fz, (float)k);
    long long sy = s.nx, sz = (long long)s.nx * s.ny;
    const float* D = s.data + i + j * sy + k * sz;
    float d000 = __ldg(D), d100 = __ldg(D + 1), d010 = __ldg(D + sy), d110 = __ldg(D + sy + 1);
    float d001 = __ldg(D + sz), d101 = __ldg(D + sz + 1), d011 = __ldg(D + sz + sy),
          d111 = __ldg(D + sz + sy + 1);
    float dx00 = lerp_rn(d000, d100, al), dx10 = lerp_rn(d010, d110, al);
    float dxy0 = lerp_rn(dx00, dx10, be);
    float dx01 = lerp_rn(d001, d101, al), dx11 = lerp_rn(d011, d111, al);
    float dxy1 = lerp_rn(dx01, dx11, be);
    float d0y0 = lerp_rn(d000, d010, be), d0y1 = lerp_rn(d001, d011, be);
    float d0yz = lerp_rn(d0y0, d0y1, ga);
    float d1y0 = lerp_rn(d100, d110, be), d1y1 = lerp_rn(d101, d111, be);
    float d1yz = lerp_rn(d1y0, d1y1, ga);
    float dx0z = lerp_rn(dx00, dx01, ga), dx1z = lerp_rn(dx10, dx11, ga);
    float n0 = __fsub_rn(d0yz, d1yz), n1 = __fsub_rn(dx0z, dx1z), n2 = __fsub_rn(dxy0, dxy1);
    float l2 = __fadd_rn(__fadd_rn(__fmul_rn(n0, n0), __fmul_rn(n1, n1)), __fmul_rn(n2, n2));
    float l = __fsqrt_rn(l2);
    if (l < 0.0001f) {
        nrm = make_float3(0.f, 0.f, 0.f);
    } else {
        float is = __fdiv_rn(1.0f, l);
        nrm = make_float3(__fmul_rn(n0, is), __fmul_rn(n1, is), __fmul_rn(n2, is));
    }
    d = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, ga), dxy0), __fmul_rn(ga, dxy1));
}

// K_ConstrainSDF body (BoundaryConstraint.cu:41-66) for caller particle `id`.
// Returns true when the particle was in contact (x, v modified).
__device__ inline bool sdf_constrain(const SdfView& s, int id, float3& x, float3& v,
                                     float normal_friction, float tangential_friction, float dt)
{
    if (s.inverted) {
        float m = fminf(fminf(fminf(x.x - s.box_lo[0], s.box_hi[0] - x.x),
                              fminf(x.y - s.box_lo[1], s.box_hi[1] - x.y)),
                        fminf(x.z - s.box_lo[2], s.box_hi[2] - x.z));
        if (m > s.margin) return false;
    }
    float dist;
    float3 n;
    sdf_distance(s, x.x, x.y, x.z, dist, n);
    if (!(dist <= 0.0f)) return false;
    float olddist = -dist;
    curandState st;
    curand_init((unsigned long long)id, 0ull, 0ull, &st);  // RandNumber(pId), CudaRand.h:12-15
    dist = __fmul_rn(0.0001f, curand_uniform(&st));
    float sh = __fadd_rn(olddist, dist);
    x.x = __fsub_rn(x.x, __fmul_rn(sh, n.x));
    x.y = __fsub_rn(x.y, __fmul_rn(sh, n.y));
    x.z = __fsub_rn(x.z, __fmul_rn(sh, n.z));
    float vn = __fadd_rn(__fadd_rn(__fmul_rn(v.x, n.x), __fmul_rn(v.y, n.y)), __fmul_rn(v.z, n.z));
    float3 vnor = make_float3(__fmul_rn(vn, n.x), __fmul_rn(vn, n.y), __fmul_rn(vn, n.z));
    float3 vtan = make_float3(__fsub_rn(v.x, vnor.x), __fsub_rn(v.y, vnor.y), __fsub_rn(v.z, vnor.z));
    if (vn > 0.0f) vnor = make_float3(-vnor.x, -vnor.y, -vnor.z);
    float fr = __fsub_rn(1.0f, normal_friction);
    vnor = make_float3(__fmul_rn(vnor.x, fr), __fmul_rn(vnor.y, fr), __fmul_rn(vnor.z, fr));
    float damp = powf(2.718281828459045f, -dt * tangential_friction);
    v = make_float3(__fmul_rn(__fadd_rn(vnor.x, vtan.x), damp),
                    __fmul_rn(__fadd_rn(vnor.y, vtan.y), damp),
                    __fmul_rn(__fadd_rn(vnor.z, vtan.z), damp));
    return true;
}

}  // namespace pk
