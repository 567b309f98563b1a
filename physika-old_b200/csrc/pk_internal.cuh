// pk_internal.cuh -- shared definitions of the sm_100a particle-constraint kernels.
//
// Data layout in HBM (per context, grown on demand, never shrunk):
//   perm[n]      sorted slot -> caller particle id (cell-key order, ids ascending in a cell)
//   inv[n]       caller particle id -> sorted slot
//   xs_pre[n]    float4 positions the neighbour list was built on (sorted order)
//   xs0/xa/xb[n] float4 solver positions (x_old and the two Jacobi buffers)
//   vs[n]        float4 velocities (sorted order)
//   rows[n*row_cap] int32 neighbour rows in sorted space:
//                bit31: j is in N(i) (i's capped list), bit30: i is in N(j),
//                bits 0-29: sorted index j.  Entries with bit31 come first.
//   rcnt[n]      int2 {#entries with bit31, #entries in the row}
//   tau[n]       uint2 {float bits of the cap-th smallest distance, its caller id}
//   cell_cnt / cell_start  dense blocked-Morton cell table (nkeys + 1 / + 2)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pk_hot.h"

namespace pk {

constexpr float kEpsilon = 1e-6f;  // cuda_utilities.h:30
constexpr int kRowFlagA = 1 << 31;
constexpr int kRowFlagB = 1 << 30;
constexpr int kRowIndexMask = (1 << 30) - 1;
// Per-particle row capacity of the hit rows and solver rows held in the main
// arrays (kRowCapMin, or 2 cap for a larger cap; kRowCapDynamic or
// max_neighbors for a dynamic list).  A particle with more hits keeps the rest of its hit row and
// of its solver row in the spill pool, so no count of particles inside one
// radius is too large for a list.
#ifndef PK_ROWCAP_MIN
#define PK_ROWCAP_MIN 128
#endif
constexpr int kRowCapMin = PK_ROWCAP_MIN;
constexpr int kRowCapDynamic = 192;  // dynamic lists by default (every hit is a row entry)
constexpr int kRowCapMax = 4096;

// Solver rows are interleaved by blocks of 32 sorted particles and quads of
// entries: entries 4q .. 4q+3 of particle s are 16 contiguous bytes at
// (((s / 32) * ceil(row_cap / 4) + q) * 32 + s % 32) * 4.  A warp whose lanes
// walk their rows in step reads 512 contiguous bytes per quad (one 16-byte
// load per lane), and at any entry index its lanes gather from a few
// neighbour cells.  The array holds ceil(n / 32) * 32 * ceil(row_cap / 4) * 4
// entries (row_slots).
__host__ __device__ inline int row_quads(int row_cap) { return (row_cap + 3) >> 2; }
__host__ __device__ inline long long row_slot(int s, int e, int row_cap)
{
    return (((long long)(s >> 5) * row_quads(row_cap) + (e >> 2)) * 32 + (s & 31)) * 4 + (e & 3);
}
__host__ __device__ inline long long row_slots(long long n, int row_cap)
{
    return ((n + 31) & ~31LL) * 4LL * row_quads(row_cap);
}

// Row entry e of sorted particle s (e < its row length): the main array up
// to the row capacity, then the particle's spill segment.
struct RowView {
    const int* rows;
    const int* rpool;
    const int* ovf;
    int rc;
    __device__ __forceinline__ int at(int s, int e) const
    {
        return e < rc ? rows[row_slot(s, e, rc)] : rpool[ovf[s] + (e - rc)];
    }
};

// Error bits latched in Ctx::d_err.
constexpr int kErrRowOverflow = 1;  // a row over the capacity of a build without spill
constexpr int kErrHitOverflow = 2;  // the spill pool ran out (it grows for the next build)
constexpr int kErrPublicOverflow = 4;
constexpr int kErrBadIndex = 8;  // a particle id outside [0, n) (pins)

// Uniform grid of the reference's GridHash (GridHash.cu:46-75): cell = radius,
// two cells of padding.  Keys are blocked Morton: 4x4x4 cell blocks in
// row-major block order, Morton order inside a block, so the 27 cells around
// a particle sit in a few contiguous key ranges.
struct Grid {
    float ds;
    float lo[3];
    int nx, ny, nz;
    int bx, by, bz;       // blocks per axis
    long long nkeys;      // keys of all scenes: nscenes * scene_keys
    long long scene_keys; // bx*by*bz*64, the keys of one scene's grid
    int nscenes;          // scenes stepped together (1: a single scene)
    const int* scene_off; // device, nscenes + 1 caller-order particle offsets (null when 1)
};

// Scene of caller particle i (0 for a single scene): scenes share one grid
// geometry and each owns a disjoint key range [scene * scene_keys, ...), so no
// particle ever meets another scene's particles.
__device__ inline int scene_of(const Grid& g, int i)
{
    if (g.nscenes <= 1) return 0;
    int lo = 0, hi = g.nscenes;  // scene_off[lo] <= i < scene_off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(g.scene_off + mid) <= i)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}
__device__ inline int scene_key_base(const Grid& g, int i) { return (int)(scene_of(g, i) * g.scene_keys); }

__host__ __device__ inline int morton2bit3(int i, int j, int k)
{
    return (i & 1) | ((j & 1) << 1) | ((k & 1) << 2) | ((i & 2) << 2) | ((j & 2) << 3) |
           ((k & 2) << 4);
}

// Key of valid cell (i,j,k); -1 if outside the grid (GridHash::getIndex, GridHash.h:37-44).
__host__ __device__ inline int cell_key(const Grid& g, int i, int j, int k)
{
    if (i < 0 || i >= g.nx || j < 0 || j >= g.ny || k < 0 || k >= g.nz) return -1;
    int b = ((k >> 2) * g.by + (j >> 2)) * g.bx + (i >> 2);
    return (b << 6) | morton2bit3(i & 3, j & 3, k & 3);
}

// GridHash::getIndex3 (GridHash.h:55-62): IEEE divide then floor.
__device__ inline int3 cell3(const Grid& g, float x, float y, float z)
{
    int3 c;
    c.x = (int)floorf(__fdiv_rn(__fsub_rn(x, g.lo[0]), g.ds));
    c.y = (int)floorf(__fdiv_rn(__fsub_rn(y, g.lo[1]), g.ds));
    c.z = (int)floorf(__fdiv_rn(__fsub_rn(z, g.lo[2]), g.ds));
    return c;
}

// offset1[27][3] (NeighborQuery.cu:14-41): visiting order of the 27 cells.
__constant__ const int kOffset27[27][3] = {
    {0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {1, 0, 0}, {0, 0, -1}, {0, -1, 0}, {-1, 0, 0},
    {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1},
    {-1, 0, -1}, {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 1, 1}, {1, 1, -1},
    {1, -1, 1}, {-1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};

// |a - b| exactly as Vector3f::norm() of the reference's device code
// (vector_3d.inl:208-212 -> glm length = sqrt(dot)), with every rounding
// explicit so the neighbour decision d < h is bit-reproducible.
#ifndef PK_NORM_VARIANT
#define PK_NORM_VARIANT 1
#endif
__device__ __forceinline__ float exact_norm3(float dx, float dy, float dz)
{
#if PK_NORM_VARIANT == 0
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
#elif PK_NORM_VARIANT == 2
    return __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))));
#else
    return __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy))));
#endif
}

__device__ __forceinline__ float exact_dist(float4 a, float4 b)
{
    return exact_norm3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}

// SpikyKernel (Kernel.h:36-57) with the constants folded per launch:
// W = cw * d^3, grad = cg * d^2, d = 1 - r/h, zero for r/h > 1.
struct Spiky {
    float h, inv_h, cw, cg;
};

__device__ __forceinline__ void spiky_wg(const Spiky& k, float r, float& w, float& g)
{
    float q = r * k.inv_h;
    if (q > 1.0f) {
        w = 0.0f;
        g = 0.0f;
    } else {
        float d = 1.0f - q;
        float d2 = d * d;
        w = k.cw * d2 * d;
        g = k.cg * d2;
    }
}

// Host-side construction of the grid (GridHash::setSpace, GridHash.cu:46-75).
Grid make_grid(float h, const float lo[3], const float hi[3]);
Spiky make_spiky(float h);

// Device kernels launched by the API layer (defined in pk_nbr.cu / pk_pbd.cu / pk_pd.cu).
struct Ctx;

}  // namespace pk
