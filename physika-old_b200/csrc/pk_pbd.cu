// pk_pbd.cu -- DensityPBD (with SummationDensity) and ParticleIntegrator.
//
// Fast path: the rows built by pk_nbr.cu in sorted space.  One Jacobi
// iteration of the reference (DensityPBD::takeOneIteration,
// DensityPBD.cu:305-365: density, lambdas, displacement with atomics,
// position update) is two gather passes here:
//   pass A: rho_i and lambda_i over N(i) (K_ComputeDensity
//           SummationDensity.cu:13-36 + K_ComputeLambdas DensityPBD.cu:46-90),
//   pass B: x_i' = x_i + sum over the row of m_ij * dp_ij, m_ij = [j in N(i)]
//           + [i in N(j)] -- the same sum the reference's scatter
//           (+dp_ij to i, -dp_ij to j, DensityPBD.cu:134-179) accumulates,
//           since dp_ji = -dp_ij bit for bit.
// One thread per particle walks its solver row; rows are interleaved by
// blocks of 32 particles (row_slot), so a warp's row reads are one line per
// entry and its gathers at one entry index touch a few neighbour cells.
// Jacobi: pass A reads x, writes (x, lambda) to xl; pass B reads xl only and
// writes x'.
#include <algorithm>

#include "pk_kernels.cuh"

namespace pk {

// Per-pair constants of the two passes (Spiky kernel, Kernel.h SpikyKernel).
struct PassK {
    float inv_h, cwm, cg, c10g;
};
__host__ __device__ inline PassK pass_k(const Spiky& k, float mass)
{
    return PassK{k.inv_h, mass * k.cw, k.cg, 10.0f * k.cg};
}
constexpr float kEps2 = kEpsilon * kEpsilon;  // r > EPSILON  <=>  r^2 > EPSILON^2

// Pair geometry shared by both passes: r from one reciprocal square root
// (r = d2 / sqrt(d2); d2 = 0 gives r = 0), 1/r, and d = 1 - r/h clamped at 0,
// so w = cw d^3 and |grad| = cg d^2 vanish beyond h as in SpikyKernel.
__device__ __forceinline__ void pair_geom(float dx, float dy, float dz, float inv_h, float& d2, float& ir,
                                          float& dd)
{
    d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    ir = rsqrtf(fmaxf(d2, 1e-30f));
    dd = fmaxf(fmaf(-(d2 * ir), inv_h, 1.0f), 0.0f);
}

#ifndef PK_PASS_BLOCK
#define PK_PASS_BLOCK 256
#endif
constexpr int kPassBlock = PK_PASS_BLOCK;  // threads per block of the Jacobi passes

// One quad of row entries (16 bytes, streaming: the rows are read once per
// pass and outgrow L2).
__device__ __forceinline__ int4 row_quad(const int4* p) { return __ldcs(p); }

// Entries of a solver row past the row capacity: the particle's spill
// segment (rows that long exist only where more particles than the capacity
// sit inside one radius).
struct Tail {
    const int* rpool;
    const int* ovf;
    __device__ __forceinline__ int entry(int s, int k) const { return __ldg(rpool + __ldg(ovf + s) + k); }
};

// Pass A: rho_i and lambda_i over N(i), one thread per particle walking its
// interleaved row.  Writes xl[s] = (x_i, lambda_i) so pass B gathers a
// neighbour's position and lambda in one 16-byte load.  sum |grad_j|^2 is taken
// as sum g_j^2 (|x_ij / r| = 1).
__global__ void __launch_bounds__(kPassBlock)
    k_pass_density(const float4* __restrict__ xs, const int* __restrict__ rows,
                   const int2* __restrict__ rcnt, int row_cap, int n, PassK k_,
                   float4* __restrict__ xl, float* __restrict__ rho_out, Tail tl)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 xi = xs[s];
    const int na_all = rcnt[s].x, na = min(na_all, row_cap);
    const int4* rq = reinterpret_cast<const int4*>(rows + row_slot(s, 0, row_cap));
    float rho = 0.f, sg = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    auto pair = [&](int v) {
        const float4 xj = __ldg(xs + (v & kRowIndexMask));
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        float d2, ir, dd;
        pair_geom(dx, dy, dz, k_.inv_h, d2, ir, dd);
        const float dd2 = dd * dd;
        rho = fmaf(k_.cwm, dd2 * dd, rho);
        const float g = d2 > kEps2 ? k_.cg * dd2 : 0.0f;
        const float gi = g * ir;
        gx = fmaf(gi, dx, gx);
        gy = fmaf(gi, dy, gy);
        gz = fmaf(gi, dz, gz);
        sg = fmaf(g, g, sg);
    };
    const int nq = (na + 3) >> 2;
    int4 nxt = nq > 0 ? row_quad(rq) : make_int4(0, 0, 0, 0);
    for (int q = 0; q < nq; ++q) {
        const int4 cur = nxt;
        if (q + 1 < nq) nxt = row_quad(rq + 32LL * (q + 1));  // next quad in flight
        const int ent[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (4 * q + k >= na) break;
            pair(ent[k]);
        }
    }
    for (int e = na; e < na_all; ++e) pair(tl.entry(s, e - na));
    float l = sg + (gx * gx + gy * gy + gz * gz);
    l = -(rho - 1000.0f) / (l + 0.1f);  // rest density hard-coded (DensityPBD.cu:87)
    xl[s] = make_float4(xi.x, xi.y, xi.z, l > 0.0f ? 0.0f : l);
    if (rho_out != nullptr) rho_out[s] = rho;
}

// Pass B: x_i' = x_i + sum over U(i) of m_ij * 10 (x_i - x_j)(lambda_i +
// lambda_j) grad(r) / r (DensityPBD.cu:158), m_ij = popcount of the two flag
// bits; one thread per particle.
__global__ void __launch_bounds__(kPassBlock)
    k_pass_disp(const float4* __restrict__ xl, const int* __restrict__ rows, const int2* __restrict__ rcnt,
                int row_cap, int n, PassK k_, float4* __restrict__ xs_out, Tail tl)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 xi = xl[s];
    const int nu_all = rcnt[s].y, nu = min(nu_all, row_cap);
    const int4* rq = reinterpret_cast<const int4*>(rows + row_slot(s, 0, row_cap));
    float ax = 0.f, ay = 0.f, az = 0.f;
    auto pair = [&](int v) {
        const float mult = (float)__popc((unsigned)v >> 30);
        const float4 xj = __ldg(xl + (v & kRowIndexMask));
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        float d2, ir, dd;
        pair_geom(dx, dy, dz, k_.inv_h, d2, ir, dd);
        const float c = d2 > kEps2 ? mult * (xi.w + xj.w) * (k_.c10g * (dd * dd)) * ir : 0.0f;
        ax = fmaf(c, dx, ax);
        ay = fmaf(c, dy, ay);
        az = fmaf(c, dz, az);
    };
    const int nq = (nu + 3) >> 2;
    int4 nxt = nq > 0 ? row_quad(rq) : make_int4(0, 0, 0, 0);
    for (int q = 0; q < nq; ++q) {
        const int4 cur = nxt;
        if (q + 1 < nq) nxt = row_quad(rq + 32LL * (q + 1));  // next quad in flight
        const int ent[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (4 * q + k >= nu) break;
            pair(ent[k]);
        }
    }
    for (int e = nu; e < nu_all; ++e) pair(tl.entry(s, e - nu));
    xs_out[s] = make_float4(xi.x + ax, xi.y + ay, xi.z + az, 0.f);
}

// ---- FP32x2 variants of the passes (sm_100 packed FFMA2/FADD2/FMUL2): two
// row entries per instruction.  Each lane runs its full quads as two entry
// pairs, then its last partial quad one entry at a time.  The sums run as two
// interleaved partial sums (even and odd entries of each pair), so the order
// of additions differs from the one-entry kernels; the arithmetic of each
// pair term is identical.  d is taken as x_j - x_i (the exact negation of
// x_i - x_j), so the accumulated gradients and displacements carry the
// opposite sign and are negated at the end.

#ifndef PK_PASS_F32X2
#define PK_PASS_F32X2 1
#endif
// Row quads each thread keeps in flight ahead of the one it works on.
#ifndef PK_PASS_PF
#define PK_PASS_PF 2
#endif
constexpr int kPassPrefetch = PK_PASS_PF;

#ifndef PK_PASS_WARPS
#define PK_PASS_WARPS 0  // resident warps per SM asked of the register allocator (0: none)
#endif
template <int BLOCK>
constexpr int pass_min_blocks()
{
    return PK_PASS_WARPS > 0 && PK_PASS_WARPS / (BLOCK / 32) > 0 ? PK_PASS_WARPS / (BLOCK / 32) : 1;
}

struct Geom2 {
    float2 dx, dy, dz, d2, ir, dd;
};

__device__ __forceinline__ void pair_geom2(const float4& a, const float4& b, const float4& xi, float inv_h, Geom2& g)
{
    g.dx = make_float2(a.x - xi.x, b.x - xi.x);
    g.dy = make_float2(a.y - xi.y, b.y - xi.y);
    g.dz = make_float2(a.z - xi.z, b.z - xi.z);
    g.d2 = __ffma2_rn(g.dz, g.dz, __ffma2_rn(g.dy, g.dy, __fmul2_rn(g.dx, g.dx)));
    g.ir = make_float2(rsqrtf(fmaxf(g.d2.x, 1e-30f)), rsqrtf(fmaxf(g.d2.y, 1e-30f)));
    const float2 t = __ffma2_rn(__fmul2_rn(g.d2, g.ir), make_float2(-inv_h, -inv_h), make_float2(1.0f, 1.0f));
    g.dd = make_float2(fmaxf(t.x, 0.0f), fmaxf(t.y, 0.0f));
}

struct DensAcc {
    float2 rho, sg, gx, gy, gz;
};

__device__ __forceinline__ void dens_pair(const float4& a, const float4& b, const float4& xi, const PassK& k_,
                                          DensAcc& s)
{
    Geom2 g;
    pair_geom2(a, b, xi, k_.inv_h, g);
    const float2 dd2 = __fmul2_rn(g.dd, g.dd);
    s.rho = __ffma2_rn(make_float2(k_.cwm, k_.cwm), __fmul2_rn(dd2, g.dd), s.rho);
    const float2 gg = __fmul2_rn(make_float2(k_.cg, k_.cg), dd2);
    const float2 w = make_float2(g.d2.x > kEps2 ? gg.x : 0.0f, g.d2.y > kEps2 ? gg.y : 0.0f);
    const float2 gi = __fmul2_rn(w, g.ir);
    s.gx = __ffma2_rn(gi, g.dx, s.gx);
    s.gy = __ffma2_rn(gi, g.dy, s.gy);
    s.gz = __ffma2_rn(gi, g.dz, s.gz);
    s.sg = __ffma2_rn(w, w, s.sg);
}

// One entry into the .x partial sums (the tail of a row).
__device__ __forceinline__ void dens_one(const float4& a, const float4& xi, const PassK& k_, DensAcc& s)
{
    const float dx = a.x - xi.x, dy = a.y - xi.y, dz = a.z - xi.z;
    float d2, ir, dd;
    pair_geom(dx, dy, dz, k_.inv_h, d2, ir, dd);
    const float dd2 = dd * dd;
    s.rho.x = fmaf(k_.cwm, dd2 * dd, s.rho.x);
    const float w = d2 > kEps2 ? k_.cg * dd2 : 0.0f;
    const float gi = w * ir;
    s.gx.x = fmaf(gi, dx, s.gx.x);
    s.gy.x = fmaf(gi, dy, s.gy.x);
    s.gz.x = fmaf(gi, dz, s.gz.x);
    s.sg.x = fmaf(w, w, s.sg.x);
}

__device__ __forceinline__ void density2_particle(int s, const float4* __restrict__ xs,
                                                  const int* __restrict__ rows, const int2* __restrict__ rcnt,
                                                  int row_cap, const PassK& k_, float4* __restrict__ xl,
                                                  float* __restrict__ rho_out, const Tail& tl)
{
    const float4 xi = xs[s];
    const int na_all = rcnt[s].x, na = min(na_all, row_cap);
    const int4* rq = reinterpret_cast<const int4*>(rows + row_slot(s, 0, row_cap));
    DensAcc a{};
    const int nfull = na >> 2, nq = (na + 3) >> 2;
    int4 ring[kPassPrefetch];  // ring[k] = quad q + k of the row
#pragma unroll
    for (int k = 0; k < kPassPrefetch; ++k) ring[k] = k < nq ? row_quad(rq + 32LL * k) : make_int4(0, 0, 0, 0);
    for (int q = 0; q < nfull; ++q) {
        const int4 cur = ring[0];
#pragma unroll
        for (int k = 0; k + 1 < kPassPrefetch; ++k) ring[k] = ring[k + 1];
        if (q + kPassPrefetch < nq) ring[kPassPrefetch - 1] = row_quad(rq + 32LL * (q + kPassPrefetch));
        const float4 x0 = __ldg(xs + (cur.x & kRowIndexMask)), x1 = __ldg(xs + (cur.y & kRowIndexMask));
        const float4 x2 = __ldg(xs + (cur.z & kRowIndexMask)), x3 = __ldg(xs + (cur.w & kRowIndexMask));
        dens_pair(x0, x1, xi, k_, a);
        dens_pair(x2, x3, xi, k_, a);
    }
    const int rest = na - 4 * nfull;
    if (rest > 0) {
        const int ent[3] = {ring[0].x, ring[0].y, ring[0].z};
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < rest) dens_one(__ldg(xs + (ent[k] & kRowIndexMask)), xi, k_, a);
    }
    for (int e = na; e < na_all; ++e) dens_one(__ldg(xs + (tl.entry(s, e - na) & kRowIndexMask)), xi, k_, a);
    const float rho = a.rho.x + a.rho.y, sg = a.sg.x + a.sg.y;
    const float gx = a.gx.x + a.gx.y, gy = a.gy.x + a.gy.y, gz = a.gz.x + a.gz.y;
    float l = sg + (gx * gx + gy * gy + gz * gz);
    l = -(rho - 1000.0f) / (l + 0.1f);  // rest density hard-coded (DensityPBD.cu:87)
    xl[s] = make_float4(xi.x, xi.y, xi.z, l > 0.0f ? 0.0f : l);
    if (rho_out != nullptr) rho_out[s] = rho;
}

// Tiles of the persistent passes: each scene's sorted range (and the range of
// the particles outside every grid) cut into tiles of one block's threads, so
// no tile holds two scenes.  Null tiles: one scene, tile t = [t B, (t+1) B).
struct SceneTiles {
    const int2* tile;
    const int* count;  // device: number of tiles
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, pass_min_blocks<BLOCK>())
    k_pass_density2(const float4* __restrict__ xs, const int* __restrict__ rows,
                    const int2* __restrict__ rcnt, int row_cap, int n, PassK k_,
                    float4* __restrict__ xl, float* __restrict__ rho_out, Tail tl)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) density2_particle(s, xs, rows, rcnt, row_cap, k_, xl, rho_out, tl);
}

// Persistent form: a grid of resident blocks walks the scene tiles.
// (32 resident warps per SM asked of the register allocator: the tile loop
// would otherwise take the kernel past 64 registers and a quarter of them)
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
    k_pass_density2_t(const float4* __restrict__ xs, const int* __restrict__ rows,
                      const int2* __restrict__ rcnt, int row_cap, int n, PassK k_,
                      float4* __restrict__ xl, float* __restrict__ rho_out, Tail tl, SceneTiles T)
{
    const int nt = T.tile ? *T.count : (n + BLOCK - 1) / BLOCK;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 r = T.tile ? T.tile[t] : make_int2(t * BLOCK, min((t + 1) * BLOCK, n));
        const int s = r.x + (int)threadIdx.x;
        if (s < r.y) density2_particle(s, xs, rows, rcnt, row_cap, k_, xl, rho_out, tl);
    }
}

struct DispAcc {
    float2 ax, ay, az;
};

__device__ __forceinline__ void disp_pair(const float4& a, const float4& b, int va, int vb, const float4& xi,
                                          const PassK& k_, DispAcc& s)
{
    Geom2 g;
    pair_geom2(a, b, xi, k_.inv_h, g);
    const float2 mult = make_float2((float)__popc((unsigned)va >> 30), (float)__popc((unsigned)vb >> 30));
    const float2 lw = make_float2(xi.w + a.w, xi.w + b.w);
    const float2 c = __fmul2_rn(__fmul2_rn(__fmul2_rn(mult, lw),
                                           __fmul2_rn(make_float2(k_.c10g, k_.c10g), __fmul2_rn(g.dd, g.dd))),
                                g.ir);
    const float2 cc = make_float2(g.d2.x > kEps2 ? c.x : 0.0f, g.d2.y > kEps2 ? c.y : 0.0f);
    s.ax = __ffma2_rn(cc, g.dx, s.ax);
    s.ay = __ffma2_rn(cc, g.dy, s.ay);
    s.az = __ffma2_rn(cc, g.dz, s.az);
}

__device__ __forceinline__ void disp_one(const float4& a, int v, const float4& xi, const PassK& k_, DispAcc& s)
{
    const float mult = (float)__popc((unsigned)v >> 30);
    const float dx = a.x - xi.x, dy = a.y - xi.y, dz = a.z - xi.z;
    float d2, ir, dd;
    pair_geom(dx, dy, dz, k_.inv_h, d2, ir, dd);
    const float c = d2 > kEps2 ? mult * (xi.w + a.w) * (k_.c10g * (dd * dd)) * ir : 0.0f;
    s.ax.x = fmaf(c, dx, s.ax.x);
    s.ay.x = fmaf(c, dy, s.ay.x);
    s.az.x = fmaf(c, dz, s.az.x);
}

__device__ __forceinline__ void disp2_particle(int s, const float4* __restrict__ xl, const int* __restrict__ rows,
                                               const int2* __restrict__ rcnt, int row_cap, const PassK& k_,
                                               float4* __restrict__ xs_out, const Tail& tl)
{
    const float4 xi = xl[s];
    const int nu_all = rcnt[s].y, nu = min(nu_all, row_cap);
    const int4* rq = reinterpret_cast<const int4*>(rows + row_slot(s, 0, row_cap));
    DispAcc a{};
    const int nfull = nu >> 2, nq = (nu + 3) >> 2;
    int4 ring[kPassPrefetch];  // ring[k] = quad q + k of the row
#pragma unroll
    for (int k = 0; k < kPassPrefetch; ++k) ring[k] = k < nq ? row_quad(rq + 32LL * k) : make_int4(0, 0, 0, 0);
    for (int q = 0; q < nfull; ++q) {
        const int4 cur = ring[0];
#pragma unroll
        for (int k = 0; k + 1 < kPassPrefetch; ++k) ring[k] = ring[k + 1];
        if (q + kPassPrefetch < nq) ring[kPassPrefetch - 1] = row_quad(rq + 32LL * (q + kPassPrefetch));
        const float4 x0 = __ldg(xl + (cur.x & kRowIndexMask)), x1 = __ldg(xl + (cur.y & kRowIndexMask));
        const float4 x2 = __ldg(xl + (cur.z & kRowIndexMask)), x3 = __ldg(xl + (cur.w & kRowIndexMask));
        disp_pair(x0, x1, cur.x, cur.y, xi, k_, a);
        disp_pair(x2, x3, cur.z, cur.w, xi, k_, a);
    }
    const int rest = nu - 4 * nfull;
    if (rest > 0) {
        const int ent[3] = {ring[0].x, ring[0].y, ring[0].z};
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < rest) disp_one(__ldg(xl + (ent[k] & kRowIndexMask)), ent[k], xi, k_, a);
    }
    for (int e = nu; e < nu_all; ++e) {
        const int v = tl.entry(s, e - nu);
        disp_one(__ldg(xl + (v & kRowIndexMask)), v, xi, k_, a);
    }
    // the sums hold -(displacement): d was x_j - x_i
    xs_out[s] = make_float4(xi.x - (a.ax.x + a.ax.y), xi.y - (a.ay.x + a.ay.y), xi.z - (a.az.x + a.az.y), 0.f);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, pass_min_blocks<BLOCK>())
    k_pass_disp2(const float4* __restrict__ xl, const int* __restrict__ rows, const int2* __restrict__ rcnt,
                 int row_cap, int n, PassK k_, float4* __restrict__ xs_out, Tail tl)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) disp2_particle(s, xl, rows, rcnt, row_cap, k_, xs_out, tl);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
    k_pass_disp2_t(const float4* __restrict__ xl, const int* __restrict__ rows, const int2* __restrict__ rcnt,
                   int row_cap, int n, PassK k_, float4* __restrict__ xs_out, Tail tl, SceneTiles T)
{
    const int nt = T.tile ? *T.count : (n + BLOCK - 1) / BLOCK;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 r = T.tile ? T.tile[t] : make_int2(t * BLOCK, min((t + 1) * BLOCK, n));
        const int s = r.x + (int)threadIdx.x;
        if (s < r.y) disp2_particle(s, xl, rows, rcnt, row_cap, k_, xs_out, tl);
    }
}

// Scene tiles from the cell table: scene s holds the sorted range
// [start[s K], start[(s+1) K]) (K keys per scene), the particles outside
// every grid [start[nkeys], n).  One thread per scene.
__global__ void __launch_bounds__(256) k_tile_count(const int* __restrict__ start, long long scene_keys,
                                                    int nscenes, long long nkeys, int tile, int* __restrict__ cnt)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > nscenes) return;
    const int b = q < nscenes ? start[(long long)q * scene_keys] : start[nkeys];
    const int e = q < nscenes ? start[(long long)(q + 1) * scene_keys] : start[nkeys + 1];
    cnt[q] = (e - b + tile - 1) / tile;
}

__global__ void __launch_bounds__(256) k_tile_fill(const int* __restrict__ start, long long scene_keys,
                                                   int nscenes, long long nkeys, int tile,
                                                   const int* __restrict__ off, int2* __restrict__ tiles)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > nscenes) return;
    const int b = q < nscenes ? start[(long long)q * scene_keys] : start[nkeys];
    const int e = q < nscenes ? start[(long long)(q + 1) * scene_keys] : start[nkeys + 1];
    int o = off[q];
    for (int a = b; a < e; a += tile) tiles[o++] = make_int2(a, min(a + tile, e));
}

// Sorted -> caller order: x, v += (x - x_old)/dt (DP_UpdateVelocity,
// DensityPBD.cu:367-378), outDensity.  One thread per caller particle i
// (s = inv[i]): the 16-byte sorted values are gathered, the caller's AoS
// arrays written contiguously.
__global__ void __launch_bounds__(256)
    k_finish(const float4* __restrict__ xf, const float4* __restrict__ x0, const float4* __restrict__ vs,
             const float* __restrict__ rho_s, const int* __restrict__ inv, int n, float dt,
             float* __restrict__ x, float* __restrict__ v, float* __restrict__ rho_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = inv[i];
    float4 p = xf[s], q = x0[s], u = vs[s];
    x[3 * i] = p.x;
    x[3 * i + 1] = p.y;
    x[3 * i + 2] = p.z;
    v[3 * i] = u.x + (p.x - q.x) / dt;
    v[3 * i + 1] = u.y + (p.y - q.y) / dt;
    v[3 * i + 2] = u.z + (p.z - q.z) / dt;
    if (rho_out != nullptr) rho_out[i] = rho_s[s];
}

// ---- ImplicitViscosity (ImplicitViscosity.cu:8-128)

// VB_VisWeight: 45/(13 pi h^3) (1 - r/h) for r <= h.
struct ViscK {
    float inv_h, cw, b;  // b = dt * viscosity / h
};

// DP_UpdateVelocity in sorted space: v = v_integrated + (x - x_old)/dt, kept
// as the viscosity's v_old and first iterate.
__global__ void __launch_bounds__(256)
    k_vel_sorted(const float4* __restrict__ xf, const float4* __restrict__ x0, float4* __restrict__ vs,
                 float4* __restrict__ vcur, int n, float dt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 p = xf[s], q = x0[s], u = vs[s];
    const float4 v = make_float4(u.x + (p.x - q.x) / dt, u.y + (p.y - q.y) / dt, u.z + (p.z - q.z) / dt, 0.f);
    vs[s] = v;
    vcur[s] = v;
}

// One K_ApplyViscosity sweep over N(i) (the rows' first |N(i)| entries):
// v_i = v_old,i/(1+b) + (sum w v_j / sum w) b/(1+b); b = 0 and sum w = 1 when
// sum w < EPSILON.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
    k_pass_visc(const float4* __restrict__ xs, const float4* __restrict__ vin, const float4* __restrict__ vold,
                const int* __restrict__ rows, const int2* __restrict__ rcnt, int row_cap, int n, ViscK k_,
                float4* __restrict__ vout, Tail tl)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 xi = xs[s];
    const int na_all = rcnt[s].x, na = min(na_all, row_cap);
    const int4* rq = reinterpret_cast<const int4*>(rows + row_slot(s, 0, row_cap));
    float tw = 0.f, dx_ = 0.f, dy_ = 0.f, dz_ = 0.f;
    auto pair = [&](int v) {
        const int j = v & kRowIndexMask;
        const float4 xj = __ldg(xs + j);
        const float4 vj = __ldg(vin + j);
        float d2, ir, dd;
        pair_geom(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z, k_.inv_h, d2, ir, dd);
        const float w = d2 > kEps2 ? k_.cw * dd : 0.0f;
        tw += w;
        dx_ = fmaf(w, vj.x, dx_);
        dy_ = fmaf(w, vj.y, dy_);
        dz_ = fmaf(w, vj.z, dz_);
    };
    const int nq = (na + 3) >> 2;
    int4 ring[kPassPrefetch];  // ring[k] = quad q + k of the row
#pragma unroll
    for (int k = 0; k < kPassPrefetch; ++k) ring[k] = k < nq ? row_quad(rq + 32LL * k) : make_int4(0, 0, 0, 0);
    for (int q = 0; q < nq; ++q) {
        const int4 cur = ring[0];
#pragma unroll
        for (int k = 0; k + 1 < kPassPrefetch; ++k) ring[k] = ring[k + 1];
        if (q + kPassPrefetch < nq) ring[kPassPrefetch - 1] = row_quad(rq + 32LL * (q + kPassPrefetch));
        const int ent[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (4 * q + k >= na) break;
            pair(ent[k]);
        }
    }
    for (int e = na; e < na_all; ++e) pair(tl.entry(s, e - na));
    const float b = tw < kEpsilon ? 0.0f : k_.b;
    const float t = tw < kEpsilon ? 1.0f : tw;
    const float4 vo = vold[s];
    vout[s] = make_float4(vo.x / (1.0f + b) + dx_ / t * b / (1.0f + b), vo.y / (1.0f + b) + dy_ / t * b / (1.0f + b),
                          vo.z / (1.0f + b) + dz_ / t * b / (1.0f + b), 0.f);
}

// Sorted -> caller order with the velocity given: x, v, outDensity (one
// thread per caller particle, as k_finish).
__global__ void __launch_bounds__(256)
    k_finish_v(const float4* __restrict__ xf, const float4* __restrict__ vf, const float* __restrict__ rho_s,
               const int* __restrict__ inv, int n, float* __restrict__ x, float* __restrict__ v,
               float* __restrict__ rho_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = inv[i];
    const float4 p = xf[s], u = vf[s];
    x[3 * i] = p.x;
    x[3 * i + 1] = p.y;
    x[3 * i + 2] = p.z;
    v[3 * i] = u.x;
    v[3 * i + 1] = u.y;
    v[3 * i + 2] = u.z;
    if (rho_out != nullptr) rho_out[i] = rho_s[s];
}

ViscK visc_k(float vis, float h, float dt)
{
    return ViscK{1.0f / h, 45.0f / (13.0f * (float)M_PI * h * h * h), dt * vis / h};
}

// Caller order -> sorted: the solver's starting state.
__global__ void __launch_bounds__(256)
    k_gather_state(const float* __restrict__ x, const float* __restrict__ v, const int* __restrict__ perm,
                   int n, float4* __restrict__ xs0, float4* __restrict__ vs)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int i = perm[s];
    xs0[s] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.f);
    vs[s] = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.f);
}

// The Jacobi passes at the block size the context's autotuner chose (128,
// 256 or 512 threads; one thread per particle, so the results do not depend
// on it).
template <template <int> class Launch, class... Args>
static void by_block(int block, Args&&... args)
{
    if (block == 128)
        Launch<128>::run(args...);
    else if (block == 512)
        Launch<512>::run(args...);
    else
        Launch<256>::run(args...);
}
template <int B>
struct LaunchDensity {
    static void run(unsigned nb, cudaStream_t st, const float4* cur, const int* rows, const int2* rcnt, int row_cap,
                    int n, PassK pk, float4* xl, float* rho, Tail tl)
    {
        k_pass_density2<B><<<nb, B, 0, st>>>(cur, rows, rcnt, row_cap, n, pk, xl, rho, tl);
    }
};
template <int B>
struct LaunchDisp {
    static void run(unsigned nb, cudaStream_t st, const float4* xl, const int* rows, const int2* rcnt, int row_cap,
                    int n, PassK pk, float4* out, Tail tl)
    {
        k_pass_disp2<B><<<nb, B, 0, st>>>(xl, rows, rcnt, row_cap, n, pk, out, tl);
    }
};
// Resident blocks per SM of a persistent pass kernel (one query per shape).
template <class K>
static int resident_blocks(K kernel, int block)
{
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
    return std::max(1, per_sm) * std::max(1, sms);
}
template <int B>
struct LaunchDensityT {
    static void run(unsigned, cudaStream_t st, const float4* cur, const int* rows, const int2* rcnt, int row_cap,
                    int n, PassK pk, float4* xl, float* rho, Tail tl, SceneTiles T)
    {
        static const int grid = resident_blocks(k_pass_density2_t<B>, B);
        k_pass_density2_t<B><<<grid, B, 0, st>>>(cur, rows, rcnt, row_cap, n, pk, xl, rho, tl, T);
    }
};
template <int B>
struct LaunchDispT {
    static void run(unsigned, cudaStream_t st, const float4* xl, const int* rows, const int2* rcnt, int row_cap,
                    int n, PassK pk, float4* out, Tail tl, SceneTiles T)
    {
        static const int grid = resident_blocks(k_pass_disp2_t<B>, B);
        k_pass_disp2_t<B><<<grid, B, 0, st>>>(xl, rows, rcnt, row_cap, n, pk, out, tl, T);
    }
};
template <int B>
struct LaunchVisc {
    static void run(unsigned nb, cudaStream_t st, const float4* xs, const float4* vin, const float4* vold,
                    const int* rows, const int2* rcnt, int row_cap, int n, ViscK vk, float4* vout, Tail tl)
    {
        k_pass_visc<B><<<nb, B, 0, st>>>(xs, vin, vold, rows, rcnt, row_cap, n, vk, vout, tl);
    }
};

int pbd_fast_solve(pk_ctx* c, int n, const Spiky& k, float mass, int iterations, float dt,
                   float* x, float* v, float* rho_out, cudaStream_t st, float viscosity, int vis_iterations)
{
    if (n <= 0) return 0;
    const int pb = c->tune.pass_block;
    const unsigned nb1 = (unsigned)((n + 255) / 256), nbp = (unsigned)((n + pb - 1) / pb);
    if (c->tune.on) cudaEventRecord(c->tune.ev[2], st);
    int launches = 0;
    const float4* cur = c->xs0;
    const PassK pk = pass_k(k, mass);
    const Tail tl{c->rpool, c->ovf};
    // resident-grid passes (an autotuner shape): scene tiles of batched frames
    // from the cell table
    const bool persist = PK_PASS_F32X2 && c->tune.persist;
    SceneTiles T{nullptr, nullptr};
    if (persist && c->grid.nscenes > 1) {
        const int ns = c->grid.nscenes;
        const unsigned nb = (unsigned)((ns + 1 + 255) / 256);
        k_tile_count<<<nb, 256, 0, st>>>(c->cell_start, c->grid.scene_keys, ns, c->grid.nkeys, pb, c->tile_cnt);
        exclusive_scan(c->tile_cnt, ns + 1, c->tile_off, c->scan_part, st);
        k_tile_fill<<<nb, 256, 0, st>>>(c->cell_start, c->grid.scene_keys, ns, c->grid.nkeys, pb, c->tile_off,
                                        c->tiles);
        T = SceneTiles{c->tiles, c->tile_off + ns + 1};
        launches += 2 + scan_launches();
    }
    // pass B reads only xl, so it may overwrite the positions pass A read
    // (except xs0, which the velocity update needs)
    for (int it = 0; it < iterations; ++it) {
        const bool last = it == iterations - 1;
        prof_begin(c, PK_PROF_DENSITY, st);
        if (persist)
            by_block<LaunchDensityT>(pb, nbp, st, cur, c->rows, c->rcnt, c->row_cap, n, pk, c->xb,
                                     last ? c->rho : nullptr, tl, T);
        else if (PK_PASS_F32X2)
            by_block<LaunchDensity>(pb, nbp, st, cur, c->rows, c->rcnt, c->row_cap, n, pk, c->xb,
                                    last ? c->rho : nullptr, tl);
        else
            k_pass_density<<<(n + kPassBlock - 1) / kPassBlock, kPassBlock, 0, st>>>(
                cur, c->rows, c->rcnt, c->row_cap, n, pk, c->xb, last ? c->rho : nullptr, tl);
        prof_end(c, PK_PROF_DENSITY, st);
        prof_begin(c, PK_PROF_DISP, st);
        if (persist)
            by_block<LaunchDispT>(pb, nbp, st, c->xb, c->rows, c->rcnt, c->row_cap, n, pk, c->xa, tl, T);
        else if (PK_PASS_F32X2)
            by_block<LaunchDisp>(pb, nbp, st, c->xb, c->rows, c->rcnt, c->row_cap, n, pk, c->xa, tl);
        else
            k_pass_disp<<<(n + kPassBlock - 1) / kPassBlock, kPassBlock, 0, st>>>(c->xb, c->rows, c->rcnt,
                                                                                 c->row_cap, n, pk, c->xa, tl);
        prof_end(c, PK_PROF_DISP, st);
        cur = c->xa;
        launches += 2;
    }
    float* rho = (rho_out != nullptr && iterations > 0) ? rho_out : nullptr;
    prof_begin(c, PK_PROF_FINISH, st);
    if (viscosity > 0.f && vis_iterations > 0) {
        // ImplicitViscosity after the solve (PositionBasedFluidModel.cpp:98), on
        // the same rows; velocities ping-pong between vv and xb
        k_vel_sorted<<<nb1, 256, 0, st>>>(cur, c->xs0, c->vs, c->vv, n, dt);
        const ViscK vk = visc_k(viscosity, k.h, dt);
        float4* vin = c->vv;
        float4* vout = c->xb;
        for (int t = 0; t < vis_iterations; ++t) {
            by_block<LaunchVisc>(pb, nbp, st, cur, vin, c->vs, c->rows, c->rcnt, c->row_cap, n, vk, vout, tl);
            float4* tmp = vin;
            vin = vout;
            vout = tmp;
        }
        k_finish_v<<<nb1, 256, 0, st>>>(cur, vin, c->rho, c->inv, n, x, v, rho);
        launches += 2 + vis_iterations;
    } else {
        k_finish<<<nb1, 256, 0, st>>>(cur, c->xs0, c->vs, c->rho, c->inv, n, dt, x, v, rho);
        ++launches;
    }
    prof_end(c, PK_PROF_FINISH, st);
    if (c->tune.on) cudaEventRecord(c->tune.ev[3], st);
    return launches;
}

// pbd_fast_solve without viscosity, keeping every Jacobi iterate for a
// reverse pass: ys[0..n) holds y_0 (the integrated positions, as sorted by
// the frame's build), iteration t reads ys[t n ..) and writes ys[(t+1) n ..)
// with the same kernels and arithmetic, so the iterates are those of the
// fused frame bit for bit.  Then x, v in caller order as k_finish writes them.
int pbd_replay_solve(pk_ctx* c, int n, const Spiky& k, float mass, int iterations, float dt, float4* ys,
                     float* x, float* v, cudaStream_t st)
{
    if (n <= 0) return 0;
    const int pb = c->tune.pass_block;
    const unsigned nb1 = (unsigned)((n + 255) / 256), nbp = (unsigned)((n + pb - 1) / pb);
    const PassK pk = pass_k(k, mass);
    const Tail tl{c->rpool, c->ovf};  // unused: the rollout's rows fit their capacity
    for (int it = 0; it < iterations; ++it) {
        by_block<LaunchDensity>(pb, nbp, st, ys + (size_t)it * n, c->rows, c->rcnt, c->row_cap, n, pk, c->xb,
                                nullptr, tl);
        by_block<LaunchDisp>(pb, nbp, st, c->xb, c->rows, c->rcnt, c->row_cap, n, pk, ys + (size_t)(it + 1) * n,
                             tl);
    }
    k_finish<<<nb1, 256, 0, st>>>(ys + (size_t)iterations * n, ys, c->vs, c->rho, c->inv, n, dt, x, v, nullptr);
    return 2 * iterations + 1;
}

int gather_state(pk_ctx* c, const float* x, const float* v, int n, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_gather_state<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, v, c->perm, n, c->xs0, c->vs);
    return 1;
}

// ------------------------------------------------------------------------
// Generic path: any NeighborList<int> in caller order (a list that did not
// come from this context's pk_nq_build).  One thread per particle, the
// displacement scattered with atomics as in the reference.

__device__ __forceinline__ int nb_size(const int* index, int cap, long long total, int n, int i)
{
    // NeighborList::getNeighborSize (NeighborList.h:27-41)
    if (cap > 0) return index[i];
    if (i >= n - 1) return (int)(total - index[i]);
    return index[i + 1] - index[i];
}
__device__ __forceinline__ long long nb_at(const int* index, int cap, int i, int k)
{
    return cap > 0 ? (long long)cap * i + k : (long long)index[i] + k;
}

// A neighbour id of a caller's list outside [0, n) is skipped (never read or
// scattered to) and latched as kErrBadIndex where the caller gave a flag word.
__device__ __forceinline__ bool valid_id(int j, int n, int* err)
{
    if (j >= 0 && j < n) return true;
    if (err) atomicOr(err, kErrBadIndex);
    return false;
}

__global__ void __launch_bounds__(256)
    k_g_density(const float* __restrict__ x, int n, const int* __restrict__ index,
                const int* __restrict__ elements, int cap, long long total, Spiky k, float mass,
                float* __restrict__ rho, int* __restrict__ err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2], acc = 0.f;
    int m = nb_size(index, cap, total, n, i);
    for (int e = 0; e < m; ++e) {
        int j = elements[nb_at(index, cap, i, e)];
        if (!valid_id(j, n, err)) continue;
        float dx = xi - x[3 * j], dy = yi - x[3 * j + 1], dz = zi - x[3 * j + 2];
        float r = sqrtf(dx * dx + dy * dy + dz * dz), w, g;
        spiky_wg(k, r, w, g);
        acc += mass * w;
    }
    rho[i] = acc;
}

__global__ void __launch_bounds__(256)
    k_g_lambda(const float* __restrict__ x, const float* __restrict__ rho, int n,
               const int* __restrict__ index, const int* __restrict__ elements, int cap,
               long long total, Spiky k, float* __restrict__ lam, float* __restrict__ dpos,
               int* __restrict__ err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
    float sg = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    int m = nb_size(index, cap, total, n, i);
    for (int e = 0; e < m; ++e) {
        int j = elements[nb_at(index, cap, i, e)];
        if (!valid_id(j, n, err)) continue;
        float dx = xi - x[3 * j], dy = yi - x[3 * j + 1], dz = zi - x[3 * j + 2];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r > kEpsilon) {
            float w, g;
            spiky_wg(k, r, w, g);
            float ir = 1.0f / r;
            float g0 = g * dx * ir, g1 = g * dy * ir, g2 = g * dz * ir;
            gx += g0; gy += g1; gz += g2;
            sg += g0 * g0 + g1 * g1 + g2 * g2;
        }
    }
    float l = sg + (gx * gx + gy * gy + gz * gz);
    l = -(rho[i] - 1000.0f) / (l + 0.1f);
    lam[i] = l > 0.0f ? 0.0f : l;
    dpos[3 * i] = 0.f;  // m_deltaPos.reset() (DensityPBD.cu:315)
    dpos[3 * i + 1] = 0.f;
    dpos[3 * i + 2] = 0.f;
}

__global__ void __launch_bounds__(256)
    k_g_disp(const float* __restrict__ x, const float* __restrict__ lam, int n,
             const int* __restrict__ index, const int* __restrict__ elements, int cap,
             long long total, Spiky k, float* __restrict__ dpos, int* __restrict__ err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2], li = lam[i];
    int m = nb_size(index, cap, total, n, i);
    for (int e = 0; e < m; ++e) {
        int j = elements[nb_at(index, cap, i, e)];
        if (!valid_id(j, n, err)) continue;
        float dx = xi - x[3 * j], dy = yi - x[3 * j + 1], dz = zi - x[3 * j + 2];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r > kEpsilon) {
            float w, g;
            spiky_wg(k, r, w, g);
            float sl = li + lam[j], ir = 1.0f / r;
            float p0 = 10.0f * dx * sl * g * ir, p1 = 10.0f * dy * sl * g * ir,
                  p2 = 10.0f * dz * sl * g * ir;
            atomicAdd(dpos + 3 * i, p0);
            atomicAdd(dpos + 3 * j, -p0);
            atomicAdd(dpos + 3 * i + 1, p1);
            atomicAdd(dpos + 3 * j + 1, -p1);
            atomicAdd(dpos + 3 * i + 2, p2);
            atomicAdd(dpos + 3 * j + 2, -p2);
        }
    }
}

__global__ void __launch_bounds__(256) k_g_add(float* __restrict__ x, const float* __restrict__ d, long long m)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) x[t] += d[t];
}

__global__ void __launch_bounds__(256)
    k_g_velocity(float* __restrict__ v, const float* __restrict__ x, const float* __restrict__ xold,
                 long long m, float dt)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) v[t] += (x[t] - xold[t]) / dt;
}

int density_generic(const float* x, int n, const int* index, const int* elements, int cap,
                    long long total, const Spiky& k, float mass, float* rho, int* err, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_g_density<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, index, elements, cap, total, k, mass, rho,
                                                              err);
    return 1;
}

int pbd_generic_solve(pk_ctx* c, float* x, float* v, int n, const int* index, const int* elements,
                      int cap, long long total, const Spiky& k, float mass, int iterations,
                      float dt, float* rho_out, cudaStream_t st)
{
    return pbd_generic_solve_scratch(x, v, n, index, elements, cap, total, k, mass, iterations, dt, rho_out,
                                     c->g_rho, c->g_lam, c->g_dpos, c->g_xold, c->d_err, st);
}

// The generic solve on caller-supplied scratch (rho_s, lam: n floats; dpos,
// xold: 3n floats): a context's arrays, or the allocation-free entry point's
// fixed array. err (nullable) receives kErrBadIndex for list ids outside [0, n).
int pbd_generic_solve_scratch(float* x, float* v, int n, const int* index, const int* elements,
                              int cap, long long total, const Spiky& k, float mass, int iterations,
                              float dt, float* rho_out, float* rho_s, float* lam, float* dpos,
                              float* xold, int* err, cudaStream_t st)
{
    if (n <= 0) return 0;
    const unsigned nb = (unsigned)((n + 255) / 256);
    const long long m3 = 3LL * n;
    const unsigned nb3 = (unsigned)((m3 + 255) / 256);
    int launches = 0;
    cudaMemcpyAsync(xold, x, sizeof(float) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
    float* rho = rho_out != nullptr ? rho_out : rho_s;
    for (int it = 0; it < iterations; ++it) {
        k_g_density<<<nb, 256, 0, st>>>(x, n, index, elements, cap, total, k, mass, rho, err);
        k_g_lambda<<<nb, 256, 0, st>>>(x, rho, n, index, elements, cap, total, k, lam, dpos, err);
        k_g_disp<<<nb, 256, 0, st>>>(x, lam, n, index, elements, cap, total, k, dpos, err);
        k_g_add<<<nb3, 256, 0, st>>>(x, dpos, m3);
        launches += 4;
    }
    k_g_velocity<<<nb3, 256, 0, st>>>(v, x, xold, m3, dt);
    return launches + 1;
}

// ------------------------------------------------ integrator and boundary

__global__ void __launch_bounds__(256)
    k_integrate(float* __restrict__ x, float* __restrict__ v, const float* __restrict__ f, int n,
                float gx, float gy, float gz, float dt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float g[3] = {gx, gy, gz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float fa = f != nullptr ? f[3 * i + a] : 0.f;
        float va = v[3 * i + a] + dt * (fa + g[a]);  // K_UpdateVelocity (ParticleIntegrator.cu:69)
        v[3 * i + a] = va;
        if (x != nullptr) x[3 * i + a] += dt * va;  // K_UpdatePosition (ParticleIntegrator.cu:111)
    }
}

int integrate_aos(float* x, float* v, const float* f, int n, const float g[3], float dt, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_integrate<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, v, f, n, g[0], g[1], g[2], dt);
    return 1;
}

__global__ void __launch_bounds__(256) k_advect(float* __restrict__ x, const float* __restrict__ v,
                                                long long m, float dt)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) x[t] += dt * v[t];
}

int advect_aos(float* x, const float* v, int n, float dt, cudaStream_t st)
{
    if (n <= 0) return 0;
    long long m = 3LL * n;
    k_advect<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(x, v, m, dt);
    return 1;
}

int velocity_from_positions(float* v, const float* x, const float* xold, int n, float dt, cudaStream_t st)
{
    if (n <= 0) return 0;
    long long m = 3LL * n;
    k_g_velocity<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(v, x, xold, m, dt);
    return 1;
}

__global__ void __launch_bounds__(256)
    k_boundary(float* __restrict__ x, float* __restrict__ v, int n, SdfView s, float nfric,
               float tfric, float dt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 p = make_float3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    float3 u = make_float3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    if (sdf_constrain(s, i, p, u, nfric, tfric, dt)) {
        x[3 * i] = p.x; x[3 * i + 1] = p.y; x[3 * i + 2] = p.z;
        v[3 * i] = u.x; v[3 * i + 1] = u.y; v[3 * i + 2] = u.z;
    }
}

int boundary_aos(float* x, float* v, int n, const SdfView& s, float nfric, float tfric, float dt,
                 cudaStream_t st)
{
    if (n <= 0) return 0;
    k_boundary<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, v, n, s, nfric, tfric, dt);
    return 1;
}

__global__ void __launch_bounds__(256) k_jitter(float* __restrict__ out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandState st;
    curand_init((unsigned long long)i, 0ull, 0ull, &st);
    out[i] = curand_uniform(&st);
}

int boundary_jitter(float* out, int n, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_jitter<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n);
    return 1;
}

SdfView sdf_view(const pk_ctx* c)
{
    SdfView s{};
    s.data = c->sdf;
    float mh = 0.f;
    for (int a = 0; a < 3; ++a) {
        s.left[a] = c->sdf_left[a];
        s.inv_h[a] = (float)(1.0 / (double)c->sdf_h[a]);
        s.box_lo[a] = c->sdf_box_lo[a];
        s.box_hi[a] = c->sdf_box_hi[a];
        mh = fmaxf(mh, c->sdf_h[a]);
    }
    s.margin = 2.0f * mh + 1e-6f;
    s.nx = c->sdf_dims[0];
    s.ny = c->sdf_dims[1];
    s.nz = c->sdf_dims[2];
    s.inverted = c->sdf_inverted;
    return s;
}


// ImplicitViscosity on any NeighborList<int> in caller order (one thread per
// particle, as K_ApplyViscosity): vout from vin (the previous iterate) and vold.
__global__ void __launch_bounds__(256)
    k_g_visc(const float* __restrict__ x, const float* __restrict__ vin, const float* __restrict__ vold,
             float* __restrict__ vout, int n, const int* __restrict__ index, const int* __restrict__ elements,
             int cap, long long total, ViscK k_, int* __restrict__ err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float xi0 = x[3 * i], xi1 = x[3 * i + 1], xi2 = x[3 * i + 2];
    float tw = 0.f, d0 = 0.f, d1 = 0.f, d2v = 0.f;
    const int m = nb_size(index, cap, total, n, i);
    for (int e = 0; e < m; ++e) {
        const int j = elements[nb_at(index, cap, i, e)];
        if (!valid_id(j, n, err)) continue;
        float d2, ir, dd;
        pair_geom(xi0 - x[3 * j], xi1 - x[3 * j + 1], xi2 - x[3 * j + 2], k_.inv_h, d2, ir, dd);
        const float w = d2 > kEps2 ? k_.cw * dd : 0.0f;
        tw += w;
        d0 = fmaf(w, vin[3 * j], d0);
        d1 = fmaf(w, vin[3 * j + 1], d1);
        d2v = fmaf(w, vin[3 * j + 2], d2v);
    }
    const float b = tw < kEpsilon ? 0.0f : k_.b;
    const float t = tw < kEpsilon ? 1.0f : tw;
    vout[3 * i] = vold[3 * i] / (1.0f + b) + d0 / t * b / (1.0f + b);
    vout[3 * i + 1] = vold[3 * i + 1] / (1.0f + b) + d1 / t * b / (1.0f + b);
    vout[3 * i + 2] = vold[3 * i + 2] / (1.0f + b) + d2v / t * b / (1.0f + b);
}

int viscosity_generic(pk_ctx* c, const float* x, float* v, int n, const int* index, const int* elements, int cap,
                      long long total, float vis, float h, int iterations, float dt, cudaStream_t st)
{
    if (n <= 0 || iterations <= 0) return 0;
    const unsigned nb = (unsigned)((n + 255) / 256);
    const size_t bytes = sizeof(float) * 3 * (size_t)n;
    const ViscK vk = visc_k(vis, h, dt);
    // velOld and velBuf copies, then the sweep (ImplicitViscosity.cu:105-124)
    cudaMemcpyAsync(c->g_xold, v, bytes, cudaMemcpyDeviceToDevice, st);
    for (int t = 0; t < iterations; ++t) {
        cudaMemcpyAsync(c->g_dpos, v, bytes, cudaMemcpyDeviceToDevice, st);
        k_g_visc<<<nb, 256, 0, st>>>(x, c->g_dpos, c->g_xold, v, n, index, elements, cap, total, vk, c->d_err);
    }
    return iterations;
}

}  // namespace pk
