// pk_sort.cu -- counting sort of particles into blocked-Morton cells.
//
// Replaces GridHash::construct (GridHash.cu:297-323): the reference counts
// with atomics, reduces on the host, scans and scatters ids with atomics (the
// order inside a cell is whatever the atomics produce), and re-mallocs `ids`
// every build.  Here: one pass computes key + in-cell rank (optionally after
// the boundary projection), a device-wide scan gives cell starts (no host
// round trip), a scatter places ids, and a per-cell fix-up sorts each cell's
// ids ascending so the order is deterministic.  A final gather builds the
// sorted float4 arrays the list build and the solver read.
#include <algorithm>

#include "pk_boundary.cuh"
#include "pk_kernels.cuh"

namespace pk {

Grid make_grid(float h, const float lo[3], const float hi[3])
{
    // GridHash::setSpace (GridHash.cu:46-75), float arithmetic as on the host.
    Grid g;
    const int padding = 2;
    g.ds = h;
    int n[3];
    for (int a = 0; a < 3; ++a) {
        float pad = (float)padding * h;
        float nseg = (hi[a] - lo[a]) / h;
        g.lo[a] = lo[a] - pad;
        n[a] = (int)(ceilf(nseg) + 1.0f + (float)(2 * padding));
    }
    g.nx = n[0];
    g.ny = n[1];
    g.nz = n[2];
    g.bx = (g.nx + 3) / 4;
    g.by = (g.ny + 3) / 4;
    g.bz = (g.nz + 3) / 4;
    g.scene_keys = (long long)g.bx * g.by * g.bz * 64;
    g.nkeys = g.scene_keys;
    g.nscenes = 1;
    g.scene_off = nullptr;
    return g;
}

Spiky make_spiky(float h)
{
    Spiky k;
    k.h = h;
    k.inv_h = 1.0f / h;
    float hh = h * h;
    k.cw = 15.0f / ((float)M_PI * hh * h);
    k.cg = -45.0f / ((float)M_PI * hh * h);
    return k;
}

// key = blocked-Morton cell key, or nkeys for particles outside the grid
// (the reference leaves those out of the hash, GridHash.cu:85,194; they still
// query).  rank = arrival order inside the cell.
template <bool kBoundary>
__global__ void __launch_bounds__(256) k_keys(float* __restrict__ x, float* __restrict__ v, int n,
                                              Grid g, int* __restrict__ key,
                                              int* __restrict__ rank, int* __restrict__ cell_cnt,
                                              SdfView sdf, float nfric, float tfric, float dt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 p = make_float3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    const int scene = scene_of(g, i);
    if (kBoundary) {
        // the jitter is seeded by the particle's id within its own scene
        const int local = g.nscenes > 1 ? i - __ldg(g.scene_off + scene) : i;
        float3 u = make_float3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        if (sdf_constrain(sdf, local, p, u, nfric, tfric, dt)) {
            x[3 * i] = p.x; x[3 * i + 1] = p.y; x[3 * i + 2] = p.z;
            v[3 * i] = u.x; v[3 * i + 1] = u.y; v[3 * i + 2] = u.z;
        }
    }
    int3 c = cell3(g, p.x, p.y, p.z);
    int k = cell_key(g, c.x, c.y, c.z);
    k = k < 0 ? (int)g.nkeys : k + (int)(scene * g.scene_keys);
    key[i] = k;
    rank[i] = atomicAdd(&cell_cnt[k], 1);
}

// ---------------------------------------------------------------- scan
// Exclusive scan of in[0..m) into out[0..m], out[m] = total.  Three passes:
// tile sums, a one-block scan of the sums, tile scans with the carried offset.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* smem_warp, int& total)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) smem_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        int w = lane < nw ? smem_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += y;
        }
        if (lane < nw) smem_warp[lane] = wi - w;
        if (lane == nw - 1) smem_warp[32] = wi;
    }
    __syncthreads();
    int res = smem_warp[warp] + incl - v;
    total = smem_warp[32];
    __syncthreads();
    return res;
}

// A thread's kScanItems consecutive values: two 16-byte loads when the array
// is 16-byte aligned and the group lies inside it (every group but the last).
__device__ __forceinline__ void scan_load(const int* __restrict__ in, long long base, long long m, bool vec,
                                          int (&vals)[kScanItems])
{
    if (vec && base + kScanItems <= m) {
        const int4 u = __ldg(reinterpret_cast<const int4*>(in + base));
        const int4 w = __ldg(reinterpret_cast<const int4*>(in + base) + 1);
        vals[0] = u.x; vals[1] = u.y; vals[2] = u.z; vals[3] = u.w;
        vals[4] = w.x; vals[5] = w.y; vals[6] = w.z; vals[7] = w.w;
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) vals[k] = base + k < m ? in[base + k] : 0;
    }
}
static_assert(kScanItems == 8, "two 16-byte loads per thread");

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* __restrict__ in, long long m,
                                                              int* __restrict__ part, bool vec)
{
    __shared__ int sw[33];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int vals[kScanItems];
    scan_load(in, base, m, vec, vals);
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += vals[k];
    int tot;
    block_exclusive_scan(s, sw, tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_parts(int* __restrict__ part, int nparts)
{
    __shared__ int sw[33];
    int carry = 0;
    for (int base = 0; base < nparts; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < nparts ? part[i] : 0;
        int tot;
        int ex = block_exclusive_scan(v, sw, tot);
        if (i < nparts) part[i] = ex + carry;
        carry += tot;
    }
}

// kItems (the cell table's scan, m = cells + 1 with the last the bucket of
// particles outside the grid): also appends the list-build work items, one
// (begin, end) sorted range per occupied cell (a warp's with one atomic) and
// one per particle of the outside bucket (each queries its own, out-of-range
// cell).
template <bool kItems>
__global__ void __launch_bounds__(kScanThreads) k_scan_down(const int* __restrict__ in, long long m,
                                                            const int* __restrict__ part,
                                                            int* __restrict__ out, bool vec,
                                                            int2* __restrict__ items, int* __restrict__ nitems)
{
    __shared__ int sw[33];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int vals[kScanItems];
    scan_load(in, base, m, vec, vals);
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += vals[k];
    int tot;
    int ex = block_exclusive_scan(s, sw, tot) + part[blockIdx.x];
    int o[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        o[k] = ex;
        ex += vals[k];
    }
    if (vec && base + kScanItems <= m) {
        reinterpret_cast<int4*>(out + base)[0] = make_int4(o[0], o[1], o[2], o[3]);
        reinterpret_cast<int4*>(out + base)[1] = make_int4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (base + k < m) out[base + k] = o[k];
    }
    if (base < m && base + kScanItems >= m) out[m] = ex;  // the thread holding the last item
    if (kItems) {
        const int lane = threadIdx.x & 31;
        int occ = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) occ += (base + k < m - 1 && vals[k] > 0) ? 1 : 0;
        int incl = occ;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        int wbase = 0;
        if (lane == 31 && incl > 0) wbase = atomicAdd(nitems, incl);
        wbase = __shfl_sync(0xffffffffu, wbase, 31);
        int q = wbase + incl - occ;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (base + k < m - 1 && vals[k] > 0) items[q++] = make_int2(o[k], o[k] + vals[k]);
        if (base <= m - 1 && m - 1 < base + kScanItems) {  // the outside bucket
            const int k = (int)(m - 1 - base);
            int cnt = 0, beg = 0;
#pragma unroll
            for (int u = 0; u < kScanItems; ++u)
                if (u == k) {
                    cnt = vals[u];
                    beg = o[u];
                }
            if (cnt > 0) {
                const int b0 = atomicAdd(nitems, cnt);
                for (int u = 0; u < cnt; ++u) items[b0 + u] = make_int2(beg + u, beg + u + 1);
            }
        }
    }
}

int scan_launches() { return 3; }

void exclusive_scan(const int* in, long long m, int* out, int* part, cudaStream_t st)
{
    long long nparts = (m + kScanTile - 1) / kScanTile;
    if (nparts < 1) nparts = 1;
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
    k_scan_reduce<<<(unsigned)nparts, kScanThreads, 0, st>>>(in, m, part, vec);
    k_scan_parts<<<1, 1024, 0, st>>>(part, (int)nparts);
    k_scan_down<false><<<(unsigned)nparts, kScanThreads, 0, st>>>(in, m, part, out, vec, nullptr, nullptr);
}

// The cell table's scan (m = cells + 1), appending the list-build items to
// items / *nitems (zeroed by the caller).
static void scan_cells(const int* in, long long m, int* out, int* part, int2* items, int* nitems,
                       cudaStream_t st)
{
    long long nparts = (m + kScanTile - 1) / kScanTile;
    if (nparts < 1) nparts = 1;
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
    k_scan_reduce<<<(unsigned)nparts, kScanThreads, 0, st>>>(in, m, part, vec);
    k_scan_parts<<<1, 1024, 0, st>>>(part, (int)nparts);
    k_scan_down<true><<<(unsigned)nparts, kScanThreads, 0, st>>>(in, m, part, out, vec, items, nitems);
}

long long scan_parts_needed(long long m) { return (m + kScanTile - 1) / kScanTile + 1; }

// ------------------------------------------------------- scatter + fix-up

__global__ void __launch_bounds__(256) k_scatter(const int* __restrict__ key, const int* __restrict__ rank,
                                                 const int* __restrict__ start, int n,
                                                 int* __restrict__ perm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[start[key[i]] + rank[i]] = i;
}

// Ascending sort of the m <= N ids at p (N a power of two) in registers: a
// bitonic network over N values padded with INT_MAX, every index fixed at
// compile time, so no step waits on a memory access.
template <int N>
__device__ __forceinline__ void sort_ids(int* __restrict__ p, int m)
{
    int v[N];
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = k < m ? p[k] : 0x7fffffff;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const int l = k ^ stride;
                if (l > k) {
                    const int lo = min(v[k], v[l]), hi = max(v[k], v[l]);
                    const bool up = (k & size) == 0;
                    v[k] = up ? lo : hi;
                    v[l] = up ? hi : lo;
                }
            }
#pragma unroll
    for (int k = 0; k < N; ++k)
        if (k < m) p[k] = v[k];
}

// Insertion sort of the m ids at p (cells above 32 ids: dense clusters and
// the outside bucket).
__device__ __forceinline__ void sort_ids_insertion(int* __restrict__ p, int m)
{
    for (int u = 1; u < m; ++u) {
        int t = p[u];
        int w = u - 1;
        while (w >= 0 && p[w] > t) {
            p[w + 1] = p[w];
            --w;
        }
        p[w + 1] = t;
    }
}

// Sorts the ids of each occupied cell ascending, so the order inside a cell
// is deterministic (the scatter's order is the atomics' arrival order): one
// thread per work item (a register network for up to 32 ids, insertion sort
// above; per-particle items of the outside bucket hold one id), and the
// outside bucket itself by one thread.  Cells above 2048 ids (only the
// outside bucket is likely to be that large) keep their arrival order.
__global__ void __launch_bounds__(256) k_sort_cells(const int* __restrict__ start, long long ncells,
                                                    int* __restrict__ perm, const int2* __restrict__ items,
                                                    const int* __restrict__ nitems)
{
    const int ni = *nitems;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ni; q += gridDim.x * blockDim.x) {
        const int2 r = items[q];
        const int m = r.y - r.x;
        if (m < 2 || m > 2048) continue;
        int* p = perm + r.x;
        if (m <= 16)
            sort_ids<16>(p, m);
        else if (m <= 32)
            sort_ids<32>(p, m);
        else
            sort_ids_insertion(p, m);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int a = start[ncells - 1], m = start[ncells] - a;
        if (m >= 2 && m <= 2048) sort_ids_insertion(perm + a, m);
    }
}

// Sorted-order gather: xs_pre = positions the list is built on; when
// kIntegrate, also ParticleIntegrator::integrate (ParticleIntegrator.cu:59-70,
// 102-112) into xs0/vs: v += dt*(f + g), x += dt*v.
template <bool kIntegrate>
__global__ void __launch_bounds__(256) k_gather(const float* __restrict__ x, const float* __restrict__ v,
                                                const float* __restrict__ f,
                                                const int* __restrict__ perm, int n,
                                                float4* __restrict__ xs_pre, float4* __restrict__ xs0,
                                                float4* __restrict__ vs, int* __restrict__ inv,
                                                float gx, float gy, float gz, float dt)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int i = perm[s];
    float px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
    xs_pre[s] = make_float4(px, py, pz, 0.0f);
    inv[i] = s;
    if (kIntegrate) {
        float vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (f) { fx = f[3 * i]; fy = f[3 * i + 1]; fz = f[3 * i + 2]; }
        vx += dt * (fx + gx);
        vy += dt * (fy + gy);
        vz += dt * (fz + gz);
        xs0[s] = make_float4(px + dt * vx, py + dt * vy, pz + dt * vz, 0.0f);
        vs[s] = make_float4(vx, vy, vz, 0.0f);
    }
}

// ------------------------------------------------------------------ host

int sort_particles(pk_ctx* c, float* x, float* v, const float* f, int n, const Grid& g,
                   bool boundary, const SdfView* sdf, float nfric, float tfric, float dt,
                   bool integrate, const float grav[3], cudaStream_t st)
{
    int launches = 0;
    long long nk = g.nkeys + 1;  // + the "outside" bucket
    prof_begin(c, PK_PROF_SORT, st);
    cudaMemsetAsync(c->cell_cnt, 0, sizeof(int) * (size_t)nk, st);
    unsigned nb = (unsigned)((n + 255) / 256);
    SdfView sv{};
    if (sdf) sv = *sdf;
    if (n > 0) {
        if (boundary)
            k_keys<true><<<nb, 256, 0, st>>>(x, v, n, g, c->key, c->rank, c->cell_cnt, sv, nfric, tfric, dt);
        else
            k_keys<false><<<nb, 256, 0, st>>>(x, v, n, g, c->key, c->rank, c->cell_cnt, sv, nfric, tfric, dt);
        ++launches;
    }
    cudaMemsetAsync(c->nitems, 0, sizeof(int), st);
    scan_cells(c->cell_cnt, nk, c->cell_start, c->scan_part, c->items, c->nitems, st);
    launches += scan_launches();
    if (n > 0) {
        k_scatter<<<nb, 256, 0, st>>>(c->key, c->rank, c->cell_start, n, c->perm);
        k_sort_cells<<<std::min(nb, 2048u), 256, 0, st>>>(c->cell_start, nk, c->perm, c->items, c->nitems);
        if (integrate)
            k_gather<true><<<nb, 256, 0, st>>>(x, v, f, c->perm, n, c->xs_pre, c->xs0, c->vs, c->inv,
                                               grav[0], grav[1], grav[2], dt);
        else
            k_gather<false><<<nb, 256, 0, st>>>(x, v, f, c->perm, n, c->xs_pre, nullptr, nullptr,
                                                c->inv, 0.f, 0.f, 0.f, 0.f);
        launches += 3;
    }
    prof_end(c, PK_PROF_SORT, st);
    return launches;
}

}  // namespace pk
