// pk_nbr.cu -- neighbour rows over the cell-sorted particles.
//
// Reference: K_ComputeNeighborFixed (NeighborQuery.cu:514-581) keeps, per
// particle, the `cap` nearest hits with d < h by replacing the current
// farthest entry; K_CalNeighborSize/K_GetNeighborElements (:245-276,337-367)
// build the uncapped list.  A capped list is asymmetric (j in N(i) does not
// imply i in N(j)) and DensityPBD scatters each pair's displacement to both
// ends (DensityPBD.cu:161-173).  To solve that with gathers only, each solver
// row holds N(i) plus {j : i in N(j)} with two flag bits, so a pair's
// multiplicity in i's displacement is known without atomics.
//
//   k_build (one warp per occupied cell, passes of up to 8 particles, 4 or 16
//     when the context's autotuner measured that faster): every lane holds the
//     pass's particles in registers and takes one candidate of each 32-wide
//     chunk of the 27 neighbour ranges (a coalesced load), so a lane runs up to
//     8 independent pair tests per chunk; one ballot per particle
//     appends the chunk's hits (sorted index, d2) to its hit row in candidate
//     order.  The hit test compares the rounded squared distance with the
//     precomputed float T (sqrt_rn(d2) < h  <=>  d2 < T, sqrt_rn being
//     monotone), so no square root is taken.
//   k_select (capped lists, a warp per over-cap row): tau_i, the cap-th
//     smallest key (d2, sorted index) of the row.  Rows of at most 128 hits
//     are held in registers and tau is taken by rounds of warp maxima over
//     64-bit keys, pivoted on the particle's tau of the previous frame so only
//     |#keys below the pivot - cap| + 1 rounds run; longer rows narrow a
//     32-bin histogram of d2 until the bin holding the cap-th key fits a warp.
//     sqrt_rn is monotone, so the key order agrees with the reference's
//     distance order except among hits at exactly equal distance, which the
//     reference orders by arrival.
//   k_spill (particles with more hits than the row capacity): the same sweep
//     for one particle, keeping the hits past the capacity in the particle's
//     segment of the spill pool, so a row of any length is in candidate order.
//   k_emit (8 lanes per particle): re-reads the hit row, marks a = key <= tau_i
//     (j in N(i)) and b = key' <= tau_j (i in N(j)), compacts in place with
//     a-entries first, then b-only entries, and writes the public NeighborList
//     in caller ids (fixed: index = count; dynamic: CSR).
// Distances use the explicit roundings of exact_norm3's squared sum, so every
// d < h decision and every ordering is bit-identical for (i, j) and (j, i)
// and matches the CPU restatement.
#include <algorithm>
#include <cmath>

#include "pk_kernels.cuh"

namespace pk {

constexpr int kBuildWarps = 4;
constexpr int kBins = 32;                // histogram of d2 over [0, T)
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool key_le(float d2, int id, uint2 tau)
{
    const float td = __uint_as_float(tau.x);
    return d2 < td || (d2 == td && id <= (int)tau.y);
}

__device__ __forceinline__ bool key_lt(float da, int ta, float db, int tb)
{
    return da < db || (da == db && ta < tb);
}

// Rounded squared distance of exact_norm3 (before its square root).
__device__ __forceinline__ float exact_d2(float4 a, float4 b)
{
    const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
#if PK_NORM_VARIANT == 0
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
#elif PK_NORM_VARIANT == 2
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
#else
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
#endif
}

struct BuildArgs {
    const float4* xs;   // positions the list is built on (sorted)
    const int* start;   // cell starts
    const int2* items;  // (begin, end) sorted ranges sharing one cell
    const int* nitems;
    Grid g;
    int n, row_cap;
    float T;            // d2 threshold of d < h
    uint2* hits;        // hit rows: (sorted index, d2 bits), candidate order
    int* hcnt;          // hits per particle (sorted order), past the row capacity too
    int* count_c;       // hits per particle in caller order (dynamic public list), or null
    const int* perm;
    int* err;
    // spill pool (pool_cap 0: none, a row past the capacity is an error)
    long long pool_cap;
    unsigned long long* spill;  // [0] entries handed out, [1] particles listed
    int* ovf;
    int* ovf_list;
    uint2* hpool;
};

// Entries past the row capacity: a segment of round4(count - row_cap) entries
// of the spill pool, and the particle listed for k_spill.
__device__ __forceinline__ void claim_spill(const BuildArgs& A, int s, int count)
{
    if (A.pool_cap <= 0) {
        atomicOr(A.err, kErrRowOverflow);
        return;
    }
    const unsigned long long need = (unsigned long long)((count - A.row_cap + 3) & ~3);
    const unsigned long long off = atomicAdd(A.spill, need);
    if (off + need <= (unsigned long long)A.pool_cap) {
        A.ovf[s] = (int)off;
        A.ovf_list[atomicAdd(A.spill + 1, 1ull)] = s;
    } else {
        A.ovf[s] = -1;
        atomicOr(A.err, kErrHitOverflow);
    }
}

// Particles of one pass, held in registers by every lane: 8 by default, 4 or
// 16 when the context's autotuner measured that faster (the hit rows are the
// same).
constexpr int kPB = 16;

// Per-warp shared state of the sweep: the 27 neighbour ranges as (begin,
// packed offset) pairs.
struct SweepSmem {
    int rbeg[32], roff[33];
};
constexpr size_t kBuildSmem = sizeof(SweepSmem) * kBuildWarps;

// Candidate g of the packed 27 ranges (t = its sorted index); past the end a
// far-away sentinel that hits nothing.
__device__ __forceinline__ float4 fetch_cand(const float4* __restrict__ xs, const SweepSmem& S, int g,
                                             int total, int& t)
{
    if (g >= total) {
        t = 0;
        return make_float4(3.0e38f, 3.0e38f, 3.0e38f, 0.f);
    }
    int r = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
        if (r + step < 27 && S.roff[r + step] <= g) r += step;
    t = S.rbeg[r] + (g - S.roff[r]);
    return __ldg(xs + t);
}

// The 27 neighbour ranges of sorted particle s's cell into S (lane o < 27
// owns offset o; the reference's visiting order), packed in that order;
// returns the candidate count.  Called by a whole warp.
__device__ __forceinline__ int sweep_ranges(const BuildArgs& A, SweepSmem& S, int s, int lane)
{
    const float4 x0 = A.xs[s];
    const int3 c = cell3(A.g, x0.x, x0.y, x0.z);
    const int base = scene_key_base(A.g, __ldg(A.perm + s));
    int beg = 0, len = 0;
    if (lane < 27) {
        const int key = cell_key(A.g, c.x + kOffset27[lane][0], c.y + kOffset27[lane][1], c.z + kOffset27[lane][2]);
        if (key >= 0) {
            beg = __ldg(A.start + base + key);
            len = __ldg(A.start + base + key + 1) - beg;
        }
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    __syncwarp();
    S.rbeg[lane] = beg;
    S.roff[lane] = incl - len;
    const int total = __shfl_sync(kFull, incl, 31);
    if (lane == 31) S.roff[32] = total;
    __syncwarp();
    return total;
}

// One chunk of 32 candidates against the pass's particles.  kChecked guards
// the row bound (hits past it are counted, and written by k_spill).
template <bool kChecked, int KPB>
__device__ __forceinline__ void sweep_chunk(const BuildArgs& A, uint2* row0, const float4& cx, int t, int m,
                                            const float (&px)[KPB], const float (&py)[KPB],
                                            const float (&pz)[KPB], int (&cnt)[KPB], unsigned lt)
{
#pragma unroll
    for (int p = 0; p < KPB; ++p) {
        if (p >= m) break;  // warp-uniform
        const float d2 = exact_d2(make_float4(px[p], py[p], pz[p], 0.f), cx);
        const bool hit = d2 < A.T;
        const unsigned b = __ballot_sync(kFull, hit);
        const int pos = cnt[p] + __popc(b & lt);
        if (hit && (!kChecked || pos < A.row_cap))
            row0[p * A.row_cap + pos] = make_uint2((unsigned)t, __float_as_uint(d2));
        cnt[p] += __popc(b);
    }
}

// One pass of the sweep: kPB particles in registers against every candidate
// chunk.  A chunk adds at most 32 hits to a row, so with the pass's largest
// count at c the next (row_cap - c) / 32 chunks cannot overflow a row: they
// run as an unchecked loop, after which the bound is refreshed; chunks left
// when no row has 32 entries to spare run checked.  (Counts are
// warp-uniform.  Deciding checked or not inside one loop, per chunk, cost
// 14% more instructions.)
template <int KPB>
__device__ __forceinline__ void sweep(const BuildArgs& A, const SweepSmem& S, int total, int p0, int m,
                                      const float (&px)[KPB], const float (&py)[KPB], const float (&pz)[KPB],
                                      int (&cnt)[KPB], int lane, unsigned lt)
{
    uint2* const row0 = A.hits + (long long)p0 * A.row_cap;
    int c0 = 0;
    while (c0 < total) {
        int mx = 0;
#pragma unroll
        for (int p = 0; p < KPB; ++p) mx = max(mx, cnt[p]);
        const int run_end = min(total, c0 + ((A.row_cap - mx) >> 5) * 32);
        if (run_end <= c0) break;
        for (; c0 < run_end; c0 += 32) {
            int t;
            const float4 cx = fetch_cand(A.xs, S, c0 + lane, total, t);
            sweep_chunk<false, KPB>(A, row0, cx, t, m, px, py, pz, cnt, lt);
        }
    }
    for (; c0 < total; c0 += 32) {
        int t;
        const float4 cx = fetch_cand(A.xs, S, c0 + lane, total, t);
        sweep_chunk<true, KPB>(A, row0, cx, t, m, px, py, pz, cnt, lt);
    }
}

// Hit rows, one warp per occupied cell in passes of up to kPB particles.
// Every lane holds the pass's particles in registers and takes one candidate
// of each 32-wide chunk of the 27 neighbour ranges: up to kPB independent
// pair tests per lane and chunk, then one ballot per particle appends the
// chunk's hits to its row (in candidate order, so rows are deterministic).
// Resident blocks per SM asked of the register allocator, per pass size: 8
// blocks (61 registers) for 8-particle passes measured 2% faster at 2M than
// the unconstrained 71 registers (7 blocks); 9 or more blocks spill.
#ifndef PK_BUILD_MINB8
#define PK_BUILD_MINB8 8
#endif
template <int KPB>
constexpr int build_min_blocks()
{
    return KPB == 8 ? PK_BUILD_MINB8 : 1;
}
template <int KPB>
__global__ void __launch_bounds__(kBuildWarps * 32, build_min_blocks<KPB>()) k_build(BuildArgs A)
{
    extern __shared__ int smem_i[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    SweepSmem& S = reinterpret_cast<SweepSmem*>(smem_i)[w];
    const int nitems = *A.nitems;
    const int gw = blockIdx.x * kBuildWarps + w, nw = gridDim.x * kBuildWarps;
    for (int item = gw; item < nitems; item += nw) {
        const int2 rng = A.items[item];
        const int total = sweep_ranges(A, S, rng.x, lane);
        for (int p0 = rng.x; p0 < rng.y; p0 += KPB) {
            const int m = min(KPB, rng.y - p0);
            float px[KPB], py[KPB], pz[KPB];
            int cnt[KPB];
#pragma unroll
            for (int p = 0; p < KPB; ++p) {
                if (p < m) {
                    const float4 q = __ldg(A.xs + p0 + p);
                    px[p] = q.x;
                    py[p] = q.y;
                    pz[p] = q.z;
                } else {
                    px[p] = py[p] = pz[p] = -3.0e38f;
                }
                cnt[p] = 0;
            }
            sweep<KPB>(A, S, total, p0, m, px, py, pz, cnt, lane, lt);
#pragma unroll
            for (int p = 0; p < KPB; ++p) {
                if (lane == p && p < m) {
                    const int s = p0 + p;
                    A.hcnt[s] = cnt[p];
                    if (A.count_c) A.count_c[A.perm[s]] = cnt[p];
                    if (cnt[p] > A.row_cap) claim_spill(A, s, cnt[p]);
                }
            }
        }
    }
}

// Hits past the row capacity: one warp per listed particle repeats the
// particle's sweep (same ranges, same candidate order) and writes the hits
// numbered row_cap and up to its spill segment.
__global__ void __launch_bounds__(kBuildWarps * 32) k_spill(BuildArgs A)
{
    extern __shared__ int smem_i[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    SweepSmem& S = reinterpret_cast<SweepSmem*>(smem_i)[w];
    const long long listed = (long long)A.spill[1];
    const long long gw = (long long)blockIdx.x * kBuildWarps + w, nw = (long long)gridDim.x * kBuildWarps;
    for (long long item = gw; item < listed; item += nw) {
        const int s = A.ovf_list[item];
        const int off = A.ovf[s];
        const int total = sweep_ranges(A, S, s, lane);
        const float4 xi = A.xs[s];
        int cnt = 0;
        for (int c0 = 0; c0 < total; c0 += 32) {
            int t;
            const float4 cx = fetch_cand(A.xs, S, c0 + lane, total, t);
            const float d2 = exact_d2(xi, cx);
            const bool hit = d2 < A.T;
            const unsigned b = __ballot_sync(kFull, hit);
            const int pos = cnt + __popc(b & lt);
            if (hit && pos >= A.row_cap) A.hpool[off + (pos - A.row_cap)] = make_uint2((unsigned)t, __float_as_uint(d2));
            cnt += __popc(b);
        }
    }
}

// ---- tau_i: the cap-th smallest key (d2, sorted index) of each hit row.
constexpr int kSelWarps = 8;
constexpr int kSelRegChunks = 4;  // rows of up to 128 hits are held in registers

// Hit e of a row held wholly in the main array.
struct PtrRow {
    const uint2* row;
    __device__ __forceinline__ uint2 at(int e) const { return __ldg(row + e); }
};
// Hit e of one particle's row: the main array up to the row capacity, then
// the particle's spill segment.
struct HitRow {
    const uint2* row;
    const uint2* pool;  // the particle's spill segment (null when none)
    int rc;
    __device__ __forceinline__ uint2 at(int e) const
    {
        if (e < rc) return __ldg(row + e);
        return pool ? __ldg(pool + (e - rc)) : make_uint2(0u, 0xffffffffu);
    }
};

struct SelSmem {
    int hist[kBins];
    uint2 slot[32];
};

__device__ __forceinline__ int sel_bin(unsigned db, float lo, float scale)
{
    return min(max((int)((__uint_as_float(db) - lo) * scale), 0), kBins - 1);
}

// Rank rr (0-based) among the c keys of a row, one warp.  The hits in play
// always form an interval [plo, phi] of d2 values (initially all of them).
// While more than 32 are in play, a 32-bin histogram over the interval
// locates the bin holding the rank, and that bin's smallest and largest d2
// become the next interval.  Bins are monotone in d2, so an interval's hits
// are exactly its bin's hits, and plo falls in bin 0 while phi falls in the
// last bin: every level shrinks the set.  At most 32 hits left are ranked
// exactly by (d2, index); more than 32 hits at one d2 value are ranked by
// index.  Src supplies the row: chunk k of 32 entries (lanes past c hold
// d2 bits 0xffffffff, outside every interval).
template <class Src, class Row>
__device__ __forceinline__ uint2 select_rank(const Src& src, int nch, const Row& row, int c, int rr, float T,
                                             SelSmem& S, int lane, unsigned lt)
{
    unsigned plo = 0u, phi = __float_as_uint(T);  // [0, T]: every hit
    float lo = 0.f, scale = (float)kBins / T;
    int np = c;
    while (np > 32 && plo != phi) {
        S.hist[lane] = 0;
        __syncwarp();
        for (int k = 0; k < nch; ++k) {
            const uint2 v = src(k);
            if (v.y >= plo && v.y <= phi) atomicAdd(&S.hist[sel_bin(v.y, lo, scale)], 1);
        }
        __syncwarp();
        const int hb = S.hist[lane];
        int incl = hb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        const int B = __ffs(__ballot_sync(kFull, incl > rr)) - 1;
        np = __shfl_sync(kFull, hb, B);
        rr -= __shfl_sync(kFull, incl - hb, B);
        // the chosen bin's extreme values
        unsigned mn = 0xffffffffu, mx = 0u;
        for (int k = 0; k < nch; ++k) {
            const uint2 v = src(k);
            if (v.y >= plo && v.y <= phi && sel_bin(v.y, lo, scale) == B) {
                mn = min(mn, v.y);
                mx = max(mx, v.y);
            }
        }
        plo = __reduce_min_sync(kFull, mn);
        phi = __reduce_max_sync(kFull, mx);
        lo = __uint_as_float(plo);
        const float width = __uint_as_float(phi) - lo;
        scale = width > 0.f ? (float)kBins / width : 0.f;
        __syncwarp();
    }
    uint2 mine = make_uint2(0u, 0x7fffffffu);
    if (np <= 32) {
        int k = 0;
        for (int q = 0; q < nch; ++q) {
            const uint2 v = src(q);
            const bool in = v.y >= plo && v.y <= phi;
            const unsigned bal = __ballot_sync(kFull, in);
            if (in) S.slot[k + __popc(bal & lt)] = v;
            k += __popc(bal);
        }
        __syncwarp();
        if (lane < k) {
            const uint2 me = S.slot[lane];
            int rank = 0;
            for (int u = 0; u < k; ++u) {
                const uint2 o = S.slot[u];
                rank += (o.y < me.y || (o.y == me.y && o.x < me.x)) ? 1 : 0;
            }
            if (rank == rr) mine = make_uint2(me.y, me.x);
        }
    } else {
        // more than 32 hits at one d2 value: the rr-th smallest index
        for (int e = lane; e < c; e += 32) {
            const uint2 v = row.at(e);
            if (v.y != plo) continue;
            int rank = 0;
            for (int u = 0; u < c; ++u) {
                const uint2 o = row.at(u);
                rank += (o.y == plo && o.x < v.x) ? 1 : 0;
            }
            if (rank == rr) mine = make_uint2(v.y, v.x);
        }
    }
    const unsigned f = __ballot_sync(kFull, mine.y != 0x7fffffffu);
    const int sl = f ? __ffs(f) - 1 : 0;
    __syncwarp();
    return make_uint2(__shfl_sync(kFull, mine.x, sl), __shfl_sync(kFull, mine.y, sl));
}

// Row chunks from registers (rows of at most 32 * kSelRegChunks hits).
struct RegSrc {
    uint2 h[kSelRegChunks];
    __device__ __forceinline__ uint2 operator()(int k) const
    {
        uint2 v = h[0];
#pragma unroll
        for (int q = 1; q < kSelRegChunks; ++q)
            if (k == q) v = h[q];
        return v;
    }
};
// Row chunks from memory (longer rows).
struct MemSrc {
    HitRow row;
    int c, lane;
    __device__ __forceinline__ uint2 operator()(int k) const
    {
        const int e = k * 32 + lane;
        return e < c ? row.at(e) : make_uint2(0u, 0xffffffffu);
    }
};

// Few keys above tau (E = c - cap small, rows of at most 128 hits): tau is
// found by rounds of warp maxima over 64-bit keys (d2 bits, index), whose
// integer order is the key order.
constexpr int kTopMax = 32;

__device__ __forceinline__ void cswap_desc(unsigned long long& a, unsigned long long& b)
{
    const unsigned long long hi = a > b ? a : b, lo = a > b ? b : a;
    a = hi;
    b = lo;
}

// The (R)-th largest of the warp's keys (R >= 1): each lane sorts its <= 4
// keys descending, then R rounds take the warp's largest head (two 32-bit
// warp maxima: high word, then low word among equal high words) and the owning
// lane advances.  Returns the last key taken as (high, low).
__device__ __forceinline__ uint2 take_largest(unsigned long long (&k)[4], int R)
{
    cswap_desc(k[0], k[1]);
    cswap_desc(k[2], k[3]);
    cswap_desc(k[0], k[2]);
    cswap_desc(k[1], k[3]);
    cswap_desc(k[1], k[2]);
    unsigned mh = 0u, ml = 0u;
    for (int r = 0; r < R; ++r) {
        const unsigned hh = (unsigned)(k[0] >> 32), hl = (unsigned)k[0];
        mh = __reduce_max_sync(kFull, hh);
        ml = __reduce_max_sync(kFull, hh == mh ? hl : 0u);
        if (hh == mh && hl == ml) {
            k[0] = k[1];
            k[1] = k[2];
            k[2] = k[3];
            k[3] = 0ull;
        }
    }
    return make_uint2(mh, ml);
}

// tau from a pivot: the previous frame's tau distance of the same particle
// (d2 bits `hint`).  With L keys at or below the pivot, tau is the
// (L - cap + 1)-th largest of those when L >= cap, else the (cap - L)-th
// smallest of the keys above it (taken as the largest of the complemented
// keys).  Positions move little between frames, so |L - cap| is small and
// few rounds run; the result is the same key whatever the pivot.  A pivot
// that saves nothing falls back to the E + 1 rounds of select_top.
// h: entries lane, lane+32, lane+64, lane+96 of the row (c <= 128).
__device__ __forceinline__ uint2 select_pivot(const uint2 (&h)[4], int c, int cap, unsigned hint, int lane)
{
    const unsigned long long P = ((unsigned long long)hint << 32) | 0xffffffffull;
    unsigned long long k[4];
    bool ok[4];
    int le = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        ok[q] = q * 32 + lane < c;
        k[q] = ((unsigned long long)h[q].y << 32) | h[q].x;
        le += (ok[q] && k[q] <= P) ? 1 : 0;
    }
    le = (int)__reduce_add_sync(kFull, (unsigned)le);
    const int E = c - cap;
    if (le >= cap && le - cap + 1 <= E) {
#pragma unroll
        for (int q = 0; q < 4; ++q) k[q] = (ok[q] && k[q] <= P) ? k[q] : 0ull;
        return take_largest(k, le - cap + 1);
    }
    if (le < cap && cap - le <= E) {
#pragma unroll
        for (int q = 0; q < 4; ++q) k[q] = (ok[q] && k[q] > P) ? ~k[q] : 0ull;
        const uint2 r = take_largest(k, cap - le);
        return make_uint2(~r.x, ~r.y);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) k[q] = ok[q] ? k[q] : 0ull;
    return take_largest(k, E + 1);
}

// A warp takes 32 consecutive particles: lane l reads the count of particle
// base + l, the particles with more than cap hits are selected one after the
// other (their rows loaded into registers when they hold at most 128 hits),
// and lane l writes tau of particle base + l.
#ifndef PK_SEL_MIN_BLOCKS
#define PK_SEL_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kSelWarps * 32, PK_SEL_MIN_BLOCKS)
    k_select(const uint2* __restrict__ hits, const int* __restrict__ hcnt, int n, int cap, int row_cap,
             float T, uint2* __restrict__ tau, const int* __restrict__ perm, unsigned* __restrict__ tau_hint,
             const uint2* __restrict__ hpool, const int* __restrict__ ovf)
{
    __shared__ SelSmem sm[kSelWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    SelSmem& S = sm[w];
    const long long gw = (long long)blockIdx.x * kSelWarps + w, nw = (long long)gridDim.x * kSelWarps;
    for (long long base = gw * 32; base < n; base += nw * 32) {
        const long long s_l = base + lane;
        const int c_l = s_l < n ? __ldg(hcnt + s_l) : 0;
        uint2 tau_l = make_uint2(0x7f800000u, 0x7fffffffu);  // every hit is in N(i)
        unsigned need = __ballot_sync(kFull, c_l > cap);
        const int id_l = c_l > cap ? __ldg(perm + s_l) : 0;
        const unsigned hint_l = c_l > cap ? tau_hint[id_l] : 0xffffffffu;
        // rows of at most 128 hits are read into registers one particle ahead,
        // so the next row's loads overlap the current selection
        uint2 hn[4];
        auto prefetch = [&](unsigned set, uint2(&h)[4]) {
            const int q = set ? __ffs(set) - 1 : 0;
            const int c = __shfl_sync(kFull, c_l, q);
            const uint2* row = hits + (base + q) * row_cap;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int e = k * 32 + lane;
                h[k] = (set && c <= 128 && e < c) ? __ldg(row + e) : make_uint2(0u, 0u);
            }
        };
        prefetch(need, hn);
        while (need) {
            const int q = __ffs(need) - 1;
            need &= need - 1;
            const int c = __shfl_sync(kFull, c_l, q);
            const uint2* row = hits + (base + q) * row_cap;
            uint2 h[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) h[k] = hn[k];
            prefetch(need, hn);
            uint2 r;
            if (c <= 32 * kSelRegChunks && c - cap + 1 <= kTopMax) {
                r = select_pivot(h, c, cap, __shfl_sync(kFull, hint_l, q), lane);
            } else if (c <= 32 * kSelRegChunks) {
                RegSrc src;
#pragma unroll
                for (int k = 0; k < kSelRegChunks; ++k) {
                    const int e = k * 32 + lane;
                    src.h[k] = e < c ? h[k] : make_uint2(0u, 0xffffffffu);
                }
                r = select_rank(src, (c + 31) / 32, PtrRow{row}, c, cap - 1, T, S, lane, lt);
            } else {
                // rows past the row capacity continue in their spill segment
                HitRow hr{row, nullptr, row_cap};
                if (c > row_cap && hpool) {
                    const int o = __ldg(ovf + base + q);
                    if (o >= 0) hr.pool = hpool + o;
                }
                r = select_rank(MemSrc{hr, c, lane}, (c + 31) / 32, hr, c, cap - 1, T, S, lane, lt);
            }
            if (lane == q) tau_l = r;
        }
        if (s_l < n) tau[s_l] = tau_l;
        if (c_l > cap) tau_hint[id_l] = tau_l.x;  // the next frame's pivot
    }
}

// Solver rows from the hit rows: G lanes per particle.  k_emit takes the
// rows that fit the row capacity (all but the longest); k_emit_spill the
// particles listed with a spill segment, whose hits and solver entries past
// the capacity live there.
constexpr int kEmitG = 8;
constexpr int kStash = 128;  // b-only entries kept per group before appending (>= kRowCapMin)
// Chunks of kEmitG entries whose loads are issued together, and resident
// blocks per SM asked of the register allocator: 2 chunks at 8 blocks (32
// registers) measured fastest at 2M, ahead of 1, 3 or 4 chunks at 4-6 blocks,
// and ahead of one thread per particle reading a quad of hits per load
// (0.72-0.81 against 0.66 ms at 2M).
#ifndef PK_EMIT_U
#define PK_EMIT_U 2
#endif
#ifndef PK_EMIT_MINB
#define PK_EMIT_MINB 8
#endif
constexpr int kEmitU = PK_EMIT_U;

struct EmitArgs {
    const int* hcnt;
    const uint2* hits;
    const uint2* hpool;  // null: no spill pool
    const int* ovf;
    const unsigned long long* spill;
    const int* ovf_list;
    const uint2* tau;
    const int* perm;
    int n, cap, rc;
    int* rows;
    int* rpool;
    int2* rcnt;
    int* pub_index;
    int* pub_elements;
    long long pub_capacity;
    const int* offs;
    int* err;
};

__global__ void __launch_bounds__(256, PK_EMIT_MINB) k_emit(EmitArgs A)
{
    __shared__ int s_b[256 / kEmitG][kStash];  // b-only entries of each group
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = gid / kEmitG, sub = gid % kEmitG, grp = threadIdx.x / kEmitG;
    const int lane = threadIdx.x & 31;
    const unsigned gmask = ((1u << kEmitG) - 1u) << (lane & ~(kEmitG - 1));
    const unsigned lt_g = ((1u << lane) - 1u) & gmask;
    int cnt = s < A.n ? A.hcnt[s] : 0;
    bool valid = s < A.n;
    if (valid && cnt > A.rc) {
        if (A.hpool && __ldg(A.ovf + s) >= 0)
            valid = false;  // k_emit_spill's
        else
            cnt = A.rc;     // no segment could be had: cut short, the error is latched
    }
    if (!valid) cnt = 0;
    const bool capped = A.cap > 0;
    int ps = 0;
    uint2 ti = make_uint2(0x7f800000u, 0x7fffffffu);
    long long pbase = 0;
    const bool pub = A.pub_elements != nullptr;
    if (valid) {
        if (capped) ti = A.tau[s];
        ps = A.perm[s];
        if (pub) pbase = capped ? (long long)ps * A.cap : (long long)A.offs[ps];
    }
    const int so = valid ? s : 0;
    const uint2* hrow = A.hits + (long long)so * A.rc;
    // entry q of the solver row: srow[(q >> 2) * 128 + (q & 3)] (row_slot)
    int* const srow = A.rows + row_slot(so, 0, A.rc);
    // every lane of the warp iterates to the longest row of the warp's groups
    int cmax = cnt;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) cmax = max(cmax, __shfl_xor_sync(kFull, cmax, o));
    int nA = 0, nB = 0;
    bool over = false;
    // kEmitU chunks per round: their hit loads, then their tau_j gathers, are
    // all in flight before the first ballot (the chunks are then decided and
    // written in order, as one chunk at a time would)
    for (int e0 = 0; e0 < cmax; e0 += kEmitG * kEmitU) {
        uint2 h[kEmitU], tj[kEmitU];
#pragma unroll
        for (int u = 0; u < kEmitU; ++u) {
            const int e = e0 + u * kEmitG + sub;
            h[u] = (valid && e < cnt) ? __ldg(hrow + e) : make_uint2(0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < kEmitU; ++u) {
            const int e = e0 + u * kEmitG + sub;
            tj[u] = (capped && valid && e < cnt) ? __ldg(A.tau + h[u].x) : make_uint2(0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < kEmitU; ++u) {
            if (e0 + u * kEmitG >= cmax) break;  // warp-uniform: cmax is the warp's maximum
            const int e = e0 + u * kEmitG + sub;
            bool fa = false, fb = false;
            const int t = (int)h[u].x;
            if (valid && e < cnt) {
                if (capped) {
                    const float d2 = __uint_as_float(h[u].y);
                    fa = key_le(d2, t, ti);
                    fb = key_le(d2, s, tj[u]);
                } else {
                    fa = fb = true;
                }
            }
            const unsigned ba = __ballot_sync(kFull, fa) & gmask;
            const unsigned bb = __ballot_sync(kFull, fb && !fa) & gmask;
            if (fa) {
                const int q = nA + __popc(ba & lt_g);
                srow[(q >> 2) * 128 + (q & 3)] = t | kRowFlagA | (fb ? kRowFlagB : 0);
                if (pub) {
                    const long long o = pbase + q;
                    if (capped ? (q < A.cap) : (o < A.pub_capacity))
                        A.pub_elements[o] = __ldg(A.perm + t);
                    else
                        over = true;
                }
            }
            if (fb && !fa) {
                // a row of at most rc <= kStash hits has at most kStash b-only entries
                const int q = nB + __popc(bb & lt_g);
                s_b[grp][q] = t | kRowFlagB;
            }
            nA += __popc(ba);
            nB += __popc(bb);
        }
    }
    __syncwarp();
    if (valid) {
        for (int e = sub; e < nB; e += kEmitG) {
            const int q = nA + e;
            srow[(q >> 2) * 128 + (q & 3)] = s_b[grp][e];
        }
        if (sub == 0) {
            A.rcnt[s] = make_int2(nA, nA + nB);
            if (A.pub_index != nullptr) A.pub_index[ps] = capped ? min(nA, A.cap) : A.offs[ps];
        }
    }
    if (__any_sync(kFull, over) && lane == 0) atomicOr(A.err, kErrPublicOverflow);
}

// The same for the particles listed with a spill segment (rows longer than
// the capacity: dense clusters only), a warp per four of them: hits and
// solver entries numbered rc and up are in the segment, and b-only entries
// past the stash are taken by a second walk over the row.
__global__ void __launch_bounds__(256) k_emit_spill(EmitArgs A)
{
    __shared__ int s_b[256 / kEmitG][kStash];
    const int lane = threadIdx.x & 31, sub = lane % kEmitG, grp = threadIdx.x / kEmitG;
    const unsigned gmask = ((1u << kEmitG) - 1u) << (lane & ~(kEmitG - 1));
    const unsigned lt_g = ((1u << lane) - 1u) & gmask;
    const long long listed = (long long)*A.spill;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    const bool capped = A.cap > 0;
    const bool pub = A.pub_elements != nullptr;
    for (long long r0 = w * 4; r0 < listed; r0 += nwarp * 4) {
        const long long item = r0 + lane / kEmitG;
        const bool valid = item < listed;
        const int s = valid ? A.ovf_list[item] : 0;
        const int cnt = valid ? A.hcnt[s] : 0;
        const int o = valid ? A.ovf[s] : 0;
        const uint2 ti = (valid && capped) ? A.tau[s] : make_uint2(0x7f800000u, 0x7fffffffu);
        const int ps = valid ? A.perm[s] : 0;
        const long long pbase = (valid && pub) ? (capped ? (long long)ps * A.cap : (long long)A.offs[ps]) : 0;
        const uint2* hrow = A.hits + (long long)s * A.rc;
        auto hit = [&](int e) { return e < A.rc ? __ldg(hrow + e) : __ldg(A.hpool + o + (e - A.rc)); };
        auto put = [&](int q, int v) {
            if (q < A.rc)
                A.rows[row_slot(s, q, A.rc)] = v;
            else
                A.rpool[o + (q - A.rc)] = v;
        };
        int cmax = cnt;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) cmax = max(cmax, __shfl_xor_sync(kFull, cmax, off));
        int nA = 0, nB = 0;
        bool over = false;
        for (int e0 = 0; e0 < cmax; e0 += kEmitG) {
            const int e = e0 + sub;
            bool fa = false, fb = false;
            int t = 0;
            if (valid && e < cnt) {
                const uint2 h = hit(e);
                t = (int)h.x;
                if (capped) {
                    const float d2 = __uint_as_float(h.y);
                    fa = key_le(d2, t, ti);
                    fb = key_le(d2, s, __ldg(A.tau + t));
                } else {
                    fa = fb = true;
                }
            }
            const unsigned ba = __ballot_sync(kFull, fa) & gmask;
            const unsigned bb = __ballot_sync(kFull, fb && !fa) & gmask;
            if (fa) {
                const int q = nA + __popc(ba & lt_g);
                put(q, t | kRowFlagA | (fb ? kRowFlagB : 0));
                if (pub) {
                    const long long po = pbase + q;
                    if (capped ? (q < A.cap) : (po < A.pub_capacity))
                        A.pub_elements[po] = __ldg(A.perm + t);
                    else
                        over = true;
                }
            }
            if (fb && !fa) {
                const int q = nB + __popc(bb & lt_g);
                if (q < kStash) s_b[grp][q] = t | kRowFlagB;
            }
            nA += __popc(ba);
            nB += __popc(bb);
        }
        __syncwarp();
        if (valid)
            for (int e = sub; e < min(nB, kStash); e += kEmitG) put(nA + e, s_b[grp][e]);
        __syncwarp();
        if (__any_sync(kFull, nB > kStash)) {
            int kb = 0;
            for (int e0 = 0; e0 < cmax; e0 += kEmitG) {
                const int e = e0 + sub;
                bool fbo = false;
                int t = 0;
                if (valid && nB > kStash && e < cnt) {
                    const uint2 h = hit(e);
                    t = (int)h.x;
                    const float d2 = __uint_as_float(h.y);
                    fbo = !key_le(d2, t, ti) && key_le(d2, s, __ldg(A.tau + t));
                }
                const unsigned bb = __ballot_sync(kFull, fbo) & gmask;
                if (fbo) {
                    const int q = kb + __popc(bb & lt_g);
                    if (q >= kStash) put(nA + q, t | kRowFlagB);
                }
                kb += __popc(bb);
            }
        }
        if (valid && sub == 0) {
            A.rcnt[s] = make_int2(nA, nA + nB);
            if (A.pub_index != nullptr) A.pub_index[ps] = capped ? min(nA, A.cap) : A.offs[ps];
        }
        if (__any_sync(kFull, over) && lane == 0) atomicOr(A.err, kErrPublicOverflow);
    }
}

// Smallest float T with sqrt_rn(T) >= h: for every float d2, sqrt_rn(d2) < h
// exactly when d2 < T (host sqrtf is correctly rounded, as __fsqrt_rn is).
static float radius_threshold(float h)
{
    float T = h * h;
    while (std::sqrt(T) < h) T = std::nextafter(T, INFINITY);
    while (T > 0.0f && std::sqrt(std::nextafter(T, 0.0f)) >= h) T = std::nextafter(T, 0.0f);
    return T;
}

int build_rows(pk_ctx* c, int n, const Grid& g, float h, int cap, int row_cap, int* pub_index,
               int* pub_elements, long long pub_capacity, cudaStream_t st, bool spill)
{
    if (n <= 0) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // a persistent grid: as many warps per SM as registers and shared memory allow
    const int pbn = c->tune.build_pb;
    if (pbn == 8)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build<8>, kBuildWarps * 32, kBuildSmem);
    else if (pbn == 4)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build<4>, kBuildWarps * 32, kBuildSmem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build<kPB>, kBuildWarps * 32, kBuildSmem);
    if (sms <= 0) sms = 148;
    if (per_sm <= 0) per_sm = 1;
    int launches = 0;
    const bool dyn_pub = cap <= 0 && pub_index != nullptr;
    const bool capped = cap > 0;
    BuildArgs A;
    A.xs = c->xs_pre;
    A.start = c->cell_start;
    A.items = c->items;
    A.nitems = c->nitems;
    A.g = g;
    A.n = n;
    A.row_cap = row_cap;
    A.T = radius_threshold(h);
    A.hits = c->hits;
    A.hcnt = c->hcnt;
    A.count_c = dyn_pub ? c->count_c : nullptr;
    A.perm = c->perm;
    A.err = c->d_err;
    A.pool_cap = spill ? c->pool_cap : 0;
    A.spill = c->spill;
    A.ovf = c->ovf;
    A.ovf_list = c->ovf_list;
    A.hpool = c->hpool;
    const int blocks = std::min((n + kBuildWarps - 1) / kBuildWarps, sms * per_sm);
    prof_begin(c, PK_PROF_SELECT, st);
    cudaMemsetAsync(c->spill, 0, 2 * sizeof(unsigned long long), st);
    if (c->tune.on) cudaEventRecord(c->tune.ev[0], st);
    if (pbn == 8)
        k_build<8><<<blocks, kBuildWarps * 32, kBuildSmem, st>>>(A);
    else if (pbn == 4)
        k_build<4><<<blocks, kBuildWarps * 32, kBuildSmem, st>>>(A);
    else
        k_build<kPB><<<blocks, kBuildWarps * 32, kBuildSmem, st>>>(A);
    if (c->tune.on) cudaEventRecord(c->tune.ev[1], st);
    ++launches;
    const uint2* hpool = A.pool_cap > 0 ? c->hpool : nullptr;
    if (hpool) {
        // the hits past the row capacity (an empty launch when no row is that long)
        k_spill<<<sms * 2, kBuildWarps * 32, kBuildSmem, st>>>(A);
        ++launches;
    }
    if (capped) {
        const int sb = (int)std::min<long long>(((long long)n + 32 * kSelWarps - 1) / (32 * kSelWarps), (long long)sms * 8);
        k_select<<<sb, kSelWarps * 32, 0, st>>>(c->hits, c->hcnt, n, cap, row_cap, A.T, c->tau, c->perm,
                                                c->tau_hint, hpool, hpool ? c->ovf : nullptr);
        ++launches;
    }
    if (dyn_pub) {
        exclusive_scan(c->count_c, n, c->offs, c->scan_part, st);
        launches += scan_launches();
    }
    prof_end(c, PK_PROF_SELECT, st);
    prof_begin(c, PK_PROF_EMIT, st);
    EmitArgs E;
    E.hcnt = c->hcnt;
    E.hits = c->hits;
    E.hpool = hpool;
    E.ovf = c->ovf;
    E.spill = c->spill + 1;
    E.ovf_list = c->ovf_list;
    E.tau = c->tau;
    E.perm = c->perm;
    E.n = n;
    E.cap = cap;
    E.rc = row_cap;
    E.rows = c->rows;
    E.rpool = c->rpool;
    E.rcnt = c->rcnt;
    E.pub_index = pub_index;
    E.pub_elements = pub_elements;
    E.pub_capacity = pub_capacity;
    E.offs = c->offs;
    E.err = c->d_err;
    k_emit<<<(unsigned)(((long long)n * kEmitG + 255) / 256), 256, 0, st>>>(E);
    if (hpool) {
        k_emit_spill<<<sms, 256, 0, st>>>(E);  // an empty launch when no row is that long
        ++launches;
    }
    prof_end(c, PK_PROF_EMIT, st);
    return launches + 1;
}

}  // namespace pk
