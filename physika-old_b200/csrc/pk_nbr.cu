// pk_nbr.cu -- neighbour rows over the cell-sorted particles.
//
// Reference: K_ComputeNeighborFixed (NeighborQuery.cu:514-581) keeps, per
// particle, the `cap` nearest hits with d < h by replacing the current
// farthest entry; K_CalNeighborSize/K_GetNeighborElements (:245-276,337-367)
// build the uncapped list.  A capped list is asymmetric (j in N(i) does not
// imply i in N(j)), and DensityPBD scatters each pair's displacement to both
// ends (DensityPBD.cu:161-173).  To solve that with gathers only, each row
// holds the union N(i) + {j : i in N(j)} with two flag bits, so a pair's
// multiplicity in i's displacement sum is known without atomics:
//   pass 1 (k_select): one warp per particle scans the 27 cells, compacts the
//     hits into shared memory, and finds tau_i = the cap-th smallest
//     (distance, sorted index) key with a 256-bin histogram of d/h and an
//     exact rank among the few hits of the boundary bin;
//   pass 2 (k_emit): the same scan marks each hit with a = key <= tau_i
//     (j in N(i)) and b = key' <= tau_j (i in N(j), tau_j gathered), writes
//     a-entries first, then b-only entries, and the public NeighborList in
//     caller ids (fixed: index = count, dynamic: CSR) on the way.
// Distances use exact_dist (explicit roundings), so the d < h decisions and
// the ordering are bit-identical for (i,j) and (j,i) and match the CPU
// restatement.
#include "pk_kernels.cuh"

namespace pk {

constexpr int kBuildWarps = 4;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool key_le(float d, int id, uint2 tau)
{
    float td = __uint_as_float(tau.x);
    return d < td || (d == td && id <= (int)tau.y);
}

template <bool kCapped>
__global__ void __launch_bounds__(kBuildWarps * 32)
    k_select(const float4* __restrict__ xs, const int* __restrict__ start, Grid g, int n, int cap,
             float h, const int* __restrict__ perm, uint2* __restrict__ tau,
             int* __restrict__ count_c, int* __restrict__ err)
{
    __shared__ float s_d[kBuildWarps][kMaxHits];
    __shared__ int s_t[kBuildWarps][kMaxHits];
    __shared__ int s_h[kBuildWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int s = blockIdx.x * kBuildWarps + w;
    if (s >= n) return;  // warp-uniform
    const unsigned lt = (1u << lane) - 1u;
    const float4 xi = xs[s];
    const int3 c = cell3(g, xi.x, xi.y, xi.z);
    int cnt = 0;
    for (int o = 0; o < 27; ++o) {
        int key = cell_key(g, c.x + kOffset27[o][0], c.y + kOffset27[o][1], c.z + kOffset27[o][2]);
        if (key < 0) continue;
        int a = __ldg(start + key), b = __ldg(start + key + 1);
        for (int t0 = a; t0 < b; t0 += 32) {
            int t = t0 + lane;
            float d = 0.f;
            bool hit = false;
            if (t < b) {
                d = exact_dist(xi, __ldg(xs + t));
                hit = d < h;
            }
            unsigned m = __ballot_sync(kFull, hit);
            if (kCapped && hit) {
                int p = cnt + __popc(m & lt);
                if (p < kMaxHits) {
                    s_d[w][p] = d;
                    s_t[w][p] = t;
                }
            }
            cnt += __popc(m);
        }
    }
    if (count_c != nullptr && lane == 0) count_c[perm[s]] = cnt;
    if (!kCapped) return;
    if (cnt <= cap || cnt > kMaxHits) {
        if (cnt > kMaxHits && lane == 0) atomicOr(err, kErrHitOverflow);
        if (lane == 0) tau[s] = make_uint2(0x7f800000u, 0x7fffffffu);  // every hit is in N(i)
        return;
    }
    // Placeholder until the selection below writes the exact key (ordered by
    // the __syncwarp that follows).
    if (lane == 0) tau[s] = make_uint2(0x7f800000u, 0x7fffffffu);
    __syncwarp();
    // ---- histogram of d over 256 equal bins of [0, h): monotone in d.
    int* hist = s_h[w];
    for (int k = lane; k < 256; k += 32) hist[k] = 0;
    __syncwarp();
    const float scale = 256.0f / h;
    for (int e = lane; e < cnt; e += 32) atomicAdd(&hist[min((int)(s_d[w][e] * scale), 255)], 1);
    __syncwarp();
    int loc[8], sum = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        loc[k] = hist[lane * 8 + k];
        sum += loc[k];
    }
    int incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(kFull, incl, off);
        if (lane >= off) incl += y;
    }
    const int excl = incl - sum;
    const int r = cap - 1;  // 0-based rank of tau
    unsigned own = __ballot_sync(kFull, excl <= r && r < incl);
    int src = __ffs(own) - 1;
    int B = 0, before = 0;
    if (lane == src) {
        int acc = excl;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (r < acc + loc[k]) {
                B = lane * 8 + k;
                before = acc;
                break;
            }
            acc += loc[k];
        }
    }
    B = __shfl_sync(kFull, B, src);
    before = __shfl_sync(kFull, before, src);
    const int rr = r - before;  // rank of tau among the hits of bin B
    __syncwarp();
    // ---- compact bin B's hits (reusing the histogram as 128 (d, t) pairs)
    int m = 0;
    for (int e0 = 0; e0 < cnt; e0 += 32) {
        int e = e0 + lane;
        bool in = false;
        float d = 0.f;
        int t = 0;
        if (e < cnt) {
            d = s_d[w][e];
            t = s_t[w][e];
            in = min((int)(d * scale), 255) == B;
        }
        unsigned mm = __ballot_sync(kFull, in);
        if (in) {
            int p = m + __popc(mm & lt);
            if (p < 128) {
                hist[2 * p] = __float_as_int(d);
                hist[2 * p + 1] = t;
            }
        }
        m += __popc(mm);
    }
    __syncwarp();
    if (m <= 128) {
        for (int q = lane; q < m; q += 32) {
            float dq = __int_as_float(hist[2 * q]);
            int tq = hist[2 * q + 1];
            int rank = 0;
            for (int u = 0; u < m; ++u) {
                float du = __int_as_float(hist[2 * u]);
                int tu = hist[2 * u + 1];
                rank += (du < dq || (du == dq && tu < tq)) ? 1 : 0;
            }
            if (rank == rr) tau[s] = make_uint2(__float_as_uint(dq), (unsigned)tq);
        }
    } else {
        // Degenerate bin (many equal distances): rank among all of bin B.
        for (int e = lane; e < cnt; e += 32) {
            float dq = s_d[w][e];
            int tq = s_t[w][e];
            if (min((int)(dq * scale), 255) != B) continue;
            int rank = 0;
            for (int u = 0; u < cnt; ++u) {
                float du = s_d[w][u];
                int tu = s_t[w][u];
                if (min((int)(du * scale), 255) != B) continue;
                rank += (du < dq || (du == dq && tu < tq)) ? 1 : 0;
            }
            if (rank == rr) tau[s] = make_uint2(__float_as_uint(dq), (unsigned)tq);
        }
    }
}

__global__ void __launch_bounds__(kBuildWarps * 32)
    k_emit(const float4* __restrict__ xs, const int* __restrict__ start, Grid g, int n, int cap,
           float h, const int* __restrict__ perm, const uint2* __restrict__ tau,
           int* __restrict__ rows, int2* __restrict__ rcnt, int row_cap,
           int* __restrict__ pub_index, int* __restrict__ pub_elements, long long pub_capacity,
           const int* __restrict__ offs, int* __restrict__ err)
{
    __shared__ int s_b[kBuildWarps][kMaxHits];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int s = blockIdx.x * kBuildWarps + w;
    if (s >= n) return;  // warp-uniform
    const unsigned lt = (1u << lane) - 1u;
    const bool capped = cap > 0;
    const float4 xi = xs[s];
    const uint2 ti = capped ? tau[s] : make_uint2(0x7f800000u, 0x7fffffffu);
    int* row = rows + (long long)s * row_cap;
    const int ps = perm[s];
    const bool pub = pub_elements != nullptr;
    long long pbase = 0;
    if (pub) pbase = capped ? (long long)ps * cap : (long long)offs[ps];
    const int3 c = cell3(g, xi.x, xi.y, xi.z);
    int nA = 0, nB = 0;
    bool pub_over = false;
    for (int o = 0; o < 27; ++o) {
        int key = cell_key(g, c.x + kOffset27[o][0], c.y + kOffset27[o][1], c.z + kOffset27[o][2]);
        if (key < 0) continue;
        int a0 = __ldg(start + key), b0 = __ldg(start + key + 1);
        for (int t0 = a0; t0 < b0; t0 += 32) {
            int t = t0 + lane;
            bool fa = false, fb = false;
            if (t < b0) {
                float d = exact_dist(xi, __ldg(xs + t));
                if (d < h) {
                    fa = key_le(d, t, ti);
                    fb = capped ? key_le(d, s, __ldg(tau + t)) : true;
                }
            }
            unsigned ma = __ballot_sync(kFull, fa);
            unsigned mb = __ballot_sync(kFull, fb && !fa);
            if (fa) {
                int p = nA + __popc(ma & lt);
                if (p < row_cap) row[p] = t | kRowFlagA | (fb ? kRowFlagB : 0);
                if (pub) {
                    long long q = pbase + p;
                    if (capped ? (p < cap) : (q < pub_capacity))
                        pub_elements[q] = __ldg(perm + t);
                    else
                        pub_over = true;
                }
            }
            if (fb && !fa) {
                int p = nB + __popc(mb & lt);
                if (p < kMaxHits) s_b[w][p] = t | kRowFlagB;
            }
            nA += __popc(ma);
            nB += __popc(mb);
        }
    }
    __syncwarp();
    const int nBw = min(nB, kMaxHits);
    for (int e = lane; e < nBw; e += 32) {
        int p = nA + e;
        if (p < row_cap) row[p] = s_b[w][e];
    }
    if (__any_sync(kFull, pub_over) && lane == 0) atomicOr(err, kErrPublicOverflow);
    if (lane == 0) {
        if (nA + nB > row_cap || nB > kMaxHits) atomicOr(err, kErrRowOverflow);
        rcnt[s] = make_int2(min(nA, row_cap), min(nA + nB, row_cap));
        if (pub_index != nullptr) pub_index[ps] = capped ? min(nA, cap) : offs[ps];
    }
}

int build_rows(pk_ctx* c, int n, const Grid& g, float h, int cap, int row_cap, int* pub_index,
               int* pub_elements, long long pub_capacity, cudaStream_t st)
{
    if (n <= 0) return 0;
    int launches = 0;
    unsigned nb = (unsigned)((n + kBuildWarps - 1) / kBuildWarps);
    const bool dyn_pub = cap <= 0 && pub_index != nullptr;
    prof_begin(c, PK_PROF_SELECT, st);
    if (cap > 0) {
        k_select<true><<<nb, kBuildWarps * 32, 0, st>>>(c->xs_pre, c->cell_start, g, n, cap, h,
                                                        c->perm, c->tau, nullptr, c->d_err);
        ++launches;
    } else if (dyn_pub) {
        k_select<false><<<nb, kBuildWarps * 32, 0, st>>>(c->xs_pre, c->cell_start, g, n, cap, h,
                                                         c->perm, c->tau, c->count_c, c->d_err);
        exclusive_scan(c->count_c, n, c->offs, c->scan_part, st);
        launches += 1 + scan_launches();
    }
    prof_end(c, PK_PROF_SELECT, st);
    prof_begin(c, PK_PROF_EMIT, st);
    k_emit<<<nb, kBuildWarps * 32, 0, st>>>(c->xs_pre, c->cell_start, g, n, cap, h, c->perm, c->tau,
                                            c->rows, c->rcnt, row_cap, pub_index, pub_elements,
                                            pub_capacity, c->offs, c->d_err);
    prof_end(c, PK_PROF_EMIT, st);
    return launches + 1;
}

}  // namespace pk
