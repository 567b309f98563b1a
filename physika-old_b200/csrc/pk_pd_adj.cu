// pk_pd_adj.cu -- the peridynamics projection as gathers, its adjoint, and
// checkpointed rollouts (float forward with a double reverse pass, and an
// all-double rollout for reference gradients).
//
// Forward: one projection iteration of ElasticityModule::solveElasticity
// (EM_EnforceElasticity, ElasticityModule.cu:123-242, + K_UpdatePosition
// :281-292) is
//     x'_i = (x_old,i + D_i(x)) / (1 + W_i)
// with, over the alive bonds i->j of i's frozen rest shape (r_ij = |rest_i -
// rest_j| > 0.01 h) and the alive bonds k->i that name i (the incoming list,
// built once because the bonds are frozen):
//     D_i = sum_{i->j} mu_ij (x_j + r n(F_i e_ij)) + la_ij (x_j + r n(x_i - x_j))
//         + sum_{k->i} mu_ki (x_k - r n(F_k e_ki)) + la_ki (x_k - r n(x_k - x_i))
//     W_i = sum_{i->j} (mu_ij + la_ij) + sum_{k->i} (mu_ki + la_ki)
// mu_ij = mu bulk_i wrr(r), la_ij = lambda bulk_i wrr(r), e_ij = rest_i -
// rest_j, n(u) = u/|u| (0 below epsilon), and F_i the deformation gradient of
// EM_EnforceElasticity's first loop (identity when det F < -0.001).  The
// reference scatters the k->i terms with atomics; here every particle gathers
// them, so the sums have a fixed order and a recomputed trajectory repeats the
// forward bit for bit, which the adjoint relies on.
//
// Adjoint of one iteration, given g = dL/dx':  a_i = g_i/(1 + W_i) (the
// adjoint of D_i and of x_old,i); then
//   kernel B (per source i): Fbar_i = sum_{i->j} mu_ij r J_n(F_i e)^T (a_i - a_j) e^T,
//     the bulk_i gradient (a bond's weight w adds w*target to D and w to W at
//     both ends: d x'/d w = (target - x')/(1 + W)),
//     and G_i = dL/dFraw_i / (tw_i h), Fraw being the unscaled first-loop sum;
//   kernel C (per particle): dL/dx_i from the linear parts, the n(x_i - x_j)
//     terms (J_n(u) = (I - n n^T)/|u|) and F (x_j enters F_i through
//     (x_j - x_i)/h: + G_i q_j at j, - G_i q_j at i).
#include "pk_kernels.cuh"
#include "pk_pd_common.cuh"

namespace pk {

template <class R>
struct V3 {
    R x, y, z;
};

template <class R>
__device__ __forceinline__ V3<R> ld3(const R* p, long long i)
{
    return V3<R>{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}
template <class R, class RX>
__device__ __forceinline__ V3<R> ld3r(const RX* p, long long i)
{
    return V3<R>{(R)p[3 * i], (R)p[3 * i + 1], (R)p[3 * i + 2]};
}
template <class R>
__device__ __forceinline__ R dot3(V3<R> a, V3<R> b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

// v.norm() > EPSILON ? v.normalize() : 0 (ElasticityModule.cu:211-212);
// normalize() gives 0 below FLT_EPSILON (vector_3d.inl:220-224).  Returns the
// length, or 0 when the result is the zero vector.
template <class R>
__device__ __forceinline__ R unit_or_zero(V3<R>& u)
{
    const R l = sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
    if (l > (R)kEpsilon && l > (R)1.1920928955078125e-7) {
        const R is = (R)1 / l;
        u.x *= is;
        u.y *= is;
        u.z *= is;
        return l;
    }
    u.x = u.y = u.z = (R)0;
    return (R)0;
}

// Adjoint of n = u/|u|: ubar = (nbar - n (n.nbar)) / |u| (0 where n was zeroed).
template <class R>
__device__ __forceinline__ V3<R> unit_vjp(V3<R> n, R l, V3<R> nbar)
{
    if (l == (R)0) return V3<R>{0, 0, 0};
    const R d = dot3(n, nbar), il = (R)1 / l;
    return V3<R>{(nbar.x - n.x * d) * il, (nbar.y - n.y * d) * il, (nbar.z - n.z * d) * il};
}

struct PdBonds {
    const int* index;
    int cap;
    long long total;
    int n;
    const int* ridx;
    const float* rpos;
    const unsigned char* alive;
    const float* invK;
    const int* in_off;   // incoming bonds k->i of particle i: in_list[in_off[i] .. in_off[i+1])
    const int2* in_list; // (source k, bond slot)
    const int* in_slot;  // the bond slots of in_list alone
    float h, mu, lambda;
    float inv_h;         // 1/h: the kernels multiply where the reference divides
};

// CorrectedKernel Weight and WeightRR (Kernel.h:99-142) with q = r * (1/h).
// The bond geometry every forward and reverse kernel evaluates -- the rest
// length r and these weights -- is written with every rounding explicit, so
// each kernel gets the same bits whatever the compiler's contraction choices
// at its call site: the reverse pass must see the forward's r (a one-ulp
// difference in r between the forward's F and the reverse's recomputation
// moved the double adjoint of a 2,000-iteration rollout by 1.4e-4).  r is
// the reference's compiled Vector3f::norm (exact_norm3).
__device__ __forceinline__ float bond_len(float e0, float e1, float e2) { return exact_norm3(e0, e1, e2); }
__device__ __forceinline__ float corr_w_f(float r, float inv_h)
{
    const float q = __fmul_rn(r, inv_h);
    const float qq = __fmul_rn(q, q);
    return q > 1.0f ? 0.0f : __fmul_rn(__fmul_rn(qq, q), __fsub_rn(1.0f, qq));
}
__device__ __forceinline__ float corr_wrr_f(float r, float inv_h)
{
    const float q = __fmul_rn(r, inv_h);
    return q > 1.0f ? 0.0f : __fmul_rn(__fmul_rn(q, __fsub_rn(1.0f, __fmul_rn(q, q))), __fmul_rn(inv_h, inv_h));
}

// unit_or_zero without the length: one reciprocal square root.
template <class R>
__device__ __forceinline__ void unit_fast(V3<R>& u)
{
    const R l2 = u.x * u.x + u.y * u.y + u.z * u.z;
    if (l2 > (R)(kEpsilon * kEpsilon) && l2 > (R)1.4210854715202004e-14) {
        const R is = rsqrt(l2);
        u.x *= is;
        u.y *= is;
        u.z *= is;
    } else {
        u.x = u.y = u.z = (R)0;
    }
}

// A bond slot holds 4 values (the bond's term and a zero pad) and is written
// whole in one store: a slot written in part leaves its 32-byte sector
// partly written, which the L2 completes by reading it from DRAM (k_pd_FP
// read 1.38 GB per launch on the 524,288-particle bar, half of it that).
__device__ __forceinline__ void store_slot(float* o, float x, float y, float z)
{
    *reinterpret_cast<float4*>(o) = make_float4(x, y, z, 0.f);
}
__device__ __forceinline__ void store_slot(double* o, double x, double y, double z)
{
    reinterpret_cast<double2*>(o)[0] = make_double2(x, y);
    reinterpret_cast<double2*>(o)[1] = make_double2(z, 0.0);
}
__device__ __forceinline__ void store_slot(float* o, float x, float y, float z, float w)
{
    *reinterpret_cast<float4*>(o) = make_float4(x, y, z, w);
}
__device__ __forceinline__ void store_slot(double* o, double x, double y, double z, double w)
{
    reinterpret_cast<double2*>(o)[0] = make_double2(x, y);
    reinterpret_cast<double2*>(o)[1] = make_double2(z, w);
}
__device__ __forceinline__ void add_slot(const float* g, float& x, float& y, float& z, float& w)
{
    const float4 q = __ldg(reinterpret_cast<const float4*>(g));
    x += q.x;
    y += q.y;
    z += q.z;
    w += q.w;
}
__device__ __forceinline__ void add_slot(const double* g, double& x, double& y, double& z, double& w)
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(g));
    const double2 b = __ldg(reinterpret_cast<const double2*>(g) + 1);
    x += a.x;
    y += a.y;
    z += b.x;
    w += b.y;
}
__device__ __forceinline__ void add_slot(const float* g, float& x, float& y, float& z)
{
    const float4 q = __ldg(reinterpret_cast<const float4*>(g));
    x += q.x;
    y += q.y;
    z += q.z;
}
__device__ __forceinline__ void add_slot(const double* g, double& x, double& y, double& z)
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(g));
    const double b = __ldg(g + 2);
    x += a.x;
    y += a.y;
    z += b;
}

// Every particle is handled by a group of kPdG lanes of one warp: lane `sub`
// takes bonds sub, sub + kPdG, ... and the group's partial sums are combined
// with xor shuffles in a fixed order (deterministic, so a replayed rollout
// repeats the forward bit for bit).
// The deformation walk loads the next bond's flag, neighbour and rest
// position (and the gather the next incoming slot) while the current one is
// used: 9.12 -> 8.35 ms per elastic-bar step, the same results.
constexpr int kPdG = 8;
constexpr int kPdBlock = 128;
constexpr unsigned kPdAll = 0xffffffffu;

template <class R>
__device__ __forceinline__ R gsum(R v)
{
#pragma unroll
    for (int o = kPdG / 2; o >= 1; o >>= 1) v += __shfl_xor_sync(kPdAll, v, o);
    return v;
}

struct PdLane {
    int i, sub;
    bool valid;
};
__device__ __forceinline__ PdLane pd_lane(int n)
{
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    PdLane L;
    L.i = gid / kPdG;
    L.sub = gid % kPdG;
    L.valid = L.i < n;
    if (!L.valid) L.i = n - 1;  // idle lanes of the last group mirror a valid particle, write nothing
    return L;
}

// First loop of EM_EnforceElasticity: F_i = (sum p q^T / tw) K^-1 with
// p = (x_j - x_i)/h, q = e wt / h, e = rest_j - rest_i, and the identity when
// det F < -0.001.  Called by all lanes of i's group; every lane gets F, tw
// and whether the identity was taken.
// With `stash`, the lane's first kPdStash bonds are kept in shared memory
// (rest vector e and the neighbour, stored as ~j for a dead bond) for a
// second walk over them.
constexpr int kPdStash = 10;  // bonds per lane: cap 80 over 8 lanes
template <class R, class RX>
__device__ void pd_deformation(const PdBonds& B, const RX* x, int i, int sub, R F[3][3], float& tw_out,
                               bool& ident, float4 (*stash)[kPdBlock] = nullptr)
{
    const long long a0 = pd_at(B.index, B.cap, i, 0);
    const float ri0 = B.rpos[3 * a0], ri1 = B.rpos[3 * a0 + 1], ri2 = B.rpos[3 * a0 + 2];
    const V3<R> ci = ld3r<R>(x, i);
    const int m = pd_size(B.index, B.cap, B.total, B.n, i);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) F[a][b] = 0;
    float tw = 0.f;
    // the next bond's flag, neighbour and rest position are loaded one bond ahead
    bool al_n = false;
    int j_n = 0;
    float r0_n = 0.f, r1_n = 0.f, r2_n = 0.f;
    auto load = [&](int ee) {
        const long long at = pd_at(B.index, B.cap, i, ee);
        al_n = B.alive[at];
        j_n = B.ridx[at];
        r0_n = B.rpos[3 * at];
        r1_n = B.rpos[3 * at + 1];
        r2_n = B.rpos[3 * at + 2];
    };
    if (sub < m) load(sub);
    for (int e = sub, k = 0; e < m; e += kPdG, ++k) {
        const bool al = al_n;
        const int j = j_n;
        const float e0 = r0_n - ri0, e1 = r1_n - ri1, e2 = r2_n - ri2;
        if (e + kPdG < m) load(e + kPdG);
        if (stash && k < kPdStash) stash[k][threadIdx.x] = make_float4(e0, e1, e2, __int_as_float(al ? j : ~j));
        if (!al) continue;
        const float r = bond_len(e0, e1, e2);
        if (r > kEpsilon) {
            const float wt = corr_w_f(r, B.inv_h);
            const V3<R> xj = ld3r<R>(x, j);
            const R ih = (R)B.inv_h;
            const R p[3] = {(xj.x - ci.x) * ih, (xj.y - ci.y) * ih, (xj.z - ci.z) * ih};
            const float qs = __fmul_rn(B.inv_h, wt);
            const R q[3] = {(R)(e0 * qs), (R)(e1 * qs), (R)(e2 * qs)};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) F[a][b] += p[a] * q[b];
            tw += wt;
        }
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) F[a][b] = gsum(F[a][b]);
    tw = gsum(tw);
    if (tw > kEpsilon) {
        const R s = (R)1 / (R)tw;
        const float* K = B.invK + 9LL * i;
        R G[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) F[a][b] *= s;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                G[a][b] = F[a][0] * (R)K[b] + F[a][1] * (R)K[3 + b] + F[a][2] * (R)K[6 + b];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) F[a][b] = G[a][b];
    }
    const R det = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                  F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                  F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    ident = det < (R)-0.001;
    if (ident)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) F[a][b] = (a == b) ? (R)1 : (R)0;
    tw_out = tw;
}

// F of every particle; with twout, also tw, stored negated when the identity
// was taken (the reverse pass reads both instead of recomputing them).
template <class R>
__global__ void __launch_bounds__(kPdBlock)
    k_pd_F(PdBonds B, const R* __restrict__ x, R* __restrict__ Fout, float* __restrict__ twout)
{
    const PdLane L = pd_lane(B.n);
    R F[3][3];
    float tw;
    bool ident;
    pd_deformation(B, x, L.i, L.sub, F, tw, ident);
    if (L.valid && L.sub == 0) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Fout[9LL * L.i + 3 * a + b] = F[a][b];
        if (twout) twout[L.i] = ident ? -1.0f - tw : tw;
    }
}

template <class R>
__device__ __forceinline__ V3<R> mat_e(const R* F, float e0, float e1, float e2)
{
    return V3<R>{F[0] * e0 + F[1] * e1 + F[2] * e2, F[3] * e0 + F[4] * e1 + F[5] * e2,
                 F[6] * e0 + F[7] * e1 + F[8] * e2};
}

// W_i (the denominator of K_UpdatePosition): constant while bulk and the bonds are.
template <class R, class RB>
__global__ void __launch_bounds__(kPdBlock) k_pd_W(PdBonds B, const RB* __restrict__ bulk, R* __restrict__ W)
{
    const PdLane L = pd_lane(B.n);
    const int i = L.i;
    const long long a0 = pd_at(B.index, B.cap, i, 0);
    const float ri0 = B.rpos[3 * a0], ri1 = B.rpos[3 * a0 + 1], ri2 = B.rpos[3 * a0 + 2];
    const int m = pd_size(B.index, B.cap, B.total, B.n, i);
    const R ml = (R)B.mu + (R)B.lambda;
    R w = 0;
    for (int e = L.sub; e < m; e += kPdG) {
        const long long at = pd_at(B.index, B.cap, i, e);
        if (!B.alive[at]) continue;
        const float e0 = ri0 - B.rpos[3 * at], e1 = ri1 - B.rpos[3 * at + 1], e2 = ri2 - B.rpos[3 * at + 2];
        const float r = bond_len(e0, e1, e2);
        if (!(r > 0.01f * B.h)) continue;
        w += ml * (R)bulk[i] * (R)corr_wrr_f(r, B.inv_h);
    }
    for (int t = B.in_off[i] + L.sub; t < B.in_off[i + 1]; t += kPdG) {
        const int2 kb = B.in_list[t];
        const long long at = kb.y;
        if (!B.alive[at]) continue;
        const long long k0 = pd_at(B.index, B.cap, kb.x, 0);
        const float e0 = B.rpos[3 * k0] - B.rpos[3 * at], e1 = B.rpos[3 * k0 + 1] - B.rpos[3 * at + 1],
                    e2 = B.rpos[3 * k0 + 2] - B.rpos[3 * at + 2];
        const float r = bond_len(e0, e1, e2);
        if (!(r > 0.01f * B.h)) continue;
        w += ml * (R)bulk[kb.x] * (R)corr_wrr_f(r, B.inv_h);
    }
    w = gsum(w);
    if (L.valid && L.sub == 0) W[i] = w;
}

// One projection iteration: xn = (xold + D(x)) / (1 + W).
template <class R>
__global__ void __launch_bounds__(kPdBlock)
    k_pd_P(PdBonds B, const R* __restrict__ x, const R* __restrict__ xold, const R* __restrict__ F,
           const R* __restrict__ bulk, const R* __restrict__ W, R* __restrict__ xn)
{
    const PdLane L = pd_lane(B.n);
    const int i = L.i;
    const long long a0 = pd_at(B.index, B.cap, i, 0);
    const float ri0 = B.rpos[3 * a0], ri1 = B.rpos[3 * a0 + 1], ri2 = B.rpos[3 * a0 + 2];
    const V3<R> ci = ld3(x, i);
    const int m = pd_size(B.index, B.cap, B.total, B.n, i);
    const R* Fi = F + 9LL * i;
    V3<R> acc{0, 0, 0};
    for (int e = L.sub; e < m; e += kPdG) {
        const long long at = pd_at(B.index, B.cap, i, e);
        if (!B.alive[at]) continue;
        const float e0 = ri0 - B.rpos[3 * at], e1 = ri1 - B.rpos[3 * at + 1], e2 = ri2 - B.rpos[3 * at + 2];
        const float r = bond_len(e0, e1, e2);
        if (!(r > 0.01f * B.h)) continue;
        const V3<R> xj = ld3(x, B.ridx[at]);
        V3<R> nf = mat_e(Fi, e0, e1, e2);
        V3<R> nc{ci.x - xj.x, ci.y - xj.y, ci.z - xj.z};
        unit_fast(nf);
        unit_fast(nc);
        const R wrr = (R)corr_wrr_f(r, B.inv_h), mu = (R)B.mu * bulk[i] * wrr, la = (R)B.lambda * bulk[i] * wrr;
        const R rr = (R)r;
        const V3<R> dj{xj.x - ci.x, xj.y - ci.y, xj.z - ci.z};
        acc.x += mu * (dj.x + rr * nf.x) + la * (dj.x + rr * nc.x);
        acc.y += mu * (dj.y + rr * nf.y) + la * (dj.y + rr * nc.y);
        acc.z += mu * (dj.z + rr * nf.z) + la * (dj.z + rr * nc.z);
    }
    for (int t = B.in_off[i] + L.sub; t < B.in_off[i + 1]; t += kPdG) {
        const int2 kb = B.in_list[t];
        const long long at = kb.y;
        if (!B.alive[at]) continue;
        const int k = kb.x;
        const long long k0 = pd_at(B.index, B.cap, k, 0);
        const float e0 = B.rpos[3 * k0] - B.rpos[3 * at], e1 = B.rpos[3 * k0 + 1] - B.rpos[3 * at + 1],
                    e2 = B.rpos[3 * k0 + 2] - B.rpos[3 * at + 2];
        const float r = bond_len(e0, e1, e2);
        if (!(r > 0.01f * B.h)) continue;
        const V3<R> xk = ld3(x, k);
        V3<R> nf = mat_e(F + 9LL * k, e0, e1, e2);
        V3<R> nc{xk.x - ci.x, xk.y - ci.y, xk.z - ci.z};
        unit_fast(nf);
        unit_fast(nc);
        const R wrr = (R)corr_wrr_f(r, B.inv_h), mu = (R)B.mu * bulk[k] * wrr, la = (R)B.lambda * bulk[k] * wrr;
        const R rr = (R)r;
        const V3<R> dk{xk.x - ci.x, xk.y - ci.y, xk.z - ci.z};
        acc.x += mu * (dk.x - rr * nf.x) + la * (dk.x - rr * nc.x);
        acc.y += mu * (dk.y - rr * nf.y) + la * (dk.y - rr * nc.y);
        acc.z += mu * (dk.z - rr * nf.z) + la * (dk.z - rr * nc.z);
    }
    acc.x = gsum(acc.x);
    acc.y = gsum(acc.y);
    acc.z = gsum(acc.z);
    if (!L.valid || L.sub != 0) return;
    // (x_old + D)/(1 + W) written about x_i: the bond targets enter as offsets
    // from x_i, which keeps float accuracy at the scale of the bonds instead of
    // the scale of the coordinates
    const R den = (R)1 + W[i];
    const V3<R> xo = ld3(xold, i);
    xn[3 * i] = ci.x + ((xo.x - ci.x) + acc.x) / den;
    xn[3 * i + 1] = ci.y + ((xo.y - ci.y) + acc.y) / den;
    xn[3 * i + 2] = ci.z + ((xo.z - ci.z) + acc.z) / den;
}

// The projection with each bond's term formed once.  A bond i->j's term in
// D_j (the incoming sum above, seen from j) uses F_i, x_i, x_j and the rest
// vector of i's shape, exactly like its term in D_i with the sign flipped:
// mu (x_i - x_j - r n(F_i e)) + la (x_i - x_j - r n(x_i - x_j)) = -t_ij.  So
// k_pd_FP computes F_i and every outgoing t_ij of particle i, keeps the sum
// in own[i] and each t_ij in its bond slot (0 for a dead or too-short bond),
// and k_pd_gather sums -t over the incoming slots: no neighbour F is
// gathered and no bond is evaluated twice.  k_pd_FP's two walks over a
// particle's bonds (F, then the terms) read the rest shape once: the first
// keeps each lane's bonds in shared memory for the second.
template <class R>
__global__ void __launch_bounds__(kPdBlock)
    k_pd_FP(PdBonds B, const R* __restrict__ x, const R* __restrict__ bulk, R* __restrict__ Fout,
            float* __restrict__ twout, R* __restrict__ own, R* __restrict__ tslot)
{
    // the first walk's bonds, read again by the second from shared memory
    // instead of from the rest shape in DRAM
    __shared__ float4 stash[kPdStash][kPdBlock];
    const PdLane L = pd_lane(B.n);
    const int i = L.i;
    R Fi[3][3];
    float tw;
    bool ident;
    pd_deformation(B, x, i, L.sub, Fi, tw, ident, stash);
    if (L.valid && L.sub == 0) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Fout[9LL * i + 3 * a + b] = Fi[a][b];
        if (twout) twout[i] = ident ? -1.0f - tw : tw;
    }
    const long long a0 = pd_at(B.index, B.cap, i, 0);
    const float ri0 = B.rpos[3 * a0], ri1 = B.rpos[3 * a0 + 1], ri2 = B.rpos[3 * a0 + 2];
    const V3<R> ci = ld3(x, i);
    const int m = pd_size(B.index, B.cap, B.total, B.n, i);
    V3<R> acc{0, 0, 0};
    R accw = 0;  // the particle's own bond weights (W, the target's share is in the slots)
    const R ml = (R)B.mu + (R)B.lambda;
    for (int e = L.sub, k = 0; e < m; e += kPdG, ++k) {
        const long long at = pd_at(B.index, B.cap, i, e);
        V3<R> t{0, 0, 0};
        R wb = 0;
        bool al;
        int j;
        float e0, e1, e2;
        if (k < kPdStash) {
            const float4 q = stash[k][threadIdx.x];
            const int jv = __float_as_int(q.w);
            al = jv >= 0;
            j = al ? jv : ~jv;
            e0 = -q.x;  // the stash holds rest_j - rest_i
            e1 = -q.y;
            e2 = -q.z;
        } else {
            al = B.alive[at];
            j = B.ridx[at];
            e0 = ri0 - B.rpos[3 * at];
            e1 = ri1 - B.rpos[3 * at + 1];
            e2 = ri2 - B.rpos[3 * at + 2];
        }
        const float r = bond_len(e0, e1, e2);
        if (al && r > 0.01f * B.h) {
            const V3<R> xj = ld3(x, j);
            V3<R> nf = V3<R>{Fi[0][0] * e0 + Fi[0][1] * e1 + Fi[0][2] * e2, Fi[1][0] * e0 + Fi[1][1] * e1 + Fi[1][2] * e2,
                             Fi[2][0] * e0 + Fi[2][1] * e1 + Fi[2][2] * e2};
            V3<R> nc{ci.x - xj.x, ci.y - xj.y, ci.z - xj.z};
            unit_fast(nf);
            unit_fast(nc);
            const R wrr = (R)corr_wrr_f(r, B.inv_h), mu = (R)B.mu * bulk[i] * wrr, la = (R)B.lambda * bulk[i] * wrr;
            const R rr = (R)r;
            const V3<R> dj{xj.x - ci.x, xj.y - ci.y, xj.z - ci.z};
            t = V3<R>{mu * (dj.x + rr * nf.x) + la * (dj.x + rr * nc.x), mu * (dj.y + rr * nf.y) + la * (dj.y + rr * nc.y),
                      mu * (dj.z + rr * nf.z) + la * (dj.z + rr * nc.z)};
            acc.x += t.x;
            acc.y += t.y;
            acc.z += t.z;
            wb = ml * bulk[i] * wrr;
            accw += wb;
        }
        if (L.valid) store_slot(tslot + 4 * at, t.x, t.y, t.z, wb);
    }
    acc.x = gsum(acc.x);
    acc.y = gsum(acc.y);
    acc.z = gsum(acc.z);
    accw = gsum(accw);
    if (L.valid && L.sub == 0) {
        own[4 * i] = acc.x;
        own[4 * i + 1] = acc.y;
        own[4 * i + 2] = acc.z;
        own[4 * i + 3] = accw;
    }
}

// xn = (xold + own - sum of the incoming bond terms) / (1 + W), written about x_i,
// W = the particle's own bond weights + those of the bonds naming it (each
// bond's weight, ml bulk_source wrr, rides in its slot's fourth value, so W
// follows broken bonds and changed stiffness without a pass of its own).
template <class R>
__global__ void __launch_bounds__(kPdBlock)
    k_pd_gather(PdBonds B, const R* __restrict__ x, const R* __restrict__ xold, const R* __restrict__ own,
                const R* __restrict__ tslot, R* __restrict__ xn)
{
    const PdLane L = pd_lane(B.n);
    const int i = L.i;
    V3<R> in{0, 0, 0};
    R win = 0;
    const int t1 = B.in_off[i + 1];
    int t = B.in_off[i] + L.sub;
    int slot_n = t < t1 ? B.in_slot[t] : 0;  // the next incoming slot, one bond ahead
    for (; t < t1; t += kPdG) {
        const R* g = tslot + 4 * (long long)slot_n;
        if (t + kPdG < t1) slot_n = B.in_slot[t + kPdG];
        add_slot(g, in.x, in.y, in.z, win);
    }
    in.x = gsum(in.x);
    in.y = gsum(in.y);
    in.z = gsum(in.z);
    win = gsum(win);
    if (!L.valid || L.sub != 0) return;
    const V3<R> ci = ld3(x, i), xo = ld3(xold, i);
    const V3<R> oi{own[4LL * i], own[4LL * i + 1], own[4LL * i + 2]};
    const R den = (R)1 + (own[4LL * i + 3] + win);
    xn[3 * i] = ci.x + ((xo.x - ci.x) + (oi.x - in.x)) / den;
    xn[3 * i + 1] = ci.y + ((xo.y - ci.y) + (oi.y - in.y)) / den;
    xn[3 * i + 2] = ci.z + ((xo.z - ci.z) + (oi.z - in.z)) / den;
}

// ---- adjoint of one iteration

// a = g/(1+W); xoldbar += a.
template <class R>
__global__ void __launch_bounds__(256)
    k_pd_adjA(int n, const R* __restrict__ g, const R* __restrict__ W, R* __restrict__ a, R* __restrict__ xoldbar)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const R den = (R)1 + W[i];
    const V3<R> gi = ld3(g, i);
    const V3<R> ai{gi.x / den, gi.y / den, gi.z / den};
    a[3 * i] = ai.x;
    a[3 * i + 1] = ai.y;
    a[3 * i + 2] = ai.z;
    xoldbar[3 * i] += ai.x;
    xoldbar[3 * i + 1] += ai.y;
    xoldbar[3 * i + 2] += ai.z;
}

// Reverse pass of one projection iteration, per source particle i (8 lanes):
// the first walk over i's bonds forms F-bar_i (through the normalisation
// Jacobian of n(F e)) and the stiffness gradient of bulk_i; every lane of the
// group then forms G_i = dL/dF_raw / (tw h) (0 when the identity was taken);
// the second walk forms dL/dx.  A bond k->i contributes to dL/dx_i through
// F_k and the n(x_k - x_i) term, and that contribution is formed by the
// source k, which holds G_k, x_k, a_k and the bond's rest vector: G_k q +
// dw a_k - u, u the normalisation adjoint of n(x_k - x_i), the same u as in
// k's own term.  k keeps its own sum in gown[k] and the partner terms in the
// bond slots, which k_pd_adjC_gather adds.  The second walk reads the first
// walk's bonds from shared memory; G never goes through global memory.
// Two kernels (F-bar/G, then dL/dx) at register caps of 80 and 64 took 799 ms
// for the 200-step backward of the 65,536-particle block; this one at 124
// registers (4 blocks per SM, no spills) 694 ms, at 96 711 ms, at 80 742 ms.
#ifndef PK_ADJBC_MINB
#define PK_ADJBC_MINB 4
#endif
template <class R, class RX>
__global__ void __launch_bounds__(kPdBlock, PK_ADJBC_MINB)
    k_pd_adjBC(PdBonds B, const RX* __restrict__ x, const RX* __restrict__ xn, const RX* __restrict__ bulk,
               const RX* __restrict__ Fst, const float* __restrict__ twst, const R* __restrict__ a,
               double* __restrict__ bulkbar, R* __restrict__ gown, R* __restrict__ slot)
{
    __shared__ float4 stash[kPdStash][kPdBlock];  // (rest_i - rest_j, j or ~j for a dead bond)
    const PdLane L = pd_lane(B.n);
    const int i = L.i;
    const long long a0 = pd_at(B.index, B.cap, i, 0);
    const float ri0 = B.rpos[3 * a0], ri1 = B.rpos[3 * a0 + 1], ri2 = B.rpos[3 * a0 + 2];
    const V3<R> ci = ld3r<R>(x, i), ai = ld3(a, i);
    const R bulk_i = (R)bulk[i];
    const int m = pd_size(B.index, B.cap, B.total, B.n, i);
    R Gi[9];
    {
        // the forward's F of this iterate, and its tw (negated: identity taken)
        R F[3][3];
        for (int p = 0; p < 3; ++p)
            for (int q = 0; q < 3; ++q) F[p][q] = (R)Fst[9LL * i + 3 * p + q];
        const V3<R> yi = ld3r<R>(xn, i);
        R Fb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        R gb = 0;  // d L / d bulk_i
        for (int e = L.sub, k = 0; e < m; e += kPdG, ++k) {
            const long long at = pd_at(B.index, B.cap, i, e);
            const bool al = B.alive[at];
            const int j = B.ridx[at];
            const float e0 = ri0 - B.rpos[3 * at], e1 = ri1 - B.rpos[3 * at + 1], e2 = ri2 - B.rpos[3 * at + 2];
            if (k < kPdStash) stash[k][threadIdx.x] = make_float4(e0, e1, e2, __int_as_float(al ? j : ~j));
            if (!al) continue;
            const float r = bond_len(e0, e1, e2);
            if (!(r > 0.01f * B.h)) continue;
            const V3<R> xj = ld3r<R>(x, j), aj = ld3(a, j);
            V3<R> nf{F[0][0] * e0 + F[0][1] * e1 + F[0][2] * e2, F[1][0] * e0 + F[1][1] * e1 + F[1][2] * e2,
                     F[2][0] * e0 + F[2][1] * e1 + F[2][2] * e2};
            V3<R> nc{ci.x - xj.x, ci.y - xj.y, ci.z - xj.z};
            const R lf = unit_or_zero(nf);
            unit_or_zero(nc);
            const R wrr = (R)corr_wrr_f(r, B.inv_h), rr = (R)r;
            const R mu = (R)B.mu * bulk_i * wrr;
            const V3<R> da{ai.x - aj.x, ai.y - aj.y, ai.z - aj.z};
            const V3<R> ub = unit_vjp(nf, lf, V3<R>{mu * rr * da.x, mu * rr * da.y, mu * rr * da.z});
            const R ev[3] = {(R)e0, (R)e1, (R)e2};
            const R ubv[3] = {ub.x, ub.y, ub.z};
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) Fb[p][q] += ubv[p] * ev[q];
            const V3<R> yj = ld3r<R>(xn, j);
            const R tmu = dot3(ai, V3<R>{xj.x + rr * nf.x - yi.x, xj.y + rr * nf.y - yi.y, xj.z + rr * nf.z - yi.z}) +
                          dot3(aj, V3<R>{ci.x - rr * nf.x - yj.x, ci.y - rr * nf.y - yj.y, ci.z - rr * nf.z - yj.z});
            const R tla = dot3(ai, V3<R>{xj.x + rr * nc.x - yi.x, xj.y + rr * nc.y - yi.y, xj.z + rr * nc.z - yi.z}) +
                          dot3(aj, V3<R>{ci.x - rr * nc.x - yj.x, ci.y - rr * nc.y - yj.y, ci.z - rr * nc.z - yj.z});
            gb += wrr * ((R)B.mu * tmu + (R)B.lambda * tla);
        }
        for (int p = 0; p < 3; ++p)
            for (int q = 0; q < 3; ++q) Fb[p][q] = gsum(Fb[p][q]);
        gb = gsum(gb);
        if (L.valid && L.sub == 0) bulkbar[i] += (double)gb;
        // G = dL/dF_raw / (tw h): F = (F_raw / tw) K, so dL/dF_raw = F-bar K^T / tw
        const float tws = twst[i];
        const bool ident = tws < 0.f;
        const float tw = ident ? -1.0f - tws : tws;
        for (int q = 0; q < 9; ++q) Gi[q] = 0;
        if (!ident) {
            if (tw > kEpsilon) {
                const float* K = B.invK + 9LL * i;
                const R sc = (R)1 / ((R)tw * (R)B.h);
                for (int p = 0; p < 3; ++p)
                    for (int c = 0; c < 3; ++c)
                        Gi[3 * p + c] = (Fb[p][0] * (R)K[3 * c] + Fb[p][1] * (R)K[3 * c + 1] + Fb[p][2] * (R)K[3 * c + 2]) * sc;
            } else {
                const R sc = (R)1 / (R)B.h;
                for (int p = 0; p < 3; ++p)
                    for (int c = 0; c < 3; ++c) Gi[3 * p + c] = Fb[p][c] * sc;
            }
        }
    }
    const R ml = (R)B.mu + (R)B.lambda;
    V3<R> out{0, 0, 0};
    for (int e = L.sub, k = 0; e < m; e += kPdG, ++k) {
        const long long at = pd_at(B.index, B.cap, i, e);
        bool al;
        int j;
        float f0, f1, f2;  // rest_j - rest_i
        if (k < kPdStash) {
            const float4 q = stash[k][threadIdx.x];
            const int jv = __float_as_int(q.w);
            al = jv >= 0;
            j = al ? jv : ~jv;
            f0 = -q.x;
            f1 = -q.y;
            f2 = -q.z;
        } else {
            al = B.alive[at];
            j = B.ridx[at];
            f0 = B.rpos[3 * at] - ri0;
            f1 = B.rpos[3 * at + 1] - ri1;
            f2 = B.rpos[3 * at + 2] - ri2;
        }
        V3<R> pt{0, 0, 0};  // the term for the bond's target
        if (al) {
            const float r = bond_len(f0, f1, f2);
            // F_i depends on x_i through -(x_i)/h q and on x_j through +(x_j)/h q
            if (r > kEpsilon) {
                const float wt = corr_w_f(r, B.inv_h);
                const float qs = __fmul_rn(B.inv_h, wt);
                const R q0 = (R)(f0 * qs), q1 = (R)(f1 * qs), q2 = (R)(f2 * qs);
                const V3<R> gq{Gi[0] * q0 + Gi[1] * q1 + Gi[2] * q2, Gi[3] * q0 + Gi[4] * q1 + Gi[5] * q2,
                               Gi[6] * q0 + Gi[7] * q1 + Gi[8] * q2};
                out.x -= gq.x;
                out.y -= gq.y;
                out.z -= gq.z;
                pt = gq;
            }
            if (r > 0.01f * B.h) {
                const V3<R> xj = ld3r<R>(x, j), aj = ld3(a, j);
                V3<R> nc{ci.x - xj.x, ci.y - xj.y, ci.z - xj.z};
                const R lc = unit_or_zero(nc);
                const R wrr = (R)corr_wrr_f(r, B.inv_h), rr = (R)r;
                const R la = (R)B.lambda * bulk_i * wrr, dw = ml * bulk_i * wrr;
                const V3<R> uc =
                    unit_vjp(nc, lc, V3<R>{la * rr * (ai.x - aj.x), la * rr * (ai.y - aj.y), la * rr * (ai.z - aj.z)});
                out.x += dw * aj.x + uc.x;
                out.y += dw * aj.y + uc.y;
                out.z += dw * aj.z + uc.z;
                pt.x += dw * ai.x - uc.x;
                pt.y += dw * ai.y - uc.y;
                pt.z += dw * ai.z - uc.z;
            }
        }
        if (L.valid) store_slot(slot + 4 * at, pt.x, pt.y, pt.z);
    }
    out.x = gsum(out.x);
    out.y = gsum(out.y);
    out.z = gsum(out.z);
    if (!L.valid || L.sub != 0) return;
    gown[3 * i] = out.x;
    gown[3 * i + 1] = out.y;
    gown[3 * i + 2] = out.z;
}

template <class R>
__global__ void __launch_bounds__(kPdBlock)
    k_pd_adjC_gather(PdBonds B, const R* __restrict__ gown, const R* __restrict__ slot, R* __restrict__ gout)
{
    const PdLane L = pd_lane(B.n);
    const int i = L.i;
    V3<R> in{0, 0, 0};
    for (int t = B.in_off[i] + L.sub; t < B.in_off[i + 1]; t += kPdG) {
        add_slot(slot + 4 * (long long)B.in_slot[t], in.x, in.y, in.z);
    }
    in.x = gsum(in.x);
    in.y = gsum(in.y);
    in.z = gsum(in.z);
    if (!L.valid || L.sub != 0) return;
    gout[3 * i] = gown[3 * i] + in.x;
    gout[3 * i + 1] = gown[3 * i + 1] + in.y;
    gout[3 * i + 2] = gown[3 * i + 2] + in.z;
}

// ---- step pieces

template <class R>
__global__ void __launch_bounds__(256)
    k_pd_integrate(int n, R* __restrict__ x, R* __restrict__ v, R gx, R gy, R gz, R dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const R g[3] = {gx, gy, gz};
    for (int c = 0; c < 3; ++c) {
        const R vv = v[3 * i + c] + dt * g[c];
        v[3 * i + c] = vv;
        x[3 * i + c] = x[3 * i + c] + dt * vv;
    }
}

template <class R>
__global__ void __launch_bounds__(256)
    k_pd_vel(long long m, R* __restrict__ v, const R* __restrict__ x, const R* __restrict__ xold, R dt)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) v[t] += (x[t] - xold[t]) / dt;
}

// Start of a step's reverse: g = xbar + vbar/dt (x_new feeds v_new), xoldbar = -vbar/dt.
template <class R>
__global__ void __launch_bounds__(256)
    k_pd_adj_head(long long m, const R* __restrict__ xbar, const R* __restrict__ vbar, R dt, R* __restrict__ g,
                  R* __restrict__ xoldbar)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    g[t] = xbar[t] + vbar[t] / dt;
    xoldbar[t] = -vbar[t] / dt;
}

// End of a step's reverse: xbar' = g + xoldbar (x' is both x_0 and x_old),
// then through x' = x + dt v', v' = v + dt gravity: vbar += dt xbar', xbar = xbar'.
template <class R>
__global__ void __launch_bounds__(256)
    k_pd_adj_tail(long long m, const R* __restrict__ g, const R* __restrict__ xoldbar, R dt, R* __restrict__ xbar,
                  R* __restrict__ vbar)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const R xb = g[t] + xoldbar[t];
    xbar[t] = xb;
    vbar[t] += dt * xb;
}

// ---- incoming bonds (transpose of the frozen rest shape)

__global__ void __launch_bounds__(256)
    k_in_count(int n, const int* __restrict__ index, int cap, long long total, const int* __restrict__ ridx,
               int* __restrict__ cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = pd_size(index, cap, total, n, i);
    for (int e = 1; e < m; ++e) {  // slot 0 is the particle itself
        const int j = ridx[pd_at(index, cap, i, e)];
        if (j != i && j >= 0 && j < n) atomicAdd(cnt + j, 1);
    }
}

__global__ void __launch_bounds__(256)
    k_in_fill(int n, const int* __restrict__ index, int cap, long long total, const int* __restrict__ ridx,
              const int* __restrict__ off, int* __restrict__ fill, int2* __restrict__ list)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = pd_size(index, cap, total, n, i);
    for (int e = 1; e < m; ++e) {
        const long long at = pd_at(index, cap, i, e);
        const int j = ridx[at];
        if (j != i && j >= 0 && j < n) list[off[j] + atomicAdd(fill + j, 1)] = make_int2(i, (int)at);
    }
}

// Each particle's incoming bonds in ascending bond slot (a fixed order).  A
// warp per particle: lists of up to 128 entries are held 4 per lane and each
// entry goes to its rank (slots are distinct within a list); longer lists are
// sorted by lane 0 in place.
constexpr int kInSortWarps = 8;
__global__ void __launch_bounds__(kInSortWarps * 32)
    k_in_sort(int n, const int* __restrict__ off, int2* __restrict__ list)
{
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kInSortWarps + (threadIdx.x >> 5);
    if (i >= n) return;  // the whole warp leaves together
    const int o = off[i], m = off[i + 1] - o;
    if (m <= 128) {
        int2 v[4];
        int rank[4] = {0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = 32 * q + lane < m ? list[o + 32 * q + lane] : make_int2(0, 0x7fffffff);
#pragma unroll
        for (int sq = 0; sq < 4; ++sq)
            for (int sl = 0; sl < 32; ++sl) {
                const int w = __shfl_sync(0xffffffffu, v[sq].y, sl);
#pragma unroll
                for (int q = 0; q < 4; ++q) rank[q] += w < v[q].y ? 1 : 0;
            }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (32 * q + lane < m) list[o + rank[q]] = v[q];
        return;
    }
    if (lane != 0) return;
    for (int a = o + 1; a < o + m; ++a) {
        const int2 v = list[a];
        int b = a - 1;
        while (b >= o && list[b].y > v.y) {
            list[b + 1] = list[b];
            --b;
        }
        list[b + 1] = v;
    }
}

// Precision conversions of the adjoint state (the adjoint runs in double).
template <class RO, class RI>
__global__ void __launch_bounds__(256) k_convert(long long m, const RI* __restrict__ in, RO* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) out[t] = in ? (RO)in[t] : (RO)0;
}

// ---------------------------------------------------------------- host side

static unsigned pd_groups_blocks(int n) { return (unsigned)(((long long)n * kPdG + kPdBlock - 1) / kPdBlock); }

// Forward state in R (float or double); the reverse state always in double:
// the adjoint differences neighbouring values (a_i - a_j, x_i - x_j) and
// sums over ~80 bonds per particle, 10 iterations per step, which float
// arithmetic does not carry over a long rollout.
template <class R>
struct PdWork {
    int cap_n = 0;
    R *F = nullptr, *W = nullptr, *xold = nullptr, *xa = nullptr, *vr = nullptr, *bulk = nullptr;
    R* own = nullptr;       // 4 per particle: the sum of its outgoing bond terms and of their weights
    R* tslot = nullptr;     // 4 per bond slot: the bond's term
    long long tslot_cap = 0;
    double* gown = nullptr;   // reverse pass: 3 per particle
    double* aslot = nullptr;  // reverse pass: 4 per bond slot
    long long aslot_cap = 0;
    double *a = nullptr, *g = nullptr, *xoldbar = nullptr, *xb = nullptr,
           *vb = nullptr, *Wa = nullptr, *bulkbar = nullptr;
    // rollout record
    int steps = 0, every = 0, n = 0;
    R gravity[3] = {0, 0, 0};
    float dt = 0.f;
    int iterations = 0;
    R* ckpt = nullptr;  // (x, v) at the start of every segment
    long long ckpt_cap = 0;
    R* seg = nullptr;   // iterates of one segment: every * (iterations + 1) * 3n
    long long seg_cap = 0;
    R* segF = nullptr;  // F of every iterate of a segment: every * iterations * 9n
    long long segF_cap = 0;
    float* segT = nullptr;  // tw of every iterate (negated: identity taken)
    long long segT_cap = 0;
};

template <class R>
static bool grow(R*& p, long long& cap, long long want)
{
    if (want <= cap) return true;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc((void**)&p, sizeof(R) * (size_t)std::max(want, 1LL)) != cudaSuccess) return false;
    cap = want;
    return true;
}

template <class T>
static bool realloc_n(T*& p, size_t count)
{
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc((void**)&p, sizeof(T) * std::max(count, (size_t)1)) == cudaSuccess;
}

template <class R>
static bool work_alloc(PdWork<R>& w, int n)
{
    if (n <= w.cap_n) return true;
    const size_t m = (size_t)n;
    bool ok = realloc_n(w.F, 9 * m) && realloc_n(w.W, m) && realloc_n(w.xold, 3 * m) && realloc_n(w.own, 4 * m) &&
              realloc_n(w.gown, 3 * m) &&
              realloc_n(w.xa, 3 * m) && realloc_n(w.vr, 3 * m) && realloc_n(w.bulk, m) &&
              realloc_n(w.a, 3 * m) && realloc_n(w.g, 3 * m) &&
              realloc_n(w.xoldbar, 3 * m) && realloc_n(w.xb, 3 * m) && realloc_n(w.vb, 3 * m) &&
              realloc_n(w.Wa, m) && realloc_n(w.bulkbar, m);
    if (!ok) return false;
    w.cap_n = n;
    return true;
}

template <class R>
static void work_free(PdWork<R>* w)
{
    if (!w) return;
    void* ps[] = {w->F, w->W, w->xold, w->xa, w->vr, w->bulk, w->own, w->tslot, w->gown, w->aslot, w->a,
                  w->g, w->xoldbar,
                  w->xb, w->vb, w->Wa, w->bulkbar, w->ckpt, w->seg, w->segF, w->segT};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete w;
}

static PdBonds bonds_of(pk_ctx* c, float horizon, float mu, float lambda)
{
    PdBonds B;
    B.index = c->pd_index;
    B.cap = c->pd_cap;
    B.total = c->pd_total;
    B.n = c->pd_n;
    B.ridx = c->pd_rest_idx;
    B.rpos = c->pd_rest_pos;
    B.alive = c->pd_alive;
    B.invK = c->pd_invK;
    B.in_off = c->pd_in_off;
    B.in_list = c->pd_in;
    B.in_slot = c->pd_in_slot;
    B.h = horizon;
    B.mu = mu;
    B.lambda = lambda;
    B.inv_h = 1.0f / horizon;
    return B;
}

template <class R>
static PdWork<R>*& work_of(pk_ctx* c);
template <>
PdWork<float>*& work_of<float>(pk_ctx* c)
{
    return reinterpret_cast<PdWork<float>*&>(c->pd_work32);
}
template <>
PdWork<double>*& work_of<double>(pk_ctx* c)
{
    return reinterpret_cast<PdWork<double>*&>(c->pd_work64);
}

void pd_work_release(pk_ctx* c)
{
    work_free(reinterpret_cast<PdWork<float>*>(c->pd_work32));
    work_free(reinterpret_cast<PdWork<double>*>(c->pd_work64));
    c->pd_work32 = c->pd_work64 = nullptr;
}

template <class R>
static PdWork<R>* ensure_work(pk_ctx* c, int n)
{
    PdWork<R>*& w = work_of<R>(c);
    if (!w) w = new PdWork<R>();
    if (!work_alloc(*w, n)) return nullptr;
    if (!grow(w->tslot, w->tslot_cap, 4 * std::max(c->pd_total, 1LL))) return nullptr;
    if (!grow(w->aslot, w->aslot_cap, 4 * std::max(c->pd_total, 1LL))) return nullptr;
    return w;
}

// The slots of the incoming lists as their own array: the gathers read 4
// bytes per incoming bond instead of the 8-byte (source, slot) pair.
__global__ void __launch_bounds__(256) k_in_slots(const int* __restrict__ total, const int2* __restrict__ list,
                                                  int* __restrict__ slots)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < *total) slots[t] = list[t].y;
}

// Builds the incoming-bond lists of the frozen rest shape (once per pd_init).
int pd_build_incoming(pk_ctx* c, cudaStream_t st)
{
    const int n = c->pd_n;
    const unsigned nb = (unsigned)((n + 255) / 256);
    cudaMemsetAsync(c->pd_in_cnt, 0, sizeof(int) * (size_t)(n + 1), st);
    k_in_count<<<nb, 256, 0, st>>>(n, c->pd_index, c->pd_cap, c->pd_total, c->pd_rest_idx, c->pd_in_cnt);
    exclusive_scan(c->pd_in_cnt, n, c->pd_in_off, c->scan_part, st);
    cudaMemsetAsync(c->pd_in_cnt, 0, sizeof(int) * (size_t)(n + 1), st);
    k_in_fill<<<nb, 256, 0, st>>>(n, c->pd_index, c->pd_cap, c->pd_total, c->pd_rest_idx, c->pd_in_off,
                                  c->pd_in_cnt, c->pd_in);
    k_in_sort<<<(unsigned)((n + kInSortWarps - 1) / kInSortWarps), kInSortWarps * 32, 0, st>>>(n, c->pd_in_off,
                                                                                           c->pd_in);
    const long long nin = std::max(c->pd_total, 1LL);
    k_in_slots<<<(unsigned)((nin + 255) / 256), 256, 0, st>>>(c->pd_in_off + n, c->pd_in, c->pd_in_slot);
    return 5 + scan_launches();
}

// One projection solve (iterations of F + P), x in place; x_old = x on entry
// (kept in w.xold).
template <class R>
static int project(PdWork<R>& w, const PdBonds& B, R* x, const R* bulk, int iterations, cudaStream_t st)
{
    const int n = B.n;
    const unsigned nb128 = pd_groups_blocks(n);
    const size_t bytes = sizeof(R) * 3 * (size_t)n;
    cudaMemcpyAsync(w.xold, x, bytes, cudaMemcpyDeviceToDevice, st);
    R* cur = x;
    R* nxt = w.xa;
    for (int it = 0; it < iterations; ++it) {
        k_pd_FP<R><<<nb128, kPdBlock, 0, st>>>(B, cur, bulk, w.F, nullptr, w.own, w.tslot);
        k_pd_gather<R><<<nb128, kPdBlock, 0, st>>>(B, cur, w.xold, w.own, w.tslot, nxt);
        R* t = cur;
        cur = nxt;
        nxt = t;
    }
    if (cur != x) cudaMemcpyAsync(x, cur, bytes, cudaMemcpyDeviceToDevice, st);
    return 2 * iterations;
}

// pk_pd_solve's projection on the gather form (float, alive mask honoured).
int pd_project_solve(pk_ctx* c, float* x, float* v, int n, float horizon, float mu, float lambda, int iterations,
                     float dt, cudaStream_t st)
{
    PdWork<float>* w = ensure_work<float>(c, n);
    if (!w) return -1;
    const PdBonds B = bonds_of(c, horizon, mu, lambda);
    int l = project<float>(*w, B, x, c->pd_bulk, iterations, st);
    const long long m3 = 3LL * n;
    k_pd_vel<float><<<(unsigned)((m3 + 255) / 256), 256, 0, st>>>(m3, v, x, w->xold, dt);
    return l + 1;
}

// The projection one step at a time (pk_pd_begin / pk_pd_enforce /
// pk_pd_update_velocity): x_old is kept in the float workspace between the
// calls (the bond weights come with every iteration's bond terms).
int pd_begin(pk_ctx* c, const float* x, int n, float /*horizon*/, float /*mu*/, float /*lambda*/, cudaStream_t st)
{
    PdWork<float>* w = ensure_work<float>(c, n);
    if (!w) return -1;
    if (n <= 0) return 0;
    cudaMemcpyAsync(w->xold, x, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, st);
    return 0;
}

int pd_enforce(pk_ctx* c, float* x, int n, float horizon, float mu, float lambda, cudaStream_t st)
{
    PdWork<float>* w = work_of<float>(c);
    if (!w || w->cap_n < n) return -1;
    if (n <= 0) return 0;
    const PdBonds B = bonds_of(c, horizon, mu, lambda);
    const unsigned nb128 = pd_groups_blocks(n);
    k_pd_FP<float><<<nb128, kPdBlock, 0, st>>>(B, x, c->pd_bulk, w->F, nullptr, w->own, w->tslot);
    k_pd_gather<float><<<nb128, kPdBlock, 0, st>>>(B, x, w->xold, w->own, w->tslot, w->xa);
    cudaMemcpyAsync(x, w->xa, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, st);
    return 2;
}

int pd_update_velocity(pk_ctx* c, const float* x, float* v, int n, float dt, cudaStream_t st)
{
    PdWork<float>* w = work_of<float>(c);
    if (!w || w->cap_n < n) return -1;
    if (n <= 0) return 0;
    const long long m3 = 3LL * n;
    k_pd_vel<float><<<(unsigned)((m3 + 255) / 256), 256, 0, st>>>(m3, v, x, w->xold, dt);
    return 1;
}

template <class R>
static int rollout(pk_ctx* c, R* x, R* v, const R* bulk_in, int n, const R g[3], const pk_pd_params* p, int steps,
                   int every, cudaStream_t st)
{
    if (n <= 0) return 0;
    PdWork<R>* w = ensure_work<R>(c, n);
    if (!w) return -1;
    const PdBonds B = bonds_of(c, p->horizon, p->mu, p->lambda);
    const size_t bytes = sizeof(R) * 3 * (size_t)n;
    cudaMemcpyAsync(w->bulk, bulk_in, sizeof(R) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    const int nseg = every > 0 ? (steps + every - 1) / every : 0;
    if (every > 0) {
        if (!grow(w->ckpt, w->ckpt_cap, 6LL * n * std::max(nseg, 1))) return -1;
        if (!grow(w->seg, w->seg_cap, 3LL * n * (p->iterations + 1) * every)) return -1;
        if (!grow(w->segF, w->segF_cap, 9LL * n * std::max(p->iterations, 1) * every)) return -1;
        if (!grow(w->segT, w->segT_cap, 1LL * n * std::max(p->iterations, 1) * every)) return -1;
    }
    w->steps = steps;
    w->every = every;
    w->n = n;
    w->dt = p->dt;
    w->iterations = p->iterations;
    for (int a = 0; a < 3; ++a) w->gravity[a] = g[a];
    const unsigned nb = (unsigned)((n + 255) / 256);
    const long long m3 = 3LL * n;
    int l = 0;
    for (int s = 0; s < steps; ++s) {
        if (every > 0 && s % every == 0) {
            R* ck = w->ckpt + 6LL * n * (s / every);
            cudaMemcpyAsync(ck, x, bytes, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(ck + 3LL * n, v, bytes, cudaMemcpyDeviceToDevice, st);
        }
        k_pd_integrate<R><<<nb, 256, 0, st>>>(n, x, v, g[0], g[1], g[2], (R)p->dt);
        l += 1 + project<R>(*w, B, x, w->bulk, p->iterations, st);
        k_pd_vel<R><<<(unsigned)((m3 + 255) / 256), 256, 0, st>>>(m3, v, x, w->xold, (R)p->dt);
        ++l;
    }
    return l;
}

template <class R>
static int rollout_backward(pk_ctx* c, const R* xbar, const R* vbar, R* gx, R* gv, double* gbulk, cudaStream_t st)
{
    PdWork<R>* w = work_of<R>(c);
    if (c->pd_n == 0) return 0;
    if (!w || w->every <= 0 || w->n != c->pd_n) return -1;
    const int n = w->n, iters = w->iterations;
    const PdBonds B = bonds_of(c, c->pd_horizon_last, c->pd_mu_last, c->pd_lambda_last);
    const size_t bytes = sizeof(R) * 3 * (size_t)n;
    const long long m3 = 3LL * n;
    const unsigned nb = (unsigned)((n + 255) / 256), nb128 = pd_groups_blocks(n),
                   nb3 = (unsigned)((m3 + 255) / 256);
    const R dt = (R)w->dt;
    k_convert<double, R><<<nb3, 256, 0, st>>>(m3, xbar, w->xb);
    k_convert<double, R><<<nb3, 256, 0, st>>>(m3, vbar, w->vb);
    cudaMemsetAsync(w->bulkbar, 0, sizeof(double) * (size_t)n, st);
    k_pd_W<double, R><<<nb128, kPdBlock, 0, st>>>(B, w->bulk, w->Wa);
    int l = 3;
    const int nseg = (w->steps + w->every - 1) / w->every;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int s0 = sg * w->every, s1 = std::min(w->steps, s0 + w->every);
        const R* ck = w->ckpt + 6LL * n * sg;
        R* xr = w->xa;
        R* vr = w->vr;
        cudaMemcpyAsync(xr, ck, bytes, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vr, ck + 3LL * n, bytes, cudaMemcpyDeviceToDevice, st);
        // replay the segment, keeping every iterate x_0 .. x_iters (x_0 = x' = x_old)
        for (int s = s0; s < s1; ++s) {
            R* it = w->seg + 3LL * n * (iters + 1) * (s - s0);
            k_pd_integrate<R><<<nb, 256, 0, st>>>(n, xr, vr, w->gravity[0], w->gravity[1], w->gravity[2], dt);
            cudaMemcpyAsync(it, xr, bytes, cudaMemcpyDeviceToDevice, st);
            for (int k = 0; k < iters; ++k) {
                const long long slot = (long long)(s - s0) * iters + k;
                R* Fk = w->segF + 9LL * n * slot;
                k_pd_FP<R><<<nb128, kPdBlock, 0, st>>>(B, it + 3LL * n * k, w->bulk, Fk, w->segT + 1LL * n * slot,
                                                       w->own, w->tslot);
                k_pd_gather<R><<<nb128, kPdBlock, 0, st>>>(B, it + 3LL * n * k, it, w->own, w->tslot,
                                                           it + 3LL * n * (k + 1));
            }
            k_pd_vel<R><<<nb3, 256, 0, st>>>(m3, vr, it + 3LL * n * iters, it, dt);
            cudaMemcpyAsync(xr, it + 3LL * n * iters, bytes, cudaMemcpyDeviceToDevice, st);
            l += 2 + 2 * iters;
        }
        for (int s = s1 - 1; s >= s0; --s) {
            const R* it = w->seg + 3LL * n * (iters + 1) * (s - s0);
            k_pd_adj_head<double><<<nb3, 256, 0, st>>>(m3, w->xb, w->vb, (double)dt, w->g, w->xoldbar);
            for (int k = iters - 1; k >= 0; --k) {
                k_pd_adjA<double><<<nb, 256, 0, st>>>(n, w->g, w->Wa, w->a, w->xoldbar);
                const long long slot = (long long)(s - s0) * iters + k;
                k_pd_adjBC<double, R><<<nb128, kPdBlock, 0, st>>>(B, it + 3LL * n * k, it + 3LL * n * (k + 1), w->bulk,
                                                              w->segF + 9LL * n * slot, w->segT + 1LL * n * slot,
                                                              w->a, w->bulkbar, w->gown, w->aslot);
                k_pd_adjC_gather<double><<<nb128, kPdBlock, 0, st>>>(B, w->gown, w->aslot, w->g);
            }
            k_pd_adj_tail<double><<<nb3, 256, 0, st>>>(m3, w->g, w->xoldbar, (double)dt, w->xb, w->vb);
            l += 2 + 3 * iters;
        }
    }
    k_convert<R, double><<<nb3, 256, 0, st>>>(m3, w->xb, gx);
    k_convert<R, double><<<nb3, 256, 0, st>>>(m3, w->vb, gv);
    cudaMemcpyAsync(gbulk, w->bulkbar, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    return l + 2;
}

int pd_rollout_f32(pk_ctx* c, float* x, float* v, int n, const float g[3], const pk_pd_params* p, int steps,
                   int every, cudaStream_t st)
{
    return rollout<float>(c, x, v, c->pd_bulk, n, g, p, steps, every, st);
}
int pd_rollout_f64(pk_ctx* c, double* x, double* v, const double* bulk, int n, const double g[3],
                   const pk_pd_params* p, int steps, int every, cudaStream_t st)
{
    return rollout<double>(c, x, v, bulk, n, g, p, steps, every, st);
}
int pd_backward_f32(pk_ctx* c, const float* xbar, const float* vbar, float* gx, float* gv, double* gbulk,
                    cudaStream_t st)
{
    return rollout_backward<float>(c, xbar, vbar, gx, gv, gbulk, st);
}
int pd_backward_f64(pk_ctx* c, const double* xbar, const double* vbar, double* gx, double* gv, double* gbulk,
                    cudaStream_t st)
{
    return rollout_backward<double>(c, xbar, vbar, gx, gv, gbulk, st);
}

}  // namespace pk
