// pk_pbd_adj.cu -- differentiable DensityPBD rollouts: checkpointed forward
// frames and hand-written reverse kernels for the Jacobi sweeps.
//
// One frame without boundary or viscosity (PositionBasedFluidModel::step,
// PositionBasedFluidModel.cpp:83-101, less ImplicitViscosity), in the sorted
// order of the frame's neighbour list, which is frozen for the frame:
//   v' = v + dt g,   y_0 = x + dt v'                (ParticleIntegrator.cu:59-112)
//   lambda_i = min(0, -(rho_i - 1000) / D_i)        (K_ComputeLambdas, DensityPBD.cu:46-90)
//     rho_i = sum_{N(i)} m W(r_ij),  S_i = sum_{N(i)} P_ij,
//     D_i = sum_{N(i)} |P_ij|^2 + |S_i|^2 + 0.1
//   y_{t+1,i} = y_{t,i} + 10 sum_j m_ij (lambda_i + lambda_j) P_ij
//                                                   (K_ComputeDisplacement :134-179 and
//                                                    K_UpdatePosition :226-237; m_ij the
//                                                    row multiplicity of the scatter)
//   x' = y_S,   v'' = v' + (y_S - y_0)/dt           (DP_UpdateVelocity :367-378)
// with P_ij = G(r) (y_i - y_j)/r for r > EPSILON, G the spiky "gradient"
// -45/(pi h^3) (1 - r/h)^2 of Kernel.h:48-57.  That G is h times dW/dr of the
// spiky weight W = 15/(pi h^3) (1 - r/h)^3 (Kernel.h:36-46), so the density's
// derivative is P/h.  The reverse of one iteration, given a = dL/dy_{t+1}:
//   lambdabar_i = 10 sum_j m_ij P_ij . (a_i - a_j)
//   rhobar_i = -lambdabar_i / D_i,  Dbar_i = -lambdabar_i lambda_i / D_i
//     (both 0 where the clamp is active)
//   dL/dy_{t,i} = a_i + sum_j J_ij v_ij + (A_ij rhobar_i + B_ij rhobar_j) m P_ij / h
//     v_ij = 10 m_ij (lambda_i + lambda_j)(a_i - a_j)
//            + A_ij 2 Dbar_i (P_ij + S_i) + B_ij 2 Dbar_j (P_ij - S_j)
//     J_ij = dP/dd = G'(r) u u^T + G(r)/r (I - u u^T),  u = (y_i - y_j)/r
// where A_ij = [j in N(i)] and B_ij = [i in N(j)] are the solver row's flags.
// Kernel r1 recomputes rho, S, D, lambda at the iterate and forms lambdabar,
// rhobar, Dbar; kernel r2 gathers the neighbours' values and forms dL/dy_t.
// The reverse state and arithmetic are double; the float rollout's iterates
// are read as given.
#include <algorithm>

#include "pk_kernels.cuh"

namespace pk {

namespace {

constexpr double kAdjEps2 = 1e-12;  // r > EPSILON (1e-6), cuda_utilities.h:30
constexpr int kAdjBlock = 128;

struct AdjK {
    double inv_h, cw, cg, m;  // W = cw (1-q)^3, G = cg (1-q)^2 = h dW/dr, G' = -2 cg (1-q)/h
};

__device__ __forceinline__ double3 ld3(const float4* p, long long s)
{
    const float4 q = __ldg(p + s);
    return make_double3(q.x, q.y, q.z);
}
__device__ __forceinline__ double3 ld3(const double4* p, long long s)
{
    const double4 q = p[s];
    return make_double3(q.x, q.y, q.z);
}
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 sub3(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }

// ---- forward in double (the reference run of the gradient checks)

__global__ void __launch_bounds__(256) k64_round(const double* __restrict__ x, long long m, float* __restrict__ xf)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) xf[t] = (float)x[t];
}

__global__ void __launch_bounds__(256)
    k64_begin(const double* __restrict__ x, const double* __restrict__ v, const int* __restrict__ perm, int n,
              double gx, double gy, double gz, double dt, double4* __restrict__ y0, double4* __restrict__ vp)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long i = perm[s];
    const double vx = v[3 * i] + dt * gx, vy = v[3 * i + 1] + dt * gy, vz = v[3 * i + 2] + dt * gz;
    vp[s] = make_double4(vx, vy, vz, 0.0);
    y0[s] = make_double4(x[3 * i] + dt * vx, x[3 * i + 1] + dt * vy, x[3 * i + 2] + dt * vz, 0.0);
}

__global__ void __launch_bounds__(kAdjBlock, 4)
    k64_pass_a(const double4* __restrict__ y, const int* __restrict__ rows, const int2* __restrict__ rcnt,
               int row_cap, int n, AdjK K, double* __restrict__ lam)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double3 yi = ld3(y, s);
    const int na = rcnt[s].x;
    double rho = 0.0, sg = 0.0;
    double3 S = make_double3(0.0, 0.0, 0.0);
    for (int e = 0; e < na; ++e) {
        const int j = rows[row_slot(s, e, row_cap)] & kRowIndexMask;
        const double3 d = sub3(yi, ld3(y, j));
        const double r2 = dot3(d, d), r = sqrt(r2);
        const double om = fmax(1.0 - r * K.inv_h, 0.0);
        rho += K.m * K.cw * om * om * om;
        if (r2 > kAdjEps2) {
            const double w1 = K.cg * om * om, c = w1 / r;
            S.x += c * d.x;
            S.y += c * d.y;
            S.z += c * d.z;
            sg += w1 * w1;
        }
    }
    const double l = -(rho - 1000.0) / (sg + dot3(S, S) + 0.1);
    lam[s] = l > 0.0 ? 0.0 : l;
}

__global__ void __launch_bounds__(kAdjBlock, 4)
    k64_pass_b(const double4* __restrict__ y, const double* __restrict__ lam, const int* __restrict__ rows,
               const int2* __restrict__ rcnt, int row_cap, int n, AdjK K, double4* __restrict__ ynext)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double3 yi = ld3(y, s);
    const double li = lam[s];
    const int nu = rcnt[s].y;
    double3 acc = make_double3(0.0, 0.0, 0.0);
    for (int e = 0; e < nu; ++e) {
        const int v = rows[row_slot(s, e, row_cap)];
        const int j = v & kRowIndexMask;
        const double mult = (double)__popc((unsigned)v >> 30);
        const double3 d = sub3(yi, ld3(y, j));
        const double r2 = dot3(d, d);
        if (!(r2 > kAdjEps2)) continue;
        const double r = sqrt(r2);
        const double om = fmax(1.0 - r * K.inv_h, 0.0);
        const double c = 10.0 * mult * (li + lam[j]) * K.cg * om * om / r;
        acc.x += c * d.x;
        acc.y += c * d.y;
        acc.z += c * d.z;
    }
    ynext[s] = make_double4(yi.x + acc.x, yi.y + acc.y, yi.z + acc.z, 0.0);
}

__global__ void __launch_bounds__(256)
    k64_finish(const double4* __restrict__ yS, const double4* __restrict__ y0, const double4* __restrict__ vp,
               const int* __restrict__ perm, int n, double inv_dt, double* __restrict__ x, double* __restrict__ v)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long i = perm[s];
    const double4 p = yS[s], q = y0[s], u = vp[s];
    x[3 * i] = p.x;
    x[3 * i + 1] = p.y;
    x[3 * i + 2] = p.z;
    v[3 * i] = u.x + (p.x - q.x) * inv_dt;
    v[3 * i + 1] = u.y + (p.y - q.y) * inv_dt;
    v[3 * i + 2] = u.z + (p.z - q.z) * inv_dt;
}

// ---- reverse

// a = dL/dy_S of a frame: dL/dx' + (dL/dv'')/dt, in the frame's sorted order.
__global__ void __launch_bounds__(256)
    k_adj_init(const int* __restrict__ perm, int n, const double* __restrict__ xb, const double* __restrict__ vb,
               double inv_dt, double4* __restrict__ a)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long i = perm[s];
    a[s] = make_double4(xb[3 * i] + vb[3 * i] * inv_dt, xb[3 * i + 1] + vb[3 * i + 1] * inv_dt,
                        xb[3 * i + 2] + vb[3 * i + 2] * inv_dt, 0.0);
}

// a = dL/dy_0 (the iterations reversed) less (dL/dv'')/dt; then
// dL/dx = dL/dy_0 and dL/dv = dL/dv'' + dt dL/dy_0, in caller order.
__global__ void __launch_bounds__(256)
    k_adj_final(const int* __restrict__ perm, int n, const double4* __restrict__ a, double dt, double inv_dt,
                double* __restrict__ xb, double* __restrict__ vb)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long i = perm[s];
    const double4 q = a[s];
    const double y0x = q.x - vb[3 * i] * inv_dt, y0y = q.y - vb[3 * i + 1] * inv_dt,
                 y0z = q.z - vb[3 * i + 2] * inv_dt;
    xb[3 * i] = y0x;
    xb[3 * i + 1] = y0y;
    xb[3 * i + 2] = y0z;
    vb[3 * i] += dt * y0x;
    vb[3 * i + 1] += dt * y0y;
    vb[3 * i + 2] += dt * y0z;
}

// r1: at iterate y_t, lambda_i, rhobar_i, Dbar_i (q1) and S_i (q2).
template <class T>
__global__ void __launch_bounds__(kAdjBlock, 4)
    k_adj_r1(const T* __restrict__ y, const double4* __restrict__ a, const int* __restrict__ rows,
             const int2* __restrict__ rcnt, int row_cap, int n, AdjK K, double4* __restrict__ q1,
             double4* __restrict__ q2)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double3 yi = ld3(y, s);
    const double4 ai4 = a[s];
    const double3 ai = make_double3(ai4.x, ai4.y, ai4.z);
    const int nu = rcnt[s].y;
    double rho = 0.0, sg = 0.0, lb = 0.0;
    double3 S = make_double3(0.0, 0.0, 0.0);
    for (int e = 0; e < nu; ++e) {
        const int v = rows[row_slot(s, e, row_cap)];
        const int j = v & kRowIndexMask;
        const bool A = v < 0;  // bit 31: j in N(i)
        const double mult = (double)__popc((unsigned)v >> 30);
        const double3 d = sub3(yi, ld3(y, j));
        const double r2 = dot3(d, d), r = sqrt(r2);
        const double om = fmax(1.0 - r * K.inv_h, 0.0);
        if (A) rho += K.m * K.cw * om * om * om;
        if (r2 > kAdjEps2) {
            const double w1 = K.cg * om * om, c = w1 / r;
            const double3 P = make_double3(c * d.x, c * d.y, c * d.z);
            if (A) {
                S.x += P.x;
                S.y += P.y;
                S.z += P.z;
                sg += w1 * w1;
            }
            const double4 aj = a[j];
            lb += mult * (P.x * (ai.x - aj.x) + P.y * (ai.y - aj.y) + P.z * (ai.z - aj.z));
        }
    }
    const double D = sg + dot3(S, S) + 0.1;
    const double lraw = -(rho - 1000.0) / D;
    const double lam = lraw > 0.0 ? 0.0 : lraw;
    const double lbar = 10.0 * lb;
    double rb = 0.0, Db = 0.0;
    if (!(lraw > 0.0)) {
        rb = -lbar / D;
        Db = -lbar * lam / D;
    }
    q1[s] = make_double4(lam, rb, Db, 0.0);
    q2[s] = make_double4(S.x, S.y, S.z, 0.0);
}

// r2: dL/dy_t.
template <class T>
__global__ void __launch_bounds__(kAdjBlock, 4)
    k_adj_r2(const T* __restrict__ y, const double4* __restrict__ a, const double4* __restrict__ q1,
             const double4* __restrict__ q2, const int* __restrict__ rows, const int2* __restrict__ rcnt,
             int row_cap, int n, AdjK K, double4* __restrict__ out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double3 yi = ld3(y, s);
    const double4 ai = a[s], qi = q1[s], Si = q2[s];
    const int nu = rcnt[s].y;
    double ox = ai.x, oy = ai.y, oz = ai.z;
    for (int e = 0; e < nu; ++e) {
        const int v = rows[row_slot(s, e, row_cap)];
        const int j = v & kRowIndexMask;
        const double3 d = sub3(yi, ld3(y, j));
        const double r2 = dot3(d, d);
        if (!(r2 > kAdjEps2)) continue;
        const double A = v < 0 ? 1.0 : 0.0, B = ((v >> 30) & 1) ? 1.0 : 0.0;
        const double r = sqrt(r2), ir = 1.0 / r;
        const double3 u = make_double3(d.x * ir, d.y * ir, d.z * ir);
        const double om = fmax(1.0 - r * K.inv_h, 0.0);
        const double w1 = K.cg * om * om, w2 = -2.0 * K.cg * om * K.inv_h;
        const double3 P = make_double3(w1 * u.x, w1 * u.y, w1 * u.z);
        const double4 aj = a[j], qj = q1[j], Sj = q2[j];
        const double cl = 10.0 * (A + B) * (qi.x + qj.x);
        const double ca = 2.0 * A * qi.z, cb = 2.0 * B * qj.z;
        const double3 vec = make_double3(cl * (ai.x - aj.x) + ca * (P.x + Si.x) + cb * (P.x - Sj.x),
                                         cl * (ai.y - aj.y) + ca * (P.y + Si.y) + cb * (P.y - Sj.y),
                                         cl * (ai.z - aj.z) + ca * (P.z + Si.z) + cb * (P.z - Sj.z));
        const double uv = dot3(u, vec);
        const double f = w1 * ir;
        const double cr = K.m * K.inv_h * (A * qi.y + B * qj.y);  // dW/dr = G/h
        ox += w2 * u.x * uv + f * (vec.x - u.x * uv) + cr * P.x;
        oy += w2 * u.y * uv + f * (vec.y - u.y * uv) + cr * P.y;
        oz += w2 * u.z * uv + f * (vec.z - u.z * uv) + cr * P.z;
    }
    out[s] = make_double4(ox, oy, oz, 0.0);
}

__global__ void __launch_bounds__(256) k_to_double(const float* __restrict__ a, long long m, double* __restrict__ b)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) b[t] = a ? (double)a[t] : 0.0;
}
__global__ void __launch_bounds__(256) k_to_float(const double* __restrict__ a, long long m, float* __restrict__ b)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) b[t] = (float)a[t];
}

// ------------------------------------------------------------ host side

// The record of the last rollout and the workspaces of its reverse pass.
struct PbdRoll {
    int n = 0, steps = 0, every = 0, iterations = 0, row_cap = 0, nseg = 0;
    bool f64 = false;
    bool valid = false;
    pk_pbf_params p{};
    Grid g{};
    float dt = 0.f, mass = 0.f;
    Spiky k{};
    // (x, v) in caller order at the start of every segment
    float* ck32 = nullptr;
    long long ck32_cap = 0;
    double* ck64 = nullptr;
    long long ck64_cap = 0;
    // one segment: every step's permutation, rows, row counts and iterates
    int* seg_perm = nullptr;
    long long seg_perm_cap = 0;
    int* seg_rows = nullptr;
    long long seg_rows_cap = 0;
    int2* seg_rcnt = nullptr;
    long long seg_rcnt_cap = 0;
    float4* seg_y32 = nullptr;
    long long seg_y32_cap = 0;
    double4* seg_y64 = nullptr;
    long long seg_y64_cap = 0;
    // double forward scratch: float copy of x for the list, y_0 and two
    // iterates, v', lambda
    float* xf = nullptr;
    double4 *y64a = nullptr, *y64b = nullptr, *y64c = nullptr, *vp64 = nullptr;
    double* lam64 = nullptr;
    // reverse state
    double4 *a = nullptr, *a2 = nullptr, *q1 = nullptr, *q2 = nullptr;
    double *xb = nullptr, *vb = nullptr;
    // replay state (caller order) of the double and of the float rollout
    double *xw64 = nullptr, *vw64 = nullptr;
    float *xw32 = nullptr, *vw32 = nullptr;
    int cap_n = 0;
};

template <class T>
bool grow_to(T*& p, long long& cap, long long want)
{
    if (want <= cap) return true;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc((void**)&p, sizeof(T) * (size_t)std::max(want, 1LL)) != cudaSuccess) return false;
    cap = want;
    return true;
}

template <class T>
bool realloc_to(T*& p, size_t count)
{
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc((void**)&p, sizeof(T) * std::max(count, (size_t)1)) == cudaSuccess;
}

PbdRoll*& roll_of(pk_ctx* c) { return reinterpret_cast<PbdRoll*&>(c->pbd_roll); }

bool ensure_roll_n(PbdRoll& R, int n)
{
    if (n <= R.cap_n) return true;
    const size_t m = (size_t)n;
    const bool ok = realloc_to(R.xf, 3 * m) && realloc_to(R.y64a, m) && realloc_to(R.y64b, m) &&
                    realloc_to(R.y64c, m) && realloc_to(R.vp64, m) && realloc_to(R.lam64, m) &&
                    realloc_to(R.a, m) && realloc_to(R.a2, m) && realloc_to(R.q1, m) && realloc_to(R.q2, m) &&
                    realloc_to(R.xb, 3 * m) && realloc_to(R.vb, 3 * m) && realloc_to(R.xw64, 3 * m) &&
                    realloc_to(R.vw64, 3 * m) && realloc_to(R.xw32, 3 * m) && realloc_to(R.vw32, 3 * m);
    if (!ok) return false;
    R.cap_n = n;
    return true;
}

AdjK adj_k(const PbdRoll& R)
{
    return AdjK{(double)R.k.inv_h, (double)R.k.cw, (double)R.k.cg, (double)R.mass};
}

unsigned blocks_of(long long m, int b) { return (unsigned)((m + b - 1) / b); }

// The context's list-build state for a frame of the rollout: rows with the
// rollout's row capacity; the fused-step list is stale afterwards.
void set_build_state(pk_ctx* c, const PbdRoll& R)
{
    c->nq_valid = false;
    c->grid = R.g;
    c->nq_n = R.n;
    c->nq_cap = R.p.nq.cap;
    c->row_cap = R.row_cap;
    c->nq_h = R.p.nq.radius;
    c->exported_index = nullptr;
    c->exported_elements = nullptr;
}

// One float frame: sort, list, Jacobi solve (every iterate kept when ys is
// given: y_0 .. y_S, each n float4; ys must then be the context's xs0).
int frame32(pk_ctx* c, const PbdRoll& R, float* x, float* v, float4* ys, cudaStream_t st)
{
    const int n = R.n;
    int l = sort_particles(c, x, v, nullptr, n, R.g, false, nullptr, 0.f, 0.f, R.dt, true, R.p.gravity, st);
    l += build_rows(c, n, R.g, R.p.nq.radius, R.p.nq.cap, R.row_cap, nullptr, nullptr, 0, st, false);
    if (ys)
        l += pbd_replay_solve(c, n, R.k, R.mass, R.iterations, R.dt, ys, x, v, st);
    else
        l += pbd_fast_solve(c, n, R.k, R.mass, R.iterations, R.dt, x, v, nullptr, st);
    return l;
}

// One double frame: the list from the positions rounded to float, then the
// integration and the Jacobi solve in double (every iterate kept in ys when
// given; otherwise y_0 stays in y64a and the iterates alternate between y64b
// and y64c).
int frame64(pk_ctx* c, PbdRoll& R, double* x, double* v, double4* ys, cudaStream_t st)
{
    const int n = R.n;
    const long long m3 = 3LL * n;
    k64_round<<<blocks_of(m3, 256), 256, 0, st>>>(x, m3, R.xf);
    int l = 1 + sort_particles(c, R.xf, R.xf, nullptr, n, R.g, false, nullptr, 0.f, 0.f, R.dt, false,
                               R.p.gravity, st);
    l += build_rows(c, n, R.g, R.p.nq.radius, R.p.nq.cap, R.row_cap, nullptr, nullptr, 0, st, false);
    const double dt = (double)R.dt;
    double4* y0 = ys ? ys : R.y64a;
    k64_begin<<<blocks_of(n, 256), 256, 0, st>>>(x, v, c->perm, n, (double)R.p.gravity[0], (double)R.p.gravity[1],
                                                (double)R.p.gravity[2], dt, y0, R.vp64);
    const AdjK K = adj_k(R);
    double4* cur = y0;
    for (int it = 0; it < R.iterations; ++it) {
        double4* nxt = ys ? ys + (size_t)(it + 1) * n : (it % 2 == 0 ? R.y64b : R.y64c);
        k64_pass_a<<<blocks_of(n, kAdjBlock), kAdjBlock, 0, st>>>(cur, c->rows, c->rcnt, R.row_cap, n, K, R.lam64);
        k64_pass_b<<<blocks_of(n, kAdjBlock), kAdjBlock, 0, st>>>(cur, R.lam64, c->rows, c->rcnt, R.row_cap, n, K,
                                                                  nxt);
        cur = nxt;
    }
    k64_finish<<<blocks_of(n, 256), 256, 0, st>>>(cur, y0, R.vp64, c->perm, n, 1.0 / dt, x, v);
    return l + 2 + 2 * R.iterations;
}

// Replays `len` steps from (x, v), keeping every step's list and iterates in
// the segment storage (the context's permutation, rows, row counts and, for
// the float frame, integrated positions are pointed at the storage meanwhile).
int replay32(pk_ctx* c, PbdRoll& R, float* x, float* v, int len, cudaStream_t st)
{
    const int n = R.n;
    const long long slots = row_slots(n, R.row_cap);
    int* perm0 = c->perm;
    int* rows0 = c->rows;
    int2* rcnt0 = c->rcnt;
    float4* xs00 = c->xs0;
    int l = 0;
    for (int j = 0; j < len; ++j) {
        c->perm = R.seg_perm + (size_t)j * n;
        c->rows = R.seg_rows + (size_t)j * slots;
        c->rcnt = R.seg_rcnt + (size_t)j * n;
        c->xs0 = R.seg_y32 + (size_t)j * (R.iterations + 1) * n;
        l += frame32(c, R, x, v, c->xs0, st);
    }
    c->perm = perm0;
    c->rows = rows0;
    c->rcnt = rcnt0;
    c->xs0 = xs00;
    return l;
}

int replay64(pk_ctx* c, PbdRoll& R, double* x, double* v, int len, cudaStream_t st)
{
    const int n = R.n;
    const long long slots = row_slots(n, R.row_cap);
    int* perm0 = c->perm;
    int* rows0 = c->rows;
    int2* rcnt0 = c->rcnt;
    int l = 0;
    for (int j = 0; j < len; ++j) {
        c->perm = R.seg_perm + (size_t)j * n;
        c->rows = R.seg_rows + (size_t)j * slots;
        c->rcnt = R.seg_rcnt + (size_t)j * n;
        l += frame64(c, R, x, v, R.seg_y64 + (size_t)j * (R.iterations + 1) * n, st);
    }
    c->perm = perm0;
    c->rows = rows0;
    c->rcnt = rcnt0;
    return l;
}

// Reverses the steps of the replayed segment, last first; R.xb / R.vb hold
// dL/dx, dL/dv of the segment's end on entry and of its start on return.
template <class T>
int reverse_segment(PbdRoll& R, const T* ys_base, int len, cudaStream_t st)
{
    const int n = R.n;
    const long long slots = row_slots(n, R.row_cap);
    const AdjK K = adj_k(R);
    const double dt = (double)R.dt, inv_dt = 1.0 / dt;
    const unsigned nb = blocks_of(n, kAdjBlock), nb256 = blocks_of(n, 256);
    int l = 0;
    for (int j = len - 1; j >= 0; --j) {
        const int* perm = R.seg_perm + (size_t)j * n;
        const int* rows = R.seg_rows + (size_t)j * slots;
        const int2* rcnt = R.seg_rcnt + (size_t)j * n;
        const T* ys = ys_base + (size_t)j * (R.iterations + 1) * n;
        k_adj_init<<<nb256, 256, 0, st>>>(perm, n, R.xb, R.vb, inv_dt, R.a);
        for (int it = R.iterations - 1; it >= 0; --it) {
            const T* y = ys + (size_t)it * n;
            k_adj_r1<T><<<nb, kAdjBlock, 0, st>>>(y, R.a, rows, rcnt, R.row_cap, n, K, R.q1, R.q2);
            k_adj_r2<T><<<nb, kAdjBlock, 0, st>>>(y, R.a, R.q1, R.q2, rows, rcnt, R.row_cap, n, K, R.a2);
            std::swap(R.a, R.a2);
        }
        k_adj_final<<<nb256, 256, 0, st>>>(perm, n, R.a, dt, inv_dt, R.xb, R.vb);
        l += 2 + 2 * R.iterations;
    }
    return l;
}

bool ensure_segment(PbdRoll& R)
{
    const long long n = R.n, every = std::max(R.every, 1);
    const long long slots = row_slots(n, R.row_cap);
    const long long ny = every * (R.iterations + 1) * n;
    bool ok = grow_to(R.seg_perm, R.seg_perm_cap, every * n) && grow_to(R.seg_rows, R.seg_rows_cap, every * slots) &&
              grow_to(R.seg_rcnt, R.seg_rcnt_cap, every * n);
    if (R.f64)
        ok = ok && grow_to(R.seg_y64, R.seg_y64_cap, ny);
    else
        ok = ok && grow_to(R.seg_y32, R.seg_y32_cap, ny);
    return ok;
}

}  // namespace

void pbd_roll_release(pk_ctx* c)
{
    PbdRoll* R = roll_of(c);
    if (!R) return;
    void* ps[] = {R->ck32, R->ck64, R->seg_perm, R->seg_rows, R->seg_rcnt, R->seg_y32, R->seg_y64, R->xf,
                  R->y64a, R->y64b, R->y64c, R->vp64, R->lam64, R->a, R->a2, R->q1, R->q2, R->xb, R->vb,
                  R->xw64, R->vw64, R->xw32, R->vw32};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete R;
    roll_of(c) = nullptr;
}

// The forward rollout (float or double): `steps` frames, (x, v) kept at the
// start of every segment of `every` steps for the reverse pass.  Returns the
// kernels launched, or -1 when memory runs out.
template <class T>
int pbd_rollout_impl(pk_ctx* c, T* x, T* v, int n, const pk_pbf_params* p, int steps, int every, int row_cap,
                     cudaStream_t st)
{
    PbdRoll*& Rp = roll_of(c);
    if (!Rp) Rp = new PbdRoll();
    PbdRoll& R = *Rp;
    const bool f64 = sizeof(T) == 8;
    R.valid = false;
    R.n = n;
    R.steps = steps;
    R.every = every > 0 ? every : std::max(steps, 1);
    R.iterations = p->pbd.iterations;
    R.row_cap = row_cap;
    R.f64 = f64;
    R.p = *p;
    R.g = make_grid(p->nq.radius, p->nq.lo, p->nq.hi);
    R.dt = p->pbd.dt;
    R.mass = effective_mass_of(&p->pbd);
    R.k = make_spiky(p->pbd.smoothing_length);
    R.nseg = (steps + R.every - 1) / R.every;
    if (!ensure_roll_n(R, n)) return -1;
    const long long m3 = 3LL * n;
    const long long ckw = 2 * m3 * std::max(R.nseg, 1);
    if (f64 ? !grow_to(R.ck64, R.ck64_cap, ckw) : !grow_to(R.ck32, R.ck32_cap, ckw)) return -1;
    T* ck_base = f64 ? (T*)(void*)R.ck64 : (T*)(void*)R.ck32;
    set_build_state(c, R);
    int l = 0;
    for (int k = 0; k < steps; ++k) {
        if (k % R.every == 0) {
            T* ck = ck_base + (size_t)(k / R.every) * 2 * m3;
            cudaMemcpyAsync(ck, x, sizeof(T) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(ck + m3, v, sizeof(T) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
        }
        if (f64)
            l += frame64(c, R, (double*)(void*)x, (double*)(void*)v, nullptr, st);
        else
            l += frame32(c, R, (float*)(void*)x, (float*)(void*)v, nullptr, st);
    }
    R.valid = true;
    return l;
}

template int pbd_rollout_impl<float>(pk_ctx*, float*, float*, int, const pk_pbf_params*, int, int, int,
                                     cudaStream_t);
template int pbd_rollout_impl<double>(pk_ctx*, double*, double*, int, const pk_pbf_params*, int, int, int,
                                      cudaStream_t);

// The reverse pass of the last rollout: dL/dx_T, dL/dv_T (caller order;
// vbar may be null) to dL/dx_0, dL/dv_0.  Returns kernels launched, -1 when
// memory runs out, -2 when no rollout of this precision is recorded.
template <class T>
int pbd_backward_impl(pk_ctx* c, const T* xbar, const T* vbar, T* gx, T* gv, cudaStream_t st)
{
    PbdRoll* Rp = roll_of(c);
    const bool f64 = sizeof(T) == 8;
    if (!Rp || !Rp->valid || Rp->f64 != f64) return -2;
    PbdRoll& R = *Rp;
    const int n = R.n;
    const long long m3 = 3LL * n;
    if (!ensure_segment(R)) return -1;
    set_build_state(c, R);
    int l = 0;
    if (f64) {
        cudaMemcpyAsync(R.xb, xbar, sizeof(double) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
        if (vbar)
            cudaMemcpyAsync(R.vb, vbar, sizeof(double) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
        else
            cudaMemsetAsync(R.vb, 0, sizeof(double) * (size_t)m3, st);
    } else {
        k_to_double<<<blocks_of(m3, 256), 256, 0, st>>>((const float*)(const void*)xbar, m3, R.xb);
        k_to_double<<<blocks_of(m3, 256), 256, 0, st>>>((const float*)(const void*)vbar, m3, R.vb);
        l += 2;
    }
    for (int sgm = R.nseg - 1; sgm >= 0; --sgm) {
        const int k0 = sgm * R.every;
        const int len = std::min(R.every, R.steps - k0);
        if (f64) {
            const double* ck = R.ck64 + (size_t)sgm * 2 * m3;
            cudaMemcpyAsync(R.xw64, ck, sizeof(double) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(R.vw64, ck + m3, sizeof(double) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
            l += replay64(c, R, R.xw64, R.vw64, len, st);
            l += reverse_segment<double4>(R, R.seg_y64, len, st);
        } else {
            const float* ck = R.ck32 + (size_t)sgm * 2 * m3;
            cudaMemcpyAsync(R.xw32, ck, sizeof(float) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(R.vw32, ck + m3, sizeof(float) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
            l += replay32(c, R, R.xw32, R.vw32, len, st);
            l += reverse_segment<float4>(R, R.seg_y32, len, st);
        }
    }
    if (f64) {
        cudaMemcpyAsync(gx, R.xb, sizeof(double) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(gv, R.vb, sizeof(double) * (size_t)m3, cudaMemcpyDeviceToDevice, st);
    } else {
        k_to_float<<<blocks_of(m3, 256), 256, 0, st>>>(R.xb, m3, (float*)(void*)gx);
        k_to_float<<<blocks_of(m3, 256), 256, 0, st>>>(R.vb, m3, (float*)(void*)gv);
        l += 2;
    }
    return l;
}

template int pbd_backward_impl<float>(pk_ctx*, const float*, const float*, float*, float*, cudaStream_t);
template int pbd_backward_impl<double>(pk_ctx*, const double*, const double*, double*, double*, cudaStream_t);

}  // namespace pk
