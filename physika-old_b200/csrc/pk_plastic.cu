// pk_plastic.cu -- ElastoplasticityModule and FractureModule
// (Dynamics/ParticleSystem/ElastoplasticityModule.cu, FractureModule.cu) on
// the context's peridynamics rest shape.  Every kernel updates only the bonds
// of its own particle, so the rest shape can be rewritten in place.  Bond
// walks split a particle's bonds over kPlG lanes; the double-precision
// eigen-decompositions run one thread per particle.
//
// The reference's SVDs come from svd3_cuda.h (McAdams et al. 2011: U and V
// rotations, the sign of det A on the smallest singular value).  What the
// modules use from them is unique: the clamped inverse V D^-1 U^T of a
// symmetric positive semi-definite matrix (its eigen-decomposition) and the
// polar rotation U V^T.  Both are formed in double from a Jacobi
// eigen-decomposition (jacobi3), with the same sign convention.
#include "pk_kernels.cuh"
#include "pk_pd_common.cuh"

namespace pk {

struct RestView {
    const int* index;
    int cap;
    long long total;
    int n;
    const int* ridx;
    float* rpos;
};

__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf((x * x + y * y) + z * z); }

// kPlG lanes per particle: lane `sub` walks bonds sub, sub + kPlG, ...; the
// group's partial sums are combined with xor shuffles in a fixed order.  The
// idle lanes of the last group mirror particle n - 1 and write nothing.
constexpr int kPlG = 8;
constexpr int kPlBlock = 128;
struct PlLane {
    int i, sub;
    bool valid;
};
__device__ __forceinline__ PlLane pl_lane(int n)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    PlLane L;
    L.i = (int)(gid / kPlG);
    L.sub = (int)(gid % kPlG);
    L.valid = L.i < n;
    if (!L.valid) L.i = n - 1;
    return L;
}
__device__ __forceinline__ float gsum8(float v)
{
#pragma unroll
    for (int o = kPlG / 2; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ void gsum8(float (&M)[3][3])
{
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) M[a][b] = gsum8(M[a][b]);
}

// Eigenpairs by decreasing eigenvalue.
__device__ inline void eig_sorted(double A[3][3], double Q[3][3], double w[3])
{
    jacobi3(A, Q, w);
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2 - a; ++b)
            if (w[b] < w[b + 1]) {
                double t = w[b];
                w[b] = w[b + 1];
                w[b + 1] = t;
                for (int k = 0; k < 3; ++k) {
                    t = Q[k][b];
                    Q[k][b] = Q[k][b + 1];
                    Q[k][b + 1] = t;
                }
            }
}

__device__ inline double det3d(const double M[3][3])
{
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

__device__ inline void unit3d(double u[3])
{
    const double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    if (l > 0) {
        u[0] /= l;
        u[1] /= l;
        u[2] /= l;
    }
}

__device__ inline void cross3d(const double a[3], const double b[3], double c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// polarDecomposition's R (MatrixFunc.inl:81-98): V from the eigenvectors of
// A^T A (v_2 flipped so det V = 1), u_0, u_1 = A v_0, A v_1 normalised,
// u_2 = u_0 x u_1; R = U V^T.  Zero matrix: identity.
__device__ inline void polar_rotation(const double A[3][3], double R[3][3])
{
    double S[3][3], V[3][3], w[3], u[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) S[a][b] = A[0][a] * A[0][b] + A[1][a] * A[1][b] + A[2][a] * A[2][b];
    eig_sorted(S, V, w);
    if (!(w[0] > 0)) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) R[a][b] = (a == b) ? 1.0 : 0.0;
        return;
    }
    if (det3d(V) < 0)
        for (int a = 0; a < 3; ++a) V[a][2] = -V[a][2];
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a) u[k][a] = A[a][0] * V[0][k] + A[a][1] * V[1][k] + A[a][2] * V[2][k];
    unit3d(u[0]);
    if (w[1] > 1e-24 * w[0]) {
        const double d = u[1][0] * u[0][0] + u[1][1] * u[0][1] + u[1][2] * u[0][2];
        for (int a = 0; a < 3; ++a) u[1][a] -= d * u[0][a];
        unit3d(u[1]);
    } else {
        double e[3] = {0, 0, 0};
        const int m = fabs(u[0][0]) <= fabs(u[0][1]) ? (fabs(u[0][0]) <= fabs(u[0][2]) ? 0 : 2)
                                                      : (fabs(u[0][1]) <= fabs(u[0][2]) ? 1 : 2);
        e[m] = 1.0;
        cross3d(u[0], e, u[1]);
        unit3d(u[1]);
    }
    cross3d(u[0], u[1], u[2]);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) R[a][b] = u[0][a] * V[b][0] + u[1][a] * V[b][1] + u[2][a] * V[b][2];
}

// V D' U^T of a symmetric positive semi-definite M: D' = 1/s above thr, fill below.
__device__ inline void clamped_inverse(const float M[3][3], double thr, double fill, float out[3][3])
{
    double A[3][3], Q[3][3], w[3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) A[a][b] = (double)M[a][b];
    jacobi3(A, Q, w);
    for (int a = 0; a < 3; ++a) {
        const double sv = fabs(w[a]);
        w[a] = sv > thr ? 1.0 / sv : fill;
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            out[a][b] = (float)(Q[a][0] * w[0] * Q[b][0] + Q[a][1] * w[1] * Q[b][1] + Q[a][2] * w[2] * Q[b][2]);
}

__device__ inline void mat_mul(const float A[3][3], const float B[3][3], float C[3][3])
{
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) C[a][b] = (A[a][0] * B[0][b] + A[a][1] * B[1][b]) + A[a][2] * B[2][b];
}

__device__ inline float det3f(const float M[3][3])
{
    return +M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

// EM_RotateRestShape (ElastoplasticityModule.cu:568-644) in three kernels:
// kPlG lanes per particle sum the deformation moment and the rest-shape
// moment over the bonds (coalesced walks), one thread per particle forms the
// rotation (two double-precision eigen-decompositions, every lane of a warp
// busy with its own particle), and kPlG lanes per particle rotate the bonds.
// Scratch per particle (kPlMk floats): mat (9), K (9), tw; then R (9).
__global__ void __launch_bounds__(kPlBlock) k_pl_rot_sums(RestView R, const float* __restrict__ x, float h,
                                                          float* __restrict__ mk)
{
    const PlLane L = pl_lane(R.n);
    const int i = L.i;
    const long long a0 = pd_at(R.index, R.cap, i, 0);
    const float ri[3] = {R.rpos[3 * a0], R.rpos[3 * a0 + 1], R.rpos[3 * a0 + 2]};
    const int m = pd_size(R.index, R.cap, R.total, R.n, i);
    float tw = 0.f, mat[3][3] = {}, K[3][3] = {};
    for (int e = L.sub; e < m; e += kPlG) {
        const long long at = pd_at(R.index, R.cap, i, e);
        const int j = R.ridx[at];
        const float* rj = R.rpos + 3 * at;
        const float r = len3(ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]);
        if (r > kEpsilon) {
            const float wt = smooth_w(r, h);
            float p[3], q[3];
            for (int a = 0; a < 3; ++a) {
                p[a] = (x[3 * j + a] - x[3 * i + a]) / h;
                q[a] = (rj[a] - ri[a]) / h;
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    mat[a][b] += p[a] * q[b] * wt;
                    K[a][b] += q[a] * q[b] * wt;
                }
            tw += wt;
        }
    }
    gsum8(mat);
    gsum8(K);
    tw = gsum8(tw);
    if (!L.valid || L.sub != 0) return;
    float* o = mk + (long long)kPlMk * i;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            o[3 * a + b] = mat[a][b];
            o[9 + 3 * a + b] = K[a][b];
        }
    o[18] = tw;
}

__global__ void __launch_bounds__(128) k_pl_rot_solve(int n, float h, float* __restrict__ mk)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* o = mk + (long long)kPlMk * i;
    float mat[3][3], K[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            mat[a][b] = o[3 * a + b];
            K[a][b] = o[9 + 3 * a + b];
        }
    const float tw = o[18];
    if (tw > kEpsilon) {
        const float s = 1.0f / tw;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                mat[a][b] *= s;
                K[a][b] *= s;
            }
    }
    float Ki[3][3], M2[3][3];
    clamped_inverse(K, (double)(0.0001f * h), 1.0, Ki);
    mat_mul(mat, Ki, M2);
    double Md[3][3], Rd[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Md[a][b] = (double)M2[a][b];
    polar_rotation(Md, Rd);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) o[3 * a + b] = (float)Rd[a][b];
}

__global__ void __launch_bounds__(kPlBlock) k_pl_rot_apply(RestView R, const float* __restrict__ mk)
{
    const PlLane L = pl_lane(R.n);
    const int i = L.i;
    const long long a0 = pd_at(R.index, R.cap, i, 0);
    const float ri[3] = {R.rpos[3 * a0], R.rpos[3 * a0 + 1], R.rpos[3 * a0 + 2]};
    const int m = pd_size(R.index, R.cap, R.total, R.n, i);
    float Rf[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Rf[a][b] = mk[(long long)kPlMk * i + 3 * a + b];
    __syncwarp();  // every lane holds rest_i before bond 0 (rest_i itself) is rewritten
    if (!L.valid) return;
    for (int e = L.sub; e < m; e += kPlG) {
        float* rj = R.rpos + 3 * pd_at(R.index, R.cap, i, e);
        const float d[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
        for (int a = 0; a < 3; ++a) rj[a] = ri[a] + ((Rf[a][0] * d[0] + Rf[a][1] * d[1]) + Rf[a][2] * d[2]);
    }
}

// I1 and the reference's J2 (PM_ComputeInvariants, ElastoplasticityModule.cu:43-128;
// the J2 loop assigns, so only the last bond over 0.01 h counts), by the
// particle's lane group: the I1 sums are combined, and J2 is the term of the
// group's largest qualifying bond index.
__device__ inline void invariants(const RestView& R, const float* __restrict__ x, float h, int i, int sub,
                                  float& I1, float& J2)
{
    const long long a0 = pd_at(R.index, R.cap, i, 0);
    const float ri[3] = {R.rpos[3 * a0], R.rpos[3 * a0 + 1], R.rpos[3 * a0 + 2]};
    const int m = pd_size(R.index, R.cap, R.total, R.n, i);
    const double lim = 0.01 * (double)h;
    float s1 = 0.f, tw = 0.f;
    for (int e = 1 + sub; e < m; e += kPlG) {
        const long long at = pd_at(R.index, R.cap, i, e);
        const int j = R.ridx[at];
        const float* rj = R.rpos + 3 * at;
        const float r = len3(ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]);
        if ((double)r > lim) {
            const float wt = corr_w(r, h);
            const float pl = len3(x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]);
            s1 += wt * (pl / r);
            tw += wt;
        }
    }
    s1 = gsum8(s1);
    tw = gsum8(tw);
    s1 = tw > kEpsilon ? s1 / tw : 1.0f;
    int last = -1;
    float j2 = 0.f;
    for (int e = 1 + sub; e < m; e += kPlG) {
        const long long at = pd_at(R.index, R.cap, i, e);
        const int j = R.ridx[at];
        const float* rj = R.rpos + 3 * at;
        const float r = len3(ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]);
        if ((double)r > lim) {
            const float wt = corr_w(r, h);
            const float pl = len3(x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]);
            const float ratio = pl / r;
            j2 = (ratio - s1) * (ratio - s1) * wt;
            last = e;
        }
    }
#pragma unroll
    for (int o = kPlG / 2; o >= 1; o >>= 1) {
        const int ol = __shfl_xor_sync(0xffffffffu, last, o);
        const float oj = __shfl_xor_sync(0xffffffffu, j2, o);
        if (ol > last) {
            last = ol;
            j2 = oj;
        }
    }
    I1 = s1;
    J2 = tw > kEpsilon ? sqrtf(j2 / tw) : 0.0f;
}

// PM_ComputeInvariants: Drucker-Prager yield (a yielding particle keeps its flag).
__global__ void __launch_bounds__(kPlBlock)
    k_pl_invariants(RestView R, const float* __restrict__ x, const float* __restrict__ bulk, float h, float A,
                    float B, float mu, float lambda, float* __restrict__ y1, float* __restrict__ y2,
                    float* __restrict__ i1, unsigned char* __restrict__ byield)
{
    const PlLane L = pl_lane(R.n);
    const int i = L.i;
    float I1, J2;
    invariants(R, x, h, i, L.sub, I1, J2);
    if (!L.valid || L.sub != 0) return;
    const float sJ2 = J2 * mu * bulk[i];
    const float sD1 = (1.0f - I1) * lambda * bulk[i];
    const float lim = A + B * sD1;
    if (sJ2 <= lim) {
        y1[i] = 0.f;
        y2[i] = 0.f;
        byield[i] = 0;
    } else if (lim > 0.f) {
        y1[i] = 0.f;
        y2[i] = (sJ2 - lim) / sJ2;
    } else {
        y1[i] = lim < -kEpsilon ? lim / (B * sD1) : 1.0f;
        y2[i] = 1.0f;
    }
    i1[i] = I1;
}

// v.norm() > EPSILON ? v.normalize() : 0 (normalize gives 0 below FLT_EPSILON).
__device__ inline void unit_or_zero3(float v[3])
{
    const float l = len3(v[0], v[1], v[2]);
    if (l > kEpsilon && l > 1.1920928955078125e-7f) {
        const float is = 1.0f / l;
        v[0] *= is;
        v[1] *= is;
        v[2] *= is;
    } else {
        v[0] = v[1] = v[2] = 0.f;
    }
}

// PM_ApplyYielding (ElastoplasticityModule.cu:165-226).
__global__ void __launch_bounds__(kPlBlock)
    k_pl_yield(RestView R, const float* __restrict__ x, const float* __restrict__ y1, const float* __restrict__ y2,
               const float* __restrict__ i1)
{
    const PlLane L = pl_lane(R.n);
    const int i = L.i;
    const long long a0 = pd_at(R.index, R.cap, i, 0);
    const float ri[3] = {R.rpos[3 * a0], R.rpos[3 * a0 + 1], R.rpos[3 * a0 + 2]};
    const int m = pd_size(R.index, R.cap, R.total, R.n, i);
    __syncwarp();  // every lane has read slot 0 before lane 0 of the group rewrites it
    if (!L.valid) return;
    for (int e = L.sub; e < m; e += kPlG) {
        const long long at = pd_at(R.index, R.cap, i, e);
        const int j = R.ridx[at];
        float* rj = R.rpos + 3 * at;
        const float s = i1[i] + i1[j];
        const float ya = (y1[i] + y1[j]) / 2, yb = (y2[i] + y2[j]) / 2;
        float p[3], q[3], nq[3], iso[3], dq[3];
        for (int a = 0; a < 3; ++a) {
            p[a] = x[3 * j + a] - x[3 * i + a];
            q[a] = rj[a] - ri[a];
            nq[a] = q[a] * s / 2;
            iso[a] = nq[a] - q[a];
            dq[a] = q[a];
        }
        unit_or_zero3(dq);
        const float pl = len3(p[0], p[1], p[2]);
        for (int a = 0; a < 3; ++a) rj[a] = (rj[a] + ya * iso[a]) + yb * (pl * dq[a] - nq[a]);
    }
}

// PM_ComputeInverseDeformation (ElastoplasticityModule.cu:389-471).
__global__ void __launch_bounds__(128)
    k_pl_invF(RestView R, const float* __restrict__ x, float h, float* __restrict__ invF)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R.n) return;
    const long long a0 = pd_at(R.index, R.cap, i, 0);
    const float ri[3] = {R.rpos[3 * a0], R.rpos[3 * a0 + 1], R.rpos[3 * a0 + 2]};
    const int m = pd_size(R.index, R.cap, R.total, R.n, i);
    float tw = 0.f, cur[3][3] = {}, ref[3][3] = {};
    for (int e = 0; e < m; ++e) {
        const long long at = pd_at(R.index, R.cap, i, e);
        const int j = R.ridx[at];
        const float* rj = R.rpos + 3 * at;
        const float r = len3(rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]);
        if (r > kEpsilon) {
            const float wt = corr_w(r, h);
            float p[3], q[3];
            for (int a = 0; a < 3; ++a) {
                p[a] = (x[3 * j + a] - x[3 * i + a]) / h;
                q[a] = (rj[a] - ri[a]) / h;
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    cur[a][b] += p[a] * p[b] * wt;
                    ref[a][b] += q[a] * p[b] * wt;
                }
            tw += wt;
        }
    }
    if (tw < kEpsilon) tw = 1.0f;
    const float s = 1.0f / tw;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            ref[a][b] *= s;
            cur[a][b] *= s;
        }
    float Ci[3][3], out[3][3];
    clamped_inverse(cur, (double)0.00001f, 1.0 / (double)0.00001f, Ci);
    mat_mul(ref, Ci, out);
    if (det3f(out) < kEpsilon)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) out[a][b] = (a == b) ? 1.0f : 0.0f;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) invF[9LL * i + 3 * a + b] = out[a][b];
}

// PM_ReconfigureRestShape (ElastoplasticityModule.cu:373-387).
__global__ void __launch_bounds__(256)
    k_pl_recon_sizes(RestView R, const unsigned char* __restrict__ byield, const int* __restrict__ nindex, int ncap,
                     long long ntotal, int* __restrict__ sizes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R.n) return;
    sizes[i] = byield[i] ? pd_size(nindex, ncap, ntotal, R.n, i) : pd_size(R.index, R.cap, R.total, R.n, i);
}

// PM_ReconstructRestShape (ElastoplasticityModule.cu:309-371) into CSR `off`.
__global__ void __launch_bounds__(128)
    k_pl_recon_fill(RestView R, const float* __restrict__ x, unsigned char* __restrict__ byield,
                    const float* __restrict__ invF, const int* __restrict__ nindex,
                    const int* __restrict__ nelements, int ncap, long long ntotal, const int* __restrict__ off,
                    int* __restrict__ new_idx, float* __restrict__ new_pos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R.n) return;
    const long long o = off[i];
    if (!byield[i]) {
        const int m = pd_size(R.index, R.cap, R.total, R.n, i);
        for (int e = 0; e < m; ++e) {
            const long long at = pd_at(R.index, R.cap, i, e);
            new_idx[o + e] = R.ridx[at];
            for (int a = 0; a < 3; ++a) new_pos[3 * (o + e) + a] = R.rpos[3 * at + a];
        }
    } else {
        const int m = pd_size(nindex, ncap, ntotal, R.n, i);
        const float* Fi = invF + 9LL * i;
        for (int e = 0; e < m; ++e) {
            const int j = nelements[pd_at(nindex, ncap, i, e)];
            const float* Fj = invF + 9LL * j;
            float M[3][3], d[3], np[3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) M[a][b] = 0.5f * (Fi[3 * a + b] + Fj[3 * a + b]);
            for (int a = 0; a < 3; ++a) d[a] = x[3 * j + a] - x[3 * i + a];
            for (int a = 0; a < 3; ++a) np[a] = x[3 * i + a] + ((M[a][0] * d[0] + M[a][1] * d[1]) + M[a][2] * d[2]);
            if (i != j || e == 0) {
                new_idx[o + e] = j;
                for (int a = 0; a < 3; ++a) new_pos[3 * (o + e) + a] = np[a];
            } else {
                new_idx[o + e] = new_idx[o];
                for (int a = 0; a < 3; ++a) new_pos[3 * (o + e) + a] = new_pos[3 * o + a];
                new_idx[o] = j;
                for (int a = 0; a < 3; ++a) new_pos[3 * o + a] = np[a];
            }
        }
    }
    byield[i] = 0;
}

// FractureModule's PM_ComputeInvariants (FractureModule.cu:15-105).
__global__ void __launch_bounds__(kPlBlock)
    k_pl_fracture(RestView R, const float* __restrict__ x, float* __restrict__ bulk, float h, float A, float B,
                  float mu, float lambda)
{
    const PlLane L = pl_lane(R.n);
    const int i = L.i;
    float I1, J2;
    invariants(R, x, h, i, L.sub, I1, J2);
    if (!L.valid || L.sub != 0) return;
    const float sJ2 = J2 * mu * bulk[i];
    const float sD1 = (1.0f - I1) * lambda * bulk[i];
    if (sJ2 > A + B * sD1) bulk[i] = 0.0f;
}

__global__ void __launch_bounds__(256) k_pl_fill_u8(unsigned char* __restrict__ p, long long m, unsigned char v)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) p[t] = v;
}

static RestView rest_view(pk_ctx* c)
{
    return RestView{c->pd_index, c->pd_cap, c->pd_total, c->pd_n, c->pd_rest_idx, c->pd_rest_pos};
}

static unsigned blocks(long long m, int b) { return (unsigned)((m + b - 1) / b); }

int pl_rotate(pk_ctx* c, const float* x, float h, cudaStream_t st)
{
    if (c->pd_n <= 0) return 0;
    const RestView R = rest_view(c);
    const unsigned g = blocks((long long)c->pd_n * kPlG, kPlBlock);
    k_pl_rot_sums<<<g, kPlBlock, 0, st>>>(R, x, h, c->pl_mk);
    k_pl_rot_solve<<<blocks(c->pd_n, 128), 128, 0, st>>>(c->pd_n, h, c->pl_mk);
    k_pl_rot_apply<<<g, kPlBlock, 0, st>>>(R, c->pl_mk);
    return 3;
}

int pl_yield(pk_ctx* c, const float* x, const pk_plastic_params* p, cudaStream_t st)
{
    const int n = c->pd_n;
    if (n <= 0) return 0;
    const RestView R = rest_view(c);
    const unsigned g = blocks((long long)n * kPlG, kPlBlock);
    k_pl_invariants<<<g, kPlBlock, 0, st>>>(R, x, c->pd_bulk, p->horizon, p->A, p->B, p->mu, p->lambda, c->pl_y1,
                                            c->pl_y2, c->pl_i1, c->pl_yield);
    k_pl_yield<<<g, kPlBlock, 0, st>>>(R, x, c->pl_y1, c->pl_y2, c->pl_i1);
    return 2;
}

int pl_fracture(pk_ctx* c, const float* x, const pk_plastic_params* p, cudaStream_t st)
{
    if (c->pd_n <= 0) return 0;
    k_pl_fracture<<<blocks((long long)c->pd_n * kPlG, kPlBlock), kPlBlock, 0, st>>>(rest_view(c), x, c->pd_bulk,
                                                                                    p->horizon, p->A, p->B, p->mu,
                                                                                    p->lambda);
    return 1;
}

int pl_enable_all(pk_ctx* c, cudaStream_t st)
{
    if (c->pd_n <= 0) return 0;
    k_pl_fill_u8<<<blocks(c->pd_n, 256), 256, 0, st>>>(c->pl_yield, c->pd_n, 1);
    return 1;
}

int pl_recon_begin(pk_ctx* c, const float* x, const int* nindex, int ncap, long long ntotal, float h,
                   cudaStream_t st)
{
    const int n = c->pd_n;
    if (n <= 0) return 0;
    const RestView R = rest_view(c);
    k_pl_recon_sizes<<<blocks(n, 256), 256, 0, st>>>(R, c->pl_yield, nindex, ncap, ntotal, c->pl_sizes);
    exclusive_scan(c->pl_sizes, n, c->pl_off, c->scan_part, st);
    k_pl_invF<<<blocks(n, 128), 128, 0, st>>>(R, x, h, c->pl_invF);
    return 2 + scan_launches();
}

int pl_recon_fill(pk_ctx* c, const float* x, const int* nindex, const int* nelements, int ncap, long long ntotal,
                  cudaStream_t st)
{
    const int n = c->pd_n;
    if (n <= 0) return 0;
    k_pl_recon_fill<<<blocks(n, 128), 128, 0, st>>>(rest_view(c), x, c->pl_yield, c->pl_invF, nindex, nelements,
                                                   ncap, ntotal, c->pl_off, c->pl_rest_idx2, c->pl_rest_pos2);
    return 1;
}

int pl_fill_alive(pk_ctx* c, long long bonds, cudaStream_t st)
{
    if (bonds <= 0) return 0;
    k_pl_fill_u8<<<blocks(bonds, 256), 256, 0, st>>>(c->pd_alive, bonds, 1);
    return 1;
}

}  // namespace pk
