// pk_pd.cu -- ElasticityModule (projective peridynamics).
//
// The rest shape (bond list + rest positions) is set at initialisation
// (ElasticityModule::resetRestShape, ElasticityModule.cu:496-517) and K^-1 is
// computed with it; the reference recomputes the same matrix every step
// (solveElasticity -> computeInverseK, :404-411), which pk_pd_compute_inverse_k
// does where plasticity moves the rest shape.  Each projection iteration
// is EM_EnforceElasticity (:123-242) + K_UpdatePosition (:281-292).
#include "pk_kernels.cuh"
#include "pk_pd_common.cuh"

namespace pk {

// K_UpdateRestShape (ElasticityModule.cu:449-494): copy the list, self to slot 0.
__global__ void __launch_bounds__(256)
    k_pd_rest(const float* __restrict__ x, int n, const int* __restrict__ index,
              const int* __restrict__ elements, int cap, long long total,
              int* __restrict__ ridx, float* __restrict__ rpos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int m = pd_size(index, cap, total, n, i);
    for (int e = 0; e < m; ++e) {
        long long at = pd_at(index, cap, i, e);
        int j = elements[at];
        if (i != j || e == 0) {
            ridx[at] = j;
            rpos[3 * at] = x[3 * j];
            rpos[3 * at + 1] = x[3 * j + 1];
            rpos[3 * at + 2] = x[3 * j + 2];
        } else {
            long long a0 = pd_at(index, cap, i, 0);
            ridx[at] = ridx[a0];
            rpos[3 * at] = rpos[3 * a0];
            rpos[3 * at + 1] = rpos[3 * a0 + 1];
            rpos[3 * at + 2] = rpos[3 * a0 + 2];
            ridx[a0] = j;
            rpos[3 * a0] = x[3 * j];
            rpos[3 * a0 + 1] = x[3 * j + 1];
            rpos[3 * a0 + 2] = x[3 * j + 2];
        }
    }
}

// EM_PrecomputeShape (ElasticityModule.cu:21-116): weighted second moment of
// the rest bonds, then the pseudo-inverse with singular values <= 1e-4*h
// replaced by 1 (polarDecomposition's SVD of a symmetric PSD matrix is its
// eigen-decomposition).  invK row-major.  Two kernels: eight lanes per
// particle sum the bonds (coalesced walks of the rest shape) into invK and
// tws, then one thread per particle takes the eigen-decomposition in place
// (every lane of a warp busy with its own double-precision solve).
__global__ void __launch_bounds__(128)
    k_pd_invk_sums(int n, const int* __restrict__ index, int cap, long long total,
                   const float* __restrict__ rpos, float h, float* __restrict__ Kout, float* __restrict__ tws)
{
    const Lane8 L = lane8_of(n);
    const int i = L.i;
    const long long a0 = pd_at(index, cap, i, 0);
    const float ri0 = rpos[3 * a0], ri1 = rpos[3 * a0 + 1], ri2 = rpos[3 * a0 + 2];
    const int m = pd_size(index, cap, total, n, i);
    float M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, tw = 0.f;
    for (int e = L.sub; e < m; e += 8) {
        const long long at = pd_at(index, cap, i, e);
        const float q0 = rpos[3 * at] - ri0, q1 = rpos[3 * at + 1] - ri1, q2 = rpos[3 * at + 2] - ri2;
        const float r = exact_norm3(q0, q1, q2);  // (rest_j - rest_i).norm(), as compiled by the reference
        if (r > kEpsilon) {
            const float wt = corr_w(r, h), sw = sqrtf(wt);
            const float q[3] = {q0 / h * sw, q1 / h * sw, q2 / h * sw};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) M[a][b] += q[a] * q[b];
            tw += wt;
        }
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) M[a][b] = sum8(M[a][b]);
    tw = sum8(tw);
    if (!L.valid || L.sub != 0) return;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Kout[9LL * i + 3 * a + b] = M[a][b];
    tws[i] = tw;
}

__global__ void __launch_bounds__(128)
    k_pd_invk_solve(int n, float h, const float* __restrict__ tws, float* __restrict__ invK)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float M[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) M[a][b] = invK[9LL * i + 3 * a + b];
    const float tw = tws[i];
    if (tw > kEpsilon) {
        const float s = 1.0f / tw;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) M[a][b] *= s;
    }
    double A[3][3], Q[3][3], w[3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) A[a][b] = (double)M[a][b];
    jacobi3(A, Q, w);
    const double thr = (double)(0.0001f * h);
    for (int a = 0; a < 3; ++a) {
        const double sv = fabs(w[a]);
        w[a] = sv > thr ? 1.0 / sv : 1.0;
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            invK[9LL * i + 3 * a + b] =
                (float)(Q[a][0] * w[0] * Q[b][0] + Q[a][1] * w[1] * Q[b][1] + Q[a][2] * w[2] * Q[b][2]);
}

static int launch_invk(pk_ctx* c, int n, int cap, long long total, float h, cudaStream_t st)
{
    k_pd_invk_sums<<<(unsigned)(((long long)n * 8 + 127) / 128), 128, 0, st>>>(n, c->pd_index, cap, total,
                                                                              c->pd_rest_pos, h, c->pd_invK,
                                                                              c->pd_ktw);
    k_pd_invk_solve<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, h, c->pd_ktw, c->pd_invK);
    return 2;
}

__global__ void __launch_bounds__(256) k_fill_f(float* __restrict__ p, long long m, float v)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) p[t] = v;
}
__global__ void __launch_bounds__(256) k_fill_u8(unsigned char* __restrict__ p, long long m, unsigned char v)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) p[t] = v;
}

// Stretch break (no reference counterpart): a bond dies for good once
// |x_i - x_j| > (1 + s) * |rest_i - rest_j|.  kBreakG lanes per particle,
// lane `sub` taking bonds sub, sub + kBreakG, ...
constexpr int kBreakG = 8;
__global__ void __launch_bounds__(256)
    k_pd_break(const float* __restrict__ x, int n, const int* __restrict__ index, int cap,
               long long total, const int* __restrict__ ridx, const float* __restrict__ rpos,
               unsigned char* __restrict__ alive, float s)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(gid / kBreakG), sub = (int)(gid % kBreakG);
    if (i >= n) return;
    long long a0 = pd_at(index, cap, i, 0);
    int m = pd_size(index, cap, total, n, i);
    for (int e = sub; e < m; e += kBreakG) {
        long long at = pd_at(index, cap, i, e);
        if (!alive[at]) continue;
        int j = ridx[at];
        float r0 = rpos[3 * at] - rpos[3 * a0], r1 = rpos[3 * at + 1] - rpos[3 * a0 + 1],
              r2 = rpos[3 * at + 2] - rpos[3 * a0 + 2];
        float c0 = x[3 * j] - x[3 * i], c1 = x[3 * j + 1] - x[3 * i + 1], c2 = x[3 * j + 2] - x[3 * i + 2];
        // lengths rounded as Vector3f::norm compiles (fma(z,z,fma(x,x,y*y)))
        float lr = __fsqrt_rn(__fmaf_rn(r2, r2, __fmaf_rn(r0, r0, __fmul_rn(r1, r1))));
        float lc = __fsqrt_rn(__fmaf_rn(c2, c2, __fmaf_rn(c0, c0, __fmul_rn(c1, c1))));
        if (lc > __fmul_rn(__fadd_rn(1.0f, s), lr)) alive[at] = 0;
    }
}

int pd_rest_shape(pk_ctx* c, const float* x, int n, const int* index, const int* elements, int cap,
                  long long total, float horizon, cudaStream_t st)
{
    if (n <= 0) return 0;
    const unsigned nb = (unsigned)((n + 255) / 256);
    long long bonds = cap > 0 ? (long long)n * cap : total;
    cudaMemcpyAsync(c->pd_index, index, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    k_pd_rest<<<nb, 256, 0, st>>>(x, n, index, elements, cap, total, c->pd_rest_idx, c->pd_rest_pos);
    const int l = launch_invk(c, n, cap, total, horizon, st);
    k_fill_f<<<nb, 256, 0, st>>>(c->pd_bulk, n, 1.0f);  // computeMaterialStiffness (:371-387)
    if (bonds > 0)
        k_fill_u8<<<(unsigned)((bonds + 255) / 256), 256, 0, st>>>(c->pd_alive, bonds, 1);
    return 4 + l;
}

int pd_inverse_k(pk_ctx* c, float horizon, cudaStream_t st)
{
    const int n = c->pd_n;
    if (n <= 0) return 0;
    return launch_invk(c, n, c->pd_cap, c->pd_total, horizon, st);
}

int pd_solve(pk_ctx* c, float* x, float* v, int n, float horizon, float mu, float lambda,
             int iterations, float dt, float break_stretch, cudaStream_t st)
{
    if (n <= 0) return 0;
    int launches = 0;
    if (break_stretch > 0.f) {
        k_pd_break<<<(unsigned)(((long long)n * kBreakG + 255) / 256), 256, 0, st>>>(x, n, c->pd_index, c->pd_cap,
                                                                                      c->pd_total,
                                                               c->pd_rest_idx, c->pd_rest_pos, c->pd_alive,
                                                               break_stretch);
        ++launches;
    }
    // the projection as gathers over outgoing and incoming bonds (pk_pd_adj.cu)
    const int l = pd_project_solve(c, x, v, n, horizon, mu, lambda, iterations, dt, st);
    return l < 0 ? l : launches + l;
}

}  // namespace pk
