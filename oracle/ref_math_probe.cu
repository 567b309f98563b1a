// ref_math_probe.cu -- TEST INFRASTRUCTURE ONLY: a driver that runs the
// reference's own device arithmetic for the hot path, compiled by nvcc from the
// reference sources where they lie (no copy, no patch), to produce golden
// vectors that pin the CPU restatement and the sm_100a library:
//   Vector3f::norm / normalize   Core/Vector/vector_3d.inl:206-224 (glm::length,
//                                glm::normalize), the distance every neighbour
//                                decision `d < h` is taken on
//                                (NeighborQuery.cu:266,357,536)
//   SpikyKernel Weight/Gradient  Dynamics/ParticleSystem/Kernel.h:29-58
//   SmoothKernel::Weight         Dynamics/ParticleSystem/Kernel.h:62-75
//   CorrectedKernel Weight/WeightRR  Dynamics/ParticleSystem/Kernel.h:90-142
//   polarDecomposition           Core/Algorithm/MatrixFunc.inl:81-98 with the
//                                vendored svd3 (Core/Algorithm/svd3_cuda.h), the
//                                rotation and SVD the plasticity kernels use
//                                (ElastoplasticityModule.cu:442-458,624-634)
// The hot-path .cu files themselves (NeighborQuery.cu, DensityPBD.cu,
// ElasticityModule.cu) do not compile unmodified outside MSVC, so they are not
// built here; see oracle/Makefile.
//
// Usage (on a machine with a GPU):
//   ref_math_probe pairs   <in.f32: n x 6 (a, b)>   <out.f32: n x 4 (|a-b|, unit(a-b))>
//   ref_math_probe kernels <h> <in.f32: n (r)>       <out.f32: n x 5 (spikyW, spikyG,
//                                                      smoothW, correctedW, correctedWRR)>
//   ref_math_probe polar <thr> <in.f32: n x 9 (A row-major)>
//                                 <out.f32: n x 21 (R row-major, D diagonal,
//                                  V D' U^T row-major with D' = 1/D above thr, 1 below)>
// Files are raw little-endian float32.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "Core/Algorithm/MatrixFunc.h"
#include "Core/DataTypes.h"
#include "Dynamics/ParticleSystem/Kernel.h"

using PhysIKA::Vector3f;

__global__ void k_pairs(const float* __restrict__ ab, float* __restrict__ out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = ab + 6 * (size_t)i;
    const Vector3f a(p[0], p[1], p[2]), b(p[3], p[4], p[5]);
    Vector3f e = a - b;
    const float d = e.norm();
    Vector3f u = e;
    u.normalize();
    out[4 * (size_t)i + 0] = d;
    out[4 * (size_t)i + 1] = u[0];
    out[4 * (size_t)i + 2] = u[1];
    out[4 * (size_t)i + 3] = u[2];
}

__global__ void k_kernels(const float* __restrict__ r, float h, float* __restrict__ out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    PhysIKA::SpikyKernel<float> spiky;
    PhysIKA::SmoothKernel<float> smooth;
    PhysIKA::CorrectedKernel<float> corrected;
    const float ri = r[i];
    out[5 * (size_t)i + 0] = spiky.Weight(ri, h);
    out[5 * (size_t)i + 1] = spiky.Gradient(ri, h);
    out[5 * (size_t)i + 2] = smooth.Weight(ri, h);
    out[5 * (size_t)i + 3] = corrected.Weight(ri, h);
    out[5 * (size_t)i + 4] = corrected.WeightRR(ri, h);
}

__global__ void k_polar(const float* __restrict__ in, float thr, float* __restrict__ out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 9 * (size_t)i;
    const PhysIKA::SquareMatrix<float, 3> A(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
    PhysIKA::SquareMatrix<float, 3> R, U, D, V;
    PhysIKA::polarDecomposition(A, R, U, D, V);
    float* o = out + 21 * (size_t)i;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o[3 * r + c] = R(r, c);
    for (int k = 0; k < 3; ++k) o[9 + k] = D(k, k);
    PhysIKA::SquareMatrix<float, 3> Di(0.0f);
    for (int k = 0; k < 3; ++k) Di(k, k) = D(k, k) > thr ? 1.0f / D(k, k) : 1.0f;
    const PhysIKA::SquareMatrix<float, 3> Inv = V * Di * U.transpose();
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o[12 + 3 * r + c] = Inv(r, c);
}

static std::vector<float> read_f32(const char* path)
{
    std::vector<float> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)bytes / sizeof(float));
    if (std::fread(v.data(), sizeof(float), v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

static bool write_f32(const char* path, const std::vector<float>& v)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v.data(), sizeof(float), v.size(), f) == v.size();
    std::fclose(f);
    return ok;
}

static int fail(const char* what)
{
    std::fprintf(stderr, "ref_math_probe: %s\n", what);
    return 1;
}

int main(int argc, char** argv)
{
    if (argc < 4) return fail("usage: pairs <in> <out> | kernels <h> <in> <out> | polar <thr> <in> <out>");
    const std::string mode = argv[1];
    const bool pairs = mode == "pairs", polar = mode == "polar";
    if (!pairs && ((mode != "kernels" && !polar) || argc < 5)) return fail("unknown mode or missing arguments");
    const char* in_path = pairs ? argv[2] : argv[3];
    const char* out_path = pairs ? argv[3] : argv[4];
    const std::vector<float> in = read_f32(in_path);
    const int per_in = pairs ? 6 : (polar ? 9 : 1), per_out = pairs ? 4 : (polar ? 21 : 5);
    if (in.empty() || in.size() % per_in) return fail("bad input file");
    const int n = (int)(in.size() / per_in);
    float *d_in = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, in.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_out, (size_t)n * per_out * sizeof(float)) != cudaSuccess)
        return fail("cudaMalloc failed");
    cudaMemcpy(d_in, in.data(), in.size() * sizeof(float), cudaMemcpyHostToDevice);
    const int blocks = (n + 255) / 256;
    if (pairs)
        k_pairs<<<blocks, 256>>>(d_in, d_out, n);
    else if (polar)
        k_polar<<<blocks, 256>>>(d_in, (float)std::atof(argv[2]), d_out, n);
    else
        k_kernels<<<blocks, 256>>>(d_in, (float)std::atof(argv[2]), d_out, n);
    std::vector<float> out((size_t)n * per_out);
    if (cudaMemcpy(out.data(), d_out, out.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(cudaGetErrorString(cudaGetLastError()));
    cudaFree(d_in);
    cudaFree(d_out);
    if (!write_f32(out_path, out)) return fail("cannot write output");
    return 0;
}
