// pk_noalloc.cu -- DensityPBD solve that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application that
// owns the GPU's memory itself (a fixed budget or its own pool, with plugins
// forbidden to allocate), or a frame loop that cannot pay the implicit device
// synchronisation of cudaMalloc/cudaFree.  pk_pbd_solve_noalloc serves them:
// it needs no context (creating one allocates) and keeps its scratch --
// density, lambda, displacement and the start positions, 8 floats per
// particle -- in one fixed device array defined in this file.
//
// That array is a __device__ symbol: in host code its name is only a
// stand-in, so its device address is fetched once per device with
// cudaGetSymbolAddress (the first call on a device does this) and passed to
// the kernels.  Every GPU that loads the library holds the 4 MiB until exit.
#include <mutex>

#include "pk_kernels.cuh"

#define PK_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int kNoAllocMaxParticles = 131072;
constexpr size_t kNoAllocFloats = 8ull * kNoAllocMaxParticles;  // rho, lambda, dpos[3], xold[3]

// The scratch of every pk_pbd_solve_noalloc call on this device.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
float* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once.
float* scratch_on_current_device(int* status)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        *status = PK_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            *status = PK_ERR_CUDA;
            return nullptr;
        }
        g_scratch_ptr[dev] = static_cast<float*>(p);
    }
    *status = PK_OK;
    return g_scratch_ptr[dev];
}

}  // namespace

PK_API int pk_noalloc_max_particles(void) { return kNoAllocMaxParticles; }

PK_API int pk_pbd_solve_noalloc(float* x, float* v, int n, const int* index, const int* elements,
                                int cap, long long total, const pk_pbd_params* p, float* rho_out,
                                pk_stream stream)
{
    if (n < 0 || !p) return PK_ERR_ARG;
    if (n > kNoAllocMaxParticles) return PK_ERR_CAPACITY;  // beyond the fixed scratch
    if (n > 0 && (!x || !v || !index || !elements)) return PK_ERR_ARG;
    if (cap < 0 || (cap == 0 && total < 0)) return PK_ERR_ARG;
    if (!(p->smoothing_length > 0.0f) || !(p->sampling_distance > 0.0f) || !(p->dt > 0.0f) ||
        p->iterations < 0 || p->smoothing_length / p->sampling_distance > 64.0f)
        return PK_ERR_ARG;
    int status = PK_OK;
    float* base = scratch_on_current_device(&status);
    if (status != PK_OK) return status;
    // Scratch layout by the maximum size; the displacement is zeroed by the
    // lambda kernel of every iteration before it is accumulated, the other
    // parts are written before they are read.
    float* rho_s = base;
    float* lam = base + kNoAllocMaxParticles;
    float* dpos = base + 2ull * kNoAllocMaxParticles;
    float* xold = base + 5ull * kNoAllocMaxParticles;
    pk::pbd_generic_solve_scratch(x, v, n, index, elements, cap, total,
                                  pk::make_spiky(p->smoothing_length), pk::effective_mass_of(p),
                                  p->iterations, p->dt, rho_out, rho_s, lam, dpos, xold,
                                  (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? PK_OK : PK_ERR_CUDA;
}
