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
// stand-in, so its device address is fetched with cudaGetSymbolAddress (the
// first call in a CUDA context does this) and passed to the kernels.  A
// symbol's address belongs to the context that loaded the module, so the
// address is kept per context, keyed by the context's process-unique id
// (cuCtxGetId): after cudaDeviceReset, or under a context the host application
// made current itself, the next call looks the address up again.  Every GPU
// that loads the library holds the 4 MiB until exit.
#include <cuda.h>

#include <mutex>

#include "pk_kernels.cuh"

#define PK_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int kNoAllocMaxParticles = 131072;
constexpr size_t kNoAllocFloats = 8ull * kNoAllocMaxParticles;  // rho, lambda, dpos[3], xold[3]

// The scratch of every pk_pbd_solve_noalloc call in a context.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
struct Cached {
    unsigned long long ctx_id = 0;  // 0: nothing cached
    float* ptr = nullptr;
};
Cached g_cache[kMaxDevices];

// The process-unique id of the calling thread's current context, or 0 when
// there is none yet (the runtime creates it on its first call that needs it)
// or the driver cannot tell.  The driver functions are reached through the
// runtime, so the library links no driver library.
unsigned long long current_context_id()
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {  // under g_mutex
        resolved = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) !=
                cudaSuccess || q1 != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
        cudaGetLastError();
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array in the current context.
float* scratch_in_current_context(int* status)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        *status = PK_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    unsigned long long id = current_context_id();
    if (id != 0 && g_cache[dev].ctx_id == id) {
        *status = PK_OK;
        return g_cache[dev].ptr;
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        *status = PK_ERR_CUDA;
        return nullptr;
    }
    // the lookup made the device's context current if it was not yet
    if (id == 0) id = current_context_id();
    g_cache[dev].ctx_id = id;  // stays 0 (looked up on every call) if the id is unknown
    g_cache[dev].ptr = static_cast<float*>(p);
    *status = PK_OK;
    return g_cache[dev].ptr;
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
    float* base = scratch_in_current_context(&status);
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
                                  p->iterations, p->dt, rho_out, rho_s, lam, dpos, xold, nullptr,
                                  (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? PK_OK : PK_ERR_CUDA;
}
