// pk_api.cu -- the extern "C" entry points declared in include/pk_hot.h.
//
// Validation happens here, on the host, before anything is enqueued; the
// kernels assume valid sizes.  Scratch grows on demand (cudaMalloc outside
// any capture; once a size has been seen nothing is allocated again).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pk_kernels.cuh"

#define PK_API extern "C" __attribute__((visibility("default")))

namespace {

int fail(pk_ctx* c, int code, const char* msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(pk_ctx* c, cudaError_t e, const char* where)
{
    if (c) {
        c->err = std::string(where) + ": " + cudaGetErrorString(e);
    }
    return PK_ERR_CUDA;
}

// Launch errors of everything enqueued since the last check.
int check_launch(pk_ctx* c, const char* where)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, where);
    return PK_OK;
}

template <class T>
bool regrow(T*& p, size_t count)
{
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void**)&p, sizeof(T) * count) == cudaSuccess;
}

int ensure_particles(pk_ctx* c, int n)
{
    if (n <= c->cap_n) return PK_OK;
    size_t m = (size_t)n;
    bool ok = regrow(c->perm, m) && regrow(c->inv, m) && regrow(c->key, m) && regrow(c->rank, m) &&
              regrow(c->count, m) && regrow(c->count_c, m) && regrow(c->offs, m + 1) &&
              regrow(c->xs_pre, m) && regrow(c->xs0, m) && regrow(c->xa, m) && regrow(c->xb, m) &&
              regrow(c->vs, m) && regrow(c->vv, m) && regrow(c->rho, m) && regrow(c->rcnt, m) &&
              regrow(c->tau, m) && regrow(c->tau_hint, m) && regrow(c->hcnt, m) && regrow(c->items, m + 1) &&
              regrow(c->nitems, 1) && regrow(c->ovf, m) && regrow(c->ovf_list, m) && regrow(c->tile_cnt, m + 2) &&
              regrow(c->tile_off, m + 2) && regrow(c->tiles, m + m / 128 + 2);
    if (!ok) {
        c->cap_n = 0;
        return fail(c, PK_ERR_NOMEM, "device allocation of particle scratch failed");
    }
    // no pivot yet: all ones sits above every distance, so the first selection
    // takes the plain rounds
    if (cudaMemset(c->tau_hint, 0xff, sizeof(unsigned) * m) != cudaSuccess)
        return fail(c, PK_ERR_CUDA, "cudaMemset of the selection pivots failed");
    c->cap_n = n;
    return PK_OK;
}

int ensure_rows(pk_ctx* c, long long m)
{
    if (m <= c->cap_rows) return PK_OK;
    if (!regrow(c->rows, (size_t)m) || !regrow(c->hits, (size_t)m)) {
        c->cap_rows = 0;
        return fail(c, PK_ERR_NOMEM, "device allocation of neighbour rows failed");
    }
    c->cap_rows = m;
    return PK_OK;
}

// The spill pool: 8 entries per particle, or what the last synchronised build
// found it needed (and a quarter more).
constexpr long long kPoolPerParticle = 8;

int ensure_pool(pk_ctx* c, int n)
{
    long long want = std::max<long long>((long long)n * kPoolPerParticle, 4096);
    if (c->pool_need > 0) want = std::max(want, c->pool_need + c->pool_need / 4);
    want = std::min<long long>((want + 3) & ~3LL, (1LL << 31) - 4);
    if (want <= c->pool_cap) return PK_OK;
    if (!regrow(c->hpool, (size_t)want) || !regrow(c->rpool, (size_t)want)) {
        c->pool_cap = 0;
        return fail(c, PK_ERR_NOMEM, "device allocation of the spill pool failed");
    }
    c->pool_cap = want;
    return PK_OK;
}

// Entries the last build handed out of the spill pool (also past its
// capacity), read after the stream's work; with offs_n, the dynamic list's
// total too, in the same synchronisation.  -1 on a CUDA error.
long long spill_used(pk_ctx* c, cudaStream_t st, int n = 0, int* offs_n = nullptr)
{
    unsigned long long used = 0;
    cudaError_t e = cudaMemcpyAsync(&used, c->spill, sizeof(used), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && offs_n) e = cudaMemcpyAsync(offs_n, c->offs + n, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return -1;
    if ((long long)used > c->pool_cap) c->pool_need = std::max(c->pool_need, (long long)used);
    return (long long)used;
}

int ensure_keys(pk_ctx* c, long long nk, int n)
{
    if (nk > c->cap_keys) {
        if (!regrow(c->cell_cnt, (size_t)nk + 1) || !regrow(c->cell_start, (size_t)nk + 2)) {
            c->cap_keys = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of the cell table failed");
        }
        c->cap_keys = nk;
    }
    long long parts = std::max(pk::scan_parts_needed(nk + 1), pk::scan_parts_needed(n));
    if (parts > c->cap_part) {
        if (!regrow(c->scan_part, (size_t)parts)) {
            c->cap_part = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of scan partials failed");
        }
        c->cap_part = parts;
    }
    return PK_OK;
}

int ensure_generic(pk_ctx* c, int n)
{
    if (n <= c->cap_g) return PK_OK;
    size_t m = (size_t)n;
    if (!(regrow(c->g_rho, m) && regrow(c->g_lam, m) && regrow(c->g_dpos, 3 * m) &&
          regrow(c->g_xold, 3 * m))) {
        c->cap_g = 0;
        return fail(c, PK_ERR_NOMEM, "device allocation of solver scratch failed");
    }
    c->cap_g = n;
    return PK_OK;
}

// Entries per particle kept in the main hit and solver rows: 128, or 2 cap
// for a larger cap; a dynamic list, whose solver rows hold every hit, 192 or
// its max_neighbors (a multiple of 4).  Longer rows continue in the spill
// pool.
int row_capacity(const pk_nq_params* p)
{
    int m = pk::kRowCapMin;
    if (p->cap > 0) m = std::max(m, 2 * p->cap);
    if (p->cap <= 0) m = p->max_neighbors > 0 ? std::max(m, p->max_neighbors) : pk::kRowCapDynamic;
    return std::min((m + 3) & ~3, pk::kRowCapMax);
}

int check_nq(pk_ctx* c, const pk_nq_params* p)
{
    if (!p) return fail(c, PK_ERR_ARG, "null neighbour-query parameters");
    if (!(p->radius > 0.0f) || !std::isfinite(p->radius))
        return fail(c, PK_ERR_ARG, "radius must be positive and finite");
    if (p->cap < 0 || p->cap > 448) return fail(c, PK_ERR_ARG, "cap must be in [0, 448]");
    if (p->max_neighbors < 0 || p->max_neighbors > pk::kRowCapMax)
        return fail(c, PK_ERR_ARG, "max_neighbors must be in [0, 4096]");
    for (int a = 0; a < 3; ++a)
        if (!(p->hi[a] > p->lo[a])) return fail(c, PK_ERR_ARG, "bounding box must have hi > lo");
    pk::Grid g = pk::make_grid(p->radius, p->lo, p->hi);
    if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0 || g.nkeys > (1LL << 30))
        return fail(c, PK_ERR_ARG, "grid too large for the radius and bounds");
    return PK_OK;
}

// SummationDensity::calculateScalingFactor (SummationDensity.cu:112-138) in
// host float arithmetic; returns factor * mass, the mass the kernels use.
float effective_mass(const pk_pbd_params* p)
{
    const float d = p->sampling_distance, H = p->smoothing_length;
    const float V = d * d * d;
    float total = 0.0f;
    const int half = (int)(H / d + 1.0f);
    for (int i = -half; i <= half; ++i)
        for (int j = -half; j <= half; ++j)
            for (int k = -half; k <= half; ++k) {
                float x = (float)i * d, y = (float)j * d, z = (float)k * d;
                float r = std::sqrt(x * x + y * y + z * z);
                float q = r / H, w = 0.0f;
                if (!(q > 1.0f)) {
                    float dd = (float)(1.0 - (double)q);
                    float hh = H * H;
                    w = 15.0f / ((float)M_PI * hh * H) * dd * dd * dd;
                }
                total += V * w;
            }
    const float factor = (float)(1.0 / (double)total);
    return factor * (p->rest_density * V);
}

int check_pbd(pk_ctx* c, const pk_pbd_params* p)
{
    if (!p) return fail(c, PK_ERR_ARG, "null DensityPBD parameters");
    if (!(p->smoothing_length > 0.0f) || !(p->sampling_distance > 0.0f) || !(p->dt > 0.0f))
        return fail(c, PK_ERR_ARG, "smoothing length, sampling distance and dt must be positive");
    if (p->iterations < 0) return fail(c, PK_ERR_ARG, "iterations must be >= 0");
    if (p->smoothing_length / p->sampling_distance > 64.0f)
        return fail(c, PK_ERR_ARG, "smoothing length / sampling distance too large");
    return PK_OK;
}

int check_list(pk_ctx* c, int n, const int* index, const int* elements, int cap, long long total)
{
    if (n > 0 && (!index || !elements)) return fail(c, PK_ERR_ARG, "null neighbour list");
    if (cap < 0) return fail(c, PK_ERR_ARG, "negative cap");
    if (cap == 0 && total < 0) return fail(c, PK_ERR_ARG, "negative list total");
    return PK_OK;
}

}  // namespace

namespace pk {

float effective_mass_of(const pk_pbd_params* p) { return effective_mass(p); }

void prof_begin(pk_ctx* c, int kind, cudaStream_t st)
{
    if (!c->prof) return;
    auto& ev = c->prof_ev[kind];
    int u = c->prof_used[kind];
    while ((int)ev.size() < u + 2) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        ev.push_back(e);
    }
    cudaEventRecord(ev[u], st);
}

void prof_end(pk_ctx* c, int kind, cudaStream_t st)
{
    if (!c->prof) return;
    auto& ev = c->prof_ev[kind];
    int u = c->prof_used[kind];
    if ((int)ev.size() < u + 2) return;
    cudaEventRecord(ev[u + 1], st);
    c->prof_used[kind] = u + 2;
}

}  // namespace pk

// ======================================================================
// context

PK_API int pk_ctx_create(pk_ctx** out, int device)
{
    if (!out) return PK_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return PK_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return PK_ERR_CUDA;
    pk_ctx* c = new pk_ctx();
    c->device = device;
    if (cudaMalloc((void**)&c->d_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&c->spill, 2 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(c->spill, 0, 2 * sizeof(unsigned long long)) != cudaSuccess) {
        if (c->d_err) cudaFree(c->d_err);
        if (c->spill) cudaFree(c->spill);
        delete c;
        return PK_ERR_NOMEM;
    }
    *out = c;
    return PK_OK;
}

PK_API int pk_graph_release(pk_ctx* c);

PK_API int pk_ctx_destroy(pk_ctx* c)
{
    if (!c) return PK_ERR_ARG;
    cudaSetDevice(c->device);
    pk_graph_release(c);
    if (c->capture_stream) cudaStreamDestroy(c->capture_stream);
    for (auto& e : c->tune.ev)
        if (e) cudaEventDestroy(e);
    void* ptrs[] = {c->d_err, c->perm, c->inv, c->key, c->rank, c->count, c->count_c, c->offs,
                    c->xs_pre, c->xs0, c->xa, c->xb, c->vs, c->vv, c->rho, c->rcnt, c->tau, c->tau_hint, c->pl_y1, c->pl_y2, c->pl_i1, c->pl_yield,
                    c->pl_invF, c->pl_sizes, c->pl_off, c->pl_rest_idx2, c->pl_rest_pos2,
                    c->hcnt, c->items, c->nitems,
                    c->rows, c->hits, c->hpool, c->rpool, c->ovf, c->ovf_list, c->spill, c->tile_cnt,
                    c->tile_off, c->tiles, c->cell_cnt, c->cell_start, c->scan_part, c->g_rho, c->g_lam,
                    c->g_dpos, c->g_xold, c->sdf, c->pd_index, c->pd_rest_idx, c->pd_rest_pos,
                    c->pd_alive, c->pd_invK, c->pd_bulk, c->pd_xold, c->pd_delta, c->pd_w,
                    c->pd_in_cnt, c->pd_in_off, c->pd_in, c->pd_in_slot, c->h_x, c->h_v, c->pd_ktw, c->pl_mk};
    pk::pd_work_release(c);
    pk::pbd_roll_release(c);
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& ev : c->prof_ev)
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    delete c;
    return PK_OK;
}

PK_API const char* pk_last_error(const pk_ctx* c)
{
    return c ? c->err.c_str() : "null context";
}

PK_API int pk_ctx_status(pk_ctx* c, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    cudaSetDevice(c->device);
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_ctx_status");
    int bits = 0;
    e = cudaMemcpy(&bits, c->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_ctx_status");
    if (bits) {
        cudaMemset(c->d_err, 0, sizeof(int));
        char msg[160];
        if (bits & pk::kErrBadIndex) {
            snprintf(msg, sizeof msg, "a particle id outside [0, n) was given in pins or a neighbour list (flags 0x%x)", bits);
            return fail(c, PK_ERR_ARG, msg);
        }
        const long long used = spill_used(c, (cudaStream_t)stream);
        if (bits & pk::kErrHitOverflow)
            snprintf(msg, sizeof msg,
                     "the spill pool of long neighbour rows ran out (flags 0x%x; %lld entries needed, %lld held; "
                     "the next build grows it)", bits, used, c->pool_cap);
        else
            snprintf(msg, sizeof msg, "capacity exceeded on the device (flags 0x%x: 1=row, 4=list)", bits);
        return fail(c, PK_ERR_CAPACITY, msg);
    }
    return PK_OK;
}

PK_API int pk_last_launch_count(const pk_ctx* c) { return c ? c->launches : -1; }

PK_API int pk_ctx_autotune(pk_ctx* c, int enable)
{
    if (!c) return PK_ERR_ARG;
    cudaSetDevice(c->device);
    auto& t = c->tune;
    t = pk_ctx::Tune{t.on, 0, t.pass_block, t.persist, t.build_pb, {0, 0, 0, 0}, {0, 0, 0},
                     {t.ev[0], t.ev[1], t.ev[2], t.ev[3]}};
    if (!enable) {
        t.on = false;
        return PK_OK;
    }
    for (auto& e : t.ev)
        if (!e && cudaEventCreate(&e) != cudaSuccess) return fail(c, PK_ERR_CUDA, "cudaEventCreate failed");
    t.on = true;
    t.frame = 0;
    return PK_OK;
}

PK_API int pk_ctx_tuning(const pk_ctx* c, int* pass_block, int* build_particles, int* active)
{
    if (!c) return PK_ERR_ARG;
    if (pass_block) *pass_block = c->tune.pass_block;
    if (build_particles) *build_particles = c->tune.build_pb;
    if (active) *active = c->tune.on ? 1 : 0;
    return PK_OK;
}

PK_API int pk_ctx_tuning_resident(const pk_ctx* c, int* resident)
{
    if (!c || !resident) return PK_ERR_ARG;
    *resident = c->tune.persist ? 1 : 0;
    return PK_OK;
}

PK_API int pk_ctx_profile(pk_ctx* c, int enable)
{
    if (!c) return PK_ERR_ARG;
    c->prof = enable != 0;
    for (int k = 0; k < PK_PROF_KINDS; ++k) c->prof_used[k] = 0;
    return PK_OK;
}

PK_API int pk_ctx_profile_read(pk_ctx* c, int kind, double* total_ms, int* launches)
{
    if (!c) return PK_ERR_ARG;
    if (kind < 0 || kind >= PK_PROF_KINDS || !total_ms || !launches)
        return fail(c, PK_ERR_ARG, "bad profile kind or output");
    cudaSetDevice(c->device);
    double sum = 0.0;
    auto& ev = c->prof_ev[kind];
    for (int u = 0; u + 1 < c->prof_used[kind]; u += 2) {
        cudaError_t e = cudaEventSynchronize(ev[u + 1]);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[u], ev[u + 1]);
        if (e != cudaSuccess) return cuda_fail(c, e, "pk_ctx_profile_read");
        sum += ms;
    }
    *total_ms = sum;
    *launches = c->prof_used[kind] / 2;
    return PK_OK;
}

// ======================================================================
// NeighborQuery

PK_API int pk_nq_build(pk_ctx* c, const float* x, int n, const pk_nq_params* p, int* index,
                       int* elements, long long elements_capacity, long long* total,
                       pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    if (n > (1 << 29)) return fail(c, PK_ERR_ARG, "more than 2^29 particles");
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    int rc = check_nq(c, p);
    if (rc) return rc;
    if (p->cap > 0 && elements && elements_capacity < (long long)n * p->cap)
        return fail(c, PK_ERR_ARG, "elements capacity below n*cap");
    if (elements && !index) return fail(c, PK_ERR_ARG, "elements given without index");
    cudaSetDevice(c->device);
    cudaStream_t st = (cudaStream_t)stream;
    pk::Grid g = pk::make_grid(p->radius, p->lo, p->hi);
    const int row_cap = row_capacity(p);
    if ((rc = ensure_particles(c, n)) || (rc = ensure_keys(c, g.nkeys + 1, n)) ||
        (rc = ensure_rows(c, pk::row_slots(n, row_cap))))
        return rc;
    c->nq_valid = false;
    c->grid = g;
    c->nq_n = n;
    c->nq_cap = p->cap;
    c->row_cap = row_cap;
    c->nq_h = p->radius;
    c->exported_index = index;
    c->exported_elements = elements;
    // rows longer than the capacity go to the spill pool; a pool too small for
    // this build is grown to what the build asked for and the build repeated
    int launches = 0;
    const bool dyn_total = total && p->cap <= 0 && index;
    int t = 0;  // the dynamic list's total, read in the same synchronisation
    for (int attempt = 0; attempt < 2; ++attempt) {
        if ((rc = ensure_pool(c, n))) return rc;
        launches = pk::sort_particles(c, const_cast<float*>(x), nullptr, nullptr, n, g, false, nullptr, 0.f, 0.f,
                                      0.f, false, nullptr, st);
        launches += pk::build_rows(c, n, g, p->radius, p->cap, row_cap, index, elements,
                                   elements ? elements_capacity : 0, st);
        if ((rc = check_launch(c, "pk_nq_build"))) return rc;
        const long long used = spill_used(c, st, n, dyn_total && n > 0 ? &t : nullptr);
        if (used < 0) return cuda_fail(c, cudaGetLastError(), "pk_nq_build");
        if (used <= c->pool_cap) break;
        cudaMemset(c->d_err, 0, sizeof(int));  // the repeated build replaces this one
    }
    c->launches = launches;
    c->nq_valid = true;
    if (total) {
        if (p->cap > 0) {
            *total = (long long)n * p->cap;
        } else if (index) {
            *total = n > 0 ? t : 0;
            if (elements && *total > elements_capacity) {
                cudaMemset(c->d_err, 0, sizeof(int));
                return fail(c, PK_ERR_CAPACITY, "dynamic neighbour list exceeds elements_capacity");
            }
        } else {
            *total = 0;
        }
    }
    return PK_OK;
}

PK_API int pk_nq_row_stats(pk_ctx* c, double* mean_list, double* mean_row, int* max_row,
                           pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (!c->nq_valid) return fail(c, PK_ERR_STATE, "no neighbour build on this context");
    cudaSetDevice(c->device);
    std::vector<int2> h((size_t)std::max(c->nq_n, 1));
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (c->nq_n > 0)
        e = cudaMemcpyAsync(h.data(), c->rcnt, sizeof(int2) * (size_t)c->nq_n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_nq_row_stats");
    double sa = 0, su = 0;
    int mx = 0;
    for (int i = 0; i < c->nq_n; ++i) {
        sa += h[i].x;
        su += h[i].y;
        mx = std::max(mx, h[i].y);
    }
    const double n = std::max(c->nq_n, 1);
    if (mean_list) *mean_list = sa / n;
    if (mean_row) *mean_row = su / n;
    if (max_row) *max_row = mx;
    return PK_OK;
}

// ======================================================================
// DensityPBD / SummationDensity / integrator

PK_API int pk_summation_density(pk_ctx* c, const float* x, int n, const int* index,
                                const int* elements, int cap, long long total,
                                const pk_pbd_params* p, float* rho, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    int rc = check_pbd(c, p);
    if (rc) return rc;
    if ((rc = check_list(c, n, index, elements, cap, total))) return rc;
    if (n > 0 && (!x || !rho)) return fail(c, PK_ERR_ARG, "null positions or density");
    cudaSetDevice(c->device);
    pk::density_generic(x, n, index, elements, cap, total, pk::make_spiky(p->smoothing_length),
                        effective_mass(p), rho, c->d_err, (cudaStream_t)stream);
    return check_launch(c, "pk_summation_density");
}

PK_API int pk_pbd_solve(pk_ctx* c, float* x, float* v, int n, const int* index, const int* elements,
                        int cap, long long total, const pk_pbd_params* p, float* rho_out,
                        pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    int rc = check_pbd(c, p);
    if (rc) return rc;
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    cudaSetDevice(c->device);
    cudaStream_t st = (cudaStream_t)stream;
    const pk::Spiky k = pk::make_spiky(p->smoothing_length);
    const float mass = effective_mass(p);
    const bool own_list = c->nq_valid && n == c->nq_n &&
                          ((index == nullptr && elements == nullptr) ||
                           (index == c->exported_index && elements == c->exported_elements &&
                            cap == c->nq_cap));
    if (own_list) {
        int l = pk::gather_state(c, x, v, n, st);
        l += pk::pbd_fast_solve(c, n, k, mass, p->iterations, p->dt, x, v, rho_out, st);
        c->launches = l;
    } else {
        if ((rc = check_list(c, n, index, elements, cap, total))) return rc;
        if ((rc = ensure_generic(c, n))) return rc;
        c->launches = pk::pbd_generic_solve(c, x, v, n, index, elements, cap, total, k, mass,
                                            p->iterations, p->dt, rho_out, st);
    }
    return check_launch(c, "pk_pbd_solve");
}

PK_API int pk_integrate(pk_ctx* c, float* x, float* v, const float* f, int n, const float gravity[3],
                        float dt, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    if (n > 0 && !v) return fail(c, PK_ERR_ARG, "null velocities");
    if (!gravity) return fail(c, PK_ERR_ARG, "null gravity");
    cudaSetDevice(c->device);
    c->launches = pk::integrate_aos(x, v, f, n, gravity, dt, (cudaStream_t)stream);
    return check_launch(c, "pk_integrate");
}

PK_API int pk_advect(pk_ctx* c, float* x, const float* v, int n, float dt, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || (n > 0 && (!x || !v))) return fail(c, PK_ERR_ARG, "bad positions or velocities");
    cudaSetDevice(c->device);
    c->launches = pk::advect_aos(x, v, n, dt, (cudaStream_t)stream);
    return check_launch(c, "pk_advect");
}

PK_API int pk_fixed_points(pk_ctx* c, float* x, float* v, int n, const int* ids, const float* target,
                           const float* vel, int count, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || count < 0 || (count > 0 && (!x || !v || !ids || !target)))
        return fail(c, PK_ERR_ARG, "bad positions, velocities, ids or targets");
    cudaSetDevice(c->device);
    c->launches = pk::fix_points(x, v, n, ids, target, vel, count, c->d_err, (cudaStream_t)stream);
    return check_launch(c, "pk_fixed_points");
}

PK_API int pk_plane_constrain(pk_ctx* c, float* x, int n, const float origin[3], const float dir[3],
                              pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || (n > 0 && !x) || !origin || !dir) return fail(c, PK_ERR_ARG, "bad arguments");
    cudaSetDevice(c->device);
    c->launches = pk::plane_constrain(x, n, origin, dir, (cudaStream_t)stream);
    return check_launch(c, "pk_plane_constrain");
}

PK_API int pk_update_velocity(pk_ctx* c, float* v, const float* x, const float* x_old, int n, float dt,
                              pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || (n > 0 && (!x || !v || !x_old))) return fail(c, PK_ERR_ARG, "bad arrays");
    if (!(dt > 0.0f)) return fail(c, PK_ERR_ARG, "dt must be positive");
    cudaSetDevice(c->device);
    c->launches = pk::velocity_from_positions(v, x, x_old, n, dt, (cudaStream_t)stream);
    return check_launch(c, "pk_update_velocity");
}

// ======================================================================
// BoundaryConstraint: the box SDF is evaluated on the host once per box with
// the float expressions of DistanceToBox / DistanceToSqure / DistanceToSegment
// (DistanceField3D.cu:14-123, K_DistanceFieldToBox :266-280), uploaded, and
// sampled by the kernels.  Host code is built without FMA contraction.

namespace {

float dot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

float segment_distance(const float* pos, const float* lo, const float* hi)
{
    float seg[3], e1[3], e2[3], nseg[3];
    for (int a = 0; a < 3; ++a) {
        seg[a] = hi[a] - lo[a];
        e1[a] = pos[a] - lo[a];
        e2[a] = pos[a] - hi[a];
        nseg[a] = -seg[a];
    }
    if (dot3(e1, seg) < 0.0f) return std::sqrt(dot3(e1, e1));
    if (dot3(e2, nseg) < 0.0f) return std::sqrt(dot3(e2, e2));
    float l1 = dot3(e1, e1);
    float len = std::sqrt(dot3(seg, seg));
    if (len > 1.1920929e-7f) {
        float is = 1.0f / std::sqrt(dot3(seg, seg));
        for (int a = 0; a < 3; ++a) seg[a] = seg[a] * is;
    } else {
        seg[0] = seg[1] = seg[2] = 0.0f;
    }
    float l2 = dot3(e1, seg);
    return std::sqrt(l1 - l2 * l2);
}

float square_distance(const float* pos, const float* lo, const float* hi, int axis)
{
    float c1[3], c2[3], c3[3], c4[3], nrm[3] = {0.f, 0.f, 0.f}, lc[2], hc[2], p[2];
    int u = axis == 0 ? 1 : 0, w = axis == 2 ? 1 : 2;  // the two in-plane axes
    for (int a = 0; a < 3; ++a) c1[a] = c2[a] = c3[a] = c4[a] = lo[a];
    // corners in the order of DistanceToSqure's switch
    if (axis == 0) {
        c2[1] = hi[1]; c3[1] = hi[1]; c3[2] = hi[2]; c4[2] = hi[2];
    } else if (axis == 1) {
        c2[2] = hi[2]; c3[0] = hi[0]; c3[2] = hi[2]; c4[0] = hi[0];
    } else {
        c2[0] = hi[0]; c3[0] = hi[0]; c3[1] = hi[1]; c4[1] = hi[1];
    }
    nrm[axis] = 1.0f;
    lc[0] = lo[u]; lc[1] = lo[w]; hc[0] = hi[u]; hc[1] = hi[w]; p[0] = pos[u]; p[1] = pos[w];
    float d1 = segment_distance(pos, c1, c2), d2 = segment_distance(pos, c2, c3);
    float d3 = segment_distance(pos, c3, c4), d4 = segment_distance(pos, c4, c1);
    float rel[3] = {pos[0] - c1[0], pos[1] - c1[1], pos[2] - c1[2]};
    float d5 = std::fabs(dot3(nrm, rel));
    if (p[0] < hc[0] && p[0] > lc[0] && p[1] < hc[1] && p[1] > lc[1]) return d5;
    return std::fmin(std::fmin(d1, d2), std::fmin(d3, d4));
}

float box_distance(const float* pos, const float* lo, const float* hi)
{
    if (pos[0] < hi[0] && pos[0] > lo[0] && pos[1] < hi[1] && pos[1] > lo[1] && pos[2] < hi[2] &&
        pos[2] > lo[2]) {
        float dx = std::fmin(std::fabs(pos[0] - hi[0]), std::fabs(pos[0] - lo[0]));
        float dy = std::fmin(std::fabs(pos[1] - hi[1]), std::fabs(pos[1] - lo[1]));
        float dz = std::fmin(std::fabs(pos[2] - hi[2]), std::fabs(pos[2] - lo[2]));
        return std::fmin(std::fmin(dx, dy), dz);
    }
    const float k0[3] = {lo[0], lo[1], lo[2]}, k1[3] = {hi[0], lo[1], lo[2]};
    const float k2[3] = {hi[0], hi[1], lo[2]}, k3[3] = {lo[0], hi[1], lo[2]};
    const float k4[3] = {lo[0], lo[1], hi[2]}, k5[3] = {hi[0], lo[1], hi[2]};
    const float k6[3] = {hi[0], hi[1], hi[2]}, k7[3] = {lo[0], hi[1], hi[2]};
    float x1 = square_distance(pos, k0, k7, 0), x2 = square_distance(pos, k1, k6, 0);
    float y1 = square_distance(pos, k0, k5, 1), y2 = square_distance(pos, k3, k6, 1);
    float z1 = square_distance(pos, k0, k2, 2), z2 = square_distance(pos, k4, k6, 2);
    return -std::fmin(std::fmin(std::fmin(x1, x2), std::fmin(y1, y2)), std::fmin(z1, z2));
}

}  // namespace

PK_API int pk_boundary_set_box(pk_ctx* c, const float lo[3], const float hi[3], float spacing,
                               int inverted, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (!lo || !hi || !(spacing > 0.0f)) return fail(c, PK_ERR_ARG, "bad box or spacing");
    int dims[3];
    float left[3], h[3];
    for (int a = 0; a < 3; ++a) {
        if (!(hi[a] > lo[a])) return fail(c, PK_ERR_ARG, "box must have hi > lo");
        int nb = (int)std::floor((hi[a] - lo[a]) / spacing) + 10;  // setCube (:111-115)
        float p0 = lo[a] - 5.0f * spacing, p1 = hi[a] + 5.0f * spacing;
        left[a] = p0;
        h[a] = (p1 - p0) * (float)(1.0 / (double)(float)(nb + 1));  // setSpace (:198)
        dims[a] = nb + 1;
    }
    long long nodes = (long long)dims[0] * dims[1] * dims[2];
    if (nodes > (1LL << 31)) return fail(c, PK_ERR_ARG, "SDF grid too large");
    std::vector<float> data((size_t)nodes);
    const float sign = inverted ? 1.0f : -1.0f;
    for (int k = 0; k < dims[2]; ++k)
        for (int j = 0; j < dims[1]; ++j)
            for (int i = 0; i < dims[0]; ++i) {
                float p[3] = {left[0] + (float)i * h[0], left[1] + (float)j * h[1], left[2] + (float)k * h[2]};
                data[((size_t)k * dims[1] + j) * dims[0] + i] = sign * box_distance(p, lo, hi);
            }
    cudaSetDevice(c->device);
    size_t bytes = sizeof(float) * (size_t)nodes;
    if (bytes > c->sdf_bytes) {
        if (c->sdf) cudaFree(c->sdf);
        c->sdf = nullptr;
        c->sdf_bytes = 0;
        if (cudaMalloc((void**)&c->sdf, bytes) != cudaSuccess)
            return fail(c, PK_ERR_NOMEM, "device allocation of the SDF failed");
        c->sdf_bytes = bytes;
    }
    cudaError_t e = cudaMemcpyAsync(c->sdf, data.data(), bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_boundary_set_box");
    for (int a = 0; a < 3; ++a) {
        c->sdf_left[a] = left[a];
        c->sdf_h[a] = h[a];
        c->sdf_dims[a] = dims[a];
        c->sdf_box_lo[a] = lo[a];
        c->sdf_box_hi[a] = hi[a];
    }
    c->sdf_inverted = inverted ? 1 : 0;
    c->has_sdf = true;
    return PK_OK;
}

PK_API int pk_boundary_constrain(pk_ctx* c, float* x, float* v, int n, float normal_friction,
                                 float tangential_friction, float dt, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (!c->has_sdf) return fail(c, PK_ERR_STATE, "no boundary box set");
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    cudaSetDevice(c->device);
    c->launches = pk::boundary_aos(x, v, n, pk::sdf_view(c), normal_friction, tangential_friction, dt,
                                   (cudaStream_t)stream);
    return check_launch(c, "pk_boundary_constrain");
}

PK_API int pk_boundary_jitter(pk_ctx* c, int n, float* out, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || (n > 0 && !out)) return fail(c, PK_ERR_ARG, "bad jitter output");
    cudaSetDevice(c->device);
    c->launches = pk::boundary_jitter(out, n, (cudaStream_t)stream);
    return check_launch(c, "pk_boundary_jitter");
}

// ======================================================================
// fused fluid step

namespace {

// One frame for one scene, or for several scenes concatenated in caller order
// (scene_off: device offsets, nscenes + 1 entries) that share the parameters.
// Reads the trial frame's build and solve times (this synchronises the
// stream) and, after the last trial, keeps the fastest shapes.
void tune_record(pk_ctx* c, int trial)
{
    auto& t = c->tune;
    float build = 0.f, solve = 0.f;
    if (cudaEventSynchronize(t.ev[3]) != cudaSuccess || cudaEventElapsedTime(&build, t.ev[0], t.ev[1]) != cudaSuccess ||
        cudaEventElapsedTime(&solve, t.ev[2], t.ev[3]) != cudaSuccess) {
        cudaGetLastError();
        t.on = false;
        t.pass_block = 256;
        t.persist = false;
        t.build_pb = 8;
        return;
    }
    const int pi = t.persist ? 3 : (t.pass_block == 128 ? 0 : (t.pass_block == 512 ? 2 : 1));
    const int bi = t.build_pb == 8 ? 1 : (t.build_pb == 4 ? 2 : 0);
    if (t.pass_ms[pi] == 0.f || solve < t.pass_ms[pi]) t.pass_ms[pi] = solve;
    if (t.build_ms[bi] == 0.f || build < t.build_ms[bi]) t.build_ms[bi] = build;
    t.frame = trial + 2;
    if (trial < 3) return;
    int best = 1;
    for (int k = 0; k < 4; ++k)
        if (t.pass_ms[k] < t.pass_ms[best]) best = k;
    t.pass_block = best == 0 ? 128 : (best == 2 ? 512 : 256);
    t.persist = best == 3;
    int bb = 0;
    for (int k = 1; k < 3; ++k)
        if (t.build_ms[k] < t.build_ms[bb]) bb = k;
    t.build_pb = bb == 1 ? 8 : (bb == 2 ? 4 : 16);
    t.on = false;
}

int pbf_step_impl(pk_ctx* c, float* x, float* v, int n, const pk_pbf_params* p, float* rho_out,
                  const int* scene_off, int nscenes, pk_stream stream, const char* what)
{
    if (!c) return PK_ERR_ARG;
    if (!p) return fail(c, PK_ERR_ARG, "null step parameters");
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    if (n > (1 << 29)) return fail(c, PK_ERR_ARG, "more than 2^29 particles");
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    int rc = check_nq(c, &p->nq);
    if (rc || (rc = check_pbd(c, &p->pbd))) return rc;
    if (p->boundary && !c->has_sdf) return fail(c, PK_ERR_STATE, "boundary requested but no box set");
    cudaSetDevice(c->device);
    cudaStream_t st = (cudaStream_t)stream;
    pk::Grid g = pk::make_grid(p->nq.radius, p->nq.lo, p->nq.hi);
    if (nscenes > 1) {
        if ((long long)nscenes * g.scene_keys > (1LL << 30))
            return fail(c, PK_ERR_ARG, "scenes x cells per scene exceeds 2^30 keys");
        g.nscenes = nscenes;
        g.scene_off = scene_off;
        g.nkeys = (long long)nscenes * g.scene_keys;
    }
    const int row_cap = row_capacity(&p->nq);
    if ((rc = ensure_particles(c, n)) || (rc = ensure_keys(c, g.nkeys + 1, n)) ||
        (rc = ensure_rows(c, pk::row_slots(n, row_cap))) || (rc = ensure_pool(c, n)))
        return rc;
    pk::SdfView sv{};
    if (p->boundary) sv = pk::sdf_view(c);
    // autotuning: this frame's trial shapes (4 frames: pass blocks 128, 256,
    // 512 and 256 as a resident grid walking scene tiles; build passes of 4,
    // 8 and 16 particles)
    static const int kTrialPass[4] = {128, 256, 512, 256}, kTrialBuild[4] = {16, 8, 4, 16};
    // (the first frame after pk_ctx_autotune runs the current shapes untimed:
    // it pays the one-time costs, first kernel loads and scratch growth,
    // that would otherwise land on the first trial)
    const int trial = c->tune.on ? c->tune.frame - 1 : -1;
    if (trial >= 0) {
        c->tune.pass_block = kTrialPass[trial];
        c->tune.persist = trial == 3;
        c->tune.build_pb = kTrialBuild[trial];
    }
    // The build state is recorded before anything is launched: the solver
    // passes read the row stride from the context.
    c->nq_valid = false;
    c->grid = g;
    c->nq_n = n;
    c->nq_cap = p->nq.cap;
    c->row_cap = row_cap;
    c->nq_h = p->nq.radius;
    c->exported_index = nullptr;
    c->exported_elements = nullptr;
    // StaticBoundary::advance, then ParticleIntegrator::begin (force zeroed),
    // NeighborQuery::compute on the current positions, integrate, DensityPBD.
    int l = pk::sort_particles(c, x, v, nullptr, n, g, p->boundary != 0, p->boundary ? &sv : nullptr,
                               p->normal_friction, p->tangential_friction, p->pbd.dt, true,
                               p->gravity, st);
    l += pk::build_rows(c, n, g, p->nq.radius, p->nq.cap, row_cap, nullptr, nullptr, 0, st);
    l += pk::pbd_fast_solve(c, n, pk::make_spiky(p->pbd.smoothing_length), effective_mass(&p->pbd),
                            p->pbd.iterations, p->pbd.dt, x, v, rho_out, st, p->viscosity,
                            p->viscosity_iterations);
    c->launches = l;
    if ((rc = check_launch(c, what))) return rc;
    c->nq_valid = true;  // for batched scenes: the union of the scenes' lists
    if (trial >= 0)
        tune_record(c, trial);
    else if (c->tune.on)
        c->tune.frame = 1;
    return PK_OK;
}

}  // namespace

PK_API int pk_pbf_step(pk_ctx* c, float* x, float* v, int n, const pk_pbf_params* p, float* rho_out,
                       pk_stream stream)
{
    return pbf_step_impl(c, x, v, n, p, rho_out, nullptr, 1, stream, "pk_pbf_step");
}

PK_API int pk_pbf_step_host(pk_ctx* c, float* x, float* v, int n, const pk_pbf_params* p, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || (n > 0 && (!x || !v)) || !p) return fail(c, PK_ERR_ARG, "pk_pbf_step_host: bad arguments");
    cudaSetDevice(c->device);
    if (n > c->h_cap) {
        if (!(regrow(c->h_x, 3 * (size_t)n) && regrow(c->h_v, 3 * (size_t)n))) {
            c->h_cap = 0;
            return fail(c, PK_ERR_NOMEM, "pk_pbf_step_host: out of device memory");
        }
        c->h_cap = n;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = sizeof(float) * 3 * (size_t)n;
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMemcpyAsync(c->h_x, x, bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->h_v, v, bytes, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(c, e, "pk_pbf_step_host: copy in");
    }
    int rc = pbf_step_impl(c, c->h_x, c->h_v, n, p, nullptr, nullptr, 1, stream, "pk_pbf_step_host");
    if (rc != PK_OK) return rc;
    if (n > 0) {
        e = cudaMemcpyAsync(x, c->h_x, bytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(v, c->h_v, bytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(c, e, "pk_pbf_step_host: copy out");
    }
    return PK_OK;
}

PK_API int pk_pbf_step_batched(pk_ctx* c, float* x, float* v, const int* scene_offsets, int nscenes,
                               int n, const pk_pbf_params* p, float* rho_out, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (nscenes < 1 || (nscenes > 1 && !scene_offsets))
        return fail(c, PK_ERR_ARG, "need at least one scene and its offsets");
    return pbf_step_impl(c, x, v, n, p, rho_out, scene_offsets, nscenes, stream, "pk_pbf_step_batched");
}

// ======================================================================
// differentiable DensityPBD rollouts

namespace {

// Hits per particle the rollout's rows hold.  Its frames keep every step's
// rows for the reverse pass, so a longer row is a capacity error there
// instead of continuing in the spill pool as in pk_pbf_step.
constexpr int kRollRowCap = 128;

int pbd_roll_check(pk_ctx* c, int n, const pk_pbf_params* p, int steps, int every, const void* x,
                   const void* v)
{
    if (!p) return fail(c, PK_ERR_ARG, "null step parameters");
    if (n <= 0 || n > (1 << 29)) return fail(c, PK_ERR_ARG, "particle count must be in [1, 2^29]");
    if (!x || !v) return fail(c, PK_ERR_ARG, "null positions or velocities");
    if (steps < 0 || every < 0) return fail(c, PK_ERR_ARG, "negative step or checkpoint count");
    int rc = check_nq(c, &p->nq);
    if (rc || (rc = check_pbd(c, &p->pbd))) return rc;
    if (p->boundary || p->viscosity > 0.0f)
        return fail(c, PK_ERR_ARG, "the differentiable frame has no boundary and no viscosity");
    if (p->nq.cap > kRollRowCap) return fail(c, PK_ERR_ARG, "cap above the rollout's 128 hits per particle");
    cudaSetDevice(c->device);
    const pk::Grid g = pk::make_grid(p->nq.radius, p->nq.lo, p->nq.hi);
    if ((rc = ensure_particles(c, n)) || (rc = ensure_keys(c, g.nkeys + 1, n)) ||
        (rc = ensure_rows(c, pk::row_slots(n, kRollRowCap))))
        return rc;
    return PK_OK;
}

template <class T>
int pbd_rollout_entry(pk_ctx* c, T* x, T* v, int n, const pk_pbf_params* p, int steps, int every,
                      pk_stream stream, const char* what)
{
    if (!c) return PK_ERR_ARG;
    int rc = pbd_roll_check(c, n, p, steps, every, x, v);
    if (rc) return rc;
    const int l = pk::pbd_rollout_impl<T>(c, x, v, n, p, steps, every, kRollRowCap, (cudaStream_t)stream);
    if (l < 0) return fail(c, PK_ERR_NOMEM, "device allocation of the rollout record failed");
    c->launches = l;
    return check_launch(c, what);
}

template <class T>
int pbd_backward_entry(pk_ctx* c, const T* xbar, const T* vbar, T* gx, T* gv, pk_stream stream, const char* what)
{
    if (!c) return PK_ERR_ARG;
    if (!xbar || !gx || !gv) return fail(c, PK_ERR_ARG, "null gradient arrays");
    cudaSetDevice(c->device);
    const int l = pk::pbd_backward_impl<T>(c, xbar, vbar, gx, gv, (cudaStream_t)stream);
    if (l == -2) return fail(c, PK_ERR_STATE, "no rollout of this precision recorded on the context");
    if (l < 0) return fail(c, PK_ERR_NOMEM, "device allocation of the reverse pass failed");
    c->launches = l;
    return check_launch(c, what);
}

}  // namespace

PK_API int pk_pbd_rollout(pk_ctx* c, float* x, float* v, int n, const pk_pbf_params* p, int steps,
                          int checkpoint_every, pk_stream stream)
{
    return pbd_rollout_entry<float>(c, x, v, n, p, steps, checkpoint_every, stream, "pk_pbd_rollout");
}

PK_API int pk_pbd_rollout_backward(pk_ctx* c, const float* xbar, const float* vbar, float* grad_x0, float* grad_v0,
                                   pk_stream stream)
{
    return pbd_backward_entry<float>(c, xbar, vbar, grad_x0, grad_v0, stream, "pk_pbd_rollout_backward");
}

PK_API int pk_pbd_rollout_f64(pk_ctx* c, double* x, double* v, int n, const pk_pbf_params* p, int steps,
                              int checkpoint_every, pk_stream stream)
{
    return pbd_rollout_entry<double>(c, x, v, n, p, steps, checkpoint_every, stream, "pk_pbd_rollout_f64");
}

PK_API int pk_pbd_rollout_backward_f64(pk_ctx* c, const double* xbar, const double* vbar, double* grad_x0,
                                       double* grad_v0, pk_stream stream)
{
    return pbd_backward_entry<double>(c, xbar, vbar, grad_x0, grad_v0, stream, "pk_pbd_rollout_backward_f64");
}

// ======================================================================
// a frame recorded as a CUDA graph

PK_API int pk_graph_release(pk_ctx* c)
{
    if (!c) return PK_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    return PK_OK;
}

PK_API int pk_graph_capture(pk_ctx* c, float* x, float* v, const int* scene_offsets, int nscenes, int n,
                            const pk_pbf_params* p, float* rho_out, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (nscenes < 1 || (nscenes > 1 && !scene_offsets))
        return fail(c, PK_ERR_ARG, "need at least one scene and its offsets");
    if (c->tune.on || c->prof) return fail(c, PK_ERR_STATE, "autotuning or profiling is on");
    cudaSetDevice(c->device);
    pk_graph_release(c);
    // one frame as usual: grows every buffer the frame touches
    int rc = pbf_step_impl(c, x, v, n, p, rho_out, nscenes > 1 ? scene_offsets : nullptr, nscenes, stream,
                           "pk_graph_capture");
    if (rc != PK_OK) return rc;
    cudaError_t e = cudaSuccess;
    if (!c->capture_stream) e = cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking);
    // the capture stream starts after the warm frame
    cudaEvent_t ready = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->capture_stream, ready, 0);
    if (ready) cudaEventDestroy(ready);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(c->capture_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_graph_capture: begin");
    rc = pbf_step_impl(c, x, v, n, p, rho_out, nscenes > 1 ? scene_offsets : nullptr, nscenes,
                       (pk_stream)c->capture_stream, "pk_graph_capture");
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(c->capture_stream, &g);
    if (rc != PK_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_graph_capture: end");
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(c, e, "pk_graph_capture: instantiate");
    }
    c->graph = g;
    c->graph_exec = ex;
    return PK_OK;
}

PK_API int pk_graph_launch(pk_ctx* c, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (!c->graph_exec) return fail(c, PK_ERR_STATE, "no frame recorded (pk_graph_capture)");
    cudaSetDevice(c->device);
    cudaError_t e = cudaGraphLaunch(c->graph_exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_graph_launch");
    return PK_OK;
}

// ======================================================================
// ImplicitViscosity

PK_API int pk_viscosity(pk_ctx* c, const float* x, float* v, int n, const int* index, const int* elements, int cap,
                        long long total, float viscosity, float smoothing_length, int iterations, float dt,
                        pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0 || iterations < 0) return fail(c, PK_ERR_ARG, "negative particle or iteration count");
    if (!(smoothing_length > 0.0f) || !(dt > 0.0f) || viscosity < 0.0f)
        return fail(c, PK_ERR_ARG, "bad smoothing length, dt or viscosity");
    int rc = check_list(c, n, index, elements, cap, total);
    if (rc) return rc;
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    cudaSetDevice(c->device);
    if ((rc = ensure_generic(c, n))) return rc;
    c->launches = pk::viscosity_generic(c, x, v, n, index, elements, cap, total, viscosity, smoothing_length,
                                        iterations, dt, (cudaStream_t)stream);
    return check_launch(c, "pk_viscosity");
}

// ======================================================================
// ElasticityModule

PK_API int pk_pd_init(pk_ctx* c, const float* x, int n, const int* index, const int* elements, int cap,
                      long long total, float horizon, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (n < 0) return fail(c, PK_ERR_ARG, "negative particle count");
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    int rc = check_list(c, n, index, elements, cap, total);
    if (rc) return rc;
    if (!(horizon > 0.0f)) return fail(c, PK_ERR_ARG, "horizon must be positive");
    cudaSetDevice(c->device);
    long long bonds = cap > 0 ? (long long)n * cap : total;
    if (n > c->pd_cap_n) {
        size_t m = (size_t)n;
        if (!(regrow(c->pd_index, m) && regrow(c->pd_invK, 9 * m) && regrow(c->pd_bulk, m) &&
              regrow(c->pd_xold, 3 * m) && regrow(c->pd_delta, 3 * m) && regrow(c->pd_w, m) && regrow(c->pd_ktw, m) &&
              regrow(c->pd_in_cnt, m + 1) && regrow(c->pd_in_off, m + 1))) {
            c->pd_cap_n = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of elasticity state failed");
        }
        c->pd_cap_n = n;
    }
    if (bonds > c->pd_cap_rest) {
        if (!(regrow(c->pd_rest_idx, (size_t)bonds) && regrow(c->pd_rest_pos, 3 * (size_t)bonds))) {
            c->pd_cap_rest = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of the rest shape failed");
        }
        c->pd_cap_rest = bonds;
    }
    if (bonds > c->pd_cap_bonds) {
        if (!(regrow(c->pd_alive, (size_t)bonds) && regrow(c->pd_in, (size_t)bonds) &&
              regrow(c->pd_in_slot, (size_t)bonds))) {
            c->pd_cap_bonds = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of the bond masks failed");
        }
        c->pd_cap_bonds = bonds;
    }
    c->pd_n = n;
    c->pd_begun = false;
    if (c->pl_yield && n > 0 && n <= c->pl_cap_n)  // m_bYield.reset() (ElastoplasticityModule.cu:665)
        cudaMemsetAsync(c->pl_yield, 0, (size_t)n, (cudaStream_t)stream);
    c->pd_cap = cap;
    c->pd_total = bonds;
    c->pd_horizon = horizon;
    if (bonds > (1LL << 31) - 1) return fail(c, PK_ERR_ARG, "more than 2^31 bonds");
    long long parts = pk::scan_parts_needed(n + 1);
    if (parts > c->cap_part) {
        if (!regrow(c->scan_part, (size_t)parts)) {
            c->cap_part = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of scan partials failed");
        }
        c->cap_part = parts;
    }
    pk::pd_rest_shape(c, x, n, index, elements, cap, bonds, horizon, (cudaStream_t)stream);
    if (n > 0) pk::pd_build_incoming(c, (cudaStream_t)stream);
    return check_launch(c, "pk_pd_init");
}

PK_API int pk_pd_set_bulk(pk_ctx* c, const float* bulk, int n, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    if (n != c->pd_n || (n > 0 && !bulk)) return fail(c, PK_ERR_ARG, "bulk size does not match");
    cudaSetDevice(c->device);
    cudaError_t e = cudaMemcpyAsync(c->pd_bulk, bulk, sizeof(float) * (size_t)n,
                                    cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_pd_set_bulk");
    return PK_OK;
}

PK_API int pk_pd_solve(pk_ctx* c, float* x, float* v, int n, const pk_pd_params* p, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (!p) return fail(c, PK_ERR_ARG, "null elasticity parameters");
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    if (n != c->pd_n) return fail(c, PK_ERR_ARG, "particle count differs from pk_pd_init");
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    if (!(p->horizon > 0.0f) || !(p->dt > 0.0f) || p->iterations < 0)
        return fail(c, PK_ERR_ARG, "bad horizon, dt or iterations");
    cudaSetDevice(c->device);
    c->launches = pk::pd_solve(c, x, v, n, p->horizon, p->mu, p->lambda, p->iterations, p->dt,
                               p->break_stretch, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_NOMEM, "device allocation of the projection workspace failed");
    return check_launch(c, "pk_pd_solve");
}

namespace {
int check_rollout(pk_ctx* c, int n, const void* x, const void* v, const pk_pd_params* p, int steps, int every)
{
    if (!p) return fail(c, PK_ERR_ARG, "null elasticity parameters");
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    if (n != c->pd_n) return fail(c, PK_ERR_ARG, "particle count differs from pk_pd_init");
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    if (!(p->horizon > 0.0f) || !(p->dt > 0.0f) || p->iterations < 0 || steps < 0 || every < 0)
        return fail(c, PK_ERR_ARG, "bad horizon, dt, iterations, steps or checkpoint interval");
    if (p->break_stretch > 0.0f)
        return fail(c, PK_ERR_ARG, "bond breaking is not differentiable: break_stretch must be 0 in a rollout");
    return PK_OK;
}
}  // namespace

PK_API int pk_pd_rollout(pk_ctx* c, float* x, float* v, int n, const float gravity[3], const pk_pd_params* p,
                         int steps, int checkpoint_every, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_rollout(c, n, x, v, p, steps, checkpoint_every);
    if (rc) return rc;
    if (!gravity) return fail(c, PK_ERR_ARG, "null gravity");
    cudaSetDevice(c->device);
    c->pd_horizon_last = p->horizon;
    c->pd_mu_last = p->mu;
    c->pd_lambda_last = p->lambda;
    c->launches = pk::pd_rollout_f32(c, x, v, n, gravity, p, steps, checkpoint_every, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_NOMEM, "device allocation of the rollout state failed");
    return check_launch(c, "pk_pd_rollout");
}

PK_API int pk_pd_rollout_backward(pk_ctx* c, const float* xbar, const float* vbar, float* grad_x0, float* grad_v0,
                                  double* grad_bulk, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n > 0 && (!xbar || !grad_x0 || !grad_v0 || !grad_bulk))
        return fail(c, PK_ERR_ARG, "null adjoint or gradient arrays");
    cudaSetDevice(c->device);
    c->launches = pk::pd_backward_f32(c, xbar, vbar, grad_x0, grad_v0, grad_bulk, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_STATE, "no checkpointed float rollout to differentiate");
    return check_launch(c, "pk_pd_rollout_backward");
}

PK_API int pk_pd_rollout_f64(pk_ctx* c, double* x, double* v, const double* bulk, int n, const double gravity[3],
                             const pk_pd_params* p, int steps, int checkpoint_every, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_rollout(c, n, x, v, p, steps, checkpoint_every);
    if (rc) return rc;
    if (!gravity || (n > 0 && !bulk)) return fail(c, PK_ERR_ARG, "null gravity or bulk");
    cudaSetDevice(c->device);
    c->pd_horizon_last = p->horizon;
    c->pd_mu_last = p->mu;
    c->pd_lambda_last = p->lambda;
    c->launches = pk::pd_rollout_f64(c, x, v, bulk, n, gravity, p, steps, checkpoint_every, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_NOMEM, "device allocation of the rollout state failed");
    return check_launch(c, "pk_pd_rollout_f64");
}

PK_API int pk_pd_rollout_backward_f64(pk_ctx* c, const double* xbar, const double* vbar, double* grad_x0,
                                      double* grad_v0, double* grad_bulk, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n > 0 && (!xbar || !grad_x0 || !grad_v0 || !grad_bulk))
        return fail(c, PK_ERR_ARG, "null adjoint or gradient arrays");
    cudaSetDevice(c->device);
    c->launches = pk::pd_backward_f64(c, xbar, vbar, grad_x0, grad_v0, grad_bulk, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_STATE, "no checkpointed double rollout to differentiate");
    return check_launch(c, "pk_pd_rollout_backward_f64");
}

// ======================================================================
// ElasticityModule step by step, ElastoplasticityModule, FractureModule

namespace {
int check_pd(pk_ctx* c, int n)
{
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    if (n != c->pd_n) return fail(c, PK_ERR_ARG, "particle count differs from pk_pd_init");
    return PK_OK;
}

int check_pd_params(pk_ctx* c, const pk_pd_params* p)
{
    if (!p) return fail(c, PK_ERR_ARG, "null elasticity parameters");
    if (!(p->horizon > 0.0f)) return fail(c, PK_ERR_ARG, "horizon must be positive");
    if (p->break_stretch > 0.0f) return fail(c, PK_ERR_ARG, "break_stretch must be 0 for step-by-step solves");
    return PK_OK;
}

int check_plastic(pk_ctx* c, int n, const float* x, const pk_plastic_params* p)
{
    int rc = check_pd(c, n);
    if (rc) return rc;
    if (!p) return fail(c, PK_ERR_ARG, "null plasticity parameters");
    if (!(p->horizon > 0.0f)) return fail(c, PK_ERR_ARG, "horizon must be positive");
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    return PK_OK;
}

// The yield state of ElastoplasticityModule::initializeImpl (m_bYield reset,
// ElastoplasticityModule.cu:659-668), allocated on first use.
int ensure_plastic(pk_ctx* c)
{
    const int n = c->pd_n;
    if (n <= c->pl_cap_n && c->pl_y1) return PK_OK;
    const size_t m = (size_t)std::max(n, 1);
    if (!(regrow(c->pl_y1, m) && regrow(c->pl_y2, m) && regrow(c->pl_i1, m) && regrow(c->pl_yield, m) &&
          regrow(c->pl_invF, 9 * m) && regrow(c->pl_mk, (size_t)pk::kPlMk * m) && regrow(c->pl_sizes, m + 1) &&
          regrow(c->pl_off, m + 1))) {
        c->pl_cap_n = 0;
        return fail(c, PK_ERR_NOMEM, "device allocation of the plasticity state failed");
    }
    cudaMemset(c->pl_yield, 0, m);
    cudaMemset(c->pl_y1, 0, sizeof(float) * m);
    cudaMemset(c->pl_y2, 0, sizeof(float) * m);
    cudaMemset(c->pl_i1, 0, sizeof(float) * m);
    c->pl_cap_n = n;
    return PK_OK;
}
}  // namespace

PK_API int pk_pd_compute_inverse_k(pk_ctx* c, float horizon, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    if (!(horizon > 0.0f)) return fail(c, PK_ERR_ARG, "horizon must be positive");
    cudaSetDevice(c->device);
    c->launches = pk::pd_inverse_k(c, horizon, (cudaStream_t)stream);
    return check_launch(c, "pk_pd_compute_inverse_k");
}

PK_API int pk_pd_begin(pk_ctx* c, const float* x, int n, const pk_pd_params* p, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_pd(c, n);
    if (rc || (rc = check_pd_params(c, p))) return rc;
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    cudaSetDevice(c->device);
    c->launches = pk::pd_begin(c, x, n, p->horizon, p->mu, p->lambda, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_NOMEM, "device allocation of the projection workspace failed");
    c->pd_begun = true;
    return check_launch(c, "pk_pd_begin");
}

PK_API int pk_pd_enforce(pk_ctx* c, float* x, int n, const pk_pd_params* p, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_pd(c, n);
    if (rc || (rc = check_pd_params(c, p))) return rc;
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    if (!c->pd_begun) return fail(c, PK_ERR_STATE, "pk_pd_begin has not been called");
    cudaSetDevice(c->device);
    c->launches = pk::pd_enforce(c, x, n, p->horizon, p->mu, p->lambda, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_STATE, "pk_pd_begin has not been called for this size");
    return check_launch(c, "pk_pd_enforce");
}

PK_API int pk_pd_update_velocity(pk_ctx* c, const float* x, float* v, int n, float dt, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_pd(c, n);
    if (rc) return rc;
    if (n > 0 && (!x || !v)) return fail(c, PK_ERR_ARG, "null positions or velocities");
    if (!(dt > 0.0f)) return fail(c, PK_ERR_ARG, "dt must be positive");
    if (!c->pd_begun) return fail(c, PK_ERR_STATE, "pk_pd_begin has not been called");
    cudaSetDevice(c->device);
    c->launches = pk::pd_update_velocity(c, x, v, n, dt, (cudaStream_t)stream);
    if (c->launches < 0) return fail(c, PK_ERR_STATE, "pk_pd_begin has not been called for this size");
    return check_launch(c, "pk_pd_update_velocity");
}

PK_API int pk_pd_rotate_rest_shape(pk_ctx* c, const float* x, int n, float horizon, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_pd(c, n);
    if (rc) return rc;
    if (!(horizon > 0.0f)) return fail(c, PK_ERR_ARG, "horizon must be positive");
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    cudaSetDevice(c->device);
    if ((rc = ensure_plastic(c))) return rc;
    c->launches = pk::pl_rotate(c, x, horizon, (cudaStream_t)stream);
    return check_launch(c, "pk_pd_rotate_rest_shape");
}

PK_API int pk_pd_apply_yielding(pk_ctx* c, const float* x, int n, const pk_plastic_params* p, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_plastic(c, n, x, p);
    if (rc) return rc;
    cudaSetDevice(c->device);
    if ((rc = ensure_plastic(c))) return rc;
    c->launches = pk::pl_yield(c, x, p, (cudaStream_t)stream);
    return check_launch(c, "pk_pd_apply_yielding");
}

PK_API int pk_pd_fracture(pk_ctx* c, const float* x, int n, const pk_plastic_params* p, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_plastic(c, n, x, p);
    if (rc) return rc;
    cudaSetDevice(c->device);
    c->launches = pk::pl_fracture(c, x, p, (cudaStream_t)stream);
    return check_launch(c, "pk_pd_fracture");
}

PK_API int pk_pd_reconstruct_rest_shape(pk_ctx* c, const float* x, int n, const int* index, const int* elements,
                                        int cap, long long total, float horizon, int reconstruct_all,
                                        pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    int rc = check_pd(c, n);
    if (rc) return rc;
    if ((rc = check_list(c, n, index, elements, cap, total))) return rc;
    if (!(horizon > 0.0f)) return fail(c, PK_ERR_ARG, "horizon must be positive");
    if (n > 0 && !x) return fail(c, PK_ERR_ARG, "null positions");
    cudaSetDevice(c->device);
    if ((rc = ensure_plastic(c))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // The yield flag is only ever raised by reconstruct_all (PM_ComputeInvariants
    // only clears it), so without it every particle keeps its bonds: once the
    // rest shape is in CSR the reconstruction copies it unchanged, and it is
    // skipped (no bond count to read back, no host synchronisation).
    if (!reconstruct_all && c->pd_cap == 0) {
        c->launches = 0;
        return PK_OK;
    }
    int l = 0;
    if (reconstruct_all) l += pk::pl_enable_all(c, st);
    l += pk::pl_recon_begin(c, x, index, cap, total, horizon, st);
    int new_total = 0;
    if (n > 0) {
        cudaError_t e = cudaMemcpyAsync(&new_total, c->pl_off + n, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(c, e, "pk_pd_reconstruct_rest_shape");
    }
    if (new_total < 0) return fail(c, PK_ERR_ARG, "more than 2^31 rest bonds");
    if (new_total > c->pl_cap_rest2) {
        if (!(regrow(c->pl_rest_idx2, (size_t)new_total) && regrow(c->pl_rest_pos2, 3 * (size_t)new_total))) {
            c->pl_cap_rest2 = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of the reconstructed rest shape failed");
        }
        c->pl_cap_rest2 = new_total;
    }
    l += pk::pl_recon_fill(c, x, index, elements, cap, total, st);
    // the new shape becomes the rest shape (CSR); the old buffers are the next spares
    std::swap(c->pd_rest_idx, c->pl_rest_idx2);
    std::swap(c->pd_rest_pos, c->pl_rest_pos2);
    std::swap(c->pd_cap_rest, c->pl_cap_rest2);
    if (new_total > c->pd_cap_bonds) {
        if (!(regrow(c->pd_alive, (size_t)new_total) && regrow(c->pd_in, (size_t)new_total) &&
              regrow(c->pd_in_slot, (size_t)new_total))) {
            c->pd_cap_bonds = 0;
            return fail(c, PK_ERR_NOMEM, "device allocation of the bond masks failed");
        }
        c->pd_cap_bonds = new_total;
    }
    if (n > 0) cudaMemcpyAsync(c->pd_index, c->pl_off, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    c->pd_cap = 0;
    c->pd_total = new_total;
    l += pk::pl_fill_alive(c, new_total, st);
    if (n > 0) l += pk::pd_build_incoming(c, st);
    c->launches = l;
    return check_launch(c, "pk_pd_reconstruct_rest_shape");
}

PK_API int pk_pd_get_yield(pk_ctx* c, float* yield_i1, float* yield_j2, float* i1, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    cudaSetDevice(c->device);
    int rc = ensure_plastic(c);
    if (rc) return rc;
    const size_t b = sizeof(float) * (size_t)c->pd_n;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (yield_i1 && b) e = cudaMemcpyAsync(yield_i1, c->pl_y1, b, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && yield_j2 && b) e = cudaMemcpyAsync(yield_j2, c->pl_y2, b, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && i1 && b) e = cudaMemcpyAsync(i1, c->pl_i1, b, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_pd_get_yield");
    return PK_OK;
}

PK_API int pk_pd_get_bulk(pk_ctx* c, float* bulk, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    cudaSetDevice(c->device);
    if (!bulk || c->pd_n == 0) return PK_OK;
    cudaError_t e = cudaMemcpyAsync(bulk, c->pd_bulk, sizeof(float) * (size_t)c->pd_n, cudaMemcpyDeviceToDevice,
                                    (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_pd_get_bulk");
    return PK_OK;
}

PK_API int pk_pd_rest_layout(pk_ctx* c, int* index, int* cap, long long* total, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    cudaSetDevice(c->device);
    if (cap) *cap = c->pd_cap;
    if (total) *total = c->pd_total;
    if (index && c->pd_n > 0) {
        cudaError_t e = cudaMemcpyAsync(index, c->pd_index, sizeof(int) * (size_t)c->pd_n, cudaMemcpyDeviceToDevice,
                                        (cudaStream_t)stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "pk_pd_rest_layout");
    }
    return PK_OK;
}

PK_API int pk_pd_get_rest_shape(pk_ctx* c, int* rest_idx, float* rest_pos, float* inv_k, pk_stream stream)
{
    if (!c) return PK_ERR_ARG;
    if (c->pd_n < 0) return fail(c, PK_ERR_STATE, "pk_pd_init has not been called");
    cudaSetDevice(c->device);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (rest_idx && c->pd_total > 0)
        e = cudaMemcpyAsync(rest_idx, c->pd_rest_idx, sizeof(int) * (size_t)c->pd_total,
                            cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && rest_pos && c->pd_total > 0)
        e = cudaMemcpyAsync(rest_pos, c->pd_rest_pos, 3 * sizeof(float) * (size_t)c->pd_total,
                            cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && inv_k && c->pd_n > 0)
        e = cudaMemcpyAsync(inv_k, c->pd_invK, 9 * sizeof(float) * (size_t)c->pd_n,
                            cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "pk_pd_get_rest_shape");
    return PK_OK;
}
