// pk_kernels.cuh -- host-side launchers shared between the kernel files.
#pragma once
#include "pk_boundary.cuh"
#include "pk_ctx.cuh"

namespace pk {

// pk_api.cu: event pairs around a kernel class when profiling is on.
void prof_begin(pk_ctx* c, int kind, cudaStream_t st);
void prof_end(pk_ctx* c, int kind, cudaStream_t st);

// pk_sort.cu
void exclusive_scan(const int* in, long long m, int* out, int* part, cudaStream_t st);
long long scan_parts_needed(long long m);
int scan_launches();
int sort_particles(pk_ctx* c, float* x, float* v, const float* f, int n, const Grid& g,
                   bool boundary, const SdfView* sdf, float nfric, float tfric, float dt,
                   bool integrate, const float grav[3], cudaStream_t st);

// pk_nbr.cu: the cap-nearest selection and the row emission over the sorted
// particles.  pub_index/pub_elements may be null.  With spill, rows longer
// than row_cap continue in the context's spill pool; without, they are a
// capacity error.  Returns kernels launched.
int build_rows(pk_ctx* c, int n, const Grid& g, float h, int cap, int row_cap,
               int* pub_index, int* pub_elements, long long pub_capacity, cudaStream_t st,
               bool spill = true);

// pk_pbd.cu
int pbd_fast_solve(pk_ctx* c, int n, const Spiky& k, float mass, int iterations, float dt,
                   float* x, float* v, float* rho_out, cudaStream_t st, float viscosity = 0.f,
                   int vis_iterations = 0);
int pbd_replay_solve(pk_ctx* c, int n, const Spiky& k, float mass, int iterations, float dt, float4* ys,
                     float* x, float* v, cudaStream_t st);
int viscosity_generic(pk_ctx* c, const float* x, float* v, int n, const int* index, const int* elements, int cap,
                      long long total, float vis, float h, int iterations, float dt, cudaStream_t st);
int pbd_generic_solve(pk_ctx* c, float* x, float* v, int n, const int* index, const int* elements,
                      int cap, long long total, const Spiky& k, float mass, int iterations,
                      float dt, float* rho_out, cudaStream_t st);
int pbd_generic_solve_scratch(float* x, float* v, int n, const int* index, const int* elements,
                              int cap, long long total, const Spiky& k, float mass, int iterations,
                              float dt, float* rho_out, float* rho_s, float* lam, float* dpos,
                              float* xold, int* err, cudaStream_t st);
// pk_api.cu: the mass the density kernels use (SummationDensity scaling).
float effective_mass_of(const pk_pbd_params* p);
int density_generic(const float* x, int n, const int* index, const int* elements, int cap,
                    long long total, const Spiky& k, float mass, float* rho, int* err, cudaStream_t st);
int gather_state(pk_ctx* c, const float* x, const float* v, int n, cudaStream_t st);
int integrate_aos(float* x, float* v, const float* f, int n, const float g[3], float dt,
                  cudaStream_t st);
int advect_aos(float* x, const float* v, int n, float dt, cudaStream_t st);
int velocity_from_positions(float* v, const float* x, const float* xold, int n, float dt, cudaStream_t st);
int fix_points(float* x, float* v, int n, const int* ids, const float* target, const float* vel, int count,
               int* err, cudaStream_t st);
int plane_constrain(float* x, int n, const float origin[3], const float dir[3], cudaStream_t st);
int boundary_aos(float* x, float* v, int n, const SdfView& s, float nfric, float tfric, float dt,
                 cudaStream_t st);
SdfView sdf_view(const pk_ctx* c);
int boundary_jitter(float* out, int n, cudaStream_t st);

// pk_pd_adj.cu
int pd_build_incoming(pk_ctx* c, cudaStream_t st);
int pd_inverse_k(pk_ctx* c, float horizon, cudaStream_t st);
int pd_begin(pk_ctx* c, const float* x, int n, float horizon, float mu, float lambda, cudaStream_t st);
int pd_enforce(pk_ctx* c, float* x, int n, float horizon, float mu, float lambda, cudaStream_t st);
int pd_update_velocity(pk_ctx* c, const float* x, float* v, int n, float dt, cudaStream_t st);
// pk_plastic.cu
constexpr int kPlMk = 20;  // floats per particle of the rotation scratch (pk_ctx::pl_mk)
int pl_rotate(pk_ctx* c, const float* x, float h, cudaStream_t st);
int pl_yield(pk_ctx* c, const float* x, const pk_plastic_params* p, cudaStream_t st);
int pl_fracture(pk_ctx* c, const float* x, const pk_plastic_params* p, cudaStream_t st);
int pl_enable_all(pk_ctx* c, cudaStream_t st);
int pl_recon_begin(pk_ctx* c, const float* x, const int* nindex, int ncap, long long ntotal, float h,
                   cudaStream_t st);
int pl_recon_fill(pk_ctx* c, const float* x, const int* nindex, const int* nelements, int ncap, long long ntotal,
                  cudaStream_t st);
int pl_fill_alive(pk_ctx* c, long long bonds, cudaStream_t st);
int pd_project_solve(pk_ctx* c, float* x, float* v, int n, float horizon, float mu, float lambda, int iterations,
                     float dt, cudaStream_t st);
int pd_rollout_f32(pk_ctx* c, float* x, float* v, int n, const float g[3], const pk_pd_params* p, int steps,
                   int every, cudaStream_t st);
int pd_rollout_f64(pk_ctx* c, double* x, double* v, const double* bulk, int n, const double g[3],
                   const pk_pd_params* p, int steps, int every, cudaStream_t st);
int pd_backward_f32(pk_ctx* c, const float* xbar, const float* vbar, float* gx, float* gv, double* gbulk,
                    cudaStream_t st);
int pd_backward_f64(pk_ctx* c, const double* xbar, const double* vbar, double* gx, double* gv, double* gbulk,
                    cudaStream_t st);
void pd_work_release(pk_ctx* c);

// pk_pbd_adj.cu: differentiable DensityPBD rollouts (float or double state);
// -1 when memory runs out, -2 (backward) when no matching rollout is recorded.
template <class T>
int pbd_rollout_impl(pk_ctx* c, T* x, T* v, int n, const pk_pbf_params* p, int steps, int every, int row_cap,
                     cudaStream_t st);
template <class T>
int pbd_backward_impl(pk_ctx* c, const T* xbar, const T* vbar, T* gx, T* gv, cudaStream_t st);
void pbd_roll_release(pk_ctx* c);

// pk_pd.cu
int pd_rest_shape(pk_ctx* c, const float* x, int n, const int* index, const int* elements,
                  int cap, long long total, float horizon, cudaStream_t st);
int pd_solve(pk_ctx* c, float* x, float* v, int n, float horizon, float mu, float lambda,
             int iterations, float dt, float break_stretch, cudaStream_t st);

}  // namespace pk
