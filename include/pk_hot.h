/*
 * pk_hot.h -- C ABI of the B200-native particle-constraint hot path.
 *
 * One shared library (physika-old_b200/lib/libpkhot.so) exports these
 * symbols.  Arguments are plain device pointers and sizes; no C++ or torch
 * types cross the boundary.  Every entry point returns an int status
 * (PK_OK = 0) and never frees caller memory.  Positions, velocities and
 * forces are the reference's DeviceArray<Vector3f>: 3 floats per particle,
 * 12-byte stride, in the caller's particle order.  Neighbour lists use the
 * reference's NeighborList<int> layouts (Framework/Topology/NeighborList.h:27-66):
 *   cap > 0  (fixed):   index[i] = count_i, elements[i*cap + k]
 *   cap == 0 (dynamic): index[i] = exclusive CSR offset, elements packed
 *
 * All work is enqueued on `stream` (NULL = legacy default stream) without a
 * host synchronisation, except where a function says it synchronises.
 * Conditions found on the device (a spill pool too small for the frame's
 * long rows, a list over its capacity) are latched in the context and
 * reported by pk_ctx_status().
 *
 * Reference paths below are relative to PhysIKA's source tree (Source/).
 */
#ifndef PK_HOT_H
#define PK_HOT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pk_ctx pk_ctx;
typedef struct CUstream_st* pk_stream; /* a cudaStream_t */

enum {
    PK_OK = 0,
    PK_ERR_ARG = 1,      /* invalid argument (null pointer, negative size, ...) */
    PK_ERR_CUDA = 2,     /* a CUDA runtime call failed */
    PK_ERR_CAPACITY = 3, /* a list or buffer capacity was exceeded */
    PK_ERR_STATE = 4,    /* call order violated (e.g. solve before init) */
    PK_ERR_NOMEM = 5     /* device allocation failed */
};

/* ------------------------------------------------------------- context */

/* Creates a context on `device`.  The context owns the module scratch (the
 * role of DensityPBD::m_lamda/m_deltaPos, GridHash::ids/counter/index,
 * ElasticityModule::m_invK/m_weights ...: DensityPBD.h:82-84,
 * GridHash.h:90-92, ElasticityModule.h:96-106).  Scratch grows on demand and
 * is kept, so steady-state steps allocate nothing. */
int pk_ctx_create(pk_ctx** out, int device);
int pk_ctx_destroy(pk_ctx* ctx);
/* Message of the last failing call on this context ("" if none). */
const char* pk_last_error(const pk_ctx* ctx);
/* Synchronises `stream`, returns and clears conditions latched on the device:
 * PK_ERR_CAPACITY if a neighbour row or list overflowed since the last call. */
int pk_ctx_status(pk_ctx* ctx, pk_stream stream);

/* ------------------------------------------------------ NeighborQuery */

typedef struct {
    float radius;      /* NeighborQuery::inRadius (NeighborQuery.h:57) */
    float lo[3];       /* scene bounds (NeighborQuery::setBoundingBox, NeighborQuery.h:30) */
    float hi[3];
    int cap;           /* setNeighborSizeLimit (NeighborQuery.h:34); 0 = dynamic list */
    int max_neighbors; /* dynamic mode: entries per particle kept in the context's main rows
                          (0 = 192, at most 4096; fixed mode keeps max(128, 2 cap)).  Not a
                          limit: longer rows continue in the context's spill pool */
} pk_nq_params;

/* NeighborQuery::compute (Framework/Topology/NeighborQuery.cu:152-199):
 * GridHash::construct (GridHash.cu:297-323) then queryNeighborFixed
 * (NeighborQuery.cu:584-605) or queryNeighborDynamic (:450-478).  Fixed mode
 * keeps the `cap` nearest; the set equals the reference's replace-the-farthest
 * result (exactly equal distances at the cap boundary are ordered
 * deterministically here, by arrival order in the reference).
 *
 * `x` is read (n AoS positions).  index/elements may be NULL (only the
 * context's internal list is built, which pk_pbd_solve/pk_pbf_step use).
 * Fixed mode writes index[n] and elements[n*cap] (elements_capacity >= n*cap).
 * Dynamic mode writes CSR offsets to index[n] and, if the total fits,
 * elements; when `total` is non-NULL this call synchronises `stream` and
 * stores the number of entries (and returns PK_ERR_CAPACITY if it exceeded
 * elements_capacity, as the reference re-sizes its list, NeighborQuery.cu:463-472).
 * Any number of particles may lie inside one radius (as for the reference):
 * rows longer than the context's row capacity continue in its spill pool, and
 * this call synchronises `stream` once to check that the pool held them,
 * growing it and repeating the build when it did not. */
int pk_nq_build(pk_ctx* ctx, const float* x, int n, const pk_nq_params* p,
                int* index, int* elements, long long elements_capacity,
                long long* total, pk_stream stream);

/* Row statistics of the context's last neighbour build (synchronises
 * `stream`): mean entries of N(i) (the capped list incl. self), mean entries
 * of the solver rows (N(i) plus the particles whose capped list holds i) and
 * the longest solver row.  No reference counterpart (measurement only). */
int pk_nq_row_stats(pk_ctx* ctx, double* mean_list, double* mean_row, int* max_row,
                    pk_stream stream);

/* ---------------------------------------------------------- DensityPBD */

typedef struct {
    float smoothing_length;  /* varSmoothingLength (DensityPBD.h:44) */
    float sampling_distance; /* varSamplingDistance (DensityPBD.h:42) */
    float rest_density;      /* varRestDensity (DensityPBD.h:40); only sets mass */
    int iterations;          /* varIterationNumber (DensityPBD.h:38) */
    float dt;                /* parent Node's dt (DensityPBD.cu:308) */
} pk_pbd_params;

/* SummationDensity::compute (Dynamics/ParticleSystem/SummationDensity.cu:58-110,
 * K_ComputeDensity :13-36) over any NeighborList<int>.  rho[n] written. */
int pk_summation_density(pk_ctx* ctx, const float* x, int n, const int* index,
                         const int* elements, int cap, long long total,
                         const pk_pbd_params* p, float* rho, pk_stream stream);

/* DensityPBD::constrain (Dynamics/ParticleSystem/DensityPBD.cu:271-302):
 * `iterations` Jacobi sweeps of density, lambda (K_ComputeLambdas :46-90) and
 * displacement (K_ComputeDisplacement :134-179, K_UpdatePosition :226-237),
 * then v += (x - x_old)/dt (DP_UpdateVelocity :367-378).  x and v are updated
 * in place; rho_out (may be NULL) receives outDensity.  When (index, elements)
 * are the arrays the last pk_nq_build on this context wrote (and n matches),
 * the solve runs on the context's sorted internal list; any other list is
 * solved as given, and a neighbour id in it outside [0, n) is skipped and
 * reported by pk_ctx_status as PK_ERR_ARG. */
int pk_pbd_solve(pk_ctx* ctx, float* x, float* v, int n, const int* index,
                 const int* elements, int cap, long long total,
                 const pk_pbd_params* p, float* rho_out, pk_stream stream);

/* ---------------------------------------------------- ParticleIntegrator */

/* ParticleIntegrator::integrate (Dynamics/ParticleSystem/ParticleIntegrator.cu:128-138):
 * v += dt*(f + g) (K_UpdateVelocity :59-70), then x += dt*v (K_UpdatePosition
 * :102-112).  f may be NULL (ParticleIntegrator::begin zeroes it, :32).  x may
 * be NULL: then only the velocity update runs (updateVelocity, :86-100). */
int pk_integrate(pk_ctx* ctx, float* x, float* v, const float* f, int n,
                 const float gravity[3], float dt, pk_stream stream);

/* ParticleIntegrator::updatePosition alone (K_UpdatePosition,
 * ParticleIntegrator.cu:102-112): x += dt*v. */
int pk_advect(pk_ctx* ctx, float* x, const float* v, int n, float dt, pk_stream stream);

/* v += (x - x_old)/dt: DensityPBD::updateVelocity (DP_UpdateVelocity,
 * DensityPBD.cu:367-392) and ElasticityModule::updateVelocity (K_UpdateVelocity,
 * ElasticityModule.cu:295-306,423-437). */
int pk_update_velocity(pk_ctx* ctx, float* v, const float* x, const float* x_old, int n,
                       float dt, pk_stream stream);

/* ---------------------------------------------------- ImplicitViscosity */

/* ImplicitViscosity::constrain (Dynamics/ParticleSystem/ImplicitViscosity.cu:98-128,
 * K_ApplyViscosity :20-62): `iterations` Jacobi sweeps of
 * v_i = v_old,i/(1+b) + (sum_j w_ij v_j / sum_j w_ij) b/(1+b) over any
 * NeighborList<int>, b = dt*viscosity/smoothing_length, w = 45/(13 pi h^3)
 * (1 - r/h) (VB_VisWeight :8-18).  x is read, v updated in place. */
int pk_viscosity(pk_ctx* ctx, const float* x, float* v, int n, const int* index, const int* elements, int cap,
                 long long total, float viscosity, float smoothing_length, int iterations, float dt,
                 pk_stream stream);

/* ---------------------------------------------------------- FixedPoints */

/* FixedPoints::constrain (Dynamics/ParticleSystem/FixedPoints.cu:110-147,
 * K_DoFixPoints :126-140): for k < count, x[ids[k]] = target[k] and
 * v[ids[k]] = 0, as the reference's pins; with vel != NULL, v[ids[k]] = vel[k]
 * instead (a pin moved kinematically, e.g. a pulled end; no reference
 * counterpart).  ids outside [0, n) are skipped and reported as PK_ERR_ARG by
 * pk_ctx_status.  target and vel are 3 floats per pin (device memory). */
int pk_fixed_points(pk_ctx* ctx, float* x, float* v, int n, const int* ids, const float* target,
                    const float* vel, int count, pk_stream stream);

/* FixedPoints::constrainPositionToPlane (FixedPoints.cu:150-169): particles
 * behind the plane through `origin` with unit normal `dir` are moved onto it. */
int pk_plane_constrain(pk_ctx* ctx, float* x, int n, const float origin[3], const float dir[3],
                       pk_stream stream);

/* ------------------------------------------------- BoundaryConstraint */

/* BoundaryConstraint::setCube (Dynamics/ParticleSystem/BoundaryConstraint.cu:108-117):
 * a box SDF on a grid of `spacing` with 5 cells of padding
 * (DistanceField3D::setSpace/loadBox, Framework/Topology/DistanceField3D.cu:194-201,266-291).
 * inverted != 0 keeps particles inside the box.  Replaces the context's box. */
int pk_boundary_set_box(pk_ctx* ctx, const float lo[3], const float hi[3], float spacing,
                        int inverted, pk_stream stream);

/* BoundaryConstraint::constrain (BoundaryConstraint.cu:84-97, K_ConstrainSDF
 * :29-67): particles with SDF distance <= 0 are projected out along the SDF
 * normal plus 1e-4*U with U = curand_uniform after curand_init(particle id,0,0),
 * their normal velocity is reflected and scaled by (1 - normal_friction). */
int pk_boundary_constrain(pk_ctx* ctx, float* x, float* v, int n, float normal_friction,
                          float tangential_friction, float dt, pk_stream stream);

/* The jitter values K_ConstrainSDF draws (BoundaryConstraint.cu:50-51):
 * out[i] = curand_uniform after curand_init(i, 0, 0) (RandNumber,
 * Core/Utility/CudaRand.h:12-24), for i < n. */
int pk_boundary_jitter(pk_ctx* ctx, int n, float* out, pk_stream stream);

/* ---------------------------------------------- fused fluid step */

typedef struct {
    pk_nq_params nq;       /* neighbour query of the step */
    pk_pbd_params pbd;     /* DensityPBD parameters (pbd.dt is the step's dt) */
    float gravity[3];      /* SceneGraph::getGravity (Framework/Framework/SceneGraph.h:57-58) */
    int boundary;          /* 1: apply the context's box boundary first */
    float normal_friction; /* BoundaryConstraint.h:32 default 0.95 */
    float tangential_friction;
    float viscosity;          /* > 0: ImplicitViscosity after the solve (the stock model sets 1, */
    int viscosity_iterations; /*      PositionBasedFluidModel.cpp:69-70, 5 sweeps); 0: off */
} pk_pbf_params;

/* One dam-break frame: StaticBoundary::advance (StaticBoundary.cpp:45-59) then
 * PositionBasedFluidModel::step (Dynamics/ParticleSystem/PositionBasedFluidModel.cpp:83-101):
 * integrator begin, NeighborQuery on the current positions, integrate,
 * DensityPBD, and ImplicitViscosity when p->viscosity > 0.
 * x, v (n AoS) are updated in place; rho_out may be NULL.  Asynchronous and
 * allocation-free once the context has seen `n` (capturable in a CUDA graph).
 * Rows longer than the row capacity continue in the context's spill pool
 * (8 entries per particle at first); a frame that needs more reports
 * PK_ERR_CAPACITY through pk_ctx_status, which records the size, and the
 * next frame runs with the pool grown to it. */
int pk_pbf_step(pk_ctx* ctx, float* x, float* v, int n, const pk_pbf_params* p,
                float* rho_out, pk_stream stream);

/* pk_pbf_step on host arrays, the view of an application that owns its
 * particles on the host and reads every frame back (the reference's
 * ParticleSystem loading and ParticleWriter dumps, ParticleWriter.cpp:49-80).
 * x, v: n AoS float triples in host memory, updated in place; page-locked
 * memory gives full PCIe speed.  Copies them into context-owned device arrays
 * (grown on first use of a larger n), runs the frame and copies the results
 * back, all on `stream`, then synchronises the stream. */
int pk_pbf_step_host(pk_ctx* ctx, float* x, float* v, int n, const pk_pbf_params* p, pk_stream stream);

/* Many independent scenes in one frame (no reference counterpart; the
 * reference steps each ParticleFluid node with its own launches).  The scenes'
 * particles are concatenated in caller order: scene s owns particles
 * [scene_offsets[s], scene_offsets[s+1]) of x, v and rho_out, with
 * scene_offsets a device array of nscenes + 1 ints (0 first, n last,
 * non-decreasing).  Every scene has its own box of the same geometry
 * (p->nq.lo/hi, the context's boundary box) and the same parameters; scenes
 * never interact.  The result for each scene is that of pk_pbf_step on that
 * scene alone (the boundary jitter is seeded by the id within the scene).
 * All scenes run in the same ~21 launches, asynchronous and allocation-free
 * once the context has seen n and nscenes, so a frame can be captured in a
 * CUDA graph. */
int pk_pbf_step_batched(pk_ctx* ctx, float* x, float* v, const int* scene_offsets, int nscenes, int n,
                        const pk_pbf_params* p, float* rho_out, pk_stream stream);

/* A frame as a CUDA graph (no reference counterpart).  pk_graph_capture
 * records one frame -- pk_pbf_step when nscenes == 1 (scene_offsets may be
 * NULL), else pk_pbf_step_batched -- with these arguments into a graph the
 * context owns, replacing any earlier one.  It first runs that frame once
 * on `stream` without capture, so every buffer the frame needs exists before
 * recording (a captured frame allocates nothing); x and v therefore advance by
 * one frame.  pk_graph_launch replays the recorded frame on `stream`: the
 * same kernels on the same pointers and parameters, one launch for the whole
 * frame.  The context's autotuning trials and profiling must be off while a
 * frame is captured (PK_ERR_STATE otherwise).  pk_graph_release frees the
 * graph; pk_ctx_destroy does too. */
int pk_graph_capture(pk_ctx* ctx, float* x, float* v, const int* scene_offsets, int nscenes, int n,
                     const pk_pbf_params* p, float* rho_out, pk_stream stream);
int pk_graph_launch(pk_ctx* ctx, pk_stream stream);
int pk_graph_release(pk_ctx* ctx);

/* Number of kernel launches the last pk_pbf_step enqueued. */
int pk_last_launch_count(const pk_ctx* ctx);

/* Autotuning of the frame kernels (no reference counterpart).  With enable,
 * the next pk_pbf_step / pk_pbf_step_batched call runs the current shapes
 * untimed (it takes the one-time costs of a first frame) and the four after it
 * are trial frames: they
 * run the Jacobi passes at 128, 256 and 512 threads per block and at 256 as a
 * resident grid walking the scene tiles (each scene's sorted range cut into
 * blocks, from the cell table), and the neighbour sweep with 4, 8 and 16
 * particles per pass, time them (each trial frame synchronises its stream, so
 * do not capture them in a graph), and keep the fastest shapes for the
 * context.  The shapes change no result.  pk_ctx_tuning reports the shapes in
 * use and whether trials remain; pk_ctx_tuning_resident whether the passes
 * run as the resident grid. */
int pk_ctx_autotune(pk_ctx* ctx, int enable);
int pk_ctx_tuning(const pk_ctx* ctx, int* pass_block, int* build_particles, int* active);
int pk_ctx_tuning_resident(const pk_ctx* ctx, int* resident);

/* Per-kernel timing with CUDA events recorded on the launching stream around
 * each kernel class of the neighbour build and the solver (no reference
 * counterpart; the reference's GTimer, Core/Utility/GTimer.h:6-23, is the
 * closest).  pk_ctx_profile(ctx, 1) clears and starts recording;
 * pk_ctx_profile_read synchronises and returns the summed milliseconds and
 * launch count of one class:
 *   0 sort (keys, cell scan, scatter, cell fix-up, gather), 1 cap selection,
 *   2 row emission, 3 density+lambda pass, 4 displacement pass, 5 write-back. */
enum { PK_PROF_SORT = 0, PK_PROF_SELECT, PK_PROF_EMIT, PK_PROF_DENSITY, PK_PROF_DISP,
       PK_PROF_FINISH, PK_PROF_KINDS };
int pk_ctx_profile(pk_ctx* ctx, int enable);
int pk_ctx_profile_read(pk_ctx* ctx, int kind, double* total_ms, int* launches);

/* ---------------------------------------------- ElasticityModule (peridynamics) */

typedef struct {
    float horizon;   /* inHorizon (ElasticityModule.h:63) */
    float mu;        /* m_mu, default 0.05 (ElasticityModule.cu:326) */
    float lambda;    /* m_lambda, default 0.1 (ElasticityModule.cu:327) */
    int iterations;  /* m_iterNum, default 10 (ElasticityModule.cu:328) */
    float dt;
    float break_stretch; /* > 0: bonds break when |x_i-x_j| > (1+s)|r_ij| (no reference counterpart) */
} pk_pd_params;

/* ElasticityModule::initializeImpl (Dynamics/ParticleSystem/ElasticityModule.cu:519-546):
 * freezes the rest shape from the neighbour list (resetRestShape +
 * K_UpdateRestShape :449-517, self moved to slot 0), sets bulk stiffness 1
 * (computeMaterialStiffness :380-387) and precomputes K^-1 once
 * (EM_PrecomputeShape :21-116; the rest shape never changes, so the
 * reference's per-step recomputation gives the same matrix). */
int pk_pd_init(pk_ctx* ctx, const float* x, int n, const int* index, const int* elements,
               int cap, long long total, float horizon, pk_stream stream);

/* The protected ElasticityModule::m_bulkCoefs (ElasticityModule.h:96) that
 * subclasses set through computeMaterialStiffness: bulk[n] is copied. */
int pk_pd_set_bulk(pk_ctx* ctx, const float* bulk, int n, pk_stream stream);

/* ElasticityModule::solveElasticity (ElasticityModule.cu:404-421): iterations
 * of EM_EnforceElasticity (:123-242) + K_UpdatePosition (:281-292), then
 * K_UpdateVelocity (:295-306).  x, v in place (n AoS). */
int pk_pd_solve(pk_ctx* ctx, float* x, float* v, int n, const pk_pd_params* p,
                pk_stream stream);

/* The steps of ElasticityModule::solveElasticity (ElasticityModule.cu:404-421)
 * one at a time, for solvers that interleave other constraints between the
 * projection iterations (ElastoplasticityModule::solveElasticity,
 * Dynamics/ParticleSystem/ElastoplasticityModule.cu:240-262, runs a one-
 * iteration DensityPBD after each):
 *   pk_pd_compute_inverse_k: K^-1 of the current rest shape (computeInverseK,
 *     ElasticityModule.cu:390-400; plasticity moves the rest shape);
 *   pk_pd_begin: m_position_old = x and the bond weights of the current bulk
 *     stiffness;
 *   pk_pd_enforce: one EM_EnforceElasticity + K_UpdatePosition against that
 *     x_old (x in place);
 *   pk_pd_update_velocity: v += (x - x_old)/dt (K_UpdateVelocity :295-306).
 * p->iterations is not used by these; p->break_stretch must be 0. */
int pk_pd_compute_inverse_k(pk_ctx* ctx, float horizon, pk_stream stream);
int pk_pd_begin(pk_ctx* ctx, const float* x, int n, const pk_pd_params* p, pk_stream stream);
int pk_pd_enforce(pk_ctx* ctx, float* x, int n, const pk_pd_params* p, pk_stream stream);
int pk_pd_update_velocity(pk_ctx* ctx, const float* x, float* v, int n, float dt, pk_stream stream);

/* ------------------------------------ ElastoplasticityModule / FractureModule */

typedef struct {
    float horizon; /* inHorizon */
    float mu;      /* ElasticityModule m_mu */
    float lambda;  /* ElasticityModule m_lambda */
    float A;       /* computeA(): 6 c cos(phi) / (3 + sin(phi)) / sqrt(3) (ElastoplasticityModule.h:53-58) */
    float B;       /* computeB(): 2 sin(phi) / (3 + sin(phi)) / sqrt(3) (:61-65) */
} pk_plastic_params;

/* ElastoplasticityModule::rotateRestShape (EM_RotateRestShape,
 * ElastoplasticityModule.cu:568-657): each particle's rest bonds rotated by
 * the polar rotation of its deformation gradient (SmoothKernel weights over
 * the rest shape). */
int pk_pd_rotate_rest_shape(pk_ctx* ctx, const float* x, int n, float horizon, pk_stream stream);

/* ElastoplasticityModule::applyYielding (:273-307): PM_ComputeInvariants
 * (:43-163, Drucker-Prager on I1 and J2 with the context's bulk stiffness)
 * then PM_ApplyYielding (:165-226, rest bonds moved by the mean yield of
 * their two ends). */
int pk_pd_apply_yielding(pk_ctx* ctx, const float* x, int n, const pk_plastic_params* p, pk_stream stream);

/* ElastoplasticityModule::reconstructRestShape (:483-531): particles flagged
 * as yielding (all of them when reconstruct_all, enableFullyReconstruction)
 * take their current neighbours (index/elements/cap/total: a NeighborList of
 * the current positions) as rest bonds placed by the inverse deformation
 * (PM_ComputeInverseDeformation :389-471, PM_ReconstructRestShape :309-371);
 * the others keep theirs.  The rest shape becomes a CSR list.  Synchronises
 * the stream (the new bond count sizes the list).  The reference raises the
 * yield flag only through reconstruct_all, so without it a CSR rest shape is
 * left as it is and the call returns at once. */
int pk_pd_reconstruct_rest_shape(pk_ctx* ctx, const float* x, int n, const int* index, const int* elements,
                                 int cap, long long total, float horizon, int reconstruct_all,
                                 pk_stream stream);

/* FractureModule::applyPlasticity (Dynamics/ParticleSystem/FractureModule.cu:107-128):
 * particles past the Drucker-Prager limit lose their bulk stiffness. */
int pk_pd_fracture(pk_ctx* ctx, const float* x, int n, const pk_plastic_params* p, pk_stream stream);

/* State readers: the yield fields of the last pk_pd_apply_yielding (n floats
 * each, any may be NULL), the bulk stiffness, and the rest-shape layout
 * (index: n counts (cap > 0) or CSR offsets (cap == 0); any may be NULL). */
int pk_pd_get_yield(pk_ctx* ctx, float* yield_i1, float* yield_j2, float* i1, pk_stream stream);
int pk_pd_get_bulk(pk_ctx* ctx, float* bulk, pk_stream stream);
int pk_pd_rest_layout(pk_ctx* ctx, int* index, int* cap, long long* total, pk_stream stream);

/* Copies the frozen rest shape out: rest_idx/rest_pos in the NeighborList
 * layout the rest shape was built with (TPair index/pos, Dynamics/ParticleSystem/NeighborData.h:6-21). */
int pk_pd_get_rest_shape(pk_ctx* ctx, int* rest_idx, float* rest_pos, float* inv_k,
                         pk_stream stream);

/* ------------------------------- differentiable peridynamics rollouts */

/* No reference counterpart.  `steps` elasticity steps on the rest shape of
 * pk_pd_init, each: v += dt*gravity, x += dt*v (ParticleIntegrator with no
 * force), then ElasticityModule::solveElasticity as in pk_pd_solve (the
 * projection's bond terms are gathered over each particle's outgoing and
 * incoming bonds, so a replay repeats the forward bit for bit).  x, v (n AoS)
 * in place; stiffness from pk_pd_set_bulk; break_stretch must be 0.  With
 * checkpoint_every > 0 the state at every checkpoint_every-th step is kept in
 * the context for pk_pd_rollout_backward. */
int pk_pd_rollout(pk_ctx* ctx, float* x, float* v, int n, const float gravity[3], const pk_pd_params* p,
                  int steps, int checkpoint_every, pk_stream stream);

/* Reverse mode of the last checkpointed pk_pd_rollout: given dL/dx_T (xbar)
 * and dL/dv_T (vbar, may be NULL), writes dL/dx_0, dL/dv_0 (n AoS) and
 * dL/dbulk (n doubles: the stiffness gradient is accumulated in double).  The
 * rollout is replayed segment by segment from its checkpoints, every
 * projection iterate of a segment is kept, and each iteration is reversed by
 * hand-written adjoint kernels.  The reverse state and its arithmetic are
 * double (the float iterates are read as given): the adjoint differences
 * neighbouring values, which float arithmetic does not carry over hundreds of
 * projection iterations. */
int pk_pd_rollout_backward(pk_ctx* ctx, const float* xbar, const float* vbar, float* grad_x0, float* grad_v0,
                           double* grad_bulk, pk_stream stream);

/* The same rollout and reverse mode in double precision (x, v, bulk doubles;
 * the rest shape and K^-1 of pk_pd_init as given): the reference against which
 * the float gradients and central finite differences are checked. */
int pk_pd_rollout_f64(pk_ctx* ctx, double* x, double* v, const double* bulk, int n, const double gravity[3],
                      const pk_pd_params* p, int steps, int checkpoint_every, pk_stream stream);
int pk_pd_rollout_backward_f64(pk_ctx* ctx, const double* xbar, const double* vbar, double* grad_x0,
                               double* grad_v0, double* grad_bulk, pk_stream stream);

/* Differentiable DensityPBD rollout (no reference counterpart: the reference
 * has no derivatives).  `steps` frames of pk_pbf_step without boundary and
 * viscosity (p->boundary and p->viscosity must be 0; each frame builds its
 * list on the frame's start positions, integrates, runs DensityPBD and
 * updates the velocity), x and v (n AoS, device) updated in place; the state
 * at the start of every checkpoint_every-th step (0: only the first) is kept
 * on the context for pk_pbd_rollout_backward.  A frame's list is a step
 * constant: the derivative is that of the frame map with the list frozen.
 * Rows hold at most 128 hits per particle (the frames' rows are kept for the
 * reverse pass, so a longer row is not spilled: pk_ctx_status reports
 * PK_ERR_CAPACITY). */
int pk_pbd_rollout(pk_ctx* ctx, float* x, float* v, int n, const pk_pbf_params* p, int steps,
                   int checkpoint_every, pk_stream stream);

/* Reverse mode of the last pk_pbd_rollout: given dL/dx_T (xbar) and dL/dv_T
 * (vbar, may be NULL), writes dL/dx_0 and dL/dv_0 (n AoS).  Each segment is
 * replayed from its checkpoint keeping every frame's rows and Jacobi iterates,
 * then every iteration, integration and velocity update is reversed by
 * hand-written kernels (the derivatives of K_ComputeLambdas' lambda, its
 * clamp, SummationDensity's density and K_ComputeDisplacement's scatter with
 * the rows' multiplicities).  The reverse state and its arithmetic are double;
 * the float iterates are read as given. */
int pk_pbd_rollout_backward(pk_ctx* ctx, const float* xbar, const float* vbar, float* grad_x0, float* grad_v0,
                            pk_stream stream);

/* The same rollout and reverse mode in double precision (lists from the
 * positions rounded to float): the reference run of the gradient checks and
 * the FP64 run the float frames are compared against. */
int pk_pbd_rollout_f64(pk_ctx* ctx, double* x, double* v, int n, const pk_pbf_params* p, int steps,
                       int checkpoint_every, pk_stream stream);
int pk_pbd_rollout_backward_f64(pk_ctx* ctx, const double* xbar, const double* vbar, double* grad_x0,
                                double* grad_v0, pk_stream stream);

/* ------------------------------------------- DensityPBD without allocation */

/* No counterpart in the reference.  For callers that may not allocate device
 * memory (a host application that owns the GPU memory budget, or a frame loop
 * that cannot take the synchronisation of cudaMalloc): the same solve as
 * pk_pbd_solve on a list that was not built by a context, with no context at
 * all.  Its scratch is one fixed device array inside the library (4 MiB, held
 * by every GPU that loads the library until exit), so n may be at most
 * pk_noalloc_max_particles() (131072); larger n returns PK_ERR_CAPACITY.
 * The first call in a CUDA context looks up the array's device address (an
 * address belongs to the context, so a call under another context, or after
 * cudaDeviceReset, looks it up again); make that first call before any stream
 * capture.  All calls share the array: calls whose work overlaps on the GPU
 * (different streams, or several host threads) race on it and must be ordered
 * by the caller.  A neighbour id outside [0, n) is skipped (there is no
 * context to report it).  Nothing is allocated or freed. */
int pk_noalloc_max_particles(void);
int pk_pbd_solve_noalloc(float* x, float* v, int n, const int* index, const int* elements,
                         int cap, long long total, const pk_pbd_params* p, float* rho_out,
                         pk_stream stream);

#ifdef __cplusplus
}
#endif
#endif
