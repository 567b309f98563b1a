/*
 * pk_oracle.h -- CPU restatement of PhysIKA's particle-constraint hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, the
 * C++ Framework mirror, the Python wrapper) may call, link or load this code.
 * It is used by tests/ as the checker, by __graft_entry__.smoke() to check one
 * small GPU invocation, and by bench.py as the timed CPU baseline
 * (cpu_baseline / --impl reference).
 *
 * Every function restates one reference kernel or host routine and cites the
 * reference file:line it follows (paths relative to the PhysIKA source tree).
 *
 * Pinning: the reference's hot-path translation units do not compile outside
 * MSVC (oracle/Makefile says where), so the reference is not run end to end.
 * Its own compiled arithmetic is: oracle/_ref/ref_math_probe builds the
 * reference's Vector3f::norm/normalize and Kernel.h from the reference
 * sources, and tests/golden/ref_math.npz holds its outputs on a B200.  The
 * distance (norm variant 1) and the Spiky / Smooth / Corrected kernels here
 * reproduce those bit for bit (tests/test_golden_ref_cpu.py); the control
 * flow around them (grid, 27-cell walk, cap selection, Jacobi passes) is
 * restated from the source and is not pinned by a reference run.
 *
 * Precision: the neighbour query, grid and SDF are float only (the reference
 * computes them in float).  The solver functions exist in two builds of the
 * same source: suffix _f (float, the reference's precision) and _d (double,
 * the FP64 oracle of the same method, used for error statements only).
 *
 * Layout: positions/velocities/forces are AoS arrays of 3 values per particle
 * (Vector3f, 12 B stride), exactly as the reference's DeviceArray<Coord>.
 * Neighbour lists use NeighborList<int>'s two layouts (NeighborList.h:27-66):
 *   cap > 0 : index[i] = count_i, elements[i*cap + k]
 *   cap == 0: index[i] = exclusive CSR offset, elements packed, `total` entries
 */
#ifndef PK_ORACLE_H
#define PK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* GridHash geometry (GridHash.cu:46-75). */
typedef struct {
    float ds;        /* cell size = radius */
    float lo[3];     /* padded lower corner */
    int nx, ny, nz;  /* cells per axis */
} pko_grid;

void  pko_grid_setup(pko_grid* g, float h, const float lo[3], const float hi[3]);
/* Which float expression computes |a-b|.  0: ((x*x+y*y)+z*z), 1:
 * fma(z,z,fma(x,x,y*y)), 2: fma(z,z,fma(y,y,x*x)).  1 (the default) is what
 * the reference's Vector3f::norm compiles to under nvcc (pinned by
 * tests/golden/ref_math.npz); it must equal the variant the CUDA library was
 * built with for neighbour sets to be bit-exact. */
void  pko_set_norm_variant(int v);
int   pko_get_norm_variant(void);
float pko_dist3(const float* a, const float* b);
/* FixedPoints::constrain (FixedPoints.cu:110-147): x[ids[k]] = target[k],
 * v[ids[k]] = vel ? vel[k] : 0; ids outside [0, n) skipped. */
void pko_fixed_points(int n, float* x, float* v, const int* ids, const float* target, const float* vel,
                      int count);
/* FixedPoints::constrainPositionToPlane (FixedPoints.cu:150-169). */
void pko_plane_constrain(int n, float* x, const float origin[3], const float dir[3]);
/* SpikyKernel Weight/Gradient, SmoothKernel::Weight, CorrectedKernel
 * Weight/WeightRR (Kernel.h:29-142) at radii r[n], float: out5[5*i + k]. */
void  pko_kernels_f(int n, const float* r, float h, float* out5);

/* NeighborQuery::compute (NeighborQuery.cu:152-199) with GridHash::construct
 * (GridHash.cu:297-323).  Fixed mode (cap > 0) follows K_ComputeNeighborFixed
 * (NeighborQuery.cu:514-581); dynamic mode (cap == 0) follows K_CalNeighborSize
 * + scan + K_GetNeighborElements (NeighborQuery.cu:245-276,337-367,450-478).
 * Particles in one cell are visited in ascending id (the reference's order is
 * whatever its atomics produced).  In dynamic mode, pass elements == NULL to
 * obtain *total only.  Returns 0, or -1 if elem_capacity is too small. */
int pko_neighbor_query(int n, const float* x, float h, const float lo[3], const float hi[3],
                       int cap, int* index, int* elements, long long elem_capacity,
                       long long* total);

/* SummationDensity::calculateScalingFactor (SummationDensity.cu:112-138):
 * factor = 1/sum(V*W) over a lattice, mass = rho0*d^3; the kernels then use
 * factor*mass (SummationDensity.cu:104-109). */
void pko_density_scaling(float sampling, float h, float rho0, float* factor, float* mass);

/* Box SDF on a grid: BoundaryConstraint::setCube (BoundaryConstraint.cu:108-117)
 * -> DistanceField3D::setSpace (DistanceField3D.cu:194-201) + loadBox
 * (DistanceField3D.cu:266-291).  `data` must hold (nx+11)*(ny+11)*(nz+11)
 * floats, nx = floor((hi-lo)/spacing); pass data == NULL to get the dims. */
typedef struct {
    float left[3];   /* m_left */
    float h[3];      /* m_h (cell size per axis) */
    int   nx, ny, nz;/* node counts (m_distance dims) */
    int   inverted;
    float* data;     /* nx*ny*nz node values, x fastest */
} pko_sdf;
void pko_sdf_box_dims(const float lo[3], const float hi[3], float spacing, int dims[3]);
void pko_sdf_box_fill(pko_sdf* s, const float lo[3], const float hi[3], float spacing, int inverted);

/* DistanceField3D::getDistance (DistanceField3D.h:113-170). */
void pko_sdf_distance(const pko_sdf* s, const float p[3], float* d, float normal[3]);

/* K_ConstrainSDF (BoundaryConstraint.cu:29-67).  rnd[i] is the value
 * curand_uniform returns after curand_init(i, 0, 0) (CudaRand.h:12-24); the
 * generator is not restated: the table is produced by curand on a GPU. */
void pko_sdf_constrain(int n, float* x, float* v, const pko_sdf* s, const float* rnd,
                       float normal_friction, float tangential_friction, float dt);

/* ---- solver, float (_f) and double (_d) builds of the same source ---- */
#define PKO_DECLARE(real, sfx)                                                               \
void pko_summation_density##sfx(int n, const real* x, const int* index, const int* elements, \
                                int cap, long long total, real h, real mass, real* rho);     \
void pko_pbd_constrain##sfx(int n, real* x, real* v, const int* index, const int* elements,  \
                            int cap, long long total, real h, real mass, int iterations,     \
                            real dt, real* rho_out);                                         \
void pko_integrate##sfx(int n, real* x, real* v, const real* f, const real g[3], real dt);  \
void pko_pd_rest_shape##sfx(int n, const real* x, const int* index, const int* elements,     \
                            int cap, long long total, int* rest_idx, real* rest_pos);        \
void pko_pd_inverse_k##sfx(int n, const int* index, int cap, long long total,                \
                           const real* rest_pos, real h, real* invK);                        \
void pko_pd_solve##sfx(int n, real* x, real* v, const int* index, int cap, long long total,  \
                       const int* rest_idx, const real* rest_pos, const unsigned char* alive,\
                       const real* invK, const real* bulk, real horizon, real mu,            \
                       real lambda, int iterations, real dt);                           \
void pko_pd_break##sfx(int n, const real* x, const int* index, int cap, long long total,     \
                       const int* rest_idx, const real* rest_pos, unsigned char* alive, real s); \
void pko_implicit_viscosity##sfx(int n, const real* x, real* v, const int* index,            \
                                 const int* elements, int cap, long long total, real vis,    \
                                 real h, int iterations, real dt);                           \
void pko_pd_enforce##sfx(int n, real* x, const real* xold, const int* index, int cap,        \
                         long long total, const int* rest_idx, const real* rest_pos,         \
                         const real* invK, const real* bulk, real horizon, real mu,          \
                         real lambda);                                                       \
void pko_pd_rotate_rest_shape##sfx(int n, const real* x, const int* index, int cap,          \
                                   long long total, const int* rest_idx, real* rest_pos,     \
                                   real h);                                                  \
void pko_pd_invariants##sfx(int n, const real* x, const int* index, int cap, long long total,\
                            const int* rest_idx, const real* rest_pos, const real* bulk,     \
                            real h, real A, real B, real mu, real lambda, real* yield_i1,    \
                            real* yield_j2, real* i1, unsigned char* byield);                \
void pko_pd_apply_yielding##sfx(int n, const real* x, const int* index, int cap,             \
                                long long total, const int* rest_idx, real* rest_pos,        \
                                const real* yield_i1, const real* yield_j2, const real* i1); \
void pko_pd_inverse_deformation##sfx(int n, const real* x, const int* index, int cap,        \
                                     long long total, const int* rest_idx,                   \
                                     const real* rest_pos, real h, real* invF);              \
void pko_pd_recon_sizes##sfx(int n, const unsigned char* byield, const int* nbr_index,       \
                             int nbr_cap, long long nbr_total, const int* index, int cap,    \
                             long long total, int* sizes);                                   \
void pko_pd_recon_fill##sfx(int n, const real* x, unsigned char* byield, const real* invF,   \
                            const int* nbr_index, const int* nbr_elements, int nbr_cap,      \
                            long long nbr_total, const int* index, int cap, long long total, \
                            const int* rest_idx, const real* rest_pos, const int* off,       \
                            int* new_idx, real* new_pos);                                    \
void pko_pd_fracture##sfx(int n, const real* x, const int* index, int cap, long long total,  \
                          const int* rest_idx, const real* rest_pos, real* bulk, real h,     \
                          real A, real B, real mu, real lambda);

PKO_DECLARE(float, _f)
PKO_DECLARE(double, _d)

/* Polar rotation (row-major 3x3) and V D' U^T of a symmetric positive
 * semi-definite matrix (D' = 1/D above thr, fill below): the quantities the
 * plasticity restatement takes from polarDecomposition (MatrixFunc.inl:81-98). */
void pko_polar_rotation(const float* A9, float* R9);
void pko_clamped_inverse(const float* M9, double thr, double fill, float* out9);

/* Threads used by the OpenMP loops (0 = library default). 1 = deterministic. */
void pko_set_threads(int t);
int  pko_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
