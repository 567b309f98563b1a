/*
 * pk_oracle.c -- CPU restatement of PhysIKA's particle-constraint hot path.
 * TEST INFRASTRUCTURE ONLY (see pk_oracle.h): the checker, never the product.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/Makefile).
 * -ffp-contract=off matters: every fused multiply-add below is an explicit
 * fmaf, so results do not depend on what the host compiler chooses to fuse.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "pk_oracle.h"

#define PKO_EPSILON 1e-6   /* cuda_utilities.h:30 */
#define PKO_INVALID (-1)   /* GridHash.h:13 */

static int g_norm_variant = 1;
void pko_set_norm_variant(int v) { g_norm_variant = v; }
int  pko_get_norm_variant(void) { return g_norm_variant; }

void pko_set_threads(int t)
{
#ifdef _OPENMP
    omp_set_num_threads(t > 0 ? t : omp_get_num_procs());
#else
    (void)t;
#endif
}
int pko_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Vector3f::norm() = glm::length = sqrt(dot(v, v)) (vector_3d.inl:208-212,
 * glm func_geometric.inl:64-71,95-99).  dot = (x*x + y*y) + z*z; which of the
 * products the CUDA compiler fuses is the only freedom, hence the variants. */
static inline float norm3f(float dx, float dy, float dz)
{
    switch (g_norm_variant) {
    case 0: return sqrtf((dx * dx + dy * dy) + dz * dz);
    case 2: return sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
    default: return sqrtf(fmaf(dz, dz, fmaf(dx, dx, dy * dy)));
    }
}

float pko_dist3(const float* a, const float* b)
{
    return norm3f(a[0] - b[0], a[1] - b[1], a[2] - b[2]);
}

/* ------------------------------------------------------------------ grid */

/* GridHash::setSpace (GridHash.cu:46-75): 2 cells of padding, cell = h. */
void pko_grid_setup(pko_grid* g, float h, const float lo[3], const float hi[3])
{
    const int padding = 2;
    int a;
    int n[3];
    g->ds = h;
    for (a = 0; a < 3; a++) {
        float pad = (float)padding * h;
        float nseg = (hi[a] - lo[a]) / h;
        g->lo[a] = lo[a] - pad;
        n[a] = (int)(ceilf(nseg) + 1.0f + (float)(2 * padding));
    }
    g->nx = n[0];
    g->ny = n[1];
    g->nz = n[2];
}

/* GridHash::getIndex3 (GridHash.h:55-62). */
static inline void grid_cell3(const pko_grid* g, const float* p, int c[3])
{
    c[0] = (int)floorf((p[0] - g->lo[0]) / g->ds);
    c[1] = (int)floorf((p[1] - g->lo[1]) / g->ds);
    c[2] = (int)floorf((p[2] - g->lo[2]) / g->ds);
}

/* GridHash::getIndex(i,j,k) (GridHash.h:37-44). */
static inline int grid_index(const pko_grid* g, int i, int j, int k)
{
    if (i < 0 || i >= g->nx) return PKO_INVALID;
    if (j < 0 || j >= g->ny) return PKO_INVALID;
    if (k < 0 || k >= g->nz) return PKO_INVALID;
    return i + j * g->nx + k * g->nx * g->ny;
}

/* offset1[27][3] (NeighborQuery.cu:14-41): the order cells are visited in. */
static const int k_offset[27][3] = {
    {0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {1, 0, 0}, {0, 0, -1}, {0, -1, 0}, {-1, 0, 0},
    {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1},
    {-1, 0, -1}, {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 1, 1}, {1, 1, -1},
    {1, -1, 1}, {-1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};

/* Counting-sort hash (GridHash::construct, GridHash.cu:297-323): cell_start
 * has ncell+1 entries; ids of one cell are ascending.  Particles whose cell is
 * INVALID are not inserted (GridHash.cu:85,194). */
static void build_hash(const pko_grid* g, int n, const float* x, int** cell_start_out, int** ids_out)
{
    long long ncell = (long long)g->nx * g->ny * g->nz;
    int* start = (int*)calloc((size_t)ncell + 1, sizeof(int));
    int* fill = (int*)calloc((size_t)ncell, sizeof(int));
    int* key = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* ids;
    long long c, total = 0;
    int i;
    for (i = 0; i < n; i++) {
        int c3[3];
        grid_cell3(g, x + 3 * i, c3);
        key[i] = grid_index(g, c3[0], c3[1], c3[2]);
        if (key[i] != PKO_INVALID) start[key[i] + 1]++;
    }
    for (c = 0; c < ncell; c++) start[c + 1] += start[c];
    total = start[ncell];
    ids = (int*)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    for (i = 0; i < n; i++)
        if (key[i] != PKO_INVALID) ids[start[key[i]] + fill[key[i]]++] = i;
    free(fill);
    free(key);
    *cell_start_out = start;
    *ids_out = ids;
}

int pko_neighbor_query(int n, const float* x, float h, const float lo[3], const float hi[3],
                       int cap, int* index, int* elements, long long elem_capacity,
                       long long* total)
{
    pko_grid g;
    int *start, *ids;
    int i;
    long long sum = 0;
    pko_grid_setup(&g, h, lo, hi);
    build_hash(&g, n, x, &start, &ids);

    if (cap > 0) {
        /* K_ComputeNeighborFixed (NeighborQuery.cu:514-581): keep the first
         * `cap` hits, then replace the current farthest when d < it. */
        if (elem_capacity < (long long)n * cap) { free(start); free(ids); return -1; }
#pragma omp parallel for schedule(dynamic, 256)
        for (i = 0; i < n; i++) {
            int nid[4096];
            float ndist[4096];
            int lim = cap < 4096 ? cap : 4096;
            int counter = 0, c, t, c3[3];
            const float* pi = x + 3 * i;
            grid_cell3(&g, pi, c3);
            for (c = 0; c < 27; c++) {
                int cid = grid_index(&g, c3[0] + k_offset[c][0], c3[1] + k_offset[c][1],
                                     c3[2] + k_offset[c][2]);
                if (cid < 0) continue;
                for (t = start[cid]; t < start[cid + 1]; t++) {
                    int nb = ids[t];
                    float d = pko_dist3(pi, x + 3 * nb);
                    if (d < h) {
                        if (counter < lim) {
                            nid[counter] = nb;
                            ndist[counter] = d;
                            counter++;
                        } else {
                            int maxId = 0, ne;
                            float maxDist = ndist[0];
                            for (ne = 1; ne < lim; ne++)
                                if (maxDist < ndist[ne]) { maxDist = ndist[ne]; maxId = ne; }
                            if (d < ndist[maxId]) { ndist[maxId] = d; nid[maxId] = nb; }
                        }
                    }
                }
            }
            index[i] = counter;
            for (t = 0; t < counter; t++) elements[(long long)i * cap + t] = nid[t];
        }
        if (total) *total = (long long)n * cap;
    } else {
        /* K_CalNeighborSize (NeighborQuery.cu:245-276), exclusive scan, then
         * K_GetNeighborElements (NeighborQuery.cu:337-367). */
        int* cnt = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
#pragma omp parallel for schedule(dynamic, 256)
        for (i = 0; i < n; i++) {
            int counter = 0, c, t, c3[3];
            const float* pi = x + 3 * i;
            grid_cell3(&g, pi, c3);
            for (c = 0; c < 27; c++) {
                int cid = grid_index(&g, c3[0] + k_offset[c][0], c3[1] + k_offset[c][1],
                                     c3[2] + k_offset[c][2]);
                if (cid < 0) continue;
                for (t = start[cid]; t < start[cid + 1]; t++)
                    if (pko_dist3(pi, x + 3 * ids[t]) < h) counter++;
            }
            cnt[i] = counter;
        }
        for (i = 0; i < n; i++) { index[i] = (int)sum; sum += cnt[i]; }
        if (total) *total = sum;
        if (elements != NULL) {
            if (elem_capacity < sum) { free(cnt); free(start); free(ids); return -1; }
#pragma omp parallel for schedule(dynamic, 256)
            for (i = 0; i < n; i++) {
                int j = 0, c, t, c3[3];
                const float* pi = x + 3 * i;
                grid_cell3(&g, pi, c3);
                for (c = 0; c < 27; c++) {
                    int cid = grid_index(&g, c3[0] + k_offset[c][0], c3[1] + k_offset[c][1],
                                         c3[2] + k_offset[c][2]);
                    if (cid < 0) continue;
                    for (t = start[cid]; t < start[cid + 1]; t++)
                        if (pko_dist3(pi, x + 3 * ids[t]) < h) elements[index[i] + j++] = ids[t];
                }
            }
        }
        free(cnt);
    }
    free(start);
    free(ids);
    return 0;
}

/* ------------------------------------------------------ density scaling */

/* SpikyKernel::Weight (Kernel.h:36-45), float. */
static float host_spiky_w(float r, float h)
{
    const float q = r / h;
    if (q > 1.0f) return 0.0f;
    {
        const float d = (float)(1.0 - (double)q);
        const float hh = h * h;
        return 15.0f / ((float)M_PI * hh * h) * d * d * d * 1.0f;
    }
}

void pko_density_scaling(float sampling, float h, float rho0, float* factor, float* mass)
{
    /* SummationDensity::calculateScalingFactor (SummationDensity.cu:112-138) */
    float d = sampling;
    float V = d * d * d;
    float total_weight = 0.0f;
    int half_res = (int)(h / d + 1.0f);
    int i, j, k;
    for (i = -half_res; i <= half_res; i++)
        for (j = -half_res; j <= half_res; j++)
            for (k = -half_res; k <= half_res; k++) {
                float xx = (float)i * d, yy = (float)j * d, zz = (float)k * d;
                float r = sqrtf(xx * xx + yy * yy + zz * zz);
                total_weight += V * host_spiky_w(r, h);
            }
    *factor = (float)(1.0 / (double)total_weight);
    *mass = rho0 * V;
}

/* ------------------------------------------------------------------ SDF */

void pko_sdf_box_dims(const float lo[3], const float hi[3], float spacing, int dims[3])
{
    int a;
    for (a = 0; a < 3; a++) {
        int nb = (int)floorf((hi[a] - lo[a]) / spacing); /* BoundaryConstraint.cu:111-113 */
        dims[a] = nb + 10 + 1;                           /* setSpace: Resize(nbx+1, ...) */
    }
}

static float seg_dist(const float* pos, const float* lo, const float* hi)
{
    /* DistanceToSegment (DistanceField3D.cu:14-33) */
    float seg[3], e1[3], e2[3], d1, d2, l1, l2, ln, inv;
    int a;
    for (a = 0; a < 3; a++) { seg[a] = hi[a] - lo[a]; e1[a] = pos[a] - lo[a]; e2[a] = pos[a] - hi[a]; }
    d1 = (e1[0] * seg[0] + e1[1] * seg[1]) + e1[2] * seg[2];
    if (d1 < 0.0f) return sqrtf((e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2]);
    d2 = (e2[0] * -seg[0] + e2[1] * -seg[1]) + e2[2] * -seg[2];
    if (d2 < 0.0f) return sqrtf((e2[0] * e2[0] + e2[1] * e2[1]) + e2[2] * e2[2]);
    l1 = (e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2];
    ln = sqrtf((seg[0] * seg[0] + seg[1] * seg[1]) + seg[2] * seg[2]);
    if (ln > 1.1920929e-7f) {
        inv = 1.0f / sqrtf((seg[0] * seg[0] + seg[1] * seg[1]) + seg[2] * seg[2]);
        for (a = 0; a < 3; a++) seg[a] = seg[a] * inv;
    } else {
        seg[0] = seg[1] = seg[2] = 0.0f;
    }
    l2 = (e1[0] * seg[0] + e1[1] * seg[1]) + e1[2] * seg[2];
    return sqrtf(l1 - l2 * l2);
}

static float square_dist(const float* pos, const float* lo, const float* hi, int axis)
{
    /* DistanceToSqure (DistanceField3D.cu:35-88) */
    float c1[3], c2[3], c3[3], c4[3], nrm[3], loC[2], hiC[2], p[2];
    float d1, d2, d3, d4, d5, t;
    if (axis == 0) {
        c1[0] = lo[0]; c1[1] = lo[1]; c1[2] = lo[2];
        c2[0] = lo[0]; c2[1] = hi[1]; c2[2] = lo[2];
        c3[0] = lo[0]; c3[1] = hi[1]; c3[2] = hi[2];
        c4[0] = lo[0]; c4[1] = lo[1]; c4[2] = hi[2];
        nrm[0] = 1.0f; nrm[1] = 0.0f; nrm[2] = 0.0f;
        loC[0] = lo[1]; loC[1] = lo[2]; hiC[0] = hi[1]; hiC[1] = hi[2]; p[0] = pos[1]; p[1] = pos[2];
    } else if (axis == 1) {
        c1[0] = lo[0]; c1[1] = lo[1]; c1[2] = lo[2];
        c2[0] = lo[0]; c2[1] = lo[1]; c2[2] = hi[2];
        c3[0] = hi[0]; c3[1] = lo[1]; c3[2] = hi[2];
        c4[0] = hi[0]; c4[1] = lo[1]; c4[2] = lo[2];
        nrm[0] = 0.0f; nrm[1] = 1.0f; nrm[2] = 0.0f;
        loC[0] = lo[0]; loC[1] = lo[2]; hiC[0] = hi[0]; hiC[1] = hi[2]; p[0] = pos[0]; p[1] = pos[2];
    } else {
        c1[0] = lo[0]; c1[1] = lo[1]; c1[2] = lo[2];
        c2[0] = hi[0]; c2[1] = lo[1]; c2[2] = lo[2];
        c3[0] = hi[0]; c3[1] = hi[1]; c3[2] = lo[2];
        c4[0] = lo[0]; c4[1] = hi[1]; c4[2] = lo[2];
        nrm[0] = 0.0f; nrm[1] = 0.0f; nrm[2] = 1.0f;
        loC[0] = lo[0]; loC[1] = lo[1]; hiC[0] = hi[0]; hiC[1] = hi[1]; p[0] = pos[0]; p[1] = pos[1];
    }
    d1 = seg_dist(pos, c1, c2);
    d2 = seg_dist(pos, c2, c3);
    d3 = seg_dist(pos, c3, c4);
    d4 = seg_dist(pos, c4, c1);
    t = (nrm[0] * (pos[0] - c1[0]) + nrm[1] * (pos[1] - c1[1])) + nrm[2] * (pos[2] - c1[2]);
    d5 = fabsf(t);
    if (p[0] < hiC[0] && p[0] > loC[0] && p[1] < hiC[1] && p[1] > loC[1]) return d5;
    return fminf(fminf(d1, d2), fminf(d3, d4));
}

static float box_dist(const float* pos, const float* lo, const float* hi)
{
    /* DistanceToBox (DistanceField3D.cu:90-123) */
    float corner0[3] = {lo[0], lo[1], lo[2]}, corner1[3] = {hi[0], lo[1], lo[2]};
    float corner2[3] = {hi[0], hi[1], lo[2]}, corner3[3] = {lo[0], hi[1], lo[2]};
    float corner4[3] = {lo[0], lo[1], hi[2]}, corner5[3] = {hi[0], lo[1], hi[2]};
    float corner6[3] = {hi[0], hi[1], hi[2]}, corner7[3] = {lo[0], hi[1], hi[2]};
    (void)corner1; (void)corner2; (void)corner3;
    if (pos[0] < hi[0] && pos[0] > lo[0] && pos[1] < hi[1] && pos[1] > lo[1] && pos[2] < hi[2] &&
        pos[2] > lo[2]) {
        float dx = fminf(fabsf(pos[0] - hi[0]), fabsf(pos[0] - lo[0]));
        float dy = fminf(fabsf(pos[1] - hi[1]), fabsf(pos[1] - lo[1]));
        float dz = fminf(fabsf(pos[2] - hi[2]), fabsf(pos[2] - lo[2]));
        return fminf(fminf(dx, dy), dz);
    } else {
        float dx1 = square_dist(pos, corner0, corner7, 0);
        float dx2 = square_dist(pos, corner1, corner6, 0);
        float dy1 = square_dist(pos, corner0, corner5, 1);
        float dy2 = square_dist(pos, corner3, corner6, 1);
        float dz1 = square_dist(pos, corner0, corner2, 2);
        float dz2 = square_dist(pos, corner4, corner6, 2);
        return -fminf(fminf(fminf(dx1, dx2), fminf(dy1, dy2)), fminf(dz1, dz2));
    }
}

void pko_sdf_box_fill(pko_sdf* s, const float lo[3], const float hi[3], float spacing, int inverted)
{
    int a, dims[3], i, j, k;
    float p0[3], p1[3];
    pko_sdf_box_dims(lo, hi, spacing, dims);
    for (a = 0; a < 3; a++) {
        float pad = 5.0f * spacing;
        int nb = dims[a] - 1;
        p0[a] = lo[a] - pad;
        p1[a] = hi[a] + pad;
        s->left[a] = p0[a];
        /* m_h = (p1 - p0) * (1.0 / Real(nb+1)) (DistanceField3D.cu:198) */
        s->h[a] = (p1[a] - p0[a]) * (float)(1.0 / (double)(float)(nb + 1));
    }
    s->nx = dims[0];
    s->ny = dims[1];
    s->nz = dims[2];
    s->inverted = inverted;
    if (s->data == NULL) return;
    /* K_DistanceFieldToBox (DistanceField3D.cu:266-280): sign +1 when inverted. */
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                float p[3];
                float sign = inverted ? 1.0f : -1.0f;
                p[0] = s->left[0] + (float)i * s->h[0];
                p[1] = s->left[1] + (float)j * s->h[1];
                p[2] = s->left[2] + (float)k * s->h[2];
                s->data[((long long)k * s->ny + j) * s->nx + i] = sign * box_dist(p, lo, hi);
            }
}

static inline float lerpf_(float a, float b, float alpha)
{
    return (1.0f - alpha) * a + alpha * b; /* DistanceField3D.h:81-83 */
}

void pko_sdf_distance(const pko_sdf* s, const float p[3], float* d, float normal[3])
{
    /* DistanceField3D::getDistance (DistanceField3D.h:113-170) */
    float inv[3], fp[3], alpha, beta, gamma, l;
    int i, j, k;
    const float* D = s->data;
    long long sx = 1, sy = s->nx, sz = (long long)s->nx * s->ny;
    float d000, d100, d010, d110, d001, d101, d011, d111;
    float dx00, dx10, dxy0, dx01, dx11, dxy1, d0y0, d0y1, d0yz, d1y0, d1y1, d1yz, dx0z, dx1z;
    inv[0] = (float)(1.0 / (double)s->h[0]);
    inv[1] = (float)(1.0 / (double)s->h[1]);
    inv[2] = (float)(1.0 / (double)s->h[2]);
    fp[0] = (p[0] - s->left[0]) * inv[0];
    fp[1] = (p[1] - s->left[1]) * inv[1];
    fp[2] = (p[2] - s->left[2]) * inv[2];
    i = (int)floorf(fp[0]);
    j = (int)floorf(fp[1]);
    k = (int)floorf(fp[2]);
    if (i < 0 || i >= s->nx - 1 || j < 0 || j >= s->ny - 1 || k < 0 || k >= s->nz - 1) {
        *d = s->inverted ? -100000.0f : 100000.0f;
        normal[0] = normal[1] = normal[2] = 0.0f;
        return;
    }
    alpha = fp[0] - (float)i;
    beta = fp[1] - (float)j;
    gamma = fp[2] - (float)k;
    {
        long long o = i * sx + j * sy + k * sz;
        d000 = D[o]; d100 = D[o + sx]; d010 = D[o + sy]; d110 = D[o + sx + sy];
        d001 = D[o + sz]; d101 = D[o + sx + sz]; d011 = D[o + sy + sz]; d111 = D[o + sx + sy + sz];
    }
    dx00 = lerpf_(d000, d100, alpha);
    dx10 = lerpf_(d010, d110, alpha);
    dxy0 = lerpf_(dx00, dx10, beta);
    dx01 = lerpf_(d001, d101, alpha);
    dx11 = lerpf_(d011, d111, alpha);
    dxy1 = lerpf_(dx01, dx11, beta);
    d0y0 = lerpf_(d000, d010, beta);
    d0y1 = lerpf_(d001, d011, beta);
    d0yz = lerpf_(d0y0, d0y1, gamma);
    d1y0 = lerpf_(d100, d110, beta);
    d1y1 = lerpf_(d101, d111, beta);
    d1yz = lerpf_(d1y0, d1y1, gamma);
    dx0z = lerpf_(dx00, dx01, gamma);
    dx1z = lerpf_(dx10, dx11, gamma);
    normal[0] = d0yz - d1yz;
    normal[1] = dx0z - dx1z;
    normal[2] = dxy0 - dxy1;
    l = sqrtf((normal[0] * normal[0] + normal[1] * normal[1]) + normal[2] * normal[2]);
    if (l < 0.0001f) {
        normal[0] = normal[1] = normal[2] = 0.0f;
    } else {
        /* Vector::normalize (vector_3d.inl:220-224): v * inversesqrt(dot) */
        float is = 1.0f / sqrtf((normal[0] * normal[0] + normal[1] * normal[1]) + normal[2] * normal[2]);
        normal[0] *= is; normal[1] *= is; normal[2] *= is;
    }
    *d = (1.0f - gamma) * dxy0 + gamma * dxy1;
}

void pko_sdf_constrain(int n, float* x, float* v, const pko_sdf* s, const float* rnd,
                       float normal_friction, float tangential_friction, float dt)
{
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++) {
        float* pos = x + 3 * i;
        float* vec = v + 3 * i;
        float dist, nrm[3];
        pko_sdf_distance(s, pos, &dist, nrm);
        if (dist <= 0.0f) {
            /* BoundaryConstraint.cu:48-63 */
            float olddist = -dist, vn, vnor[3], vtan[3], f;
            int a;
            dist = 0.0001f * rnd[i];
            for (a = 0; a < 3; a++) pos[a] -= (olddist + dist) * nrm[a];
            vn = (vec[0] * nrm[0] + vec[1] * nrm[1]) + vec[2] * nrm[2];
            for (a = 0; a < 3; a++) { vnor[a] = vn * nrm[a]; vtan[a] = vec[a] - vnor[a]; }
            if (vn > 0.0f) for (a = 0; a < 3; a++) vnor[a] = -vnor[a];
            for (a = 0; a < 3; a++) vnor[a] *= (1.0f - normal_friction);
            f = powf((float)M_E, -dt * tangential_friction);
            for (a = 0; a < 3; a++) vec[a] = (vnor[a] + vtan[a]) * f;
        }
    }
}

/* ----------------------------------------- solver: float and double builds */
#define real float
#define SFX(name) name##_f
#define RSQRT sqrtf
#define FMA fmaf
#include "pk_oracle_solver.inc"
#include "pk_oracle_plastic.inc"
#undef real
#undef SFX
#undef RSQRT
#undef FMA

/* FixedPoints (FixedPoints.cu:126-162): pins and the plane constraint. */
void pko_fixed_points(int n, float* x, float* v, const int* ids, const float* target, const float* vel,
                      int count)
{
    int k, a;
    for (k = 0; k < count; k++) {
        const int i = ids[k];
        if (i < 0 || i >= n) continue;
        for (a = 0; a < 3; a++) {
            x[3 * i + a] = target[3 * k + a];
            v[3 * i + a] = vel ? vel[3 * k + a] : 0.0f;
        }
    }
}

void pko_plane_constrain(int n, float* x, const float origin[3], const float dir[3])
{
    int i, a;
    for (i = 0; i < n; i++) {
        const float ex = x[3 * i] - origin[0], ey = x[3 * i + 1] - origin[1], ez = x[3 * i + 2] - origin[2];
        /* glm dot as nvcc fuses it: fma(z, z', fma(x, x', y*y')) */
        const float tmp = fmaf(dir[2], ez, fmaf(dir[0], ex, dir[1] * ey));
        if (tmp < 0.0f)
            for (a = 0; a < 3; a++) x[3 * i + a] = fmaf(-tmp, dir[a], x[3 * i + a]);
    }
}

/* The polar rotation and the clamped inverse the plasticity restatement
 * forms (pk_oracle_plastic.inc), for checking against the reference's
 * compiled polarDecomposition (MatrixFunc.inl:81-98, svd3).  Row-major. */
void pko_polar_rotation(const float* A9, float* R9)
{
    double A[3][3], R[3][3];
    int a, b;
    for (a = 0; a < 3; a++)
        for (b = 0; b < 3; b++) A[a][b] = (double)A9[3 * a + b];
    polar_rotation_f(A, R);
    for (a = 0; a < 3; a++)
        for (b = 0; b < 3; b++) R9[3 * a + b] = (float)R[a][b];
}

void pko_clamped_inverse(const float* M9, double thr, double fill, float* out9)
{
    float M[3][3], O[3][3];
    int a, b;
    for (a = 0; a < 3; a++)
        for (b = 0; b < 3; b++) M[a][b] = M9[3 * a + b];
    clamped_inverse_f(M, thr, fill, O);
    for (a = 0; a < 3; a++)
        for (b = 0; b < 3; b++) out9[3 * a + b] = O[a][b];
}

/* The float kernel functions the solver uses, for checking against the
 * reference's compiled SpikyKernel / SmoothKernel / CorrectedKernel. */
void pko_kernels_f(int n, const float* r, float h, float* out5)
{
    int i;
    for (i = 0; i < n; i++) {
        out5[5 * i + 0] = spiky_w_f(r[i], h);
        out5[5 * i + 1] = spiky_g_f(r[i], h);
        out5[5 * i + 2] = smooth_w_f(r[i], h);
        out5[5 * i + 3] = corr_w_f(r[i], h);
        out5[5 * i + 4] = corr_wrr_f(r[i], h);
    }
}

#define real double
#define SFX(name) name##_d
#define RSQRT sqrt
#define FMA fma
#include "pk_oracle_solver.inc"
#include "pk_oracle_plastic.inc"
#undef real
#undef SFX
#undef RSQRT
