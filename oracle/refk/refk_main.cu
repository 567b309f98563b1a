// pkref_driver: runs PhysIKA's own hot-path kernels on small seeded inputs and
// writes their results, for the golden fixtures that pin the CPU restatement.
//
// TEST INFRASTRUCTURE ONLY. Built by `make -C oracle refk` into oracle/_ref/;
// run by tests/golden/make_ref_steps.py on a GPU machine.
//
//   pkref_driver nq  <in> <out>   one NeighborQuery::compute
//   pkref_driver pbf <in> <out>   PositionBasedFluidModel::step frames without
//                                 viscosity or boundary: query on the frame's
//                                 start positions, integrate, DensityPBD
//   pkref_driver pd  <in> <out>   ParticleElasticBody::advance steps: integrate,
//                                 ElasticityModule::solveElasticity
//
// Files are raw little-endian int32/float32 records in the order read below.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <vector>
#include "refk.h"

using namespace refk;

namespace {
struct In {
    FILE* f;
    explicit In(const char* p) : f(fopen(p, "rb")) { if (!f) { perror(p); exit(2); } }
    ~In() { fclose(f); }
    int i() { int v; if (fread(&v, 4, 1, f) != 1) die(); return v; }
    float r() { float v; if (fread(&v, 4, 1, f) != 1) die(); return v; }
    Coord c() { float a = r(), b = r(), d = r(); return Coord(a, b, d); }
    template <typename T> std::vector<T> arr(size_t n) {
        std::vector<T> v(n);
        if (n && fread(v.data(), sizeof(T), n, f) != n) die();
        return v;
    }
    static void die() { fprintf(stderr, "pkref_driver: short input\n"); exit(2); }
};
struct Out {
    FILE* f;
    explicit Out(const char* p) : f(fopen(p, "wb")) { if (!f) { perror(p); exit(2); } }
    ~Out() { fclose(f); }
    void i(int v) { fwrite(&v, 4, 1, f); }
    void r(float v) { fwrite(&v, 4, 1, f); }
    template <typename T> void arr(const std::vector<T>& v) { fwrite(v.data(), sizeof(T), v.size(), f); }
};
void check(cudaError_t e) { if (e != cudaSuccess) { fprintf(stderr, "CUDA: %s\n", cudaGetErrorString(e)); exit(3); } }
template <typename T> void upload(DArr<T>& d, const std::vector<T>& h) {
    d.resize((int)h.size());
    check(cudaMemcpy(d.getDataPtr(), h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
}
template <typename T> std::vector<T> download(DArr<T>& d, size_t n) {
    std::vector<T> h(n);
    if (n) check(cudaMemcpy(h.data(), d.getDataPtr(), sizeof(T) * n, cudaMemcpyDeviceToHost));
    return h;
}
std::vector<Coord> coords(const std::vector<float>& a) {
    std::vector<Coord> c(a.size() / 3);
    for (size_t k = 0; k < c.size(); k++) c[k] = Coord(a[3 * k], a[3 * k + 1], a[3 * k + 2]);
    return c;
}
std::vector<float> floats(const std::vector<Coord>& c) {
    std::vector<float> a(3 * c.size());
    for (size_t k = 0; k < c.size(); k++) { a[3 * k] = c[k][0]; a[3 * k + 1] = c[k][1]; a[3 * k + 2] = c[k][2]; }
    return a;
}
void need_multiple_of_64(int n) {
    if (n <= 0 || n % 64) { fprintf(stderr, "pkref_driver: n must be a positive multiple of 64\n"); exit(2); }
}
// The list as written to the output: index (counts or CSR offsets) and the
// elements (cap-strided or packed).
void write_list(Out& o, NList<int>& nbr, int n, int total) {
    o.i(total);
    o.arr(download(nbr.getIndex(), n));
    o.arr(download(nbr.getElements(), total));
}

int cmd_nq(const char* in_path, const char* out_path) {
    In in(in_path);
    int n = in.i(), cap = in.i();
    float h = in.r();
    Coord lo = in.c(), hi = in.c();
    need_multiple_of_64(n);
    std::vector<float> x = in.arr<float>(3 * (size_t)n);
    DArr<Coord> pos;
    upload(pos, coords(x));
    NList<int> nbr;
    int total = neighbor_query(pos, h, lo, hi, cap, nbr);
    Out o(out_path);
    write_list(o, nbr, n, total);
    return 0;
}

int cmd_pbf(const char* in_path, const char* out_path) {
    In in(in_path);
    int n = in.i(), cap = in.i(), iters = in.i(), steps = in.i(), ndump = in.i();
    float h = in.r(), spacing = in.r(), rho0 = in.r(), dt = in.r();
    Coord g = in.c(), lo = in.c(), hi = in.c();
    need_multiple_of_64(n);
    std::vector<int> dumps = in.arr<int>(ndump);
    std::vector<float> x = in.arr<float>(3 * (size_t)n), v = in.arr<float>(3 * (size_t)n);
    std::set<int> dump_set(dumps.begin(), dumps.end());

    DArr<Coord> pos, vel, force, pos_old, dpos;
    DArr<Real> rho, lambda;
    upload(pos, coords(x));
    upload(vel, coords(v));
    force.resize(n); pos_old.resize(n); dpos.resize(n); rho.resize(n); lambda.resize(n);
    Real mass = 0;
    Real factor = density_factor(spacing, h, rho0, &mass);
    Out o(out_path);
    o.r(factor);
    o.r(mass);
    for (int k = 1; k <= steps; k++) {
        NList<int> nbr;
        int total = neighbor_query(pos, h, lo, hi, cap, nbr);
        integrate(pos, vel, force, g, dt);
        check(cudaMemcpy(pos_old.getDataPtr(), pos.getDataPtr(), sizeof(Coord) * n, cudaMemcpyDeviceToDevice));
        for (int it = 0; it < iters; it++) pbd_iteration(pos, vel, nbr, rho, lambda, dpos, h, dt, factor * mass);
        pbd_update_velocity(vel, pos_old, pos, dt);
        if (dump_set.count(k)) {
            o.i(k);
            o.arr(floats(download(pos, n)));
            o.arr(floats(download(vel, n)));
            o.arr(download(rho, n));
            write_list(o, nbr, n, total);
        }
        nbr.release();
    }
    return 0;
}

int cmd_pd(const char* in_path, const char* out_path) {
    In in(in_path);
    int n = in.i(), cap = in.i(), iters = in.i(), steps = in.i(), ndump = in.i();
    float horizon = in.r(), mu = in.r(), lam = in.r(), dt = in.r();
    Coord g = in.c(), lo = in.c(), hi = in.c();
    need_multiple_of_64(n);
    std::vector<int> dumps = in.arr<int>(ndump);
    std::vector<float> x = in.arr<float>(3 * (size_t)n), v = in.arr<float>(3 * (size_t)n);
    std::vector<float> bulk_h = in.arr<float>(n);
    std::set<int> dump_set(dumps.begin(), dumps.end());

    DArr<Coord> pos, vel, force, pos_old, disp;
    DArr<Real> weights, bulk;
    DArr<Matrix> invK;
    upload(pos, coords(x));
    upload(vel, coords(v));
    upload(bulk, bulk_h);
    force.resize(n); pos_old.resize(n); disp.resize(n); weights.resize(n); invK.resize(n);
    // ElasticityModule::initializeImpl: the rest shape from the neighbourhood of
    // the initial positions (ParticleElasticBody queries it once, at set-up).
    NList<int> nbr;
    int total = neighbor_query(pos, horizon, lo, hi, cap, nbr);
    NList<NPair> shape;
    pd_rest_shape(shape, nbr, pos);
    pd_inverse_k(invK, shape, horizon);
    Out o(out_path);
    write_list(o, nbr, n, total);
    {
        std::vector<NPair> s = download(shape.getElements(), total);
        std::vector<int> idx(total);
        std::vector<float> rp(3 * (size_t)total);
        for (int k = 0; k < total; k++) {
            idx[k] = s[k].index;
            rp[3 * k] = s[k].pos[0]; rp[3 * k + 1] = s[k].pos[1]; rp[3 * k + 2] = s[k].pos[2];
        }
        o.arr(idx);
        o.arr(rp);
        std::vector<Matrix> K = download(invK, n);
        std::vector<float> kf(9 * (size_t)n);
        for (int p = 0; p < n; p++)
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) kf[9 * p + 3 * a + b] = K[p](a, b);
        o.arr(kf);
    }
    for (int k = 1; k <= steps; k++) {
        integrate(pos, vel, force, g, dt);
        check(cudaMemcpy(pos_old.getDataPtr(), pos.getDataPtr(), sizeof(Coord) * n, cudaMemcpyDeviceToDevice));
        pd_inverse_k(invK, shape, horizon);
        for (int it = 0; it < iters; it++)
            pd_enforce(pos, pos_old, disp, weights, bulk, invK, shape, horizon, mu, lam);
        pd_update_velocity(vel, pos_old, pos, dt);
        if (dump_set.count(k)) {
            o.i(k);
            o.arr(floats(download(pos, n)));
            o.arr(floats(download(vel, n)));
        }
    }
    return 0;
}
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: pkref_driver nq|pbf|pd <in> <out>\n");
        return 2;
    }
    if (!strcmp(argv[1], "nq")) return cmd_nq(argv[2], argv[3]);
    if (!strcmp(argv[1], "pbf")) return cmd_pbf(argv[2], argv[3]);
    if (!strcmp(argv[1], "pd")) return cmd_pd(argv[2], argv[3]);
    fprintf(stderr, "pkref_driver: unknown command %s\n", argv[1]);
    return 2;
}
