// pk_pybind.cpp -- the pybind11 layer of the differentiable rollouts.
//
// The torch.autograd.Functions of pk_torch.py call these functions, which
// check their tensors (CUDA, contiguous, shape, dtype), take torch's current
// stream of the tensors' device and call the C ABI of include/pk_hot.h
// (pk_pd_rollout*, pk_pd_rollout_backward*, pk_pbd_rollout*,
// pk_pbd_rollout_backward*, pk_pd_set_bulk).  Tensors are handled through
// their Python interface (data_ptr, shape, dtype), so the module needs the
// Python and pybind11 headers but not torch's; it links libpkhot.so.
// A failing call raises RuntimeError("pk error <code>: <pk_last_error>").
#include <pybind11/pybind11.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/pk_hot.h"

namespace py = pybind11;

namespace {

pk_ctx* as_ctx(std::uintptr_t h)
{
    if (!h) throw std::invalid_argument("null pk context");
    return reinterpret_cast<pk_ctx*>(h);
}

void check(pk_ctx* c, int rc)
{
    if (rc != PK_OK) throw std::runtime_error("pk error " + std::to_string(rc) + ": " + pk_last_error(c));
}

py::object torch() { return py::module_::import("torch"); }

// A contiguous CUDA tensor of the given dtype and leading size n (and second
// size `cols` when cols > 0); returns its device address.
void* tensor_ptr(const py::object& t, const char* what, const py::object& dtype, long long n, long long cols)
{
    if (!t.attr("is_cuda").cast<bool>() || !t.attr("is_contiguous")().cast<bool>())
        throw std::invalid_argument(std::string(what) + ": expected a contiguous CUDA tensor");
    if (!py::object(t.attr("dtype")).equal(dtype)) throw std::invalid_argument(std::string(what) + ": wrong dtype");
    const py::tuple shape = t.attr("shape");
    const bool ok = cols > 0 ? (shape.size() == 2 && shape[0].cast<long long>() == n && shape[1].cast<long long>() == cols)
                             : (shape.size() == 1 && shape[0].cast<long long>() == n);
    if (!ok) throw std::invalid_argument(std::string(what) + ": wrong shape");
    return reinterpret_cast<void*>(t.attr("data_ptr")().cast<std::uintptr_t>());
}

// torch's current stream on the tensor's device.
pk_stream stream_of(const py::object& t)
{
    const py::object s = torch().attr("cuda").attr("current_stream")(t.attr("device"));
    return reinterpret_cast<pk_stream>(s.attr("cuda_stream").cast<std::uintptr_t>());
}

bool is_f64(const py::object& t) { return py::object(t.attr("dtype")).equal(torch().attr("float64")); }

long long rows_of(const py::object& t) { return py::tuple(t.attr("shape"))[0].cast<long long>(); }

// (Every tensor is checked before the stream is taken: no device call is made
// for a bad argument.)
void pd_set_bulk(std::uintptr_t h, const py::object& bulk)
{
    pk_ctx* c = as_ctx(h);
    const long long n = rows_of(bulk);
    const auto* b = static_cast<const float*>(tensor_ptr(bulk, "bulk", torch().attr("float32"), n, 0));
    check(c, pk_pd_set_bulk(c, b, (int)n, stream_of(bulk)));
}

// pk_pd_rollout / pk_pd_rollout_f64: x, v (n, 3) updated in place; for double
// tensors bulk64 (n,) is the stiffness, for float ones the context's.
void pd_rollout(std::uintptr_t h, const py::object& x, const py::object& v, float horizon, float mu, float lam,
                int iterations, float dt, int steps, int every, const py::tuple& gravity, const py::object& bulk64)
{
    pk_ctx* c = as_ctx(h);
    const long long n = rows_of(x);
    const pk_pd_params p{horizon, mu, lam, iterations, dt, 0.0f};
    if (is_f64(x)) {
        const py::object f64 = torch().attr("float64");
        const double g[3] = {gravity[0].cast<double>(), gravity[1].cast<double>(), gravity[2].cast<double>()};
        if (bulk64.is_none()) throw std::invalid_argument("a double rollout needs bulk64");
        auto* px = static_cast<double*>(tensor_ptr(x, "x", f64, n, 3));
        auto* pv = static_cast<double*>(tensor_ptr(v, "v", f64, n, 3));
        const auto* pb = static_cast<const double*>(tensor_ptr(bulk64, "bulk64", f64, n, 0));
        check(c, pk_pd_rollout_f64(c, px, pv, pb, (int)n, g, &p, steps, every, stream_of(x)));
    } else {
        const py::object f32 = torch().attr("float32");
        const float g[3] = {gravity[0].cast<float>(), gravity[1].cast<float>(), gravity[2].cast<float>()};
        auto* px = static_cast<float*>(tensor_ptr(x, "x", f32, n, 3));
        auto* pv = static_cast<float*>(tensor_ptr(v, "v", f32, n, 3));
        check(c, pk_pd_rollout(c, px, pv, (int)n, g, &p, steps, every, stream_of(x)));
    }
}

// Reverse mode of the last pd rollout of xbar's precision: (dL/dx0, dL/dv0,
// dL/dbulk as doubles).
py::tuple pd_rollout_backward(std::uintptr_t h, const py::object& xbar, const py::object& vbar)
{
    pk_ctx* c = as_ctx(h);
    const long long n = rows_of(xbar);
    const py::object tt = torch();
    const py::object dt = xbar.attr("dtype");
    void* px = tensor_ptr(xbar, "xbar", dt, n, 3);
    void* pv = vbar.is_none() ? nullptr : tensor_ptr(vbar, "vbar", dt, n, 3);
    py::object gx = tt.attr("empty_like")(xbar), gv = tt.attr("empty_like")(xbar);
    py::object gb = tt.attr("empty")(n, py::arg("dtype") = tt.attr("float64"), py::arg("device") = xbar.attr("device"));
    void* pgx = tensor_ptr(gx, "gx", dt, n, 3);
    void* pgv = tensor_ptr(gv, "gv", dt, n, 3);
    auto* pb = static_cast<double*>(tensor_ptr(gb, "grad_bulk", tt.attr("float64"), n, 0));
    const pk_stream st = stream_of(xbar);
    if (is_f64(xbar))
        check(c, pk_pd_rollout_backward_f64(c, static_cast<const double*>(px), static_cast<const double*>(pv),
                                            static_cast<double*>(pgx), static_cast<double*>(pgv), pb, st));
    else
        check(c, pk_pd_rollout_backward(c, static_cast<const float*>(px), static_cast<const float*>(pv),
                                        static_cast<float*>(pgx), static_cast<float*>(pgv), pb, st));
    return py::make_tuple(gx, gv, gb);
}

// pk_pbd_rollout / _f64: `params` is the address of a pk_pbf_params.
void pbd_rollout(std::uintptr_t h, const py::object& x, const py::object& v, std::uintptr_t params, int steps,
                 int every)
{
    pk_ctx* c = as_ctx(h);
    if (!params) throw std::invalid_argument("null step parameters");
    const long long n = rows_of(x);
    const auto* p = reinterpret_cast<const pk_pbf_params*>(params);
    const bool f64 = is_f64(x);
    const py::object dt = torch().attr(f64 ? "float64" : "float32");
    void* px = tensor_ptr(x, "x", dt, n, 3);
    void* pv = tensor_ptr(v, "v", dt, n, 3);
    const pk_stream st = stream_of(x);
    if (f64)
        check(c, pk_pbd_rollout_f64(c, static_cast<double*>(px), static_cast<double*>(pv), (int)n, p, steps, every, st));
    else
        check(c, pk_pbd_rollout(c, static_cast<float*>(px), static_cast<float*>(pv), (int)n, p, steps, every, st));
}

py::tuple pbd_rollout_backward(std::uintptr_t h, const py::object& xbar, const py::object& vbar)
{
    pk_ctx* c = as_ctx(h);
    const long long n = rows_of(xbar);
    const py::object tt = torch();
    const py::object dt = xbar.attr("dtype");
    void* px = tensor_ptr(xbar, "xbar", dt, n, 3);
    void* pv = vbar.is_none() ? nullptr : tensor_ptr(vbar, "vbar", dt, n, 3);
    py::object gx = tt.attr("empty_like")(xbar), gv = tt.attr("empty_like")(xbar);
    void* pgx = tensor_ptr(gx, "gx", dt, n, 3);
    void* pgv = tensor_ptr(gv, "gv", dt, n, 3);
    const pk_stream st = stream_of(xbar);
    if (is_f64(xbar))
        check(c, pk_pbd_rollout_backward_f64(c, static_cast<const double*>(px), static_cast<const double*>(pv),
                                             static_cast<double*>(pgx), static_cast<double*>(pgv), st));
    else
        check(c, pk_pbd_rollout_backward(c, static_cast<const float*>(px), static_cast<const float*>(pv),
                                         static_cast<float*>(pgx), static_cast<float*>(pgv), st));
    return py::make_tuple(gx, gv);
}

}  // namespace

PYBIND11_MODULE(_pkbind, m)
{
    m.doc() = "pybind11 layer of the differentiable rollouts (pk_hot.h)";
    m.def("pd_set_bulk", &pd_set_bulk, py::arg("ctx"), py::arg("bulk"));
    m.def("pd_rollout", &pd_rollout, py::arg("ctx"), py::arg("x"), py::arg("v"), py::arg("horizon"), py::arg("mu"),
          py::arg("lam"), py::arg("iterations"), py::arg("dt"), py::arg("steps"), py::arg("checkpoint_every"),
          py::arg("gravity"), py::arg("bulk64") = py::none());
    m.def("pd_rollout_backward", &pd_rollout_backward, py::arg("ctx"), py::arg("xbar"), py::arg("vbar") = py::none());
    m.def("pbd_rollout", &pbd_rollout, py::arg("ctx"), py::arg("x"), py::arg("v"), py::arg("params"),
          py::arg("steps"), py::arg("checkpoint_every"));
    m.def("pbd_rollout_backward", &pbd_rollout_backward, py::arg("ctx"), py::arg("xbar"),
          py::arg("vbar") = py::none());
}
