"""Python binding of libpkhot.so (include/pk_hot.h) through ctypes.

Torch is used only for device memory and streams: every call passes raw
device pointers of contiguous float32/int32 CUDA tensors plus the current
CUDA stream to the C ABI.  There is no CPU fallback: if the library is not
built, or no GPU is present, the calls raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpkhot.so")

PK_OK, PK_ERR_ARG, PK_ERR_CUDA, PK_ERR_CAPACITY, PK_ERR_STATE, PK_ERR_NOMEM = range(6)

EXPORTED = [
    "pk_ctx_create", "pk_ctx_destroy", "pk_last_error", "pk_ctx_status", "pk_last_launch_count",
    "pk_ctx_profile", "pk_ctx_profile_read", "pk_ctx_autotune", "pk_ctx_tuning", "pk_ctx_tuning_resident",
    "pk_nq_build", "pk_nq_row_stats", "pk_summation_density", "pk_pbd_solve", "pk_integrate",
    "pk_advect", "pk_update_velocity", "pk_fixed_points", "pk_plane_constrain", "pk_viscosity",
    "pk_boundary_set_box", "pk_boundary_constrain", "pk_boundary_jitter", "pk_pbf_step",
    "pk_pbf_step_batched", "pk_pbf_step_host", "pk_graph_capture", "pk_graph_launch", "pk_graph_release",
    "pk_pd_init", "pk_pd_set_bulk", "pk_pd_solve", "pk_pd_get_rest_shape",
    "pk_pd_compute_inverse_k", "pk_pd_begin", "pk_pd_enforce", "pk_pd_update_velocity",
    "pk_pd_rotate_rest_shape", "pk_pd_apply_yielding", "pk_pd_reconstruct_rest_shape", "pk_pd_fracture",
    "pk_pd_get_yield", "pk_pd_get_bulk", "pk_pd_rest_layout",
    "pk_pd_rollout", "pk_pd_rollout_backward", "pk_pd_rollout_f64", "pk_pd_rollout_backward_f64",
    "pk_pbd_rollout", "pk_pbd_rollout_backward", "pk_pbd_rollout_f64", "pk_pbd_rollout_backward_f64",
    "pk_noalloc_max_particles", "pk_pbd_solve_noalloc",
]


class PkError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pk error {code}: {msg}")
        self.code = code


class NqParams(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_float), ("lo", ctypes.c_float * 3), ("hi", ctypes.c_float * 3),
                ("cap", ctypes.c_int), ("max_neighbors", ctypes.c_int)]


class PbdParams(ctypes.Structure):
    _fields_ = [("smoothing_length", ctypes.c_float), ("sampling_distance", ctypes.c_float),
                ("rest_density", ctypes.c_float), ("iterations", ctypes.c_int), ("dt", ctypes.c_float)]


class PbfParams(ctypes.Structure):
    _fields_ = [("nq", NqParams), ("pbd", PbdParams), ("gravity", ctypes.c_float * 3),
                ("boundary", ctypes.c_int), ("normal_friction", ctypes.c_float),
                ("tangential_friction", ctypes.c_float), ("viscosity", ctypes.c_float),
                ("viscosity_iterations", ctypes.c_int)]


class PdParams(ctypes.Structure):
    _fields_ = [("horizon", ctypes.c_float), ("mu", ctypes.c_float), ("lambda_", ctypes.c_float),
                ("iterations", ctypes.c_int), ("dt", ctypes.c_float), ("break_stretch", ctypes.c_float)]


class PlasticParams(ctypes.Structure):
    _fields_ = [("horizon", ctypes.c_float), ("mu", ctypes.c_float), ("lambda_", ctypes.c_float),
                ("A", ctypes.c_float), ("B", ctypes.c_float)]


_lib = None


def load():
    """Loads libpkhot.so and declares the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built (run __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    P, I, F, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_longlong
    sig = {
        "pk_ctx_create": ([ctypes.POINTER(P), I], I),
        "pk_ctx_destroy": ([P], I),
        "pk_last_error": ([P], ctypes.c_char_p),
        "pk_ctx_status": ([P, P], I),
        "pk_last_launch_count": ([P], I),
        "pk_ctx_profile": ([P, I], I),
        "pk_ctx_profile_read": ([P, I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(I)], I),
        "pk_nq_build": ([P, P, I, ctypes.POINTER(NqParams), P, P, LL, ctypes.POINTER(LL), P], I),
        "pk_nq_row_stats": ([P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                             ctypes.POINTER(I), P], I),
        "pk_summation_density": ([P, P, I, P, P, I, LL, ctypes.POINTER(PbdParams), P, P], I),
        "pk_pbd_solve": ([P, P, P, I, P, P, I, LL, ctypes.POINTER(PbdParams), P, P], I),
        "pk_integrate": ([P, P, P, P, I, ctypes.POINTER(F * 3), F, P], I),
        "pk_advect": ([P, P, P, I, F, P], I),
        "pk_update_velocity": ([P, P, P, P, I, F, P], I),
        "pk_fixed_points": ([P, P, P, I, P, P, P, I, P], I),
        "pk_viscosity": ([P, P, P, I, P, P, I, LL, F, F, I, F, P], I),
        "pk_plane_constrain": ([P, P, I, ctypes.POINTER(F * 3), ctypes.POINTER(F * 3), P], I),
        "pk_boundary_set_box": ([P, ctypes.POINTER(F * 3), ctypes.POINTER(F * 3), F, I, P], I),
        "pk_boundary_constrain": ([P, P, P, I, F, F, F, P], I),
        "pk_boundary_jitter": ([P, I, P, P], I),
        "pk_pbf_step": ([P, P, P, I, ctypes.POINTER(PbfParams), P, P], I),
        "pk_pbf_step_batched": ([P, P, P, P, I, I, ctypes.POINTER(PbfParams), P, P], I),
        "pk_pbf_step_host": ([P, P, P, I, ctypes.POINTER(PbfParams), P], I),
        "pk_graph_capture": ([P, P, P, P, I, I, ctypes.POINTER(PbfParams), P, P], I),
        "pk_graph_launch": ([P, P], I),
        "pk_graph_release": ([P], I),
        "pk_pd_init": ([P, P, I, P, P, I, LL, F, P], I),
        "pk_pd_set_bulk": ([P, P, I, P], I),
        "pk_pd_solve": ([P, P, P, I, ctypes.POINTER(PdParams), P], I),
        "pk_pd_get_rest_shape": ([P, P, P, P, P], I),
        "pk_ctx_autotune": ([P, I], I),
        "pk_ctx_tuning": ([P, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I)], I),
        "pk_ctx_tuning_resident": ([P, ctypes.POINTER(I)], I),
        "pk_pd_compute_inverse_k": ([P, F, P], I),
        "pk_pd_begin": ([P, P, I, ctypes.POINTER(PdParams), P], I),
        "pk_pd_enforce": ([P, P, I, ctypes.POINTER(PdParams), P], I),
        "pk_pd_update_velocity": ([P, P, P, I, F, P], I),
        "pk_pd_rotate_rest_shape": ([P, P, I, F, P], I),
        "pk_pd_apply_yielding": ([P, P, I, ctypes.POINTER(PlasticParams), P], I),
        "pk_pd_reconstruct_rest_shape": ([P, P, I, P, P, I, LL, F, I, P], I),
        "pk_pd_fracture": ([P, P, I, ctypes.POINTER(PlasticParams), P], I),
        "pk_pd_get_yield": ([P, P, P, P, P], I),
        "pk_pd_get_bulk": ([P, P, P], I),
        "pk_pd_rest_layout": ([P, P, ctypes.POINTER(I), ctypes.POINTER(LL), P], I),
        "pk_pd_rollout": ([P, P, P, I, ctypes.POINTER(F * 3), ctypes.POINTER(PdParams), I, I, P], I),
        "pk_pd_rollout_backward": ([P, P, P, P, P, P, P], I),
        "pk_pd_rollout_f64": ([P, P, P, P, I, ctypes.POINTER(ctypes.c_double * 3), ctypes.POINTER(PdParams),
                               I, I, P], I),
        "pk_pd_rollout_backward_f64": ([P, P, P, P, P, P, P], I),
        "pk_pbd_rollout": ([P, P, P, I, ctypes.POINTER(PbfParams), I, I, P], I),
        "pk_pbd_rollout_backward": ([P, P, P, P, P, P], I),
        "pk_pbd_rollout_f64": ([P, P, P, I, ctypes.POINTER(PbfParams), I, I, P], I),
        "pk_pbd_rollout_backward_f64": ([P, P, P, P, P, P], I),
        "pk_noalloc_max_particles": ([], I),
        "pk_pbd_solve_noalloc": ([P, P, I, P, P, I, LL, ctypes.POINTER(PbdParams), P, P], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _f3(v):
    return (ctypes.c_float * 3)(*[float(a) for a in v])


def nq_params(radius, lo, hi, cap, max_neighbors=0):
    return NqParams(float(radius), _f3(lo), _f3(hi), int(cap), int(max_neighbors))


def pbd_params(smoothing_length, sampling_distance, rest_density=1000.0, iterations=5, dt=1e-3):
    return PbdParams(float(smoothing_length), float(sampling_distance), float(rest_density),
                     int(iterations), float(dt))


def pbf_params(nq, pbd, gravity=(0.0, -9.8, 0.0), boundary=True, normal_friction=0.95,
               tangential_friction=0.0, viscosity=0.0, viscosity_iterations=5):
    return PbfParams(nq, pbd, _f3(gravity), int(bool(boundary)), float(normal_friction),
                     float(tangential_friction), float(viscosity), int(viscosity_iterations))


class Context:
    """One pk_ctx: the module scratch of NeighborQuery/DensityPBD/ElasticityModule."""

    def __init__(self, device=0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("pkhot needs a CUDA device; there is no CPU path")
        self.L = load()
        self.device = device
        torch.cuda.set_device(device)
        h = ctypes.c_void_p()
        rc = self.L.pk_ctx_create(ctypes.byref(h), device)
        if rc != PK_OK:
            raise PkError(rc, "pk_ctx_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pk_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != PK_OK:
            raise PkError(rc, self.L.pk_last_error(self.h).decode())

    def status(self):
        return self.L.pk_ctx_status(self.h, _stream())

    def check_status(self):
        self._check(self.status())

    def launch_count(self):
        return self.L.pk_last_launch_count(self.h)

    PROF_KINDS = ("sort", "select", "emit", "density", "disp", "finish")

    def profile(self, enable=True):
        self._check(self.L.pk_ctx_profile(self.h, int(bool(enable))))

    def profile_read(self):
        """{kind: (total_ms, launches)} of the kernel classes since profile(True)."""
        out = {}
        for k, name in enumerate(self.PROF_KINDS):
            ms, nl = ctypes.c_double(), ctypes.c_int()
            self._check(self.L.pk_ctx_profile_read(self.h, k, ctypes.byref(ms), ctypes.byref(nl)))
            out[name] = (ms.value, nl.value)
        return out

    # ---- NeighborQuery
    def nq_build(self, x, radius, lo, hi, cap, max_neighbors=0, want_list=True):
        """Returns (index, elements, total) as the reference's NeighborList."""
        import torch
        n = x.shape[0]
        p = nq_params(radius, lo, hi, cap, max_neighbors)
        tot = ctypes.c_longlong(0)
        if not want_list:
            self._check(self.L.pk_nq_build(self.h, _ptr(x), n, ctypes.byref(p), None, None, 0,
                                           None, _stream()))
            return None, None, 0
        index = torch.empty(max(n, 1), dtype=torch.int32, device=x.device)
        if cap > 0:
            elements = torch.full((max(n * cap, 1),), -1, dtype=torch.int32, device=x.device)
            self._check(self.L.pk_nq_build(self.h, _ptr(x), n, ctypes.byref(p), _ptr(index),
                                           _ptr(elements), n * cap, ctypes.byref(tot), _stream()))
            return index[:n], elements, tot.value
        # dynamic: one build into a buffer sized from the last dynamic total (and an
        # eighth more); only a list that outgrew it is built again at its size (the
        # reference also reads the total back and resizes, NeighborQuery.cu:463-472)
        hint = getattr(self, "_dyn_hint", 0)
        if hint > 0:
            elements = torch.empty(hint, dtype=torch.int32, device=x.device)
            rc = self.L.pk_nq_build(self.h, _ptr(x), n, ctypes.byref(p), _ptr(index), _ptr(elements), hint,
                                    ctypes.byref(tot), _stream())
            if rc == PK_OK:
                self._dyn_hint = max(hint, tot.value + tot.value // 8)
                return index[:n], elements[: tot.value], tot.value
            if rc != PK_ERR_CAPACITY:
                self._check(rc)
        else:
            self._check(self.L.pk_nq_build(self.h, _ptr(x), n, ctypes.byref(p), _ptr(index), None, 0,
                                           ctypes.byref(tot), _stream()))
        elements = torch.empty(max(tot.value, 1), dtype=torch.int32, device=x.device)
        self._check(self.L.pk_nq_build(self.h, _ptr(x), n, ctypes.byref(p), _ptr(index),
                                       _ptr(elements), tot.value, ctypes.byref(tot), _stream()))
        self._dyn_hint = tot.value + tot.value // 8
        return index[:n], elements[: tot.value], tot.value

    def row_stats(self):
        """(mean capped-list length incl. self, mean solver-row length, longest row)."""
        a, u, m = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(self.L.pk_nq_row_stats(self.h, ctypes.byref(a), ctypes.byref(u), ctypes.byref(m),
                                           _stream()))
        return a.value, u.value, m.value

    # ---- DensityPBD / SummationDensity
    def summation_density(self, x, index, elements, cap, total, params):
        import torch
        n = x.shape[0]
        rho = torch.empty(max(n, 1), dtype=torch.float32, device=x.device)
        self._check(self.L.pk_summation_density(self.h, _ptr(x), n, _ptr(index), _ptr(elements), cap,
                                                total, ctypes.byref(params), _ptr(rho), _stream()))
        return rho[:n]

    def pbd_solve(self, x, v, index, elements, cap, total, params, rho_out=None):
        self._check(self.L.pk_pbd_solve(self.h, _ptr(x), _ptr(v), x.shape[0], _ptr(index),
                                        _ptr(elements), cap, total, ctypes.byref(params),
                                        _ptr(rho_out), _stream()))

    def integrate(self, x, v, gravity, dt, f=None):
        self._check(self.L.pk_integrate(self.h, _ptr(x), _ptr(v), _ptr(f), x.shape[0],
                                        ctypes.byref(_f3(gravity)), float(dt), _stream()))

    def advect(self, x, v, dt):
        self._check(self.L.pk_advect(self.h, _ptr(x), _ptr(v), x.shape[0], float(dt), _stream()))

    def update_velocity(self, v, x, x_old, dt):
        self._check(self.L.pk_update_velocity(self.h, _ptr(v), _ptr(x), _ptr(x_old), x.shape[0],
                                              float(dt), _stream()))

    def viscosity(self, x, v, index, elements, cap, total, viscosity, smoothing_length, iterations=5, dt=1e-3):
        self._check(self.L.pk_viscosity(self.h, _ptr(x), _ptr(v), x.shape[0], _ptr(index), _ptr(elements), cap,
                                        total, float(viscosity), float(smoothing_length), int(iterations),
                                        float(dt), _stream()))

    # ---- FixedPoints
    def fixed_points(self, x, v, ids, target, vel=None):
        """x[ids[k]] = target[k]; v[ids[k]] = vel[k] (or 0). ids int32, target/vel (count, 3)."""
        self._check(self.L.pk_fixed_points(self.h, _ptr(x), _ptr(v), x.shape[0], _ptr(ids), _ptr(target),
                                           _ptr(vel), ids.shape[0], _stream()))

    def plane_constrain(self, x, origin, direction):
        self._check(self.L.pk_plane_constrain(self.h, _ptr(x), x.shape[0], ctypes.byref(_f3(origin)),
                                              ctypes.byref(_f3(direction)), _stream()))

    # ---- boundary
    def boundary_set_box(self, lo, hi, spacing, inverted=True):
        self._check(self.L.pk_boundary_set_box(self.h, ctypes.byref(_f3(lo)), ctypes.byref(_f3(hi)),
                                               float(spacing), int(bool(inverted)), _stream()))

    def boundary_constrain(self, x, v, dt, normal_friction=0.95, tangential_friction=0.0):
        self._check(self.L.pk_boundary_constrain(self.h, _ptr(x), _ptr(v), x.shape[0],
                                                 float(normal_friction), float(tangential_friction),
                                                 float(dt), _stream()))

    def boundary_jitter(self, n):
        import torch
        out = torch.empty(max(n, 1), dtype=torch.float32, device=f"cuda:{self.device}")
        self._check(self.L.pk_boundary_jitter(self.h, n, _ptr(out), _stream()))
        return out[:n]

    # ---- fused step
    def pbf_step(self, x, v, params, rho_out=None):
        self._check(self.L.pk_pbf_step(self.h, _ptr(x), _ptr(v), x.shape[0], ctypes.byref(params),
                                       _ptr(rho_out), _stream()))

    def pbf_step_host(self, x, v, params):
        """pbf_step on contiguous float32 CPU tensors (n, 3), updated in place;
        pinned tensors give full PCIe speed.  Returns after the copies back."""
        import torch
        for t in (x, v):
            if t.is_cuda or not t.is_contiguous() or t.dtype != torch.float32 or t.shape != x.shape:
                raise ValueError("expected a contiguous float32 CPU tensor")
        self._check(self.L.pk_pbf_step_host(self.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                            x.shape[0], ctypes.byref(params), _stream()))

    def pbf_step_batched(self, x, v, scene_offsets, params, rho_out=None):
        """One frame of len(scene_offsets) - 1 independent scenes concatenated in x, v."""
        self._check(self.L.pk_pbf_step_batched(self.h, _ptr(x), _ptr(v), _ptr(scene_offsets),
                                               scene_offsets.shape[0] - 1, x.shape[0],
                                               ctypes.byref(params), _ptr(rho_out), _stream()))

    def graph_capture(self, x, v, params, scene_offsets=None, rho_out=None):
        """Records one frame (batched when scene_offsets is given) as a CUDA graph
        owned by the context; the call also runs that frame once, uncaptured."""
        ns = 1 if scene_offsets is None else scene_offsets.shape[0] - 1
        self._check(self.L.pk_graph_capture(self.h, _ptr(x), _ptr(v), _ptr(scene_offsets), ns, x.shape[0],
                                            ctypes.byref(params), _ptr(rho_out), _stream()))

    def graph_launch(self):
        self._check(self.L.pk_graph_launch(self.h, _stream()))

    def graph_release(self):
        self._check(self.L.pk_graph_release(self.h))

    # ---- ElasticityModule
    def pd_init(self, x, index, elements, cap, total, horizon):
        self._check(self.L.pk_pd_init(self.h, _ptr(x), x.shape[0], _ptr(index), _ptr(elements), cap,
                                      total, float(horizon), _stream()))

    def pd_set_bulk(self, bulk):
        self._check(self.L.pk_pd_set_bulk(self.h, _ptr(bulk), bulk.shape[0], _stream()))

    def pd_solve(self, x, v, horizon, mu=0.05, lam=0.1, iterations=10, dt=1e-3, break_stretch=0.0):
        p = PdParams(float(horizon), float(mu), float(lam), int(iterations), float(dt), float(break_stretch))
        self._check(self.L.pk_pd_solve(self.h, _ptr(x), _ptr(v), x.shape[0], ctypes.byref(p), _stream()))

    def pd_rollout(self, x, v, horizon, mu=0.05, lam=0.1, iterations=10, dt=1e-3, steps=1,
                   checkpoint_every=0, gravity=(0.0, -9.8, 0.0), bulk64=None):
        """`steps` peridynamics steps (integrate + projection) in place, keeping a
        checkpoint every `checkpoint_every` steps for pd_rollout_backward.  x, v
        float32 (bulk from pd_set_bulk) or float64 (then bulk64 is the stiffness)."""
        import torch
        p = PdParams(float(horizon), float(mu), float(lam), int(iterations), float(dt), 0.0)
        if x.dtype == torch.float64:
            g = (ctypes.c_double * 3)(*[float(a) for a in gravity])
            self._check(self.L.pk_pd_rollout_f64(self.h, _ptr(x), _ptr(v), _ptr(bulk64), x.shape[0],
                                                 ctypes.byref(g), ctypes.byref(p), int(steps),
                                                 int(checkpoint_every), _stream()))
        else:
            self._check(self.L.pk_pd_rollout(self.h, _ptr(x), _ptr(v), x.shape[0], ctypes.byref(_f3(gravity)),
                                             ctypes.byref(p), int(steps), int(checkpoint_every), _stream()))

    def pd_rollout_backward(self, xbar, vbar=None):
        """Gradients (dL/dx0, dL/dv0, dL/dbulk) of the last checkpointed rollout of
        xbar's precision, given dL/dx_T (and dL/dv_T)."""
        import torch
        gx, gv = torch.empty_like(xbar), torch.empty_like(xbar)
        gb = torch.empty(xbar.shape[0], dtype=torch.float64, device=xbar.device)
        fn = self.L.pk_pd_rollout_backward_f64 if xbar.dtype == torch.float64 else self.L.pk_pd_rollout_backward
        self._check(fn(self.h, _ptr(xbar), _ptr(vbar), _ptr(gx), _ptr(gv), _ptr(gb), _stream()))
        return gx, gv, gb

    def pbd_rollout(self, x, v, params, steps=1, checkpoint_every=0):
        """`steps` DensityPBD frames (no boundary, no viscosity) in place, keeping
        a checkpoint every `checkpoint_every` steps for pbd_rollout_backward.
        x, v float32 or float64 (the double run of the same method)."""
        import torch
        fn = self.L.pk_pbd_rollout_f64 if x.dtype == torch.float64 else self.L.pk_pbd_rollout
        self._check(fn(self.h, _ptr(x), _ptr(v), x.shape[0], ctypes.byref(params), int(steps),
                       int(checkpoint_every), _stream()))

    def pbd_rollout_backward(self, xbar, vbar=None):
        """(dL/dx0, dL/dv0) of the last rollout of xbar's precision, given dL/dx_T
        (and dL/dv_T)."""
        import torch
        gx, gv = torch.empty_like(xbar), torch.empty_like(xbar)
        fn = self.L.pk_pbd_rollout_backward_f64 if xbar.dtype == torch.float64 else self.L.pk_pbd_rollout_backward
        self._check(fn(self.h, _ptr(xbar), _ptr(vbar), _ptr(gx), _ptr(gv), _stream()))
        return gx, gv

    # ---- autotuning of the frame kernels
    def autotune(self, enable=True):
        self._check(self.L.pk_ctx_autotune(self.h, int(bool(enable))))

    def tuning(self):
        """(pass threads per block, build particles per pass, trials remaining?)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.L.pk_ctx_tuning(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, bool(c.value)

    def tuning_resident(self):
        """Whether the Jacobi passes run as a resident grid walking the scene tiles."""
        r = ctypes.c_int()
        self._check(self.L.pk_ctx_tuning_resident(self.h, ctypes.byref(r)))
        return bool(r.value)

    # ---- ElasticityModule step by step, ElastoplasticityModule, FractureModule
    def pd_compute_inverse_k(self, horizon):
        self._check(self.L.pk_pd_compute_inverse_k(self.h, float(horizon), _stream()))

    def pd_begin(self, x, horizon, mu=0.05, lam=0.1, dt=1e-3):
        p = PdParams(float(horizon), float(mu), float(lam), 1, float(dt), 0.0)
        self._check(self.L.pk_pd_begin(self.h, _ptr(x), x.shape[0], ctypes.byref(p), _stream()))

    def pd_enforce(self, x, horizon, mu=0.05, lam=0.1, dt=1e-3):
        p = PdParams(float(horizon), float(mu), float(lam), 1, float(dt), 0.0)
        self._check(self.L.pk_pd_enforce(self.h, _ptr(x), x.shape[0], ctypes.byref(p), _stream()))

    def pd_update_velocity(self, x, v, dt):
        self._check(self.L.pk_pd_update_velocity(self.h, _ptr(x), _ptr(v), x.shape[0], float(dt), _stream()))

    def pd_rotate_rest_shape(self, x, horizon):
        self._check(self.L.pk_pd_rotate_rest_shape(self.h, _ptr(x), x.shape[0], float(horizon), _stream()))

    def pd_apply_yielding(self, x, horizon, A, B, mu=0.05, lam=0.1):
        p = PlasticParams(float(horizon), float(mu), float(lam), float(A), float(B))
        self._check(self.L.pk_pd_apply_yielding(self.h, _ptr(x), x.shape[0], ctypes.byref(p), _stream()))

    def pd_fracture(self, x, horizon, A, B, mu=0.05, lam=0.1):
        p = PlasticParams(float(horizon), float(mu), float(lam), float(A), float(B))
        self._check(self.L.pk_pd_fracture(self.h, _ptr(x), x.shape[0], ctypes.byref(p), _stream()))

    def pd_reconstruct_rest_shape(self, x, index, elements, cap, total, horizon, reconstruct_all=False):
        self._check(self.L.pk_pd_reconstruct_rest_shape(self.h, _ptr(x), x.shape[0], _ptr(index), _ptr(elements),
                                                        int(cap), int(total), float(horizon),
                                                        int(bool(reconstruct_all)), _stream()))

    def pd_get_yield(self, n):
        import torch
        out = [torch.zeros(n, device="cuda") for _ in range(3)]
        self._check(self.L.pk_pd_get_yield(self.h, *[_ptr(t) for t in out], _stream()))
        return out

    def pd_get_bulk(self, n):
        import torch
        b = torch.zeros(n, device="cuda")
        self._check(self.L.pk_pd_get_bulk(self.h, _ptr(b), _stream()))
        return b

    def pd_rest_layout(self, n):
        """(index tensor, cap, total) of the current rest shape."""
        import torch
        idx = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
        cap, tot = ctypes.c_int(), ctypes.c_longlong()
        self._check(self.L.pk_pd_rest_layout(self.h, _ptr(idx), ctypes.byref(cap), ctypes.byref(tot), _stream()))
        return idx[:n], cap.value, tot.value

    def pd_get_rest_shape(self, rest_idx=None, rest_pos=None, inv_k=None):
        self._check(self.L.pk_pd_get_rest_shape(self.h, _ptr(rest_idx), _ptr(rest_pos), _ptr(inv_k),
                                                _stream()))
