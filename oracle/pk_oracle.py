"""ctypes binding of the CPU restatement (oracle/libpkoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py for the timed CPU baseline.  The product never imports
this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libpkoracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        c_int, c_float, c_ll = ctypes.c_int, ctypes.c_float, ctypes.c_longlong
        L.pko_set_norm_variant.argtypes = [c_int]
        L.pko_get_norm_variant.restype = c_int
        L.pko_set_threads.argtypes = [c_int]
        L.pko_max_threads.restype = c_int
        L.pko_dist3.argtypes = [_f32p, _f32p]
        L.pko_dist3.restype = c_float
        L.pko_kernels_f.argtypes = [c_int, _f32p, c_float, _f32p]
        L.pko_fixed_points.argtypes = [c_int, _f32p, _f32p, _i32p, _f32p, ctypes.c_void_p, c_int]
        L.pko_plane_constrain.argtypes = [c_int, _f32p, _f32p, _f32p]
        L.pko_neighbor_query.argtypes = [c_int, _f32p, c_float, _f32p, _f32p, c_int,
                                         ctypes.c_void_p, ctypes.c_void_p, c_ll,
                                         ctypes.POINTER(c_ll)]
        L.pko_neighbor_query.restype = c_int
        L.pko_density_scaling.argtypes = [c_float, c_float, c_float,
                                          ctypes.POINTER(c_float), ctypes.POINTER(c_float)]
        L.pko_sdf_box_dims.argtypes = [_f32p, _f32p, c_float, _i32p]
        L.pko_polar_rotation.argtypes = [_f32p, _f32p]
        L.pko_clamped_inverse.argtypes = [_f32p, ctypes.c_double, ctypes.c_double, _f32p]
        for sfx, rp, rt in (("_f", _f32p, c_float), ("_d", _f64p, ctypes.c_double)):
            getattr(L, "pko_summation_density" + sfx).argtypes = [
                c_int, rp, _i32p, _i32p, c_int, c_ll, rt, rt, rp]
            getattr(L, "pko_pbd_constrain" + sfx).argtypes = [
                c_int, rp, rp, _i32p, _i32p, c_int, c_ll, rt, rt, c_int, rt, ctypes.c_void_p]
            getattr(L, "pko_integrate" + sfx).argtypes = [
                c_int, rp, rp, ctypes.c_void_p, rp, rt]
            getattr(L, "pko_pd_rest_shape" + sfx).argtypes = [
                c_int, rp, _i32p, _i32p, c_int, c_ll, _i32p, rp]
            getattr(L, "pko_pd_inverse_k" + sfx).argtypes = [
                c_int, _i32p, c_int, c_ll, rp, rt, rp]
            getattr(L, "pko_implicit_viscosity" + sfx).argtypes = [
                c_int, rp, rp, _i32p, _i32p, c_int, c_ll, rt, rt, c_int, rt]
            getattr(L, "pko_pd_break" + sfx).argtypes = [
                c_int, rp, _i32p, c_int, c_ll, _i32p, rp, _u8p, rt]
            getattr(L, "pko_pd_solve" + sfx).argtypes = [
                c_int, rp, rp, _i32p, c_int, c_ll, _i32p, rp, ctypes.c_void_p, rp, rp,
                rt, rt, rt, c_int, rt]
            getattr(L, "pko_pd_enforce" + sfx).argtypes = [
                c_int, rp, rp, _i32p, c_int, c_ll, _i32p, rp, rp, rp, rt, rt, rt]
            getattr(L, "pko_pd_rotate_rest_shape" + sfx).argtypes = [
                c_int, rp, _i32p, c_int, c_ll, _i32p, rp, rt]
            getattr(L, "pko_pd_invariants" + sfx).argtypes = [
                c_int, rp, _i32p, c_int, c_ll, _i32p, rp, rp, rt, rt, rt, rt, rt, rp, rp, rp, _u8p]
            getattr(L, "pko_pd_apply_yielding" + sfx).argtypes = [
                c_int, rp, _i32p, c_int, c_ll, _i32p, rp, rp, rp, rp]
            getattr(L, "pko_pd_inverse_deformation" + sfx).argtypes = [
                c_int, rp, _i32p, c_int, c_ll, _i32p, rp, rt, rp]
            getattr(L, "pko_pd_recon_sizes" + sfx).argtypes = [
                c_int, _u8p, _i32p, c_int, c_ll, _i32p, c_int, c_ll, _i32p]
            getattr(L, "pko_pd_recon_fill" + sfx).argtypes = [
                c_int, rp, _u8p, rp, _i32p, _i32p, c_int, c_ll, _i32p, c_int, c_ll, _i32p, rp, _i32p,
                _i32p, rp]
            getattr(L, "pko_pd_fracture" + sfx).argtypes = [
                c_int, rp, _i32p, c_int, c_ll, _i32p, rp, rp, rt, rt, rt, rt, rt]
        _LIB = L
    return _LIB


class _Sdf(ctypes.Structure):
    _fields_ = [("left", ctypes.c_float * 3), ("h", ctypes.c_float * 3),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("inverted", ctypes.c_int), ("data", ctypes.POINTER(ctypes.c_float))]


def set_norm_variant(v):
    lib().pko_set_norm_variant(int(v))


def set_threads(t):
    """OpenMP threads of the restatement; t <= 0 means one per host processor."""
    lib().pko_set_threads(int(t))


def max_threads():
    """Threads the next parallel region will use (as last set)."""
    return lib().pko_max_threads()


def dist3(a, b):
    return lib().pko_dist3(np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32))


def dist3_many(pairs):
    """|a - b| for each row (a, b) of an (n, 6) float32 array."""
    p = np.ascontiguousarray(pairs, np.float32)
    L = lib()
    return np.array([L.pko_dist3(np.ascontiguousarray(q[:3]), np.ascontiguousarray(q[3:])) for q in p],
                    np.float32)


def kernels(r, h):
    """(n, 5): SpikyKernel W, G; SmoothKernel W; CorrectedKernel W, WRR (float)."""
    r = np.ascontiguousarray(r, np.float32)
    out = np.zeros((r.shape[0], 5), np.float32)
    lib().pko_kernels_f(r.shape[0], r, float(h), out)
    return out


def fixed_points(x, v, ids, target, vel=None):
    x = np.array(x, np.float32, copy=True)
    v = np.array(v, np.float32, copy=True)
    ids = np.ascontiguousarray(ids, np.int32)
    target = np.ascontiguousarray(target, np.float32)
    velp = None if vel is None else np.ascontiguousarray(vel, np.float32)
    lib().pko_fixed_points(x.shape[0], x, v, ids, target,
                           None if velp is None else velp.ctypes.data_as(ctypes.c_void_p), ids.shape[0])
    return x, v


def plane_constrain(x, origin, direction):
    x = np.array(x, np.float32, copy=True)
    lib().pko_plane_constrain(x.shape[0], x, _v3(origin), _v3(direction))
    return x


def _v3(a):
    return np.ascontiguousarray(np.asarray(a, np.float32).reshape(3))


def neighbor_query(x, h, lo, hi, cap):
    """NeighborQuery::compute.  Returns (index, elements) in NeighborList layout."""
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
    n = x.shape[0]
    L = lib()
    index = np.zeros(max(n, 1), np.int32)
    total = ctypes.c_longlong(0)
    if cap > 0:
        elements = np.full(max(n * cap, 1), -1, np.int32)
        rc = L.pko_neighbor_query(n, x.reshape(-1), h, _v3(lo), _v3(hi), cap,
                                  index.ctypes.data, elements.ctypes.data, n * cap,
                                  ctypes.byref(total))
    else:
        rc = L.pko_neighbor_query(n, x.reshape(-1), h, _v3(lo), _v3(hi), 0,
                                  index.ctypes.data, None, 0, ctypes.byref(total))
        elements = np.zeros(max(total.value, 1), np.int32)
        rc = L.pko_neighbor_query(n, x.reshape(-1), h, _v3(lo), _v3(hi), 0,
                                  index.ctypes.data, elements.ctypes.data, total.value,
                                  ctypes.byref(total))
        elements = elements[: total.value]
    if rc != 0:
        raise RuntimeError("pko_neighbor_query failed")
    return index[:n], elements


def density_scaling(sampling, h, rho0):
    f, m = ctypes.c_float(), ctypes.c_float()
    lib().pko_density_scaling(sampling, h, rho0, ctypes.byref(f), ctypes.byref(m))
    return f.value, m.value


def _rt(dtype):
    return ("_f", np.float32) if np.dtype(dtype) == np.float32 else ("_d", np.float64)


def _total(index, elements, cap):
    return int(index.shape[0] * cap) if cap > 0 else int(elements.shape[0])


def summation_density(x, index, elements, cap, h, mass, dtype=np.float32):
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    n = x.shape[0] // 3
    rho = np.zeros(max(n, 1), dt_)
    getattr(lib(), "pko_summation_density" + sfx)(
        n, x, np.ascontiguousarray(index, np.int32), np.ascontiguousarray(elements, np.int32),
        cap, _total(index, elements, cap), h, mass, rho)
    return rho[:n]


def pbd_constrain(x, v, index, elements, cap, h, mass, iterations, dt, dtype=np.float32):
    """DensityPBD::constrain in place on copies; returns (x, v, rho)."""
    sfx, dt_ = _rt(dtype)
    x = np.array(x, dt_).reshape(-1)
    v = np.array(v, dt_).reshape(-1)
    n = x.shape[0] // 3
    rho = np.zeros(max(n, 1), dt_)
    getattr(lib(), "pko_pbd_constrain" + sfx)(
        n, x, v, np.ascontiguousarray(index, np.int32), np.ascontiguousarray(elements, np.int32),
        cap, _total(index, elements, cap), h, mass, iterations, dt, rho.ctypes.data)
    return x.reshape(-1, 3), v.reshape(-1, 3), rho[:n]


def implicit_viscosity(x, v, index, elements, cap, vis, h, iterations, dt, dtype=np.float32):
    """ImplicitViscosity::constrain on copies; returns v."""
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    v = np.array(v, dt_).reshape(-1)
    getattr(lib(), "pko_implicit_viscosity" + sfx)(
        x.shape[0] // 3, x, v, np.ascontiguousarray(index, np.int32), np.ascontiguousarray(elements, np.int32),
        cap, _total(index, elements, cap), vis, h, iterations, dt)
    return v.reshape(-1, 3)


def integrate(x, v, g, dt, f=None, dtype=np.float32):
    sfx, dt_ = _rt(dtype)
    x = np.array(x, dt_).reshape(-1)
    v = np.array(v, dt_).reshape(-1)
    n = x.shape[0] // 3
    fp = None
    if f is not None:
        f = np.ascontiguousarray(f, dt_).reshape(-1)
        fp = f.ctypes.data
    getattr(lib(), "pko_integrate" + sfx)(n, x, v, fp, np.asarray(g, dt_), dt)
    return x.reshape(-1, 3), v.reshape(-1, 3)


def sdf_box(lo, hi, spacing, inverted=True):
    """Returns the pko_sdf structure (kept alive with its data array)."""
    dims = np.zeros(3, np.int32)
    lib().pko_sdf_box_dims(_v3(lo), _v3(hi), spacing, dims)
    data = np.zeros(int(dims[0]) * int(dims[1]) * int(dims[2]), np.float32)
    s = _Sdf()
    s.data = data.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    lib().pko_sdf_box_fill.argtypes = [ctypes.POINTER(_Sdf), _f32p, _f32p, ctypes.c_float, ctypes.c_int]
    lib().pko_sdf_box_fill(ctypes.byref(s), _v3(lo), _v3(hi), spacing, int(bool(inverted)))
    s._keep = data
    return s


def sdf_constrain(x, v, sdf, rnd, normal_friction=0.95, tangential_friction=0.0, dt=0.001):
    L = lib()
    L.pko_sdf_constrain.argtypes = [ctypes.c_int, _f32p, _f32p, ctypes.POINTER(_Sdf), _f32p,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_float]
    x = np.array(x, np.float32).reshape(-1)
    v = np.array(v, np.float32).reshape(-1)
    n = x.shape[0] // 3
    L.pko_sdf_constrain(n, x, v, ctypes.byref(sdf), np.ascontiguousarray(rnd, np.float32),
                        normal_friction, tangential_friction, dt)
    return x.reshape(-1, 3), v.reshape(-1, 3)


def pd_rest_shape(x, index, elements, cap, dtype=np.float32):
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    n = x.shape[0] // 3
    tot = _total(index, elements, cap)
    ridx = np.zeros(max(tot, 1), np.int32)
    rpos = np.zeros(3 * max(tot, 1), dt_)
    getattr(lib(), "pko_pd_rest_shape" + sfx)(
        n, x, np.ascontiguousarray(index, np.int32), np.ascontiguousarray(elements, np.int32),
        cap, tot, ridx, rpos)
    return ridx, rpos


def pd_inverse_k(index, cap, total, rest_pos, h, dtype=np.float32):
    sfx, dt_ = _rt(dtype)
    n = index.shape[0]
    invK = np.zeros(9 * max(n, 1), dt_)
    getattr(lib(), "pko_pd_inverse_k" + sfx)(
        n, np.ascontiguousarray(index, np.int32), cap, total,
        np.ascontiguousarray(rest_pos, dt_), h, invK)
    return invK[: 9 * n].reshape(n, 3, 3)


def pd_break(x, index, cap, total, rest_idx, rest_pos, alive, s, dtype=np.float32):
    """Stretch break (mirrors the library's k_pd_break); updates `alive` in place."""
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    getattr(lib(), "pko_pd_break" + sfx)(
        x.shape[0] // 3, x, np.ascontiguousarray(index, np.int32), cap, total,
        np.ascontiguousarray(rest_idx, np.int32), np.ascontiguousarray(rest_pos, dt_), alive, s)
    return alive


def pd_solve(x, v, index, cap, total, rest_idx, rest_pos, invK, bulk, horizon, mu, lam,
             iterations, dt, alive=None, dtype=np.float32):
    sfx, dt_ = _rt(dtype)
    x = np.array(x, dt_).reshape(-1)
    v = np.array(v, dt_).reshape(-1)
    n = x.shape[0] // 3
    ap = None
    if alive is not None:
        alive = np.ascontiguousarray(alive, np.uint8)
        ap = alive.ctypes.data
    getattr(lib(), "pko_pd_solve" + sfx)(
        n, x, v, np.ascontiguousarray(index, np.int32), cap, total,
        np.ascontiguousarray(rest_idx, np.int32), np.ascontiguousarray(rest_pos, dt_), ap,
        np.ascontiguousarray(invK, dt_).reshape(-1), np.ascontiguousarray(bulk, dt_),
        horizon, mu, lam, iterations, dt)
    return x.reshape(-1, 3), v.reshape(-1, 3)


# ---- ElastoplasticityModule / FractureModule (pk_oracle_plastic.inc)

class RestShape:
    """A peridynamics rest shape in the NeighborList<TPair> layouts: fixed
    (cap > 0, index = counts) or CSR (cap == 0, index = offsets)."""

    def __init__(self, index, cap, total, idx, pos):
        self.index = np.ascontiguousarray(index, np.int32)
        self.cap, self.total = int(cap), int(total)
        self.idx = np.ascontiguousarray(idx, np.int32)
        self.pos = np.ascontiguousarray(pos).reshape(-1)

    def args(self, dt_):
        self.pos = np.ascontiguousarray(self.pos, dt_)
        return self.index, self.cap, self.total, self.idx, self.pos

    def copy(self):
        return RestShape(self.index.copy(), self.cap, self.total, self.idx.copy(), self.pos.copy())


def pd_enforce(x, xold, rs, invK, bulk, horizon, mu, lam, dtype=np.float32):
    """One EM_EnforceElasticity + K_UpdatePosition against x_old; returns x."""
    sfx, dt_ = _rt(dtype)
    x = np.array(x, dt_).reshape(-1)
    index, cap, total, idx, pos = rs.args(dt_)
    getattr(lib(), "pko_pd_enforce" + sfx)(
        x.shape[0] // 3, x, np.ascontiguousarray(xold, dt_).reshape(-1), index, cap, total, idx, pos,
        np.ascontiguousarray(invK, dt_).reshape(-1), np.ascontiguousarray(bulk, dt_), horizon, mu, lam)
    return x.reshape(-1, 3)


def pd_rotate_rest_shape(x, rs, h, dtype=np.float32):
    """EM_RotateRestShape on a copy of the rest shape; returns the new RestShape."""
    sfx, dt_ = _rt(dtype)
    out = rs.copy()
    index, cap, total, idx, pos = out.args(dt_)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    getattr(lib(), "pko_pd_rotate_rest_shape" + sfx)(x.shape[0] // 3, x, index, cap, total, idx, pos, h)
    return out


def pd_invariants(x, rs, bulk, h, A, B, mu, lam, byield, dtype=np.float32):
    """PM_ComputeInvariants: (yield_I1, yield_J2, I1, byield)."""
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    n = x.shape[0] // 3
    index, cap, total, idx, pos = rs.args(dt_)
    y1, y2, i1 = np.zeros(max(n, 1), dt_), np.zeros(max(n, 1), dt_), np.zeros(max(n, 1), dt_)
    by = np.array(byield, np.uint8)
    getattr(lib(), "pko_pd_invariants" + sfx)(n, x, index, cap, total, idx, pos, np.ascontiguousarray(bulk, dt_),
                                               h, A, B, mu, lam, y1, y2, i1, by)
    return y1[:n], y2[:n], i1[:n], by


def pd_apply_yielding(x, rs, y1, y2, i1, dtype=np.float32):
    """PM_ApplyYielding on a copy of the rest shape; returns the new RestShape."""
    sfx, dt_ = _rt(dtype)
    out = rs.copy()
    index, cap, total, idx, pos = out.args(dt_)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    getattr(lib(), "pko_pd_apply_yielding" + sfx)(
        x.shape[0] // 3, x, index, cap, total, idx, pos, np.ascontiguousarray(y1, dt_),
        np.ascontiguousarray(y2, dt_), np.ascontiguousarray(i1, dt_))
    return out


def pd_inverse_deformation(x, rs, h, dtype=np.float32):
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    n = x.shape[0] // 3
    index, cap, total, idx, pos = rs.args(dt_)
    invF = np.zeros(9 * max(n, 1), dt_)
    getattr(lib(), "pko_pd_inverse_deformation" + sfx)(n, x, index, cap, total, idx, pos, h, invF)
    return invF[: 9 * n].reshape(n, 3, 3)


def pd_reconstruct(x, rs, byield, nbr_index, nbr_elements, nbr_cap, h, dtype=np.float32):
    """ElastoplasticityModule::reconstructRestShape: (new CSR RestShape, cleared byield)."""
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    n = x.shape[0] // 3
    nbr_index = np.ascontiguousarray(nbr_index, np.int32)
    nbr_elements = np.ascontiguousarray(nbr_elements, np.int32)
    nbr_total = _total(nbr_index, nbr_elements, nbr_cap)
    by = np.array(byield, np.uint8)
    index, cap, total, idx, pos = rs.args(dt_)
    sizes = np.zeros(max(n, 1), np.int32)
    getattr(lib(), "pko_pd_recon_sizes" + sfx)(n, by, nbr_index, nbr_cap, nbr_total, index, cap, total, sizes)
    sizes = sizes[:n]
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    tot = int(off[-1])
    off32 = np.ascontiguousarray(off[:max(n, 1)], np.int32)
    invF = pd_inverse_deformation(x, rs, h, dtype).reshape(-1)
    new_idx = np.zeros(max(tot, 1), np.int32)
    new_pos = np.zeros(3 * max(tot, 1), dt_)
    getattr(lib(), "pko_pd_recon_fill" + sfx)(n, x, by, np.ascontiguousarray(invF, dt_), nbr_index, nbr_elements,
                                               nbr_cap, nbr_total, index, cap, total, idx, pos, off32, new_idx,
                                               new_pos)
    return RestShape(off32[:n], 0, tot, new_idx[:max(tot, 1)], new_pos), by


def pd_fracture(x, rs, bulk, h, A, B, mu, lam, dtype=np.float32):
    """FractureModule::applyPlasticity: returns the new bulk stiffness."""
    sfx, dt_ = _rt(dtype)
    x = np.ascontiguousarray(x, dt_).reshape(-1)
    b = np.array(bulk, dt_)
    index, cap, total, idx, pos = rs.args(dt_)
    getattr(lib(), "pko_pd_fracture" + sfx)(x.shape[0] // 3, x, index, cap, total, idx, pos, b, h, A, B, mu, lam)
    return b


def drucker_prager(c, phi):
    """ElastoplasticityModule::computeA/computeB (ElastoplasticityModule.h:53-64),
    phi as stored by the module (setFrictionAngle divides degrees by 180)."""
    A = 6.0 * c * np.cos(phi) / (3.0 + np.sin(phi)) / np.sqrt(3.0)
    B = 2.0 * np.sin(phi) / (3.0 + np.sin(phi)) / np.sqrt(3.0)
    return float(np.float32(A)), float(np.float32(B))


def polar_rotation(A):
    """The polar rotation of each row-major 3x3 in A (n, 9)."""
    A = np.ascontiguousarray(A, np.float32).reshape(-1, 9)
    out = np.zeros_like(A)
    for k in range(A.shape[0]):
        lib().pko_polar_rotation(A[k], out[k])
    return out


def clamped_inverse(M, thr, fill=1.0):
    """V D' U^T of each symmetric PSD row-major 3x3 in M (n, 9)."""
    M = np.ascontiguousarray(M, np.float32).reshape(-1, 9)
    out = np.zeros_like(M)
    for k in range(M.shape[0]):
        lib().pko_clamped_inverse(M[k], float(thr), float(fill), out[k])
    return out
