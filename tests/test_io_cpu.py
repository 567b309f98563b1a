"""Particle I/O of the Framework mirror on the host: ParticleWriter frames
(ParticleWriter.cpp:44-88: int32 count, then x, y, z, color as float32 per
particle), the OBJ point reader (PointSet.cu:30-86) and the lattice fills of
ParticleSystem::loadParticles (ParticleSystem.cpp:34-97), against numpy
restatements.  Bit-exact: these are byte and float-addition formats."""
import ctypes
import os

import numpy as np
import pytest

import pkhot

LIB = os.path.join(os.path.dirname(pkhot.LIB_PATH), "libpkframework.so")
F = ctypes.POINTER(ctypes.c_float)


@pytest.fixture(scope="module")
def fw():
    if not os.path.exists(LIB):
        pytest.skip("libpkframework.so not built")
    L = ctypes.CDLL(LIB)
    L.pkf_write_frame.argtypes = [ctypes.c_char_p, F, F, ctypes.c_int]
    L.pkf_read_frame.argtypes = [ctypes.c_char_p, F, F, ctypes.c_int]
    L.pkf_load_obj_points.argtypes = [ctypes.c_char_p, F, F, ctypes.c_int]
    L.pkf_lattice_box.argtypes = [F, F, ctypes.c_float, F, ctypes.c_int]
    L.pkf_lattice_ball.argtypes = [F, ctypes.c_float, ctypes.c_float, F, ctypes.c_int]
    return L


def fp(a):
    return a.ctypes.data_as(F) if a is not None else None


def f3(v):
    return np.ascontiguousarray(np.asarray(v, np.float32))


@pytest.mark.parametrize("n", [0, 1, 1000])
def test_frame_round_trip(fw, tmp_path, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, 3)).astype(np.float32)
    c = rng.uniform(size=n).astype(np.float32)
    path = str(tmp_path / f"frame_{n}.txt").encode()
    assert fw.pkf_write_frame(path, fp(x), fp(c), n) == 0
    raw = open(path, "rb").read()
    assert len(raw) == 4 + 16 * n
    assert int(np.frombuffer(raw[:4], np.int32)[0]) == n
    rec = np.frombuffer(raw[4:], np.float32).reshape(n, 4)
    assert np.array_equal(rec[:, :3], x) and np.array_equal(rec[:, 3], c)
    xr, cr = np.zeros((max(n, 1), 3), np.float32), np.zeros(max(n, 1), np.float32)
    assert fw.pkf_read_frame(path, fp(xr), fp(cr), n) == n
    assert np.array_equal(xr[:n], x) and np.array_equal(cr[:n], c)


def test_frame_errors(fw, tmp_path):
    assert fw.pkf_read_frame(str(tmp_path / "missing.txt").encode(), None, None, 0) == -1
    short = tmp_path / "short.txt"
    short.write_bytes(np.int32(5).tobytes() + np.zeros(7, np.float32).tobytes())
    assert fw.pkf_read_frame(str(short).encode(), None, None, 0) == -1


def test_obj_points(fw, tmp_path):
    text = ("# a comment\r\n"
            "v 0.5 1.25 -3e-2\r\n"
            "vn 0 1 0\n"
            "v\t1e-3 2 3\n"
            "vt 0.5 0.5\n"        # read as a point by the reference: (0, 0, 0)
            "v 7 8\n"             # missing z: 0
            "f 1 2 3\n"
            "vn 1 0 0\n"
            "v 0.1 0.2 0.3")      # no newline at the end
    p = tmp_path / "pts.obj"
    p.write_text(text)
    want = np.float32([[0.5, 1.25, -3e-2], [1e-3, 2, 3], [0, 0, 0], [7, 8, 0], [0.1, 0.2, 0.3]])
    # "vn" lines skip one character ('v') and then fail on "n", so every
    # normal the reference reads is 0; the list is padded to the vertex count
    want_n = np.zeros((5, 3), np.float32)
    x, nrm = np.zeros((8, 3), np.float32), np.zeros((8, 3), np.float32)
    assert fw.pkf_load_obj_points(str(p).encode(), fp(x), fp(nrm), 8) == 5
    assert np.array_equal(x[:5], want)
    assert np.array_equal(nrm[:5], want_n)
    # counting without buffers
    assert fw.pkf_load_obj_points(str(p).encode(), None, None, 0) == 5


def test_obj_refused(fw, tmp_path):
    q = tmp_path / "pts.txt"
    q.write_text("v 1 2 3\n")
    assert fw.pkf_load_obj_points(str(q).encode(), None, None, 0) == -1
    assert fw.pkf_load_obj_points(str(tmp_path / "none.obj").encode(), None, None, 0) == -1


def np_box(lo, hi, d):
    lo, hi, d = f3(lo), f3(hi), np.float32(d)
    out = []
    x = lo[0]
    while x <= hi[0]:
        y = lo[1]
        while y <= hi[1]:
            z = lo[2]
            while z <= hi[2]:
                out.append((x, y, z))
                z = np.float32(z + d)
            y = np.float32(y + d)
        x = np.float32(x + d)
    return np.array(out, np.float32).reshape(-1, 3)


def np_ball(c, r, d):
    c, r = f3(c), np.float32(r)
    box = np_box(c - r, c + r, d)
    dd = box - c
    n2 = np.float32(np.float32(dd[:, 0] * dd[:, 0] + dd[:, 1] * dd[:, 1]) + dd[:, 2] * dd[:, 2])
    return box[np.sqrt(n2) < r]


@pytest.mark.parametrize("lo,hi,d", [((0, 0, 0), (0.1, 0.05, 0.02), 0.005),
                                     ((-0.3, 0.1, 0.2), (0.2, 0.3, 0.21), 0.0125)])
def test_lattice_box(fw, lo, hi, d):
    want = np_box(lo, hi, d)
    got = np.zeros((want.shape[0] + 1, 3), np.float32)
    assert fw.pkf_lattice_box(fp(f3(lo)), fp(f3(hi)), d, fp(got), got.shape[0]) == want.shape[0]
    assert np.array_equal(got[:want.shape[0]], want)


def test_lattice_ball(fw):
    c, r, d = (0.5, 0.4, 0.3), 0.05, 0.005
    want = np_ball(c, r, d)
    got = np.zeros((want.shape[0] + 1, 3), np.float32)
    assert fw.pkf_lattice_ball(fp(f3(c)), r, d, fp(got), got.shape[0]) == want.shape[0]
    assert np.array_equal(got[:want.shape[0]], want)
    assert 3000 < want.shape[0] < 5000  # ~ (4/3) pi (r/d)^3
