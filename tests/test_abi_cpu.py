"""The C ABI library loads on a machine without a GPU and exports exactly
what include/pk_hot.h declares; argument errors are reported without
touching a device."""
import ctypes
import os
import re
import subprocess

import pkhot

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "pk_hot.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pk_\w+)\s*\(", txt, re.M)))


def test_header_and_exports_agree():
    names = declared()
    assert len(names) >= 16
    out = subprocess.run(["nm", "-D", "--defined-only", pkhot.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted({l.split()[-1] for l in out.splitlines() if " T " in l})
    assert exported == names
    assert sorted(pkhot.EXPORTED) == names


def test_library_loads_without_gpu():
    L = pkhot.load()
    for n in declared():
        assert hasattr(L, n)


def test_argument_errors_need_no_device():
    L = pkhot.load()
    assert L.pk_ctx_destroy(None) == pkhot.PK_ERR_ARG
    assert L.pk_ctx_create(None, 0) == pkhot.PK_ERR_ARG
    assert L.pk_pbf_step_host(None, None, None, 0, None, None) == pkhot.PK_ERR_ARG
    p = pkhot.nq_params(0.01, (0, 0, 0), (1, 1, 1), 60)
    assert L.pk_nq_build(None, None, 0, ctypes.byref(p), None, None, 0, None, None) == pkhot.PK_ERR_ARG
    assert L.pk_last_error(None) == b"null context"


def test_pybind_layer_loads_and_checks_its_tensors_without_gpu():
    # the pybind11 layer of the differentiable rollouts (pk_torch's path):
    # loads against the same libpkhot.so and refuses bad arguments before any
    # device call
    import pytest
    import torch
    import pk_torch
    B = pk_torch._pkbind
    for name in ("pd_set_bulk", "pd_rollout", "pd_rollout_backward", "pbd_rollout", "pbd_rollout_backward"):
        assert hasattr(B, name)
    x = torch.zeros((4, 3))
    with pytest.raises(ValueError, match="null pk context"):
        B.pbd_rollout(0, x, x, 1, 1, 0)
    with pytest.raises(ValueError, match="contiguous CUDA tensor"):
        B.pd_rollout(1, x, x, 0.01, 0.05, 0.1, 10, 1e-3, 1, 0, (0.0, -9.8, 0.0))
    with pytest.raises(ValueError, match="contiguous CUDA tensor"):
        B.pbd_rollout_backward(1, x)
