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
