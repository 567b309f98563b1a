import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "physika-old_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a library")


def _ensure_built():
    import build as pkbuild
    pkbuild.build_oracle(verbose=False)
    lib = os.path.join(ROOT, "physika-old_b200", "lib", "libpkhot.so")
    if not os.path.exists(lib):
        pkbuild.build_pkhot(verbose=False)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    import pk_oracle as po
    po.set_threads(1)
    po.set_norm_variant(1)
    return po


@pytest.fixture(scope="session")
def ctx():
    import pkhot
    c = pkhot.Context(0)
    yield c
    c.close()
