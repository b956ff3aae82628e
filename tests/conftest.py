import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "applied-multiphysics_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built():
    # the libraries are built in-tree by __graft_entry__.build(); build them here if missing
    need = [os.path.join(ROOT, "applied-multiphysics_b200", "libampsolve.so"),
            os.path.join(ROOT, "applied-multiphysics_b200", "libampwork.so"),
            os.path.join(ROOT, "oracle", "_build", "libamporacle.so")]
    if not all(os.path.exists(p) for p in need):
        sys.path.insert(0, ROOT)
        import __graft_entry__

        __graft_entry__.build()
