"""Shared test setup.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu``); everything
else runs on CPU.  The oracle (tests' checker) is built on first use.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def session_fill():
    """LDB200_FILL_SCRATCH=<byte> (e.g. 0xff): the byte every device allocation
    of the library is filled with for the whole session, or -1."""
    v = os.environ.get("LDB200_FILL_SCRATCH")
    return -1 if v is None else int(v, 0)


@pytest.fixture(scope="session", autouse=True)
def _session_scratch_fill():
    """With LDB200_FILL_SCRATCH set, every test runs with the library's new
    device allocations filled with that byte (0xff: NaN doubles), so that a
    result depending on memory no kernel wrote fails its parity check."""
    fill = session_fill()
    if fill < 0:
        yield
        return
    from abi import Abi

    Abi.check(Abi.lib().ld_debug_fill_scratch(fill))
    yield
    Abi.lib().ld_debug_fill_scratch(-1)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build(with_ref=None)
    return oracle


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_names(prefix=""):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith(prefix))


def sf24():
    from libdescriptor_b200.workloads import sf24_params

    return sf24_params()


def sf_mixed():
    types = ["g1", "g2", "g3", "g4", "g5"]
    sizes = [1, 1, 2, 2, 2, 1, 3, 3, 2, 3]
    params = [0.0, 0.05, 1.5, 0.3, 2.5, 1.3, 2.7, 1.5, 1.0, 0.02, 2.0, -1.0, 0.05, 3.3, 1.0, 0.005,
              1.0, -1.0, 0.01, 2.5, 1.0, 0.03]
    return types, sizes, params
