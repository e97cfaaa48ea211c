"""GPU: no kernel reads device memory that no kernel wrote.

``ld_debug_fill_scratch(0xff)`` fills every new device allocation of the
library (grow-only buffers and scratch-pool blocks) with NaN bytes before
use.  With the fill on, every golden case's descriptors and gradient must
still match the reference and the oracle: a read of unwritten work space
(for instance Y rows of a bispectrum layer whose triples no output needs, as
with the style-2 odd-layer rule of src/Bispectrum.cpp:391-468) would turn into
NaN on every run instead of depending on what the memory held before.
"""
import numpy as np
import pytest

from abi import Abi
from conftest import golden_names, load_golden
from helpers import DESC_RTOL, GRAD_RTOL, assert_close, gpu_for, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture
def filled_scratch():
    L = Abi.lib()
    Abi.check(L.ld_debug_fill_scratch(0xFF))
    try:
        yield
    finally:
        Abi.check(L.ld_debug_fill_scratch(-1))


@pytest.mark.parametrize("name", golden_names())
def test_results_with_nan_filled_allocations(oracle_mod, filled_scratch, name):
    g = load_golden(name)
    h = gpu_for(name, g)                # fresh handle: its buffers are allocated (and filled) now
    o = oracle_for(name, g)
    n = int(g["n_atoms"])
    desc = h.compute(n, g["species"], g["nbl"], g["counts"], g["coords"])
    assert_close(desc, g["desc"], DESC_RTOL, name + " desc")
    dE = np.random.default_rng(11).normal(size=(n, h.width))
    dc, desc2 = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE, want_desc=True)
    _, dco = o.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=dE)
    assert_close(dc, dco, GRAD_RTOL, name + " grad")
    assert_close(desc2, g["desc"], DESC_RTOL, name + " desc of the fused pass")
