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
from conftest import golden_names, load_golden, session_fill
from helpers import DESC_RTOL, GRAD_RTOL, assert_close, gpu_for, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture
def filled_scratch():
    L = Abi.lib()
    Abi.check(L.ld_debug_fill_scratch(0xFF))
    try:
        yield
    finally:
        Abi.check(L.ld_debug_fill_scratch(session_fill()))


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


@pytest.mark.parametrize("style", [2, 3])
def test_batched_pass_with_nan_filled_work_space(filled_scratch, style):
    """The resident batched pass owns its work space (a torch buffer, not the
    library's allocations): filled with NaN bytes before the pass, the results
    still equal the per-configuration host calls."""
    import torch

    import libdescriptor_b200 as lds
    from libdescriptor_b200 import batch as B
    from libdescriptor_b200 import workloads as W

    cfgs = []
    for c in range(4):
        x, cell = W.diamond_cell(1 + c % 2, 1, 2, jitter=0.1, strain=0.03, seed=300 + c)
        cfgs.append(W.prepare(x, cell, (np.arange(len(x)) % 2).astype(np.int32), 5.0))
    b = W.concat(cfgs)
    h = Abi.create_bs(0.99363, 4, style, 0.0, 1, 0, 2, np.full((2, 2), 5.0), [1.0, 0.5])
    k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 4, style, 0, 0.0, 1, 0,
                                           5.0, ["A", "B"], [1.0, 0.5])
    dE = np.random.default_rng(12).normal(size=(b.n_rows, h.width))
    desc_ref = h.compute_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords)
    dc_ref = h.gradient_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords, dE)
    db = B.DeviceBatch.from_batch(b, k)
    ps = B.BatchedPass(k, db, torch.from_numpy(dE).to("cuda"))
    ps.work.fill_(0xFF)
    ps.desc.fill_(float("nan"))
    torch.cuda.synchronize()
    ps.run()
    ps.sync_status()
    assert_close(ps.desc.cpu().numpy(), desc_ref, DESC_RTOL, f"style {style} batched desc")
    grad = ps.grad.cpu().numpy()
    for c, cfg in enumerate(cfgs):
        p = int(b.config_ptr[c])
        ref = W.fold(dc_ref[p:p + cfg.n_total], cfg.n_atoms, cfg.image)
        assert_close(grad[p:p + cfg.n_atoms], ref, GRAD_RTOL, f"style {style} batched forces cfg {c}")
