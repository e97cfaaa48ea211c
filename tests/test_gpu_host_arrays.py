"""GPU: the host API at megabyte sizes, with the caller's arrays in pageable
memory (plain numpy) and in pinned memory.  At 7,999 atoms (input and result
sizes of about a megabyte, none a round number of pages) both kinds must give
the oracle's descriptors and gradient, and the same numbers as each other.
Results of 64 KiB and up come back in pinned host memory.  Invalid
indices raise before any kernel runs and leave the handle usable.
"""
import numpy as np
import pytest

from helpers import DESC_RTOL, GRAD_RTOL, assert_close

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


@pytest.mark.parametrize("kind", ["sf24", "bs4"])
def test_pageable_and_pinned_inputs_give_oracle_results(oracle_mod, kind):
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W
    from oracle import OracleDescriptor

    x, cell, sp = W.random_packing(7999, density=0.05, dmin=2.0, n_species=2, seed=31)
    cfg = W.prepare(x, cell, sp, 5.0)
    cm = np.full((2, 2), 5.0)
    if kind == "sf24":
        t, sz, p = W.sf24_params()
        k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["A", "B"], "cos", 5.0,
                                               t, sz, p)
        o = OracleDescriptor.symmetry_functions(2, cm, t, np.asarray(sz).reshape(-1, 2), np.asarray(p, float))
    else:
        k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 4, 3, 0, 0.0, 1, 0,
                                               5.0, ["A", "B"], [1.0, 0.5])
        o = OracleDescriptor.bispectrum(0.99363, 4, 3, 0.0, 1, 0, 2, cm, [1.0, 0.5])
    n, w = cfg.n_atoms, int(k.width)
    dE = np.random.default_rng(32).normal(size=(n, w))
    assert dE.nbytes >= 256 << 10 and dE.nbytes % 4096 != 0
    assert cfg.nbl.nbytes >= 256 << 10
    args = (cfg.species, cfg.nbl, cfg.counts, cfg.coords)
    desc_pg, grad_pg = lds.compute_and_gradient(k, n, *args, dE)
    desc_pn, grad_pn = lds.compute_and_gradient(k, n, *[_pinned(a) for a in args], _pinned(dE))
    desc_o, grad_o = o.run(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE=dE)
    assert_close(desc_pg, desc_o, DESC_RTOL, f"{kind} desc, pageable inputs")
    assert_close(grad_pg, grad_o, GRAD_RTOL, f"{kind} grad, pageable inputs")
    # the two routes agree to rounding (sums that meet in FP64 atomics vary in
    # their order from run to run)
    np.testing.assert_allclose(desc_pn, desc_pg, rtol=1e-13, atol=1e-13 * np.max(np.abs(desc_pg)))
    np.testing.assert_allclose(grad_pn, grad_pg, rtol=1e-12, atol=1e-12 * np.max(np.abs(grad_pg)))
    # forward only
    d2 = lds.compute(k, n, *args)
    assert_close(d2, desc_o, DESC_RTOL, f"{kind} forward-only desc, pageable inputs")
    # results of 64 KiB and up come back in pinned host memory, whose
    # blocks are recycled when the arrays are freed: repeated calls that drop
    # their results reuse them and still return the right numbers
    import torch

    assert torch.from_numpy(desc_pg).is_pinned() and torch.from_numpy(d2).is_pinned()
    assert torch.from_numpy(grad_pg).is_pinned()
    del desc_pn, grad_pn, d2
    for _ in range(3):
        d3, g3 = lds.compute_and_gradient(k, n, *args, dE)
        assert_close(d3, desc_o, DESC_RTOL, f"{kind} desc, recycled result blocks")
        assert_close(g3, grad_o, GRAD_RTOL, f"{kind} grad, recycled result blocks")
        del d3, g3


@pytest.mark.parametrize("kind", ["sf24", "bs4"])
def test_bad_indices_raise_and_leave_the_handle_usable(oracle_mod, kind):
    """A neighbour index outside the coordinates or a species outside the
    descriptor's list is an invalid argument (ValueError, nothing launched);
    the same handle then computes a valid call correctly."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W
    from oracle import OracleDescriptor

    x, cell, sp = W.random_packing(300, density=0.05, dmin=2.0, n_species=2, seed=33)
    cfg = W.prepare(x, cell, sp, 5.0)
    cm = np.full((2, 2), 5.0)
    if kind == "sf24":
        t, sz, p = W.sf24_params()
        k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["A", "B"], "cos", 5.0,
                                               t, sz, p)
        o = OracleDescriptor.symmetry_functions(2, cm, t, np.asarray(sz).reshape(-1, 2), np.asarray(p, float))
    else:
        k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 4, 3, 0, 0.0, 1, 0,
                                               5.0, ["A", "B"], [1.0, 0.5])
        o = OracleDescriptor.bispectrum(0.99363, 4, 3, 0.0, 1, 0, 2, cm, [1.0, 0.5])
    n, w = cfg.n_atoms, int(k.width)
    dE = np.random.default_rng(34).normal(size=(n, w))
    bad_nbl = cfg.nbl.copy()
    bad_nbl[len(bad_nbl) // 2] = cfg.n_total
    with pytest.raises(ValueError, match="neighbor_list"):
        lds.compute_and_gradient(k, n, cfg.species, bad_nbl, cfg.counts, cfg.coords, dE)
    bad_sp = cfg.species.copy()
    bad_sp[n // 3] = 2
    with pytest.raises(ValueError, match="species"):
        lds.compute(k, n, bad_sp, cfg.nbl, cfg.counts, cfg.coords)
    # more centre rows than coordinates: rejected before any buffer is sized
    n_big = cfg.n_total + 1
    counts_big = np.concatenate([cfg.counts, np.zeros(n_big - n, np.int32)]).astype(np.int32)
    dE_big = np.zeros((n_big, w))
    with pytest.raises(ValueError, match="n_atoms exceeds"):
        lds.compute_and_gradient(k, n_big, cfg.species, cfg.nbl, counts_big, cfg.coords, dE_big)
    desc, grad = lds.compute_and_gradient(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE)
    desc_o, grad_o = o.run(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE=dE)
    assert_close(desc, desc_o, DESC_RTOL, f"{kind} desc after rejected calls")
    assert_close(grad, grad_o, GRAD_RTOL, f"{kind} grad after rejected calls")


def test_pinned_result_blocks_are_bounded_and_recycled():
    """ld_host_alloc / ld_host_free through the C ABI: blocks of 200 MiB are
    handed out until 512 MiB would be outstanding (then LD_ERR_CAPACITY, and
    the module falls back to pageable arrays); a released block is kept and
    handed out again for a request of the same size."""
    import ctypes as C

    import libdescriptor_b200  # noqa: F401  (loads the library and a CUDA context)
    from abi import Abi

    L = Abi.lib()
    L.ld_host_alloc.argtypes = [C.c_size_t, C.POINTER(C.c_void_p)]
    L.ld_host_alloc.restype = C.c_int
    L.ld_host_free.argtypes = [C.c_void_p]
    L.ld_host_free.restype = None
    size = 200 << 20
    a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
    assert L.ld_host_alloc(size, C.byref(a)) == 0 and a.value
    assert L.ld_host_alloc(size, C.byref(b)) == 0 and b.value
    try:
        assert L.ld_host_alloc(size, C.byref(c)) == 3      # LD_ERR_CAPACITY
        assert not c.value
        L.ld_host_free(b)
        assert L.ld_host_alloc(size, C.byref(c)) == 0 and c.value == b.value
        # the memory is usable host memory
        C.memset(c.value, 7, 4096)
        assert C.string_at(c.value, 4)[0] == 7
    finally:
        L.ld_host_free(a)
        L.ld_host_free(c)
    L.ld_host_free(None)
    L.ld_host_free(C.c_void_p(12345))                      # not from ld_host_alloc: ignored
