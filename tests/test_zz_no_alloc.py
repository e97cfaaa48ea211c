"""GPU: the descriptor + VJP entry point that allocates no device memory.

Callers such as MD engines that own every device buffer through their own
pool, or serving loops that forbid allocation while evaluating forces,
cannot let the library call cudaMalloc.  ld_gradient_counts_dev_noalloc
keeps its work space in a fixed array of the library's own device memory.
This file checks it through the C ABI against the regular device entry
point (ld_neighbor_offsets_dev + ld_gradient_dev), on two calls in a row,
with the parity tolerances of the other tests.  It is collected last so a
stop-at-first-failure run has already run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from abi import Abi
from conftest import load_golden
from helpers import DESC_RTOL, GRAD_RTOL, assert_close, gpu_for

pytestmark = pytest.mark.gpu

LD_ERR_CAPACITY = 3


def _declare(L):
    L.ld_gradient_counts_dev_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_void_p]
    L.ld_gradient_counts_dev_noalloc.restype = C.c_int
    return L


@pytest.mark.parametrize("name", ["sf24_diamond64", "bs_j8_style3_sw1_packing64"])
def test_noalloc_matches_regular_entry_point(name):
    import torch

    L = _declare(Abi.lib())
    g = load_golden(name)
    h = gpu_for(name, g)
    n = int(g["n_atoms"])
    dev = torch.device("cuda", 0)
    sp = torch.as_tensor(g["species"], device=dev)
    nbl = torch.as_tensor(g["nbl"], device=dev)
    cnt = torch.as_tensor(g["counts"], device=dev)
    x = torch.as_tensor(g["coords"], device=dev)
    dE = torch.as_tensor(np.random.default_rng(4).normal(size=(n, h.width)), device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # regular device entry point
    off = torch.empty(n + 1, dtype=torch.int64, device=dev)
    mx = C.c_int(0)
    Abi.check(L.ld_neighbor_offsets_dev(h.h, n, cnt.data_ptr(), off.data_ptr(), C.byref(mx), stream))
    dc_ref = torch.zeros_like(x)
    desc_ref = torch.empty((n, h.width), dtype=torch.float64, device=dev)
    Abi.check(L.ld_gradient_dev(h.h, n, None, sp.data_ptr(), nbl.data_ptr(), off.data_ptr(), mx.value,
                                x.data_ptr(), dE.data_ptr(), dc_ref.data_ptr(), desc_ref.data_ptr(), None,
                                stream))
    Abi.check(L.ld_sync_status(h.h, stream))
    for call in range(2):
        dc = torch.zeros_like(x)
        desc = torch.full((n, h.width), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        allocs0, launches0 = L.ld_alloc_count(), L.ld_launch_count()
        rc = L.ld_gradient_counts_dev_noalloc(h.h, n, None, sp.data_ptr(), nbl.data_ptr(), cnt.data_ptr(),
                                              mx.value, x.data_ptr(), dE.data_ptr(), dc.data_ptr(),
                                              desc.data_ptr(), None, stream)
        Abi.check(rc)
        torch.cuda.synchronize()
        # the library's own allocation counter (grow-only buffers and its
        # scratch pool) stays put, while the pass itself did launch: the
        # row-offset scan and at least one descriptor kernel
        assert L.ld_alloc_count() == allocs0, f"call {call} allocated device memory"
        assert L.ld_launch_count() - launches0 >= 2
        assert_close(dc.cpu().numpy(), dc_ref.cpu().numpy(), GRAD_RTOL, f"{name} gradient, call {call}")
        assert_close(desc.cpu().numpy(), desc_ref.cpu().numpy(), DESC_RTOL, f"{name} desc, call {call}")
        assert_close(desc.cpu().numpy(), g["desc"], DESC_RTOL, f"{name} desc vs reference, call {call}")


def test_noalloc_limits_and_status_reset():
    import torch

    L = _declare(Abi.lib())
    name = "sf24_diamond64"
    g = load_golden(name)
    h = gpu_for(name, g)
    n = int(g["n_atoms"])
    dev = torch.device("cuda", 0)
    sp = torch.as_tensor(g["species"], device=dev)
    nbl = torch.as_tensor(g["nbl"], device=dev)
    cnt = torch.as_tensor(g["counts"], device=dev)
    x = torch.as_tensor(g["coords"], device=dev)
    dE = torch.ones((n, h.width), dtype=torch.float64, device=dev)
    dc = torch.zeros_like(x)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # beyond the fixed row limit: rejected before any device work
    rc = L.ld_gradient_counts_dev_noalloc(h.h, (1 << 18) + 1, None, sp.data_ptr(), nbl.data_ptr(),
                                          cnt.data_ptr(), 64, x.data_ptr(), dE.data_ptr(), dc.data_ptr(),
                                          None, None, stream)
    assert rc == LD_ERR_CAPACITY
    assert b"262144" in Abi.lib().ld_error_message()
    # a row above max_neigh raises the device status ...
    mx = int(g["counts"].max())
    rc = L.ld_gradient_counts_dev_noalloc(h.h, n, None, sp.data_ptr(), nbl.data_ptr(), cnt.data_ptr(), mx - 2,
                                          x.data_ptr(), dE.data_ptr(), dc.data_ptr(), None, None, stream)
    assert rc == LD_ERR_CAPACITY
    # ... and the next call starts from a cleared status word
    dc.zero_()
    Abi.check(L.ld_gradient_counts_dev_noalloc(h.h, n, None, sp.data_ptr(), nbl.data_ptr(), cnt.data_ptr(), mx,
                                               x.data_ptr(), dE.data_ptr(), dc.data_ptr(), None, None, stream))
    want = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], np.ones((n, h.width)))
    assert_close(dc.cpu().numpy(), want, GRAD_RTOL, "after status reset")
