"""GPU: failures made on the host, with the device left usable.

* Out of device memory: ``ld_fail_next_allocation`` makes the library's next
  device allocation fail as a failed cudaMalloc would.  The call returns
  LD_ERR_OOM (the Python module raises RuntimeError), nothing is launched,
  and the same handle computes the reference's results on the next call.
  The reference's failure surface is exceptions (src/Descriptors.cpp:100,
  114, 258); this is the status-code form of the same contract.
* Cancellation: requests withdrawn from the serving engine while they wait
  (pending or admitted, not launched) get no results and free their ring
  space; every other request's results are those it gets alone.
* Bounded waits: a bulk-copy wait armed for a copy that never comes gives up
  after its limit and reports LD_ERR_TIMEOUT; the device stays usable.
"""
import numpy as np
import pytest

from abi import Abi, AbiError
from conftest import load_golden
from helpers import DESC_RTOL, GRAD_RTOL, assert_close, gpu_for

pytestmark = pytest.mark.gpu

LD_ERR_OOM = 4


@pytest.mark.parametrize("name", ["sf24_diamond64", "bs_j8_style3_sw1_packing64"])
def test_injected_oom_leaves_handle_usable(name):
    L = Abi.lib()
    g = load_golden(name)
    h = gpu_for(name, g)               # fresh handle: its buffers are not allocated yet
    n = int(g["n_atoms"])
    dE = np.random.default_rng(2).normal(size=(n, h.width))
    launches0 = L.ld_launch_count()
    Abi.check(L.ld_fail_next_allocation(1))
    with pytest.raises(AbiError) as e:
        h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE)
    assert e.value.code == LD_ERR_OOM
    assert "injected" in str(e.value)
    assert L.ld_launch_count() == launches0, "a kernel ran after the failed allocation"
    # the failure was a one-off: the same handle now gives the reference's descriptors
    dc, desc = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE, want_desc=True)
    assert_close(desc, g["desc"], DESC_RTOL, f"{name} desc after OOM")
    ref = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE)
    assert_close(dc, ref, GRAD_RTOL, f"{name} gradient after OOM")


def test_injected_oom_in_scratch_pool_and_python_error():
    """The stream-ordered scratch pool (device API without a caller work
    space) fails the same way, and the Python module raises RuntimeError."""
    import ctypes as C

    import torch

    import libdescriptor_b200 as lds

    L = Abi.lib()
    name = "bs_j8_style3_sw1_packing64"
    g = load_golden(name)
    h = gpu_for(name, g)
    n = int(g["n_atoms"])
    dev = torch.device("cuda", 0)
    t = {k: torch.as_tensor(g[k], device=dev) for k in ("species", "nbl", "counts", "coords")}
    dE = torch.as_tensor(np.random.default_rng(3).normal(size=(n, h.width)), device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    off = torch.empty(n + 1, dtype=torch.int64, device=dev)
    mx = C.c_int(0)
    Abi.check(L.ld_neighbor_offsets_dev(h.h, n, t["counts"].data_ptr(), off.data_ptr(), C.byref(mx), s))
    dc = torch.zeros_like(t["coords"])
    desc = torch.empty((n, h.width), dtype=torch.float64, device=dev)

    def call():
        return L.ld_gradient_dev(h.h, n, None, t["species"].data_ptr(), t["nbl"].data_ptr(), off.data_ptr(),
                                 mx.value, t["coords"].data_ptr(), dE.data_ptr(), dc.data_ptr(), desc.data_ptr(),
                                 None, s)

    Abi.check(call())                  # the handle's own buffers exist after one call
    Abi.check(L.ld_sync_status(h.h, s))
    Abi.check(L.ld_fail_next_allocation(1))
    assert call() == LD_ERR_OOM        # the per-call scratch from the pool fails
    Abi.check(L.ld_sync_status(h.h, s))
    dc.zero_()
    Abi.check(call())
    Abi.check(L.ld_sync_status(h.h, s))
    assert_close(desc.cpu().numpy(), g["desc"], DESC_RTOL, "device API after OOM")
    # the Python module: RuntimeError, then a normal call on the same kind
    kind = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, float(g["rfac0"]),
                                              int(g["twojmax"]), int(g["style"]), 0, float(g["rmin0"]),
                                              int(g["switch_flag"]), 0, float(g["cutoff"]), ["A", "B"],
                                              list(g["weights"]))
    Abi.check(L.ld_fail_next_allocation(1))
    with pytest.raises(RuntimeError, match="injected"):
        lds.compute(kind, n, g["species"], g["nbl"], g["counts"], g["coords"])
    got = lds.compute(kind, n, g["species"], g["nbl"], g["counts"], g["coords"])
    assert_close(got, g["desc"], DESC_RTOL, "module after OOM")


def test_cancelled_requests_leave_the_rest_unchanged():
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import serving as S
    from libdescriptor_b200 import workloads as W

    t, sz, p = W.sf24_params()
    kinds = {"sf": lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["A", "B"], "cos",
                                                      5.0, t, sz, p),
             "bs": lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 8, 3, 0, 0.0, 1,
                                                      0, 5.0, ["A", "B"], [1.0, 0.5])}
    widths = {k: int(v.width) for k, v in kinds.items()}
    pool = S.packing_pool(8, n_min=16, n_max=600, seed=12)
    reqs = S.make_requests(pool, 36, widths, {"sf": 0.6, "bs": 0.4}, seed=13)
    alone = []
    for r in reqs:
        d, gr = lds.compute_and_gradient(kinds[r.lane], r.n_atoms, r.species, r.nbl, r.counts, r.coords, r.dE)
        alone.append((d, S.fold_host(gr, r.n_atoms, r.image)))
    # a small budget keeps most of the burst waiting for admission; at the
    # first completion every third request not yet launched is withdrawn
    eng = S.ServingEngine(kinds, budget_bytes=18 << 20, max_batch_rows=2048, stage_bytes=8 << 20)
    withdrawn = []

    def on_done(req):
        if not withdrawn:
            for r in reqs[2::3]:
                if eng.cancel(r):
                    withdrawn.append(r)

    st = eng.serve(reqs, None, keep_results=True, on_done=on_done)
    assert withdrawn, "nothing was waiting at the first completion"
    assert st["cancelled"] == len(withdrawn) and st["requests"] == len(reqs) - len(withdrawn)
    for r, (d, gr) in zip(reqs, alone):
        if any(r is w for w in withdrawn):
            assert r.state == "cancelled" and r.desc is None
            continue
        assert r.state == "done"
        assert_close(r.desc, d, DESC_RTOL, f"request {r.rid} desc")
        assert_close(r.grad, gr, GRAD_RTOL, f"request {r.rid} forces")
    for rings in eng.sched.rings.values():
        assert all(ring.used == 0 for ring in rings)


def test_bounded_bulk_wait_runs_out_and_device_stays_usable():
    """The Z kernel's wait for its bulk-copied tile is bounded: armed for a
    copy that never comes, the same wait gives up after its limit and the CTA
    reports a timeout (LD_ERR_TIMEOUT) instead of hanging; the device then
    computes the reference's results as before."""
    import time

    L = Abi.lib()
    t0 = time.perf_counter()
    assert L.ld_debug_bulk_wait_timeout(2_000_000) == 6      # LD_ERR_TIMEOUT after ~2 ms of device time
    assert time.perf_counter() - t0 < 30.0
    assert "ran out" in L.ld_error_message().decode()
    g = load_golden("bs_j8_style3_sw1_packing64")
    h = gpu_for("bs_j8_style3_sw1_packing64", g)
    desc = h.compute(int(g["n_atoms"]), g["species"], g["nbl"], g["counts"], g["coords"])
    assert_close(desc, g["desc"], DESC_RTOL, "descriptors after the timed-out wait")
