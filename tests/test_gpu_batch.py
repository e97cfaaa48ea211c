"""GPU: batched rows (ragged neighbour arena), launch-shape tuning, the
persistent batched pass under a CUDA graph, and the torch.autograd.Function.

Every result is compared with the per-configuration host API (itself pinned
to the reference and the oracle by test_gpu_parity.py) at the parity bars:
descriptors 1e-10, gradients 1e-8 relative.
"""
import ctypes as C

import numpy as np
import pytest

from abi import Abi
from helpers import DESC_RTOL, GRAD_RTOL, assert_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _cells(n=5, n_max=2, seed=0, two_species=True):
    from libdescriptor_b200 import workloads as W

    rng = np.random.default_rng(seed)
    cfgs = []
    for c in range(n):
        n1, n2, n3 = (int(v) for v in rng.integers(1, n_max + 1, 3))
        x, cell = W.diamond_cell(n1, n2, n3, jitter=0.1, strain=0.03, seed=100 + c)
        sp = (np.arange(len(x)) % 2).astype(np.int32) if two_species else np.zeros(len(x), np.int32)
        cfgs.append(W.prepare(x, cell, sp, 5.0))
    return cfgs


def _abi_handle(kind):
    from libdescriptor_b200 import workloads as W

    if kind == "sf":
        t, sz, p = W.sf24_params()
        return Abi.create_sf(2, np.full((2, 2), 5.0), t, sz, p)
    return Abi.create_bs(0.99363, 6, 3, 0.0, 1, 0, 2, np.full((2, 2), 5.0), [1.0, 0.5])


def _module_kind(kind):
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W

    if kind == "sf":
        t, sz, p = W.sf24_params()
        return lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["A", "B"], "cos",
                                                  5.0, t, sz, p)
    return lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 6, 3, 0, 0.0, 1, 0,
                                              5.0, ["A", "B"], [1.0, 0.5])


def _host_reference(h, b, dE):
    desc = h.compute_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords)
    dc = h.gradient_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords, dE)
    return desc, dc


def _dev(a, dt):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dt)


def _rows_call(h, rows, nbl_arena, begin, counts_perm, b, dE_perm, work=True, image=None, want_desc=True):
    """ld_gradient_rows_dev over rows in the given order; returns desc, grad."""
    L = Abi.lib()
    n = len(rows)
    counts = _dev(counts_perm, torch.int32)
    off = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    mx = C.c_int()
    Abi.check(L.ld_neighbor_offsets_dev(h.h, n, counts.data_ptr(), off.data_ptr(), C.byref(mx), None))
    centre = _dev(b.row_centre[rows], torch.int32)
    nb = _dev(begin, torch.int64)
    sp = _dev(b.species, torch.int32)
    nbl = _dev(nbl_arena, torch.int32)
    x = _dev(b.coords, torch.float64)
    dE = _dev(dE_perm, torch.float64)
    dc = torch.zeros((b.coords.shape[0], 3), dtype=torch.float64, device="cuda")
    desc = torch.zeros((n, h.width), dtype=torch.float64, device="cuda")
    img = _dev(image, torch.int32) if image is not None else None
    wb = h.rows_work_bytes(n, 1)
    wk = torch.empty(wb + 256, dtype=torch.uint8, device="cuda") if work else None
    wptr = ((wk.data_ptr() + 255) & ~255) if work else None
    torch.cuda.synchronize()
    Abi.check(L.ld_gradient_rows_dev(h.h, n, centre.data_ptr(), nb.data_ptr(), sp.data_ptr(), nbl.data_ptr(),
                                     off.data_ptr(), max(mx.value, 1), x.data_ptr(), dE.data_ptr(), dc.data_ptr(),
                                     desc.data_ptr() if want_desc else None,
                                     img.data_ptr() if img is not None else None, wptr, wb if work else 0, None))
    Abi.check(L.ld_sync_status(h.h, None))
    return desc.cpu().numpy(), dc.cpu().numpy()


@pytest.mark.parametrize("kind", ["sf", "bs"])
@pytest.mark.parametrize("queue", [0, 1])
@pytest.mark.parametrize("work", [True, False])
def test_rows_api_ragged_arena_matches_batch(kind, queue, work):
    """Rows in a shuffled order whose neighbour lists sit at scattered
    positions (with gaps) of a larger arena give the per-row results of the
    contiguous batch."""
    from libdescriptor_b200 import workloads as W

    cfgs = _cells()
    b = W.concat(cfgs)
    h = _abi_handle(kind)
    dE = np.random.default_rng(1).normal(size=(b.n_rows, h.width))
    desc_ref, dc_ref = _host_reference(h, b, dE)
    rng = np.random.default_rng(2)
    rows = rng.permutation(b.n_rows)
    off = np.concatenate([[0], np.cumsum(b.counts)])
    # scatter every row's list into an arena with random gaps, in a random order
    order = rng.permutation(b.n_rows)
    begin = np.zeros(b.n_rows, np.int64)
    pos = 0
    pieces = []
    for r in order:
        gap = int(rng.integers(0, 7))
        pieces.append(np.full(gap, -7, np.int32))   # never read
        pos += gap
        begin[r] = pos
        pieces.append(b.nbl[off[r]:off[r + 1]])
        pos += int(b.counts[r])
    arena = np.concatenate(pieces).astype(np.int32)
    h.set_tuning(3, queue)
    desc, dc = _rows_call(h, rows, arena, begin[rows], b.counts[rows], b, dE[rows], work=work)
    assert_close(desc, desc_ref[rows], DESC_RTOL, "rows desc")
    assert_close(dc, dc_ref, GRAD_RTOL, "rows grad")


@pytest.mark.parametrize("kind", ["sf", "bs"])
def test_tuning_does_not_change_results(kind):
    from libdescriptor_b200 import tuner
    from libdescriptor_b200 import workloads as W

    b = W.concat(_cells(4, seed=3))
    h = _abi_handle(kind)
    dE = np.random.default_rng(4).normal(size=(b.n_rows, h.width))
    desc_ref, dc_ref = _host_reference(h, b, dE)
    keys = {"sf_warps": 0, "ctas_per_sm": 1, "pair_grid_mult": 2, "dynamic_queue": 3}
    for shape in tuner.candidates(0 if kind == "sf" else 1):
        for name, key in keys.items():
            h.set_tuning(key, shape.get(name, 0))
            assert h.get_tuning(key) == shape.get(name, 0)
        desc = h.compute_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords)
        dc = h.gradient_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords, dE)
        assert_close(desc, desc_ref, DESC_RTOL, f"desc {shape}")
        assert_close(dc, dc_ref, GRAD_RTOL, f"grad {shape}")


def test_tuning_rejects_bad_values():
    from abi import AbiError

    h = _abi_handle("sf")
    with pytest.raises(AbiError):
        h.set_tuning(0, 3)     # warps per CTA must be 1, 2 or 4
    with pytest.raises(AbiError):
        h.set_tuning(9, 1)     # unknown key
    with pytest.raises(AbiError):
        h.set_tuning(3, 3)     # row queue: 0 built-in, 1 on, 2 off
    h.set_tuning(3, 2)
    assert h.get_tuning(3) == 2


@pytest.mark.parametrize("kind", ["sf", "bs"])
def test_batched_pass_graph_and_loop_match_host_api(kind):
    from libdescriptor_b200 import batch as B
    from libdescriptor_b200 import workloads as W

    cfgs = _cells(9, n_max=3, seed=7, two_species=True)
    b = W.concat(cfgs)
    k = _module_kind(kind)
    h = _abi_handle(kind)
    dE_np = np.random.default_rng(8).normal(size=(b.n_rows, h.width))
    desc_ref, dc_ref = _host_reference(h, b, dE_np)
    db = B.DeviceBatch.from_batch(b, k)
    ps = B.BatchedPass(k, db, _dev(dE_np, torch.float64))
    B.set_tuning(k, {"dynamic_queue": 1})
    outs = []
    ps.run()
    ps.sync_status()
    outs.append((ps.desc.cpu().numpy(), ps.grad.cpu().numpy()))
    ps.capture()
    for _ in range(2):
        ps.desc.zero_()
        ps.replay()
        ps.stream.synchronize()
        outs.append((ps.desc.cpu().numpy(), ps.grad.cpu().numpy()))
    n = ps.run_per_config()
    assert n >= len(cfgs)
    ps.stream.synchronize()
    outs.append((ps.desc.cpu().numpy(), ps.grad.cpu().numpy()))
    # folded reference forces per configuration
    for desc, grad in outs:
        assert_close(desc, desc_ref, DESC_RTOL, "batched desc")
        for c, cfg in enumerate(cfgs):
            p = int(b.config_ptr[c])
            ref = W.fold(dc_ref[p:p + cfg.n_total], cfg.n_atoms, cfg.image)
            assert_close(grad[p:p + cfg.n_atoms], ref, GRAD_RTOL, f"batched forces cfg {c}")


@pytest.mark.parametrize("kind", ["sf", "bs"])
def test_torch_autograd_function(kind):
    from libdescriptor_b200 import torch_ops as T

    cfg = _cells(1, n_max=2, seed=11)[0]
    k = _module_kind(kind)
    h = _abi_handle(kind)
    rows = T.Rows.build(k, cfg.species, cfg.nbl, cfg.counts)
    x = _dev(cfg.coords, torch.float64).requires_grad_(True)
    w = np.random.default_rng(12).normal(size=(cfg.n_atoms, h.width))
    wt = _dev(w, torch.float64)
    desc = T.descriptors(k, x, rows)
    loss = (desc * wt).sum()
    loss.backward()
    T.sync_status(k)
    ref_desc = h.compute(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords)
    ref_grad = h.gradient(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords, w)
    assert_close(desc.detach().cpu().numpy(), ref_desc, DESC_RTOL, "torch desc")
    assert_close(x.grad.cpu().numpy(), ref_grad, GRAD_RTOL, "torch grad")
    # central finite differences, h = 1e-5 A, on a few coordinates of atoms
    # whose neighbours stay clear of the cutoff
    hstep = 1e-5
    g = x.grad.cpu().numpy()
    rng = np.random.default_rng(13)
    with torch.no_grad():
        for _ in range(6):
            a = int(rng.integers(cfg.n_atoms))
            d = int(rng.integers(3))
            xp = x.detach().clone()
            xm = x.detach().clone()
            xp[a, d] += hstep
            xm[a, d] -= hstep
            lp = float((T.descriptors(k, xp, rows) * wt).sum())
            lm = float((T.descriptors(k, xm, rows) * wt).sum())
            fd = (lp - lm) / (2 * hstep)
            assert abs(fd - g[a, d]) <= 1e-6 * max(1.0, abs(g[a, d])), (a, d, fd, g[a, d])


@pytest.mark.parametrize("generic", [False, True])
def test_large_sf_batch_split_launches_match_per_config(generic):
    """A symmetry-function batch of at least 8192 rows runs its two-body and
    three-body sums as two launches; each of its 4096-atom cells alone runs
    the single kernel.  Both give the same descriptors and forces, for the
    factored kernel and for the table-driven one (forced)."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import batch as B
    from libdescriptor_b200 import workloads as W

    cfgs = []
    for c in range(8):
        x, cell = W.diamond_cell(8, 8, 8, jitter=0.1, strain=0.02, seed=200 + c)
        cfgs.append(W.prepare(x, cell, np.zeros(len(x), np.int32), 5.0))
    b = W.concat(cfgs)
    assert b.n_rows >= 8192
    k = _module_kind("sf")
    if generic:
        B.set_tuning(k, {"sf_generic": 1})
    dE = np.random.default_rng(31).normal(size=(b.n_rows, int(k.width)))
    db = B.DeviceBatch.from_batch(b, k)
    ps = B.BatchedPass(k, db, _dev(dE, torch.float64))
    ps.run()
    ps.sync_status()
    desc, grad = ps.desc.cpu().numpy(), ps.grad.cpu().numpy()
    r0 = 0
    for c, cfg in enumerate(cfgs):
        n = cfg.n_atoms
        d1, g1 = lds.compute_and_gradient(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE[r0:r0 + n])
        p = int(b.config_ptr[c])
        assert_close(desc[r0:r0 + n], d1, DESC_RTOL, f"cell {c} desc")
        assert_close(grad[p:p + n], W.fold(g1, n, cfg.image), GRAD_RTOL, f"cell {c} forces")
        r0 += n
