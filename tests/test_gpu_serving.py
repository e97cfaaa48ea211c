"""GPU: the continuous-batching serving loop.  Every request's descriptors
and folded forces are the same in the mix as alone (one plain
``compute_and_gradient`` call), within the parity bars (descriptors 1e-10,
gradients 1e-8 relative), for a burst that must wait for HBM admission and
for a Poisson stream."""
import numpy as np
import pytest

from helpers import DESC_RTOL, GRAD_RTOL, assert_close

pytestmark = pytest.mark.gpu


def _kinds():
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W

    t, sz, p = W.sf24_params()
    sf = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["A", "B"], "cos", 5.0,
                                            t, sz, p)
    bs = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 8, 3, 0, 0.0, 1, 0, 5.0,
                                            ["A", "B"], [1.0, 0.5])
    return {"sf": sf, "bs": bs}


@pytest.fixture(scope="module")
def stream_setup():
    from libdescriptor_b200 import serving as S

    kinds = _kinds()
    pool = S.packing_pool(10, n_min=16, n_max=700, seed=5)
    widths = {k: int(v.width) for k, v in kinds.items()}
    reqs = S.make_requests(pool, 40, widths, {"sf": 0.7, "bs": 0.3}, seed=6)
    alone = []
    for r in reqs:
        import libdescriptor_b200 as lds

        d, g = lds.compute_and_gradient(kinds[r.lane], r.n_atoms, r.species, r.nbl, r.counts, r.coords, r.dE)
        alone.append((d, S.fold_host(g, r.n_atoms, r.image)))
    return kinds, pool, widths, alone


def _check(reqs, alone):
    for r, (d, g) in zip(reqs, alone):
        assert_close(r.desc, d, DESC_RTOL, f"request {r.rid} ({r.lane}, {r.n_atoms} atoms) desc")
        assert_close(r.grad, g, GRAD_RTOL, f"request {r.rid} ({r.lane}, {r.n_atoms} atoms) forces")


def test_burst_with_admission_waits_matches_alone(stream_setup):
    from libdescriptor_b200 import serving as S

    kinds, pool, widths, alone = stream_setup
    reqs = S.make_requests(pool, 40, widths, {"sf": 0.7, "bs": 0.3}, seed=6)
    eng = S.ServingEngine(kinds, budget_bytes=18 << 20, max_batch_rows=2048, stage_bytes=8 << 20)
    st = eng.serve(reqs, None, keep_results=True)
    assert st["admission_waits"] > 0, st
    assert st["max_batch_requests"] > 1, st
    _check(reqs, alone)


def test_poisson_stream_matches_alone(stream_setup):
    from libdescriptor_b200 import serving as S

    kinds, pool, widths, alone = stream_setup
    reqs = S.make_requests(pool, 40, widths, {"sf": 0.7, "bs": 0.3}, seed=6)
    eng = S.ServingEngine(kinds, budget_bytes=256 << 20, max_batch_rows=4096, stage_bytes=16 << 20)
    st = eng.serve(reqs, S.poisson_arrivals(len(reqs), 4000.0, seed=9), keep_results=True)
    assert st["requests"] == 40 and st["p99_ms"] >= st["p50_ms"] > 0
    _check(reqs, alone)


def test_style2_bispectrum_lane_with_nan_filled_work_space():
    """A bispectrum lane whose odd layers hold no needed triples (style 2):
    the served batches' work space (a torch buffer) filled with NaN bytes
    before serving, every request's results still equal its plain call."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import serving as S

    kinds = {"bs": lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 4, 2, 0, 0.0, 1,
                                                      0, 5.0, ["A", "B"], [1.0, 0.5])}
    pool = S.packing_pool(6, n_min=16, n_max=400, seed=15)
    widths = {k: int(v.width) for k, v in kinds.items()}
    reqs = S.make_requests(pool, 16, widths, {"bs": 1.0}, seed=16)
    alone = []
    for r in reqs:
        d, g = lds.compute_and_gradient(kinds["bs"], r.n_atoms, r.species, r.nbl, r.counts, r.coords, r.dE)
        alone.append((d, S.fold_host(g, r.n_atoms, r.image)))
    eng = S.ServingEngine(kinds, budget_bytes=64 << 20, max_batch_rows=2048, stage_bytes=8 << 20)
    for ln in eng.lanes.values():
        ln.work.fill_(0xFF)
    import torch

    torch.cuda.synchronize()
    eng.serve(reqs, None, keep_results=True)
    eng.close()
    _check(reqs, alone)


def test_requests_without_neighbours_in_the_mix(stream_setup):
    """Requests whose atoms have no neighbours at all (an empty neighbour
    field in their staging chunk) between ordinary ones: every result equals
    its plain call (isolated atoms: zero forces, the descriptors of an empty
    environment)."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import serving as S

    kinds, pool, widths, _ = stream_setup
    reqs = S.make_requests(pool, 12, widths, {"sf": 0.5, "bs": 0.5}, seed=21)
    rng = np.random.default_rng(22)
    mixed = []
    for i, r in enumerate(reqs):
        mixed.append(r)
        n = 1 + i % 3
        lane = "sf" if i % 2 else "bs"
        coords = rng.normal(size=(n, 3)) * 20.0          # far apart: no neighbours within 5 A
        mixed.append(S.Request(1000 + i, lane, n, coords, np.zeros(n, np.int32), np.arange(n, dtype=np.int32),
                               np.zeros(n, np.int32), np.zeros(0, np.int32),
                               rng.normal(size=(n, widths[lane]))))
    for k, r in enumerate(mixed):
        r.rid = k
    alone = []
    for r in mixed:
        d, g = lds.compute_and_gradient(kinds[r.lane], r.n_atoms, r.species, r.nbl, r.counts, r.coords, r.dE)
        alone.append((d, S.fold_host(g, r.n_atoms, r.image)))
    eng = S.ServingEngine(kinds, budget_bytes=64 << 20, max_batch_rows=2048, stage_bytes=8 << 20)
    eng.serve(mixed, None, keep_results=True)
    eng.close()
    _check(mixed, alone)


def test_request_with_bad_index_raises_and_frees_staging(stream_setup):
    """A request whose neighbour list points outside its atoms fails its
    host-side index check during staging: ``serve`` raises, and the staging
    blocks reserved for that round are given back."""
    from libdescriptor_b200 import serving as S

    kinds, pool, widths, _ = stream_setup
    reqs = S.make_requests(pool, 3, widths, {"sf": 1.0}, seed=31)
    bad = reqs[1]
    nbl = np.array(bad.nbl, copy=True)
    nbl[0] = bad.n_total + 5
    reqs[1] = S.Request(bad.rid, bad.lane, bad.n_atoms, bad.coords, bad.species, bad.image, bad.counts, nbl, bad.dE)
    eng = S.ServingEngine(kinds, budget_bytes=64 << 20, max_batch_rows=2048, stage_bytes=8 << 20)
    with pytest.raises((ValueError, RuntimeError), match="outside"):
        eng.serve(reqs, None)
    assert all(ln.stage_ring.used == 0 for ln in eng.lanes.values())
    eng.close()
