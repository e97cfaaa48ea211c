"""GPU: parity at the benchmark's own configurations, against the oracle.

The same seeded inputs the benchmark builds, at full size:

* 4096-atom Si diamond 8x8x8 (a = 5.43 A, jitter N(0, 0.1 A)), 24-d
  symmetry functions, descriptors + VJP;
* 8192-atom two-species random packing (0.05 A^-3, d_min 2 A), bispectrum
  2J = 8 (rfac0 0.99363, switching on, weights {1.0, 0.5}), descriptors + VJP;
* 512 strained, jittered diamond supercells (n_i ~ U{1..6}) through the
  CUDA-graph batched pass, symmetry functions and bispectrum 2J = 6, checked
  cell by cell on a sample of 24 cells;
* one served burst of the mixed stream whose batches hold 8192+ rows per
  lane (so the atomic row queue and the two-launch symmetry-function split
  are on), every request checked.

Bars (tests/helpers.py): descriptors 1e-10, gradients 1e-8 relative, against
the oracle's forward and its independent analytic adjoint; the forward of
the single configurations also against the reference's own C++
(SymmetryFunctions::compute, src/SymmetryFunctions.cpp:141-259;
Bispectrum::compute, src/Bispectrum.cpp:229-297) where that library is built.
"""
import os

import numpy as np
import pytest

from helpers import DESC_RTOL, GRAD_RTOL, assert_close

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _sf24(species):
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W

    t, sz, p = W.sf24_params()
    kind = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, species, "cos", 5.0, t, sz, p)
    return kind, ("sf", t, sz, p)


def _bs(J, species, weights):
    import libdescriptor_b200 as lds

    kind = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, J, 3, 0, 0.0, 1, 0, 5.0,
                                              species, weights)
    return kind, ("bs", J, weights)


def _oracle(spec, ns):
    from oracle import OracleDescriptor

    cm = np.full((ns, ns), 5.0)
    if spec[0] == "sf":
        return OracleDescriptor.symmetry_functions(ns, cm, spec[1], spec[2], spec[3])
    return OracleDescriptor.bispectrum(0.99363, spec[1], 3, 0.0, 1, 0, ns, cm, spec[2])


def _reference(spec, ns):
    from oracle import Reference, ReferenceDescriptor

    if not Reference.available():
        return None
    cm = np.full((ns, ns), 5.0)
    if spec[0] == "sf":
        return ReferenceDescriptor.symmetry_functions(ns, cm, spec[1], spec[2], spec[3])
    return ReferenceDescriptor.bispectrum(0.99363, spec[1], 3, 0.0, 1, 0, ns, cm, spec[2])


def _single(cfg, kind, spec, ns, seed, what):
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W

    n = cfg.n_atoms
    dE = np.random.default_rng(seed).normal(size=(n, int(kind.width)))
    desc, grad = lds.compute_and_gradient(kind, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE)
    d_ref, g_ref = _oracle(spec, ns).run(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE=dE, n_threads=THREADS)
    assert_close(desc, d_ref, DESC_RTOL, f"{what}: descriptors vs oracle")
    assert_close(grad, g_ref, GRAD_RTOL, f"{what}: gradient vs oracle")
    # forces folded onto the contributing atoms (the reference's assemble_forces)
    assert_close(W.fold(grad, n, cfg.image), W.fold(g_ref, n, cfg.image), GRAD_RTOL, f"{what}: folded forces")
    ref = _reference(spec, ns)
    if ref is not None:
        d_cpp = ref.compute(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, n_threads=THREADS)
        assert_close(desc, d_cpp, DESC_RTOL, f"{what}: descriptors vs the reference's C++")


def test_diamond_4096_sf24_desc_and_vjp():
    from libdescriptor_b200 import workloads as W

    x, cell = W.diamond_cell(8, 8, 8, jitter=0.1, seed=1)
    cfg = W.prepare(x, cell, np.zeros(len(x), np.int32), 5.0)
    assert cfg.n_atoms == 4096 and 25 <= cfg.counts.mean() <= 32
    kind, spec = _sf24(["Si"])
    _single(cfg, kind, spec, 1, 100, "diamond 4096, sf24")


def test_packing_8192_bs2J8_desc_and_vjp():
    from libdescriptor_b200 import workloads as W

    x, cell, sp = W.random_packing(8192, density=0.05, dmin=2.0, n_species=2, seed=1)
    cfg = W.prepare(x, cell, sp, 5.0)
    assert cfg.n_atoms == 8192 and 22 <= cfg.counts.mean() <= 30
    kind, spec = _bs(8, ["A", "B"], [1.0, 0.5])
    assert int(kind.width) == 55
    _single(cfg, kind, spec, 2, 101, "packing 8192, bs 2J=8")


@pytest.mark.parametrize("which", ["sf24", "bs6"])
def test_batch512_graph_pass_sample_of_cells(which):
    import torch

    from libdescriptor_b200 import batch as B
    from libdescriptor_b200 import workloads as W

    cfgs = B.diamond_batch(512, seed=1)
    b = W.concat(cfgs)
    kind, spec = _sf24(["Si"]) if which == "sf24" else _bs(6, ["Si"], [1.0])
    dev = torch.device("cuda", 0)
    db = B.DeviceBatch.from_batch(b, kind, device=dev)
    dE_h = np.random.default_rng(7).normal(size=(db.n_rows, int(kind.width)))
    ps = B.BatchedPass(kind, db, torch.as_tensor(dE_h, device=dev))
    ps.capture()
    ps.replay()
    ps.replay()                       # replays start from zeroed gradients
    ps.stream.synchronize()
    ps.sync_status()
    desc = ps.desc.cpu().numpy()
    grad = ps.grad.cpu().numpy()
    ora = _oracle(spec, 1)
    sample = list(range(0, 512, 21)) + [int(np.argmax(b.n_atoms))]
    for c in sample:
        cfg = cfgs[c]
        r0, r1 = int(db.row_ptr[c]), int(db.row_ptr[c + 1])
        p = int(db.config_ptr[c])
        d_ref, g_ref = ora.run(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE=dE_h[r0:r1],
                               n_threads=THREADS)
        assert_close(desc[r0:r1], d_ref, DESC_RTOL, f"batch512 {which} cell {c}: descriptors")
        assert_close(grad[p:p + cfg.n_atoms], W.fold(g_ref, cfg.n_atoms, cfg.image), GRAD_RTOL,
                     f"batch512 {which} cell {c}: forces")
        assert not np.any(grad[p + cfg.n_atoms:p + cfg.n_total]), "ghost rows of the folded gradient"


def test_served_step_with_large_batches():
    import libdescriptor_b200 as lds  # noqa: F401
    from libdescriptor_b200 import serving as S
    from libdescriptor_b200 import workloads as W

    sf, sf_spec = _sf24(["A", "B"])
    bs, bs_spec = _bs(8, ["A", "B"], [1.0, 0.5])
    kinds = {"sf": sf, "bs": bs}
    widths = {k: int(v.width) for k, v in kinds.items()}
    pool = S.packing_pool(12, n_min=1500, n_max=6000, seed=3)
    reqs = S.make_requests(pool, 60, widths, {"sf": 0.7, "bs": 0.3}, seed=4)
    eng = S.ServingEngine(kinds, budget_bytes=8 << 30)
    st = eng.serve(reqs, None, keep_results=True)
    assert st["requests"] == 60
    for lane in kinds:
        rows = [n for n, k in zip(eng.sched.batch_rows, eng.sched.batch_lanes) if k == lane]
        assert max(rows) >= 8192, f"{lane}: largest batch {max(rows)} rows"
    oracles = {"sf": _oracle(sf_spec, 2), "bs": _oracle(bs_spec, 2)}
    memo = {}
    for r in reqs:
        key = (id(r.coords), r.lane, id(r.dE))
        if key not in memo:
            d_ref, g_ref = oracles[r.lane].run(r.n_atoms, r.species, r.nbl, r.counts, r.coords, dE=r.dE,
                                               n_threads=THREADS)
            memo[key] = (d_ref, W.fold(g_ref, r.n_atoms, r.image))
        d_ref, f_ref = memo[key]
        assert_close(r.desc, d_ref, DESC_RTOL, f"served request {r.rid} ({r.lane}, {r.n_atoms} atoms): descriptors")
        assert_close(r.grad, f_ref, GRAD_RTOL, f"served request {r.rid} ({r.lane}, {r.n_atoms} atoms): forces")
