"""CPU: host-side logic of the serving loop (rings, admission by footprint,
continuous batching, retirement order) driven by a fake device, and the
autotuner's candidate space and cache."""
import json
import os

import numpy as np
import pytest

from libdescriptor_b200 import serving as S


# ----------------------------------------------------------------- rings
def _occupied(ring):
    occ = np.zeros(ring.cap, dtype=int)
    for s, n in ring.live:
        occ[s:s + n] += 1
    return occ


def test_ring_random_ops_never_overlap():
    rng = np.random.default_rng(0)
    for cap in (1, 7, 64, 1000):
        ring = S.Ring(cap)
        for _ in range(3000):
            if ring.live and rng.random() < 0.45:
                ring.free(ring.live[0][0])
            else:
                n = int(rng.integers(1, max(2, cap // 3 + 1)))
                s = ring.alloc(n)
                if s is not None:
                    assert 0 <= s and s + n <= cap
            occ = _occupied(ring)
            assert occ.max(initial=0) <= 1, "overlapping ranges"


def test_ring_fifo_and_wrap():
    r = S.Ring(10)
    a = r.alloc(4)
    b = r.alloc(4)
    assert (a, b) == (0, 4)
    assert r.alloc(3) is None          # only 2 left at the end, 0 at the start
    r.free(a)
    c = r.alloc(3)                     # wraps to the start
    assert c == 0
    assert r.alloc(2) is None          # [3, 4) free but only 1 slot; the end [8, 10) is behind the wrap
    with pytest.raises(RuntimeError):
        r.free(c)                      # not the oldest
    r.free(b)
    r.free(c)
    assert r.alloc(10) == 0


def test_ring_rejects_oversize():
    r = S.Ring(5)
    assert r.alloc(6) is None
    assert not r.fits_ever(6)


# ------------------------------------------------------------ scheduler
class FakeDevice:
    """Backend that records calls; a batch finishes when release() says so."""

    def __init__(self):
        self.staged = []
        self.launched = []
        self.finished = set()

    def stage(self, req):
        self.staged.append(req.rid)

    def launch(self, plan):
        plan.handle = len(self.launched)
        self.launched.append(plan)

    def done(self, plan):
        return plan.handle in self.finished

    def finish(self, plan):
        for r in plan.reqs:
            r.desc = ("desc", r.rid)

    def release_all(self):
        self.finished.update(p.handle for p in self.launched)


def _req(rid, lane, n, nt=None, nnz=None):
    nt = nt or n
    nnz = n * 4 if nnz is None else nnz
    return S.Request(rid, lane, n, np.zeros((nt, 3)), np.zeros(nt, np.int32), np.arange(nt, dtype=np.int32) % n,
                     np.full(n, nnz // n, np.int32), np.zeros(nnz, np.int32), np.zeros((n, 2)))


def test_admission_waits_for_memory_and_batches_continuously():
    caps = {"sf": S.LaneCaps(rows=100, atoms=300, entries=400), "bs": S.LaneCaps(rows=50, atoms=150, entries=200)}
    dev = FakeDevice()
    sch = S.Scheduler(caps, dev, max_batch_rows=64, depth=2, out_rows=128)
    reqs = [_req(i, "sf" if i % 3 else "bs", 20) for i in range(12)]
    for r in reqs:
        sch.submit(r)
    sch.admit(0.0)
    # sf: 8 requests x 20 rows, ring of 100 -> 5 admitted; bs: 4 x 20, ring of 50 -> 2
    assert len(sch.admitted["sf"]) == 5 and len(sch.pending["sf"]) == 3
    assert len(sch.admitted["bs"]) == 2 and len(sch.pending["bs"]) == 2
    sch.launch()
    # max 64 rows per batch: sf batches of 3 and 2 requests, bs one batch of 2
    sizes = sorted((p.lane, len(p.reqs)) for p in dev.launched)
    assert sizes == [("bs", 2), ("sf", 2), ("sf", 3)]
    for p in dev.launched:
        assert p.n_rows == sum(r.n_atoms for r in p.reqs)
        assert [r.slots[0] for r in p.reqs] == [p.row0 + 20 * i for i in range(len(p.reqs))]
    # nothing completes until the device says so; then memory frees and the
    # waiting requests are admitted and launched
    assert sch.poll(1.0) == []
    dev.release_all()
    done = sch.poll(2.0)
    assert sorted(r.rid for r in done) == sorted(r.rid for p in dev.launched for r in p.reqs)
    assert all(r.done_at == 2.0 for r in done)
    sch.admit(2.0)
    sch.launch()
    while not sch.idle():
        dev.release_all()
        sch.step(3.0)
    assert sorted(r.rid for r in sch.completed) == list(range(12))
    # FIFO per lane
    for lane in ("sf", "bs"):
        rids = [r.rid for r in sch.completed if r.lane == lane]
        assert rids == sorted(rids)
    assert all(ring.used == 0 for rings in sch.rings.values() for ring in rings)


def test_ring_release_out_of_order_reclaims_after_older_ranges():
    r = S.Ring(12)
    a, b, c = r.alloc(4), r.alloc(4), r.alloc(4)
    r.release(b)                       # middle range: space held until a is freed
    assert r.alloc(1) is None
    with pytest.raises(RuntimeError):
        r.release(b)                   # already released
    r.free(a)                          # a and the released b come back together
    assert [s for s, _ in r.live] == [c]
    assert r.alloc(8) == 0
    r.release(c)
    r.free(0)
    assert r.used == 0 and r.alloc(12) == 0


def test_ring_random_release_never_overlaps():
    rng = np.random.default_rng(3)
    ring = S.Ring(50)
    for _ in range(4000):
        live = [s for s, _ in ring.live if s not in ring.dead]
        u = rng.random()
        if live and u < 0.25:
            ring.free(ring.live[0][0]) if ring.live[0][0] not in ring.dead else None
        elif live and u < 0.45:
            ring.release(live[int(rng.integers(len(live)))])
        else:
            ring.alloc(int(rng.integers(1, 12)))
        occ = _occupied(ring)
        assert occ.max(initial=0) <= 1


def test_cancel_pending_and_admitted_requests():
    caps = {"sf": S.LaneCaps(rows=60, atoms=180, entries=240)}
    dev = FakeDevice()
    sch = S.Scheduler(caps, dev, max_batch_rows=40, depth=1, out_rows=80)
    reqs = [_req(i, "sf", 10) for i in range(10)]
    for r in reqs:
        sch.submit(r)
    sch.admit(0.0)                     # 6 admitted (60 rows), 4 pending
    sch.launch()                       # depth 1: one batch of 4 requests (40 rows) launched
    assert [r.state for r in reqs[:4]] == ["launched"] * 4
    assert [r.state for r in reqs[4:6]] == ["admitted"] * 2 and reqs[6].state == "pending"
    assert not sch.cancel(reqs[0])     # on the GPU: completes as usual
    assert sch.cancel(reqs[4])         # admitted: its ring space is released
    assert sch.cancel(reqs[7])         # pending: leaves the queue
    assert not sch.cancel(reqs[7])
    late = _req(99, "sf", 10)
    assert sch.cancel(late) and late.state == "cancelled"   # before submission
    while not sch.idle():
        dev.release_all()
        sch.step(1.0)
    done = sorted(r.rid for r in sch.completed)
    assert done == [0, 1, 2, 3, 5, 6, 8, 9]
    assert [r.rid for r in sch.cancelled] == [4, 7, 99]
    assert reqs[4].desc is None and reqs[7].desc is None
    # every batch still covers contiguous rows, and all ring space came back
    for p in dev.launched:
        assert [r.slots[0] for r in p.reqs] == [p.row0 + 10 * i for i in range(len(p.reqs))]
    assert all(ring.used == 0 for rings in sch.rings.values() for ring in rings)


def test_oversized_request_is_rejected_up_front():
    caps = {"sf": S.LaneCaps(rows=10, atoms=30, entries=40)}
    sch = S.Scheduler(caps, FakeDevice(), max_batch_rows=8, out_rows=16)
    with pytest.raises(ValueError):
        sch.submit(_req(0, "sf", 11))
    with pytest.raises(ValueError):
        sch.submit(_req(1, "sf", 9))       # more rows than one batch


def test_batch_stops_at_row_ring_wrap():
    caps = {"sf": S.LaneCaps(rows=50, atoms=1000, entries=1000)}
    dev = FakeDevice()
    sch = S.Scheduler(caps, dev, max_batch_rows=50, depth=1, out_rows=100)
    for i in range(2):
        sch.submit(_req(i, "sf", 20))
    sch.step(0.0)                       # admits 0, 1; launches [0, 1]
    dev.release_all()
    sch.submit(_req(2, "sf", 20))       # rows 40..50 too short -> wraps to 0
    sch.submit(_req(3, "sf", 5))
    sch.step(1.0)
    assert [r.slots[0] for r in (sch.completed[0], sch.completed[1])] == [0, 20]
    last = dev.launched[-1]
    assert [r.rid for r in last.reqs] == [2, 3] and last.row0 == 0


def test_plan_caps_respects_budget():
    caps = S.plan_caps(1 << 30, {"sf": 24, "bs": 55}, {"sf": 1.0, "bs": 1.0}, {"sf": 1 << 20, "bs": 1 << 25})
    used = 0
    for k, w in (("sf", 24), ("bs", 55)):
        c = caps[k]
        used += c.rows * S.lane_bytes_per_row(w) + c.atoms * 32 + c.entries * 4
    assert used + (1 << 20) + (1 << 25) <= 1 << 30
    with pytest.raises(ValueError):
        S.plan_caps(1 << 20, {"sf": 24}, {"sf": 1.0}, {"sf": 1 << 21})


def test_fold_host_matches_add_at():
    rng = np.random.default_rng(1)
    n, nt = 13, 50
    g = rng.normal(size=(nt, 3))
    img = np.concatenate([np.arange(n), rng.integers(0, n, nt - n)]).astype(np.int32)
    ref = g[:n].copy()
    np.add.at(ref, img[n:], g[n:])
    np.testing.assert_allclose(S.fold_host(g, n, img), ref, rtol=1e-14, atol=1e-14)


def test_poisson_arrivals_rate():
    a = S.poisson_arrivals(20000, 5000.0, seed=3)
    assert np.all(np.diff(a) >= 0)
    assert abs(len(a) / a[-1] - 5000.0) / 5000.0 < 0.03


# ---------------------------------------------------------------- tuner
def test_tuner_candidates_and_cache(tmp_path, monkeypatch):
    from libdescriptor_b200 import tuner

    sf = tuner.candidates(0)
    bs = tuner.candidates(1)
    assert {c["sf_warps"] for c in sf} == {1, 2, 4}
    assert {c["dynamic_queue"] for c in sf + bs} == {1, 2}   # explicit on / off (0 is the built-in choice)
    assert {c["pair_grid_mult"] for c in bs} == {2, 4, 8, 16}
    assert tuner.shape_key("B200", "x", 1000, 30) == tuner.shape_key("B200", "x", 1024, 30)
    assert tuner.shape_key("B200", "x", 1025, 30) != tuner.shape_key("B200", "x", 1024, 30)

    applied = []
    monkeypatch.setattr(tuner.B, "set_tuning", lambda kind, shape: applied.append(dict(shape or {})))

    class FakeTorchCuda:
        @staticmethod
        def get_device_name(dev):
            return "FakeGPU"

    class FakeTorch:
        cuda = FakeTorchCuda

    class FakeDB:
        n_rows, max_neigh = 5000, 31

    class FakeDesc:
        device = None

    class FakePass:
        torch = FakeTorch
        kind = object()
        db = FakeDB
        desc = FakeDesc

    cost = {json.dumps(c, sort_keys=True): 1.0 + i for i, c in enumerate(bs)}
    best_shape = bs[5]
    cost[json.dumps(best_shape, sort_keys=True)] = 0.1
    path = os.path.join(tmp_path, "tune.json")
    t = tuner.Autotuner(cache_path=path)
    monkeypatch.setattr(t, "time_shape", lambda p, shape: cost[json.dumps(shape, sort_keys=True)])
    got = t.tune(FakePass, "bs8", 1)
    assert got == best_shape and applied[-1] == best_shape
    # cached: a fresh tuner reads the file and times nothing
    t2 = tuner.Autotuner(cache_path=path)
    monkeypatch.setattr(t2, "time_shape", lambda p, s: pytest.fail("timed a cached shape"))
    assert t2.tune(FakePass, "bs8", 1) == best_shape


# ------------------------------------------------------- request staging
def _stage(n, nt, nbl, counts, image, W=2, slots=(5, 100, 1000)):
    import ctypes as C

    from abi import Abi

    L = Abi.lib()
    rng = np.random.default_rng(2)
    coords = rng.normal(size=(nt, 3))
    species = (np.arange(nt) % 2).astype(np.int32)
    dE = rng.normal(size=(n, W))
    nb = C.c_size_t()
    Abi.check(L.ld_stage_bytes(n, nt, len(nbl), W, C.byref(nb)))
    raw = np.zeros(nb.value + 512, np.uint8)
    base = (raw.ctypes.data + 255) & ~255
    fake = [C.c_void_p(1 << 20)] * 8      # never dereferenced on the host
    rc = L.ld_stage_request(n, nt, len(nbl), W, slots[0], slots[1], slots[2], np.ascontiguousarray(coords).ravel(),
                            species, np.asarray(image, np.int32), np.asarray(nbl, np.int32),
                            np.asarray(counts, np.int32), dE.ravel(), C.c_void_p(base), nb.value, *fake, None)
    buf = raw[base - raw.ctypes.data:]
    return rc, buf, coords, species, dE


def test_stage_request_rebases_indices_into_staging():
    """Host side of ld_stage_request: the staging layout holds the inputs
    with indices rebased to the ring slots (the uploads need a device and
    fail here with the no-device status, after the staging is written)."""
    n, nt = 3, 5
    counts = [2, 0, 3]
    nbl = [1, 4, 0, 2, 3]
    image = [0, 1, 2, 0, 2]
    rc, buf, coords, species, dE = _stage(n, nt, nbl, counts, image)
    assert rc != 0
    up = lambda b: (b + 255) & ~255
    sizes = [nt * 24, nt * 4, nt * 4, len(nbl) * 4, n * 4, n * 8, n * 4, n * 2 * 8]
    offs = np.concatenate([[0], np.cumsum([up(s) for s in sizes])])
    v = lambda i, dt, cnt: buf[offs[i]:offs[i] + cnt * np.dtype(dt).itemsize].view(dt)
    np.testing.assert_array_equal(v(0, np.float64, 3 * nt), coords.ravel())
    np.testing.assert_array_equal(v(1, np.int32, nt), species)
    np.testing.assert_array_equal(v(2, np.int32, nt), np.asarray(image) + 5)
    np.testing.assert_array_equal(v(3, np.int32, 5), np.asarray(nbl) + 100)
    np.testing.assert_array_equal(v(4, np.int32, n), 100 + np.arange(n))
    np.testing.assert_array_equal(v(5, np.int64, n), [1000, 1002, 1002])
    np.testing.assert_array_equal(v(6, np.int32, n), counts)
    np.testing.assert_array_equal(v(7, np.float64, 2 * n), dE.ravel())


def test_stage_pack_writes_what_stage_request_writes():
    """ld_stage_pack, the host half the serving engine runs on its packing
    threads, fills the staging area byte for byte as ld_stage_request does
    (and touches no device: it succeeds without one)."""
    import ctypes as C

    from abi import Abi

    n, nt = 3, 5
    counts, nbl, image = [2, 0, 3], [1, 4, 0, 2, 3], [0, 1, 2, 0, 2]
    _, want, coords, species, dE = _stage(n, nt, nbl, counts, image)
    L = Abi.lib()
    nb = C.c_size_t()
    Abi.check(L.ld_stage_bytes(n, nt, len(nbl), 2, C.byref(nb)))
    raw = np.zeros(nb.value + 512, np.uint8)
    base = (raw.ctypes.data + 255) & ~255
    Abi.check(L.ld_stage_pack(n, nt, len(nbl), 2, 5, 100, 1000, np.ascontiguousarray(coords).ravel(), species,
                              np.asarray(image, np.int32), np.asarray(nbl, np.int32), np.asarray(counts, np.int32),
                              dE.ravel(), C.c_void_p(base), nb.value))
    got = raw[base - raw.ctypes.data:][:nb.value]
    np.testing.assert_array_equal(got, want[:nb.value])
    assert L.ld_stage_pack(n, nt, len(nbl), 2, 5, 100, 1000, np.ascontiguousarray(coords).ravel(), species,
                           np.asarray([0, 1, 2, 3, 2], np.int32), np.asarray(nbl, np.int32),
                           np.asarray(counts, np.int32), dE.ravel(), C.c_void_p(base), nb.value) == 2


def test_stage_chunks_follow_ring_contiguity_and_cap():
    """Requests in consecutive slots of all three rings share a chunk; a wrap
    (or any gap) in one ring, or the byte cap, starts a new one."""
    from libdescriptor_b200.serving import field_bytes, stage_chunks

    W = 4
    items = [(3, 5, 6, W, (0, 0, 0)), (2, 4, 3, W, (3, 5, 6)), (1, 1, 0, W, (5, 9, 9)),
             (2, 2, 2, W, (0, 10, 9)),            # row ring wrapped
             (2, 3, 1, W, (2, 12, 11)),
             (4, 4, 4, W, (4, 16, 12))]           # atom gap (16 != 15)
    assert stage_chunks(items, 1 << 30) == [[0, 1, 2], [3, 4], [5]]
    b0 = sum(field_bytes(3, 5, 6, W))
    assert stage_chunks(items[:3], b0) == [[0], [1, 2]]
    assert stage_chunks([], 1 << 20) == []


def test_chunk_pack_fields_equal_per_request_staging():
    """Two requests in consecutive slots packed field by field into one chunk
    (ld_stage_pack_fields through the module, no device) hold exactly the
    fields ld_stage_pack writes for each request alone, in admission order."""
    import ctypes as C

    from abi import Abi
    from libdescriptor_b200 import _ext
    from libdescriptor_b200.serving import chunk_layout

    W = 2
    reqs = [dict(n=3, nt=5, counts=[2, 0, 3], nbl=[1, 4, 0, 2, 3], image=[0, 1, 2, 0, 2]),
            dict(n=2, nt=3, counts=[1, 2], nbl=[2, 0, 1], image=[0, 1, 1])]
    rng = np.random.default_rng(4)
    slots, r0, a0, e0 = [], 7, 40, 300
    for q in reqs:
        q["coords"] = rng.normal(size=(q["nt"], 3))
        q["species"] = (np.arange(q["nt"]) % 2).astype(np.int32)
        q["dE"] = rng.normal(size=(q["n"], W))
        slots.append((r0, a0, e0))
        r0, a0, e0 = r0 + q["n"], a0 + q["nt"], e0 + len(q["nbl"])
    items = [(q["n"], q["nt"], len(q["nbl"]), W, sl) for q, sl in zip(reqs, slots)]
    starts, totals, offsets, nbytes = chunk_layout(items)
    raw = np.zeros(nbytes + 512, np.uint8)
    base = (raw.ctypes.data + 255) & ~255
    for q, sl, off in zip(reqs, slots, offsets):
        _ext._stage_pack_fields(q["n"], q["nt"], len(q["nbl"]), W, sl[0], sl[1], sl[2],
                                np.ascontiguousarray(q["coords"]).ravel(), q["species"],
                                np.asarray(q["image"], np.int32), np.asarray(q["nbl"], np.int32),
                                np.asarray(q["counts"], np.int32), q["dE"].ravel(),
                                [base + st + o for st, o in zip(starts, off)])
    chunk = raw[base - raw.ctypes.data:][:nbytes]
    # each request alone through ld_stage_pack, fields concatenated in order
    L = Abi.lib()
    want = [b"" for _ in range(8)]
    for q, sl in zip(reqs, slots):
        nb = C.c_size_t()
        Abi.check(L.ld_stage_bytes(q["n"], q["nt"], len(q["nbl"]), W, C.byref(nb)))
        r = np.zeros(nb.value + 512, np.uint8)
        rb = (r.ctypes.data + 255) & ~255
        Abi.check(L.ld_stage_pack(q["n"], q["nt"], len(q["nbl"]), W, sl[0], sl[1], sl[2],
                                  np.ascontiguousarray(q["coords"]).ravel(), q["species"],
                                  np.asarray(q["image"], np.int32), np.asarray(q["nbl"], np.int32),
                                  np.asarray(q["counts"], np.int32), q["dE"].ravel(), C.c_void_p(rb), nb.value))
        buf = r[rb - r.ctypes.data:]
        sizes = [q["nt"] * 24, q["nt"] * 4, q["nt"] * 4, len(q["nbl"]) * 4, q["n"] * 4, q["n"] * 8, q["n"] * 4,
                 q["n"] * W * 8]
        off = 0
        for f, sz in enumerate(sizes):
            want[f] += buf[off:off + sz].tobytes()
            off += (sz + 255) // 256 * 256
    for f in range(8):
        assert chunk[starts[f]:starts[f] + totals[f]].tobytes() == want[f], f"field {f}"


def test_stage_upload_fields_checks_its_list():
    from libdescriptor_b200 import _ext

    with pytest.raises(ValueError):
        _ext._stage_upload_fields([1, 2], [3], [8, 8], 0)
    with pytest.raises((RuntimeError, ValueError)):
        _ext._stage_upload_fields([0], [4096], [8], 0)      # NULL source with bytes to copy
    _ext._stage_upload_fields([0], [0], [0], 0)             # nothing to copy: no device needed


@pytest.mark.parametrize("bad", ["nbl", "image", "counts"])
def test_stage_request_rejects_bad_indices(bad):
    from abi import Abi

    n, nt = 3, 5
    counts, nbl, image = [2, 0, 3], [1, 4, 0, 2, 3], [0, 1, 2, 0, 2]
    if bad == "nbl":
        nbl = [1, 5, 0, 2, 3]          # 5 >= n_total
    elif bad == "image":
        image = [0, 1, 2, 3, 2]        # master 3 >= n_atoms
    else:
        counts = [2, 0, 2]             # does not add up to nnz
    rc, *_ = _stage(n, nt, nbl, counts, image)
    assert rc == 2, Abi.lib().ld_error_message().decode()   # LD_ERR_INVALID_ARG


# ------------------------------------------------------- served stream
def test_stream_requests_are_fresh_periodic_packings():
    """Every request of the served stream has its own log-uniform atom count
    and its own periodic packing: minimum distance d_min under the request's
    own periodicity, density 0.05 A^-3; request i is rebuilt alone from
    (seed, i)."""
    from scipy.spatial import cKDTree

    from libdescriptor_b200 import synth

    src = synth.PackingSource(n_base=1, base_atoms=4096, seed=2)
    widths = {"sf": 24, "bs": 55}
    sizes, lanes = synth.stream_draws(400, {"sf": 0.7, "bs": 0.3}, n_max=4096, seed=2)
    assert len(set(sizes.tolist())) > 200 and sizes.min() >= 16 and sizes.max() <= 4096
    assert 0.6 < lanes.count("sf") / 400 < 0.8
    reqs = S.request_stream(12, widths, {"sf": 0.7, "bs": 0.3}, n_max=4096, seed=2, source=src)
    for r in reqs:
        L = float(r.cfg.cell[0, 0])
        x = r.coords[:r.n_atoms]
        assert np.all((x >= 0) & (x < L))
        d, _ = cKDTree(x, boxsize=L).query(x, k=2)
        assert d[:, 1].min() >= 2.0 - 1e-9
        assert abs(r.n_atoms - sizes[r.rid]) <= 4 * np.sqrt(sizes[r.rid]) + 4
        assert r.dE.shape == (r.n_atoms, widths[r.lane])
        assert r.counts.shape == (r.n_atoms,) and r.nbl.shape == (int(r.counts.sum()),)
    again = S.request_stream(8, widths, {"sf": 0.7, "bs": 0.3}, n_max=4096, seed=2, source=src, first=7)[0]
    assert again.rid == 7
    np.testing.assert_array_equal(again.coords, reqs[7].coords)
    np.testing.assert_array_equal(again.dE, reqs[7].dE)
