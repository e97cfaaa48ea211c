"""Continuous-batching request loop for descriptor + VJP requests.

A request is one configuration in the reference's call layout (coordinates
with ghosts, species, ghost -> master image, neighbour counts and list) plus
an upstream gradient dL/d(desc); its answer is the descriptors and the force
VJP folded onto the contributing atoms (the reference's ``compute`` +
``gradient`` + ``assemble_forces``, src/Descriptors.cpp:121-215,
python_package/libdescriptor/neighbor.py:227-263).

Resident state.  Each descriptor kind (lane) owns three device rings sized
from the HBM budget: atoms (coordinates, species, image), neighbour entries
and rows (centre, neighbour-list start, count, dL/d(desc), descriptors,
forces).  A request is *admitted* when contiguous space for its atoms,
neighbours and rows is free in every ring of its lane (admission by HBM
footprint, first come first served per lane); its inputs are then written,
with indices rebased to the ring slots, into a pinned host staging ring (the
requests admitted together are packed on a pool of host threads) and copied
to the device on the lane's copy stream in admission order.

Continuous batching.  While fewer than ``depth`` batches of a lane are on the
GPU, every admitted request that is not yet launched joins the next batch
(up to ``max_batch_rows`` rows, ending where a ring wraps).  One batch is one
``ld_gradient_rows_dev`` launch over rows that are contiguous in the row ring;
the neighbour-list starts are per row, so nothing is gathered.  Requests
arriving while batches run are admitted as memory frees and join the next
batch; the lanes' batches run in launch order on one compute stream (or on
a stream per lane with ``overlap_lanes``), while uploads and copy-backs run on
each lane's copy streams beside them.  Results are copied to a pinned
host output ring per batch; a request completes when its batch's copy-back
has finished, and its device ring space is freed when it is retired.

``Scheduler`` holds the policy and the ring bookkeeping and runs without a
GPU (the CPU tests drive it with a fake device); ``ServingEngine`` binds it
to CUDA streams, events and the library's kernels.
"""
from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np


# ------------------------------------------------------------------ rings
class Ring:
    """FIFO allocator of contiguous ranges in [0, cap): a range never wraps
    past the end (the tail left unused at a wrap is reclaimed when the range
    before it is freed).  Ranges are freed in allocation order (``free``);
    ``release`` frees one out of order (a cancelled request), and its space
    comes back once every older range has been freed."""

    def __init__(self, cap: int):
        if cap <= 0:
            raise ValueError("ring capacity must be positive")
        self.cap = int(cap)
        self.head = 0
        self.live: collections.deque = collections.deque()   # (start, size)
        self.dead: set = set()                               # released, not yet reclaimed

    def alloc(self, n: int):
        """Start of a free range of n >= 1 elements, or None."""
        n = max(int(n), 1)
        if n > self.cap:
            return None
        if not self.live:
            self.head = 0
            start = 0
        else:
            tail = self.live[0][0]
            if self.head > tail:
                if self.head + n <= self.cap:
                    start = self.head
                elif n <= tail:
                    start = 0
                else:
                    return None
            else:
                # live ranges wrap: free space is [head, tail)
                if self.head + n <= tail:
                    start = self.head
                else:
                    return None
        self.live.append((start, n))
        self.head = start + n
        return start

    def _reclaim(self) -> None:
        while self.live and self.live[0][0] in self.dead:
            self.dead.discard(self.live.popleft()[0])
        if not self.live:
            self.head = 0

    def free(self, start: int) -> None:
        self._reclaim()
        if not self.live or self.live[0][0] != start:
            raise RuntimeError("ring ranges must be freed in allocation order")
        self.live.popleft()
        self._reclaim()

    def release(self, start: int) -> None:
        """Free a live range out of allocation order."""
        if not any(s == start for s, _ in self.live) or start in self.dead:
            raise RuntimeError(f"ring range at {start} is not live")
        self.dead.add(start)
        self._reclaim()

    @property
    def used(self) -> int:
        return sum(n for _, n in self.live)

    def fits_ever(self, n: int) -> bool:
        return max(int(n), 1) <= self.cap


# --------------------------------------------------------------- requests
@dataclasses.dataclass
class Request:
    """One descriptor + VJP request (host arrays, local indices)."""

    rid: int
    lane: str
    n_atoms: int
    coords: np.ndarray          # (n_total, 3) f64: contributing atoms, then ghosts
    species: np.ndarray         # (n_total,) i32
    image: np.ndarray           # (n_total,) i32 master row of every coordinate row
    counts: np.ndarray          # (n_atoms,) i32
    nbl: np.ndarray             # (nnz,) i32 local coordinate rows
    dE: np.ndarray              # (n_atoms, width) f64
    arrival: float = 0.0
    max_neigh: int = -1
    # filled by the scheduler; state: new -> pending -> admitted -> launched
    # -> done, or cancelled (from new, pending or admitted)
    state: str = "new"
    slots: tuple | None = None  # (row0, atom0, entry0)
    staged: object = None
    admitted_at: float = 0.0
    done_at: float = 0.0
    desc: np.ndarray | None = None
    grad: np.ndarray | None = None

    def __post_init__(self):
        if self.max_neigh < 0:
            self.max_neigh = int(self.counts.max()) if self.counts.size else 0

    @property
    def n_total(self) -> int:
        return int(self.coords.shape[0])

    @property
    def nnz(self) -> int:
        return int(self.nbl.shape[0])


@dataclasses.dataclass
class LaneCaps:
    rows: int
    atoms: int
    entries: int


@dataclasses.dataclass
class BatchPlan:
    lane: str
    reqs: list
    row0: int
    n_rows: int
    max_neigh: int
    out0: int = -1
    handle: object = None


def lane_bytes_per_row(width: int) -> int:
    """Device bytes per row slot: centre, start, count, dL/d(desc), desc, force."""
    return 4 + 8 + 4 + 8 * width + 8 * width + 24


def plan_caps(budget_bytes: int, widths: dict, shares: dict, work_bytes: dict,
              atoms_per_row: float = 3.0, entries_per_row: float = 40.0) -> dict:
    """Ring capacities of every lane from the HBM budget: lane k gets
    shares[k] of what the batch work spaces leave, split between its rings
    in the given atom / neighbour-entry ratios per row."""
    left = budget_bytes - sum(work_bytes.values())
    if left <= 0:
        raise ValueError("HBM budget below the batch work spaces")
    tot = sum(shares.values())
    caps = {}
    for k, w in widths.items():
        b = left * shares[k] / tot
        per_row = lane_bytes_per_row(w) + atoms_per_row * 32 + entries_per_row * 4
        r = int(b // per_row)
        caps[k] = LaneCaps(rows=max(r, 1), atoms=max(int(r * atoms_per_row), 1),
                           entries=max(int(r * entries_per_row), 1))
    return caps


class Scheduler:
    """Admission, batching and retirement policy (no device calls).

    The device side is a ``backend`` with ``stage(req)`` (write and upload
    inputs), ``launch(plan)`` (one batched pass + copy-back), ``done(plan)``
    (poll) and ``finish(plan)`` (hand results to the requests)."""

    def __init__(self, caps: dict, backend, max_batch_rows: int = 1 << 19, depth: int = 2,
                 out_rows: int | None = None):
        self.caps = caps
        self.backend = backend
        self.max_batch_rows = int(max_batch_rows)
        self.depth = int(depth)
        self.rings = {k: (Ring(c.rows), Ring(c.atoms), Ring(c.entries)) for k, c in caps.items()}
        self.out = {k: Ring(out_rows or min(c.rows, 2 * self.max_batch_rows)) for k, c in caps.items()}
        self.pending = {k: collections.deque() for k in caps}
        self.admitted = {k: collections.deque() for k in caps}
        self.inflight = {k: collections.deque() for k in caps}
        self.completed: list = []
        self.cancelled: list = []
        self._out_pending: list = []   # output ranges released at the next poll
        self.n_batches = 0
        self.admission_waits = 0
        self.batch_rows: list = []
        self.batch_reqs: list = []
        self.batch_lanes: list = []

    # -- admission ------------------------------------------------------
    def submit(self, req: Request) -> None:
        rr, ra, re = self.rings[req.lane]
        if not (rr.fits_ever(req.n_atoms) and ra.fits_ever(req.n_total) and re.fits_ever(req.nnz)):
            raise ValueError(f"request {req.rid} ({req.n_atoms} atoms) exceeds the lane's whole HBM budget")
        if req.n_atoms > min(self.max_batch_rows, self.out[req.lane].cap):
            raise ValueError(f"request {req.rid} has more rows than one batch holds")
        req.state = "pending"
        self.pending[req.lane].append(req)

    def cancel(self, req: Request) -> bool:
        """Withdraw a request that is not on the GPU yet: a pending one leaves
        its queue; an admitted one (inputs staged, not launched) also gives
        back its ring space.  Returns False for a launched or finished
        request, which completes as usual."""
        if req.state == "new":
            req.state = "cancelled"
            self.cancelled.append(req)
            return True
        for q in (self.pending.get(req.lane, ()), self.admitted.get(req.lane, ())):
            for i, r in enumerate(q):
                if r is req:
                    del q[i]
                    if req.state == "admitted":
                        for ring, start in zip(self.rings[req.lane], req.slots):
                            ring.release(start)
                    req.state = "cancelled"
                    self.cancelled.append(req)
                    return True
        return False

    def _try_admit(self, req: Request) -> bool:
        rr, ra, re = self.rings[req.lane]
        r0 = rr.alloc(req.n_atoms)
        if r0 is None:
            return False
        a0 = ra.alloc(req.n_total)
        if a0 is None:
            self._undo(rr, r0)
            return False
        e0 = re.alloc(req.nnz)
        if e0 is None:
            self._undo(ra, a0)
            self._undo(rr, r0)
            return False
        req.slots = (r0, a0, e0)
        return True

    @staticmethod
    def _undo(ring: Ring, start: int) -> None:
        # the newest range is the one being undone
        s, n = ring.live.pop()
        assert s == start
        ring.head = ring.live[-1][0] + ring.live[-1][1] if ring.live else 0

    def admit(self, now: float, max_rows: int | None = None) -> int:
        """Admit pending requests in arrival order per lane while their
        footprint fits; with ``max_rows``, stop a lane once that many rows
        were staged in this call (so launches are not held back by a long
        run of staging)."""
        n = 0
        for k, q in self.pending.items():
            rows = 0
            while q and (max_rows is None or rows < max_rows):
                req = q[0]
                if not self._try_admit(req):
                    self.admission_waits += 1
                    break
                q.popleft()
                req.admitted_at = now
                req.state = "admitted"
                self.backend.stage(req)
                self.admitted[k].append(req)
                rows += req.n_atoms
                n += 1
        flush = getattr(self.backend, "flush", None)
        if flush is not None:
            flush()
        return n

    # -- batching -------------------------------------------------------
    def _next_plan(self, k: str):
        q = self.admitted[k]
        if not q:
            return None
        first = q[0]
        row0 = first.slots[0]
        reqs, rows, mx = [], 0, 0
        cap = min(self.max_batch_rows, self.out[k].cap)
        for req in q:
            # rows must be contiguous in the row ring (a wrap ends the batch);
            # atoms and neighbour entries are addressed per row
            if req.slots[0] != row0 + rows or rows + req.n_atoms > cap:
                break
            reqs.append(req)
            rows += req.n_atoms
            mx = max(mx, req.max_neigh)
        out0 = self.out[k].alloc(rows)
        if out0 is None:
            return None
        for req in reqs:
            q.popleft()
            req.state = "launched"
        return BatchPlan(k, reqs, row0, rows, mx, out0)

    def launch(self) -> int:
        n = 0
        for k in self.caps:
            while len(self.inflight[k]) < self.depth:
                plan = self._next_plan(k)
                if plan is None:
                    break
                self.backend.launch(plan)
                self.inflight[k].append(plan)
                self.n_batches += 1
                self.batch_rows.append(plan.n_rows)
                self.batch_reqs.append(len(plan.reqs))
                self.batch_lanes.append(k)
                n += 1
        return n

    # -- completion -----------------------------------------------------
    def poll(self, now: float) -> list:
        """Completed requests.  Their ``desc`` / ``grad`` are views of the
        pinned output ring, valid until the next ``poll``."""
        for plan in self._out_pending:
            self.out[plan.lane].free(plan.out0)
        self._out_pending = []
        done = []
        for k, q in self.inflight.items():
            while q and self.backend.done(q[0]):
                plan = q.popleft()
                self.backend.finish(plan)
                for req in plan.reqs:
                    req.done_at = now
                    req.state = "done"
                    done.append(req)
                self._retire(plan)
        self.completed.extend(done)
        return done

    def _retire(self, plan: BatchPlan) -> None:
        rr, ra, re = self.rings[plan.lane]
        for req in plan.reqs:
            r0, a0, e0 = req.slots
            rr.free(r0)
            ra.free(a0)
            re.free(e0)
        self._out_pending.append(plan)

    def idle(self) -> bool:
        return not any(self.pending[k] or self.admitted[k] or self.inflight[k] for k in self.caps)

    def step(self, now: float) -> list:
        done = self.poll(now)
        self.admit(now)
        self.launch()
        return done


# ------------------------------------------------------------ staging plan
# per staged field: bytes per atom (coords, species, image), per entry (nbl)
# or per row (centre, begin, counts; dE takes 8 * width)
_FIELD_UNITS = (("atom", 24), ("atom", 4), ("atom", 4), ("entry", 4), ("row", 4), ("row", 8), ("row", 4),
                ("row", None))


def field_bytes(n: int, nt: int, nnz: int, width: int) -> list:
    """Bytes of each staged field of one request (ld_stage_pack's order)."""
    per = {"atom": nt, "entry": nnz, "row": n}
    return [per[k] * (8 * width if b is None else b) for k, b in _FIELD_UNITS]


def stage_chunks(items: list, cap_bytes: int) -> list:
    """Split requests (in admission order) into staging chunks.

    items: (n_atoms, n_total, nnz, width, (row0, atom0, entry0)) per request.
    A chunk is a run of requests whose ring slots continue one another in
    all three rings (no wrap in between), so that each field of the run is
    one contiguous device range; a chunk is closed before it would exceed
    cap_bytes of staging (a larger request stands alone).  Returns lists of
    indices into items."""
    chunks, cur, nxt, size = [], [], None, 0
    for i, (n, nt, nnz, w, slots) in enumerate(items):
        b = sum(field_bytes(n, nt, nnz, w))
        if cur and tuple(slots) == nxt and size + b <= cap_bytes:
            cur.append(i)
            size += b
        else:
            if cur:
                chunks.append(cur)
            cur, size = [i], b
        nxt = (slots[0] + n, slots[1] + nt, slots[2] + nnz)
    if cur:
        chunks.append(cur)
    return chunks


def chunk_layout(items: list, align: int = 256):
    """Field-by-field layout of one chunk's staging block.

    Returns (starts, totals, offsets, block_bytes): the byte offset of each
    field's run in the block (aligned), each run's length, and per request
    the byte offset of its part inside each run."""
    sizes = [field_bytes(n, nt, nnz, w) for n, nt, nnz, w, _ in items]
    totals = [sum(col) for col in zip(*sizes)] if sizes else [0] * len(_FIELD_UNITS)
    starts, t = [], 0
    for tot in totals:
        starts.append(t)
        t += (tot + align - 1) // align * align
    offsets, run = [], [0] * len(totals)
    for sz in sizes:
        offsets.append(list(run))
        run = [a + b for a, b in zip(run, sz)]
    return starts, totals, offsets, t


# ------------------------------------------------------------ device side
class _Lane:
    """Device rings, pinned staging and streams of one descriptor kind."""

    def __init__(self, torch, name, kind, caps: LaneCaps, max_batch_rows, out_rows, stage_bytes, dev):
        from . import _ext

        self.torch = torch
        self.name = name
        self.kind = kind
        self.W = int(kind.width)
        W = self.W
        f64, i32, i64 = torch.float64, torch.int32, torch.int64
        self.coords = torch.zeros((caps.atoms, 3), dtype=f64, device=dev)
        self.species = torch.zeros(caps.atoms, dtype=i32, device=dev)
        self.image = torch.zeros(caps.atoms, dtype=i32, device=dev)
        self.nbl = torch.zeros(caps.entries, dtype=i32, device=dev)
        self.centre = torch.zeros(caps.rows, dtype=i32, device=dev)
        self.begin = torch.zeros(caps.rows, dtype=i64, device=dev)
        self.counts = torch.zeros(caps.rows, dtype=i32, device=dev)
        self.dE = torch.zeros((caps.rows, W), dtype=f64, device=dev)
        self.desc = torch.zeros((caps.rows, W), dtype=f64, device=dev)
        self.grad = torch.zeros((caps.rows, 3), dtype=f64, device=dev)
        self.off = torch.zeros(max_batch_rows + 1, dtype=i64, device=dev)
        self.work_bytes = int(_ext._rows_work_bytes(kind, max_batch_rows, True))
        self.work = torch.empty(self.work_bytes + 256, dtype=torch.uint8, device=dev)
        self.work_ptr = (self.work.data_ptr() + 255) & ~255
        self.out_desc = torch.empty((out_rows, W), dtype=f64, pin_memory=True)
        self.out_grad = torch.empty((out_rows, 3), dtype=f64, pin_memory=True)
        self.stage = torch.empty(stage_bytes, dtype=torch.uint8, pin_memory=True)
        self.stage_ring = Ring(stage_bytes // 256)      # in 256-byte units
        self.staged = collections.deque()                  # (unit0, event)
        self.s_h2d = torch.cuda.Stream(dev)
        self.s_comp = torch.cuda.Stream(dev)
        self.s_d2h = torch.cuda.Stream(dev)


class ServingEngine:
    """Continuous-batching descriptor + VJP server on one GPU.

    ``lanes`` maps a lane name to a ``DescriptorKind``; ``budget_bytes`` is
    the HBM the lanes' rings, work spaces and offsets may hold in total."""

    def __init__(self, lanes: dict, budget_bytes: int = 40 << 30, shares: dict | None = None,
                 max_batch_rows: int = 1 << 19, depth: int = 2, stage_bytes: int = 512 << 20,
                 out_rows: int | None = None, device=None, tuning: dict | None = None,
                 pack_threads: int | None = None, overlap_lanes: bool = False):
        import concurrent.futures
        import os

        import torch

        from . import _ext
        from . import batch as B

        if not torch.cuda.is_available():
            raise RuntimeError("ServingEngine needs a CUDA device")
        self.torch = torch
        self._ext = _ext
        dev = torch.device(device or "cuda")
        shares = shares or {k: 1.0 for k in lanes}
        widths = {k: int(v.width) for k, v in lanes.items()}
        work = {k: int(_ext._rows_work_bytes(v, max_batch_rows, True)) + 8 * (max_batch_rows + 1)
                for k, v in lanes.items()}
        caps = plan_caps(budget_bytes, widths, shares, work)
        out_rows = out_rows or 2 * max_batch_rows
        self.lanes = {k: _Lane(torch, k, v, caps[k], max_batch_rows, min(out_rows, caps[k].rows), stage_bytes, dev)
                      for k, v in lanes.items()}
        # overlap_lanes: each lane's kernels on its own stream, so batches of
        # different lanes share the SMs; otherwise one compute stream runs the
        # lanes' batches in launch order (their copies still overlap them).  A
        # bispectrum Z CTA needs a whole SM's shared memory and waits while
        # symmetry-function CTAs hold part of one: on the B200 overlapped
        # lanes ran no faster than lanes in turn, and up to 6% slower
        self.overlap_lanes = bool(overlap_lanes)
        if not self.overlap_lanes:
            shared = torch.cuda.Stream(dev)
            for ln in self.lanes.values():
                ln.s_comp = shared
        for k, v in lanes.items():
            if tuning and k in tuning:
                B.set_tuning(v, tuning[k])
        self.sched = Scheduler(caps, self, max_batch_rows=max_batch_rows, depth=depth,
                               out_rows=min(out_rows, min(c.rows for c in caps.values())))
        self.caps = caps
        self.launches = 0
        self.host_stage_s = 0.0
        # host threads that pack admitted requests into pinned staging (the
        # packing releases the interpreter lock)
        self._pack_threads = max(1, pack_threads if pack_threads is not None else min(16, os.cpu_count() or 1))
        self._pool = (concurrent.futures.ThreadPoolExecutor(self._pack_threads, thread_name_prefix="ld-pack")
                      if self._pack_threads > 1 else None)
        self._jobs: list = []
        self.t0 = time.perf_counter()

    def clock(self) -> float:
        return time.perf_counter() - self.t0

    def close(self) -> None:
        """Stop the packing threads (the device rings go with the engine)."""
        if self._pool is not None:
            self._pool.shutdown(wait=True)
            self._pool = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- backend interface --------------------------------------------------
    def _reclaim_staging(self, ln: _Lane) -> None:
        while ln.staged and ln.staged[0][1].query():
            u0, _ = ln.staged.popleft()
            ln.stage_ring.free(u0)

    def stage(self, req: Request) -> None:
        """Queue one admitted request for staging; ``flush`` packs the
        admitted requests into pinned staging chunk by chunk
        (``ld_stage_pack_fields``, native, indices rebased) and uploads each
        chunk with one copy per field (``ld_stage_upload_fields``)."""
        torch = self.torch
        torch.cuda.nvtx.range_push(f"serve: stage request {req.rid}")
        try:
            self._stage(req)
        finally:
            torch.cuda.nvtx.range_pop()

    def _stage(self, req: Request) -> None:
        self._jobs.append((req, self.lanes[req.lane]))

    def _pack(self, job) -> None:
        req, outs = job
        r0, a0, e0 = req.slots
        self._ext._stage_pack_fields(req.n_atoms, req.n_total, req.nnz, self.lanes[req.lane].W, r0, a0, e0,
                                     req.coords, req.species, req.image, req.nbl, req.counts, req.dE, outs)

    def _pack_group(self, jobs) -> None:
        for job in jobs:
            self._pack(job)

    def flush(self) -> None:
        """Stage the queued requests: per lane, runs of requests in
        consecutive ring slots form chunks (``stage_chunks``); each chunk
        gets one pinned staging block laid out field by field, its requests
        are packed into it (on host threads when there is enough to copy),
        and it is uploaded with one copy per field, marked by one event."""
        if not self._jobs:
            return
        t_in = time.perf_counter()
        jobs, self._jobs = self._jobs, []
        by_lane: dict = {}
        for req, ln in jobs:
            by_lane.setdefault(ln.name, (ln, []))[1].append(req)
        for ln, reqs in by_lane.values():
            cap = max(1 << 20, ln.stage.numel() // 4)
            items = [(r.n_atoms, r.n_total, r.nnz, ln.W, r.slots) for r in reqs]
            pending = []
            for ch in stage_chunks(items, cap):
                lay = chunk_layout([items[i] for i in ch])
                units = max((lay[3] + 255) // 256, 1)
                self._reclaim_staging(ln)
                u0 = ln.stage_ring.alloc(units)
                while u0 is None:
                    # staging full: pack and upload what is reserved, else
                    # wait for the oldest upload to free its block
                    if pending:
                        self._pack_upload(ln, pending)
                        pending = []
                    elif not ln.staged:
                        raise RuntimeError("request larger than the pinned staging ring")
                    else:
                        ln.staged[0][1].synchronize()
                    self._reclaim_staging(ln)
                    u0 = ln.stage_ring.alloc(units)
                pending.append(([reqs[i] for i in ch], u0, lay))
            if pending:
                self._pack_upload(ln, pending)
        self.host_stage_s += time.perf_counter() - t_in

    def _pack_upload(self, ln: _Lane, chunks: list) -> None:
        torch = self.torch
        base = ln.stage.data_ptr()
        jobs, total = [], 0
        for reqs, u0, (starts, totals, offsets, nbytes) in chunks:
            blk = base + 256 * u0
            for req, off in zip(reqs, offsets):
                jobs.append((req, [blk + st + o for st, o in zip(starts, off)]))
            total += nbytes
        try:
            if self._pool is None or len(jobs) == 1 or total < (4 << 20):
                self._pack_group(jobs)
            else:
                # longest first onto the least loaded of the workers
                groups = [[] for _ in range(min(self._pack_threads, len(jobs)))]
                load = [0] * len(groups)
                for job in sorted(jobs, key=lambda j: -(j[0].n_total + j[0].nnz + j[0].n_atoms * ln.W)):
                    g = load.index(min(load))
                    groups[g].append(job)
                    load[g] += job[0].n_total + job[0].nnz + job[0].n_atoms * ln.W
                for f in [self._pool.submit(self._pack_group, g) for g in groups]:
                    f.result()
        except Exception:
            # a request failed its index checks: give the chunks' staging
            # blocks back before the error reaches the caller
            for _, u0, _ in chunks:
                ln.stage_ring.release(u0)
            raise
        W = ln.W
        for reqs, u0, (starts, totals, offsets, nbytes) in chunks:
            r0, a0, e0 = reqs[0].slots
            blk = base + 256 * u0
            dst = [ln.coords.data_ptr() + 24 * a0, ln.species.data_ptr() + 4 * a0, ln.image.data_ptr() + 4 * a0,
                   ln.nbl.data_ptr() + 4 * e0, ln.centre.data_ptr() + 4 * r0, ln.begin.data_ptr() + 8 * r0,
                   ln.counts.data_ptr() + 4 * r0, ln.dE.data_ptr() + 8 * W * r0]
            self._ext._stage_upload_fields([blk + st for st in starts], dst, list(totals), ln.s_h2d.cuda_stream)
            ev = torch.cuda.Event()
            ev.record(ln.s_h2d)
            ln.staged.append((u0, ev))
            for req in reqs:
                req.staged = ev

    def launch(self, plan: BatchPlan) -> None:
        torch = self.torch
        torch.cuda.nvtx.range_push(f"serve: {plan.lane} batch of {plan.n_rows} rows")
        try:
            self._launch(plan)
        finally:
            torch.cuda.nvtx.range_pop()

    def _launch(self, plan: BatchPlan) -> None:
        torch = self.torch
        ln = self.lanes[plan.lane]
        r0, n = plan.row0, plan.n_rows
        W = ln.W
        comp = ln.s_comp
        comp.wait_event(plan.reqs[-1].staged)
        n0 = self._ext._launch_count()
        with torch.cuda.stream(comp):
            ln.grad[r0:r0 + n].zero_()
            s = comp.cuda_stream
            self._ext._neighbor_offsets_dev(ln.kind, n, ln.counts.data_ptr() + 4 * r0, ln.off.data_ptr(), False, s)
            self._ext._gradient_rows_dev(ln.kind, n, ln.centre.data_ptr() + 4 * r0, ln.begin.data_ptr() + 8 * r0,
                                         ln.species.data_ptr(), ln.nbl.data_ptr(), ln.off.data_ptr(),
                                         max(plan.max_neigh, 1), ln.coords.data_ptr(), ln.dE.data_ptr() + 8 * W * r0,
                                         ln.grad.data_ptr(), ln.desc.data_ptr() + 8 * W * r0, ln.image.data_ptr(),
                                         ln.work_ptr, ln.work_bytes, s)
            ev_c = torch.cuda.Event()
            ev_c.record(comp)
        self.launches += int(self._ext._launch_count() - n0)
        o = plan.out0
        with torch.cuda.stream(ln.s_d2h):
            ln.s_d2h.wait_event(ev_c)
            ln.out_desc[o:o + n].copy_(ln.desc[r0:r0 + n], non_blocking=True)
            ln.out_grad[o:o + n].copy_(ln.grad[r0:r0 + n], non_blocking=True)
            ev_d = torch.cuda.Event()
            ev_d.record(ln.s_d2h)
        plan.handle = ev_d

    def done(self, plan: BatchPlan) -> bool:
        return plan.handle.query()

    def finish(self, plan: BatchPlan) -> None:
        ln = self.lanes[plan.lane]
        o = plan.out0
        for req in plan.reqs:
            k = req.slots[0] - plan.row0
            req.desc = ln.out_desc[o + k:o + k + req.n_atoms].numpy()
            req.grad = ln.out_grad[o + k:o + k + req.n_atoms].numpy()

    # -- driving ------------------------------------------------------------
    def cancel(self, req: Request) -> bool:
        """Withdraw a request that has not been launched (``Scheduler.cancel``);
        callable from ``serve``'s ``on_done`` callback.  A cancelled request
        gets no results and counts as finished for ``serve``."""
        return self.sched.cancel(req)

    def check_status(self) -> None:
        for ln in self.lanes.values():
            self._ext._sync_status(ln.kind, ln.s_comp.cuda_stream)

    def serve(self, requests: list, arrivals: np.ndarray | None = None, keep_results: bool = False,
              on_done=None, admit_rows: int = 1 << 16) -> dict:
        """Run an open-loop stream: request i is submitted at time
        arrivals[i] (seconds from the start; None: all at once).  Results
        are copied out of the output ring when ``keep_results`` (else only
        ``on_done(req)`` sees them before the ring space is reused)."""
        order = np.argsort(arrivals, kind="stable") if arrivals is not None else np.arange(len(requests))
        arr = np.asarray(arrivals, dtype=np.float64) if arrivals is not None else np.zeros(len(requests))
        self.t0 = time.perf_counter()
        self.host_stage_s = 0.0
        nxt = 0
        n = len(requests)
        done = 0
        sched = self.sched
        c0 = len(sched.cancelled)
        while done + len(sched.cancelled) - c0 < n:
            now = self.clock()
            while nxt < n and arr[order[nxt]] <= now:
                req = requests[order[nxt]]
                req.arrival = float(arr[order[nxt]])
                if req.state != "cancelled":
                    sched.submit(req)
                nxt += 1
            for req in sched.poll(now):
                if keep_results:
                    req.desc = np.array(req.desc)
                    req.grad = np.array(req.grad)
                if on_done is not None:
                    on_done(req)
                done += 1
            sched.admit(now, admit_rows)
            sched.launch()
        self.torch.cuda.synchronize()
        self.check_status()
        served = [r for r in requests if r.state == "done"]
        lat = np.array([r.done_at - r.arrival for r in served]) if served else np.zeros(1)
        atoms = int(sum(r.n_atoms for r in served))
        t_first = float(arr.min()) if n else 0.0
        t_last = max(r.done_at for r in served) if served else 0.0
        span = max(t_last - t_first, 1e-9)
        return {"requests": len(served), "cancelled": n - len(served), "atoms": atoms, "seconds": span,
                "atoms_per_s": atoms / span,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "batches": sched.n_batches, "mean_batch_rows": float(np.mean(sched.batch_rows)) if sched.batch_rows else 0.0,
                "max_batch_requests": int(max(sched.batch_reqs)) if sched.batch_reqs else 0,
                "admission_waits": sched.admission_waits,
                "host_staging_s": self.host_stage_s,
                "gpu_launches": self.launches}


def serve_plain(kinds: dict, requests: list, arrivals: np.ndarray | None = None, keep_results: bool = False) -> dict:
    """The plain per-call path: one ``compute_and_gradient`` call per request
    in arrival order (host buffers in and out, synchronous), forces folded
    onto the contributing atoms on the host."""
    from . import _ext

    n = len(requests)
    arr = np.asarray(arrivals, dtype=np.float64) if arrivals is not None else np.zeros(n)
    order = np.argsort(arr, kind="stable")
    t0 = time.perf_counter()
    n0 = _ext._launch_count()
    done_at = np.zeros(n)
    for i in order:
        req = requests[i]
        while time.perf_counter() - t0 < arr[i]:
            pass
        desc, g = _ext.compute_and_gradient(kinds[req.lane], req.n_atoms, req.species, req.nbl, req.counts,
                                            req.coords, req.dE)
        f = fold_host(g, req.n_atoms, req.image)
        done_at[i] = time.perf_counter() - t0
        if keep_results:
            req.desc, req.grad = desc, f
    lat = done_at - arr
    atoms = int(sum(r.n_atoms for r in requests))
    span = max(float(done_at.max() - arr.min()), 1e-9) if n else 1e-9
    return {"requests": n, "atoms": atoms, "seconds": span, "atoms_per_s": atoms / span,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "gpu_launches": int(_ext._launch_count() - n0)}


def fold_host(grad: np.ndarray, n_atoms: int, image: np.ndarray) -> np.ndarray:
    """Ghost gradient rows added onto their masters (assemble_forces)."""
    out = np.array(grad[:n_atoms], dtype=np.float64, copy=True)
    if grad.shape[0] > n_atoms:
        img = image[n_atoms:]
        for d in range(3):
            out[:, d] += np.bincount(img, weights=grad[n_atoms:, d], minlength=n_atoms)[:n_atoms]
    return out


# ------------------------------------------------------------- workloads
def packing_pool(n_pool: int, n_min: int = 16, n_max: int = 32768, density: float = 0.05, dmin: float = 2.0,
                 cutoff: float = 5.0, seed: int = 0) -> list:
    """Periodic two-species random packings with atom counts drawn
    log-uniformly from [n_min, n_max], prepared (ghosts + neighbour lists)."""
    from . import workloads as Wk

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_pool)).astype(int)
    pool = []
    for i, n in enumerate(sizes):
        x, cell, sp = Wk.random_packing(int(n), density=density, dmin=dmin, n_species=2, seed=seed * 1000 + i)
        pool.append(Wk.prepare(x, cell, sp, cutoff))
    return pool


def request_stream(n_req: int, widths: dict, mix: dict, n_min: int = 16, n_max: int = 32768,
                   density: float = 0.05, dmin: float = 2.0, cutoff: float = 5.0, seed: int = 0,
                   source=None, grads=None, first: int = 0, last: int | None = None, device=None,
                   processes: int = 1) -> list:
    """Requests first .. last-1 of the served stream (``synth.stream_requests``):
    per request its own log-uniform atom count, lane and periodic two-species
    packing, ghosts and neighbour lists built on the device when one is given
    (``workloads.prepare_dev``, identical to the host builder's lists) else on
    the host, and a run of N(0, 1) dL/d(desc) rows.  ``processes`` > 1 cuts
    the packings in that many spawned worker processes."""
    from . import synth
    from . import workloads as Wk

    if device is not None:
        def prep(x, cell, sp, rc):
            return Wk.prepare_dev(x, cell, sp, rc, device=device).to_host(cell)
    else:
        prep = Wk.prepare
    reqs = []
    for i, lane, cfg, dE in synth.stream_requests(n_req, widths, mix, prep, n_min, n_max, density, dmin, cutoff,
                                                  seed, source, grads, first, last, processes):
        r = Request(i, lane, cfg.n_atoms, cfg.coords, cfg.species, cfg.image, cfg.counts, cfg.nbl, dE)
        r.cfg = cfg
        reqs.append(r)
    return reqs


def make_requests(pool: list, n_req: int, widths: dict, mix: dict, seed: int = 0) -> list:
    """n_req requests drawing configurations uniformly from ``pool`` and lanes
    by the probabilities in ``mix``; each gets an N(0, 1) dL/d(desc) (shared
    per pool entry and lane, so memory stays bounded)."""
    rng = np.random.default_rng(seed)
    names = list(mix)
    p = np.array([mix[k] for k in names], dtype=np.float64)
    p /= p.sum()
    dE = {}
    reqs = []
    for i in range(n_req):
        c = int(rng.integers(len(pool)))
        k = names[int(rng.choice(len(names), p=p))]
        cfg = pool[c]
        if (c, k) not in dE:
            dE[(c, k)] = np.random.default_rng(seed * 7919 + c * 31 + len(k)).normal(size=(cfg.n_atoms, widths[k]))
        reqs.append(Request(i, k, cfg.n_atoms, cfg.coords, cfg.species, cfg.image, cfg.counts, cfg.nbl, dE[(c, k)]))
    return reqs


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))
