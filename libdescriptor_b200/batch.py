"""Many configurations of uneven size in one persistent launch per descriptor.

The reference's ``compute_batch`` / ``gradient_batch``
(src/Descriptors.cpp:138-163, 190-215) loop over configurations on the host
and call the per-configuration kernel once each.  Here the rows of all
configurations sit in one device arena (the ``compute_batch`` layout: centre
of row (c, j) is ``j + config_ptr[c]``, neighbour indices global) and one
descriptor + VJP pass covers them all: the kernels are persistent (grid =
SMs x resident CTAs) and claim centre rows from one global atomic counter
(the built-in choice for batches of 8192 rows or more; the ``dynamic_queue``
tuning forces it on (1) or off (2)).  ``BatchedPass.capture()`` records the pass
(gradient zeroing, row-queue reset, the kernels) in a CUDA graph;
``replay()`` re-issues it with one call.  The per-configuration launch loop,
the shape the reference's batch API has, is ``BatchedPass.run_per_config``.

Launch shapes come from ``tuner.Autotuner`` (warps per centre / CTA, CTAs per
SM, pair-kernel chunking, static vs. dynamic row queue).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _ext
from . import workloads as W

TUNE_KEYS = {"sf_warps": 0, "ctas_per_sm": 1, "pair_grid_mult": 2, "dynamic_queue": 3, "sf_generic": 4}


def set_tuning(kind, tuning: dict | None) -> None:
    """Apply a launch-shape tuning (keys of ``TUNE_KEYS``; missing keys and
    values <= 0 restore the built-in choice)."""
    tuning = tuning or {}
    for name, key in TUNE_KEYS.items():
        _ext._set_tuning(kind, key, int(tuning.get(name, 0)))


def get_tuning(kind) -> dict:
    return {name: int(_ext._get_tuning(kind, key)) for name, key in TUNE_KEYS.items()}


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("libdescriptor_b200.batch needs a CUDA device")
    return torch


@dataclass
class DeviceBatch:
    """A ``workloads.Batch`` resident on the device."""

    n_rows: int
    n_total: int
    n_atoms: np.ndarray       # host copy: atoms per configuration
    row_ptr: np.ndarray       # host: first row of every configuration (+ end)
    config_ptr: np.ndarray    # host: first coordinate row of every configuration
    coords: object            # (n_total, 3) f64
    species: object           # (n_total,) i32
    image: object             # (n_total,) i32, global master coordinate row
    nbl: object               # (nnz,) i32
    counts: object            # (n_rows,) i32
    off: object               # (n_rows + 1,) i64
    row_centre: object        # (n_rows,) i32
    max_neigh: int

    @classmethod
    def from_batch(cls, b: W.Batch, kind, device=None, stream=None) -> "DeviceBatch":
        torch = _torch()
        dev = torch.device(device or "cuda")

        def t(a, dt):
            # torch tensors (e.g. pinned host buffers) are copied without
            # blocking the host, numpy arrays through a pageable copy
            if isinstance(a, torch.Tensor):
                return a.to(device=dev, dtype=dt, non_blocking=True)
            return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)

        n_rows = int(b.n_rows)
        counts = t(b.counts, torch.int32)
        off = torch.empty(n_rows + 1, dtype=torch.int64, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        mx = int(_ext._neighbor_offsets_dev(kind, n_rows, counts.data_ptr(), off.data_ptr(), True, s.cuda_stream))
        row_ptr = np.concatenate([[0], np.cumsum(b.n_atoms)]).astype(np.int64)
        nbl = b.nbl if (b.nbl.numel() if isinstance(b.nbl, torch.Tensor) else b.nbl.size) else np.zeros(1, np.int32)
        return cls(n_rows, int(b.coords.shape[0]), np.asarray(b.n_atoms), row_ptr, np.asarray(b.config_ptr),
                   t(b.coords, torch.float64), t(b.species, torch.int32), t(b.image, torch.int32),
                   t(nbl, torch.int32), counts, off, t(b.row_centre, torch.int32), max(mx, 1))

    @property
    def n_configs(self) -> int:
        return int(self.n_atoms.shape[0])


class BatchedPass:
    """Descriptor + force VJP over a ``DeviceBatch`` in one pass.

    ``desc`` (n_rows, width) receives the descriptors, ``grad`` (n_total, 3)
    the VJP folded onto each configuration's contributing atoms (rows
    ``config_ptr[c] .. config_ptr[c] + n_atoms[c]``; ghost rows stay 0).
    The work space is owned here, so a pass allocates nothing and can be
    captured in a CUDA graph.
    """

    def __init__(self, kind, db: DeviceBatch, dE, stream=None):
        torch = _torch()
        self.torch = torch
        self.kind = kind
        self.db = db
        self.width = int(kind.width)
        dev = db.coords.device
        if tuple(dE.shape) != (db.n_rows, self.width) or dE.dtype != torch.float64 or not dE.is_contiguous():
            raise ValueError(f"dE must be a contiguous float64 tensor of shape ({db.n_rows}, {self.width})")
        self.dE = dE
        self.desc = torch.empty((db.n_rows, self.width), dtype=torch.float64, device=dev)
        self.grad = torch.zeros((db.n_total, 3), dtype=torch.float64, device=dev)
        self.work_bytes = int(_ext._rows_work_bytes(kind, db.n_rows, True))
        self.work = torch.empty(self.work_bytes + 256, dtype=torch.uint8, device=dev)
        wp = self.work.data_ptr()
        self.work_ptr = (wp + 255) & ~255
        self.stream = stream if stream is not None else torch.cuda.Stream(dev)
        self.graph = None
        self.launches_per_pass = None

    # one persistent pass over every row of every configuration
    def _issue(self, s) -> None:
        db = self.db
        self.grad.zero_()
        _ext._gradient_rows_dev(self.kind, db.n_rows, db.row_centre.data_ptr(), db.off.data_ptr(),
                                db.species.data_ptr(), db.nbl.data_ptr(), db.off.data_ptr(), db.max_neigh,
                                db.coords.data_ptr(), self.dE.data_ptr(), self.grad.data_ptr(),
                                self.desc.data_ptr(), db.image.data_ptr(), self.work_ptr, self.work_bytes,
                                s.cuda_stream)

    def run(self) -> None:
        """Issue one pass on ``self.stream`` (asynchronous)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            n0 = _ext._launch_count()
            self._issue(self.stream)
            self.launches_per_pass = int(_ext._launch_count() - n0)

    def capture(self) -> None:
        """Record one pass in a CUDA graph (after one eager warm-up pass)."""
        torch = self.torch
        self.run()
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream, capture_error_mode="relaxed"):
            self._issue(self.stream)
        self.graph = g

    def replay(self) -> None:
        if self.graph is None:
            raise RuntimeError("capture() first")
        with self.torch.cuda.stream(self.stream):
            self.graph.replay()

    def run_per_config(self) -> int:
        """The per-configuration launch loop: one descriptor + VJP call per
        configuration over the same arena (the reference's batch loop).
        Returns the number of library kernel launches issued."""
        torch = self.torch
        db = self.db
        n0 = _ext._launch_count()
        with torch.cuda.stream(self.stream):
            self.grad.zero_()
            s = self.stream.cuda_stream
            W_ = self.width
            for c in range(db.n_configs):
                r0, r1 = int(db.row_ptr[c]), int(db.row_ptr[c + 1])
                n = r1 - r0
                if n == 0:
                    continue
                _ext._gradient_dev(self.kind, n, db.row_centre.data_ptr() + 4 * r0, db.species.data_ptr(),
                                   db.nbl.data_ptr(), db.off.data_ptr() + 8 * r0, db.max_neigh,
                                   db.coords.data_ptr(), self.dE.data_ptr() + 8 * W_ * r0, self.grad.data_ptr(),
                                   self.desc.data_ptr() + 8 * W_ * r0, db.image.data_ptr(), s)
        return int(_ext._launch_count() - n0)

    def sync_status(self) -> None:
        _ext._sync_status(self.kind, self.stream.cuda_stream)

    def forces(self, c: int):
        """Folded VJP rows of configuration c (a view)."""
        p = int(self.db.config_ptr[c])
        return self.grad[p:p + int(self.db.n_atoms[c])]

    def descriptors(self, c: int):
        return self.desc[int(self.db.row_ptr[c]):int(self.db.row_ptr[c + 1])]


def diamond_batch(n_configs=512, n_max=6, strain=0.03, jitter=0.1, cutoff=5.0, seed=0):
    """Uneven batch of periodic Si diamond supercells: n1, n2, n3 drawn
    uniformly from {1..n_max}, each cell-matrix entry strained by
    U(-strain, strain) and every coordinate jittered by N(0, jitter)."""
    rng = np.random.default_rng(seed)
    cfgs = []
    for c in range(n_configs):
        n1, n2, n3 = (int(v) for v in rng.integers(1, n_max + 1, 3))
        x, cell = W.diamond_cell(n1, n2, n3, jitter=jitter, strain=strain, seed=int(rng.integers(1 << 31)))
        cfgs.append(W.prepare(x, cell, np.zeros(len(x), np.int32), cutoff))
    return cfgs
