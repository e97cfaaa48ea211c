"""Launch-shape autotuner for the descriptor + VJP kernels.

For one descriptor and one batch shape it times every candidate launch shape
(warps per centre CTA for symmetry functions, resident CTAs per SM, the
pair-kernel chunking of the bispectrum gradient, static grid-stride vs.
dynamic atomic row queue) on the real batch with CUDA events and keeps the
fastest.  Choices are cached in a JSON file keyed by device name, descriptor
signature and the batch's shape class (rows rounded to a power of two,
maximum neighbour count), so a served or repeated workload tunes once.

Results never depend on the tuning beyond the order of floating-point
atomic additions; the tests check that.
"""
from __future__ import annotations

import itertools
import json
import math
import os
import statistics

from . import batch as B

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "libdescriptor_b200", "tuning.json")


def candidates(kind_code: int) -> list[dict]:
    """Candidate launch shapes for descriptor kind 0 (symmetry functions) or
    1 (bispectrum)."""
    if kind_code == 0:
        return [dict(sf_warps=w, ctas_per_sm=c, dynamic_queue=q)
                for w, c, q in itertools.product((1, 2, 4), (0, 8), (1, 2))]
    return [dict(ctas_per_sm=c, pair_grid_mult=m, dynamic_queue=q)
            for c, m, q in itertools.product((0, 1), (2, 4, 8, 16), (1, 2))]


def shape_key(device_name: str, signature: str, n_rows: int, max_neigh: int) -> str:
    bucket = 1 << max(0, int(math.ceil(math.log2(max(n_rows, 1)))))
    return f"{device_name}|{signature}|rows<= {bucket}|max_neigh={max_neigh}"


class Autotuner:
    """Tune-and-cache.  ``tune(pass_, signature)`` returns the chosen shape
    and leaves it applied to ``pass_.kind``."""

    def __init__(self, cache_path: str | None = DEFAULT_CACHE, reps: int = 3):
        self.cache_path = cache_path
        self.reps = int(reps)
        self.cache: dict = {}
        self.log: list = []
        if cache_path and os.path.exists(cache_path):
            try:
                with open(cache_path) as f:
                    self.cache = json.load(f)
            except (OSError, ValueError):
                self.cache = {}

    def _save(self) -> None:
        if not self.cache_path:
            return
        os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def time_shape(self, pass_: "B.BatchedPass", shape: dict) -> float:
        """Median milliseconds of one pass with ``shape`` applied."""
        torch = pass_.torch
        B.set_tuning(pass_.kind, shape)
        pass_.run()  # warm-up (first use also sets kernel attributes)
        ts = []
        for _ in range(self.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(pass_.stream)
            pass_.run()
            e1.record(pass_.stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    def tune(self, pass_: "B.BatchedPass", signature: str, kind_code: int, force: bool = False) -> dict:
        torch = pass_.torch
        dev = torch.cuda.get_device_name(pass_.desc.device)
        key = shape_key(dev, signature, pass_.db.n_rows, pass_.db.max_neigh)
        if not force and key in self.cache:
            shape = self.cache[key]["shape"]
            B.set_tuning(pass_.kind, shape)
            return shape
        results = []
        for shape in candidates(kind_code):
            results.append((self.time_shape(pass_, shape), shape))
        results.sort(key=lambda t: t[0])
        best_ms, best = results[0]
        self.cache[key] = {"shape": best, "ms": best_ms,
                           "table": [{"ms": ms, "shape": sh} for ms, sh in results]}
        self.log.append((key, best_ms, best))
        self._save()
        B.set_tuning(pass_.kind, best)
        return best
