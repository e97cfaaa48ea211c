#!/usr/bin/env python
"""Benchmark of the descriptor + VJP hot path on B200 (one JSON line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workloads (seeded synthetic inputs; the reference names no dataset):

  serve     (default) the served mixed stream of 20,000 requests: each request
            draws its own atom count log-uniformly from [16, 32768] and its own
            periodic two-species random packing (0.05 A^-3, d_min 2 A, rc 5 A);
            70% 24-d symmetry functions / 30% bispectrum 2J=8, desc + VJP vs
            N(0,1) upstream, Poisson arrivals.  value: the batched resident pass
            over steps of 200 requests (inputs in HBM); e2e: the
            continuous-batching server over the whole stream, host arrays in and
            out, beside the plain per-call path (one compute_and_gradient per
            request) on the same stream, p50/p99 of both at 1k / 10k / 50k
            requests/s.
  batch512  512 strained, jittered Si diamond supercells n_i ~ U{1..6}, each
            with 24-d symmetry functions and bispectrum 2J=6, desc + VJP: one
            persistent launch per descriptor under a CUDA graph (autotuned
            launch shape) vs the per-configuration launch loop.
  bs8       8192-atom two-species packing, bispectrum 2J=8, desc + VJP
  sf24      4096-atom Si diamond 8x8x8 (jitter 0.1 A), 24-d symmetry functions

After the timed regions the CPU leg runs the oracle on a bounded sample of
the same inputs (the baseline rate) and checks the GPU results of that sample
against it (descriptors 1e-10, gradients 1e-8 relative); a failed check
stops the benchmark.

--impl reference: the reference-side CPU path of the same workload on all
host cores (desc + VJP by the oracle's analytic adjoint, since the
reference's Enzyme gradient cannot be built offline; the reference's own C++
forward from oracle/_ref timed beside it).  Its inputs are built by the same
generators (synth.py, loaded by file path) and the reference's own
neighbour-list builder, so that process loads nothing of this library.

Multi-GPU (torchrun): replicas only -- every rank runs its own independent
work (the path has no exchange step); value = all ranks' atoms / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from dataclasses import dataclass, field

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "desc+VJP atoms/s, 1 B200: served batch vs plain call; p50/p99 ms @≤1e-10 rel"
# DRAM bytes (read + write) per centre atom of the dominant kernels, from one
# ncu capture each (profiles/, cold caches): bispectrum 2J=8 pass (U kernel
# bsU 1.34 MB, Z kernel bsZ 41.50 MB -- of which the 37.4 MB U blocks that
# the U kernel has just written, an L2 hit outside the profiler -- and the
# pair gradient bsR 21.98 MB, 8192-atom launch) and the factored
# symmetry-function kernel (4096-atom launch: 1.73 MB).  Traffic grows with
# the centres processed, so other launch sizes are scaled by their atom counts.
DRAM_BYTES_PER_ATOM = {"bs8": (1.344512e6 + 41.504768e6 + 21.98016e6) / 8192, "sf24": 1.731328e6 / 4096}
BS_KERNELS = "bsU_kernel<8> (U) + bsZ_kernel<8,1,1> (Z, B, Y) + bsR_kernel<8> (pair gradient)"
RATES = (1000.0, 10000.0, 50000.0)
N_STREAM = 20000
REQ_PER_STEP = 200
MIX = {"sf": 0.7, "bs": 0.3}
DESC_RTOL, GRAD_RTOL = 1e-10, 1e-8


def _synth():
    """synth.py loaded by file path: importing the package would load its
    native extension, which the reference arm must not."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("ldb200_synth", os.path.join(ROOT, "libdescriptor_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@dataclass
class HostCfg:
    """One configuration in the reference's input layout (host arrays)."""

    n_atoms: int
    coords: np.ndarray
    species: np.ndarray
    image: np.ndarray
    counts: np.ndarray
    nbl: np.ndarray
    cell: np.ndarray = field(default=None)

    @property
    def n_total(self) -> int:
        return int(self.coords.shape[0])


def ref_prepare(x, cell, species, cutoff, pbc=(1, 1, 1)):
    """Ghosts and full neighbour lists from the reference's own builder
    (nbl_create_paddings / nbl_build, compiled from its sources into
    oracle/_ref): the reference arm's inputs, identical to this library's
    builder's."""
    from oracle import Reference

    x = np.ascontiguousarray(x, dtype=np.float64)
    species = np.ascontiguousarray(species, dtype=np.int32)
    n = x.shape[0]
    pc, ps, pi = Reference.create_paddings(cutoff, np.asarray(cell), list(pbc), x, species)
    allx = np.ascontiguousarray(np.concatenate([x, pc]))
    need = np.zeros(allx.shape[0], np.int32)
    need[:n] = 1
    counts, nbl = Reference.neighbor_list(allx, cutoff, need, n)
    image = np.concatenate([np.arange(n, dtype=np.int32), pi.astype(np.int32)])
    return HostCfg(n, allx, np.concatenate([species, ps]).astype(np.int32), image, counts.astype(np.int32),
                   nbl.astype(np.int32), np.asarray(cell))


def rel_err(x, ref):
    """max |x - ref| / max(|ref|, 1e-3 * column scale) (the tests' rule)."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if ref.size == 0:
        return 0.0
    r2 = ref.reshape(ref.shape[0], -1)
    x2 = x.reshape(r2.shape)
    den = np.maximum(np.abs(r2), 1e-3 * np.max(np.abs(r2), axis=0, keepdims=True))
    den = np.where(den == 0, 1.0, den)
    if not np.all(np.isfinite(x2)):
        return float("inf")
    return float(np.max(np.abs(x2 - r2) / den))


def fold(grad, n_atoms, image):
    out = np.array(grad[:n_atoms], dtype=np.float64, copy=True)
    if grad.shape[0] > n_atoms:
        for d in range(3):
            out[:, d] += np.bincount(image[n_atoms:], weights=grad[n_atoms:, d], minlength=n_atoms)[:n_atoms]
    return out


class Parity:
    """Running maximum of the GPU-vs-oracle errors of a bench's sample."""

    def __init__(self):
        self.n, self.atoms, self.ed, self.eg = 0, 0, 0.0, 0.0

    def add(self, what, desc, desc_ref, grad=None, grad_ref=None):
        ed = rel_err(desc, desc_ref)
        eg = rel_err(grad, grad_ref) if grad is not None else 0.0
        if not (ed <= DESC_RTOL and eg <= GRAD_RTOL):
            raise RuntimeError(f"parity check failed for {what}: descriptors {ed:.3e}, gradient {eg:.3e}")
        self.n += 1
        self.atoms += int(np.asarray(desc).shape[0])
        self.ed, self.eg = max(self.ed, ed), max(self.eg, eg)

    def summary(self, against):
        return {"checked": self.n, "centres": self.atoms, "desc_max_rel": self.ed, "grad_max_rel": self.eg,
                "bars": {"desc": DESC_RTOL, "grad": GRAD_RTOL}, "against": against}


# --------------------------------------------------------------- specs
def sf24_spec(species):
    t, sz, p = _synth().sf24_params()
    return dict(kind="sf", types=t, sizes=sz, params=p, cutoff=5.0, species=list(species))


def bs_spec(J, species, weights):
    return dict(kind="bs", rfac0=0.99363, twojmax=J, style=3, rmin0=0.0, switch_flag=1, bzero_flag=0, cutoff=5.0,
                species=list(species), weights=list(weights))


def gpu_prepare(x, cell, species, cutoff, pbc=(1, 1, 1)):
    from libdescriptor_b200 import workloads as W

    return W.prepare(x, cell, species, cutoff, pbc)


def make_workload(name: str, seed: int, prepare=gpu_prepare):
    """The single-configuration workloads; ``prepare`` builds ghosts and
    neighbour lists (this library's builder, or the reference's in the
    reference arm: the lists are identical)."""
    sy = _synth()
    if name == "bs8":
        x, cell, sp = sy.random_packing(8192, density=0.05, dmin=2.0, n_species=2, seed=seed)
        cfg = prepare(x, cell, sp, 5.0)
        spec = bs_spec(8, ["A", "B"], [1.0, 0.5])
        desc = {"workload": "bispectrum_2J8_random_packing_8192", "atoms": 8192, "twojmax": 8, "width": 55,
                "species": 2, "density": 0.05, "cutoff": 5.0, "box_side": float(cell[0, 0])}
    elif name == "sf24":
        x, cell = sy.diamond_cell(8, 8, 8, jitter=0.1, seed=seed)
        sp = np.zeros(len(x), np.int32)
        cfg = prepare(x, cell, sp, 5.0)
        spec = sf24_spec(["Si"])
        desc = {"workload": "symmetry_functions_24_diamond_8x8x8", "atoms": 4096, "width": 24, "cutoff": 5.0}
    else:
        raise SystemExit(f"unknown workload {name}")
    desc["mean_neighbours"] = float(cfg.counts.mean())
    return cfg, spec, desc


def diamond_cells(n_configs=512, seed=1, prepare=gpu_prepare, n_max=6, strain=0.03, jitter=0.1, cutoff=5.0):
    """The 512-cell batch (the same draws as libdescriptor_b200.batch.diamond_batch)."""
    sy = _synth()
    rng = np.random.default_rng(seed)
    cfgs = []
    for _ in range(n_configs):
        n1, n2, n3 = (int(v) for v in rng.integers(1, n_max + 1, 3))
        x, cell = sy.diamond_cell(n1, n2, n3, jitter=jitter, strain=strain, seed=int(rng.integers(1 << 31)))
        cfgs.append(prepare(x, cell, np.zeros(len(x), np.int32), cutoff))
    return cfgs


def make_descriptor(spec):
    import libdescriptor_b200 as lds

    if spec["kind"] == "bs":
        return lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, spec["rfac0"],
                                                  spec["twojmax"], spec["style"], 0, spec["rmin0"],
                                                  spec["switch_flag"], spec["bzero_flag"], spec["cutoff"],
                                                  spec["species"], spec["weights"])
    return lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, spec["species"], "cos",
                                              spec["cutoff"], spec["types"], spec["sizes"], spec["params"])


def make_oracle(spec):
    from oracle import OracleDescriptor

    ns = len(spec["species"])
    cm = np.full((ns, ns), spec["cutoff"])
    if spec["kind"] == "bs":
        return OracleDescriptor.bispectrum(spec["rfac0"], spec["twojmax"], spec["style"], spec["rmin0"],
                                           spec["switch_flag"], spec["bzero_flag"], ns, cm, spec["weights"])
    return OracleDescriptor.symmetry_functions(ns, cm, spec["types"], spec["sizes"], spec["params"])


def algorithmic_flops(spec, cfg, weights):
    """Algorithmic FP64 flops of one desc+VJP pass over cfg's centres."""
    from libdescriptor_b200 import flops as F

    if spec["kind"] == "bs":
        n_in = float(cfg.counts.sum())
        per = F.bs_flops_per_atom(spec["twojmax"], spec["style"], 0.0, True, weights)
        nb = F.bs_flops_per_atom(spec["twojmax"], spec["style"], 1.0, True, weights) - per
        return per * cfg.n_atoms + nb * n_in
    # symmetry functions (8 g2 + 16 g4 rows (zeta, lambda, eta)): triplets
    # counted exactly from the neighbour lists
    if cfg.n_atoms == 0:
        return 0.0
    trip = float(np.sum(cfg.counts * (cfg.counts - 1) / 2.0))
    n_eta = len(set(np.asarray(spec["params"])[16 + 2::3]))
    return F.sf_flops_per_atom(float(cfg.counts.mean()), 8, 16, n_eta, True,
                               n_in_pairs=trip / cfg.n_atoms, w=weights) * cfg.n_atoms


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.t:
                self.t.join(timeout=2)

    def summary(self, windows):
        """Median SM clock and active throttle reasons of the samples taken
        inside the timed windows [(t0, t1), ...]."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for (t, ln) in self.lines if any(a <= t <= b for a, b in windows)]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- CPU legs
def oracle_sample(spec, cfgs, budget_s=10.0, threads=None, dEs=None, seed=7):
    """Oracle desc+VJP on all host threads over a bounded sample: whole
    configurations of ``cfgs`` in order until about budget_s of work (the
    last one may be cut to its first rows).  dEs[i]: the upstream gradient
    of cfgs[i] (default: seeded N(0, 1)).  Returns (atoms/s, atoms, threads,
    [(i, desc, unfolded gradient)] of the configurations done whole)."""
    ora = make_oracle(spec)
    threads = threads or os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    atoms, secs, whole = 0, 0.0, []
    for i, cfg in enumerate(cfgs):
        n = cfg.n_atoms
        if secs > 0 and atoms > 0:
            # cap the last configuration so the sample stays near the budget
            n = int(min(n, max(16, (budget_s - secs) * atoms / secs)))
        dE = (dEs[i] if dEs is not None else rng.normal(size=(cfg.n_atoms, ora.width)))[:n]
        t0 = time.perf_counter()
        d, g = ora.run(np.array([n], np.int32), cfg.species, cfg.nbl, cfg.counts[:n], cfg.coords, dE=dE,
                       n_configs=1, config_ptr=np.array([0], np.int32), n_threads=threads)
        secs += time.perf_counter() - t0
        atoms += n
        if n == cfg.n_atoms:
            whole.append((i, d, g))
        if secs >= budget_s:
            break
    return atoms / secs, atoms, threads, whole


def reference_forward_rate(spec, cfgs, budget_s=4.0, threads=None):
    """The reference's own C++ forward (SymmetryFunctions::compute /
    Bispectrum::compute from oracle/_ref) on all host threads over whole
    configurations of ``cfgs`` in order until about budget_s; None where
    that library is not built."""
    from oracle import Reference, ReferenceDescriptor

    if not Reference.available():
        return None
    threads = threads or os.cpu_count() or 1
    ns = len(spec["species"])
    cm = np.full((ns, ns), spec["cutoff"])
    if spec["kind"] == "bs":
        ref = ReferenceDescriptor.bispectrum(spec["rfac0"], spec["twojmax"], spec["style"], spec["rmin0"],
                                             spec["switch_flag"], spec["bzero_flag"], ns, cm, spec["weights"])
    else:
        ref = ReferenceDescriptor.symmetry_functions(ns, cm, spec["types"], spec["sizes"], spec["params"])
    atoms, secs = 0, 0.0
    for cfg in cfgs:
        t0 = time.perf_counter()
        ref.compute(np.array([cfg.n_atoms], np.int32), cfg.species, cfg.nbl, cfg.counts, cfg.coords, n_configs=1,
                    config_ptr=np.array([0], np.int32), n_threads=threads)
        secs += time.perf_counter() - t0
        atoms += cfg.n_atoms
        if secs >= budget_s:
            break
    return atoms / secs if secs > 0 else None


def mix_cpu(specs, requests, budget_s):
    """CPU desc+VJP atoms/s of the request mix: each lane's rate on a sample
    of its own requests (oracle desc+VJP, and the reference's own C++
    forward), combined by the lanes' atom shares.  Returns (rate, sample
    text, threads, reference forward rate, {rid: (desc, folded forces)} of
    the requests sampled whole)."""
    threads = os.cpu_count() or 1
    atoms = {k: sum(r.n_atoms for r in requests if r.lane == k) for k in specs}
    tot = sum(atoms.values())
    spa, spa_fwd, samples, outputs = 0.0, 0.0, [], {}
    for k, spec in specs.items():
        rs = [r for r in requests if r.lane == k]
        if not rs:
            continue
        share = atoms[k] / tot
        rate, n, _, whole = oracle_sample(spec, rs, budget_s=budget_s * share, threads=threads,
                                          dEs=[r.dE for r in rs])
        spa += share / rate
        samples.append(f"{n} {k} centres")
        for i, d, g in whole:
            outputs[rs[i].rid] = (d, fold(g, rs[i].n_atoms, rs[i].image))
        fwd = reference_forward_rate(spec, rs, budget_s=budget_s * share / 3, threads=threads)
        spa_fwd = None if (fwd is None or spa_fwd is None) else spa_fwd + share / fwd
    return 1.0 / spa, ", ".join(samples), threads, (1.0 / spa_fwd if spa_fwd else None), outputs


# ------------------------------------------------------------------ serve
def serve_specs():
    return {"sf": sf24_spec(["A", "B"]), "bs": bs_spec(8, ["A", "B"], [1.0, 0.5])}


def run_serve(args, torch, lds, dev, world, rank, local, dist):
    from libdescriptor_b200 import batch as B
    from libdescriptor_b200 import flops as F
    from libdescriptor_b200 import serving as S
    from libdescriptor_b200 import workloads as W
    from libdescriptor_b200.replicas import replica_throughput

    specs = serve_specs()
    kinds = {k: make_descriptor(s) for k, s in specs.items()}
    widths = {k: int(v.width) for k, v in kinds.items()}
    K = args.steps
    t_gen = time.perf_counter()
    reqs = S.request_stream(N_STREAM, widths, MIX, seed=11 + rank, device=dev,
                            processes=max(1, min(16, (os.cpu_count() or 1) // max(world, 1))))
    gen_s = time.perf_counter() - t_gen
    # the resident pass: K steps over (at most 10 distinct) groups of 200 requests
    steps = [reqs[i * REQ_PER_STEP:(i + 1) * REQ_PER_STEP] for i in range(min(K, 10, N_STREAM // REQ_PER_STEP))]

    peak = lds.measure_fp64_peak(4096)
    weights = F.measure_weights(peak)

    # ---- value: one batched resident pass per lane over each step's requests
    passes = []
    for st in steps:
        per = {}
        for k in kinds:
            rs = [r for r in st if r.lane == k]
            if not rs:
                continue
            db = B.DeviceBatch.from_batch(W.concat(rs), kinds[k], device=dev)
            dE = torch.as_tensor(np.concatenate([r.dE for r in rs]), device=dev)
            per[k] = (B.BatchedPass(kinds[k], db, dE), sum(algorithmic_flops(specs[k], r, weights) for r in rs))
        passes.append(per)
    stream = torch.cuda.Stream(device=dev)
    for per in passes:
        for ps, _ in per.values():
            ps.stream = stream
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            for ps, _ in passes[0].values():
                ps.run()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    evs = {k: [] for k in kinds}
    seq_ev = []
    l0 = lds.launch_count()
    windows = []
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        t_a = time.time()
        with torch.cuda.stream(stream):
            for i in range(K):
                s0_ev = torch.cuda.Event(enable_timing=True)
                s0_ev.record(stream)
                for k, (ps, _) in passes[i % len(passes)].items():
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ps.run()
                    e1.record(stream)
                    evs[k].append((e0, e1))
                s1_ev = torch.cuda.Event(enable_timing=True)
                s1_ev.record(stream)
                seq_ev.append((s0_ev, s1_ev))
        torch.cuda.synchronize()
        windows.append((t_a, time.time()))
        seq_launches = lds.launch_count() - l0
        for ps, _ in passes[0].values():
            ps.sync_status()
        # per-lane kernel times (the roofline's denominators): lanes in turn
        ms = {k: sum(a.elapsed_time(b) for a, b in v) for k, v in evs.items()}
        seq_ms = sum(a.elapsed_time(b) for a, b in seq_ev)
        # the same steps with the two lanes concurrently, one stream each (the
        # server with overlap_lanes); a step is timed from its first launch to
        # the end of its slower lane
        lane_streams = {k: torch.cuda.Stream(device=dev) for k in kinds}
        for per in passes:
            for k, (ps, _) in per.items():
                ps.stream = lane_streams[k]
        s0 = lane_streams[next(iter(kinds))]

        def concurrent_step(i, evpair=None):
            per = passes[i % len(passes)]
            start = torch.cuda.Event(enable_timing=evpair is not None)
            start.record(s0)
            for k, (ps, _) in per.items():
                lane_streams[k].wait_event(start)
                ps.run()
            for k in per:
                if lane_streams[k] is not s0:
                    done = torch.cuda.Event()
                    done.record(lane_streams[k])
                    s0.wait_event(done)
            if evpair is not None:
                end = torch.cuda.Event(enable_timing=True)
                end.record(s0)
                evpair.append((start, end))

        for i in range(args.warmup):
            concurrent_step(i)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        steps_ev = []
        l0 = lds.launch_count()
        t_c = time.time()
        for i in range(K):
            concurrent_step(i, steps_ev)
        torch.cuda.synchronize()
        windows.append((t_c, time.time()))
        conc_launches = lds.launch_count() - l0
        for ps, _ in passes[0].values():
            ps.sync_status()
        conc_ms = sum(a.elapsed_time(b) for a, b in steps_ev)
        step_atoms = [sum(r.n_atoms for r in st) for st in steps]
        atoms_timed = sum(step_atoms[i % len(steps)] for i in range(K))
        # value: the steps as the server issues them (lanes in turn on one
        # compute stream, or overlapped with --overlap-lanes)
        launches = conc_launches if args.overlap_lanes else seq_launches
        value, tot_ms, _ = replica_throughput(atoms_timed, conc_ms if args.overlap_lanes else seq_ms, dist, dev)
        flops_timed = {k: sum(per[k][1] for i in range(K) for per in [passes[i % len(passes)]] if k in per)
                       for k in kinds}
        bs_atoms_timed = sum(sum(r.n_atoms for r in steps[i % len(steps)] if r.lane == "bs") for i in range(K))
        del passes
        torch.cuda.empty_cache()

        # ---- e2e: the server over the whole stream at every rate, then the
        # plain per-call path on the same stream at every rate
        eng = S.ServingEngine(kinds, budget_bytes=40 << 30, shares={"sf": 0.45, "bs": 0.55}, device=dev,
                              overlap_lanes=args.overlap_lanes)
        eng.serve(reqs[:64], None)
        kept = {}                       # results of the first step's requests, top rate

        def keep_first_step(req):
            if req.rid < REQ_PER_STEP:
                kept[req.rid] = (np.array(req.desc), np.array(req.grad))

        sweep, served, plain = [], {}, {}
        for rate in sorted(RATES):
            sch = eng.sched
            sch.batch_rows, sch.batch_reqs, sch.batch_lanes, sch.n_batches = [], [], [], 0
            eng.launches = 0
            t_b = time.time()
            res = eng.serve(reqs, S.poisson_arrivals(N_STREAM, rate, seed=21),
                            on_done=keep_first_step if rate == max(RATES) else None)
            windows.append((t_b, time.time()))
            served[rate] = res
        eng.close()
        del eng
        torch.cuda.empty_cache()
        for rate in sorted(RATES):
            plain[rate] = S.serve_plain(kinds, reqs, S.poisson_arrivals(N_STREAM, rate, seed=21))
        for rate in sorted(RATES):
            sv, pl = served[rate], plain[rate]
            sweep.append({"rate_per_s": rate,
                          "served": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in sv.items()},
                          "plain": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in pl.items()},
                          "served_over_plain": sv["atoms_per_s"] / pl["atoms_per_s"]})
        # whole-job end-to-end rates: every rank's atoms over the slowest
        # rank's span (each rank serves its own stream)
        top = max(RATES)
        e2e_served, _, _ = replica_throughput(served[top]["atoms"], 1e3 * served[top]["seconds"], dist, dev)
        e2e_plain, _, _ = replica_throughput(plain[top]["atoms"], 1e3 * plain[top]["seconds"], dist, dev)
    if rank != 0:
        return None
    top, low = max(RATES), min(RATES)
    ach_bs = flops_timed["bs"] / (ms["bs"] * 1e-3) / 1e12 if ms.get("bs") else 0.0
    ach_sf = flops_timed["sf"] / (ms["sf"] * 1e-3) / 1e12 if ms.get("sf") else 0.0
    roof = {"bound": "fp64", "achieved": ach_bs, "peak": peak, "unit": "TFLOP/s", "frac": ach_bs / peak,
            "traffic": DRAM_BYTES_PER_ATOM["bs8"] * bs_atoms_timed / K,
            "traffic_note": "bytes per step of the bispectrum lane, ncu DRAM bytes per atom of the 8192-atom "
                            "launch (profiles/) times the lane's atoms per step",
            "kernel": BS_KERNELS + " (bispectrum 2J=8 lane of the batched pass)",
            "flops_per_step": flops_timed["bs"] / K, "share_of_pass_time": ms.get("bs", 0.0) / sum(ms.values()),
            "timing": "per-lane CUDA events with the lanes in turn on one stream",
            "flop_count": "libdescriptor_b200/flops.py: U recursion + Z/B/Y + the reverse-mode pair sweep",
            "peak_source": "bench.py FP64 FMA probe (ld_measure_fp64_peak), same run; MEASURED_PEAKS.json has no "
                           "FP64 figure",
            "call_weights_flops": {k: round(v, 1) for k, v in weights.items()},
            "sf_lane": {"achieved": ach_sf, "frac": ach_sf / peak, "kernel": "sfg_kernel<1,1,0>",
                        "share_of_pass_time": ms.get("sf", 0.0) / sum(ms.values())}}
    cpu, parity = None, None
    if not args.no_cpu_baseline and world == 1:
        r, sample, thr, fwd, outs = mix_cpu(specs, reqs[:REQ_PER_STEP], budget_s=12.0)
        cpu = {"value": r, "unit": "atoms/s", "cores": thr, "kind": "port",
               "sample": f"{sample} of the stream's first {REQ_PER_STEP} requests (whole requests in order), "
                         f"desc+VJP by the oracle's analytic adjoint on all host threads, combined by the mix's "
                         f"atom shares",
               "reference_forward": {"value": fwd, "unit": "atoms/s", "kind": "reference",
                                     "what": "the reference's own C++ forward (oracle/_ref) alone, same requests"}}
        chk = Parity()
        for rid, (d_ref, f_ref) in outs.items():
            if rid in kept:
                chk.add(f"served request {rid}", kept[rid][0], d_ref, kept[rid][1], f_ref)
        parity = chk.summary("oracle desc + analytic VJP, served results at the top rate")
    n_steps_stream = N_STREAM / REQ_PER_STEP
    h2d_bytes = sum(r.coords.nbytes + r.species.nbytes + r.image.nbytes + r.nbl.nbytes + r.counts.nbytes
                    + r.dE.nbytes + 12 * r.n_atoms for r in reqs)
    d2h_bytes = sum(8 * r.n_atoms * (widths[r.lane] + 3) for r in reqs)
    atoms_total = sum(r.n_atoms for r in reqs)
    e2e = {"value": e2e_served, "unit": "atoms/s",
           "h2d_bytes_per_step": int(h2d_bytes / n_steps_stream), "d2h_bytes_per_step": int(d2h_bytes / n_steps_stream),
           "api": "libdescriptor_b200.serving.ServingEngine.serve (host numpy requests in, host results out), "
                  f"{N_STREAM} requests, Poisson arrivals at {int(top)}/s",
           "p50_ms": served[top]["p50_ms"], "p99_ms": served[top]["p99_ms"],
           "plain_call": {"value": e2e_plain, "p50_ms": plain[top]["p50_ms"],
                          "p99_ms": plain[top]["p99_ms"],
                          "api": "libdescriptor_b200.compute_and_gradient per request + host fold"},
           "served_over_plain": e2e_served / e2e_plain,
           "rate_sweep": sweep}
    cdesc = {"workload": "served_mixed_stream_sf24_70_bs2J8_30", "requests": N_STREAM,
             "requests_per_step": REQ_PER_STEP, "atoms": int(atoms_total),
             "atoms_per_request": "log-uniform in [16, 32768], drawn per request; each request its own periodic "
                                  "packing cut from 4 random packings of 32768 atoms",
             "density": 0.05, "d_min": 2.0, "cutoff": 5.0, "mix": MIX, "hbm_budget_gb": 40,
             "stream_setup_s": round(gen_s, 1),
             "l2": "inputs of every step (>= 100 MB per lane pass) exceed the 126 MB L2 footprint reuse; no flush",
             "value": "batched resident pass (one launch per lane per step, inputs in HBM), "
                      + ("the two lanes concurrently on their own streams" if args.overlap_lanes
                         else "the lanes in turn on one compute stream") + ", as the server issues them",
             "step_ms": {"lanes_in_turn": seq_ms / K, "lanes_overlapped": conc_ms / K},
             "server_overlap_lanes": bool(args.overlap_lanes),
             "parallelism": f"replicas x{world}"}
    return {
        "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": tot_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded packings, no dataset)", "config": cdesc, "roofline": roof,
        "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "gpu_launches": int(launches),
        "clocks": clk.summary(windows),
        # latency below saturation (the lowest swept rate): above it both paths
        # queue without bound and p50/p99 measure the backlog of the stream
        "p50_ms": served[low]["p50_ms"], "p99_ms": served[low]["p99_ms"], "latency_rate_per_s": low,
        "plain_p50_ms": plain[low]["p50_ms"], "plain_p99_ms": plain[low]["p99_ms"],
    }


# --------------------------------------------------------------- batch512
def run_batch512(args, torch, lds, dev, world, rank, local, dist):
    from libdescriptor_b200 import batch as B
    from libdescriptor_b200 import flops as F
    from libdescriptor_b200 import serving as S
    from libdescriptor_b200 import tuner
    from libdescriptor_b200 import workloads as W

    from libdescriptor_b200.replicas import replica_throughput

    cfgs = B.diamond_batch(512, seed=1 + rank)
    b = W.concat(cfgs)
    specs = {"sf24": sf24_spec(["Si"]), "bs6": bs_spec(6, ["Si"], [1.0])}
    kinds = {k: make_descriptor(s) for k, s in specs.items()}
    peak = lds.measure_fp64_peak(4096)
    weights = F.measure_weights(peak)
    # the launch-shape choices are cached per process (a fresh box each run)
    tu = tuner.Autotuner(cache_path=None)
    passes, chosen, loop_ms, dE_pass = {}, {}, {}, {}
    stream = torch.cuda.Stream(device=dev)
    rng_p = np.random.default_rng(3 + rank)
    for k, kind in kinds.items():
        db = B.DeviceBatch.from_batch(b, kind, device=dev)
        dE_pass[k] = rng_p.normal(size=(db.n_rows, int(kind.width)))
        dE = torch.as_tensor(dE_pass[k], device=dev)
        ps = B.BatchedPass(kind, db, dE, stream=stream)
        chosen[k] = tu.tune(ps, k, 0 if k.startswith("sf") else 1)
        # the per-configuration launch loop (same arena, one call per cell)
        ps.run_per_config()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ps.run_per_config()
        e1.record(stream)
        e1.synchronize()
        loop_ms[k] = e0.elapsed_time(e1)
        ps.capture()
        passes[k] = ps
    n_rows = b.n_rows
    for _ in range(args.warmup):
        for ps in passes.values():
            ps.replay()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    evs = {k: [] for k in passes}
    l0 = lds.launch_count()
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        t_a = time.time()
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                for k, ps in passes.items():
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ps.replay()
                    e1.record(stream)
                    evs[k].append((e0, e1))
        torch.cuda.synchronize()
        # value: both descriptors' graphs concurrently, one stream each; a step
        # is timed from its first replay to the end of the slower one (the
        # per-descriptor times above, graphs in turn, give the roofline)
        streams = {k: (stream if i == 0 else torch.cuda.Stream(device=dev)) for i, k in enumerate(passes)}
        for k, ps in passes.items():
            ps.stream = streams[k]

        def concurrent_step(evpair=None):
            start = torch.cuda.Event(enable_timing=evpair is not None)
            start.record(stream)
            for k, ps in passes.items():
                streams[k].wait_event(start)
                ps.replay()
            for k in passes:
                if streams[k] is not stream:
                    done = torch.cuda.Event()
                    done.record(streams[k])
                    stream.wait_event(done)
            if evpair is not None:
                end = torch.cuda.Event(enable_timing=True)
                end.record(stream)
                evpair.append((start, end))

        for _ in range(args.warmup):
            concurrent_step()
        torch.cuda.synchronize()
        steps_ev = []
        for _ in range(args.steps):
            concurrent_step(steps_ev)
        torch.cuda.synchronize()
        t_b = time.time()
    for ps in passes.values():
        ps.sync_status()
    # graph replays: count kernels per captured pass (the concurrent steps)
    launches = sum(ps.launches_per_pass for ps in passes.values()) * args.steps
    ms = {k: sum(a.elapsed_time(b_) for a, b_ in v) / args.steps for k, v in evs.items()}
    conc_ms = sum(a.elapsed_time(b_) for a, b_ in steps_ev) / args.steps
    value, step_ms, _ = replica_throughput(n_rows, conc_ms, dist, dev)
    # e2e through the batch API: the host batch (pinned, as a server keeps its
    # buffers) uploaded once for both descriptors, one pass per descriptor,
    # descriptors and forces read back into pinned host buffers, every step;
    # a copy stream sends the next descriptor's dE and reads back the last
    # one's results while a pass runs
    def pinned(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dt).pin_memory()

    import dataclasses

    hb = dataclasses.replace(b, coords=pinned(b.coords, torch.float64), species=pinned(b.species, torch.int32),
                             image=pinned(b.image, torch.int32), nbl=pinned(b.nbl, torch.int32),
                             counts=pinned(b.counts, torch.int32), row_centre=pinned(b.row_centre, torch.int32))
    rng_e = np.random.default_rng(5)
    dE_h = {k: pinned(rng_e.normal(size=(n_rows, int(kd.width))), torch.float64) for k, kd in kinds.items()}
    out_h = {k: (torch.empty((n_rows, int(kd.width)), dtype=torch.float64, pin_memory=True),
                 torch.empty((int(b.coords.shape[0]), 3), dtype=torch.float64, pin_memory=True))
             for k, kd in kinds.items()}

    copy_stream = torch.cuda.Stream(device=dev)

    def e2e_step():
        keep = []
        names = list(kinds)
        with torch.cuda.stream(copy_stream):
            dEd = {k: dE_h[k].to(device=dev, non_blocking=True) for k in names}
            ready = {}
            for k in names:
                ready[k] = torch.cuda.Event()
                ready[k].record(copy_stream)
        with torch.cuda.stream(stream):
            db = B.DeviceBatch.from_batch(hb, kinds[names[0]], device=dev, stream=stream)
            for k in names:
                stream.wait_event(ready[k])
                ps = B.BatchedPass(kinds[k], db, dEd[k], stream=stream)
                ps.run()
                done = torch.cuda.Event()
                done.record(stream)
                copy_stream.wait_event(done)
                with torch.cuda.stream(copy_stream):
                    out_h[k][0].copy_(ps.desc, non_blocking=True)
                    out_h[k][1].copy_(ps.grad, non_blocking=True)
                keep.append(ps)
        stream.synchronize()
        copy_stream.synchronize()
        for k, kd in kinds.items():
            _ext_sync(kd)

    def _ext_sync(kd):
        lds._ext._sync_status(kd, stream.cuda_stream)

    for _ in range(2):
        e2e_step()
    ke = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(ke):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / ke
    # the descriptors read back through the copy stream are those of the
    # timed device passes over the same batch (to rounding: sums that meet in
    # atomics vary in order)
    for k, ps in passes.items():
        ref = ps.desc.cpu()
        if not torch.allclose(out_h[k][0], ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max())):
            raise RuntimeError(f"batch512 e2e: {k} descriptors read back differ from the device pass")
    h2d = (hb.coords.nbytes + hb.species.nbytes + hb.image.nbytes + hb.nbl.nbytes + hb.counts.nbytes
           + hb.row_centre.nbytes) + sum(v.nbytes for v in dE_h.values())
    d2h = sum(a.nbytes + g.nbytes for a, g in out_h.values())
    # the same 512 cells x 2 descriptors as 1024 requests to the server
    reqs = []
    rng = np.random.default_rng(5)
    for i, c in enumerate(cfgs):
        for k, kind in kinds.items():
            reqs.append(S.Request(len(reqs), k, c.n_atoms, c.coords, c.species, c.image, c.counts, c.nbl,
                                  rng.normal(size=(c.n_atoms, int(kind.width)))))
    eng = S.ServingEngine(kinds, budget_bytes=8 << 30, device=dev, tuning=chosen)
    eng.serve(reqs[:64], None)
    for r in reqs:
        r.slots = None
    t0 = time.perf_counter()
    st = eng.serve(reqs, None)
    serve_s = time.perf_counter() - t0
    eng.close()
    # whole-job rates: all ranks' atoms over the slowest rank's time
    e2e_rate, _, _ = replica_throughput(n_rows, 1e3 * e2e_s, dist, dev)
    serve_rate, _, _ = replica_throughput(n_rows, 1e3 * serve_s, dist, dev)
    if rank != 0:
        return None
    flop = {k: sum(algorithmic_flops(specs[k], c, weights) for c in cfgs) for k in specs}
    dom = max(ms, key=ms.get)
    ach = flop[dom] / (ms[dom] * 1e-3) / 1e12
    roof = {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
            "kernel": f"{dom} batched pass", "flops_per_step": flop[dom],
            "share_of_step_time": ms[dom] / sum(ms.values()),
            "timing": "per-descriptor graph replays in turn (before the concurrent steps that give value)",
            "peak_source": "bench.py FP64 FMA probe (ld_measure_fp64_peak), same run"}
    cpu, parity = None, None
    if not args.no_cpu_baseline and world == 1:
        secs, secs_fwd = 0.0, 0.0
        samples = []
        chk = Parity()
        rp = passes[next(iter(passes))].db.row_ptr
        for k, spec in specs.items():
            dEs = [dE_pass[k][rp[c]:rp[c + 1]] for c in range(len(cfgs))]
            r, n, thr, whole = oracle_sample(spec, cfgs, budget_s=6.0, dEs=dEs)
            secs += 1.0 / r
            fwd = reference_forward_rate(spec, cfgs, budget_s=2.0)
            secs_fwd = None if (fwd is None or secs_fwd is None) else secs_fwd + 1.0 / fwd
            samples.append(f"{n} centres ({k})")
            ps = passes[k]
            for c, d, g in whole:
                chk.add(f"batch512 {k} cell {c}", ps.descriptors(c).cpu().numpy(), d,
                        ps.forces(c).cpu().numpy(), fold(g, cfgs[c].n_atoms, cfgs[c].image))
        parity = chk.summary("oracle desc + analytic VJP, cells of the timed graph passes")
        cpu = {"value": 1.0 / secs, "unit": "atoms/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": ", ".join(samples) + " of the cells in order; every atom gets both descriptors, desc+VJP "
                                               "by the oracle on all host threads",
               "reference_forward": {"value": (1.0 / secs_fwd) if secs_fwd else None, "unit": "atoms/s",
                                     "kind": "reference",
                                     "what": "the reference's own C++ forward (oracle/_ref), both descriptors"}}
    cdesc = {"workload": "batched_512_diamond_cells_sf24_and_bs2J6", "cells": 512, "atoms": int(n_rows),
             "n_cells_per_axis": "U{1..6}", "strain": 0.03, "jitter": 0.1, "cutoff": 5.0,
             "tuned_launch_shape": chosen,
             "per_config_loop_ms": loop_ms, "graph_pass_ms": ms, "concurrent_step_ms": conc_ms,
             "per_config_loop_atoms_per_s": world * n_rows / (sum(loop_ms.values()) * 1e-3),
             "l2": "inputs exceed L2 (549,722 coordinate rows, ~20 MB neighbour lists, 100+ MB dL/d(desc)); no flush",
             "parallelism": f"replicas x{world}"}
    return {
        "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cells, no dataset)", "config": cdesc,
        "roofline": roof, "cpu_baseline": cpu, "parity": parity,
        "e2e": {"value": e2e_rate, "unit": "atoms/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_s,
                "api": "batch.DeviceBatch.from_batch once (pinned host batch) + BatchedPass.run per descriptor, "
                       "dE up and descriptors and forces back to pinned host memory on a copy stream that "
                       "overlaps the passes, synchronised, every step",
                "serving_engine": {"value": serve_rate, "ms_per_step": 1e3 * serve_s,
                                   "api": "ServingEngine.serve of the 1024 (cell, descriptor) requests, host numpy "
                                          "in/out", "batches": st["batches"]}},
        "gpu_launches": int(launches), "clocks": clk.summary([(t_a, t_b)]),
    }


# ----------------------------------------------------------- single cell
def run_single(args, torch, lds, dev, world, rank, local, dist):
    from libdescriptor_b200 import flops as F
    from libdescriptor_b200.replicas import replica_throughput

    cfg, spec, cdesc = make_workload(args.workload, seed=1 + rank)
    ds = make_descriptor(spec)
    W = ds.width
    n = cfg.n_atoms
    stream = torch.cuda.Stream(device=dev)
    sp = torch.as_tensor(cfg.species, device=dev)
    nbl = torch.as_tensor(cfg.nbl, device=dev)
    cnt = torch.as_tensor(cfg.counts, device=dev)
    x = torch.as_tensor(cfg.coords, device=dev)
    off = torch.empty(n + 1, dtype=torch.int64, device=dev)
    rng = np.random.default_rng(100 + rank)
    dE_h = rng.normal(size=(n, W))
    dE = torch.as_tensor(dE_h, device=dev)
    desc = torch.empty((n, W), dtype=torch.float64, device=dev)
    dc = torch.zeros((cfg.n_total, 3), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    s = stream.cuda_stream
    with torch.cuda.stream(stream):
        maxn = lds._ext._neighbor_offsets_dev(ds, n, cnt.data_ptr(), off.data_ptr(), True, s)

    def step():
        dc.zero_()
        lds._ext._gradient_dev(ds, n, 0, sp.data_ptr(), nbl.data_ptr(), off.data_ptr(), maxn, x.data_ptr(),
                               dE.data_ptr(), dc.data_ptr(), desc.data_ptr(), 0, s)

    peak = lds.measure_fp64_peak(4096)
    weights = F.measure_weights(peak)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        lds._ext._sync_status(ds, s)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    l0 = lds.launch_count()
    with ClockSampler(local) as clk:
        time.sleep(0.5)
        t_begin = time.time()
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(float(k))            # evict L2 between steps (outside the events)
                evs[k][0].record(stream)
                step()
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        t_end = time.time()
        time.sleep(0.1)
    launches = lds.launch_count() - l0
    lds._ext._sync_status(ds, s)
    tot_ms = float(sum(a.elapsed_time(b) for a, b in evs))
    value, tot_ms, _ = replica_throughput(n * args.steps, tot_ms, dist, dev)
    ms_per_step = tot_ms / args.steps
    # the call a user makes, with its inputs staged in pinned host memory
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    h_sp, h_nbl, h_cnt, h_x, h_dE = (pinned(cfg.species), pinned(cfg.nbl), pinned(cfg.counts), pinned(cfg.coords),
                                     pinned(dE_h))
    for _ in range(2):
        lds.compute_and_gradient(ds, n, h_sp, h_nbl, h_cnt, h_x, h_dE)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ke = max(3, min(args.steps, 10))
    for _ in range(ke):
        lds.compute_and_gradient(ds, n, h_sp, h_nbl, h_cnt, h_x, h_dE)
    e2e_s = (time.perf_counter() - t0) / ke
    e2e_rate, _, _ = replica_throughput(n, 1e3 * e2e_s, dist, dev)
    h2d = cfg.species.nbytes + cfg.nbl.nbytes + cfg.counts.nbytes + cfg.coords.nbytes + dE_h.nbytes + 8 * (n + 1)
    d2h = 8 * n * W + 8 * 3 * cfg.n_total
    e2e = {"value": e2e_rate, "unit": "atoms/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_s,
           "api": "libdescriptor_b200.compute_and_gradient (numpy inputs in pinned host memory, numpy results out, one fused pass)"}
    if rank != 0:
        return None
    flop = algorithmic_flops(spec, cfg, weights)
    achieved = flop / (ms_per_step * 1e-3) / 1e12
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": DRAM_BYTES_PER_ATOM[args.workload] * n,
            "traffic_note": "ncu DRAM read + write bytes of one launch (profiles/)",
            "kernel": BS_KERNELS if spec["kind"] == "bs" else "sfg_kernel<1,1,0>",
            "flops_per_step": flop, "peak_source": "bench.py FP64 FMA probe (ld_measure_fp64_peak), same run",
            "call_weights_flops": {k: round(v, 1) for k, v in weights.items()},
            "hbm_bytes_per_step_algorithmic": int(cfg.coords.nbytes + cfg.nbl.nbytes + 8 * n * W * 2
                                                  + 24 * cfg.n_total)}
    cpu, parity = None, None
    if not args.no_cpu_baseline and world == 1:
        r, sample, thr, whole = oracle_sample(spec, [cfg], budget_s=10.0, dEs=[dE_h])
        fwd = reference_forward_rate(spec, [cfg], budget_s=4.0)
        cpu = {"value": r, "unit": "atoms/s", "cores": thr, "kind": "port",
               "sample": f"{sample} of {n} centres, desc+VJP by the oracle's analytic adjoint on all host threads",
               "reference_forward": {"value": fwd, "unit": "atoms/s", "kind": "reference",
                                     "what": "the reference's own C++ forward (oracle/_ref) alone, same cell"}}
        chk = Parity()
        for _, d, g in whole:
            chk.add(args.workload, desc.cpu().numpy(), d, dc.cpu().numpy(), g)
        parity = chk.summary("oracle desc + analytic VJP, the last timed pass")
    return {
        "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no dataset)",
        "config": dict(cdesc, l2="flushed between steps (256 MB write outside the timed events)",
                       parallelism=f"replicas x{world}"),
        "roofline": roof, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "gpu_launches": int(launches),
        "clocks": clk.summary([(t_begin, t_end)]),
    }


# -------------------------------------------------------- reference arm
def run_reference(args):
    """The reference-side CPU path of the same workload on all host threads:
    desc+VJP by the oracle's analytic adjoint (a restatement of the
    reference's algorithm; its Enzyme gradient cannot be built offline), the
    reference's own C++ forward (oracle/_ref) timed beside it.  Inputs come
    from the same generators (synth.py by file path) with the reference's
    own neighbour-list builder: nothing of this library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    rates, fwd_rates, sample = [], [], None
    if args.workload == "serve":
        sy = _synth()
        specs = serve_specs()
        widths = {"sf": 24, "bs": 55}
        reqs = []
        for i, lane, cfg, dE in sy.stream_requests(N_STREAM, widths, MIX, ref_prepare, seed=11, last=REQ_PER_STEP):
            cfg.rid, cfg.lane, cfg.dE = i, lane, dE
            reqs.append(cfg)

        def one(budget):
            r, smp, thr, fwd, _ = mix_cpu(specs, reqs, budget)
            return r, smp, fwd

        cdesc = {"workload": "served_mixed_stream_sf24_70_bs2J8_30", "requests": N_STREAM,
                 "requests_per_step": REQ_PER_STEP, "mix": MIX, "atoms_log_uniform": [16, 32768],
                 "sampled": f"the stream's first {REQ_PER_STEP} requests"}
    elif args.workload == "batch512":
        cfgs = diamond_cells(512, seed=1, prepare=ref_prepare)
        specs = {"sf24": sf24_spec(["Si"]), "bs6": bs_spec(6, ["Si"], [1.0])}

        def one(budget):
            secs, secs_fwd, smp = 0.0, 0.0, []
            for k, spec in specs.items():
                r, n, _, _ = oracle_sample(spec, cfgs, budget_s=budget / 2)
                secs += 1.0 / r
                fwd = reference_forward_rate(spec, cfgs, budget_s=budget / 6)
                secs_fwd = None if (fwd is None or secs_fwd is None) else secs_fwd + 1.0 / fwd
                smp.append(f"{n} centres ({k})")
            return 1.0 / secs, ", ".join(smp), (1.0 / secs_fwd if secs_fwd else None)

        cdesc = {"workload": "batched_512_diamond_cells_sf24_and_bs2J6", "cells": 512}
    else:
        cfg, spec, cdesc = make_workload(args.workload, seed=1, prepare=ref_prepare)

        def one(budget):
            r, n, _, _ = oracle_sample(spec, [cfg], budget_s=budget)
            return r, f"{n} of {cfg.n_atoms} centres", reference_forward_rate(spec, [cfg], budget_s=budget / 3)

    for _ in range(args.warmup):
        one(1.0)
    walls = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r, sample, fwd = one(6.0)
        walls.append(time.perf_counter() - t0)
        rates.append(r)
        if fwd is not None:
            fwd_rates.append(fwd)
    value = statistics.mean(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cdesc,
        "cpu_baseline": {"value": value, "unit": "atoms/s", "cores": threads, "kind": "port",
                         "sample": f"per step about 6 s of desc+VJP work: {sample}, by the oracle's analytic "
                                   f"adjoint (the reference's Enzyme gradient cannot be built offline)",
                         "reference_forward": {"value": statistics.mean(fwd_rates) if fwd_rates else None,
                                               "unit": "atoms/s", "kind": "reference",
                                               "what": "the reference's own C++ forward (oracle/_ref) alone, "
                                                       "same inputs"}},
        "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- GPU
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="serve", choices=["serve", "batch512", "bs8", "sf24"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--overlap-lanes", action="store_true",
                    help="serve: each lane's kernels on its own stream (value and server), instead of the lanes "
                         "in turn on one compute stream")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.steps is None:
        args.steps = {"serve": 10, "batch512": 20}.get(args.workload, 200)
        if args.impl == "reference":
            args.steps = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    import libdescriptor_b200 as lds

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    runner = {"serve": run_serve, "batch512": run_batch512}.get(args.workload, run_single)
    line = runner(args, torch, lds, dev, world, rank, local, dist)
    if line is not None:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
