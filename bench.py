#!/usr/bin/env python
"""Benchmark of the descriptor + VJP hot path on B200 (one JSON line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one fused descriptor + force-VJP pass (FP64) over one batch of
synthetic input, with inputs resident in HBM.  Workloads (seeded, synthetic):

  bs8   8192-atom two-species random packing (0.05 A^-3, d_min 2 A, rc 5 A),
        bispectrum 2J=8 (55 components), desc + VJP vs N(0,1) upstream
  sf24  4096-atom Si diamond 8x8x8 (jitter 0.1 A), 24-d symmetry functions,
        desc + VJP

Multi-GPU (torchrun): replicas only -- every rank runs its own independent
batch (the path has no exchange step); value = all ranks' atoms / max time.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "desc+VJP atoms/s"


# --------------------------------------------------------------- workloads
def make_workload(name: str, seed: int):
    from libdescriptor_b200 import workloads as W

    if name == "bs8":
        x, cell, sp = W.random_packing(8192, density=0.05, dmin=2.0, n_species=2, seed=seed)
        cfg = W.prepare(x, cell, sp, 5.0)
        spec = dict(kind="bs", rfac0=0.99363, twojmax=8, style=3, rmin0=0.0, switch_flag=1, bzero_flag=0,
                    cutoff=5.0, species=["A", "B"], weights=[1.0, 0.5])
        desc = {"workload": "bispectrum_2J8_random_packing_8192", "atoms": 8192, "twojmax": 8, "width": 55,
                "species": 2, "density": 0.05, "cutoff": 5.0, "box_side": float(cell[0, 0])}
    elif name == "sf24":
        x, cell = W.diamond_cell(8, 8, 8, jitter=0.1, seed=seed)
        sp = np.zeros(len(x), np.int32)
        cfg = W.prepare(x, cell, sp, 5.0)
        t, sz, p = W.sf24_params()
        spec = dict(kind="sf", types=t, sizes=sz, params=p, cutoff=5.0, species=["Si"])
        desc = {"workload": "symmetry_functions_24_diamond_8x8x8", "atoms": 4096, "width": 24, "cutoff": 5.0}
    else:
        raise SystemExit(f"unknown workload {name}")
    desc["mean_neighbours"] = float(cfg.counts.mean())
    return cfg, spec, desc


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
    from libdescriptor_b200 import flops as F

    if spec["kind"] == "bs":
        n_in = float(cfg.counts.sum())
        per = F.bs_flops_per_atom(spec["twojmax"], spec["style"], 0.0, True, weights)
        nb = F.bs_flops_per_atom(spec["twojmax"], spec["style"], 1.0, True, weights) - per
        return per * cfg.n_atoms + nb * n_in
    # symmetry functions (8 g2 + 16 g4 rows (zeta, lambda, eta)): triplets
    # counted exactly from the neighbour lists
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

    def summary(self, t0=None, t1=None):
        """Median SM clock and active throttle reasons of the samples taken
        inside [t0, t1] (the timed region)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for (t, ln) in self.lines if (t0 is None or t >= t0) and (t1 is None or t <= t1)]
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
def cpu_desc_vjp_rate(spec, cfg, budget_s=12.0, threads=None):
    """Oracle desc+VJP atoms/s on a bounded sample of the same workload."""
    ora = make_oracle(spec)
    threads = threads or os.cpu_count() or 1
    rng = np.random.default_rng(7)

    def run(nrows):
        rows = np.arange(nrows, dtype=np.int32)
        dE = rng.normal(size=(nrows, ora.width))
        t0 = time.perf_counter()
        ora.run(np.array([nrows], np.int32), cfg.species, cfg.nbl, cfg.counts[:nrows], cfg.coords, dE=dE,
                n_configs=1, config_ptr=np.array([0], np.int32), n_threads=threads)
        del rows
        return time.perf_counter() - t0

    n0 = min(cfg.n_atoms, max(threads, 16))
    t0 = run(n0)
    n1 = int(min(cfg.n_atoms, max(n0, n0 * budget_s / max(t0, 1e-6))))
    t1 = run(n1)
    return n1 / t1, n1, threads


def reference_forward_rate(spec, cfg, budget_s=5.0, threads=None):
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

    def run(n):
        t0 = time.perf_counter()
        ref.compute(np.array([n], np.int32), cfg.species, cfg.nbl, cfg.counts[:n], cfg.coords, n_configs=1,
                    config_ptr=np.array([0], np.int32), n_threads=threads)
        return time.perf_counter() - t0

    n0 = min(cfg.n_atoms, max(threads, 16))
    t0 = run(n0)
    n1 = int(min(cfg.n_atoms, max(n0, n0 * budget_s / max(t0, 1e-6))))
    return n1 / run(n1)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, spec, cdesc = make_workload(args.workload, seed=1)
    threads = os.cpu_count() or 1
    rates = []
    sample = None
    for _ in range(args.warmup):
        cpu_desc_vjp_rate(spec, cfg, budget_s=2.0, threads=threads)
    for _ in range(args.steps):
        r, n, _ = cpu_desc_vjp_rate(spec, cfg, budget_s=6.0, threads=threads)
        rates.append(r)
        sample = n
    value = statistics.mean(rates)
    fwd = reference_forward_rate(spec, cfg, threads=threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sample / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cdesc,
        "cpu_baseline": {"value": value, "unit": "atoms/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} centres of the workload per step, desc+VJP by the oracle's "
                                   f"analytic adjoint (the reference's Enzyme gradient cannot be built "
                                   f"offline); reference C++ forward alone: "
                                   f"{fwd if fwd is None else round(fwd, 1)} atoms/s"},
        "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- GPU
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="bs8", choices=["bs8", "sf24"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    import libdescriptor_b200 as lds
    from libdescriptor_b200 import flops as F

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
        time.sleep(0.5)                          # let the sampler start before the timed region
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
    times = [a.elapsed_time(b) for a, b in evs]
    tot_ms = float(sum(times))
    if dist:
        t = torch.tensor([tot_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
    ms_per_step = tot_ms / args.steps
    value = world * n / (ms_per_step * 1e-3)

    # ---- end to end through the public API: host buffers in, host results out
    e2e = None
    if rank == 0 or world > 1:
        for _ in range(2):
            lds.compute_and_gradient(ds, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE_h)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ke = max(3, min(args.steps, 10))
        for _ in range(ke):
            lds.compute_and_gradient(ds, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE_h)
        e2e_s = (time.perf_counter() - t0) / ke
        h2d = cfg.species.nbytes + cfg.nbl.nbytes + cfg.counts.nbytes + cfg.coords.nbytes + dE_h.nbytes + 8 * (n + 1)
        d2h = 8 * n * W + 8 * 3 * cfg.n_total
        e2e = {"value": world * n / e2e_s, "unit": "atoms/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_s,
               "api": "libdescriptor_b200.compute_and_gradient (host numpy in/out, one fused pass)"}

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    flop = algorithmic_flops(spec, cfg, weights)
    achieved = flop / (ms_per_step * 1e-3) / 1e12
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": None, "kernel": "bs_kernel<VJP>" if spec["kind"] == "bs" else "sf_kernel<VJP>",
            "flops_per_step": flop, "peak_source": "bench.py FP64 FMA probe (ld_measure_fp64_peak), same run",
            "call_weights_flops": {k: round(v, 1) for k, v in weights.items()},
            "hbm_bytes_per_step_algorithmic": int(cfg.coords.nbytes + cfg.nbl.nbytes + 8 * n * W * 2
                                                  + 24 * cfg.n_total)}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        r, sample, thr = cpu_desc_vjp_rate(spec, cfg, budget_s=10.0)
        fwd = reference_forward_rate(spec, cfg, budget_s=4.0)
        cpu = {"value": r, "unit": "atoms/s", "cores": thr, "kind": "port",
               "sample": f"{sample} of {n} centres, desc+VJP by the oracle's analytic adjoint on all host "
                         f"threads; reference C++ forward alone: {None if fwd is None else round(fwd, 1)} atoms/s"}
    line = {
        "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no dataset)",
        "config": dict(cdesc, l2="flushed between steps (256 MB write outside the timed events)",
                       parallelism=f"replicas x{world}"),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
        "clocks": clk.summary(t_begin, t_end),
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
