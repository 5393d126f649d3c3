"""Benchmark of the TE hot path: all ordered-pair TE of 10k genes x 20k cells.

Workload (the config the headline metric is quoted on): 10,000 genes x 20,000
cells of uint8 bins, 95% of genes with b ~ U{2..16} and 5% heavy genes with
b ~ U{64..256}, values from a per-gene Dirichlet(1) over its bins (lag-1 AR on
5% of genes), seeded synthetic data; tau = 1, K = 1; 99,990,000 ordered pairs.
One step = dense remap of the resident bins, coarsening of the heavy genes to
the B200 shared-memory limit (38, the reference rule) and the full TE matrix
(float32, 400 MB) — the Adaptive-SMEM path. The 200 MB of bins exceed the
126 MB L2, so steps run back to back without an L2 flush.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Profiling options (not the headline run): --genes / --cells shrink the
workload, --pairs times only the first pair ids, --launch T,C,W fixes the
launch shape (threads, CTAs per SM, sources per work item) instead of running
the autotuner, --no-e2e, --no-cpu-baseline, --no-surrogate, --no-fdr,
--no-configs, --no-next and --no-reference-gpu skip those legs; --only NAME prints
one leg.
Side objects of the line:
  surrogate      NetWeaver's surrogate test on cfg5 (full 100-shuffle test and
                 the learned null, wall seconds, edge agreement)
  binary_path    the cfg2 GEMM-B2 matrix, 4-bit and int8 operand forms, each
                 against its live tensor-pipe probe and against the GEMM's own
                 MMA sequence issued back to back (tenex_probe_tc_gemm_b2)
  fdr            NetWeaver's default FDR method on the cfg4 matrix
  cfg3, cfg1     the other TE configs: device time and roofline, end to end,
                 and the CPU oracle on the same workload
  next_rows      the hot path's neighbouring rows: the source-filter pair list,
                 the multi-lag surrogate combine, binarisation and the
                 coarsening-off overflow launch (device time, roofline, end to end
                 and the CPU oracle where each applies)
  reference_gpu  the reference's own CUDA wrappers (installed under
                 baseline/_ref) on the same GPU, in a child process that imports
                 nothing of this repository (context, not the reference arm)
The CPU figures (cpu_baseline objects and --impl reference) all come from one
routine: the C oracle on seed-fixed uniform samples of 100,000 ordered pairs.

N > 1 (torchrun, one process per GPU): the pair-id range is split into
contiguous chunks of ceil(pairs / N), the reference's split (no data-path
collective); total work is fixed (strong scaling); time is the max over ranks.
--impl reference: rank 0 times the CPU oracle (a C restatement of the
reference's counting and TE formula, all host threads) on uniform samples of
100,000 pairs of the same coarsened bins, one sample per step.
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

N_GENES, N_CELLS, TAU = 10_000, 20_000, 1
METRIC = "TE pairs/s @10k genes x 20k cells (all ordered pairs, Adaptive-SMEM)"
WORKLOAD = "cfg4: 10000 genes x 20000 cells, 95% b~U{2..16}, 5% b~U{64..256} coarsened to 38"


def make_bins(genes: int = N_GENES, cells: int = N_CELLS):
    from tenex_b200 import workloads as W
    return W.cfg4_bins(genes, cells, seed=1004)


class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows: list[list[str]] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def profile_traffic():
    """DRAM bytes per launch of the TE kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "te_pair_tile_cfg4.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("dram_bytes_per_launch_full")
    return None


def sample_pairs(n: int, count: int, seed: int) -> np.ndarray:
    """A seed-fixed uniform sample (with replacement, then deduplicated and
    sorted) of `count` ordered pairs of n genes as [target, source] rows."""
    rng = np.random.default_rng(seed)
    ids = np.unique(rng.integers(0, n * (n - 1), count, dtype=np.int64))
    tgt = ids // (n - 1)
    sl = ids - tgt * (n - 1)
    return np.stack([tgt, sl + (sl >= tgt)], axis=1)


def cpu_oracle_rate(bins, npv, seconds: float, seed: int, sample: int = 100_000,
                    min_samples: int = 1) -> dict:
    """The CPU oracle (C, exact integer counts, float64 TE, every host thread) on
    seed-fixed uniform samples of `sample` ordered pairs, one sample after another
    until `seconds` have elapsed (at least `min_samples`). The bins are converted
    to the oracle's int32 rows once, outside the timed calls. Both the GPU arm's
    cpu_baseline and the --impl reference arm time the CPU path through here."""
    from oracle import oracle as O
    b = np.asarray(bins)
    n = b.shape[0]
    flat = np.ascontiguousarray(b.reshape(n, -1), dtype=np.int32)
    npv = np.asarray(npv, np.int32)
    nthreads = os.cpu_count() or 1
    done, busy, k = 0, 0.0, 0
    while k < min_samples or busy < seconds:
        pairs = sample_pairs(n, sample, seed + k)
        t0 = time.perf_counter()
        O.te_pairs(flat, npv, pairs, TAU, threads=nthreads)
        busy += time.perf_counter() - t0
        done += len(pairs)
        k += 1
    return {"value": done / busy, "unit": "pairs/s", "cores": nthreads, "kind": "port",
            "sample": f"{k} seed-fixed uniform samples of {sample} ordered pairs ({done} pairs, "
                      f"{busy:.1f} s on {nthreads} threads; C oracle: exact counts, float64 TE)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    x, npv = make_bins()
    cb, cnpv, bmax = O.coarsen(x, npv, 38)
    flat = np.ascontiguousarray(cb, dtype=np.int32)
    sample = args.ref_pairs
    for w in range(args.warmup):
        cpu_oracle_rate(flat, cnpv, 0.0, seed=900 + w, sample=min(sample, 20_000))
    rates = [cpu_oracle_rate(flat, cnpv, 0.0, seed=1000 + k, sample=sample)
             for k in range(args.steps)]
    busy = sum(sample / r["value"] for r in rates)
    v = args.steps * sample / busy
    line = {"metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": busy / args.steps * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "pairs_per_step": sample, "tau": TAU},
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": rates[0]["cores"],
                             "kind": "port",
                             "sample": f"per step a seed-fixed uniform sample of {sample} ordered "
                                       f"pairs of the coarsened bins, C oracle"},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from tenex_b200 import native
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.adaptive_smem import AdaptiveSMEMKernel, compute_smem_bin_limit
    from tenex_b200.preprocess import remap_bins

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    G, C = args.genes, args.cells
    x, npv = make_bins(G, C)
    total = G * (G - 1) if args.pairs is None else min(args.pairs, G * (G - 1))
    from tenex_b200.distributed import pair_range
    p0, p1 = pair_range(total, rank, world)
    kern = AdaptiveSMEMKernel()
    smem_optin = native.device_info(local).smem_optin
    limit = compute_smem_bin_limit(smem_optin, warps=32)

    raw_d = torch.from_numpy(x).to(dev)            # resident raw bins (uint8, 200 MB)
    out = torch.zeros((G, G), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    te_times = []

    def step(record_te: bool = False):
        db, npv_d, bmax = remap_bins(raw_d, 1, dev)                 # 1 launch
        db, npv_d, bmax = kern.prepare(db, npv_d, bmax, tau=TAU,    # 2 launches
                                       smem_optin=smem_optin)
        if record_te:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        kern.compute_pairfree_device(db, npv_d, bmax, TAU, p0, p1 - p0, matrix=True,
                                     out=out)                       # 3 launches
        if record_te:
            e1.record(stream)
            te_times.append((e0, e1))
        return db, npv_d, bmax

    # launch shape from the autotuner (timed once on a slice of the pair range, cached)
    from tenex_b200.kernels.pair_tile import autotune
    if args.launch:
        th, cps, w = (int(v) for v in args.launch.split(","))
        kern.cfg = dict(threads=th, ctas_per_sm=cps, src_chunk=w)
    else:
        db0, npv0, bmax0 = step()
        kern.cfg = dict(autotune(db0, npv0, bmax0, TAU))
        del db0, npv0
    bmax_run = None
    for _ in range(args.warmup):
        _, _, bmax_run = step()
    if bmax_run is None:
        _, _, bmax_run = step()
    torch.cuda.synchronize(dev)
    # the shape the library resolves for this launch (0 fields of the requested
    # config = its defaults)
    launch_resolved = native.te_launch_shape(C, TAU, int(bmax_run), kern.cfg)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step(record_te=True)
        t1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    te_ms = sum(a.elapsed_time(b) for a, b in te_times) / len(te_times)
    if world > 1:
        tt = torch.tensor([ms, te_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, te_ms = float(tt[0]), float(tt[1])
    pairs_per_step = total  # all ranks together
    value = pairs_per_step * args.steps / (ms / 1e3)

    # ---- end to end through the kernel plugin API (host bins -> host matrix) ----
    x_pin = torch.from_numpy(x).pin_memory()
    out_pin = torch.empty((G, G), dtype=torch.float32).pin_memory()
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 3))

    def e2e_step():
        xd = x_pin.to(dev, non_blocking=True)
        db, npv_d, bmax = remap_bins(xd, 1, dev)
        db, npv_d, bmax = kern.prepare(db, npv_d, bmax, tau=TAU, smem_optin=smem_optin)
        m = kern.compute_pairfree_device(db, npv_d, bmax, TAU, p0, p1 - p0, matrix=True)
        out_pin.copy_(m, non_blocking=True)

    e2e = None
    if e2e_steps:
        e2e_step()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        b.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = a.elapsed_time(b)
        if world > 1:
            tt = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_ms = float(tt[0])
        e2e = {"value": pairs_per_step * e2e_steps / (e2e_ms / 1e3), "unit": "pairs/s",
               "h2d_bytes_per_step": int(x.nbytes),
               "d2h_bytes_per_step": int(out_pin.numel() * 4),
               "path": "AdaptiveSMEMKernel: pinned host bins -> remap -> prepare -> "
                       "compute_pairfree_device -> pinned host matrix"}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel (te_pair_tile_kernel) ----
    N = C - TAU
    incr = (p1 - p0) * N                                   # histogram increments per launch
    peak_atomic = max(native.probe_smem_atomics(0, 8192) for _ in range(3))
    peak_scatter = max(native.probe_smem_atomics(2, 8192) for _ in range(3))
    achieved = incr / (te_ms / 1e3)
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")
    compulsory = G * x.shape[1] + (p1 - p0) * 4            # bins once + fp32 outputs
    roofline = {"bound": "smem_atomic", "achieved": achieved / 1e9, "peak": peak_atomic / 1e9,
                "unit": "Gincr/s", "frac": achieved / peak_atomic,
                "traffic": profile_traffic(),
                "note": "achieved = pairs x (T - tau) histogram increments per launch / mean "
                        "launch time (CUDA events); peak = conflict-free shared-memory atomicAdd "
                        "rate measured live by tenex_probe_smem_atomics (mode 0) on this GPU "
                        "(MEASURED_PEAKS.json has no shared-memory-atomic figure)",
                "scatter_peak": peak_scatter / 1e9,
                "frac_of_scatter": achieved / peak_scatter,
                "scatter_note": "second denominator, for context: the same probe with each lane "
                                "adding into a random word of a 16 KB histogram (mode 2), the "
                                "access pattern of a histogram of random cells",
                "te_kernel_ms": te_ms}
    roofline_hbm = {"bound": "hbm", "achieved": compulsory / (te_ms / 1e3) / 1e9,
                    "peak": hbm_peak, "unit": "GB/s",
                    "frac": (compulsory / (te_ms / 1e3) / 1e9 / hbm_peak) if hbm_peak else None,
                    "note": "compulsory bytes (bins read once + float32 outputs) / launch time; "
                            "peak = MEASURED_PEAKS.json hbm_gbs (of measured)"}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:                      # rank 0 at N=1 only
        cb, cnpv, _ = _coarsened_host(x, npv, limit)
        cpu = cpu_oracle_rate(cb, cnpv, 10.0, seed=1000)
    sur = (surrogate_leg(dev, with_cpu=not args.no_cpu_baseline)
           if (world == 1 and not args.no_surrogate) else None)
    binl = binary_leg(dev) if (world == 1 and not args.no_surrogate) else None
    c3 = (cfg3_leg(dev, peak_atomic, with_cpu=not args.no_cpu_baseline)
          if (world == 1 and not args.no_configs) else None)
    c1 = (cfg1_leg(dev, peak_atomic, with_cpu=not args.no_cpu_baseline)
          if (world == 1 and not args.no_configs) else None)
    nxt = (next_rows_leg(dev, peak_atomic, with_cpu=not args.no_cpu_baseline)
           if (world == 1 and not args.no_configs and not args.no_next) else None)
    refg = (reference_gpu_leg(dev) if (world == 1 and not args.no_reference_gpu
                                        and total == G * (G - 1)) else None)
    fdrl = fdr_leg(dev, out) if (world == 1 and not args.no_fdr and total == G * (G - 1)) else None
    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if (G, C, total) == (N_GENES, N_CELLS,
                                                                 N_GENES * (N_GENES - 1))
                       else f"cfg4-shaped slice: {G} genes x {C} cells, pair ids [0, {total})",
                       "genes": G, "cells": C, "tau": TAU,
                       "pairs": total, "step": "remap + coarsen + all-pairs TE matrix",
                       "parallelism": f"pair-range x{world}", "l2": "inputs (200 MB) > L2",
                       "launch": kern.cfg, "launch_resolved": launch_resolved},
            "gpu_launches": 6 * args.steps,  # remap, coarsen x2, prepass, order, TE tile
            "roofline": roofline, "roofline_hbm": roofline_hbm,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "surrogate": sur,
            "binary_path": binl, "fdr": fdrl, "cfg3": c3, "cfg1": c1, "next_rows": nxt,
            "reference_gpu": refg}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _te_device_ms(kern, db, npv_t, bmax, reps: int = 3) -> float:
    """Median device time (CUDA events on the launching stream) of one all-pairs
    TE matrix launch from resident bins, after two warm-up launches."""
    import torch
    out = torch.zeros((db.n, db.n), dtype=torch.float32, device=db.data.device)
    for _ in range(2):
        kern.compute_pairfree_device(db, npv_t, bmax, TAU, matrix=True, out=out)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    s = torch.cuda.current_stream()
    for a, b in ev:
        a.record(s)
        kern.compute_pairfree_device(db, npv_t, bmax, TAU, matrix=True, out=out)
        b.record(s)
    torch.cuda.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ev)


def _smem_roofline(pairs: int, N: int, ms: float, peak: float) -> dict:
    achieved = pairs * N / (ms / 1e3)
    return {"bound": "smem_atomic", "achieved": achieved / 1e9, "peak": peak / 1e9,
            "unit": "Gincr/s", "frac": achieved / peak,
            "note": "pairs x (T - tau) histogram increments / device time of the TE launch; "
                    "peak = conflict-free shared-memory atomic probe (tenex_probe_smem_atomics "
                    "mode 0) measured live"}


def cfg3_leg(dev, peak: float, with_cpu: bool = True) -> dict:
    """5,000 genes x 10,000 cells, b ~ U{2..32} (Full-SMEM, all 24,995,000 pairs
    in one persistent launch): device time from resident bins against the
    shared-memory atomic probe, end to end through FullSMEMKernel from pinned host
    bins to a pinned host matrix, and the CPU oracle on a uniform pair sample."""
    import torch

    from tenex_b200 import workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    x, npv = W.cfg3_bins()
    bins = np.ascontiguousarray(x, dtype=np.uint8)
    n, T = bins.shape
    bmax = int(npv.max())
    kern = FullSMEMKernel()
    db = D.pack_bins(bins, dev)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=dev)
    ms = _te_device_ms(kern, db, npv_t, bmax)
    pairs = n * (n - 1)
    # end to end: pinned host bins -> padded device rows -> TE matrix -> pinned host matrix
    x_pin = torch.from_numpy(bins).pin_memory()
    out_pin = torch.empty((n, n), dtype=torch.float32).pin_memory()
    npv_pin = torch.from_numpy(np.asarray(npv, np.int32)).pin_memory()
    s = torch.cuda.current_stream()

    def e2e_step():
        d = D.empty_bins(n, T, 1, dev)
        d.data[:, :T].copy_(x_pin, non_blocking=True)
        nd = npv_pin.to(dev, non_blocking=True)
        m = kern.compute_pairfree_device(d, nd, bmax, TAU, matrix=True)
        out_pin.copy_(m, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(2):
        e2e_step()
    b.record(s)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b) / 2
    return {"workload": "cfg3: 5000 genes x 10000 cells, b~U{2..32} Dirichlet(1), 5% AR lag-1 "
                        "(Full-SMEM, all 24,995,000 ordered pairs)",
            "pairs_per_s": pairs / (ms / 1e3), "ms": ms,
            "roofline": _smem_roofline(pairs, T - TAU, ms, peak),
            "e2e": {"value": pairs / (e2e_ms / 1e3), "unit": "pairs/s",
                    "h2d_bytes_per_step": int(bins.nbytes + npv_pin.numel() * 4),
                    "d2h_bytes_per_step": int(n * n * 4),
                    "path": "FullSMEMKernel: pinned host bins -> padded device rows -> "
                            "compute_pairfree_device -> pinned host matrix"},
            "cpu_baseline": cpu_oracle_rate(bins, npv, 5.0, seed=3000) if with_cpu else None}


def _median_event_ms(fn, reps: int = 3, warm: int = 2) -> float:
    """Median device time (CUDA events on the current stream) of fn() after `warm`
    untimed calls."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    for a, b in ev:
        a.record(s)
        fn()
        b.record(s)
    torch.cuda.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ev)


def _median_wall_s(fn, reps: int = 3) -> float:
    """Median wall seconds of fn() (which returns host data) after one warm-up call."""
    fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts)


def _oracle_pairs_rate(bins, npv, pairs: np.ndarray, seconds: float, seed: int,
                       sample: int = 100_000, tau: int = TAU) -> dict:
    """The C oracle (every host thread) on seed-fixed samples of `sample` rows of a
    given [target, source] pair list, one after another for `seconds`."""
    from oracle import oracle as O
    b = np.asarray(bins)
    flat = np.ascontiguousarray(b.reshape(b.shape[0], -1), dtype=np.int32)
    npv = np.asarray(npv, np.int32)
    nthreads = os.cpu_count() or 1
    k = min(sample, pairs.shape[0])
    done, busy, i = 0, 0.0, 0
    while i < 1 or busy < seconds:
        rng = np.random.default_rng(seed + i)
        smp = pairs[np.sort(rng.choice(pairs.shape[0], k, replace=False))]
        t0 = time.perf_counter()
        O.te_pairs(flat, npv, smp, tau, threads=nthreads)
        busy += time.perf_counter() - t0
        done += k
        i += 1
    return {"value": done / busy, "unit": "pairs/s", "cores": nthreads, "kind": "port",
            "sample": f"{i} seed-fixed samples of {k} pairs of the list ({busy:.1f} s on "
                      f"{nthreads} threads; C oracle, exact counts, float64 TE)"}


def source_filter_leg(dev, peak: float, with_cpu: bool = True) -> dict:
    """Source-filter (TF) pair list, the reference's compute_single_gpu with explicit
    pairs: the cfg3-shaped bins (5,000 genes x 10,000 cells, b ~ U{2..32}) with 500
    seed-chosen sources, every target against every source (2,499,500 [target,
    source] pairs): device time of the tenex_te_pairs launch from resident bins and
    a resident pair list against the shared-memory atomic probe; end to end through
    the plugin call (host bins and host pairs in, host TE vector out); the C oracle
    on samples of the same list."""
    import torch

    from tenex_b200 import native, workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    from tenex_b200.kernels.pair_list import item_table
    x, npv = W.cfg3_bins()
    bins = np.ascontiguousarray(x, dtype=np.uint8)
    n, T = bins.shape
    bmax = int(npv.max())
    rng = np.random.default_rng(3100)
    srcs = np.sort(rng.choice(n, 500, replace=False)).astype(np.int64)
    tgt = np.repeat(np.arange(n, dtype=np.int64), srcs.size)
    src = np.tile(srcs, n)
    keep = tgt != src
    pairs = np.ascontiguousarray(np.stack([tgt[keep], src[keep]], axis=1))   # by target
    P = pairs.shape[0]
    db = D.pack_bins(bins, dev)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=dev)
    items = item_table(pairs[:, 0], 128)
    pairs_d = torch.from_numpy(pairs).to(dev)
    items_d = torch.from_numpy(items).to(dev)
    ws = D.workspace(dev, n, db.row_len, bmax)
    out = torch.empty(P, dtype=torch.float32, device=dev)

    def launch():
        native.call("tenex_te_pairs", db.ptr(), db.ld, npv_t.data_ptr(), bmax, n, db.row_len,
                    TAU * db.K, pairs_d.data_ptr(), P, items_d.data_ptr(), items.shape[0] - 1,
                    out.data_ptr(), ws.data_ptr(), ws.numel(), None, native.stream_ptr())

    ms = _median_event_ms(launch)
    native.call("tenex_workspace_status", ws.data_ptr(), native.stream_ptr())
    kern = FullSMEMKernel()
    e2e_s = _median_wall_s(lambda: kern.compute_single_gpu(bins, pairs, bmax, npv, TAU, None,
                                                           dev))
    return {"workload": "source filter: cfg3-shaped bins (5000 genes x 10000 cells, "
                        "b~U{2..32}), 500 sources, all 5000 targets (2,499,500 pairs)",
            "pairs_per_s": P / (ms / 1e3), "ms": ms,
            "roofline": _smem_roofline(P, T - TAU, ms, peak),
            "e2e": {"value": P / e2e_s, "unit": "pairs/s", "seconds": e2e_s,
                    "h2d_bytes_per_step": int(bins.nbytes + pairs.nbytes),
                    "d2h_bytes_per_step": int(P * 4),
                    "path": "FullSMEMKernel.compute_single_gpu(host bins, host pairs) -> "
                            "host TE vector"},
            "cpu_baseline": (_oracle_pairs_rate(bins, npv, pairs, 5.0, seed=3200)
                             if with_cpu else None)}


def multi_lag_leg(dev, with_cpu: bool = True) -> dict:
    """Multi-lag surrogate combine (Pipeline.infer with taus): 2,000 genes x 5,000
    cells of expression (the cfg1 generator at cfg5's shape), FSBW-L bins, a TE
    matrix and the 100-shuffle surrogate test at tau = 1 and at tau = 2, merged per
    pair by lag_combine="max" with BH-FDR 0.05: wall seconds of the whole call from
    the host matrix (one timed call after a warm-up call); the CPU figure is the C
    oracle's estimate of the same two tests (the surrogate leg's routine on these
    bins, times the number of lags)."""
    import torch

    from tenex_b200 import Pipeline, TransferEntropyEngine, workloads as W
    x, _ = W.cfg1_expression(2000, 5000, seed=1006)
    n = x.shape[0]
    names = np.array([f"g{i}" for i in range(n)])
    taus, S = [1, 2], 100

    def call():
        return Pipeline(TransferEntropyEngine(x, names)).infer(
            "surrogate_test", taus=taus, lag_combine="max", n_surrogates=S, fdr=0.05,
            device=str(dev))

    call()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = call()
    wall = time.perf_counter() - t0
    cpu = None
    if with_cpu:
        te = TransferEntropyEngine(x, names).compute(accelerator="gpu", devices=[dev.index or 0])
        one = surrogate_cpu_baseline(te.bin_arrs[:, :, 0].astype(np.int32), te.n_per_var, S,
                                     int(res.block_length), 42, dev)
        cpu = dict(one, est_full_test_s=one["est_full_test_s"] * len(taus),
                   note="per-lag estimate of the tau = 1 test, times the number of lags")
    return {"workload": "multi-lag surrogate test: 2000 genes x 5000 cells expression "
                        "(FSBW-L), taus [1, 2], 100 block shuffles per lag, lag_combine='max', "
                        "BH-FDR 0.05",
            "metric": "Pipeline.infer('surrogate_test', taus=[1, 2]) wall seconds from the host "
                      "matrix (one call after a warm-up call)",
            "seconds": wall, "edges": int(len(res.grn)),
            "pair_surrogate_tes_per_s": n * (n - 1) * (S + 1) * len(taus) / wall,
            "cpu_baseline": cpu}


def binarize_leg(dev, with_cpu: bool = True) -> dict:
    """Binarisation, the GEMM-B2 path's input step: 10,000 genes x 20,000 cells of
    float32 expression (half zeros, 800 MB) binarised from a device-resident matrix
    by 'nonzero', 'mean' and 'median' (device time, median of 3 after 2 warm-ups)
    against the measured HBM copy rate, algorithmic bytes = the matrix read once
    plus the uint8 bins written once; end to end for 'median' from the host matrix
    to host bins; the C / numpy oracle (the reference's arithmetic) on 200 rows,
    extrapolated to the matrix."""
    import torch

    from oracle import oracle as O
    from tenex_b200.binarize import binarize
    from tenex_b200.kernels import device as D
    rng = np.random.default_rng(4000)
    n, T = 10_000, 20_000
    x = rng.standard_normal((n, T), dtype=np.float32)
    np.maximum(x, 0.0, out=x)
    xd = torch.from_numpy(x).to(dev)
    hbm = measured_peaks().get("hbm_gbs")
    algo = x.nbytes + n * T
    out = {"workload": "binarisation: 10000 genes x 20000 cells float32 (half zeros)"}
    for m in ("nonzero", "mean", "median"):
        ms = _median_event_ms(lambda m=m: binarize(xd, m, dev))
        gbs = algo / (ms / 1e3) / 1e9
        obj = {"ms": ms,
               "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                            "frac": gbs / hbm if hbm else None,
                            "note": "matrix read once + uint8 bins written once / device time; "
                                    "peak = MEASURED_PEAKS.json hbm_gbs (of measured)"}}
        if with_cpu:
            t0 = time.perf_counter()
            O.binarize(x[:200], m)
            dt = time.perf_counter() - t0
            obj["cpu_baseline"] = {"value": 200 * T / dt, "unit": "elements/s", "cores": 1,
                                   "kind": "port", "est_matrix_s": dt * n / 200,
                                   "sample": "200 rows, numpy (the reference's arithmetic)"}
        out[m] = obj
    del xd
    e2e_s = _median_wall_s(lambda: D.to_host(binarize(x, "median", dev)[0].unpadded()))
    out["e2e"] = {"method": "median", "seconds": e2e_s, "value": n * T / e2e_s,
                  "unit": "elements/s", "h2d_bytes_per_step": int(x.nbytes),
                  "d2h_bytes_per_step": int(n * T),
                  "path": "host float32 matrix -> binarize -> host uint8 bins"}
    return out


def overflow_leg(dev, peak: float, with_cpu: bool = True) -> dict:
    """Coarsening off (the reference's coarsening=False path): 400 genes x 20,000
    cells from the cfg4 generator (5% genes with b in [64, 256], not coarsened), all
    159,600 ordered pairs in one call. Pairs whose histogram does not fit shared
    memory (every pair with a heavy gene) run in the global-memory overflow launch,
    the rest in the shared-memory launch; device time of the call, its histogram
    increments against the shared-memory atomic probe (context: the overflow pairs
    count with global-memory atomics, three per sample), and the C oracle on
    samples of the same pairs."""
    import torch

    from tenex_b200 import workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.preprocess import remap_bins
    x, _ = W.cfg4_bins(400, 20_000, seed=1007)
    db, npv_d, bmax = remap_bins(torch.from_numpy(np.ascontiguousarray(x)).to(dev), 1, dev)
    npv = npv_d.cpu().numpy()
    bins_h = D.to_host(db.unpadded())            # the dense bins the kernel counts
    n, T = db.n, db.T
    P = n * (n - 1)
    heavy = int((npv > 38).sum())
    out = torch.empty(P, dtype=torch.float32, device=dev)
    ms = _median_event_ms(lambda: D.te_pairfree(db, npv_d, bmax, TAU, 0, P, out=out,
                                                check_data=False))
    rng = np.random.default_rng(4100)
    ids = np.sort(rng.choice(P, 20_000, replace=False))
    tg = ids // (n - 1)
    sl = ids - tg * (n - 1)
    pairs = np.stack([tg, sl + (sl >= tg)], axis=1)
    roof = _smem_roofline(P, T - TAU, ms, peak)
    roof["note"] = ("pairs x (T - tau) histogram increments / device time of the call, against "
                    "the shared-memory atomic probe for context: the overflow pairs count with "
                    "global-memory atomics (three per sample), which the probe does not bound")
    return {"workload": f"coarsening off: 400 genes x 20000 cells (cfg4 generator, {heavy} genes "
                        f"with b up to {bmax}), all {P} ordered pairs",
            "pairs_per_s": P / (ms / 1e3), "ms": ms, "roofline": roof,
            "cpu_baseline": (_oracle_pairs_rate(bins_h, npv, pairs, 5.0, seed=4200,
                                                sample=2000) if with_cpu else None)}


def next_rows_leg(dev, peak: float, with_cpu: bool = True) -> dict:
    """The hot path's neighbouring rows, each measured: source-filter pair list,
    multi-lag surrogate combine, binarisation and the coarsening-off overflow
    launch."""
    return {"source_filter": source_filter_leg(dev, peak, with_cpu),
            "multi_lag": multi_lag_leg(dev, with_cpu),
            "binarize": binarize_leg(dev, with_cpu),
            "overflow": overflow_leg(dev, peak, with_cpu)}


def cfg1_leg(dev, peak: float, with_cpu: bool = True, reps: int = 5) -> dict:
    """100 genes x 1,000 cells of expression (float32 log1p of zero-inflated NB
    counts) through TransferEntropyEngine.compute(accelerator="gpu"): wall seconds
    of the whole call (host matrix in, host TE matrix out: FSBW-L, remap, kernel
    choice, all 9,900 pairs) with a new engine per call, the TE launch's device
    time, and the CPU oracle on the same path (FSBW-L, remap, all pairs)."""
    import torch

    from tenex_b200 import TransferEntropyEngine, workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    from oracle import oracle as O
    x, _ = W.cfg1_expression()
    n, T = x.shape
    names = np.array([f"g{i}" for i in range(n)])
    ts, res = [], None
    for _ in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = TransferEntropyEngine(x, names).compute(accelerator="gpu", devices=[dev.index or 0])
        ts.append(time.perf_counter() - t0)
    wall = statistics.median(ts[1:])
    bins = res.bin_arrs[:, :, 0].astype(np.uint8)
    npv = res.n_per_var
    db = D.pack_bins(bins, dev)
    ms = _te_device_ms(FullSMEMKernel(), db, torch.as_tensor(npv, device=dev), int(npv.max()))
    pairs = n * (n - 1)
    cpu = None
    if with_cpu:
        nthreads = os.cpu_count() or 1
        t0 = time.perf_counter()
        k = 0
        while k < 3 or time.perf_counter() - t0 < 2.0:
            rb, _ = O.fsbwl(x, 0.5)
            cb, cnpv, _ = O.remap(rb)
            O.te_pairfree(cb, cnpv, TAU, threads=nthreads)
            k += 1
        dt = (time.perf_counter() - t0) / k
        cpu = {"value": pairs / dt, "unit": "pairs/s", "cores": nthreads, "kind": "port",
               "sample": f"the whole 9,900-pair matrix from the float32 data (FSBW-L, remap, "
                         f"TE), {k} runs, {dt * 1e3:.1f} ms each; C oracle"}
    return {"workload": "cfg1: 100 genes x 1000 cells expression, FSBW-L, Full-SMEM "
                        "(9,900 ordered pairs)",
            "metric": "TransferEntropyEngine.compute(accelerator='gpu') wall seconds from the "
                      "host matrix (median of %d after a warm-up call)" % reps,
            "seconds": wall, "pairs_per_s": pairs / wall, "te_kernel_ms": ms,
            "roofline": _smem_roofline(pairs, T - TAU, ms, peak),
            "e2e": {"value": pairs / wall, "unit": "pairs/s", "h2d_bytes_per_step": int(x.nbytes),
                    "d2h_bytes_per_step": int(n * n * 4),
                    "path": "TransferEntropyEngine(x, names).compute(accelerator='gpu')"},
            "kernel": res.kernel, "cpu_baseline": cpu}


def surrogate_leg(dev, reps: int = 3, with_cpu: bool = True) -> dict:
    """Wall seconds of NetWeaver's surrogate test on cfg5 (2,000 genes x 5,000 cells,
    100 block shuffles of length 50, seed 42, BH-FDR 0.05, parametric p): the full
    test against the learned null, each after one warm-up call, with the edge-set
    agreement of the two."""
    import torch

    from tenex_b200 import workloads as W
    from tenex_b200.inference.surrogate_test import SurrogateTestMethod
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    x, npv, _ = W.cfg5_bins(seed=1005)
    n = x.shape[0]
    names = np.array([f"g{i}" for i in range(n)])
    db = D.pack_bins(x, dev)
    obs = FullSMEMKernel().compute_pairfree_device(
        db, torch.as_tensor(npv, device=dev), int(npv.max()), 1, matrix=True).cpu().numpy()
    kw = dict(bin_data=x, n_per_var=npv, b_max=int(npv.max()), kernel="Full-SMEM", tau=1,
              n_surrogates=100, block_length=50, fdr=0.05, seed=42)
    m = SurrogateTestMethod()

    def timed(reps=reps, **extra):
        ts, res = [], None
        for _ in range(reps + 1):                      # first call is the warm-up
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            res = m.infer(obs, names, dev, **kw, **extra)
            torch.cuda.synchronize(dev)
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts[1:]), res

    t_full, full = timed()
    t_lrn, lrn = timed(reps=5, null="learned")
    cpu = surrogate_cpu_baseline(x, npv, 100, 50, 42, dev) if with_cpu else None
    e1 = set(map(tuple, full.grn.pairs.tolist()))
    e2 = set(map(tuple, lrn.grn.pairs.tolist()))
    inter = len(e1 & e2)
    return {"workload": "cfg5: 2000 genes x 5000 cells, b~U{2..16} Markov, 100 block shuffles "
                        "(block length 50, seed 42), BH-FDR 0.05, parametric p",
            "metric": "surrogate_test wall seconds (median of %d full / 5 learned runs after a "
                      "warm-up call)" % reps,
            "full_s": t_full, "learned_s": t_lrn, "speedup": t_full / t_lrn,
            "n_edges_full": len(e1), "n_edges_learned": len(e2),
            "jaccard": inter / max(1, len(e1 | e2)), "precision": inter / max(1, len(e2)),
            "recall": inter / max(1, len(e1)),
            "verified_fraction": lrn.info.get("fallback_fraction"),
            "band": lrn.info.get("band"), "cpu_baseline": cpu}


def surrogate_cpu_baseline(x, npv, S: int, bl: int, seed: int, dev, n_pairs: int = 100_000,
                           n_shuffles: int = 5) -> dict:
    """The CPU oracle on the surrogate workload: the first `n_shuffles` of the
    test's own block shuffles (same permutations), `n_pairs` pair ids each, on all
    host threads; the full test's CPU time extrapolated linearly in pairs x shuffles."""
    from oracle import oracle as O
    from tenex_b200.inference.surrogate_test import build_block_perm
    n, T = x.shape[0], x.shape[1]
    perms, blk, _ = build_block_perm(n, T, "block", bl, 0, n_shuffles, seed, dev)
    perms = perms.cpu().numpy()
    nthreads = os.cpu_count() or 1
    total = n * (n - 1)
    p0 = (total - n_pairs) // 2
    dt = 0.0
    for k in range(n_shuffles):
        sh = O.block_shuffle(x, perms[k], blk)
        t0 = time.time()
        O.te_pairfree(sh, npv, 1, p0, n_pairs, threads=nthreads)
        dt += time.time() - t0
    rate = n_pairs * n_shuffles / dt
    return {"value": rate, "unit": "pair-surrogate TEs/s", "cores": nthreads, "kind": "port",
            "est_full_test_s": total * S / rate,
            "sample": f"{n_shuffles} of the test's block shuffles x pair ids [{p0}, {p0 + n_pairs}) "
                      f"({dt:.1f} s on {nthreads} threads; C oracle, float64 TE)"}


def binary_leg(dev, reps: int = 5) -> dict:
    """cfg2 binary path (2,000 genes x 5,000 cells, GEMM-B2 on tcgen05): device time of
    one full TE matrix (pack kernel + GEMM with the TE epilogue) for the default
    4-bit operand form (kind::mxf4) against the live 4-bit tensor-pipe probe, and
    the int8 form (kind::i8) against the live INT8 probe."""
    import torch

    from tenex_b200 import native, workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.gemm_b2 import te_binary_matrix, tile_width
    x, _ = W.cfg2_binary()
    n, T = x.shape
    db = D.pack_bins(x, dev)
    out = torch.zeros((n, n), dtype=torch.float32, device=dev)
    L = T - 1
    tiles = -(-n // 128)
    tn = tile_width(n)
    forms = {}
    for form, kpad, probe in (("fp4", 256, native.probe_tc_fp4), ("int8", 128, native.probe_tc_int8)):
        for _ in range(3):
            te_binary_matrix(db, 1, out=out, operands=form)
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(reps)]
        for a, b in ev:
            a.record()
            te_binary_matrix(db, 1, out=out, check=False, operands=form)
            b.record()
        torch.cuda.synchronize(dev)
        ms = statistics.median(a.elapsed_time(b) for a, b in ev)
        Lpad = -(-L // kpad) * kpad
        ops = 6.0 * (tiles * 128) ** 2 * Lpad      # 3 GEMMs of (n x Lpad) x (Lpad x n)
        peak = max(probe(100_000) for _ in range(2))
        # the GEMM's own MMA sequence issued back to back (no copies, no waits): the
        # instruction-mix bound of its main loop; the work the MMAs execute is
        # 6 x (sources padded to 128) x (targets padded to the tile width) x L_pad
        seq = max(native.probe_tc_gemm_b2(form, tn, 2000) for _ in range(2))
        ops_exec = 6.0 * (tiles * 128) * (-(-n // tn) * tn) * Lpad
        forms[form] = {"ms": ms, "pairs_per_s": n * (n - 1) / (ms / 1e3),
                       "roofline": {"bound": "tensor", "achieved": ops / (ms / 1e3) / 1e12,
                                    "peak": peak / 1e12,
                                    "unit": "TOP/s (%s)" % ("e2m1" if form == "fp4" else "int8"),
                                    "frac": ops / (ms / 1e3) / peak,
                                    "note": "achieved = 6*n_pad^2*L_pad ops (C, D, E) / device "
                                            "time of pack + GEMM; peak = the live %s probe"
                                            % ("tenex_probe_tc_fp4" if form == "fp4"
                                               else "tenex_probe_tc_int8"),
                                    "sequence_peak": seq / 1e12,
                                    "frac_of_sequence": ops_exec / (ms / 1e3) / seq,
                                    "sequence_note": "the GEMM's own MMA sequence (tile width "
                                                     "%d) back to back on every SM "
                                                     "(tenex_probe_tc_gemm_b2), against the "
                                                     "MMA work executed per call" % tn}}
    # end to end: pinned host bins -> padded device rows -> matrix -> pinned host matrix
    # (the reference's compute_te_gemm_b2 is timed the same way, host to host)
    x_pin = torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint8)).pin_memory()
    out_pin = torch.empty((n, n), dtype=torch.float32).pin_memory()

    def e2e_step():
        d8 = D.empty_bins(n, T, 1, dev)
        d8.data[:, :T].copy_(x_pin, non_blocking=True)
        m = te_binary_matrix(d8, 1, check=False)
        out_pin.copy_(m, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        e2e_step()
    b.record()
    torch.cuda.synchronize(dev)
    e2e_ms = a.elapsed_time(b) / reps
    d = forms["fp4"]
    return {"workload": "cfg2: 2000 genes x 5000 cells, binary Markov bins, GEMM-B2",
            "pairs_per_s": d["pairs_per_s"], "ms": d["ms"], "operands": "fp4 (kind::mxf4)",
            "tile_n": tn,
            "roofline": d["roofline"], "int8_form": forms["int8"],
            "e2e": {"value": n * (n - 1) / (e2e_ms / 1e3), "unit": "pairs/s", "ms": e2e_ms,
                    "h2d_bytes_per_step": int(x.size), "d2h_bytes_per_step": int(n * n * 4),
                    "path": "pinned host bins -> padded device rows -> te_binary_matrix -> "
                            "pinned host matrix"}}


def fdr_leg(dev, mat, reps: int = 2) -> dict:
    """NetWeaver's default method on the TE matrix just computed: z-score, BH-FDR
    0.01 and DPI trimming (FDRMethod.infer from a host matrix, wall seconds, median
    of `reps` after a warm-up call), and the DPI kernel's device time on the
    thresholded network against the live FP32 min/max probe."""
    import torch

    from tenex_b200 import native
    from tenex_b200.inference.fdr import FDRMethod, dpi_trim_matrix
    n = mat.shape[0]
    names = np.array([f"g{i}" for i in range(n)])
    host = mat.cpu().numpy()
    m = FDRMethod()
    ts = []
    for _ in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        grn, trimmed = m.infer(host, names, dev, fdr=0.01)
        torch.cuda.synchronize(dev)
        ts.append(time.perf_counter() - t0)
    arr = torch.zeros((n, n), dtype=torch.float32, device=dev)
    if len(grn):
        p = torch.as_tensor(grn.pairs, dtype=torch.long, device=dev)
        arr[p[:, 0], p[:, 1]] = torch.as_tensor(grn.te, device=dev)
    med = arr.sum(dim=1) > 0
    res = torch.empty_like(arr)
    dpi_trim_matrix(arr, med, None, 0.0, out=res)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    for a, b in ev:
        a.record()
        dpi_trim_matrix(arr, med, None, 0.0, out=res)
        b.record()
    torch.cuda.synchronize(dev)
    ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    instr = 1.5 * float(n) ** 3          # one min per k, one three-input max per two k
    peak = max(native.probe_minmax() for _ in range(2))
    # sparse form on the same network: CSR build + kernel, device time
    from tenex_b200.inference.fdr import _sparse_pays, dpi_trim_sparse
    pos = arr > 0
    work = float((pos.sum(0).double() * pos.sum(1).double() * med.double()).sum().item())
    dpi_trim_sparse(arr, med, None, 0.0)
    torch.cuda.synchronize(dev)
    for a, b in ev:
        a.record()
        dpi_trim_sparse(arr, med, None, 0.0)
        b.record()
    torch.cuda.synchronize(dev)
    ms_sp = statistics.median(a.elapsed_time(b) for a, b in ev)
    return {"workload": f"TE matrix of {n} genes, fdr=0.01, DPI trimming (threshold 0)",
            "metric": "FDRMethod.infer wall seconds from a host matrix (median of %d after a "
                      "warm-up call)" % reps,
            "seconds": statistics.median(ts[1:]), "edges": len(grn), "edges_trimmed": len(trimmed),
            "density": len(grn) / float(n * (n - 1)), "dpi_ms": ms,
            "dpi_sparse": {"ms": ms_sp, "updates": work,
                           "updates_per_s": work / (ms_sp / 1e3) if ms_sp > 0 else None,
                           "note": "CSR build (torch nonzero/bincount) + tenex_dpi_trim_sparse; "
                                   "updates = sum over mediators of positive in x out degree"},
            "dpi_auto": "sparse" if _sparse_pays(arr, med) else "dense",
            "roofline": {"bound": "fp32 min/max issue", "achieved": instr / (ms / 1e3) / 1e12,
                         "peak": peak / 1e12, "unit": "T instr/s", "frac": instr / (ms / 1e3) / peak,
                         "note": "achieved = 1.5 n^3 min/max instructions / DPI kernel device "
                                 "time; peak = tenex_probe_minmax measured live"}}


REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def _reference_gpu_worker(path: str) -> None:
    """Runs in a separate process with only the installed reference importable
    (nothing of this repository is imported): times the reference's own GPU
    wrappers on the workloads saved in `path` and prints one JSON object.
    Device time = CUDA events around the wrapper call (the wrappers also copy
    their float32 result to the host, which is included)."""
    import torch
    sys.path.insert(0, REF_DIR)
    import tenex
    from tenex.kernels.adaptive_smem import compute_te_adaptive_smem_pairfree
    from tenex.kernels.full_smem import compute_te_smem_pairfree
    from tenex.kernels.gemm_b2 import compute_te_gemm_b2
    dev = torch.device("cuda", 0)
    d = np.load(path)

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return min(ts)

    out = {"reference": os.path.dirname(tenex.__file__)}
    # cfg4 slice: Adaptive-SMEM pair-free on the coarsened bins (int8)
    b4 = torch.from_numpy(d["cfg4_bins"].astype(np.int8)[:, :, None]).to(dev)
    n4 = torch.from_numpy(d["cfg4_npv"].astype(np.int32)).to(dev)
    n = b4.shape[0]
    p0, cnt = int(d["cfg4_p0"]), int(d["cfg4_pairs"])
    ms = timed(lambda: compute_te_adaptive_smem_pairfree(b4, n4, n, 1, p0, cnt))
    out["cfg4"] = {"entry": "tenex.kernels.adaptive_smem.compute_te_adaptive_smem_pairfree",
                   "pairs": cnt, "ms": ms, "pairs_per_s": cnt / (ms / 1e3),
                   "sample": f"pair ids [{p0}, {p0 + cnt}) of the coarsened 10,000 x 20,000 bins"}
    del b4, n4
    # cfg3: Full-SMEM pair-free, all pairs (int32 bins as its wrapper expects)
    b3 = torch.from_numpy(d["cfg3_bins"].astype(np.int32)[:, :, None]).to(dev)
    n3 = b3.shape[0]
    bm3 = int(d["cfg3_npv"].max())
    ms = timed(lambda: compute_te_smem_pairfree(b3, bm3, n3, 1), reps=1)
    out["cfg3"] = {"entry": "tenex.kernels.full_smem.compute_te_smem_pairfree",
                   "pairs": n3 * (n3 - 1), "ms": ms, "pairs_per_s": n3 * (n3 - 1) / (ms / 1e3)}
    del b3
    # cfg2: GEMM-B2 (torch.mm + Triton epilogue)
    x2 = d["cfg2_bins"].astype(np.int32)
    n2 = x2.shape[0]
    ms = timed(lambda: compute_te_gemm_b2(x2, tau=1, device=dev), reps=3)
    out["cfg2"] = {"entry": "tenex.kernels.gemm_b2.compute_te_gemm_b2 (torch.mm + Triton)",
                   "pairs": n2 * (n2 - 1), "ms": ms, "pairs_per_s": n2 * (n2 - 1) / (ms / 1e3),
                   "note": "from host bins to a host matrix, as the wrapper is called"}
    # cfg5: SurrogateTestMethod.infer, 100 block shuffles on the GPU
    from tenex.inference.surrogate_test import SurrogateTestMethod
    x5 = d["cfg5_bins"].astype(np.int32)
    npv5 = d["cfg5_npv"].astype(np.int32)
    obs = d["cfg5_obs"]
    names = np.array([f"g{i}" for i in range(x5.shape[0])])
    kw = dict(bin_data=x5[:, :, None], n_per_var=npv5, b_max=int(npv5.max()), kernel="Full-SMEM",
              tau=1, n_surrogates=100, block_length=50, fdr=0.05, seed=42)
    m = SurrogateTestMethod()
    m.infer(obs, names, dev, **dict(kw, n_surrogates=2))       # warm-up (compile, load)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = m.infer(obs, names, dev, **kw)
    torch.cuda.synchronize()
    out["cfg5"] = {"entry": "tenex.inference.surrogate_test.SurrogateTestMethod.infer "
                            "(kernel='Full-SMEM', 100 block shuffles)",
                   "seconds": time.perf_counter() - t0, "n_edges": int(len(r.grn))}
    print(json.dumps(out), flush=True)


def reference_gpu_leg(dev, timeout_s: int = 900) -> dict | None:
    """The reference's own CUDA kernels timed on this GPU (context, not the
    driver's reference arm): cfg4 on a 4M-pair slice, cfg3 and cfg2 whole, the
    cfg5 surrogate test whole, each through the reference's Python wrapper, in a
    child process that imports only the reference installed under baseline/_ref."""
    import subprocess
    import tempfile

    import torch

    from tenex_b200 import workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    from oracle import oracle as O
    if not os.path.isdir(os.path.join(REF_DIR, "tenex")):
        return {"unavailable": "the reference is not installed under baseline/_ref"}
    x4, npv4 = make_bins()
    cb, cnpv, _ = O.coarsen(x4, npv4, 38)
    n4 = cb.shape[0]
    x3, npv3 = W.cfg3_bins()
    x2, _ = W.cfg2_binary()
    x5, npv5, _ = W.cfg5_bins(seed=1005)
    obs = FullSMEMKernel().compute_pairfree_device(
        D.pack_bins(x5, dev), torch.as_tensor(npv5, device=dev), int(npv5.max()), 1,
        matrix=True).cpu().numpy()
    mid = (n4 * (n4 - 1) // 2) // (n4 - 1) * (n4 - 1)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "ref_gpu_inputs.npz")
        np.savez(path, cfg4_bins=cb.astype(np.uint8), cfg4_npv=cnpv, cfg4_p0=mid,
                 cfg4_pairs=4_000_000, cfg3_bins=x3, cfg3_npv=npv3, cfg2_bins=x2,
                 cfg5_bins=x5, cfg5_npv=npv5, cfg5_obs=obs)
        env = dict(os.environ, PYTHONPATH=REF_DIR)
        try:
            r = subprocess.run([sys.executable, os.path.abspath(__file__),
                                "--reference-gpu-worker", path], capture_output=True, text=True,
                               timeout=timeout_s, env=env, cwd=tmp)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"the reference's GPU run exceeded {timeout_s} s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"unavailable": f"reference GPU worker exit {r.returncode}: "
                               f"{(r.stderr or r.stdout)[-400:]}"}
    return json.loads(lines[-1])


def _coarsened_host(x, npv, limit):
    from oracle import oracle as O
    cb, cnpv, bmax = O.coarsen(x, npv, limit)
    return cb, cnpv, bmax


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-pairs", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-fdr", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the cfg1 / cfg3 objects of the line")
    ap.add_argument("--no-next", action="store_true",
                    help="skip the next_rows object (source filter, multi-lag, binarisation, "
                         "overflow)")
    ap.add_argument("--only", choices=["binary", "surrogate", "fdr", "cfg1", "cfg3", "next",
                                       "reference_gpu"],
                    default=None,
                    help="run one side leg alone and print its JSON object (profiling)")
    ap.add_argument("--genes", type=int, default=N_GENES)
    ap.add_argument("--cells", type=int, default=N_CELLS)
    ap.add_argument("--pairs", type=int, default=None)
    ap.add_argument("--launch", default=None)
    ap.add_argument("--reference-gpu-worker", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference_gpu object (the reference's CUDA kernels)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.reference_gpu_worker:
        _reference_gpu_worker(args.reference_gpu_worker)
    elif args.impl == "reference":
        run_reference(args)
    elif args.only == "binary":
        import torch
        print(json.dumps(binary_leg(torch.device("cuda", 0))), flush=True)
    elif args.only == "reference_gpu":
        import torch
        print(json.dumps(reference_gpu_leg(torch.device("cuda", 0))), flush=True)
    elif args.only in ("cfg1", "cfg3", "next"):
        import torch

        from tenex_b200 import native
        dev = torch.device("cuda", 0)
        peak = max(native.probe_smem_atomics(0, 8192) for _ in range(3))
        leg = {"cfg1": cfg1_leg, "cfg3": cfg3_leg, "next": next_rows_leg}[args.only]
        print(json.dumps(leg(dev, peak, with_cpu=not args.no_cpu_baseline)), flush=True)
    elif args.only == "surrogate":
        import torch
        print(json.dumps(surrogate_leg(torch.device("cuda", 0))), flush=True)
    elif args.only == "fdr":
        import torch

        from tenex_b200 import workloads as W
        from tenex_b200.kernels import device as D
        from tenex_b200.kernels.full_smem import FullSMEMKernel
        dev = torch.device("cuda", 0)
        x, npv, _ = W.cfg5_bins(seed=1005)
        mat = FullSMEMKernel().compute_pairfree_device(
            D.pack_bins(x, dev), torch.as_tensor(npv, device=dev), int(npv.max()), 1, matrix=True)
        print(json.dumps(fdr_leg(dev, mat)), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
