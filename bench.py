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
the autotuner, --no-e2e, --no-cpu-baseline and --no-surrogate skip those legs.
The line's "surrogate" object times NetWeaver's surrogate test on cfg5 (full
100-shuffle test against the learned null, wall seconds, edge agreement), and
"binary_path" the cfg2 GEMM-B2 matrix against the measured INT8 tensor peak
(both skipped by --no-surrogate).

N > 1 (torchrun, one process per GPU): the pair-id range is split into
contiguous chunks of ceil(pairs / N), the reference's split (no data-path
collective); total work is fixed (strong scaling); time is the max over ranks.
--impl reference: rank 0 times the CPU oracle (a C restatement of the
reference's counting and TE formula, all host threads) on a bounded sample of
the same pairs.
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


def cpu_baseline(bins, npv, b_max_c, seconds: float = 12.0, chunk: int = 20_000) -> dict:
    """The CPU oracle on consecutive pair-id chunks until `seconds` elapsed."""
    from oracle import oracle as O
    nthreads = os.cpu_count() or 1
    done, t0 = 0, time.time()
    n = bins.shape[0]
    total = n * (n - 1)
    while time.time() - t0 < seconds and done < total:
        c = min(chunk, total - done)
        O.te_pairfree(bins, npv, TAU, done, c, threads=nthreads)
        done += c
    dt = time.time() - t0
    return {"value": done / dt, "unit": "pairs/s", "cores": nthreads, "kind": "port",
            "sample": f"pair ids [0, {done}) of the same coarsened cfg4 bins "
                      f"({dt:.1f} s on {nthreads} threads; C oracle, exact counts, float64 TE)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    x, npv = make_bins()
    cb, cnpv, bmax = O.coarsen(x, npv, 38)
    nthreads = os.cpu_count() or 1
    sample = args.ref_pairs
    for w in range(args.warmup):
        O.te_pairfree(cb, cnpv, TAU, 0, min(sample, 20_000), threads=nthreads)
    t0 = time.time()
    for k in range(args.steps):
        O.te_pairfree(cb, cnpv, TAU, (k * sample) % (N_GENES * (N_GENES - 1) - sample), sample,
                      threads=nthreads)
    dt = time.time() - t0
    v = args.steps * sample / dt
    line = {"metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "pairs_per_step": sample, "tau": TAU},
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": nthreads, "kind": "port",
                             "sample": f"{sample} consecutive pair ids per step, C oracle"},
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
        kern.cfg = autotune(db0, npv0, bmax0, TAU)
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
    cpu = (cpu_baseline(*_coarsened_host(x, npv, limit))
           if (world == 1 and not args.no_cpu_baseline) else None)   # rank 0 at N=1 only
    sur = (surrogate_leg(dev, with_cpu=not args.no_cpu_baseline)
           if (world == 1 and not args.no_surrogate) else None)
    binl = binary_leg(dev) if (world == 1 and not args.no_surrogate) else None
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
            "binary_path": binl, "fdr": fdrl}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


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
    one full TE matrix (pack kernel + INT8 GEMM with the TE epilogue), against the
    live INT8 tensor-pipe probe."""
    import torch

    from tenex_b200 import native, workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.gemm_b2 import te_binary_matrix
    x, _ = W.cfg2_binary()
    n, T = x.shape
    db = D.pack_bins(x, dev)
    out = torch.zeros((n, n), dtype=torch.float32, device=dev)
    for _ in range(3):
        te_binary_matrix(db, 1, out=out)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    for a, b in ev:
        a.record()
        te_binary_matrix(db, 1, out=out, check=False)
        b.record()
    torch.cuda.synchronize(dev)
    ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    L = T - 1
    Lpad = -(-L // 128) * 128
    tiles = -(-n // 128)
    ops = 6.0 * (tiles * 128) ** 2 * Lpad          # 3 int8 GEMMs of (n x Lpad) x (Lpad x n)
    peak = max(native.probe_tc_int8(100_000) for _ in range(2))
    return {"workload": "cfg2: 2000 genes x 5000 cells, binary Markov bins, GEMM-B2",
            "pairs_per_s": n * (n - 1) / (ms / 1e3), "ms": ms,
            "roofline": {"bound": "tensor", "achieved": ops / (ms / 1e3) / 1e12,
                         "peak": peak / 1e12, "unit": "TOP/s (int8)",
                         "frac": ops / (ms / 1e3) / peak,
                         "note": "achieved = 6*n_pad^2*L_pad int8 ops (C, D, E) / device time of "
                                 "pack + GEMM; peak = tenex_probe_tc_int8 measured live"}}


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
    ap.add_argument("--only", choices=["binary", "surrogate", "fdr"], default=None,
                    help="run one side leg alone and print its JSON object (profiling)")
    ap.add_argument("--genes", type=int, default=N_GENES)
    ap.add_argument("--cells", type=int, default=N_CELLS)
    ap.add_argument("--pairs", type=int, default=None)
    ap.add_argument("--launch", default=None)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.only == "binary":
        import torch
        print(json.dumps(binary_leg(torch.device("cuda", 0))), flush=True)
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
