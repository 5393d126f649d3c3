"""Surrogate (time-shuffle) significance test of the TE matrix.

Mirrors tenex/inference/surrogate_test.py (SurrogateTestResult :74-104,
_build_block_perm :165-207, SurrogateTestMethod.infer :599-948): same
arguments, validation, RNG schedule (surrogate k draws its permutations from a
torch generator seeded with seed + k, on the same device), statistics
(float64 sums of float32 TE, population std, parametric z-test or Monte Carlo
p-values, BH-FDR over the off-diagonal or source-filtered pairs, edges where
the adjusted p < fdr and the effective TE > 0).

On the device: every surrogate is one block-shuffle kernel plus one TE launch
whose epilogue adds the surrogate's TE into the float64 sum / sum-of-squares and
the int32 count of TE_k >= observed (the stats mode of te_pair_tile_kernel;
tcgen05 GEMM-B2 plus an elementwise update for binary data). The S-surrogate
loop is launched eagerly (each launch runs for milliseconds, so launch overhead
is hidden); use_graph=True captures it into one CUDA graph after one eager
iteration instead.

null="learned" replaces most of the surrogates by a learned null model
(tenex_b200.inference.learned_null): see that module.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from tenex_b200 import _log, native
from tenex_b200.inference.grn import GRN, bh_fdr_gpu, build_pairs, make_grn
from tenex_b200.kernels import device as D


@dataclass
class SurrogateTestResult:
    observed_te: np.ndarray
    mean_surrogate_te: np.ndarray
    std_surrogate_te: np.ndarray
    effective_te: np.ndarray
    p_values: np.ndarray
    grn: GRN
    n_surrogates: int
    shuffle_method: str
    block_length: int | None
    p_method: str
    fdr: float
    null_model: str = "full"
    info: dict = field(default_factory=dict)


def build_block_perm(n_vars: int, T: int, shuffle_method: str, block_length: int, k_start: int,
                     k_end: int, seed: int, device) -> tuple[torch.Tensor, int, int]:
    """(S, n, n_blocks) int32 permutations with the reference's RNG schedule:
    surrogate k uses torch.Generator(device).manual_seed(seed + k) and
    argsort(rand(n, n_blocks)) (block) or argsort(rand(n, T)) (random)."""
    random_mode = shuffle_method == "random" or block_length <= 1 or block_length >= T
    bl = 1 if random_mode else int(block_length)
    n_blocks = T if random_mode else T // bl
    out = torch.empty((k_end - k_start, n_vars, n_blocks), dtype=torch.int32, device=device)
    gen = torch.Generator(device=device)
    for ki, k in enumerate(range(k_start, k_end)):
        gen.manual_seed(seed + k)
        rnd = torch.rand(n_vars, n_blocks, device=device, generator=gen)
        out[ki].copy_(torch.argsort(rnd, dim=1).to(torch.int32))
    return out, bl, n_blocks


class SurrogateAccumulator:
    """Device state of one surrogate run: shuffled-bins buffer, workspaces and
    the float64/int32 accumulators, with one routine per surrogate."""

    def __init__(self, db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int,
                 observed: torch.Tensor, binary: bool, cfg=None,
                 pair_offset: int = 0, n_pairs: int | None = None):
        dev = db.data.device
        n = db.n
        self.db, self.npv, self.b_max, self.tau, self.binary = db, npv, int(b_max), tau, binary
        self.obs = observed
        self.cfg = cfg
        self.p0 = pair_offset
        self.np_ = n * (n - 1) - pair_offset if n_pairs is None else n_pairs
        self.shuf = D.empty_bins(n, db.T, db.K, dev)
        self.sum = torch.zeros((n, n), dtype=torch.float64, device=dev)
        self.sumsq = torch.zeros((n, n), dtype=torch.float64, device=dev)
        self.cnt = torch.zeros((n, n), dtype=torch.int32, device=dev)
        self.ws = D.workspace(dev, n, db.row_len, self.b_max)
        if binary:
            self.tmp = torch.zeros((n, n), dtype=torch.float32, device=dev)
            nb = int(native.lib().tenex_b2_workspace_bytes(n, db.row_len, tau * db.K))
            self.b2ws = torch.empty(nb, dtype=torch.uint8, device=dev)

    def add(self, perm: torch.Tensor, block_length: int) -> None:
        D.block_shuffle(self.db, perm, block_length, out=self.shuf)
        s = native.stream_ptr()
        if self.binary:
            n = self.db.n
            native.call("tenex_te_binary_matrix", self.shuf.ptr(), self.shuf.ld, n,
                        self.shuf.row_len, self.tau * self.db.K, self.tmp.data_ptr(), n,
                        self.b2ws.data_ptr(), self.b2ws.numel(), s)
            native.call("tenex_stats_accumulate", self.tmp.data_ptr(), self.obs.data_ptr(),
                        self.sum.data_ptr(), self.sumsq.data_ptr(), self.cnt.data_ptr(), n, s)
        else:
            D.surrogate_accumulate(self.shuf, self.npv, self.b_max, self.tau, self.obs, self.sum,
                                   self.sumsq, self.cnt, self.p0, self.np_, cfg=self.cfg,
                                   ws=self.ws)

    def check(self) -> None:
        s = native.stream_ptr()
        if self.binary:
            native.call("tenex_b2_status", self.b2ws.data_ptr(), self.db.n, self.shuf.row_len,
                        self.tau * self.db.K, s)
        else:
            native.call("tenex_workspace_status", self.ws.data_ptr(), s)


def run_surrogates(acc: SurrogateAccumulator, perms: torch.Tensor, block_length: int,
                   use_graph: bool = False) -> None:
    """Adds all surrogates of `perms` (S, n, n_blocks) into `acc`."""
    S = perms.shape[0]
    if S == 0:
        return
    acc.add(perms[0], block_length)  # eager: loads kernels, sets attributes
    acc.check()
    if S == 1:
        return
    if use_graph:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for k in range(1, S):
                acc.add(perms[k], block_length)
        g.replay()
        torch.cuda.synchronize(perms.device)
        del g
    else:
        for k in range(1, S):
            acc.add(perms[k], block_length)
    acc.check()


def surrogate_statistics(observed_te: np.ndarray, sum_surr: np.ndarray, sum_sq_surr: np.ndarray,
                         count_ge: np.ndarray, n_surrogates: int, p_method: str):
    """mean, std (population), effective TE and p-values, computed with the
    reference's numpy expressions (tenex/inference/surrogate_test.py:890-912)."""
    out = pair_statistics(observed_te, sum_surr, sum_sq_surr, count_ge, n_surrogates, p_method)
    np.fill_diagonal(out[3], 1.0)
    return out


def pair_statistics(observed_te: np.ndarray, sum_surr: np.ndarray, sum_sq_surr: np.ndarray,
                    count_ge: np.ndarray, n_surrogates: int, p_method: str):
    """The elementwise part of surrogate_statistics, for arrays of any shape
    (the learned null applies it to its verified pairs only)."""
    mean_surr = (sum_surr / n_surrogates).astype(np.float32)
    var_surr = sum_sq_surr / n_surrogates - (sum_surr / n_surrogates) ** 2
    std_surr = np.sqrt(np.maximum(var_surr, 0.0)).astype(np.float32)
    effective_te = (observed_te - mean_surr).astype(np.float32)
    if p_method == "parametric":
        from scipy.special import erfc
        eps = np.float32(1e-12)
        z = (observed_te - mean_surr) / np.maximum(std_surr, eps)
        p_values = (0.5 * erfc(z / np.sqrt(2.0))).astype(np.float32)
    else:
        p_values = ((1.0 + count_ge) / (1.0 + n_surrogates)).astype(np.float32)
    return mean_surr, std_surr, effective_te, p_values


def pair_statistics_device(observed_te: torch.Tensor, sum_surr: torch.Tensor,
                           sum_sq_surr: torch.Tensor, count_ge: torch.Tensor, n_surrogates: int,
                           p_method: str):
    """pair_statistics on device tensors, op for op: float64 mean and population
    variance (sum_sq / S - (sum / S)^2, the square as one multiply), float32 mean,
    std and effective TE, z in float32, p = erfc(z / sqrt 2) / 2 in float64. Every
    step is a separate correctly rounded IEEE operation as in numpy; only erfc is
    CUDA's instead of scipy's (both within ~1 ulp of double, so the float32 p
    agrees except where a value sits on a float32 rounding boundary)."""
    m64 = sum_surr / n_surrogates
    mean_surr = m64.float()
    var_surr = sum_sq_surr / n_surrogates - m64 * m64
    std_surr = torch.sqrt(torch.clamp(var_surr, min=0.0)).float()
    effective_te = observed_te - mean_surr
    if p_method == "parametric":
        z = effective_te / torch.clamp(std_surr, min=np.float32(1e-12).item())
        p_values = (0.5 * torch.special.erfc(z.double() / np.sqrt(2.0))).float()
    else:
        p_values = ((1.0 + count_ge.double()) / (1.0 + n_surrogates)).float()
    return mean_surr, std_surr, effective_te, p_values


def tested_mask(n: int, variable_names, sources, device) -> torch.Tensor:
    """(n, n) bool: the pairs BH runs over (the source-filtered pairs, or every
    off-diagonal pair)."""
    if sources is not None:
        pb = build_pairs(np.asarray(variable_names), sources)
        mask = torch.zeros((n, n), dtype=torch.bool, device=device)
        mask[torch.as_tensor(pb[:, 0], device=device), torch.as_tensor(pb[:, 1], device=device)] = True
        return mask
    return ~torch.eye(n, dtype=torch.bool, device=device)


def bh_edges_device(p: torch.Tensor, eff: torch.Tensor, tested: torch.Tensor, variable_names,
                    fdr: float) -> GRN:
    """bh_edges on device matrices: BH over p[tested] (row-major, float32), edges
    with adjusted p < fdr and effective TE > 0; the same edges as bh_edges gives
    for the same float32 values."""
    adj = bh_fdr_gpu(p[tested], alpha=fdr)
    sig = torch.zeros_like(tested)
    sig[tested] = adj < fdr
    sig &= eff > 0
    idx = torch.nonzero(sig)
    pairs = idx.cpu().numpy().astype(np.int64)
    te = eff[idx[:, 0], idx[:, 1]].cpu().numpy()
    return make_grn(np.asarray(variable_names), pairs, te)


def bh_edges(p_values: np.ndarray, effective_te: np.ndarray, variable_names, sources, fdr: float,
             device) -> tuple[GRN, np.ndarray]:
    """BH-FDR over the tested pairs; edges with adjusted p < fdr and effective TE > 0.
    Returns the GRN and the boolean (n, n) significance mask."""
    n = p_values.shape[0]
    if sources is not None:
        pairs_bh = build_pairs(np.asarray(variable_names), sources)
        mask = np.zeros((n, n), dtype=bool)
        mask[pairs_bh[:, 0], pairs_bh[:, 1]] = True
    else:
        mask = ~np.eye(n, dtype=bool)
    p_off = p_values[mask]
    fdr_adj = bh_fdr_gpu(torch.from_numpy(p_off).to(device), alpha=fdr).cpu().numpy()
    sig = np.zeros((n, n), dtype=bool)
    sig[mask] = fdr_adj < fdr
    sig &= effective_te > 0
    pairs = np.argwhere(sig).astype(np.int64)
    grn = make_grn(np.asarray(variable_names), pairs, effective_te[pairs[:, 0], pairs[:, 1]])
    return grn, sig


class SurrogateTestMethod:
    """Time-axis shuffle surrogate test (block or random), on one CUDA device."""

    name = "surrogate_test"

    def infer(self, te_matrix, variable_names, device, **kwargs) -> SurrogateTestResult:
        bin_data = kwargs.get("bin_data")
        n_per_var = kwargs.get("n_per_var")
        b_max = kwargs.get("b_max")
        kernel_name = kwargs.get("kernel")
        if bin_data is None or n_per_var is None or b_max is None or not kernel_name:
            raise ValueError("surrogate_test requires bin_data, n_per_var, b_max, and kernel. "
                             "Pass a TransferEntropyResult to NetWeaver (these are auto-filled).")
        tau = int(kwargs.get("tau", 1))
        n_surrogates = int(kwargs.get("n_surrogates", 100))
        shuffle_method = kwargs.get("shuffle_method", "block")
        block_length = kwargs.get("block_length")
        p_method = kwargs.get("p_method", "parametric")
        fdr = float(kwargs.get("fdr", 0.01))
        seed = int(kwargs.get("seed", 42))
        null = kwargs.get("null", "full")
        # 2 x S launches of ~10 ms each: eager launching is cheaper than capturing and
        # instantiating a graph for a single replay (measured on cfg5: 1.376 vs 1.399 s)
        use_graph = bool(kwargs.get("use_graph", False))
        if shuffle_method not in ("block", "random"):
            raise ValueError(f"shuffle_method must be 'block' or 'random' (got {shuffle_method!r})")
        if n_surrogates < 2:
            raise ValueError(f"n_surrogates must be >= 2 (got {n_surrogates}); parametric "
                             f"z-test needs a non-degenerate std estimate and MC p-values need "
                             f"at least two samples to be informative.")
        if p_method not in ("parametric", "mc"):
            raise ValueError(f"p_method must be 'parametric' or 'mc' (got {p_method!r})")
        if null not in ("full", "learned"):
            raise ValueError(f"null must be 'full' or 'learned' (got {null!r})")
        # fused= picks the reference's per-pair fused kernel (float32 running sums,
        # the default below L = 1500) or its loop path (float64 sums). This build has
        # one path for both: a full TE launch per surrogate whose epilogue adds into
        # float64 sums, i.e. the loop path's accumulation for every L. The argument is
        # validated as the reference validates it.
        fused = kwargs.get("fused")
        if fused not in (None, True, False):
            raise ValueError(f"fused must be None, True or False (got {fused!r})")
        if fused is True and kernel_name not in ("Full-SMEM", "Adaptive-SMEM"):
            raise ValueError(f"fused=True requested but kernel {kernel_name!r} has no fused "
                             f"variant (supported: 'Full-SMEM', 'Adaptive-SMEM')")
        bin_data = np.asarray(bin_data)
        if bin_data.ndim == 2:
            bin_data = bin_data[..., None]
        n_vars, T, K = bin_data.shape
        if T - tau < 2:
            raise ValueError(f"T - tau = {T - tau} is too short for TE computation")
        if block_length is None:
            block_length = max(2, int(np.sqrt(T - tau)))
        block_length = int(block_length)
        dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("the surrogate test runs on a CUDA device")
        devices = kwargs.get("devices")
        device_ids = [int(d) for d in devices] if devices else [dev.index or 0]
        dev = torch.device("cuda", device_ids[0])
        torch.cuda.set_device(dev)
        observed_te = np.asarray(te_matrix, dtype=np.float32)
        if null == "learned":
            from tenex_b200.inference.learned_null import learned_surrogate_test
            return learned_surrogate_test(self, observed_te, variable_names, dev, bin_data,
                                          np.asarray(n_per_var), int(b_max), kernel_name, tau,
                                          n_surrogates, shuffle_method, block_length, p_method,
                                          fdr, seed, kwargs)
        _log.vprint(f"[TENEX] surrogate_test: {n_surrogates} shuffles (method={shuffle_method}, "
                    f"block_length={block_length}, kernel={kernel_name}, p={p_method})")
        # the binary path updates the whole matrix per surrogate (sub-millisecond each):
        # it stays on the first device
        if len(device_ids) == 1 or kernel_name == "GEMM-B2":
            # sums stay on the device: statistics and BH there, one copy back
            sums = self.accumulate(observed_te, dev, bin_data, n_per_var, int(b_max),
                                   kernel_name, tau, n_surrogates, shuffle_method, block_length,
                                   seed, use_graph, as_numpy=False)
            obs_d = torch.as_tensor(observed_te).to(dev)
            stats = pair_statistics_device(obs_d, *sums, n_surrogates, p_method)
            diag = torch.arange(observed_te.shape[0], device=dev)
            stats[3][diag, diag] = 1.0
            grn = bh_edges_device(stats[3], stats[2],
                                  tested_mask(observed_te.shape[0], variable_names,
                                              kwargs.get("sources"), dev),
                                  variable_names, fdr)
            mean_surr, std_surr, effective_te, p_values = D.to_host(torch.stack(stats))
        else:
            sum_surr, sum_sq_surr, count_ge = self._accumulate_devices(
                observed_te, device_ids, bin_data, n_per_var, int(b_max), kernel_name, tau,
                n_surrogates, shuffle_method, block_length, seed, use_graph)
            mean_surr, std_surr, effective_te, p_values = surrogate_statistics(
                observed_te, sum_surr, sum_sq_surr, count_ge, n_surrogates, p_method)
            grn, _ = bh_edges(p_values, effective_te, variable_names, kwargs.get("sources"), fdr,
                              dev)
        _log.vprint(f"[TENEX] surrogate_test: {len(grn)} significant edges (FDR<{fdr})")
        return SurrogateTestResult(observed_te=observed_te, mean_surrogate_te=mean_surr,
                                   std_surrogate_te=std_surr, effective_te=effective_te,
                                   p_values=p_values, grn=grn, n_surrogates=n_surrogates,
                                   shuffle_method=shuffle_method,
                                   block_length=block_length if shuffle_method == "block"
                                   else None, p_method=p_method, fdr=fdr)

    @classmethod
    def _accumulate_devices(cls, observed_te, device_ids, bin_data, n_per_var, b_max,
                            kernel_name, tau, n_surrogates, shuffle_method, block_length, seed,
                            use_graph=False):
        """The reference's multi-GPU split of the fused path
        (tenex/inference/surrogate_test.py:812-842): pair-id boundaries
        linspace(0, n(n-1), devices + 1), one host thread per device running every
        surrogate on its pairs; the disjoint per-device sums add exactly, and the
        diagonal's count_ge is added once."""
        from concurrent.futures import ThreadPoolExecutor
        n = bin_data.shape[0]
        bnd = np.linspace(0, n * (n - 1), len(device_ids) + 1, dtype=np.int64)

        def work(rank: int):
            torch.cuda.set_device(device_ids[rank])
            d = torch.device("cuda", device_ids[rank])
            return cls.accumulate(observed_te, d, bin_data, n_per_var, b_max, kernel_name, tau,
                                  n_surrogates, shuffle_method, block_length, seed, use_graph,
                                  pair_offset=int(bnd[rank]),
                                  n_pairs=int(bnd[rank + 1] - bnd[rank]), diag_count=False)

        with ThreadPoolExecutor(max_workers=len(device_ids)) as ex:
            parts = list(ex.map(work, range(len(device_ids))))
        s1, s2, c = (sum(p[i] for p in parts) for i in range(3))
        diag = np.arange(n)
        c[diag, diag] += n_surrogates
        return s1, s2, c

    @staticmethod
    def accumulate(observed_te, dev, bin_data, n_per_var, b_max, kernel_name, tau, n_surrogates,
                   shuffle_method, block_length, seed, use_graph=False, k_start=0,
                   pair_offset=0, n_pairs=None, diag_count=True, as_numpy=True):
        """float64 sum, sum of squares and int32 count_ge (numpy, (n, n)) over
        surrogates [k_start, k_start + n_surrogates), diagonal count included."""
        n_vars, T, K = bin_data.shape
        db = D.pack_bins(bin_data, dev)
        npv = torch.as_tensor(np.asarray(n_per_var), dtype=torch.int32).to(dev)
        binary = kernel_name == "GEMM-B2"
        obs_d = torch.as_tensor(observed_te, dtype=torch.float32).to(dev).contiguous()
        from tenex_b200.kernels import get_kernel
        kobj = get_kernel(kernel_name)
        cfg = getattr(kobj, "cfg", None)
        if cfg is None and not binary and hasattr(kobj, "launch_cfg"):
            # launch shape tuned once on the observed bins (the shuffles keep every
            # gene's bin counts, so the tuned shape carries over)
            cfg = kobj.launch_cfg(db, npv, b_max, tau, autotune_shape=True)
        acc = SurrogateAccumulator(db, npv, b_max, tau, obs_d, binary, cfg, pair_offset, n_pairs)
        perms, bl, _ = build_block_perm(n_vars, T, shuffle_method, block_length, k_start,
                                        k_start + n_surrogates, seed, dev)
        run_surrogates(acc, perms, bl, use_graph)
        if diag_count:  # te_k >= observed holds on the diagonal (0 >= 0)
            diag = torch.arange(n_vars, device=acc.cnt.device)
            acc.cnt[diag, diag] += n_surrogates
        if not as_numpy:
            return acc.sum, acc.sumsq, acc.cnt
        return acc.sum.cpu().numpy(), acc.sumsq.cpu().numpy(), acc.cnt.cpu().numpy()
