"""Benchmark: LMM association SNPs/s at n = 20,000 samples, all tests (-lmm 4).

One step = the association hot path over one chunk of SNPs of a resident cohort:
device decode of packed .bed records -> mean imputation -> eigenvector rotation ->
per-SNP Score / MLE+LRT / REML+Wald search and statistics.  The cohort's kinship and
eigendecomposition are set-up work, timed and reported separately (kinship_s, eigh_s).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own shard of SNP chunks of a replica cohort (weak
scaling, no data-path collective); the timed region is bracketed by barriers and the
max over ranks is reported.  ``--impl reference`` times the CPU oracle (jamma's path
restated in NumPy/SciPy) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_PEAK_FALLBACK = 6650.0
BF16_PEAK_FALLBACK = 1590.0
# DRAM read + write bytes of one INT8 rotation launch, measured once with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) for the configuration in the key:
# (n, SNPs per launch, missing calls present, rotation kernel variant, tile schedule).
# Any other configuration reports traffic null rather than a stale figure.
ROT_DRAM_BYTES = {(20000, 8192, True, 0, (9, 16)): 30.39e9,
                  (20000, 8192, True, 0, (5, 32)): 36.25e9,
                  (20000, 8192, True, 0, (17, 8)): 25.26e9,
                  (20000, 8192, True, 0, (3, 64)): 56.31e9,
                  (20000, 8192, True, 0, (36, 4)): 32.89e9}


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every 20 ms while
    the timed region runs (read-only queries).  The NVML device is matched to the CUDA
    device by PCI bus id, so CUDA_VISIBLE_DEVICES remapping does not matter."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, index: int):
        self.index = index
        self.sm: list[float] = []
        self.max_sm: float | None = None
        self.reasons: set[str] = set()
        self.error: str | None = None
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.index)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def _run(self):
        try:
            nv, h = self._handle()
            self.max_sm = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            while not self._stop.is_set():
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                mask = int(get_reasons(h))
                self.reasons.update(v for k, v in self.REASONS.items() if mask & k)
                self._stop.wait(0.02)
        except Exception as e:  # reported in the summary, never fatal to the bench
            self.error = f"{type(e).__name__}: {e}"

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_sm, "reasons": ["unsampled"],
                    "error": self.error}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_sm,
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args) -> None:
    """CPU arm: the oracle (jamma's JAX path restated in NumPy) on a bounded sample."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    from threadpoolctl import threadpool_info

    from oracle import lmm as OL

    n, m, c = args.n, args.ref_snps, args.n_cvt
    rng = np.random.default_rng(20261203)
    t0 = time.perf_counter()
    # cohort of the same shape: kinship from a SNP sample, FP64 eigh (set-up, not timed)
    gk = rng.binomial(2, rng.uniform(0.05, 0.5, 2000), size=(n, 2000)).astype(np.float64)
    gk -= gk.mean(0)
    K = gk @ gk.T / 2000
    evals, U = OL.eigh_threshold(K)
    W = np.column_stack([np.ones(n), rng.normal(size=(n, c - 1))])
    y = rng.normal(size=n)
    UT = np.ascontiguousarray(U.T)
    UtW, Uty = UT @ W, UT @ y
    lam0, l0 = OL.null_model_mle(evals, UtW, Uty)
    setup_s = time.perf_counter() - t0
    per_step = []
    for it in range(args.warmup + args.steps):
        g = rng.binomial(2, rng.uniform(0.05, 0.5, m), size=(n, m)).astype(np.float64)
        g[rng.random((n, m)) < args.miss] = np.nan
        t = time.perf_counter()
        mu = np.nanmean(g.astype(np.float32), 0).astype(np.float64)
        g = np.where(np.isnan(g), mu[None, :], g)
        OL.lmm_chunk(args.mode, evals, UtW, Uty, UT @ g, l0, lam0)
        if it >= args.warmup:
            per_step.append(time.perf_counter() - t)
    sec = float(np.mean(per_step))
    value = m / sec
    cores = max([i.get("num_threads", 0) for i in threadpool_info() if i.get("user_api") == "blas"] or [1])
    line = {
        "impl": "reference", "metric": "lmm_assoc_snps_per_s", "value": value, "unit": "SNPs/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": _config(args, per_step_snps=m),
        "cpu_baseline": {"value": value, "unit": "SNPs/s", "cores": cores, "kind": "port",
                         "sample": f"{m} SNPs per step at n={n}, c={c}, -lmm {args.mode}; "
                                   f"set-up (eigh n={n}) {setup_s:.1f}s untimed"},
        "e2e": {"value": value, "unit": "SNPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _config(args, per_step_snps) -> dict:
    return {"workload": f"lmm -lmm {args.mode} n={args.n} c={args.n_cvt} phenotypes=1, "
                        f"{per_step_snps} SNPs per step, {args.miss:.0%} missing calls",
            "n_samples": args.n, "n_cvt": args.n_cvt, "lmm_mode": args.mode,
            "snps_per_step": per_step_snps, "precision": args.precision,
            "l2": "inputs > L2 (each step's imputed FP64 chunk is n*m*8 bytes)",
            "parallelism": f"replicas{_dist()[0]}"}


def _int8_gemm_peak(size: int = 8192, reps: int = 10) -> float:
    """cuBLASLt INT8 GEMM (torch._int_mm, int8 x int8 -> int32) on this GPU: best of
    ``reps`` CUDA-event-timed size^3 products, in TOP/s (2 ops per multiply-add)."""
    import torch

    a = torch.randint(-127, 127, (size, size), dtype=torch.int8, device="cuda")
    b = torch.randint(-127, 127, (size, size), dtype=torch.int8, device="cuda").t().contiguous().t()
    for _ in range(3):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * size ** 3 / (best / 1e3) / 1e12


def _kinship_phases(ev, n: int, p: int, i8_peak: float) -> dict | None:
    """Device time of the INT8 kinship's two phases: the per-chunk layout + correction
    kernels, and the Gram + finalisation (one tcgen05 GEMM of n(n+1)p int8 ops)."""
    if ev is None:
        return None
    chunks_ms, gram_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    tops = n * (n + 1.0) * p / (gram_ms / 1e3) / 1e12
    return {"chunks_ms": _r(chunks_ms), "gram_finalize_ms": _r(gram_ms), "gram_tops": _r(tops),
            "gram_frac_int8_measured": _r(tops / i8_peak)}


def _r(x, sig: int = 3):
    """Round to `sig` significant digits (keeps the JSON line short)."""
    if x is None or not np.isfinite(x) or x == 0:
        return None if x is None else (float(x) if np.isfinite(x) else None)
    return float(f"{x:.{sig - 1}e}")


P_FIELDS = ("p_wald", "p_lrt", "p_score")
ACC_FIELDS = ("beta", "se", "logl_h1", "lambda_remle", "lambda_mle") + P_FIELDS


def _accuracy(got: dict, ref: dict, rows=slice(None)) -> dict:
    """Errors of one form's statistics against another's on the same SNPs.  Per field the
    max / median relative error and the number of SNPs whose NaN pattern differs; for
    p-values also the fraction within 1e-6 relative, the max |log10 p| difference and the
    number of significance calls that differ at 5e-8."""
    out = {}
    for k in ACC_FIELDS:
        if k not in got or k not in ref:
            continue
        a = np.asarray(got[k], dtype=np.float64).ravel()[rows]
        b = np.asarray(ref[k], dtype=np.float64).ravel()[rows]
        ok = np.isfinite(a) & np.isfinite(b)
        rel = np.abs(a[ok] - b[ok]) / np.maximum(np.abs(b[ok]), 1e-300)
        e = {"max_rel": float(rel.max()) if rel.size else None,
             "median_rel": float(np.median(rel)) if rel.size else None,
             "nonfinite_mismatch": int(np.sum(np.isfinite(a) != np.isfinite(b)))}
        if k in P_FIELDS:
            e["frac_rel_le_1e-6"] = float(np.mean(rel <= 1e-6)) if rel.size else None
            e["max_abs_dlog10"] = float(np.max(np.abs(np.log10(a[ok]) - np.log10(b[ok])))) \
                if rel.size else None
            e["calls_differ_5e-8"] = int(np.sum((a[ok] < 5e-8) != (b[ok] < 5e-8)))
        out[k] = e
    return out


def _accuracy_compact(acc: dict) -> dict:
    """One number per non-p field (max rel) and [max rel, fraction <= 1e-6, max |dlog10 p|,
    calls differing at 5e-8] per p-value field; NaN-pattern mismatches summed."""
    out = {}
    for k, e in acc.items():
        key = {"lambda_remle": "l_remle", "lambda_mle": "l_mle"}.get(k, k)
        if k in P_FIELDS:
            out[key] = [_r(e["max_rel"]), _r(e["frac_rel_le_1e-6"], 4), _r(e["max_abs_dlog10"]),
                        e["calls_differ_5e-8"]]
        else:
            out[key] = _r(e["max_rel"])
    out["nan_mismatch"] = int(sum(e["nonfinite_mismatch"] for e in acc.values()))
    return out


def _oracle_check(args, packed_host: np.ndarray, evals_h: np.ndarray, UT: np.ndarray,
                  W: np.ndarray, y: np.ndarray) -> tuple[dict, dict]:
    """The oracle (jamma's path restated in NumPy/SciPy) on the first SNPs of a timed chunk:
    the same packed records, decoded on the host, mean-imputed with the float32 pass-1
    mean, rotated with the same eigenvectors on host BLAS, and searched.  Returns the
    oracle's statistics and the CPU baseline: rotation + search of these SNPs timed on the
    host cores (the null model is cohort set-up and runs before the timer)."""
    from threadpoolctl import threadpool_info

    from oracle import lmm as OL
    from oracle.kinship import stream_pass1_means
    from oracle.plink import decode_packed

    n = args.n
    g = decode_packed(packed_host, n)  # (n, m) float64, NaN = missing
    mean32, _, _ = stream_pass1_means(g)
    g = np.where(np.isnan(g), np.asarray(mean32, dtype=np.float64)[None, :], g)
    UtW, Uty = UT @ W, UT @ y
    lam0 = l0 = None
    if args.mode in (2, 3, 4):
        lam0, l0 = OL.null_model_mle(evals_h, UtW, Uty)
    t = time.perf_counter()
    ref = OL.lmm_chunk(args.mode, evals_h, UtW, Uty, UT @ g, l0, lam0)
    sec = time.perf_counter() - t
    m = g.shape[1]
    cores = max([i.get("num_threads", 0) for i in threadpool_info() if i.get("user_api") == "blas"]
                or [1])
    cpu = {"value": m / sec, "unit": "SNPs/s", "cores": cores, "kind": "port",
           "sample": f"the first {m} SNPs of a timed chunk (same records, 1 % missing calls) at "
                     f"n={n}, -lmm {args.mode}: host-BLAS rotation + NumPy/SciPy search"}
    return ref, cpu


def _e2e_streaming(args, w, U, W, y, packed_host: np.ndarray) -> dict:
    """The metric end to end through jamma's public streaming runner on a PLINK file:
    ``run_lmm_association_streaming(bfile, ..., precision="mixed")`` with the cohort's
    eigendecomposition.  Its association stage (every chunk's .bed read into pinned host
    memory, host-to-device copy, the chunk's CUDA graph, device-to-host copy of the
    results) is timed by the runner on the host wall clock; the whole call (pass-1
    statistics over the file, cohort set-up from the eigenvectors, the result objects) is
    reported beside it."""
    import shutil
    import tempfile

    import torch

    from jamma_b200 import run_lmm_association_streaming
    from jamma_b200.io import write_plink_records

    n, m = args.n, args.chunk
    tmp = Path(tempfile.mkdtemp(prefix="jb_e2e_"))
    try:
        prefix = tmp / "cohort"
        write_plink_records(prefix, packed_host, n)
        timing: dict = {}
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = run_lmm_association_streaming(prefix, y, eigenvalues=w, eigenvectors=U,
                                            covariates=W if W.shape[1] > 1 else None,
                                            lmm_mode=args.mode, precision="mixed",
                                            timing=timing)
        call_s = time.perf_counter() - t
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    tested = timing["n_tested"]
    bps = (n + 3) // 4
    n_out = 9 if args.mode == 4 else 5
    return {"value": tested / timing["association_s"], "unit": "SNPs/s",
            "h2d_bytes_per_step": m * bps + m * 8, "d2h_bytes_per_step": n_out * m * 8,
            "path": "jamma_b200.run_lmm_association_streaming(bfile, precision='mixed', "
                    f"lmm_mode={args.mode}) on a written .bed: association stage (pinned "
                    "double-buffered .bed chunks, side-stream H2D, CUDA-graph replay, async D2H) "
                    "on the host wall clock",
            "snps": tested, "chunk": m, "association_s": _r(timing["association_s"], 4),
            "whole_call_snps_per_s": _r(tested / call_s, 4),
            "whole_call_s": {"total": _r(call_s, 4), "pass1": _r(timing["stats_s"], 4),
                             "setup": _r(timing["setup_s"], 4), "results": _r(timing["write_s"], 4)},
            "results_returned": len(res)}


def run_serving(args, seed: int = 7) -> dict:
    """A Poisson stream of GWAS jobs through the continuous-batching server.

    Default: a reduced version of the serving configuration so that the default bench
    stays within minutes -- ``args.serve_jobs`` jobs, n ~ log-uniform in [2 000, 8 000],
    SNPs ~ log-uniform in [10 000, 40 000], 1-4 phenotypes.  ``--serve-c4``: the serving
    configuration itself -- 200 jobs, n ~ log-uniform in [2 000, 40 000], SNPs ~
    log-uniform in [10 000, 200 000], 1-8 phenotypes.  Both: lmm mode drawn from
    {1, 2, 3, 4}, 30 % of jobs reusing a resident cohort's eigenvectors, 1 % missing calls.
    """
    import torch

    from jamma_b200 import synth
    from jamma_b200.serve import GwasJob, GwasServer

    c4 = args.serve_c4
    n_jobs = 200 if c4 else args.serve_jobs
    n_lo, n_hi = (2000, 40000) if c4 else (2000, 8000)
    p_lo, p_hi = (10000, 200000) if c4 else (10000, 40000)
    phi_hi = 8 if c4 else 4
    rng = np.random.default_rng(seed)
    cohorts = {}
    jobs = []
    t = 0.0
    for i in range(n_jobs):
        if cohorts and rng.random() < 0.3:
            cid = list(cohorts)[rng.integers(len(cohorts))]
        else:
            cid = f"c{i}"
            n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
            p = int(np.exp(rng.uniform(np.log(p_lo), np.log(p_hi))))
            cohorts[cid] = (n, synth.packed_records_device(n, p, 0.01, seed=5000 + i).cpu().numpy())
        n, packed = cohorts[cid]
        phi = int(rng.integers(1, phi_hi + 1))
        y = rng.normal(size=(n, phi))
        cov = np.column_stack([np.ones(n), rng.normal(size=n)]) if rng.random() < 0.5 else None
        t += rng.exponential(args.serve_gap)
        jobs.append((t, GwasJob(f"j{i}", cid, packed, n, y if phi > 1 else y[:, 0], cov,
                                int(rng.integers(1, 5)))))
    # the full configuration issues chunks eagerly: under its memory pressure a chunk-graph
    # capture failed and the failed graph's teardown aborted the process
    srv = GwasServer(hbm_budget_bytes=int(args.serve_budget_gb * (1 << 30)), max_active=4,
                     chunk=4096, capture_graphs=not c4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    srv.run(jobs)
    wall = time.perf_counter() - t0
    out = srv.latency_summary()
    total_snps = sum(j.snp_indices.size * (1 if np.ndim(j.phenotypes) == 1 else j.phenotypes.shape[1])
                     for _, j in jobs)
    out.update(workload=(f"{'serving configuration' if c4 else 'reduced serving mix'}: {n_jobs} jobs, "
                         f"Poisson gaps {args.serve_gap}s, n {n_lo}-{n_hi}, SNPs {p_lo}-{p_hi}, "
                         f"1-{phi_hi} phenotypes, modes 1-4, 30% cohort reuse"),
               hbm_budget_gb=args.serve_budget_gb, max_active=4, wall_s=wall,
               snp_phenotype_pairs=int(total_snps),
               new_cohorts=int(sum(1 for _, j in jobs if j.new_cohort)))
    return out


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    from jamma_b200 import _build

    if rank == 0:
        _build.build()
    if world > 1:
        dist.barrier()
    if args.rot_kernel is not None:
        from jamma_b200 import _native as _nat

        _nat.call("jb_rotate_set_kernel", args.rot_kernel)
    from jamma_b200 import _native, engine as eng, synth
    from jamma_b200.device import ptr, stream_handle
    from jamma_b200.kinship import _KinshipAccumulator, _KinshipI8, snp_stats_from_counts

    n, m, c = args.n, args.chunk, args.n_cvt
    nsteps = args.warmup + args.steps
    bps = (n + 3) // 4
    st = torch.cuda.current_stream()

    # ---------------- cohort set-up: kinship (INT8 Gram and plain FP64 Gram) + eigh
    kin_p = args.kin_snps
    kin_rec = synth.packed_records_device(n, kin_p, args.miss, seed=100 + rank)
    kc = 16384
    kin_counts = []
    for s in range(0, kin_p, kc):
        _, cnt = eng.decode_packed(kin_rec[s:s + kc], n, None, n)
        kin_counts.append(cnt.cpu().numpy())
    kin_counts = np.concatenate(kin_counts)
    poly = snp_stats_from_counts(kin_counts, n)[2]
    keep = np.where(poly)[0]

    kin_events = {}

    def kinship(form: str):
        acc = _KinshipI8(n, keep.size) if form == "int8" else _KinshipAccumulator(n, 4096)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(st)
        for s in range(0, keep.size, kc):
            sub = keep[s:s + kc]
            rec_k = kin_rec.index_select(0, torch.from_numpy(sub).cuda())
            codes_k, _ = eng.decode_packed(rec_k, n, None, n)
            cc = kin_counts[sub]
            mu = torch.from_numpy(cc[:, 1] / np.maximum(cc[:, 0], 1)).cuda()
            if form == "int8":
                acc.add(codes_k, mu, bool(np.any(cc[:, 0] < n)), n_missing=int((n - cc[:, 0]).sum()))
                acc.add_sum_mu2(cc[:, 1] / np.maximum(cc[:, 0], 1))
            else:
                acc.add(codes_k, mu)
        ev[1].record(st)
        K_out = acc.finish()
        ev[2].record(st)
        kin_events[form] = ev
        return K_out

    # one small INT8 kinship first, so the timed one excludes one-time costs (kernel
    # module loads, allocator growth); it covers the first chunk's SNPs only
    acc_w = _KinshipI8(n, min(kc, keep.size))
    sub_w = keep[: min(kc, keep.size)]
    cc_w = kin_counts[sub_w]
    codes_w, _ = eng.decode_packed(kin_rec.index_select(0, torch.from_numpy(sub_w).cuda()), n, None, n)
    acc_w.add(codes_w, torch.from_numpy(cc_w[:, 1] / np.maximum(cc_w[:, 0], 1)).cuda(),
              bool(np.any(cc_w[:, 0] < n)), n_missing=int((n - cc_w[:, 0]).sum()))
    acc_w.finish()
    del acc_w, codes_w
    torch.cuda.synchronize()
    t = time.perf_counter()
    if args.profile_phase == "kinship":  # the INT8 kinship is the profiler range
        torch.cuda.profiler.start()
    K = kinship("int8")
    torch.cuda.synchronize()
    if args.profile_phase == "kinship":
        torch.cuda.profiler.stop()
    kinship_s = time.perf_counter() - t
    kinship_fp64_s = None
    if not args.skip_fp64_kinship:
        t = time.perf_counter()
        K64 = kinship("fp64")
        torch.cuda.synchronize()
        kinship_fp64_s = time.perf_counter() - t
        kin_maxdiff = float((K64 - K).abs().max().item() / K64.abs().max().item())
        del K64
    else:
        kin_maxdiff = None
    del kin_rec
    t = time.perf_counter()
    w, U = eng.eigh_device(K)
    torch.cuda.synchronize()
    eigh_s = time.perf_counter() - t
    rng = np.random.default_rng(5)
    W = np.column_stack([np.ones(n), rng.normal(size=(n, c - 1))])
    y = rng.normal(size=n)
    cohort = eng.DeviceCohort(w, U, W, y, lmm_mode=args.mode)

    # ---------------- SNP chunks (device-resident packed records + pass-1 means)
    rec = synth.packed_records_device(n, nsteps * m, args.miss, seed=1000 + rank)
    means = []
    for s in range(nsteps):
        _, cnt = eng.decode_packed(rec[s * m:(s + 1) * m], n, None, n)
        cc = cnt.cpu().numpy().astype(np.float64)
        means.append(torch.from_numpy((cc[:, 1] / np.maximum(cc[:, 0], 1)).astype(np.float32)
                                      .astype(np.float64)).cuda())
    ld = (n + 127) // 128 * 128
    G = eng.empty((m, n))
    UtG = eng.empty((m, n))
    codes = torch.empty((m, ld), dtype=torch.int8, device="cuda")
    counts = torch.empty((m, 4), dtype=torch.int32, device="cuda")
    has_missing = args.miss > 0

    def run_form(precision: str, steps: int):
        """Warm up, then time `steps` chunks of one precision form with CUDA events."""
        c = cohort_mixed if precision == "mixed" else cohort
        outs = c.alloc_out(m)
        ev = {k: [] for k in ("decode", "rotate", "rotate_gemm", "lmm")}

        def mark():
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            return e

        def step(s, record):
            e0 = mark()
            _native.call("jb_decode_bed", ptr(rec[s * m:(s + 1) * m]), bps, m, None, n, ptr(codes),
                         ld, ptr(counts), stream_handle())
            e1 = mark()
            er = []
            if precision == "mixed":
                c.rotate_codes_i8(codes, means[s], has_missing, out=UtG,
                                  after_rotation=lambda: er.append(mark()))
            else:
                _native.call("jb_impute_f64", ptr(codes), ld, n, m, ptr(means[s]), ptr(G), n,
                             stream_handle())
                eng.rotate(c.U, G, out=UtG)
            e2 = mark()
            c.associate_rotated(UtG, outs)
            e3 = mark()
            if record:
                for k, a, b in (("decode", e0, e1), ("rotate", e1, e2), ("lmm", e2, e3)):
                    ev[k].append((a, b))
                if er:
                    ev["rotate_gemm"].append((e1, er[0]))

        for s in range(args.warmup):
            step(s, False)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # the mixed form's timed steps are the profiler range (ncu --profile-from-start off)
        prof = precision == "mixed" and args.profile_phase == "assoc"
        with ClockSampler(local) as clk:
            if prof:
                torch.cuda.profiler.start()
            a.record(st)
            for s in range(args.warmup, args.warmup + steps):
                step(s, True)
            b.record(st)
            torch.cuda.synchronize()
            if prof:
                torch.cuda.profiler.stop()
        ms = a.elapsed_time(b)
        if world > 1:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
            dist.barrier()
        kern = {k: float(np.mean([x.elapsed_time(y) for x, y in v])) for k, v in ev.items() if v}
        return ms, kern, clk.summary(), outs

    cohort_mixed = eng.DeviceCohort(w, U, W, y, lmm_mode=args.mode, precision="mixed")
    tuned = None
    if not args.no_autotune:  # rotation tile schedule (applied) and best chunk width (reported)
        from jamma_b200 import autotune

        tuned = autotune.tune(cohort_mixed, use_cache=False)
    ms, kern_ms, clocks, outs = run_form("mixed", args.steps)
    if c_status := cohort_mixed.rotate_status():
        raise RuntimeError(f"INT8 rotation pipeline status {c_status}")
    if args.traffic_sweep:  # one rotation per candidate tile schedule, as the profiler range
        from jamma_b200 import autotune as _at

        gm0, gn0 = np.zeros(1, np.int32), np.zeros(1, np.int32)
        _native.call("jb_rotate_get_schedule", gm0.ctypes.data, gn0.ctypes.data)
        k0 = _native.load().jb_rotate_get_kernel()
        _native.call("jb_rotate_set_kernel", 0)
        _native.call("jb_decode_bed", ptr(rec[:m]), bps, m, None, n, ptr(codes), ld, ptr(counts),
                     stream_handle())
        for gm, gn in _at.SCHEDULES:
            _native.call("jb_rotate_set_schedule", gm, gn)
            torch.cuda.synchronize()
            torch.cuda.profiler.start()
            cohort_mixed.rotate_codes_i8(codes, means[0], has_missing, out=UtG)
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
        _native.call("jb_rotate_set_kernel", k0)
        _native.call("jb_rotate_set_schedule", int(gm0[0]), int(gn0[0]))
    snps = args.steps * m * world
    value = snps / (ms / 1e3)
    fp64_steps = max(1, min(args.steps, args.fp64_steps))
    ms64, kern64, _, _ = run_form("fp64", fp64_steps)
    value64 = fp64_steps * m * world / (ms64 / 1e3)

    # ---------------- accuracy on one timed chunk (untimed): both GPU forms on the whole
    # chunk, and the oracle on its first SNPs (same records, eigendecomposition and phenotype)
    s_acc = args.warmup

    def one_chunk(precision: str, s: int) -> dict:
        c = cohort_mixed if precision == "mixed" else cohort
        o = c.alloc_out(m)
        _native.call("jb_decode_bed", ptr(rec[s * m:(s + 1) * m]), bps, m, None, n, ptr(codes), ld,
                     ptr(counts), stream_handle())
        if precision == "mixed":
            c.rotate_codes_i8(codes, means[s], has_missing, out=UtG)
        else:
            _native.call("jb_impute_f64", ptr(codes), ld, n, m, ptr(means[s]), ptr(G), n,
                         stream_handle())
            eng.rotate(c.U, G, out=UtG)
        c.associate_rotated(UtG, o)
        return {k: v.cpu().numpy()[0] for k, v in o.items()}

    got_mixed, got_fp64 = one_chunk("mixed", s_acc), one_chunk("fp64", s_acc)
    acc_mixed_fp64 = _accuracy(got_mixed, got_fp64)
    acc_oracle = cpu = None
    if rank == 0 and not args.no_cpu:
        k = min(args.oracle_snps, m)
        UT = U.cpu().numpy()  # row j = eigenvector j
        ref, cpu = _oracle_check(args, rec[s_acc * m:s_acc * m + k].cpu().numpy(), w.cpu().numpy(),
                                 UT, W, y)
        del UT
        acc_oracle = {"snps": k, "mixed": _accuracy(got_mixed, ref, slice(0, k)),
                      "fp64": _accuracy(got_fp64, ref, slice(0, k))}

    # ---------------- end to end through the public streaming runner on a .bed file
    e2e = None
    if rank == 0 and not args.no_e2e:
        del G
        e2e = _e2e_streaming(args, w, U, W, y, rec.cpu().numpy())
        G = eng.empty((m, n))

    # ---------------- many phenotypes per cohort (one SNP chunk, all phenotypes per warp set)
    multi = None
    if rank == 0 and args.phenotypes > 1:
        phi = args.phenotypes
        mp = min(m, args.pheno_chunk)
        Y = rng.normal(size=(n, phi))
        coh_p = eng.DeviceCohort(w, U, W, Y, lmm_mode=args.pheno_mode, precision="mixed")
        outs_p = coh_p.alloc_out(mp)
        Xp = UtG[:mp]

        def pstep(s):
            _native.call("jb_decode_bed", ptr(rec[s * m:s * m + mp]), bps, mp, None, n, ptr(codes),
                         ld, ptr(counts), stream_handle())
            coh_p.rotate_codes_i8(codes[:mp], means[s][:mp], has_missing, out=Xp)
            coh_p.associate_rotated(Xp, outs_p)
        for s in range(args.warmup):
            pstep(s)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ps = max(1, min(args.steps, 3))
        if args.profile_phase == "multi":  # the multi-phenotype steps are the profiler range
            torch.cuda.profiler.start()
        a.record(st)
        for s in range(args.warmup, args.warmup + ps):
            pstep(s)
        b.record(st)
        torch.cuda.synchronize()
        if args.profile_phase == "multi":
            torch.cuda.profiler.stop()
        pms = a.elapsed_time(b) / ps
        multi = {"phenotypes": phi, "lmm_mode": args.pheno_mode, "snps_per_step": mp,
                 "ms_per_step": _r(pms, 4), "snp_phenotype_pairs_per_s": _r(mp * phi / (pms / 1e3), 4),
                 "snps_per_s_all_phenotypes": _r(mp / (pms / 1e3), 4), "steps": ps,
                 "series_from_int8_calls": coh_p.series_ws is not None}
        del coh_p, outs_p

    serving = None
    if rank == 0 and not args.no_serving:
        # start the server from a clean allocator: the earlier legs' freed buffers go back
        # to the device instead of fragmenting the jobs' allocations
        import gc

        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        serving = run_serving(args)

    if rank == 0:
        peaks = _peaks()
        bf16 = peaks.get("bf16_tflops")
        bf16_src = "measured (MEASURED_PEAKS.json bf16_tflops, burst)" if bf16 else "fallback"
        bf16 = bf16 or BF16_PEAK_FALLBACK
        # dominant kernel of the mixed form: the INT8 tcgen05 rotation GEMM.  Algorithmic
        # work of one launch: one rotation U^T G, 2 n^2 m flops (independent of how the
        # product is split); the implementation issues 4 digit planes x (calls [+ masks])
        # int8 products.
        rot_ms = kern_ms.get("rotate_gemm", kern_ms["rotate"])
        alg_flops = 2.0 * n * n * m
        planes = 4 * (2 if has_missing else 1)
        i8_measured = _int8_gemm_peak()
        achieved = alg_flops / (rot_ms / 1e3) / 1e12
        impl_tops = alg_flops * planes / (rot_ms / 1e3) / 1e12
        variant = int(_native.load().jb_rotate_get_kernel())
        gm, gn = np.zeros(1, np.int32), np.zeros(1, np.int32)
        _native.call("jb_rotate_get_schedule", gm.ctypes.data, gn.ctypes.data)
        traffic = ROT_DRAM_BYTES.get((n, m, has_missing, variant, (int(gm[0]), int(gn[0]))))
        roofline = {
            "kernel": "i8_gemm_kernel<RotEpi> (tcgen05 kind::i8, digit-plane rotation U^T G)",
            "bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
            "frac": achieved / bf16, "traffic": traffic,
            "peak_source": f"{bf16_src}: dense bf16 cuBLAS GEMM, the tensor-pipe roofline",
            "algorithmic": "2 n^2 m flops per launch (one rotation; n samples, m SNPs)",
            "launch_ms": _r(rot_ms, 4),
            "impl_int8_ops_per_launch": alg_flops * planes,
            "impl_tops": _r(impl_tops, 4), "int8_measured_tops": _r(i8_measured, 4),
            "impl_frac_of_int8_measured": _r(impl_tops / i8_measured, 4),
            "algorithmic_bytes": 4 * n * n + 2 * n * m + 8 * n * m,
        }
        n_tests_f = int(args.mode in (1, 4)) + int(args.mode in (3, 4))
        series = cohort_mixed.series_ws is not None
        # own kernels per step (no library kernel in the mixed form): decode, [pack pairs],
        # tiles + rotation GEMM, [tiles + series GEMM], squared sums + their reduction,
        # search, [F-test p-values]
        launches = (1 + int(has_missing) + 2 + 2 * int(series) + 2 + 1 + int(n_tests_f > 0)) \
            * args.steps
        line = {
            "metric": "lmm_assoc_snps_per_s", "value": value, "unit": "SNPs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8+f64",
            "data": "synthetic (seeded device RNG; Binomial(2,p) genotypes, p~U(0.05,0.5))",
            "config": _config(args, m),
            "gpu_launches": launches,
            "kernel_ms_per_step": {k: _r(v, 4) for k, v in kern_ms.items()},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "kinship_s": kinship_s, "kinship_form": "int8 tcgen05 Gram + FP64 corrections",
            "kinship_fp64_s": kinship_fp64_s, "kinship_snps": int(keep.size),
            "kinship_int8_vs_fp64_max_rel_diff": kin_maxdiff, "eigh_s": eigh_s,
            "accuracy_detail": {"mixed_vs_fp64_form": acc_mixed_fp64,
                                "vs_oracle": acc_oracle},
            "serving": serving,
            "multi_phenotype": multi,
            "autotune": None if tuned is None else {
                "kernel": ["one CTA per tile", "CTA pairs (cta_group::2)"][tuned["kernel"]],
                "schedule": tuned["schedule"], "best_chunk": tuned["chunk"],
                "best_chunk_snps_per_s": _r(tuned["snps_per_s"], 4), "trials": len(tuned["trials"])},
            "hbm_peak_gbs": peaks.get("hbm_gbs", HBM_PEAK_FALLBACK),
            # ---- north-star evidence last (read from the end of the line)
            "kinship_phases": _kinship_phases(kin_events.get("int8"), n, int(keep.size), i8_measured),
            "accuracy_mixed_vs_fp64_form": dict(snps=m, **_accuracy_compact(acc_mixed_fp64)),
            "accuracy_vs_oracle": None if acc_oracle is None else {
                "snps": acc_oracle["snps"], "n": n,
                "key": "non-p: max rel; p: [max rel, frac <= 1e-6, max |dlog10 p|, calls differ 5e-8]",
                "mixed": _accuracy_compact(acc_oracle["mixed"]),
                "fp64": _accuracy_compact(acc_oracle["fp64"])},
            "fp64_form": {"value": _r(value64, 4), "unit": "SNPs/s", "steps": fp64_steps,
                          "kernel_ms_per_step": {k: _r(v, 4) for k, v in kern64.items()}},
            "speedup_mixed_vs_fp64": _r(value / value64, 4),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_serving_only(args) -> None:
    """The serving configuration alone (``--serve-c4``): one JSON line with its latency
    percentiles, phase split and aggregate throughput.

    Cohorts of 2 000 to 40 000 samples come and go, so the process keeps PyTorch's caching
    allocator from splitting blocks above 256 MB: with splitting, the freed multi-GB
    kinship and eigensolver buffers were cut up by later, smaller allocations until a 5 GB
    request failed with 91 GB cached but unallocated.  (Expandable segments avoided that
    but invalidated a concurrent chunk-graph capture.)"""
    os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "max_split_size_mb:256")
    import torch

    from jamma_b200 import _build

    torch.cuda.set_device(_dist()[2])
    _build.build()
    with ClockSampler(_dist()[2]) as clk:
        serving = run_serving(args)
    line = {"metric": "serving_p99_latency_s", "value": serving["p99_s"], "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "dtype": "int8+f64",
            "data": "synthetic (seeded device RNG; Binomial(2,p) genotypes, p~U(0.05,0.5))",
            "config": {"workload": serving["workload"]}, "clocks": clk.summary(),
            "serving": serving}
    print(json.dumps(line), flush=True)


def run_batched_cohort(args) -> None:
    """The batched configuration at its stated size (``--batched``): one cohort of
    n = 20 000 samples x 500 000 SNPs (1 % missing calls), INT8 kinship over every
    polymorphic SNP, one FP64 eigendecomposition, 64 phenotypes (h2 ~ U(0.1, 0.8), 50
    causal SNPs each with beta ~ N(0, 0.3^2), a polygenic term drawn from the kinship
    itself and N(0, 1) noise), all tests (-lmm 4, which includes Wald and LRT) in SNP
    chunks of 5 000 through the mixed form.  Packed records stay resident in HBM; each
    chunk is decoded, rotated and searched for all phenotypes, and its statistics are
    copied to pinned host memory on the same stream.  One JSON line: set-up times, the
    association's SNP-phenotype pairs/s (device events and host wall clock), the first
    chunk against the plain FP64 form, and the recovery of the causal SNPs at 5e-8."""
    import torch

    from jamma_b200 import _build, _native, engine as eng, synth
    from jamma_b200.device import ptr, stream_handle
    from jamma_b200.kinship import _KinshipI8, filter_mask, snp_stats_from_counts

    torch.cuda.set_device(_dist()[2])
    _build.build()
    n, p, phi, m = args.n, args.batched_snps, args.phenotypes, args.batched_chunk
    st = torch.cuda.current_stream()
    rec = synth.packed_records_device(n, p, args.miss, seed=20261203)
    bps = rec.shape[1]
    kc = 16384
    counts = np.concatenate([eng.decode_packed(rec[s:s + kc], n, None, n)[1].cpu().numpy()
                             for s in range(0, p, kc)])

    # ---- kinship (defaults maf 0, miss 1: every polymorphic SNP) and eigendecomposition
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    kin_mean, kin_miss, poly = snp_stats_from_counts(counts, n, np.float64)
    kin_idx = np.where(poly)[0]
    acc = _KinshipI8(n, kin_idx.size)
    for s in range(0, kin_idx.size, kc):
        sub = kin_idx[s:s + kc]
        codes_k, _ = eng.decode_packed(rec.index_select(0, torch.from_numpy(sub).cuda()), n, None, n)
        cc = counts[sub]
        mu = cc[:, 1] / np.maximum(cc[:, 0], 1)
        acc.add(codes_k, torch.from_numpy(mu).cuda(), bool(np.any(cc[:, 0] < n)),
                n_missing=int((n - cc[:, 0]).sum()))
        acc.add_sum_mu2(mu)
    del codes_k
    K = acc.finish()
    torch.cuda.synchronize()
    kinship_s = time.perf_counter() - t0
    del acc
    t0 = time.perf_counter()
    w, U = eng.eigh_device(K)
    torch.cuda.synchronize()
    eigh_s = time.perf_counter() - t0
    del K

    # ---- association SNP set (maf >= 0.01, miss <= 0.05) and the phenotypes
    mean32, miss, poly = snp_stats_from_counts(counts, n, np.float32)
    keep, _ = filter_mask(mean32, miss, poly, n, 0.01, 0.05)
    idx = np.where(keep)[0]
    pk = idx.size
    means_all = torch.from_numpy(mean32[idx].astype(np.float64)).cuda()
    rng = np.random.default_rng(20261203)
    h2 = rng.uniform(0.1, 0.8, phi)
    causal = np.stack([rng.choice(pk, 50, replace=False) for _ in range(phi)])
    beta = rng.normal(0.0, 0.3, (phi, 50))
    cu = np.unique(causal)
    ccodes, _ = eng.decode_packed(rec.index_select(0, torch.from_numpy(idx[cu]).cuda()), n, None, n)
    xc = ccodes[:, :n].to(torch.float64)
    mu_c = means_all[torch.from_numpy(cu).cuda()][:, None]
    xc = torch.where(ccodes[:, :n] == 3, mu_c, xc) - mu_c  # imputed, centred (|cu|, n)
    pos = {int(j): r for r, j in enumerate(cu)}
    B = torch.zeros((cu.size, phi), dtype=torch.float64, device="cuda")
    for f in range(phi):
        for j, b in zip(causal[f], beta[f]):
            B[pos[int(j)], f] += b
    fixed = xc.t() @ B                                            # (n, phi)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(20261204)
    xi = torch.randn((n, phi), generator=gen, dtype=torch.float64, device="cuda")
    g = U.t() @ (w.clamp_min(0).sqrt()[:, None] * xi)             # polygenic ~ N(0, K)
    g *= torch.from_numpy(np.sqrt(h2 / (1 - h2))).cuda() / g.std(0)
    Y = (fixed + g + torch.randn((n, phi), generator=gen, dtype=torch.float64, device="cuda"))
    Y = Y.cpu().numpy()
    del xc, ccodes, fixed, g, xi

    t0 = time.perf_counter()
    coh = eng.DeviceCohort(w, U, None, Y, lmm_mode=4, precision="mixed")
    torch.cuda.synchronize()
    cohort_s = time.perf_counter() - t0
    ld = (n + 127) // 128 * 128
    codes = torch.empty((m, ld), dtype=torch.int8, device="cuda")
    cnt = torch.empty((m, 4), dtype=torch.int32, device="cuda")
    UtG = eng.empty((m, n))
    outs = coh.alloc_out(m)
    n_chunks = (pk + m - 1) // m
    host = {k: torch.empty((n_chunks, phi, m), dtype=torch.float64, pin_memory=True) for k in outs}
    idx_dev = torch.from_numpy(idx).cuda()
    rec_kept = rec if pk == p else rec.index_select(0, idx_dev)
    del rec
    has_missing = args.miss > 0

    m_last = pk - (n_chunks - 1) * m
    outs_last = outs if m_last == m else coh.alloc_out(m_last)

    def chunk(ci: int, dst: dict | None) -> None:
        s = ci * m
        e = min(pk, s + m)
        mc = e - s
        o = outs if mc == m else outs_last
        _native.call("jb_decode_bed", ptr(rec_kept[s:e]), bps, mc, None, n, ptr(codes), ld, ptr(cnt),
                     stream_handle())
        coh.associate_rotated(coh.rotate_codes_i8(codes[:mc], means_all[s:e], has_missing,
                                                  out=UtG[:mc]), o)
        if dst is not None:  # stream-ordered: the next chunk's kernels queue after the copies
            for k, v in o.items():
                dst[k][ci, :, :mc].copy_(v, non_blocking=True)

    # warm-up: the first chunk once (module loads, workspaces)
    chunk(0, None)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(_dist()[2]) as clk:
        t0 = time.perf_counter()
        a.record(st)
        for ci in range(n_chunks):
            chunk(ci, host)
        b.record(st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    dev_s = a.elapsed_time(b) / 1e3
    if status := coh.rotate_status():
        raise RuntimeError(f"INT8 rotation pipeline status {status}")
    res = {k: v.numpy().transpose(1, 0, 2).reshape(phi, -1)[:, :pk] for k, v in host.items()}

    # ---- first chunk against the plain FP64 form (same records, eigendecomposition, phenotypes)
    coh64 = eng.DeviceCohort(w, U, None, Y, lmm_mode=4, precision="fp64")
    G = eng.empty((m, n))
    mc = min(m, pk)
    _native.call("jb_decode_bed", ptr(rec_kept[:mc]), bps, mc, None, n, ptr(codes), ld, ptr(cnt),
                 stream_handle())
    _native.call("jb_impute_f64", ptr(codes), ld, n, mc, ptr(means_all[:mc]), ptr(G), n, stream_handle())
    o64 = coh64.associate_rotated(eng.rotate(coh64.U, G[:mc], out=UtG[:mc]))
    ref = {k: v.cpu().numpy() for k, v in o64.items()}
    got = {k: v[:, :mc] for k, v in res.items()}
    acc64 = _accuracy_compact(_accuracy(got, ref))

    # ---- recovery of the causal SNPs at 5e-8 (Wald), and hits elsewhere
    pw = res["p_wald"]
    cmask = np.zeros((phi, pk), dtype=bool)
    for f in range(phi):
        cmask[f, causal[f]] = True
    hits = pw < 5e-8
    line = {
        "metric": "batched_snp_phenotype_pairs_per_s", "value": _r(pk * phi / dev_s, 4),
        "unit": "SNP-phenotype pairs/s", "higher_is_better": True, "n_gpus": 1, "dtype": "int8+f64",
        "data": "synthetic (seeded; Binomial(2,p) genotypes, p~U(0.05,0.5), 1% missing; phenotypes "
                "with 50 causal SNPs, beta~N(0,0.3^2), polygenic ~ N(0, K), h2~U(0.1,0.8))",
        "config": {"workload": f"one cohort n={n} x {p} SNPs ({pk} tested), {phi} phenotypes, -lmm 4 "
                               f"(Wald + LRT + Score), SNP chunk {m}, records resident in HBM",
                   "n_samples": n, "snps": p, "snps_tested": int(pk), "phenotypes": phi,
                   "chunk": m, "kinship_snps": int(kin_idx.size)},
        "kinship_s": _r(kinship_s, 4), "eigh_s": _r(eigh_s, 4), "cohort_setup_s": _r(cohort_s, 4),
        "association_device_s": _r(dev_s, 4), "association_wall_s": _r(wall, 4),
        "wall_pairs_per_s": _r(pk * phi / wall, 4), "snps_per_s_all_phenotypes": _r(pk / dev_s, 4),
        "chunks": n_chunks, "clocks": clk.summary(),
        "causal_found_5e-8": int(np.sum(hits & cmask)), "causal_total": int(cmask.sum()),
        "noncausal_hits_5e-8": int(np.sum(hits & ~cmask)),
        "accuracy_first_chunk_vs_fp64_form": dict(snps=int(mc), phenotypes=phi, **acc64),
    }
    print(json.dumps(line), flush=True)


def run_loco(args) -> None:
    """LOCO at config C5's shape (n samples, `--loco-chromosomes` x `--loco-snps` SNPs):
    the INT8 LOCO kinships at full size (one full-genome Gram and one Gram per chromosome,
    every K_loco formed), one LOCO eigendecomposition, and mixed-form Wald throughput with
    that chromosome's eigenvectors; the whole run's time is extrapolated with one
    eigendecomposition per chromosome.  Synthetic device-resident records stand in for the
    .bed file (1 % missing calls), so no file I/O is timed.  Prints one JSON line."""
    import torch

    from jamma_b200 import _native, engine as eng, synth
    from jamma_b200.device import empty, ptr, stream_handle
    from jamma_b200.kinship import _KinshipI8, snp_stats_from_counts

    n, n_chr, per, m = args.n, args.loco_chromosomes, args.loco_snps, args.chunk
    p = n_chr * per
    rec = synth.packed_records_device(n, p, args.miss, seed=500)
    kc = 16384
    counts = np.concatenate([eng.decode_packed(rec[s:s + kc], n, None, n)[1].cpu().numpy()
                             for s in range(0, p, kc)])
    keep = np.where(snp_stats_from_counts(counts, n)[2])[0]
    chrom = keep // per

    def accumulate(sub: np.ndarray) -> _KinshipI8:
        acc = _KinshipI8(n, sub.size)
        for s in range(0, sub.size, kc):
            part = sub[s:s + kc]
            codes, _ = eng.decode_packed(rec.index_select(0, torch.from_numpy(part).cuda()), n, None, n)
            c = counts[part]
            mu = c[:, 1] / np.maximum(c[:, 0], 1)
            acc.add(codes, torch.from_numpy(mu).cuda(), bool(np.any(c[:, 0] < n)),
                    n_missing=int((n - c[:, 0]).sum()))
            acc.add_sum_mu2(mu)
        return acc

    accumulate(keep[:kc]).finish()  # one-time costs (module loads) outside the timed region
    torch.cuda.synchronize()
    t = time.perf_counter()
    full = accumulate(keep)
    C_full = full.gram()
    torch.cuda.synchronize()
    full_s = time.perf_counter() - t
    st = stream_handle()
    K = empty((n, n))
    chr_s = []
    for ci in range(n_chr):
        t = time.perf_counter()
        part = accumulate(keep[chrom == ci])
        C_c = part.gram()
        q_full, q_c = full.RT, part.RT
        if (q_full is None) != (q_c is None):
            if q_full is None:
                full.RT = q_full = torch.zeros_like(q_c)
            else:
                q_c = torch.zeros_like(q_full)
        _native.call("jb_kinship_i8_finalize_loco", ptr(C_full), ptr(C_c), n, n, ptr(full.a),
                     ptr(part.a), ptr(full.b), ptr(part.b), full.sum_mu2 - part.sum_mu2,
                     ptr(q_full), ptr(q_c), n, keep.size - int((chrom == ci).sum()), ptr(K), n, st)
        del part, C_c, q_c
        torch.cuda.synchronize()
        chr_s.append(time.perf_counter() - t)
    del full, C_full, q_full
    torch.cuda.empty_cache()
    t = time.perf_counter()
    w, U = eng.eigh_device(K)  # the last chromosome's K_loco
    torch.cuda.synchronize()
    eigh_s = time.perf_counter() - t
    rng = np.random.default_rng(5)
    cohort = eng.DeviceCohort(w, U, np.ones((n, 1)), rng.normal(size=n), lmm_mode=1,
                              precision="mixed")
    del K, U
    torch.cuda.empty_cache()
    bps = (n + 3) // 4
    ld = (n + 127) // 128 * 128
    codes = torch.empty((m, ld), dtype=torch.int8, device="cuda")
    cnt = torch.empty((m, 4), dtype=torch.int32, device="cuda")
    UtG = eng.empty((m, n))
    outs = cohort.alloc_out(m)
    means = [torch.from_numpy((counts[s * m:(s + 1) * m, 1] / np.maximum(counts[s * m:(s + 1) * m, 0], 1))
                              .astype(np.float32).astype(np.float64)).cuda()
             for s in range(args.warmup + args.steps)]

    def step(s):
        _native.call("jb_decode_bed", ptr(rec[s * m:(s + 1) * m]), bps, m, None, n, ptr(codes), ld,
                     ptr(cnt), stream_handle())
        cohort.rotate_codes_i8(codes, means[s], args.miss > 0, out=UtG)
        cohort.associate_rotated(UtG, outs)

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(torch.cuda.current_stream())
    for s in range(args.warmup, args.warmup + args.steps):
        step(s)
    b.record(torch.cuda.current_stream())
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    if cohort.rotate_status():
        raise RuntimeError("INT8 rotation pipeline reported a timeout")
    wald = args.steps * m / (ms / 1e3)
    kin_s = full_s + sum(chr_s)
    line = {
        "metric": "loco_run_s_extrapolated", "value": kin_s + n_chr * eigh_s + keep.size / wald,
        "unit": "s", "higher_is_better": False, "n_gpus": 1, "dtype": "int8+f64",
        "data": "synthetic (seeded device RNG; Binomial(2,p) genotypes, p~U(0.05,0.5))",
        "config": {"workload": f"LOCO -lmm 1 n={n}, {n_chr} chromosomes x {per} SNPs, "
                               f"{args.miss:.0%} missing calls", "n_samples": n,
                   "snps": int(keep.size), "chromosomes": n_chr, "chunk": m},
        "loco_kinship_s": kin_s, "kinship_full_genome_s": full_s,
        "kinship_per_chromosome_s": {"mean": float(np.mean(chr_s)), "max": float(np.max(chr_s))},
        "eigh_s_one_chromosome": eigh_s, "wald_snps_per_s": wald,
        "extrapolation": "loco_kinship_s + chromosomes x eigh_s_one_chromosome + SNPs / "
                         "wald_snps_per_s (every chromosome's eigendecomposition costs the same)",
    }
    print(json.dumps(line), flush=True)



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=20000)
    ap.add_argument("--n-cvt", type=int, default=1)
    ap.add_argument("--mode", type=int, default=4)
    ap.add_argument("--chunk", type=int, default=8192)
    ap.add_argument("--miss", type=float, default=0.01)
    ap.add_argument("--kin-snps", type=int, default=500000)
    ap.add_argument("--skip-fp64-kinship", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--int8-peak-tops", type=float, default=4500.0)
    ap.add_argument("--int8-peak-source", default="nominal B200 dense INT8 (4.5 POP/s); "
                    "MEASURED_PEAKS.json has no INT8 figure")
    ap.add_argument("--oracle-snps", type=int, default=64,
                    help="SNPs of a timed chunk checked against the CPU oracle (also the CPU baseline)")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end run through run_lmm_association_streaming")
    ap.add_argument("--ref-snps", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-jobs", type=int, default=24)
    ap.add_argument("--serve-gap", type=float, default=0.2)
    ap.add_argument("--serve-budget-gb", type=float, default=60.0)
    ap.add_argument("--serve-c4", action="store_true",
                    help="serve the full serving configuration (200 jobs, n up to 40 000, SNPs up "
                         "to 200 000) and print only the serving summary")
    ap.add_argument("--phenotypes", type=int, default=64,
                    help="phenotypes of the multi-phenotype sub-measurement (1 = skip)")
    ap.add_argument("--pheno-chunk", type=int, default=2048)
    ap.add_argument("--pheno-mode", type=int, default=4)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--traffic-sweep", action="store_true",
                    help="after the timed steps, one rotation per candidate tile schedule (one-CTA "
                         "kernel) as the profiler range, for ncu's DRAM byte counts")
    ap.add_argument("--profile-phase", choices=["assoc", "kinship", "multi", "none"], default="assoc",
                    help="which phase torch.cuda.profiler.start/stop brackets")
    ap.add_argument("--rot-kernel", type=int, choices=[0, 1], default=None,
                    help="fix the INT8 rotation kernel (0 one CTA per tile, 1 CTA pairs)")
    ap.add_argument("--loco", action="store_true",
                    help="measure LOCO at config C5's shape instead (use --n 50000)")
    ap.add_argument("--loco-chromosomes", type=int, default=20)
    ap.add_argument("--loco-snps", type=int, default=50000, help="SNPs per chromosome")
    ap.add_argument("--batched", action="store_true",
                    help="measure the batched configuration at its stated size instead (one cohort "
                         "of n x --batched-snps SNPs, --phenotypes phenotypes, -lmm 4)")
    ap.add_argument("--batched-snps", type=int, default=500000)
    ap.add_argument("--batched-chunk", type=int, default=5000)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.serve_c4:
        run_serving_only(args)
    elif args.loco:
        run_loco(args)
    elif args.batched:
        run_batched_cohort(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
