"""Autotuner for the association hot path: SNP chunk width and rotation tile schedule.

Two knobs set how fast one cohort's SNP chunks go through the device:

* the chunk width m (SNPs per launch sequence): larger chunks amortise launches and fill
  the 148 SMs' persistent tiles evenly, but hold n*m*8 bytes of rotated genotypes and
  more workspace, and delay the first results;
* the INT8 rotation kernel: one CTA per output tile or CTA pairs sharing a 256-row tile
  (``jb_rotate_set_kernel``), and its tile-group shape (``jb_rotate_set_schedule``): which
  operand slices the persistent CTAs share in L2.

``tune(cohort)`` times real chunks of the given cohort on synthetic calls of its shape
(CUDA events, warm-up excluded) over the candidates that fit the memory budget, applies
the best schedule and returns the best chunk width.  Results are cached per GPU model and
problem shape in a JSON file (``$JAMMA_B200_CACHE`` or ``~/.cache/jamma_b200/autotune.json``)
guarded by a process-wide lock, so a shape is measured once per machine.
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path

import numpy as np
import torch

from jamma_b200 import _native
from jamma_b200.device import require_cuda

CHUNKS = (2048, 4096, 8192, 16384)
SCHEDULES = ((9, 16), (5, 32), (17, 8), (3, 64), (36, 4))
KERNELS = (0, 1)  # one CTA per tile, CTA pairs
_lock = threading.Lock()


def cache_path() -> Path:
    p = os.environ.get("JAMMA_B200_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "jamma_b200" / "autotune.json"


def _key(cohort, gpu: str) -> str:
    return f"{gpu}|n={cohort.n}|c={cohort.c}|phi={cohort.phi}|mode={cohort.mode}|{cohort.precision}"


def _load() -> dict:
    p = cache_path()
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return {}


def _store(entries: dict) -> None:
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(entries, indent=1, sort_keys=True))
    tmp.replace(p)


def set_schedule(group_m: int, group_n: int) -> None:
    _native.call("jb_rotate_set_schedule", int(group_m), int(group_n))


def set_kernel(variant: int) -> None:
    _native.call("jb_rotate_set_kernel", int(variant))


def get_kernel() -> int:
    return int(_native.load().jb_rotate_get_kernel())


def get_schedule() -> tuple[int, int]:
    a = np.zeros(2, dtype=np.int32)
    _native.call("jb_rotate_get_schedule", a.ctypes.data, a.ctypes.data + 4)
    return int(a[0]), int(a[1])


def chunk_bytes(cohort, m: int) -> int:
    """Device bytes one chunk of width m holds beyond the cohort's resident state."""
    lib = _native.load()
    n = cohort.n
    b = lib.jb_lmm_chunk_workspace_size(n, cohort.c, cohort.phi, cohort.n_grid, m)
    b += m * n * 8 + m * cohort.code_ld + 9 * cohort.phi * m * 8  # rotated chunk, codes, out
    if cohort.precision == "mixed":
        b += lib.jb_rotate_i8_workspace_size(n, m)
    else:
        b += m * n * 8  # imputed FP64 chunk
    return int(b)


def _synthetic_chunk(n: int, m: int, ld: int, seed: int = 0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    p = torch.rand((m, 1), generator=g, device="cuda") * 0.45 + 0.05
    u = torch.rand((m, n), generator=g, device="cuda")
    calls = (u < p * p).to(torch.int8) + (u < 2 * p - p * p).to(torch.int8)  # Binomial(2, p)
    calls[torch.rand((m, n), generator=g, device="cuda") < 0.01] = 3
    codes = torch.zeros((m, ld), dtype=torch.int8, device="cuda")
    codes[:, :n] = calls
    obs = (calls != 3)
    means = (calls.where(obs, torch.zeros_like(calls)).double().sum(1)
             / obs.sum(1).clamp(min=1).double()).float().double()
    return codes.contiguous(), means.contiguous()


def _time_chunk(cohort, codes, means, reps: int = 3) -> float:
    """Mean ms of one chunk (rotation + series + search) after one warm-up run."""
    out = cohort.alloc_out(codes.shape[0])
    bufs = {"UtG": torch.empty((codes.shape[0], cohort.n), dtype=torch.float64, device="cuda")}
    cohort.associate_codes(codes, means, out=out, bufs=bufs, has_missing=True)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        cohort.associate_codes(codes, means, out=out, bufs=bufs, has_missing=True)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune(cohort, memory_budget: int | None = None, chunks=CHUNKS, schedules=SCHEDULES,
         kernels=KERNELS, use_cache: bool = True, reps: int = 3) -> dict:
    """Pick the chunk width, rotation kernel and schedule for ``cohort``; returns
    {"chunk": m, "kernel": k, "schedule": [gm, gn], "snps_per_s": best, "trials": [...]}
    and applies kernel and schedule.  ``memory_budget`` caps the per-chunk device bytes
    (default: half of the free device memory)."""
    require_cuda()
    gpu = torch.cuda.get_device_name()
    key = _key(cohort, gpu)
    with _lock:
        if use_cache:
            hit = _load().get(key)
            if hit is not None:
                set_kernel(hit.get("kernel", 0))
                set_schedule(*hit["schedule"])
                return hit
        if memory_budget is None:
            memory_budget = torch.cuda.mem_get_info()[0] // 2
        fits = [m for m in chunks if chunk_bytes(cohort, m) <= memory_budget] or [min(chunks)]
        trials = []
        m_big = max(fits)
        codes, means = _synthetic_chunk(cohort.n, m_big, cohort.code_ld)
        best_sched, best_kernel, best_t = None, None, None
        if cohort.precision == "mixed":  # kernel + schedule first, at the largest chunk that fits
            for kern in kernels:
                set_kernel(kern)
                for sched in schedules:
                    set_schedule(*sched)
                    t = _time_chunk(cohort, codes, means, reps)
                    trials.append({"chunk": m_big, "kernel": kern, "schedule": list(sched), "ms": t})
                    if best_t is None or t < best_t:
                        best_sched, best_kernel, best_t = sched, kern, t
            set_kernel(best_kernel)
            set_schedule(*best_sched)
        else:
            best_sched, best_kernel = get_schedule(), get_kernel()
        best_m, best_rate = None, -1.0
        for m in fits:
            t = _time_chunk(cohort, codes[:m], means[:m], reps)
            trials.append({"chunk": m, "kernel": best_kernel, "schedule": list(best_sched), "ms": t})
            rate = m / (t / 1e3)
            if rate > best_rate:
                best_m, best_rate = m, rate
        res = {"chunk": int(best_m), "kernel": int(best_kernel), "schedule": list(best_sched),
               "snps_per_s": best_rate, "trials": trials, "gpu": gpu}
        if use_cache:
            entries = _load()
            entries[key] = res
            _store(entries)
        return res
