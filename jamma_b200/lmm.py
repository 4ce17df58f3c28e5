"""LMM association runners with jamma's API (``run_lmm_association_streaming`` and
``run_lmm_association_jax``), executed on the GPU through libjamma_b200.

Host responsibilities are the ones jamma's runners keep on the host: sample and SNP
masks, the order of results, and text output.  Genotype decoding, imputation,
rotation, the null model, the lambda searches and all statistics run on the device.
"""

from __future__ import annotations

import time
from pathlib import Path

import numpy as np
import torch

from jamma_b200 import engine as eng
from jamma_b200.device import require_cuda
from jamma_b200.eigen import eigendecompose_kinship_device
from jamma_b200.io import (
    MODE_TEST,
    AssocResult,
    BedFile,
    IncrementalAssocWriter,
    apply_snp_list_mask,
    format_assoc_line,
    get_plink_metadata,
    pack_genotypes,
    snp_info_from_meta,
)
from jamma_b200.kinship import filter_mask, snp_stats_from_counts

_FIELD = {  # engine output key -> AssocResult field
    "lambda_remle": "l_remle",
    "logl_h1": "logl_H1",
    "beta": "beta",
    "se": "se",
    "p_wald": "p_wald",
    "lambda_mle": "l_mle",
    "p_lrt": "p_lrt",
    "p_score": "p_score",
}


def device_chunk_for(n: int, budget_bytes: float = 4e9, cap: int = 8192) -> int:
    """SNPs per device chunk: imputed + rotated FP64 columns (16 n bytes / SNP) in budget."""
    return int(max(256, min(cap, budget_bytes // (16 * max(n, 1)))))


def valid_sample_mask(phenotypes: np.ndarray, covariates: np.ndarray | None) -> np.ndarray:
    """``~isnan(y) & y != -9 & covariates complete`` (runner_streaming.py:188-198)."""
    y = np.asarray(phenotypes, dtype=np.float64)
    if y.ndim == 2:
        mask = np.all(~np.isnan(y) & (y != -9.0), axis=1)
    else:
        mask = ~np.isnan(y) & (y != -9.0)
    if covariates is not None:
        mask &= np.all(~np.isnan(np.asarray(covariates, dtype=np.float64)), axis=1)
    return mask


def hwe_pvalues(n_aa, n_ab, n_bb) -> np.ndarray:
    """Chi-square (df 1) HWE p-values (``compute_hwe_pvalues``, core/snp_filter.py:94-150)."""
    from math import erfc, sqrt

    n_aa, n_ab, n_bb = (np.asarray(v, dtype=np.float64) for v in (n_aa, n_ab, n_bb))
    n = n_aa + n_ab + n_bb
    with np.errstate(invalid="ignore", divide="ignore"):
        p = (2 * n_aa + n_ab) / (2 * n)
        q = 1.0 - p
        e_aa, e_ab, e_bb = n * p**2, 2 * n * p * q, n * q**2
        chi = (n_aa - e_aa) ** 2 / e_aa + (n_ab - e_ab) ** 2 / e_ab + (n_bb - e_bb) ** 2 / e_bb
    chi = np.where(np.isnan(chi), 0.0, chi)
    return np.array([erfc(sqrt(max(c, 0.0) / 2.0)) for c in chi])


class _Stats:
    """Per-SNP pass-1 statistics and the filter for one analysed sample set."""

    def __init__(self, counts: np.ndarray, n: int, mean_dtype, maf, miss, snps_indices=None,
                 hwe_threshold: float = 0.0):
        self.counts = counts
        self.mean, self.miss, poly = snp_stats_from_counts(counts, n, mean_dtype)
        keep, self.af = filter_mask(self.mean, self.miss, poly, n, maf, miss)
        if snps_indices is not None:
            apply_snp_list_mask(keep, snps_indices, keep.size, "SNP list filter")
        if hwe_threshold > 0:
            hom0 = counts[:, 0] - counts[:, 2] - counts[:, 3]
            keep &= hwe_pvalues(hom0, counts[:, 2], counts[:, 3]) >= hwe_threshold
        self.idx = np.where(keep)[0]


_ORDER = ("beta", "se", "logl_H1", "l_remle", "p_wald", "p_score", "l_mle", "p_lrt")


def _build_results(mode: int, snp_idx, af, n_miss, snp_info, arrays, f: int = 0):
    """One AssocResult per tested SNP (``_build_results_*``, src/jamma/lmm/results.py:37-286).

    Built column-wise: each AssocResult field is one list over the SNPs, and the records
    are made positionally from their zip (mode 2 has no beta/se: NaN; other absent
    statistics are None)."""
    idx = np.asarray(snp_idx).tolist()
    k = len(idx)
    info = [snp_info[j] for j in idx]
    nan = float("nan")
    stats = {field: arrays[key][f].tolist() for key, field in _FIELD.items()
             if key in arrays and not (mode == 2 and field in ("beta", "se"))}
    cols = [
        [s["chr"] for s in info],
        [s["rs"] for s in info],
        [s.get("pos", s.get("ps", 0)) for s in info],
        np.asarray(n_miss).astype(int).tolist(),
        [s.get("a1", s.get("allele1", "")) for s in info],
        [s.get("a0", s.get("allele0", "")) for s in info],
        np.asarray(af, dtype=np.float64).tolist(),
    ]
    for field in _ORDER:
        cols.append(stats[field] if field in stats else
                    [nan] * k if field in ("beta", "se") else [None] * k)
    return [AssocResult(*row) for row in zip(*cols)]


def associate_records(cohort: eng.DeviceCohort, records, n_file: int, sample_idx, means: np.ndarray,
                      device_chunk: int | None = None, on_chunk=None,
                      n_miss: np.ndarray | None = None) -> dict[str, np.ndarray]:
    """Run the association for packed .bed records (m, bytes_per_snp) of kept SNPs.

    ``records`` is a host uint8 array, or a callable ``records(s, e, out)`` that writes
    rows s..e into the (e - s, bytes_per_snp) uint8 array ``out``; ``means`` are the
    per-SNP imputation values.  Returns (phi, m) arrays.

    The chunks stream through the device as the device loop of
    src/jamma/lmm/runner_streaming.py:412-586 does, with every stage overlapped:

    * the chunk's whole device pipeline (decode, rotation, series sums, search and
      statistics) is captured once as a CUDA graph (:class:`engine.ChunkGraph`) and
      replayed per chunk on the caller's stream;
    * the host reads chunk k+1's records into one of two pinned buffers while the GPU
      replays chunk k, and their host-to-device copy runs on a side stream into one of two
      device staging buffers; the replay stream takes the staged chunk with one
      device-to-device copy into the graph's input buffers;
    * results return by asynchronous copies into pinned buffers and are collected on the
      host one chunk behind, so the GPU always has the next chunk queued.
    """
    m = len(means)
    res = {k: np.empty((cohort.phi, m)) for k in eng.MODE_KEYS[cohort.mode]}
    if m == 0:
        return res
    step = min(int(device_chunk or device_chunk_for(cohort.n)), m)
    bps = (n_file + 3) // 4
    sidx = None if sample_idx is None else torch.from_numpy(
        np.asarray(sample_idx, dtype=np.int32)).to("cuda")
    means = np.asarray(means, dtype=np.float64)
    has_missing = True if n_miss is None else bool(np.any(np.asarray(n_miss) > 0))
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream()
    pin_rec = [torch.empty((step, bps), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    pin_mu = [torch.empty((step,), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    dev_rec = [torch.empty((step, bps), dtype=torch.uint8, device="cuda") for _ in range(2)]
    dev_mu = [torch.empty((step,), dtype=torch.float64, device="cuda") for _ in range(2)]
    copied = [None, None]    # pinned buffer b read, staging buffer b filled
    consumed = [None, None]  # replay stream: staging buffer b copied into the graph inputs
    returned = [None, None]  # replay stream: results of the chunk in buffer b are in pin_out[b]

    def fill(b: int, s: int, e: int) -> None:
        if callable(records):
            records(s, e, pin_rec[b].numpy()[: e - s])
        else:
            pin_rec[b].numpy()[: e - s] = records[s:e]
        pin_mu[b].numpy()[: e - s] = means[s:e]

    def first_chunk(g: eng.ChunkGraph) -> None:
        # the graph's eager warm-up run computes chunk 0
        fill(0, 0, step)
        g.packed.copy_(pin_rec[0], non_blocking=True)
        g.means.copy_(pin_mu[0], non_blocking=True)

    graph = eng.ChunkGraph(cohort, step, n_file, sidx, has_missing=has_missing,
                           prefill=first_chunk)
    pin_out = [{k: torch.empty((cohort.phi, step), dtype=torch.float64, pin_memory=True)
                for k in graph.out} for _ in range(2)]

    def collect(b: int, s: int, e: int) -> None:
        returned[b].synchronize()
        for k, v in pin_out[b].items():
            res[k][:, s:e] = v[:, : e - s].numpy()
        if on_chunk is not None:
            on_chunk(s, e)

    def send_back(b: int, rows: int) -> None:
        for k, v in graph.out.items():
            pin_out[b][k][:, :rows].copy_(v[:, :rows], non_blocking=True)
        returned[b] = torch.cuda.Event()
        returned[b].record(main)

    copied[0] = torch.cuda.Event()
    copied[0].record(main)  # the constructor's copies from pin_rec[0] precede this
    send_back(0, step)
    pending = (0, 0, step)
    for ci, s in enumerate(range(step, m, step), start=1):
        e = min(s + step, m)
        b, rows = ci % 2, e - s
        if copied[b] is not None:
            copied[b].synchronize()  # chunk ci-2's upload has read pin_rec[b]
        fill(b, s, e)
        with torch.cuda.stream(side):
            if consumed[b] is not None:
                side.wait_event(consumed[b])
            dev_rec[b][:rows].copy_(pin_rec[b][:rows], non_blocking=True)
            dev_mu[b][:rows].copy_(pin_mu[b][:rows], non_blocking=True)
            copied[b] = torch.cuda.Event()
            copied[b].record(side)
        main.wait_event(copied[b])
        graph.packed[:rows].copy_(dev_rec[b][:rows], non_blocking=True)
        graph.means[:rows].copy_(dev_mu[b][:rows], non_blocking=True)
        consumed[b] = torch.cuda.Event()
        consumed[b].record(main)
        graph.replay()
        send_back(b, rows)
        collect(*pending)
        pending = (b, s, e)
    collect(*pending)
    if cohort.precision == "mixed" and (status := cohort.rotate_status()):
        raise RuntimeError(f"INT8 rotation pipeline reported status {status} (a bounded "
                           "tensor-core pipeline wait ran out)")
    return res


def _prepare_cohort(kinship, eigenvalues, eigenvectors, covariates, y, lmm_mode, l_min, l_max,
                    n_grid, n_refine, precision="fp64"):
    if eigenvalues is not None:
        evals, U = eigenvalues, eigenvectors
    else:
        K = torch.from_numpy(np.ascontiguousarray(np.asarray(kinship, dtype=np.float64))).to("cuda")
        evals, U = eigendecompose_kinship_device(K)
    return eng.DeviceCohort(evals, U, covariates, y, lmm_mode, l_min, l_max, n_grid, n_refine,
                            precision=precision)


def run_lmm_association_streaming(
    bed_path, phenotypes: np.ndarray, kinship: np.ndarray | None = None, snp_info: list | None = None,
    covariates: np.ndarray | None = None, eigenvalues: np.ndarray | None = None,
    eigenvectors: np.ndarray | None = None, maf_threshold: float = 0.01, miss_threshold: float = 0.05,
    l_min: float = 1e-5, l_max: float = 1e5, n_grid: int = 50, n_refine: int = 10,
    chunk_size: int = 10_000, use_gpu: bool = True, check_memory: bool = True,
    show_progress: bool = True, output_path: Path | None = None, lmm_mode: int = 1,
    snps_indices: np.ndarray | None = None, hwe_threshold: float = 0.0,
    validate_genotypes: bool = True, timing: dict | None = None, precision: str = "fp64",
) -> list[AssocResult]:
    """Two-pass streaming association from a PLINK prefix (runner_streaming.py:94-628).

    ``use_gpu`` is accepted for signature compatibility: the computation always runs on
    the GPU.  ``timing`` (optional dict) receives per-stage seconds.
    """
    t0 = time.perf_counter()
    if (eigenvalues is None) != (eigenvectors is None):
        raise ValueError(
            "Must provide both eigenvalues and eigenvectors, or neither. "
            f"Got eigenvalues={eigenvalues is not None}, eigenvectors={eigenvectors is not None}"
        )
    if kinship is None and eigenvalues is None:
        raise ValueError("Either kinship or pre-computed eigendecomposition (eigenvalues + "
                         "eigenvectors) must be provided")
    if lmm_mode not in (1, 2, 3, 4):
        raise ValueError(f"lmm_mode must be 1, 2, 3 or 4, got {lmm_mode}")
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
    meta = get_plink_metadata(bed_path)
    require_cuda()  # after the argument checks, so they raise as jamma's do on any host
    n_file, p = meta["n_samples"], meta["n_snps"]
    if snp_info is None:
        snp_info = snp_info_from_meta(meta)
    y = np.asarray(phenotypes, dtype=np.float64)
    valid = valid_sample_mask(y, covariates)
    sample_idx = None if np.all(valid) else np.where(valid)[0].astype(np.int32)
    y = y[valid]
    cov = None if covariates is None else np.asarray(covariates, dtype=np.float64)[valid]
    if kinship is not None and sample_idx is not None:
        kinship = np.asarray(kinship)[np.ix_(valid, valid)]
    n = y.shape[0]
    bed = BedFile(bed_path, n_file, p)

    # pass 1: per-SNP counts on the device (float32 means, as jamma's streaming path)
    sidx = None if sample_idx is None else torch.from_numpy(sample_idx).to("cuda")
    counts = eng.pass1_counts(bed, sidx, n, max(chunk_size, 16384))
    st = _Stats(counts, n, np.float32, maf_threshold, miss_threshold, snps_indices, hwe_threshold)
    t1 = time.perf_counter()
    if st.idx.size == 0:
        return []

    cohort = _prepare_cohort(kinship, eigenvalues, eigenvectors, cov, y, lmm_mode, l_min, l_max,
                             n_grid, n_refine, precision)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    res = associate_records(cohort, lambda a, b, out: bed.take_into(st.idx[a:b], out), n_file,
                            sample_idx,
                            st.mean[st.idx].astype(np.float64), n_miss=st.miss[st.idx])
    t3 = time.perf_counter()
    results = _build_results(lmm_mode, st.idx, st.af[st.idx], st.miss[st.idx], snp_info, res)
    if output_path is not None:
        with IncrementalAssocWriter(output_path, MODE_TEST[lmm_mode]) as w:
            w.write_lines([format_assoc_line(r, MODE_TEST[lmm_mode]) for r in results])
        results = []
    if timing is not None:
        timing.update(stats_s=t1 - t0, setup_s=t2 - t1, association_s=t3 - t2,
                      write_s=time.perf_counter() - t3, n_tested=int(st.idx.size))
    return results


def run_lmm_association_jax(
    genotypes: np.ndarray, phenotypes: np.ndarray, kinship: np.ndarray, snp_info: list,
    covariates: np.ndarray | None = None, eigenvalues: np.ndarray | None = None,
    eigenvectors: np.ndarray | None = None, maf_threshold: float = 0.01,
    miss_threshold: float = 0.05, l_min: float = 1e-5, l_max: float = 1e5, n_grid: int = 50,
    n_refine: int = 10, use_gpu: bool = True, check_memory: bool = True,
    show_progress: bool = True, lmm_mode: int = 1, precision: str = "fp64",
) -> list[AssocResult]:
    """In-memory genotype runner (runner_jax.py:52-481): statistics and imputation means
    in the genotype array's own dtype (float64 means for float64 input)."""
    if (eigenvalues is None) != (eigenvectors is None):
        raise ValueError("Must provide both eigenvalues and eigenvectors, or neither.")
    if lmm_mode not in (1, 2, 3, 4):
        raise ValueError(f"lmm_mode must be 1, 2, 3 or 4, got {lmm_mode}")
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
    require_cuda()
    g = np.asarray(genotypes)
    y = np.asarray(phenotypes, dtype=np.float64)
    valid = valid_sample_mask(y, covariates)
    if not np.all(valid):
        g = g[valid]
        y = y[valid]
        if kinship is not None:
            kinship = np.asarray(kinship)[np.ix_(valid, valid)]
        if covariates is not None:
            covariates = np.asarray(covariates)[valid]
    n = y.shape[0]
    packed = pack_genotypes(g)
    packed_d = torch.from_numpy(packed).to("cuda")
    _, c = eng.decode_packed(packed_d, n, None, n)
    mean_dtype = np.float32 if g.dtype == np.float32 else np.float64
    st = _Stats(c.cpu().numpy(), n, mean_dtype, maf_threshold, miss_threshold)
    if st.idx.size == 0:
        return []
    cohort = _prepare_cohort(kinship, eigenvalues, eigenvectors, covariates, y, lmm_mode, l_min,
                             l_max, n_grid, n_refine, precision)
    res = associate_records(cohort, packed[st.idx], n, None, st.mean[st.idx].astype(np.float64),
                            n_miss=st.miss[st.idx])
    return _build_results(lmm_mode, st.idx, st.af[st.idx], st.miss[st.idx], snp_info, res)
