"""Leave-one-chromosome-out (LOCO) kinship and association on the GPU.

``compute_loco_kinship`` restates ``compute_loco_kinship_streaming``
(src/jamma/kinship/compute.py:693-916): pass-1 float32 statistics over all samples
choose the SNPs, and each chromosome's kinship K_loco = (S_full - S_c) / (p - p_c) comes
from the full-genome and per-chromosome sums -- exact int32 INT8 Grams plus FP64
corrections (``precision="int8"``) or FP64 centred Grams (``precision="fp64"``).

``run_lmm_loco`` restates ``run_lmm_loco`` (src/jamma/lmm/loco.py:54-252): chromosomes
in sorted-name order, K_loco restricted to the analysed samples and eigendecomposed on
the device, then that chromosome's SNPs are tested with float64 statistics and
imputation means over the analysed samples (``_run_lmm_for_chromosome``, 255-593).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

from jamma_b200 import _native
from jamma_b200 import engine as eng
from jamma_b200.device import empty, ptr, require_cuda, stream_handle
from jamma_b200.eigen import eigendecompose_kinship_device
from jamma_b200.io import (
    MODE_TEST,
    AssocResult,
    BedFile,
    IncrementalAssocWriter,
    apply_snp_list_mask,
    format_assoc_line,
    get_plink_metadata,
    snp_info_from_meta,
    write_kinship_matrix,
)
from jamma_b200.kinship import _KinshipAccumulator, _KinshipI8, filter_mask, snp_stats_from_counts
from jamma_b200.lmm import _build_results, _Stats, associate_records, valid_sample_mask


def chromosome_partitions(chroms) -> dict[str, np.ndarray]:
    """SNP indices per chromosome name, keys in first-appearance order
    (``get_chromosome_partitions``, src/jamma/io/plink.py:139-175)."""
    chroms = np.asarray(chroms).astype(str)
    _, first = np.unique(chroms, return_index=True)
    return {chroms[i]: np.where(chroms == chroms[i])[0] for i in np.sort(first)}


def _counts_all(bed: BedFile, chunk: int) -> np.ndarray:
    return eng.pass1_counts(bed, None, bed.n_samples, max(chunk, 16384))


def compute_loco_kinship(bfile, maf_threshold: float = 0.0, miss_threshold: float = 1.0,
                         chunk_size: int = 10000, precision: str = "int8",
                         ksnps_indices: np.ndarray | None = None):
    """Yield (chromosome, K_loco) device tensors (n x n, all samples), sorted by name."""
    if precision not in ("int8", "fp64"):
        raise ValueError("precision must be 'int8' or 'fp64'")
    require_cuda()
    meta = get_plink_metadata(bfile)
    chroms = np.asarray(meta["chromosome"]).astype(str)
    bed = BedFile(bfile, meta["n_samples"], meta["n_snps"])
    n = bed.n_samples
    counts = _counts_all(bed, chunk_size)
    mean, miss, poly = snp_stats_from_counts(counts, n, np.float32)
    keep, _ = filter_mask(mean, miss, poly, n, maf_threshold, miss_threshold)
    if ksnps_indices is not None:
        apply_snp_list_mask(keep, ksnps_indices, keep.size, "Kinship SNP list")
    idx = np.where(keep)[0]
    if idx.size == 0:
        raise ValueError("No SNPs passed filtering")
    names = sorted(set(chroms.tolist()))

    def accumulate(sub: np.ndarray):
        acc = _KinshipI8(n, sub.size) if precision == "int8" else _KinshipAccumulator(n, 4096)
        for s in range(0, sub.size, chunk_size):
            part = sub[s:s + chunk_size]
            rec = torch.from_numpy(bed.take(part)).cuda()
            codes, _ = eng.decode_packed(rec, n, None, n)
            c = counts[part]
            mu = torch.from_numpy(c[:, 1] / np.maximum(c[:, 0], 1)).cuda()
            if precision == "int8":
                acc.add(codes, mu, bool(np.any(c[:, 0] < n)), n_missing=int((n - c[:, 0]).sum()))
                acc.add_sum_mu2(c[:, 1] / np.maximum(c[:, 0], 1))
            else:
                acc.add(codes, mu)
        return acc

    full = accumulate(idx)
    if precision == "int8":
        C_full = full.gram()
    st = stream_handle()
    for c in names:
        sub = idx[chroms[idx] == c]
        if sub.size == 0:
            continue
        p_loco = idx.size - sub.size
        if p_loco == 0:
            raise ValueError(f"Cannot compute LOCO kinship: all {idx.size} filtered SNPs are on "
                             f"chromosome '{c}'.")
        part = accumulate(sub)
        K = empty((n, n))
        if precision == "int8":
            C_c = part.gram()
            q_full = full.RT
            q_c = part.RT
            if (q_full is None) != (q_c is None):  # one side without missing calls
                if q_full is None:
                    full.RT = q_full = torch.zeros_like(q_c)
                else:
                    q_c = torch.zeros_like(q_full)
            _native.call("jb_kinship_i8_finalize_loco", ptr(C_full), ptr(C_c), n, n, ptr(full.a),
                         ptr(part.a), ptr(full.b), ptr(part.b), full.sum_mu2 - part.sum_mu2,
                         ptr(q_full), ptr(q_c), n, p_loco, ptr(K), n, st)
        else:
            _native.call("jb_kinship_loco_f64", ptr(full.K), ptr(part.K), n, n, p_loco, ptr(K), n, st)
        yield c, K


def run_lmm_loco(bed_path, phenotypes: np.ndarray, covariates: np.ndarray | None = None,
                 maf_threshold: float = 0.01, miss_threshold: float = 0.05, lmm_mode: int = 1,
                 output_path: Path | None = None, check_memory: bool = True,
                 show_progress: bool = True, save_kinship: bool = False,
                 kinship_output_dir: Path | None = None, kinship_output_prefix: str = "result",
                 snps_indices: np.ndarray | None = None, ksnps_indices: np.ndarray | None = None,
                 precision: str = "fp64", kinship_precision: str = "int8") -> list[AssocResult]:
    """LOCO association; results in sorted-chromosome order (empty when written to disk)."""
    if lmm_mode not in (1, 2, 3, 4):
        raise ValueError(f"lmm_mode must be 1, 2, 3 or 4, got {lmm_mode}")
    meta = get_plink_metadata(bed_path)
    chroms = np.asarray(meta["chromosome"]).astype(str)
    parts = chromosome_partitions(chroms)
    if len(parts) < 2:
        raise ValueError("LOCO requires SNPs on multiple chromosomes. "
                         f"Found only {len(parts)} chromosome(s): {list(parts)}")
    y = np.asarray(phenotypes, dtype=np.float64)
    valid = valid_sample_mask(y, covariates)
    if not np.any(valid):
        raise ValueError("No samples with valid phenotypes")
    require_cuda()  # after the argument and file checks, which raise as jamma's do
    n_file = meta["n_samples"]
    sample_idx = None if np.all(valid) else np.where(valid)[0].astype(np.int32)
    sidx = None if sample_idx is None else torch.from_numpy(sample_idx).cuda()
    vsel = torch.from_numpy(np.where(valid)[0]).cuda()
    yv = y[valid]
    cov = None if covariates is None else np.asarray(covariates, dtype=np.float64)[valid]
    n = yv.size
    bed = BedFile(bed_path, n_file, meta["n_snps"])
    snp_info = snp_info_from_meta(meta)
    results: list[AssocResult] = []
    writer = IncrementalAssocWriter(output_path, MODE_TEST[lmm_mode]) if output_path else None
    if writer:
        writer.__enter__()
    try:
        for c, K in compute_loco_kinship(bed_path, maf_threshold, miss_threshold,
                                         precision=kinship_precision, ksnps_indices=ksnps_indices):
            if save_kinship and kinship_output_dir is not None:
                write_kinship_matrix(K.cpu().numpy(),
                                     Path(kinship_output_dir) / f"{kinship_output_prefix}.loco.cXX.chr{c}.txt")
            Kv = K if sample_idx is None else K.index_select(0, vsel).index_select(1, vsel).contiguous()
            del K
            evals, U = eigendecompose_kinship_device(Kv)
            cols = parts[c]
            cnt = np.empty((cols.size, 4), dtype=np.int32)
            for s in range(0, cols.size, 8192):
                _, cc = eng.decode_packed(torch.from_numpy(bed.take(cols[s:s + 8192])).cuda(), n_file,
                                          sidx, n)
                cnt[s:s + 8192] = cc.cpu().numpy()
            local_sel = None
            if snps_indices is not None:
                local_sel = np.where(np.isin(cols, np.asarray(snps_indices)))[0]
            st = _Stats(cnt, n, np.float64, maf_threshold, miss_threshold, local_sel)
            if st.idx.size == 0:
                continue
            cohort = eng.DeviceCohort(evals, U, cov, yv, lmm_mode, precision=precision)
            glob = cols[st.idx]
            res = associate_records(cohort, lambda a, b, out: bed.take_into(glob[a:b], out), n_file,
                                    sample_idx,
                                    st.mean[st.idx].astype(np.float64), n_miss=st.miss[st.idx])
            chr_results = _build_results(lmm_mode, glob, st.af[st.idx], st.miss[st.idx], snp_info, res)
            if writer:
                writer.write_lines([format_assoc_line(r, MODE_TEST[lmm_mode]) for r in chr_results])
            else:
                results.extend(chr_results)
            del cohort, evals, U, Kv
    finally:
        if writer:
            writer.__exit__(None, None, None)
    return [] if output_path is not None else results
