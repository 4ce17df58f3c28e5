"""Oracle restatement of jamma's SNP statistics, filters and centered kinship."""

from __future__ import annotations

import numpy as np


def snp_stats(g: np.ndarray):
    """Per-SNP (mean, miss_count, var) as ``compute_snp_stats`` computes them.

    Restates ``src/jamma/core/snp_filter.py:36-56`` (and the pass-1 loop of
    ``src/jamma/lmm/runner_streaming.py:246-256``): NaN-aware mean and variance in
    the input dtype, NaN results (all-missing SNPs) replaced by 0.
    """
    miss = np.sum(np.isnan(g), axis=0)
    with np.errstate(invalid="ignore"), np.testing.suppress_warnings() as sup:
        sup.filter(RuntimeWarning)
        mean = np.nanmean(g, axis=0)
        var = np.nanvar(g, axis=0)
    return np.nan_to_num(mean, nan=0.0), miss, np.nan_to_num(var, nan=0.0)


def filter_mask(mean, miss, var, n_samples, maf_threshold, miss_threshold):
    """``compute_snp_filter_mask`` (``src/jamma/core/snp_filter.py:59-91``).

    Returns (mask, allele_freqs) with af = mean/2 (not folded), maf = min(af, 1-af),
    keep iff maf >= maf_threshold and miss/n <= miss_threshold and var > 0.
    """
    mean = np.asarray(mean, dtype=np.float64)
    miss_rates = miss / n_samples
    af = mean / 2.0
    maf = np.minimum(af, 1.0 - af)
    mask = (maf >= maf_threshold) & (miss_rates <= miss_threshold) & (np.asarray(var) > 0)
    return mask, af


def centered_kinship(
    g: np.ndarray, batch_size: int = 10000, maf_threshold: float = 0.0, miss_threshold: float = 1.0
) -> np.ndarray:
    """GEMMA -gk 1 centered relatedness matrix, FP64.

    Restates ``compute_centered_kinship`` (``src/jamma/kinship/compute.py:93-226``):
    filter with stats in the input dtype (``_filter_snps`` 60-90; monomorphic SNPs
    always dropped), then per 10k-SNP batch ``impute_and_center``
    (``src/jamma/kinship/missing.py:22-61``: float64 nanmean, NaN -> mean, subtract
    mean) and ``K += Xc Xc^T``; finally ``K /= p_kept``.
    """
    n, _ = g.shape
    mean, miss, var = snp_stats(g)
    mask, _ = filter_mask(mean, miss, var, n, maf_threshold, miss_threshold)
    p = int(mask.sum())
    if p == 0:
        raise ValueError("No SNPs passed filtering")
    x = np.asarray(g[:, mask], dtype=np.float64)
    k = np.zeros((n, n))
    for s in range(0, p, batch_size):
        xb = x[:, s : s + batch_size]
        with np.testing.suppress_warnings() as sup:
            sup.filter(RuntimeWarning)
            mu = np.nan_to_num(np.nanmean(xb, axis=0, keepdims=True), nan=0.0)
        xc = np.where(np.isnan(xb), mu, xb) - mu
        k += xc @ xc.T
    return k / p


def stream_pass1_means(g32: np.ndarray):
    """Pass-1 statistics of the streaming runner on float32 genotypes.

    ``src/jamma/lmm/runner_streaming.py:224-256`` decodes chunks as float32 and takes
    ``np.nanmean``/``np.nanvar`` there.  Sums of 0/1/2 counts are exact in float32
    (n < 2**23), and NumPy divides the float32 sum by the integer count in float64
    before storing into float32, so the mean is ``float32(sum / n_obs)``.
    """
    return snp_stats(np.asarray(g32, dtype=np.float32))


def loco_kinships(g: np.ndarray, chroms, maf_threshold: float = 0.0, miss_threshold: float = 1.0):
    """Leave-one-chromosome-out kinships, in sorted chromosome-name order.

    Restates ``compute_loco_kinship_streaming`` (``src/jamma/kinship/compute.py:693-916``):
    float32 pass-1 statistics over all samples pick the SNPs (MAF / missing / monomorphic),
    float64 ``impute_and_center`` per SNP, S_full = sum of all kept SNPs' Xc Xc^T and
    S_c per chromosome, K_loco_c = (S_full - S_c) / (p - p_c).  Yields (chr, K_loco_c).
    """
    chroms = np.asarray(chroms).astype(str)
    n, _ = g.shape
    mean, miss, var = snp_stats(np.asarray(g, dtype=np.float32))
    mask, _ = filter_mask(mean, miss, var, n, maf_threshold, miss_threshold)
    idx = np.where(mask)[0]
    if idx.size == 0:
        raise ValueError("No SNPs passed filtering")
    x = np.asarray(g[:, idx], dtype=np.float64)
    with np.testing.suppress_warnings() as sup:
        sup.filter(RuntimeWarning)
        mu = np.nan_to_num(np.nanmean(x, axis=0, keepdims=True), nan=0.0)
    xc = np.where(np.isnan(x), mu, x) - mu
    s_full = xc @ xc.T
    kept_chr = chroms[idx]
    for c in sorted(set(chroms.tolist())):
        sel = kept_chr == c
        if not np.any(sel):
            continue
        p_loco = idx.size - int(sel.sum())
        if p_loco == 0:
            raise ValueError(f"all filtered SNPs are on chromosome {c}")
        s_c = xc[:, sel] @ xc[:, sel].T
        yield c, (s_full - s_c) / p_loco


def standardized_kinship(g: np.ndarray, batch_size: int = 10000, maf_threshold: float = 0.0,
                         miss_threshold: float = 1.0) -> np.ndarray:
    """GEMMA -gk 2 standardized relatedness matrix, FP64.

    Restates ``compute_standardized_kinship`` (``src/jamma/kinship/compute.py:229-360``):
    the same SNP filter as -gk 1 (stats in the input dtype, monomorphic SNPs dropped), then
    per batch ``impute_center_and_standardize`` (``src/jamma/kinship/missing.py:64-119``):
    float64 nanmean, NaN -> mean, centre, var = mean over all n of x_imputed^2 - mean^2,
    z = centred / sqrt(var) (0 where the sd is 0); ``K += Z Z^T``; finally ``K /= p_kept``.
    """
    n, _ = g.shape
    mean, miss, var = snp_stats(g)
    mask, _ = filter_mask(mean, miss, var, n, maf_threshold, miss_threshold)
    p = int(mask.sum())
    if p == 0:
        raise ValueError("No SNPs passed filtering")
    x = np.asarray(g[:, mask], dtype=np.float64)
    k = np.zeros((n, n))
    for s in range(0, p, batch_size):
        xb = x[:, s : s + batch_size]
        with np.testing.suppress_warnings() as sup:
            sup.filter(RuntimeWarning)
            mu = np.nan_to_num(np.nanmean(xb, axis=0, keepdims=True), nan=0.0)
        xi = np.where(np.isnan(xb), mu, xb)
        sd = np.sqrt(np.mean(xi * xi, axis=0, keepdims=True) - mu * mu)
        with np.errstate(invalid="ignore", divide="ignore"):
            z = np.where(sd > 0, (xi - mu) / sd, 0.0)
        k += z @ z.T
    return k / p
