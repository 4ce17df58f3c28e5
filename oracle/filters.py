"""Oracle restatement of jamma's host-side SNP filters: the Hardy-Weinberg chi-square
test and the -snps / -ksnps SNP lists (test infrastructure only)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
from scipy import stats


def hwe_pvalues(n_aa, n_ab, n_bb) -> np.ndarray:
    """``compute_hwe_pvalues`` (``src/jamma/core/snp_filter.py:94-150``): expected counts
    n p^2, 2 n p q, n q^2 with p = (2 n_aa + n_ab) / 2n; chi-square with one degree of
    freedom; NaN statistics (no calls, monomorphic) -> 0 -> p = 1.  JAX's ``chi2.sf`` is
    stood in for by SciPy's."""
    n_aa, n_ab, n_bb = (np.asarray(v, dtype=np.float64) for v in (n_aa, n_ab, n_bb))
    n = n_aa + n_ab + n_bb
    with np.errstate(invalid="ignore", divide="ignore"):
        p = (2 * n_aa + n_ab) / (2 * n)
        q = 1.0 - p
        e_aa, e_ab, e_bb = n * p ** 2, 2 * n * p * q, n * q ** 2
        chi = (n_aa - e_aa) ** 2 / e_aa + (n_ab - e_ab) ** 2 / e_ab + (n_bb - e_bb) ** 2 / e_bb
    chi = np.where(np.isnan(chi), 0.0, chi)
    return stats.chi2.sf(chi, df=1)


def genotype_counts(g: np.ndarray):
    """(n_aa, n_ab, n_bb) = counts of observed 0 / 1 / 2 calls per SNP, as the streaming
    runner's pass 1 accumulates them (``src/jamma/lmm/runner_streaming.py:264-268``)."""
    ok = ~np.isnan(g)
    return (np.sum((g == 0) & ok, axis=0), np.sum((g == 1) & ok, axis=0),
            np.sum((g == 2) & ok, axis=0))


def snp_list_indices(path, bim_sids) -> np.ndarray:
    """``read_snp_list_file`` + ``resolve_snp_list_to_indices``
    (``src/jamma/io/snp_list.py:13-88``): first token of each non-empty line, exact
    (case-sensitive) match against the .bim ids, sorted indices; FileNotFoundError /
    ValueError for a missing file, an empty list or no match."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(str(path))
    ids = set()
    for line in path.read_text().splitlines():
        if line.strip():
            ids.add(line.strip().split()[0])
    if not ids:
        raise ValueError("empty SNP list")
    found = sorted(i for i, s in enumerate(bim_sids) if s in ids)
    if not found:
        raise ValueError("no SNP of the list is in the .bim")
    return np.array(found, dtype=np.intp)
