"""Host-side SNP filters against the oracle: the Hardy-Weinberg chi-square p-values
(src/jamma/core/snp_filter.py:94-150) with degenerate SNPs, the -snps / -ksnps list files
(src/jamma/io/snp_list.py:13-88) and the in-place list mask (snp_filter.py:15-33)."""

from __future__ import annotations

import numpy as np
import pytest

from jamma_b200 import io as jio
from jamma_b200.kinship import filter_mask, snp_stats_from_counts
from jamma_b200.lmm import _Stats, hwe_pvalues
from oracle import filters as OF
from oracle import kinship as OK


def _counts_from_genotypes(g):
    """Device-layout counts {n_obs, sum, n_het, n_hom2} per SNP, computed on the host."""
    ok = ~np.isnan(g)
    return np.stack([ok.sum(0), np.nansum(g, 0), ((g == 1) & ok).sum(0),
                     ((g == 2) & ok).sum(0)], axis=1).astype(np.int32)


def test_hwe_pvalues_match_the_oracle_including_degenerate_snps():
    rng = np.random.default_rng(5)
    aa = rng.integers(0, 400, 500)
    ab = rng.integers(0, 400, 500)
    bb = rng.integers(0, 400, 500)
    # degenerate rows (p = 1 by convention): no calls, one homozygote class only, a single
    # call; row 3 (heterozygotes only) is a genuine departure
    aa[:6] = [0, 50, 0, 0, 1, 0]
    ab[:6] = [0, 0, 0, 30, 0, 0]
    bb[:6] = [0, 0, 70, 0, 0, 1]
    # strong departures (tiny p) and exact equilibrium
    aa[6:9], ab[6:9], bb[6:9] = [500, 0, 250], [0, 1000, 500], [500, 0, 250]
    got, ref = hwe_pvalues(aa, ab, bb), OF.hwe_pvalues(aa, ab, bb)
    deg = [0, 1, 2, 4, 5]
    assert np.all(got[deg] == 1.0) and np.all(ref[deg] == 1.0)
    assert got[3] < 1e-7 and got[8] == 1.0 and ref[8] == 1.0
    tiny = ref < 1e-300
    np.testing.assert_array_equal(got[tiny] < 1e-290, True)
    np.testing.assert_allclose(got[~tiny], ref[~tiny], rtol=1e-11, atol=0)


def test_hwe_filter_of_the_runner_keeps_the_oracle_snp_set():
    rng = np.random.default_rng(6)
    n, p = 300, 400
    af = rng.uniform(0.05, 0.5, p)
    g = rng.binomial(2, af, size=(n, p)).astype(np.float64)
    # push some SNPs out of equilibrium: heterozygotes to homozygotes
    bad = rng.choice(p, 40, replace=False)
    for j in bad:
        het = np.where(g[:, j] == 1)[0]
        g[het[: len(het) * 3 // 4], j] = rng.choice([0.0, 2.0], len(het) * 3 // 4)
    g[rng.random((n, p)) < 0.02] = np.nan
    g[:, 0] = np.nan  # all missing
    g[:, 1] = 1.0     # monomorphic heterozygote
    counts = _counts_from_genotypes(g)
    for thr in (1e-6, 1e-3, 0.05):
        st = _Stats(counts, n, np.float32, 0.01, 0.05, hwe_threshold=thr)
        mean, miss, var = OK.snp_stats(g.astype(np.float32))
        mask, _ = OK.filter_mask(mean, miss, var, n, 0.01, 0.05)
        mask &= OF.hwe_pvalues(*OF.genotype_counts(g)) >= thr
        np.testing.assert_array_equal(st.idx, np.where(mask)[0], err_msg=f"threshold {thr}")
    assert np.intersect1d(st.idx, bad).size < bad.size  # the filter removed some


def test_snp_list_files_resolve_like_the_oracle(tmp_path):
    sids = np.array([f"rs{i}" for i in range(50)] + ["RS7", "chr1:100"])
    f = tmp_path / "snps.txt"
    f.write_text("rs3\n\n  rs10 extra columns here\nrs7\nrs7\nmissing_id\nRS7\nchr1:100\trest\n")
    got = jio.resolve_snp_list_to_indices(jio.read_snp_list_file(f), sids)
    ref = OF.snp_list_indices(f, sids)
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(got, [3, 7, 10, 50, 51])
    mask = np.ones(sids.size, dtype=bool)
    mask[3] = False
    jio.apply_snp_list_mask(mask, got, sids.size, "SNP list")
    np.testing.assert_array_equal(np.where(mask)[0], [7, 10, 50, 51])


def test_snp_list_errors_follow_jamma(tmp_path):
    with pytest.raises(FileNotFoundError):
        jio.read_snp_list_file(tmp_path / "absent.txt")
    empty = tmp_path / "empty.txt"
    empty.write_text("\n  \n")
    with pytest.raises(ValueError, match="empty"):
        jio.read_snp_list_file(empty)
    with pytest.raises(ValueError, match="matched"):
        jio.resolve_snp_list_to_indices({"zz"}, np.array(["a", "b"]))
    with pytest.raises(ValueError, match="out of range"):
        jio.apply_snp_list_mask(np.ones(4, dtype=bool), np.array([1, 4]), 4, "SNP list")


def test_snp_list_restricts_the_runner_filter():
    rng = np.random.default_rng(8)
    n, p = 200, 60
    g = rng.binomial(2, rng.uniform(0.05, 0.5, p), size=(n, p)).astype(np.float64)
    g[:, 5] = 0.0  # monomorphic: filtered even when listed
    counts = _counts_from_genotypes(g)
    sel = np.array([2, 5, 9, 40, 59])
    st = _Stats(counts, n, np.float32, 0.01, 0.05, snps_indices=sel)
    mean, miss, poly = snp_stats_from_counts(counts, n)
    keep, _ = filter_mask(mean, miss, poly, n, 0.01, 0.05)
    np.testing.assert_array_equal(st.idx, [j for j in sel if keep[j]])
    assert 5 not in st.idx
