"""GPU edge cases that jamma's own tests pin, against the CPU oracle.

- Degenerate SNP columns and eigenvalue spectra (tests/test_hypothesis.py:480-700 in
  jamma): an all-zero rotated genotype has P_xx = 0 exactly, so beta, se, p_wald and
  p_score are NaN (src/jamma/lmm/stats.py:138-150); a constant genotype collinear with
  the intercept leaves a last-bit residual of either sign, so it must come out finite or
  NaN but never infinite; kinships with zero eigenvalues and with negative eigenvalues
  (non-PSD) keep the oracle's values and NaN pattern.  The mixed form evaluates
  non-PSD cohorts directly in FP64 (no series over a pole of 1/(lambda e + 1)).
- Missingness edge SNPs (tests/test_missingness.py:149-275 in jamma): all-missing,
  single-observation and two-observation SNPs through the streaming runner in both forms,
  with default and permissive filters, give the oracle's SNP set and statistics; a
  cohort whose SNPs all fail the filter returns no results.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import kinship as OK
from oracle import lmm as OL
from oracle import plink as OP

from _parity import _arrays, assert_assoc_parity, assert_mixed_parity

pytestmark = pytest.mark.gpu

KEYS = ("lambda_remle", "logl_h1", "beta", "se", "p_wald", "lambda_mle", "logl_mle", "p_lrt",
        "p_score")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


def _check(precision, got, ref, keys):
    if precision == "fp64":
        assert_assoc_parity(got, ref, keys, min_frac=0.9)
    else:
        assert_mixed_parity(got, ref, keys)


def _spectrum(kind: str, n: int, rng) -> np.ndarray:
    if kind == "positive":
        return np.abs(rng.standard_normal(n)) + 0.1
    if kind == "zeros":  # thresholded eigenvalues of a rank-deficient kinship
        return np.sort(np.r_[np.zeros(n // 10), np.abs(rng.standard_normal(n - n // 10)) + 0.1])
    return np.sort(rng.standard_normal(n))  # non-PSD: about half negative


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kind", ["positive", "zeros", "negative"])
@pytest.mark.parametrize("n", [50, 333])
def test_degenerate_columns_and_spectra_follow_the_oracle(precision, kind, n):
    from jamma_b200 import engine as eng

    rng = np.random.default_rng(1000 + n)
    ev = _spectrum(kind, n, rng)
    U = np.eye(n)  # rotated vectors are the inputs themselves, as in jamma's unit tests
    y = rng.standard_normal(n)
    m_rand = 29
    X = np.column_stack([np.zeros(n), np.r_[2.0, np.ones(n - 1)],
                         rng.standard_normal((n, m_rand))])
    const = np.column_stack([np.ones(n), 2.0 * np.ones(n)])
    lam0, l0 = OL.null_model_mle(ev, np.ones((n, 1)), y)
    ref = OL.lmm_chunk(4, ev, np.ones((n, 1)), y, X, logl_h0=l0, lam0=lam0)

    coh = eng.DeviceCohort(ev, U, None, y, lmm_mode=4, precision=precision)
    if precision == "mixed" and kind == "negative":
        assert coh.search == 0  # direct FP64 probes: the series would cross a pole
    Xd = torch.from_numpy(np.ascontiguousarray(np.column_stack([X, const]).T)).cuda()
    out = {k: v.cpu().numpy()[0] for k, v in coh.associate_rotated(Xd).items()}
    got = {k: v[: X.shape[1]] for k, v in out.items()}

    # x = 0: P_xx = 0 exactly -> no Wald or score statistics, like jamma
    for k in ("beta", "se", "p_wald", "p_score"):
        assert np.isnan(got[k][0]) and np.isnan(ref[k][0]), k
    keys = [k for k in KEYS if k in got and not np.all(np.isnan(ref[k]))]
    _check(precision, got, ref, keys)
    # constant genotypes: finite or NaN, never infinite
    for k in KEYS:
        if k in out:
            assert not np.any(np.isinf(out[k][X.shape[1]:])), k


@pytest.fixture(scope="module")
def missing_cohort(tmp_path_factory):
    d = tmp_path_factory.mktemp("edge")
    n, p = 300, 400
    g = synth.genotypes(n, p, 0.02, seed=21)
    g[:, 0] = np.nan  # all missing
    g[:, 1] = np.nan
    g[0, 1] = 1.0  # one observed call: zero variance
    g[:, 2] = np.nan
    g[0, 2], g[1, 2] = 0.0, 2.0  # two observed calls: polymorphic
    rows = np.random.default_rng(3).random(n) < 0.6
    g[rows, 3] = np.nan  # 60 % missing
    g[:, 4] = np.where(np.arange(n) % 2 == 0, np.nan, 2.0)  # monomorphic where observed
    g[::7, 5:40] = np.nan  # heterogeneous missingness on a block of SNPs
    y = synth.phenotypes(np.nan_to_num(g, nan=1.0), n_causal=8, h2=0.5, seed=5)
    OP.write_plink(d / "edge", g, phenotypes=y)
    K = OK.centered_kinship(g.astype(np.float32))
    return d / "edge", g, y, K


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("maf,miss", [(0.01, 0.05), (0.0, 1.0)])
def test_missingness_edge_snps_match_oracle(missing_cohort, precision, maf, miss):
    from jamma_b200 import run_lmm_association_streaming

    prefix, g, y, K = missing_cohort
    res = run_lmm_association_streaming(prefix, y, kinship=K, lmm_mode=4, chunk_size=128,
                                        maf_threshold=maf, miss_threshold=miss,
                                        precision=precision, show_progress=False)
    ref = OL.lmm_association(g, y, kinship=K, lmm_mode=4, maf_threshold=maf,
                             miss_threshold=miss)
    rs = np.array([int(r.rs[2:]) for r in res])
    np.testing.assert_array_equal(rs, ref.snp_indices)
    assert 0 not in rs and 1 not in rs and 4 not in rs  # all-missing, one call, monomorphic
    assert (2 in rs) == (miss >= 1.0)  # two calls pass only the permissive filter
    np.testing.assert_array_equal([r.af for r in res], ref.af)
    np.testing.assert_array_equal([r.n_miss for r in res], ref.n_miss)
    got = _arrays(res)
    keys = [k for k in got if k in ref.stats and not np.all(np.isnan(ref.stats[k]))]
    _check(precision, got, ref.stats, keys)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_all_snps_filtered_returns_no_results(tmp_path, precision):
    from jamma_b200 import run_lmm_association_streaming

    n, p = 60, 12
    g = synth.genotypes(n, p, 0.0, seed=4)
    g[:, :6] = np.nan
    g[:, 6:] = 1.0
    y = np.random.default_rng(2).standard_normal(n)
    OP.write_plink(tmp_path / "none", g, phenotypes=y)
    K = np.eye(n)
    res = run_lmm_association_streaming(tmp_path / "none", y, kinship=K, lmm_mode=4,
                                        precision=precision, show_progress=False)
    assert res == []
