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


@pytest.mark.parametrize("mode,n_cov", [(4, 1), (3, 1), (4, 2)])
def test_mixed_form_at_the_upper_lambda_bound(mode, n_cov):
    """Phenotypes whose variance is all genetic drive the null and alternative lambdas to
    the upper bound 1e5, where the weighted sums the statistics use shrink by ~1/(lambda e)
    and the series' fixed absolute error would dominate them; the mixed form evaluates
    those optima with direct FP64 sums and must keep every p-value within 1e-6 of the
    plain FP64 form (before, 3-5 % of such pairs were off by up to 2e-4).  With a second
    covariate column the mixed form runs one pair per warp instead of two."""
    from jamma_b200 import _native
    from jamma_b200 import engine as eng
    from jamma_b200.device import ptr, stream_handle

    n, m = 3000, 512
    g_k = synth.genotypes(n, 6000, 0.0, seed=21)
    K = OK.centered_kinship(g_k)
    w, U = np.linalg.eigh(K)
    w = np.where(np.abs(w) < 1e-10, 0.0, w)
    rng = np.random.default_rng(22)
    genetic = U @ (np.sqrt(np.maximum(w, 0))[:, None] * rng.standard_normal((n, 2)))
    mixed_h2 = genetic[:, :1] + 0.5 * rng.standard_normal((n, 1))
    Y = np.column_stack([genetic, mixed_h2, rng.standard_normal(n)])
    W = None if n_cov == 1 else np.column_stack([np.ones(n), rng.standard_normal(n)])
    g = synth.genotypes(n, m, 0.01, seed=23)
    packed = torch.from_numpy(OP.encode_genotypes(g)).cuda()
    mu = torch.from_numpy(np.nan_to_num(np.nanmean(g, 0)).astype(np.float32).astype(np.float64)).cuda()
    out = {}
    for precision in ("fp64", "mixed"):
        coh = eng.DeviceCohort(w, U, W, Y, lmm_mode=mode, precision=precision)
        codes, _ = eng.decode_packed(packed, n, None, n, ld=coh.code_ld)
        if precision == "mixed":
            assert coh.search == 1
            X = coh.rotate_codes_i8(codes, mu, True)
        else:
            G = eng.empty((m, n))
            _native.call("jb_impute_f64", ptr(codes), coh.code_ld, n, m, ptr(mu), ptr(G), n,
                         stream_handle())
            X = eng.rotate(coh.U, G)
        out[precision] = ({k: v.cpu().numpy() for k, v in coh.associate_rotated(X).items()},
                          coh.null_model()[0])
    (a, lam0), (b, _) = out["mixed"], out["fp64"]
    assert np.all(lam0[:2] > 1e4), f"the all-genetic phenotypes should reach the bound: {lam0}"
    if mode == 4:
        assert np.all(a["lambda_mle"][:2] > 1e4)
    # score and LRT: the null lambda is the plain form's and the MLE optimum sits on the
    # bound in both forms, so every pair must agree; Wald: the REML optimum is searched on
    # the series, and a golden-section step decided differently (a near tie) moves a few
    # p-values by ~1e-6, as between any two FP64 summation orders
    checks = (("p_wald", 0.99), ("p_lrt", 0.998), ("p_score", 0.998)) if mode == 4 else \
        (("p_score", 0.998),)
    for k, frac in checks:
        for f in range(Y.shape[1]):
            x, y = a[k][f], b[k][f]
            rel = np.abs(x - y) / np.abs(y)
            assert np.mean(rel <= 1e-6) >= frac, f"{k} phenotype {f}: worst {rel.max():.2e}"
            assert np.max(np.abs(np.log10(x) - np.log10(y))) < 1e-4, (k, f)
            for t in (0.05, 1e-3, 5e-8):
                np.testing.assert_array_equal(x < t, y < t)
