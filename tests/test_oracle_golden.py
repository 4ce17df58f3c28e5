"""Pin the CPU oracle against jamma's golden vectors (no GPU).

Two sources: GEMMA fixture outputs (kinship, Wald / LRT / Score / all-tests, with
and without covariates; null-model log-likelihoods) at jamma's own tolerances
(``JAX_GEMMA_TOLERANCES`` = ToleranceConfig(lambda_rtol=5e-5), tests/test_lmm_validation.py:32
in jamma), and jamma's NumPy likelihood module evaluated by
``tests/golden/make_golden.py`` (tight, FP64 round-off level).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import kinship as OK
from oracle import lmm as OL

# jamma ToleranceConfig defaults with lambda_rtol=5e-5 (src/jamma/validation/tolerances.py)
TOL = {"beta": 1e-2, "se": 1e-5, "p_wald": 1e-4, "p_lrt": 1e-4, "p_score": 1e-4,
       "l_remle": 5e-5, "l_mle": 5e-5}
ATOL = 1e-12
COLS = {"beta": "beta", "se": "se", "l_remle": "lambda_remle", "p_wald": "p_wald",
        "l_mle": "lambda_mle", "p_lrt": "p_lrt", "p_score": "p_score"}


def _assert_close(a, b, rtol, atol=ATOL, name=""):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    bad = ~(np.abs(a - b) <= atol + rtol * np.abs(b))
    assert not bad.any(), f"{name}: {bad.sum()} mismatches, worst rel " \
        f"{np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)):.3e}"


def test_kinship_matches_gemma(gemma, gemma_geno):
    k = OK.centered_kinship(gemma_geno.astype(np.float32))
    np.testing.assert_allclose(k, gemma["kinship"], rtol=1e-8, atol=1e-9)


@pytest.mark.parametrize("case,mode,cov", [
    ("wald", 1, False), ("lrt", 2, False), ("score", 3, False), ("all", 4, False),
    ("cov_wald", 1, True), ("cov_lrt", 2, True), ("cov_score", 3, True), ("cov_all", 4, True),
])
def test_association_matches_gemma(gemma, gemma_geno, case, mode, cov):
    covariates = gemma["covariates"] if cov else None
    r = OL.lmm_association(gemma_geno.astype(np.float32), gemma["pheno"], kinship=gemma["kinship"],
                           covariates=covariates, lmm_mode=mode)
    checked = 0
    for col, key in COLS.items():
        ref_key = f"{case}__{col}"
        if ref_key not in gemma:
            continue
        # beta for near-zero effects needs jamma's absolute tolerance
        atol = 1e-6 if col == "beta" else ATOL
        _assert_close(r.stats[key], gemma[ref_key], TOL[col], atol, name=f"{case}:{col}")
        checked += 1
    assert checked >= 2
    np.testing.assert_allclose(r.af, gemma[f"{case}__af"], atol=5e-4)


def test_null_logl_matches_gemma_log(gemma, gemma_geno):
    evals, U = OL.eigh_threshold(gemma["kinship"])
    y = gemma["pheno"]
    UtW = U.T @ np.ones((y.size, 1))
    Uty = U.T @ y
    _, l0 = OL.null_model_mle(evals, UtW, Uty)
    np.testing.assert_allclose(l0, gemma["lrt__null_mle"], rtol=1e-5)


def test_pab_and_logl_match_reference_module(ref_lik):
    evals = ref_lik["evals"]
    lambdas = ref_lik["lambdas"]
    for tag in ("ic", "cov"):
        UtW, Uty, UtG = ref_lik[f"{tag}__UtW"], ref_lik[f"{tag}__Uty"], ref_lik[f"{tag}__UtG"]
        c = UtW.shape[1]
        uab = OL.build_uab(UtW, Uty, UtG)
        iab = OL.pab_recursion(c, uab.sum(axis=1))
        m = UtG.shape[1]
        for k, lam in enumerate(lambdas):
            lv = np.full(m, lam)
            np.testing.assert_allclose(OL.reml_alt(c, lv, evals, uab, iab), ref_lik[f"{tag}__reml"][:, k],
                                       rtol=1e-11)
            np.testing.assert_allclose(OL.mle_alt(c, lv, evals, uab), ref_lik[f"{tag}__mle"][:, k],
                                       rtol=1e-11)
            hi = 1.0 / (lam * evals + 1.0)
            np.testing.assert_allclose(OL.calc_pab(c, hi, uab), ref_lik[f"{tag}__pab"][:, k],
                                       rtol=1e-9, atol=1e-12)


def test_null_model_matches_reference_module(ref_lik):
    evals = ref_lik["evals"]
    for tag in ("ic", "cov"):
        UtW, Uty = ref_lik[f"{tag}__UtW"], ref_lik[f"{tag}__Uty"]
        lam, logl = OL.null_model_mle(evals, UtW, Uty)
        np.testing.assert_allclose([lam, logl], ref_lik[f"{tag}__null_mle"], rtol=1e-12)


def test_golden_refine_is_deterministic_and_bracketed():
    # a smooth concave function of log-lambda with its maximum at log(3)
    f = lambda lg: -(lg - np.log(3.0)) ** 2  # noqa: E731
    ll = OL.grid_log_lambdas(1e-5, 1e5, 50)
    grid = np.stack([f(np.full(4, v)) for v in ll])
    lam, val = OL.golden_refine(f, grid, ll, 50, 20)
    np.testing.assert_allclose(lam, 3.0, rtol=5e-5)
    assert np.all(val <= 0)


def test_standardized_kinship_known_answer():
    """The reference's hand-computed -gk 2 case (tests/test_kinship_compute.py:257-273):
    3 samples x 2 SNPs, each SNP mean 1 and variance 2/3 over all samples."""
    x = np.array([[0.0, 2.0], [1.0, 1.0], [2.0, 0.0]])
    sd = np.sqrt(2.0 / 3.0)
    z = np.array([[-1.0 / sd, 1.0 / sd], [0.0, 0.0], [1.0 / sd, -1.0 / sd]])
    np.testing.assert_allclose(OK.standardized_kinship(x), z @ z.T / 2, rtol=0, atol=1e-12)


def test_standardized_kinship_missing_and_monomorphic():
    """Missing calls are imputed before the variance (they shrink it, n in the
    denominator); monomorphic SNPs are filtered out of p."""
    x = np.array([[0.0, 1.0, 2.0], [np.nan, 1.0, 1.0], [2.0, 1.0, 0.0], [1.0, 1.0, np.nan]])
    k = OK.standardized_kinship(x)
    cols = []
    for j in (0, 2):  # SNP 1 is monomorphic and dropped
        c = x[:, j]
        mu = np.nanmean(c)
        ci = np.where(np.isnan(c), mu, c)
        cols.append((ci - mu) / np.sqrt(np.mean(ci**2) - mu**2))
    z = np.column_stack(cols)
    np.testing.assert_allclose(k, z @ z.T / 2, rtol=1e-13, atol=1e-14)
