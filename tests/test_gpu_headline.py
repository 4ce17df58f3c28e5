"""Both GPU forms against the FP64 oracle at the headline configuration: n = 20 000
samples, intercept only, all tests (-lmm 4), 1 % missing calls.

The cohort's eigendecomposition comes from the device (the oracle is handed the same
eigenvalues and eigenvectors, as jamma's runner is when eigen files are given), and 64 SNPs
with four strong causal effects are tested by the plain FP64 form, the mixed form (INT8
tcgen05 rotation, series-interpolated lambda search) and jamma's path restated in NumPy
(src/jamma/lmm/runner_streaming.py:392-586, likelihood_jax.py:491-798).

* plain form: on every SNP whose REML (MLE) lambda matches the oracle's to 1e-12 -- every
  golden-section decision taken the same way, at least half of the SNPs -- beta, se,
  logl_H1 and p_wald (logl_mle) agree to 1e-10 relative and p_lrt to 1e-8 (it also carries
  the null model's logl_H0, whose own golden search can end one step apart at an FP64 tie);
  with the oracle's null lambda0, every p_score agrees to 1e-10;
  lambda itself always within the golden bracket; identical calls at 5e-8.
* mixed form: every |log10 p| error below 1e-4 and identical calls at 5e-8; p within 1e-6
  relative for at least 98 % of SNPs (the rest are golden-section steps on flat
  likelihoods that a 1e-9 perturbation of the rotated genotypes resolves differently).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from _parity import assert_strict, strict_fp64_report
from jamma_b200 import synth
from oracle import lmm as OL
from oracle import plink as OP

pytestmark = pytest.mark.gpu

N, SNPS, KIN_SNPS, MISS = 20000, 64, 3000, 0.01


@pytest.fixture(scope="module")
def cohort20k():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build
    from jamma_b200 import engine as eng

    _build.build()
    gk = torch.from_numpy(synth.genotypes(N, KIN_SNPS, 0.0, seed=2020)).cuda()
    gk -= gk.mean(0, keepdim=True)
    K = gk @ gk.T / KIN_SNPS  # test set-up: a centered kinship of KIN_SNPS SNPs
    del gk
    w_d, U_d = eng.eigh_device(K)
    g = synth.genotypes(N, SNPS, MISS, seed=2021)
    gi = np.where(np.isnan(g), np.nanmean(g, axis=0, keepdims=True), g)
    y = synth.phenotypes(synth.genotypes(N, 400, 0.0, seed=2022), n_causal=20, h2=0.5, seed=2023)
    y = y + gi[:, :4] @ np.array([0.15, -0.1, 0.08, 0.06])  # four associated SNPs
    ref = OL.lmm_association(g, y, eigenvalues=w_d.cpu().numpy(),
                             eigenvectors=U_d.cpu().numpy().T, lmm_mode=4, maf_threshold=0.0,
                             miss_threshold=1.0)
    return w_d, U_d, g, y, ref


def _run(cohort20k, precision):
    from jamma_b200 import engine as eng
    from jamma_b200.lmm import associate_records

    w_d, U_d, g, y, _ = cohort20k
    cohort = eng.DeviceCohort(w_d, U_d, None, y, lmm_mode=4, precision=precision)
    mu32 = np.nanmean(g.astype(np.float32), axis=0).astype(np.float64)
    out = associate_records(cohort, OP.encode_genotypes(g), N, None, mu32,
                            n_miss=np.isnan(g).sum(0))
    return {k: v[0] for k, v in out.items()}, float(cohort.null_model()[0][0])


def _pvalue_checks(got, ref, strict_frac):
    fracs = {}
    for k in ("p_wald", "p_lrt", "p_score"):
        a, b = np.asarray(got[k]), ref.stats[k]
        np.testing.assert_array_equal(np.isfinite(a), np.isfinite(b), err_msg=f"{k}: NaN pattern")
        ok = np.isfinite(a)
        dlog = np.abs(np.log10(a[ok]) - np.log10(b[ok]))
        assert dlog.max() < 1e-4, f"{k}: |dlog10 p| {dlog.max():.2e}"
        np.testing.assert_array_equal(a[ok] < 5e-8, b[ok] < 5e-8, err_msg=f"{k}: calls at 5e-8")
        fracs[k] = float(np.mean(np.abs(a[ok] - b[ok]) / b[ok] <= 1e-6))
        assert fracs[k] >= strict_frac, f"{k}: {fracs[k]:.3f} within 1e-6"
    return fracs


def test_headline_fp64_form_matches_oracle(cohort20k):
    got, lam0 = _run(cohort20k, "fp64")
    ref = cohort20k[4]
    assert np.any(ref.stats["p_wald"] < 5e-8), "the cohort should hold genome-wide hits"
    _pvalue_checks(got, ref, 0.98)
    reml = strict_fp64_report(got, ref.stats)
    mle = strict_fp64_report(got, ref.stats, keys=("logl_mle", "p_lrt"), lam_key="lambda_mle",
                             tols={"p_lrt": 1e-8})
    print(f"headline fp64 form vs oracle: {reml} {mle}")
    assert_strict(reml, 0.5, "REML")
    assert_strict(mle, 0.5, "MLE")
    for k in ("lambda_remle", "lambda_mle"):
        rel = np.abs(got[k] - ref.stats[k]) / ref.stats[k]
        assert rel.max() <= 1e-4, f"{k}: {rel.max():.2e} outside the golden bracket"
    if abs(lam0 - ref.lam0) <= 1e-12 * ref.lam0:
        a, b = got["p_score"], ref.stats["p_score"]
        assert np.max(np.abs(a - b) / b) <= 1e-10


def test_headline_mixed_form_matches_oracle(cohort20k):
    got, _ = _run(cohort20k, "mixed")
    _pvalue_checks(got, cohort20k[4], 0.98)
    beta = np.abs(got["beta"] - cohort20k[4].stats["beta"]) / np.abs(cohort20k[4].stats["beta"])
    assert np.median(beta) < 1e-6
