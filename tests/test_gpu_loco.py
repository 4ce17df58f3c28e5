"""LOCO kinship and association on the GPU against the oracle's restatement of jamma's
LOCO path (chromosome names sorted as strings, K_loco = (S_full - S_c)/(p - p_c),
per-chromosome float64 statistics over the analysed samples)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import kinship as OK
from oracle import lmm as OL
from oracle import plink as OP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


@pytest.fixture(scope="module")
def loco_cohort(tmp_path_factory):
    d = tmp_path_factory.mktemp("loco")
    n, p = 260, 900
    g = synth.genotypes(n, p, 0.01, seed=21)
    chroms = np.repeat(["1", "2", "10"], [300, 350, 250])
    y = synth.phenotypes(g, n_causal=8, h2=0.5, seed=22)
    y[[4, 100]] = np.nan
    cov = synth.covariates(n, 1, seed=23)
    OP.write_plink(d / "loco", g, phenotypes=y, chrom=chroms)
    return d / "loco", g, chroms, y, cov


@pytest.mark.parametrize("precision", ["int8", "fp64"])
def test_loco_kinship_matches_oracle(loco_cohort, precision):
    from jamma_b200.loco import compute_loco_kinship

    prefix, g, chroms, _, _ = loco_cohort
    got = [(c, K.cpu().numpy()) for c, K in compute_loco_kinship(prefix, 0.01, 0.05, chunk_size=200,
                                                                  precision=precision)]
    ref = list(OK.loco_kinships(g, chroms, 0.01, 0.05))
    assert [c for c, _ in got] == [c for c, _ in ref] == ["1", "10", "2"]
    for (_, a), (_, b) in zip(got, ref):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
        np.testing.assert_array_equal(a, a.T)


@pytest.mark.parametrize("mode", [1, 4])
def test_run_lmm_loco_matches_oracle(loco_cohort, mode):
    from jamma_b200.loco import run_lmm_loco

    prefix, g, chroms, y, cov = loco_cohort
    res = run_lmm_loco(prefix, y, covariates=cov, lmm_mode=mode)
    ref = OL.loco_association(g, y, chroms, covariates=cov, lmm_mode=mode)
    ref_idx = np.concatenate([r[1] for r in ref])
    np.testing.assert_array_equal([int(r.rs[2:]) for r in res], ref_idx)
    np.testing.assert_array_equal([r.n_miss for r in res], np.concatenate([r[3] for r in ref]))
    np.testing.assert_allclose([r.af for r in res], np.concatenate([r[2] for r in ref]), rtol=0,
                               atol=1e-15)
    keys = {"p_wald": "p_wald", "beta": "beta", "l_remle": "lambda_remle"}
    if mode == 4:
        keys.update(p_lrt="p_lrt", p_score="p_score")
    for field, key in keys.items():
        a = np.array([getattr(r, field) for r in res])
        b = np.concatenate([r[4][key] for r in ref])
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
        assert np.mean(rel < 1e-8) >= 0.99, f"{field}: worst {rel.max():.3e}"


def test_loco_needs_two_chromosomes(tmp_path):
    from jamma_b200.loco import run_lmm_loco

    g = synth.genotypes(50, 40, 0.0, seed=1)
    OP.write_plink(tmp_path / "one", g, chrom=["1"] * 40)
    with pytest.raises(ValueError, match="multiple chromosomes"):
        run_lmm_loco(tmp_path / "one", np.ones(50))


def test_int8_kinship_with_sample_subset_and_missing(tmp_path):
    from jamma_b200 import compute_kinship_from_bed

    g = synth.genotypes(180, 500, 0.03, seed=31)
    OP.write_plink(tmp_path / "s", g)
    sel = np.sort(np.random.default_rng(1).choice(180, 150, replace=False))
    k = compute_kinship_from_bed(tmp_path / "s", chunk_size=128, sample_idx=sel, precision="int8")
    ref = OK.centered_kinship(g[sel].astype(np.float32))
    assert np.abs(k - ref).max() <= 1e-10 * np.abs(ref).max()


def test_int8_kinship_is_bit_reproducible(tmp_path):
    """The sparse missing-call correction sums in SNP order, so repeated runs agree bitwise."""
    from jamma_b200 import compute_kinship_from_bed

    g = synth.genotypes(300, 2600, 0.05, seed=41)
    OP.write_plink(tmp_path / "r", g)
    k1 = compute_kinship_from_bed(tmp_path / "r", chunk_size=2600, precision="int8")
    k2 = compute_kinship_from_bed(tmp_path / "r", chunk_size=2600, precision="int8")
    np.testing.assert_array_equal(k1, k2)
