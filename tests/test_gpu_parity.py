"""GPU parity: the CUDA path against the CPU oracle on identical seeded inputs.

Tolerances (plain FP64 form): the device evaluates the same sequence of likelihoods as
jamma's JAX path; only the order of the length-n sums differs, so

- decode / counts / SNP sets / af / n_miss: bit-exact;
- kinship: 1e-10 relative to the largest entry;
- eigenvalues: 1e-10 relative to the largest; eigenvectors up to sign, 1e-8;
- lambda (l_remle, l_mle): 1e-9 relative for >= 99% of SNPs and within the golden
  section's own final bracket (1e-4 relative) for all -- a near tie fc ~ fd that
  the two summation orders resolve differently moves the bracket;
- beta, se, logl, p-values: 1e-8 relative for >= 99% of SNPs, every p-value within
  1e-6 relative or 1e-12 absolute of the oracle, and identical significance calls at
  0.05 / 1e-3 / 5e-8.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import kinship as OK
from oracle import lmm as OL
from oracle import plink as OP

from _parity import _arrays, assert_assoc_parity

pytestmark = pytest.mark.gpu

@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


# ------------------------------------------------------------------ decode
def test_decode_bed_matches_oracle():
    from jamma_b200.engine import decode_packed

    g = synth.genotypes(203, 157, 0.05, seed=11)
    packed = OP.encode_genotypes(g)
    sel = np.sort(np.random.default_rng(0).choice(203, 150, replace=False)).astype(np.int32)
    codes, counts = decode_packed(torch.from_numpy(packed).cuda(), 203,
                                  torch.from_numpy(sel).cuda(), 150, ld=160)
    codes = codes.cpu().numpy()
    counts = counts.cpu().numpy()
    gs = g[sel]
    exp = np.where(np.isnan(gs), 3, np.nan_to_num(gs)).T.astype(np.int8)
    np.testing.assert_array_equal(codes[:, :150], exp)
    assert np.all(codes[:, 150:] == 0)
    np.testing.assert_array_equal(counts[:, 0], (~np.isnan(gs)).sum(0))
    np.testing.assert_array_equal(counts[:, 1], np.nansum(gs, 0))
    np.testing.assert_array_equal(counts[:, 2], (gs == 1).sum(0))
    np.testing.assert_array_equal(counts[:, 3], (gs == 2).sum(0))


# all samples, no subset: 16 samples per thread from one record word (n = 29 with a partial
# last word, n = 208), 4 samples per thread (ld a multiple of 4), one sample per thread
@pytest.mark.parametrize("n,ld", [(29, 32), (208, 208), (203, 204), (201, 201)])
def test_decode_bed_all_samples_matches_oracle(n, ld):
    from jamma_b200.engine import decode_packed

    g = synth.genotypes(n, 131, 0.05, seed=n)
    packed = OP.encode_genotypes(g)
    codes, counts = decode_packed(torch.from_numpy(packed).cuda(), n, None, n, ld=ld)
    codes = codes.cpu().numpy()
    counts = counts.cpu().numpy()
    exp = np.where(np.isnan(g), 3, np.nan_to_num(g)).T.astype(np.int8)
    np.testing.assert_array_equal(codes[:, :n], exp)
    assert np.all(codes[:, n:] == 0)
    np.testing.assert_array_equal(counts[:, 0], (~np.isnan(g)).sum(0))
    np.testing.assert_array_equal(counts[:, 1], np.nansum(g, 0))
    np.testing.assert_array_equal(counts[:, 2], (g == 1).sum(0))
    np.testing.assert_array_equal(counts[:, 3], (g == 2).sum(0))


# ------------------------------------------------------------------ kinship
def test_kinship_gemma_fixture(gemma, gemma_geno):
    from jamma_b200 import compute_centered_kinship

    k = compute_centered_kinship(gemma_geno.astype(np.float32))
    np.testing.assert_allclose(k, OK.centered_kinship(gemma_geno.astype(np.float32)), rtol=0,
                               atol=1e-12)
    np.testing.assert_allclose(k, gemma["kinship"], rtol=1e-8, atol=1e-9)


@pytest.mark.parametrize("n,p,miss,maf", [(300, 2000, 0.02, 0.0), (129, 517, 0.1, 0.05)])
def test_kinship_synthetic_with_missing(n, p, miss, maf):
    from jamma_b200 import compute_centered_kinship

    g = synth.genotypes(n, p, miss, seed=n)
    g[:, 3] = 1.0  # monomorphic: always dropped
    k = compute_centered_kinship(g, maf_threshold=maf)
    ref = OK.centered_kinship(g, maf_threshold=maf)
    assert np.abs(k - ref).max() <= 1e-10 * np.abs(ref).max()
    np.testing.assert_array_equal(k, k.T)


def test_kinship_from_bed_matches(tmp_path):
    from jamma_b200 import compute_kinship_from_bed

    g = synth.genotypes(150, 700, 0.01, seed=5)
    OP.write_plink(tmp_path / "c", g)
    k = compute_kinship_from_bed(tmp_path / "c", chunk_size=128)
    ref = OK.centered_kinship(g.astype(np.float32))
    assert np.abs(k - ref).max() <= 1e-10 * np.abs(ref).max()


# ------------------------------------------------------------------ eigen
def test_eigh_matches_numpy():
    from jamma_b200 import eigendecompose_kinship

    g = synth.genotypes(240, 900, 0.0, seed=3)
    K = OK.centered_kinship(g)
    w, U = eigendecompose_kinship(K)
    wr, Ur = OL.eigh_threshold(K)
    assert np.abs(w - wr).max() <= 1e-10 * np.abs(wr).max()
    assert w[0] == 0.0  # centred kinship has a null vector, thresholded to exactly 0
    big = np.abs(wr) > 1e-6
    dots = np.abs(np.sum(U[:, big] * Ur[:, big], axis=0))
    np.testing.assert_allclose(dots, 1.0, atol=1e-8)
    np.testing.assert_allclose(U.T @ U, np.eye(240), atol=1e-10)


# ------------------------------------------------------------------ association
@pytest.mark.parametrize("mode", [1, 2, 3, 4])
@pytest.mark.parametrize("cov", [False, True])
def test_association_gemma_fixture(gemma, gemma_geno, mode, cov):
    from jamma_b200 import run_lmm_association_jax

    covariates = gemma["covariates"] if cov else None
    info = [{"chr": "1", "rs": f"rs{j}", "pos": j, "a1": "A", "a0": "G"} for j in range(500)]
    res = run_lmm_association_jax(gemma_geno.astype(np.float32), gemma["pheno"], gemma["kinship"],
                                  info, covariates=covariates, lmm_mode=mode)
    ref = OL.lmm_association(gemma_geno.astype(np.float32), gemma["pheno"], kinship=gemma["kinship"],
                             covariates=covariates, lmm_mode=mode)
    got = _arrays(res)
    keys = [k for k in got if k in ref.stats and not np.all(np.isnan(ref.stats[k]))]
    assert len(res) == 500 and keys
    assert_assoc_parity(got, ref.stats, keys)
    # and against GEMMA itself at jamma's tolerances
    case = ("cov_" if cov else "") + {1: "wald", 2: "lrt", 3: "score", 4: "all"}[mode]
    for col, key, tol in (("p_wald", "p_wald", 1e-4), ("p_lrt", "p_lrt", 1e-4),
                          ("p_score", "p_score", 1e-4), ("se", "se", 1e-5)):
        if f"{case}__{col}" in gemma and key in got:
            b = gemma[f"{case}__{col}"]
            assert np.all(np.abs(got[key] - b) <= 1e-12 + tol * np.abs(b)), col


@pytest.fixture(scope="module")
def cohort_files(tmp_path_factory):
    d = tmp_path_factory.mktemp("cohort")
    n, p = 420, 2600
    g = synth.genotypes(n, p, 0.01, seed=42)
    g[:, 10] = 0.0  # monomorphic -> filtered
    g[:, 11] = np.where(np.arange(n) < 2, 1.0, 0.0)  # maf < 0.01 -> filtered
    y = synth.phenotypes(g, n_causal=10, h2=0.5, seed=7)
    y[[3, 77]] = np.nan
    y[5] = -9.0
    cov = synth.covariates(n, 2, seed=9)
    cov[8, 1] = np.nan
    OP.write_plink(d / "coh", g, phenotypes=y)
    K = OK.centered_kinship(g.astype(np.float32))
    return d / "coh", g, y, cov, K


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_streaming_runner_matches_oracle(cohort_files, mode, tmp_path):
    from jamma_b200 import run_lmm_association_streaming

    prefix, g, y, cov, K = cohort_files
    res = run_lmm_association_streaming(prefix, y, kinship=K, covariates=cov, lmm_mode=mode,
                                        chunk_size=700)
    ref = OL.lmm_association(g, y, kinship=K, covariates=cov, lmm_mode=mode)
    assert len(res) == ref.snp_indices.size
    rs = np.array([int(r.rs[2:]) for r in res])
    np.testing.assert_array_equal(rs, ref.snp_indices)
    np.testing.assert_array_equal([r.af for r in res], ref.af)
    np.testing.assert_array_equal([r.n_miss for r in res], ref.n_miss)
    got = _arrays(res)
    keys = [k for k in got if k in ref.stats and not np.all(np.isnan(ref.stats[k]))]
    assert_assoc_parity(got, ref.stats, keys)
    # written file has the GEMMA layout
    out = tmp_path / "r.assoc.txt"
    run_lmm_association_streaming(prefix, y, kinship=K, covariates=cov, lmm_mode=mode,
                                  output_path=out)
    lines = out.read_text().splitlines()
    assert len(lines) == len(res) + 1


def _assert_mostly_equal(a, b, name, rtol=1e-12, frac=0.99):
    """Equal to rtol for >= frac of entries and within the golden bracket (1e-4) for all.

    The grid and bracket sums come from cuBLAS DGEMMs whose kernels (and so their last
    bits) depend on the chunk width; a last-bit change can flip a near-tied golden-section
    comparison, which moves lambda by at most the final bracket width.
    """
    a, b = np.asarray(a), np.asarray(b)
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b), err_msg=name)
    ok = ~np.isnan(a)
    rel = np.abs(a[ok] - b[ok]) / np.maximum(np.abs(b[ok]), 1e-300)
    assert np.mean(rel <= rtol) >= frac, f"{name}: {np.mean(rel <= rtol):.4f} within {rtol}, " \
        f"worst {rel.max():.3e}"
    if name.startswith("lambda"):
        assert rel.max() <= 1e-4, f"{name}: worst {rel.max():.3e}"


def test_chunking_and_phenotype_batching_are_invariant(cohort_files):
    """Per-SNP results do not depend on the chunk width or on the phenotype batch."""
    from jamma_b200 import engine as eng

    _, g, y, cov, K = cohort_files
    valid = ~np.isnan(y) & (y != -9) & ~np.isnan(cov).any(1)
    gv, yv, cv = g[valid], y[valid], cov[valid]
    w, U = OL.eigh_threshold(K[np.ix_(valid, valid)])
    y2 = np.column_stack([yv, yv[::-1], yv * 0.5 + 1.0])
    packed = OP.encode_genotypes(gv[:, :600])
    mu = np.nan_to_num(np.nanmean(gv[:, :600], 0))
    miss = np.isnan(gv[:, :600]).sum(0)
    from jamma_b200.lmm import associate_records

    for precision in ("fp64", "mixed"):
        multi = eng.DeviceCohort(w, U, cv, y2, lmm_mode=4, precision=precision)
        r_a = associate_records(multi, packed, gv.shape[0], None, mu, device_chunk=256, n_miss=miss)
        r_b = associate_records(multi, packed, gv.shape[0], None, mu, device_chunk=97, n_miss=miss)
        for k in r_a:
            _assert_mostly_equal(r_a[k], r_b[k], f"{k} ({precision}, chunking)")
        for f in range(3):
            # a single-phenotype cohort rotates y with a 1-column cuBLAS product instead of
            # a 3-column one, so U^T y may differ in the last bit
            single = eng.DeviceCohort(w, U, cv, y2[:, f], lmm_mode=4, precision=precision)
            r_s = associate_records(single, packed, gv.shape[0], None, mu, device_chunk=97,
                                    n_miss=miss)
            # ... and that last bit also reaches the null model (lambda0, logl_H0), whose
            # likelihood can be flat enough for a golden-section near tie: compare at the
            # 1e-6 relative tolerance of the p-values
            for k in r_s:
                _assert_mostly_equal(r_s[k][0], r_a[k][f], f"{k} ({precision}, phenotype {f})",
                                     rtol=1e-6)


def test_device_null_model_matches_oracle(cohort_files):
    from jamma_b200 import engine as eng

    _, g, y, cov, K = cohort_files
    valid = ~np.isnan(y) & (y != -9) & ~np.isnan(cov).any(1)
    w, U = OL.eigh_threshold(K[np.ix_(valid, valid)])
    c = eng.DeviceCohort(w, U, cov[valid], y[valid], lmm_mode=2)
    lam, logl = c.null_model()
    lr, llr = OL.null_model_mle(w, U.T @ cov[valid], U.T @ y[valid])
    np.testing.assert_allclose(lam[0], lr, rtol=1e-9)
    np.testing.assert_allclose(logl[0], llr, rtol=1e-12)


def test_errors_are_raised_like_jamma(cohort_files):
    from jamma_b200 import run_lmm_association_streaming

    prefix, g, y, cov, K = cohort_files
    with pytest.raises(ValueError):
        run_lmm_association_streaming(prefix, y, kinship=K, lmm_mode=5)
    with pytest.raises(ValueError):
        run_lmm_association_streaming(prefix, y)
    with pytest.raises(ValueError):
        run_lmm_association_streaming(prefix, y, eigenvalues=np.ones(3))
    assert run_lmm_association_streaming(prefix, y, kinship=K, maf_threshold=0.6) == []
