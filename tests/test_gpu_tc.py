"""tcgen05 INT8 tensor-core kernels: exactness of the Gram and the mixed kinship path."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import kinship as OK

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


def _gram(Z: np.ndarray) -> np.ndarray:
    """Run jb_gram_i8 on a host int8 (n, p) matrix; return the int32 upper triangle."""
    from jamma_b200 import _native
    from jamma_b200.device import ptr, stream_handle, workspace

    n, p = Z.shape
    ldz = (p + 127) // 128 * 128
    Zd = torch.zeros((n, ldz), dtype=torch.int8, device="cuda")
    Zd[:, :p] = torch.from_numpy(Z).cuda()
    C = torch.full((n, n), -7, dtype=torch.int32, device="cuda")
    ws = workspace(_native.load().jb_gram_i8_workspace_size(n))
    st = stream_handle()
    _native.call("jb_gram_i8", ptr(Zd), n, p, ldz, ptr(C), n, ptr(ws), ws.numel(), st)
    status = np.zeros(1, dtype=np.int32)
    _native.call("jb_gram_status", ptr(ws), status.ctypes.data, st)
    assert status[0] == 0, f"pipeline status {status[0]}"
    # C is column-major: C[j*n + i] holds (i, j), i <= j
    return C.cpu().numpy().T


@pytest.mark.parametrize("n,p", [(128, 128), (300, 1000), (1, 5), (129, 257), (513, 4096)])
def test_gram_i8_is_exact(n, p):
    rng = np.random.default_rng(n * 7 + p)
    Z = rng.integers(0, 3, size=(n, p), dtype=np.int8)
    got = _gram(Z)
    ref = Z.astype(np.int64) @ Z.T.astype(np.int64)
    iu = np.triu_indices(n)
    np.testing.assert_array_equal(got[iu], ref[iu])


def test_gram_i8_signed_extremes():
    rng = np.random.default_rng(3)
    Z = rng.choice(np.array([-128, -1, 0, 1, 127], dtype=np.int8), size=(200, 640))
    got = _gram(Z)
    ref = Z.astype(np.int64) @ Z.T.astype(np.int64)
    iu = np.triu_indices(200)
    np.testing.assert_array_equal(got[iu], ref[iu])


@pytest.mark.parametrize("n,p,miss", [(300, 2000, 0.0), (300, 2000, 0.02), (257, 777, 0.1)])
def test_int8_kinship_matches_oracle(n, p, miss):
    from jamma_b200 import compute_centered_kinship

    g = synth.genotypes(n, p, miss, seed=p + n)
    k = compute_centered_kinship(g, precision="int8")
    ref = OK.centered_kinship(g)
    assert np.abs(k - ref).max() <= 1e-10 * np.abs(ref).max()
    np.testing.assert_array_equal(k, k.T)


def test_int8_kinship_gemma_fixture(gemma, gemma_geno):
    from jamma_b200 import compute_centered_kinship

    k = compute_centered_kinship(gemma_geno.astype(np.float32), precision="int8")
    np.testing.assert_allclose(k, gemma["kinship"], rtol=1e-8, atol=1e-9)


def test_int8_kinship_from_bed(tmp_path):
    from jamma_b200 import compute_kinship_from_bed
    from oracle import plink as OP

    g = synth.genotypes(200, 900, 0.01, seed=9)
    OP.write_plink(tmp_path / "k", g)
    k = compute_kinship_from_bed(tmp_path / "k", chunk_size=256, precision="int8")
    ref = OK.centered_kinship(g.astype(np.float32))
    assert np.abs(k - ref).max() <= 1e-10 * np.abs(ref).max()


# ------------------------------------------------------------------ INT8 rotation
def _orthogonal(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n))
    _, u = np.linalg.eigh(a @ a.T)
    return u


@pytest.mark.parametrize("n,m,miss", [(300, 700, 0.02), (256, 512, 0.0), (97, 33, 0.1),
                                      (1000, 300, 0.01)])
def test_rotate_i8_matches_fp64(n, m, miss):
    from jamma_b200 import engine as eng
    from oracle import plink as OP

    U = _orthogonal(n, n + m)
    g = synth.genotypes(n, m, miss, seed=m)
    mu = np.nan_to_num(np.nanmean(g, axis=0)).astype(np.float32).astype(np.float64)
    gi = np.where(np.isnan(g), mu[None, :], g)
    ref = U.T @ gi
    cohort = eng.DeviceCohort(np.ones(n), U, None, np.zeros(n), lmm_mode=1, precision="mixed")
    codes, _ = eng.decode_packed(torch.from_numpy(OP.encode_genotypes(g)).cuda(), n, None, n,
                                 ld=cohort.code_ld)
    X = cohort.rotate_codes_i8(codes, torch.from_numpy(mu).cuda(), has_missing=miss > 0)
    assert cohort.rotate_status() == 0
    got = X.cpu().numpy().T
    # four base-254 digits: |U - split| <= 0.5 * 254^-3 * max|U_col| / 127 ~ 2.4e-10 max|U_col|
    bound = np.abs(U).max(axis=0)[:, None] * np.abs(gi).sum(axis=0)[None, :] * 2.0 ** -31
    assert np.all(np.abs(got - ref) <= bound + 1e-300)
    assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.parametrize("mode", [1, 4])
def test_mixed_association_matches_oracle(mode, tmp_path):
    from jamma_b200 import run_lmm_association_streaming
    from oracle import lmm as OL
    from oracle import plink as OP

    n, p = 500, 1500
    g = synth.genotypes(n, p, 0.01, seed=77)
    y = synth.phenotypes(g, n_causal=15, h2=0.6, seed=3)
    cov = synth.covariates(n, 2, seed=4)
    OP.write_plink(tmp_path / "m", g, phenotypes=y)
    K = OK.centered_kinship(g.astype(np.float32))
    res = run_lmm_association_streaming(tmp_path / "m", y, kinship=K, covariates=cov, lmm_mode=mode,
                                        precision="mixed")
    ref = OL.lmm_association(g, y, kinship=K, covariates=cov, lmm_mode=mode)
    keys = ("p_wald", "p_lrt", "p_score") if mode == 4 else ("p_wald",)
    for k in keys:
        a = np.array([getattr(r, k) for r in res])
        b = ref.stats[k]
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
        assert np.mean(rel < 1e-6) >= 0.99, f"{k}: worst {rel.max():.3e}"
        assert np.max(np.abs(np.log10(a) - np.log10(b))) < 1e-4
        for t in (0.05, 1e-3, 5e-8):
            np.testing.assert_array_equal(a < t, b < t)
    beta = np.array([r.beta for r in res])
    relb = np.abs(beta - ref.stats["beta"]) / np.abs(ref.stats["beta"])
    assert np.mean(relb < 1e-6) >= 0.99


@pytest.mark.parametrize("n_cvt,miss", [(1, 0.02), (2, 0.0)])
def test_series_sums_from_int8_calls_match_the_dgemm_form(n_cvt, miss):
    """Linear series sums formed from the int8 calls (basis U A_lin^T on the INT8 rotation
    core, precision 2) give the same statistics as the DGEMM over the rotated chunk
    (precision 1): both carry the 4-digit split's ~1e-9 relative error, so p-values agree
    to 1e-6 and significance calls exactly."""
    from jamma_b200 import engine as eng
    from oracle import plink as OP

    n, m = 640, 900
    g = synth.genotypes(n, m, miss, seed=5)
    K = np.corrcoef(np.nan_to_num(g, nan=1.0))
    w, U = np.linalg.eigh(K)
    y = synth.phenotypes(np.nan_to_num(g, nan=1.0), n_causal=10, h2=0.5, seed=6)
    cov = synth.covariates(n, n_cvt, seed=7)
    cohort = eng.DeviceCohort(np.where(np.abs(w) < 1e-10, 0.0, w), U, cov, y, lmm_mode=4,
                              precision="mixed")
    assert cohort.series_ws is not None
    mu = np.nan_to_num(np.nanmean(g, axis=0)).astype(np.float32).astype(np.float64)
    codes, _ = eng.decode_packed(torch.from_numpy(OP.encode_genotypes(g)).cuda(), n, None, n,
                                 ld=cohort.code_ld)
    means = torch.from_numpy(mu).cuda()
    X = cohort.rotate_codes_i8(codes, means, has_missing=miss > 0)
    got = {k: v.cpu().numpy() for k, v in cohort.associate_rotated(X).items()}  # precision 2
    assert cohort.rotate_status() == 0
    ref = {k: v.cpu().numpy() for k, v in cohort.associate_rotated(X).items()}  # precision 1
    for k in ("p_wald", "p_lrt", "p_score"):
        rel = np.abs(got[k] - ref[k]) / np.abs(ref[k])
        assert np.mean(rel < 1e-6) >= 0.99, f"{k}: worst {rel.max():.2e}"
        np.testing.assert_array_equal(got[k] < 5e-8, ref[k] < 5e-8)
        np.testing.assert_array_equal(got[k] < 1e-3, ref[k] < 1e-3)
    np.testing.assert_allclose(got["p_score"], ref["p_score"], rtol=1e-7)


@pytest.mark.parametrize("n,m,miss", [(300, 700, 0.02), (256, 512, 0.0), (97, 33, 0.1),
                                      (1000, 300, 0.01), (2500, 1100, 0.01)])
def test_rotate_pair_kernel_equals_single_cta_kernel(n, m, miss):
    """CTA-pair (cta_group::2, M = 256) rotation == one-CTA rotation, bit for bit; odd
    numbers of eigenvector blocks leave the second CTA of the last pair on zero rows."""
    from jamma_b200 import _native
    from jamma_b200 import engine as eng
    from oracle import plink as OP

    U = _orthogonal(n, 3 * n + m)
    g = synth.genotypes(n, m, miss, seed=n + m)
    mu = np.nan_to_num(np.nanmean(g, axis=0)).astype(np.float32).astype(np.float64)
    cohort = eng.DeviceCohort(np.ones(n), U, None, np.zeros(n), lmm_mode=1, precision="mixed")
    codes, _ = eng.decode_packed(torch.from_numpy(OP.encode_genotypes(g)).cuda(), n, None, n,
                                 ld=cohort.code_ld)
    means = torch.from_numpy(mu).cuda()
    prev = _native.load().jb_rotate_get_kernel()
    try:
        out = {}
        for variant in (0, 1):
            _native.call("jb_rotate_set_kernel", variant)
            out[variant] = cohort.rotate_codes_i8(codes, means, has_missing=miss > 0).cpu().numpy()
            assert cohort.rotate_status() == 0, variant
    finally:
        _native.call("jb_rotate_set_kernel", prev)
    np.testing.assert_array_equal(out[1], out[0])


@pytest.mark.parametrize("miss", [0.01, 0.05])
def test_tensor_core_and_sparse_missing_corrections_agree(miss, monkeypatch):
    """The missing-call correction on INT8 tensor cores (digit planes of mu) and the sparse
    walk give the same kinship, both within 1e-10 of the oracle."""
    from jamma_b200 import kinship as KM

    n, p = 700, 1024
    g = synth.genotypes(n, p, miss, seed=int(miss * 1000))
    ref = OK.centered_kinship(g)
    out = {}
    for name, thr in (("tc", 0.0), ("sparse", 2.0)):
        monkeypatch.setattr(KM, "TC_MISSING_DENSITY", thr)
        out[name] = KM.compute_centered_kinship(g, batch_size=256, precision="int8")
        assert np.abs(out[name] - ref).max() <= 1e-10 * np.abs(ref).max(), name
    # four base-254 digits carry mu_j to 4.8e-10; summed over a sample's missing SNPs and
    # divided by p that stays near 1e-11 of the kinship's scale
    assert np.abs(out["tc"] - out["sparse"]).max() <= 5e-11 * np.abs(ref).max()
    np.testing.assert_array_equal(out["tc"], out["tc"].T)
