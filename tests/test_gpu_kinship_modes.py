"""-gk 2 standardized kinship, -ksnps kinship subsets and eigen-file reuse on the GPU
against the oracle."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import kinship as OK
from oracle import plink as OP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


@pytest.mark.parametrize("n,p,miss", [(3, 2, 0.0), (120, 800, 0.03), (257, 1500, 0.0)])
def test_standardized_kinship_matches_oracle(n, p, miss):
    from jamma_b200 import compute_standardized_kinship

    if n == 3:
        g = np.array([[0.0, 2.0], [1.0, 1.0], [2.0, 0.0]])
    else:
        g = synth.genotypes(n, p, miss, seed=n)
    ref = OK.standardized_kinship(g)
    got = compute_standardized_kinship(g)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    np.testing.assert_array_equal(got, got.T)


def test_standardized_kinship_from_bed_and_filters(tmp_path):
    from jamma_b200 import compute_kinship_from_bed

    g = synth.genotypes(150, 1000, 0.02, seed=8)
    OP.write_plink(tmp_path / "s", g)
    got = compute_kinship_from_bed(tmp_path / "s", 0.05, 0.05, chunk_size=300, kinship_mode=2)
    ref = OK.standardized_kinship(g.astype(np.float32), maf_threshold=0.05, miss_threshold=0.05)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    with pytest.raises(ValueError, match="FP64"):
        compute_kinship_from_bed(tmp_path / "s", kinship_mode=2, precision="int8")


@pytest.mark.parametrize("precision", ["fp64", "int8"])
def test_ksnps_subset_kinship(tmp_path, precision):
    from jamma_b200 import compute_kinship_from_bed

    g = synth.genotypes(140, 900, 0.02, seed=9)
    OP.write_plink(tmp_path / "k", g)
    sub = np.sort(np.random.default_rng(2).choice(900, 300, replace=False))
    got = compute_kinship_from_bed(tmp_path / "k", chunk_size=128, ksnps_indices=sub,
                                   precision=precision)
    ref = OK.centered_kinship(g[:, sub].astype(np.float32))
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_eigen_files_roundtrip_gives_same_association(tmp_path):
    """gk -eigen writes GEMMA eigen files; lmm -d/-u with them reproduces lmm -k."""
    from jamma_b200 import cli
    from jamma_b200.io import read_eigen_files

    g = synth.genotypes(90, 400, 0.01, seed=10)
    y = synth.phenotypes(np.nan_to_num(g, nan=1.0), n_causal=4, h2=0.5, seed=11)
    OP.write_plink(tmp_path / "e", g, phenotypes=y)
    out = tmp_path / "out"
    assert cli.main(["-outdir", str(out), "-o", "kin", "gk", "-bfile", str(tmp_path / "e"),
                     "-gk", "1", "-eigen"]) == 0
    for suffix in ("cXX.txt", "eigenD.txt", "eigenU.txt", "log.txt"):
        assert (out / f"kin.{suffix}").exists(), suffix
    evals, evecs = read_eigen_files(out / "kin.eigenD.txt", out / "kin.eigenU.txt", 90)
    assert evecs.shape == (90, 90)
    log = (out / "kin.log.txt").read_text()
    assert "## Command Line Input =" in log and "## kinship_mode = 1" in log
    assert cli.main(["-outdir", str(out), "-o", "a", "lmm", "-bfile", str(tmp_path / "e"),
                     "-k", str(out / "kin.cXX.txt"), "-lmm", "4"]) == 0
    assert cli.main(["-outdir", str(out), "-o", "b", "lmm", "-bfile", str(tmp_path / "e"),
                     "-d", str(out / "kin.eigenD.txt"), "-u", str(out / "kin.eigenU.txt"),
                     "-lmm", "4"]) == 0
    a = np.loadtxt(out / "a.assoc.txt", skiprows=1, usecols=range(6, 15))
    b = np.loadtxt(out / "b.assoc.txt", skiprows=1, usecols=range(6, 15))
    # eigen files hold 10 significant digits: statistics agree to ~1e-7 relative
    np.testing.assert_allclose(b, a, rtol=2e-5, atol=1e-12)
    assert (out / "a.log.txt").exists()
