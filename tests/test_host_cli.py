"""CLI argument and error handling that is decided on the host before any device work:
errors print ``Error: ...`` and return exit status 1 (jamma's src/jamma/cli.py:485-487)."""

from __future__ import annotations

import pytest

from jamma_b200 import cli


def _run(argv, capsys):
    rc = cli.main(argv)
    return rc, capsys.readouterr().err


def test_lmm_needs_a_kinship_source(capsys, tmp_path):
    rc, err = _run(["-outdir", str(tmp_path), "lmm", "-bfile", str(tmp_path / "x")], capsys)
    assert rc == 1 and err.startswith("Error: lmm needs -k, -d/-u or -loco")


def test_eigen_files_come_in_pairs(capsys, tmp_path):
    rc, err = _run(["-outdir", str(tmp_path), "lmm", "-bfile", str(tmp_path / "x"), "-d",
                    str(tmp_path / "a.eigenD.txt")], capsys)
    assert rc == 1 and "-d and -u must be given together" in err


def test_invalid_kinship_mode(capsys, tmp_path):
    rc, err = _run(["-outdir", str(tmp_path), "gk", "-bfile", str(tmp_path / "x"), "-gk", "3"],
                   capsys)
    assert rc == 1 and "invalid kinship mode 3" in err


def test_missing_bed_file(capsys, tmp_path):
    rc, err = _run(["-outdir", str(tmp_path), "gk", "-bfile", str(tmp_path / "nothere")], capsys)
    assert rc == 1 and err.startswith("Error: PLINK .bed file not found")


def test_unknown_precision_is_an_argument_error(capsys, tmp_path):
    with pytest.raises(SystemExit) as e:
        cli.main(["gk", "-bfile", str(tmp_path / "x"), "-precision", "fp16"])
    assert e.value.code == 2


@pytest.mark.parametrize("kwargs,msg", [
    ({"precision": "fp16"}, "precision must be"),
    ({"lmm_mode": 5}, "lmm_mode must be 1, 2, 3 or 4"),
    ({"loco": True, "kinship_file": "k.cXX.txt"}, "mutually exclusive"),
    ({"eigenvalue_file": "d.txt"}, "provided together"),
])
def test_gwas_argument_errors(kwargs, msg, tmp_path):
    """gwas() rejects inconsistent arguments with ValueError before reading any file
    (src/jamma/gwas.py:40-167)."""
    from jamma_b200.gwas import gwas

    with pytest.raises(ValueError, match=msg):
        gwas(tmp_path / "x", **kwargs)


def test_package_gwas_can_be_called_repeatedly(tmp_path):
    """``jamma_b200.gwas`` stays the function after the submodule has been imported (a
    lazily imported submodule would rebind the package attribute to itself)."""
    import jamma_b200
    import jamma_b200.gwas  # noqa: F401

    for _ in range(2):
        with pytest.raises(ValueError, match="lmm_mode"):
            jamma_b200.gwas(tmp_path / "x", lmm_mode=9)


def test_runner_argument_errors_come_before_the_device(tmp_path):
    """The association runners and the eigendecomposition check their arguments first, so
    a bad call raises jamma's ValueError (or FileNotFoundError) on any host."""
    import numpy as np

    from jamma_b200 import eigendecompose_kinship, run_lmm_association_jax
    from jamma_b200 import run_lmm_association_streaming as stream
    from jamma_b200.loco import run_lmm_loco

    y = np.zeros(4)
    with pytest.raises(ValueError, match="both eigenvalues and eigenvectors"):
        stream(tmp_path / "x", y, eigenvalues=np.ones(4))
    with pytest.raises(ValueError, match="Either kinship or pre-computed"):
        stream(tmp_path / "x", y)
    with pytest.raises(ValueError, match="lmm_mode"):
        stream(tmp_path / "x", y, kinship=np.eye(4), lmm_mode=0)
    with pytest.raises(ValueError, match="precision"):
        stream(tmp_path / "x", y, kinship=np.eye(4), precision="bf16")
    with pytest.raises(FileNotFoundError):
        stream(tmp_path / "x", y, kinship=np.eye(4))
    with pytest.raises(ValueError, match="lmm_mode"):
        run_lmm_association_jax(np.zeros((4, 2)), y, np.eye(4), [], lmm_mode=7)
    with pytest.raises(ValueError, match="square"):
        eigendecompose_kinship(np.ones((3, 4)))
    with pytest.raises(ValueError, match="lmm_mode"):
        run_lmm_loco(tmp_path / "x", y, lmm_mode=5)


def test_gwas_file_checks_before_the_device(tmp_path):
    """No valid phenotype, or eigen files of the wrong size, are errors before any device
    work (jamma's pipeline.py:286-291 and its n_samples cross-check of the eigen files)."""
    import numpy as np

    from jamma_b200.gwas import gwas
    from jamma_b200.io import write_eigen_files
    from oracle import plink as OP

    g = np.random.default_rng(0).binomial(2, 0.3, (6, 5)).astype(float)
    OP.write_plink(tmp_path / "a", g, phenotypes=np.full(6, -9.0))
    with pytest.raises(ValueError, match="No samples with valid phenotypes"):
        gwas(tmp_path / "a", kinship_file=tmp_path / "k.cXX.txt")
    OP.write_plink(tmp_path / "b", g, phenotypes=np.array([1.0, 2, np.nan, 4, 5, 6]))
    d, u = write_eigen_files(np.ones(6), np.eye(6), tmp_path, "e")
    with pytest.raises(ValueError, match="does not match expected"):
        gwas(tmp_path / "b", eigenvalue_file=d, eigenvector_file=u)


def test_no_cpu_fallback(tmp_path, monkeypatch):
    """Without a CUDA device the product path raises instead of computing on the host."""
    import numpy as np
    import torch

    from jamma_b200 import device
    from jamma_b200.kinship import compute_centered_kinship

    monkeypatch.setattr(device, "_checked", False)
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        device.require_cuda()
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        compute_centered_kinship(np.zeros((4, 3)))
