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
