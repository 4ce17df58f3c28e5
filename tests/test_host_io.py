"""Host-side file formats not covered elsewhere (no GPU): eigen files, .fam phenotypes,
the .log.txt writer, the per-test .assoc.txt line formatters and the int8 code layout."""

from __future__ import annotations

import numpy as np
import pytest

from jamma_b200 import io as jio


def test_eigen_files_round_trip_and_checks(tmp_path):
    rng = np.random.default_rng(1)
    w = np.array([0.0, 1.5e-3, 2.0, 12345.678901234])
    u = rng.standard_normal((4, 4))
    d_path, u_path = jio.write_eigen_files(w, u, tmp_path / "out", "run")
    assert d_path.name == "run.eigenD.txt" and u_path.name == "run.eigenU.txt"
    assert d_path.read_text().splitlines() == ["0", "0.0015", "2", "12345.6789"]
    first = u_path.read_text().splitlines()[0].split("\t")
    assert len(first) == 4 and first[0] == f"{u[0, 0]:.10g}"
    w2, u2 = jio.read_eigen_files(d_path, u_path, n_samples=4)
    np.testing.assert_allclose(w2, w, rtol=1e-9)
    np.testing.assert_allclose(u2, u, rtol=1e-9, atol=1e-12)
    with pytest.raises(ValueError, match="does not match expected"):
        jio.read_eigen_files(d_path, u_path, n_samples=5)
    (tmp_path / "bad.eigenU.txt").write_text("1\t2\t3\n4\t5\t6\n")
    with pytest.raises(ValueError, match="square"):
        jio.read_eigen_files(d_path, tmp_path / "bad.eigenU.txt")


def test_fam_phenotypes(tmp_path):
    (tmp_path / "c.fam").write_text("f1 i1 0 0 1 1.5 7\nf2 i2 0 0 2 -9 8\nf3 i3 0 0 1 NA 9\n")
    y = jio.read_phenotypes(tmp_path / "c")
    assert y[0] == 1.5 and np.isnan(y[1]) and np.isnan(y[2])
    np.testing.assert_array_equal(jio.read_phenotypes(tmp_path / "c", column=2), [7, 8, 9])
    with pytest.raises(ValueError, match="exceeds"):
        jio.read_phenotypes(tmp_path / "c", column=3)
    with pytest.raises(ValueError, match="1-based"):
        jio.read_phenotypes(tmp_path / "c", column=0)


def test_gemma_log(tmp_path):
    p = jio.write_gemma_log(tmp_path / "o", "run", {"n_samples": 10, "lmm_mode": 4},
                            {"kinship": 1.5, "lmm": 2}, "jamma lmm -bfile x", version="9.9")
    lines = p.read_text().splitlines()
    assert p.name == "run.log.txt" and lines[0] == "##" and lines[-1] == "##"
    assert "## JAMMA Version = 9.9" in lines
    assert "## Command Line Input = jamma lmm -bfile x" in lines
    assert "## n_samples = 10" in lines and "## lmm_mode = 4" in lines
    assert "## kinship time = 1.50 seconds" in lines and "## lmm time = 2 seconds" in lines


def test_assoc_formatters_per_test(tmp_path):
    r = jio.AssocResult("3", "rs9", 55, 2, "T", "C", 0.1234, -0.5, 0.25, -10.0, 0.3, 1e-3,
                        2e-3, 0.4, 3e-3)
    assert jio.format_assoc_line_score(r) == jio.format_assoc_line(r, "score")
    assert jio.format_assoc_line_lrt(r) == jio.format_assoc_line(r, "lrt")
    assert jio.format_assoc_line_all(r) == jio.format_assoc_line(r, "all")
    assert jio.format_assoc_line(r, "score").split("\t")[6:] == [
        "0.123", "-5.000000e-01", "2.500000e-01", "2.000000e-03"]
    assert jio.format_assoc_line(r, "all").split("\t")[7:] == [
        f"{v:.6e}" for v in (-0.5, 0.25, -10.0, 0.3, 0.4, 1e-3, 3e-3, 2e-3)]
    nan_row = jio.AssocResult("3", "rs9", 55, 2, "T", "C", 0.5, float("nan"), float("nan"),
                              l_mle=1.0, p_lrt=0.5)
    assert jio.format_assoc_line(nan_row, "lrt").endswith("\t0.500\t1.000000e+00\t5.000000e-01")
    path = tmp_path / "a.assoc.txt"
    jio.write_assoc_results([r, r], path, "all")
    lines = path.read_text().splitlines()
    assert lines[0] == jio.HEADER_ALL and len(lines) == 3
    assert len(lines[1].split("\t")) == len(jio.HEADER_ALL.split("\t")) == 15


def test_int8_code_layout():
    g = np.array([[0, 1, np.nan], [2, np.nan, 1]], dtype=np.float64)  # 2 samples x 3 SNPs
    codes = jio.encode_codes(g)
    assert codes.dtype == np.int8 and codes.shape == (3, 2)
    np.testing.assert_array_equal(codes, [[0, 2], [1, 3], [3, 1]])
    with pytest.raises(ValueError, match="allele counts"):
        jio.encode_codes(np.array([[0.5]]))


def test_chromosome_partitions_keep_first_appearance_order():
    from jamma_b200.loco import chromosome_partitions

    parts = chromosome_partitions(["2", "2", "10", "1", "10", "2"])
    assert list(parts) == ["2", "10", "1"]
    np.testing.assert_array_equal(parts["2"], [0, 1, 5])
    np.testing.assert_array_equal(parts["10"], [2, 4])
    assert sorted(parts) == ["1", "10", "2"]  # the string order LOCO processes them in


def test_eigen_warnings():
    import warnings

    from jamma_b200.eigen import _warn

    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        _warn(np.array([-1e-3, 0.0, 0.0, 1.0]), 1e-10)
    msgs = [str(x.message) for x in w]
    assert any("1 negative eigenvalue" in m for m in msgs)
    assert any("2 eigenvalues close to zero" in m for m in msgs)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        _warn(np.array([0.0, 0.5, 1.0]), 1e-10)  # one zero eigenvalue: no warning
    assert not w


def test_autotune_cache_survives_a_corrupt_file(tmp_path, monkeypatch):
    from jamma_b200 import autotune

    monkeypatch.setenv("JAMMA_B200_CACHE", str(tmp_path / "t" / "tune.json"))
    assert autotune._load() == {}
    autotune._store({"k": {"chunk": 4096}})
    assert autotune._load() == {"k": {"chunk": 4096}}
    autotune.cache_path().write_text("{not json")
    assert autotune._load() == {}
