"""Host-side logic of the product package checked against the oracle (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from jamma_b200 import io as jio
from jamma_b200.kinship import filter_mask, snp_stats_from_counts
from jamma_b200.lmm import valid_sample_mask
from oracle import kinship as OK
from oracle import plink as OP


def _random_genotypes(n, p, miss, seed):
    rng = np.random.default_rng(seed)
    af = rng.uniform(0.05, 0.5, p)
    g = rng.binomial(2, af, size=(n, p)).astype(np.float64)
    g[rng.random((n, p)) < miss] = np.nan
    return g


@pytest.mark.parametrize("n", [1, 3, 4, 5, 100, 257])
def test_pack_matches_oracle_decode(n):
    g = _random_genotypes(n, 37, 0.05, n)
    packed = jio.pack_genotypes(g)
    back = OP.decode_packed(packed, n)
    np.testing.assert_array_equal(np.isnan(back), np.isnan(g))
    np.testing.assert_array_equal(np.nan_to_num(back, nan=-1), np.nan_to_num(g, nan=-1))


def test_pack_rejects_dosages():
    with pytest.raises(ValueError):
        jio.pack_genotypes(np.array([[0.5, 1.0]]))


def _counts(g):
    obs = ~np.isnan(g)
    return np.stack([obs.sum(0), np.nansum(g, 0), (g == 1).sum(0), (g == 2).sum(0)], 1).astype(np.int32)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stats_from_counts_match_numpy_nanmean(dtype):
    g = _random_genotypes(211, 400, 0.03, 7)
    g[:, 0] = np.nan  # all missing
    g[:, 1] = 1.0  # monomorphic
    g[:5, 2] = np.nan
    mean, miss, poly = snp_stats_from_counts(_counts(g), g.shape[0], dtype)
    ref_mean, ref_miss, ref_var = OK.snp_stats(g.astype(dtype))
    np.testing.assert_array_equal(mean, ref_mean)  # bit-exact
    np.testing.assert_array_equal(miss, ref_miss)
    np.testing.assert_array_equal(poly, ref_var > 0)
    m1, af1 = filter_mask(mean, miss, poly, g.shape[0], 0.01, 0.05)
    m2, af2 = OK.filter_mask(ref_mean, ref_miss, ref_var, g.shape[0], 0.01, 0.05)
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_array_equal(af1, af2)


def test_valid_sample_mask():
    y = np.array([1.0, np.nan, -9.0, 2.0, 3.0])
    cov = np.array([[1, 0.1], [1, 0.2], [1, 0.3], [1, np.nan], [1, 0.5]])
    np.testing.assert_array_equal(valid_sample_mask(y, None), [1, 0, 0, 1, 1])
    np.testing.assert_array_equal(valid_sample_mask(y, cov), [1, 0, 0, 0, 1])


def test_assoc_formats_and_writer(tmp_path):
    r = jio.AssocResult("1", "rs1", 1000, 0, "A", "G", 0.70512, 0.683, 0.153, -140.1, 1e-5, 2.1e-5,
                        4.2e-3, 1e5, 2.7e-4)
    assert jio.format_assoc_line(r) == (
        "1\trs1\t1000\t0\tA\tG\t0.705\t6.830000e-01\t1.530000e-01\t-1.401000e+02\t1.000000e-05\t"
        "2.100000e-05")
    assert jio.format_assoc_line(r, "lrt").endswith("\t0.705\t1.000000e+05\t2.700000e-04")
    assert len(jio.format_assoc_line(r, "all").split("\t")) == 15
    p = tmp_path / "x.assoc.txt"
    with jio.IncrementalAssocWriter(p, "score") as w:
        w.write(r)
    lines = p.read_text().splitlines()
    assert lines[0] == jio.HEADER_SCORE and len(lines) == 2 and w.count == 1


def test_kinship_and_covariate_io(tmp_path):
    k = np.array([[1.0, 0.123456789012], [0.123456789012, 2.0]])
    p = tmp_path / "k.cXX.txt"
    jio.write_kinship_matrix(k, p)
    assert p.read_text().splitlines()[0] == "1\t0.123456789"
    np.testing.assert_allclose(jio.read_kinship_matrix(p), k, rtol=1e-9)
    bad = tmp_path / "bad.txt"
    bad.write_text("1 2\n3 4\n")
    with pytest.raises(ValueError):
        jio.read_kinship_matrix(bad)
    c = tmp_path / "c.txt"
    c.write_text("1 0.5\n1 NA\n\n1 2\n")
    cov, ind = jio.read_covariate_file(c)
    assert cov.shape == (3, 2) and np.isnan(cov[1, 1]) and list(ind) == [1, 0, 1]


def test_bed_file_roundtrip(tmp_path):
    g = _random_genotypes(13, 9, 0.1, 3)
    OP.write_plink(tmp_path / "t", g)
    bed = jio.BedFile(tmp_path / "t")
    np.testing.assert_array_equal(bed.read(0, 9), OP.encode_genotypes(g))
    meta = jio.get_plink_metadata(tmp_path / "t")
    assert meta["n_samples"] == 13 and meta["n_snps"] == 9
    (tmp_path / "t.bed").write_bytes((tmp_path / "t.bed").read_bytes()[:-1])
    with pytest.raises(ValueError):
        jio.BedFile(tmp_path / "t")


def test_sd_from_counts_matches_imputed_variance():
    """sd per SNP from device counts == sqrt(mean(x_imputed^2) - mean^2) over all samples."""
    from jamma_b200.kinship import snp_sd_from_counts

    rng = np.random.default_rng(4)
    g = rng.binomial(2, 0.3, size=(50, 40)).astype(float)
    g[rng.random(g.shape) < 0.1] = np.nan
    g[:, 3] = 1.0  # monomorphic
    obs = ~np.isnan(g)
    gz = np.nan_to_num(g)
    counts = np.column_stack([obs.sum(0), gz.sum(0), (gz == 1).sum(0), (gz == 2).sum(0)])
    sd = snp_sd_from_counts(counts, 50)
    mu = np.nanmean(g, axis=0)
    gi = np.where(obs, g, mu)
    ref = np.sqrt(np.maximum(np.mean(gi**2, axis=0) - mu**2, 0))
    np.testing.assert_allclose(sd, ref, rtol=1e-13, atol=1e-15)
    assert sd[3] == 0.0


def test_bed_positioned_reads_match_the_records(tmp_path):
    """BedFile.read_into / take_into (positioned reads into a caller buffer, used to fill
    the pinned staging buffers) return the same bytes as the memory-mapped records, for
    runs of consecutive SNPs and scattered ones."""
    from jamma_b200.io import BedFile, write_plink_records

    rng = np.random.default_rng(3)
    rec = rng.integers(0, 256, size=(700, 26), dtype=np.uint8)
    write_plink_records(tmp_path / "c", rec, 101)
    bed = BedFile(tmp_path / "c")
    out = np.zeros((40, 26), dtype=np.uint8)
    bed.read_into(650, 690, out)
    np.testing.assert_array_equal(out, rec[650:690])
    idx = np.array([0, 1, 2, 9, 10, 300, 698, 699])
    got = np.zeros((idx.size, 26), dtype=np.uint8)
    bed.take_into(idx, got)
    np.testing.assert_array_equal(got, rec[idx])
    np.testing.assert_array_equal(bed.records[idx], rec[idx])
