"""PLINK 1 binary (.bed/.bim/.fam) restatement for the oracle.

jamma reads genotypes through bed-reader 1.0.6 (a Rust wheel pinned in the
reference's ``uv.lock:20``, called at ``src/jamma/io/plink.py:79,299``) with its
default ``count_A1=True``: the two-bit codes of a SNP-major .bed file map to
allele-1 counts ``00 -> 2, 01 -> missing (NaN), 10 -> 1, 11 -> 0``.  Sample ``i``
of a SNP lives in byte ``i // 4`` of that SNP's ``ceil(n/4)``-byte record, at
bit offset ``2 * (i % 4)``.  The file starts with the magic ``6c 1b 01``.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

BED_MAGIC = bytes([0x6C, 0x1B, 0x01])

# 2-bit code -> allele-1 count (count_A1=True); code 1 is missing.
_CODE_TO_COUNT = np.array([2.0, np.nan, 1.0, 0.0])


def _count_lines(path: Path) -> int:
    with open(path, "rb") as f:
        return sum(1 for line in f if line.strip())


def read_fam(prefix) -> list[list[str]]:
    """Rows of the .fam file (FID IID father mother sex pheno...)."""
    with open(f"{prefix}.fam") as f:
        return [line.split() for line in f if line.strip()]


def read_bim(prefix) -> list[dict]:
    """SNP metadata in the dict form jamma's runners use.

    Mirrors the ``snp_info`` built at ``src/jamma/lmm/runner_streaming.py:172-182``
    (chr, rs, pos, a1 = allele_1 = .bim column 5, a0 = allele_2 = column 6).
    """
    out = []
    with open(f"{prefix}.bim") as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            out.append({"chr": t[0], "rs": t[1], "pos": int(t[3]), "a1": t[4], "a0": t[5]})
    return out


def read_bed_packed(prefix) -> tuple[np.ndarray, int, int]:
    """Raw packed .bed records as a (p, ceil(n/4)) uint8 array."""
    n = _count_lines(Path(f"{prefix}.fam"))
    p = _count_lines(Path(f"{prefix}.bim"))
    raw = np.fromfile(f"{prefix}.bed", dtype=np.uint8)
    if raw.size < 3 or bytes(raw[:3]) != BED_MAGIC:
        raise ValueError(f"{prefix}.bed: not a SNP-major PLINK .bed file")
    bps = (n + 3) // 4
    if raw.size != 3 + bps * p:
        raise ValueError(
            f"{prefix}.bed: size {raw.size} does not match {n} samples x {p} SNPs"
        )
    return raw[3:].reshape(p, bps), n, p


def decode_packed(packed: np.ndarray, n: int, dtype=np.float64) -> np.ndarray:
    """Decode (p, ceil(n/4)) packed records to an (n, p) allele-1 count matrix."""
    p = packed.shape[0]
    codes = np.empty((p, packed.shape[1] * 4), dtype=np.uint8)
    for k in range(4):
        codes[:, k::4] = (packed >> (2 * k)) & 3
    g = _CODE_TO_COUNT[codes[:, :n]].T.astype(dtype)
    return np.ascontiguousarray(g)


def read_bed(prefix, dtype=np.float64, start: int = 0, end: int | None = None) -> np.ndarray:
    """(n, p) genotypes with NaN for missing, optionally a SNP window [start, end)."""
    packed, n, p = read_bed_packed(prefix)
    end = p if end is None else end
    return decode_packed(packed[start:end], n, dtype)


def encode_genotypes(g: np.ndarray) -> np.ndarray:
    """Inverse of :func:`decode_packed`: (n, p) counts with NaN -> (p, ceil(n/4)) bytes."""
    n, p = g.shape
    codes = np.full((p, ((n + 3) // 4) * 4), 3, dtype=np.uint8)  # pad with "0 copies"
    gt = g.T
    c = np.full(gt.shape, 1, dtype=np.uint8)  # missing
    c[gt == 2] = 0
    c[gt == 1] = 2
    c[gt == 0] = 3
    codes[:, :n] = c
    packed = np.zeros((p, codes.shape[1] // 4), dtype=np.uint8)
    for k in range(4):
        packed |= (codes[:, k::4] << (2 * k)).astype(np.uint8)
    return packed


def write_plink(prefix, g: np.ndarray, phenotypes=None, chrom=None, rs=None) -> None:
    """Write a .bed/.bim/.fam triple (used to materialise synthetic cohorts)."""
    n, p = g.shape
    packed = encode_genotypes(g)
    with open(f"{prefix}.bed", "wb") as f:
        f.write(BED_MAGIC)
        f.write(packed.tobytes())
    with open(f"{prefix}.bim", "w") as f:
        for j in range(p):
            c = chrom[j] if chrom is not None else 1
            r = rs[j] if rs is not None else f"rs{j:07d}"
            f.write(f"{c}\t{r}\t0\t{1000 * (j + 1)}\tA\tG\n")
    with open(f"{prefix}.fam", "w") as f:
        for i in range(n):
            ph = "-9" if phenotypes is None else repr(float(phenotypes[i]))
            f.write(f"FAM{i:06d}\tIND{i:06d}\t0\t0\t0\t{ph}\n")
