"""File formats kept from jamma: PLINK inputs, covariates, .cXX.txt kinship, .assoc.txt.

Host-side text and byte handling only.  Layouts follow jamma:
``src/jamma/io/plink.py`` (metadata), ``src/jamma/io/covariate.py:19-95``,
``src/jamma/kinship/io.py:9-67`` and ``src/jamma/lmm/io.py:12-262``.
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

BED_MAGIC = bytes([0x6C, 0x1B, 0x01])


# ---------------------------------------------------------------- PLINK
def _lines(path: Path) -> list[str]:
    with open(path) as f:
        return [line for line in f if line.strip()]


def get_plink_metadata(bfile) -> dict:
    """Dimensions and SNP/sample metadata (``get_plink_metadata``, plink.py:92-136)."""
    bed = Path(f"{bfile}.bed")
    if not bed.exists():
        raise FileNotFoundError(f"PLINK .bed file not found: {bed}")
    fam = [line.split() for line in _lines(Path(f"{bfile}.fam"))]
    bim = [line.split() for line in _lines(Path(f"{bfile}.bim"))]
    return {
        "n_samples": len(fam),
        "n_snps": len(bim),
        "iid": np.array([[r[0], r[1]] for r in fam]),
        "sid": np.array([r[1] for r in bim]),
        "chromosome": np.array([r[0] for r in bim]),
        "bp_position": np.array([int(r[3]) for r in bim]),
        "allele_1": np.array([r[4] for r in bim]),
        "allele_2": np.array([r[5] for r in bim]),
    }


def snp_info_from_meta(meta: dict) -> list[dict]:
    """``snp_info`` dicts as the streaming runner builds them (runner_streaming.py:172-182)."""
    return [
        {"chr": str(c), "rs": str(r), "pos": int(p), "a1": str(a1), "a0": str(a0)}
        for c, r, p, a1, a0 in zip(meta["chromosome"], meta["sid"], meta["bp_position"],
                                   meta["allele_1"], meta["allele_2"])
    ]


_READ_THREADS = 4
_READ_SPLIT_BYTES = 8 << 20
_READ_POOL = None


def _read_pool():
    global _READ_POOL
    if _READ_POOL is None:
        from concurrent.futures import ThreadPoolExecutor

        _READ_POOL = ThreadPoolExecutor(max_workers=_READ_THREADS, thread_name_prefix="jb-bed")
    return _READ_POOL


class BedFile:
    """Memory-mapped SNP-major .bed records: ``records[j]`` is SNP j's packed bytes."""

    def __init__(self, bfile, n_samples: int | None = None, n_snps: int | None = None):
        self.path = Path(f"{bfile}.bed")
        if not self.path.exists():
            raise FileNotFoundError(f"PLINK .bed file not found: {self.path}")
        if n_samples is None or n_snps is None:
            meta = get_plink_metadata(bfile)
            n_samples, n_snps = meta["n_samples"], meta["n_snps"]
        self.n_samples, self.n_snps = int(n_samples), int(n_snps)
        self.bytes_per_snp = (self.n_samples + 3) // 4
        # copy-on-write: the views handed to torch.from_numpy are writable, the file is never
        # written
        raw = np.memmap(self.path, dtype=np.uint8, mode="c")
        if raw.size < 3 or bytes(raw[:3]) != BED_MAGIC:
            raise ValueError(f"{self.path}: not a SNP-major PLINK .bed file")
        expect = 3 + self.bytes_per_snp * self.n_snps
        if raw.size != expect:
            raise ValueError(
                f"{self.path}: {raw.size} bytes, expected {expect} for "
                f"{self.n_samples} samples x {self.n_snps} SNPs"
            )
        self.records = raw[3:].reshape(self.n_snps, self.bytes_per_snp)
        self._fd = os.open(self.path, os.O_RDONLY)

    def __del__(self):
        fd = getattr(self, "_fd", None)
        if fd is not None:
            os.close(fd)

    def read(self, start: int, end: int) -> np.ndarray:
        return np.ascontiguousarray(self.records[start:end])

    def take(self, idx: np.ndarray) -> np.ndarray:
        return np.ascontiguousarray(self.records[np.asarray(idx)])

    def _pread(self, mv: memoryview, off: int) -> None:
        done = 0
        while done < len(mv):
            got = os.preadv(self._fd, [mv[done:]], off + done)
            if got <= 0:
                raise OSError(f"{self.path}: short read at byte {off + done}")
            done += got

    def read_into(self, start: int, end: int, out: np.ndarray) -> None:
        """Records of SNPs start..end into the C-contiguous uint8 array ``out`` (e.g. a
        pinned staging buffer) by positioned reads -- far faster than touching the memory
        map page by page -- split over a few threads for large reads (the reads release
        the GIL)."""
        mv = memoryview(out).cast("B")[: (end - start) * self.bytes_per_snp]
        off = 3 + start * self.bytes_per_snp
        parts = min(_READ_THREADS, len(mv) // _READ_SPLIT_BYTES)
        if parts <= 1:
            self._pread(mv, off)
            return
        step = -(-len(mv) // parts)
        futs = [_read_pool().submit(self._pread, mv[a:a + step], off + a)
                for a in range(0, len(mv), step)]
        for f in futs:
            f.result()

    def take_into(self, idx: np.ndarray, out: np.ndarray) -> None:
        """Copy the records of SNPs ``idx`` into ``out`` (len(idx), bytes_per_snp), one
        positioned read per run of consecutive SNPs."""
        idx = np.asarray(idx, dtype=np.int64)
        if idx.size == 0:
            return
        cut = np.flatnonzero(np.diff(idx) != 1) + 1
        starts = np.concatenate(([0], cut))
        ends = np.concatenate((cut, [idx.size]))
        for a, b in zip(starts.tolist(), ends.tolist()):
            self.read_into(int(idx[a]), int(idx[a]) + (b - a), out[a:b])


def read_snp_list_file(path) -> set[str]:
    """SNP ids of a GEMMA-style list file (``read_snp_list_file``,
    src/jamma/io/snp_list.py:13-49): the first whitespace-delimited token of every
    non-empty line.  Raises FileNotFoundError for a missing file and ValueError when the
    file holds no id."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"SNP list file not found: {path}")
    ids: set[str] = set()
    with open(path) as f:
        for line in f:
            tok = line.split()
            if tok:
                ids.add(tok[0])
    if not ids:
        raise ValueError(f"SNP list file is empty or contains no valid IDs: {path}")
    return ids


def resolve_snp_list_to_indices(snp_ids, bim_sids) -> np.ndarray:
    """Sorted .bim column indices of the listed ids, case-sensitive
    (``resolve_snp_list_to_indices``, src/jamma/io/snp_list.py:52-88).  Ids absent from the
    .bim are skipped; ValueError when none matches."""
    pos = {sid: i for i, sid in enumerate(bim_sids)}
    idx = sorted(pos[s] for s in snp_ids if s in pos)
    if not idx:
        raise ValueError(f"No SNPs from the list matched the BIM file (requested {len(snp_ids)} SNPs)")
    return np.array(idx, dtype=np.intp)


def apply_snp_list_mask(snp_mask: np.ndarray, indices, n_snps: int, label: str) -> None:
    """AND ``snp_mask`` in place with the listed indices (``apply_snp_list_mask``,
    src/jamma/core/snp_filter.py:15-33); ValueError for an index past the last SNP."""
    indices = np.asarray(indices, dtype=np.int64)
    if indices.size and indices.max() >= n_snps:
        raise ValueError(f"{label} index {indices.max()} out of range for {n_snps} SNPs")
    keep = np.zeros(n_snps, dtype=bool)
    keep[indices] = True
    snp_mask &= keep


def write_plink_records(prefix, records: np.ndarray, n_samples: int, chrom=None,
                        phenotypes=None) -> None:
    """Write a .bed/.bim/.fam triple from packed SNP-major records (p, ceil(n/4)) --
    e.g. records already in the device layout -- without decoding them."""
    records = np.ascontiguousarray(records, dtype=np.uint8)
    p, bps = records.shape
    if bps != (n_samples + 3) // 4:
        raise ValueError(f"records have {bps} bytes per SNP; {n_samples} samples need "
                         f"{(n_samples + 3) // 4}")
    with open(f"{prefix}.bed", "wb") as f:
        f.write(BED_MAGIC)
        records.tofile(f)
    with open(f"{prefix}.bim", "w") as f:
        f.writelines(f"{chrom[j] if chrom is not None else 1}\trs{j:07d}\t0\t{1000 * (j + 1)}\tA\tG\n"
                     for j in range(p))
    with open(f"{prefix}.fam", "w") as f:
        f.writelines(f"FAM{i:06d}\tIND{i:06d}\t0\t0\t0\t"
                     f"{'-9' if phenotypes is None else repr(float(phenotypes[i]))}\n"
                     for i in range(n_samples))


def encode_codes(genotypes: np.ndarray) -> np.ndarray:
    """(n, p) float genotypes -> (p, n) int8 codes: 0/1/2, 3 = missing (NaN).

    Raises ValueError for values other than 0, 1, 2 and NaN (the int8 device layout
    holds allele counts; jamma's own data path only produces these values).
    """
    g = np.asarray(genotypes)
    nan = np.isnan(g)
    ok = nan | (g == 0) | (g == 1) | (g == 2)
    if not np.all(ok):
        raise ValueError("genotypes must be allele counts 0/1/2 or NaN for missing")
    codes = np.where(nan, 3, np.nan_to_num(g, nan=0.0)).astype(np.int8)
    return np.ascontiguousarray(codes.T)


def read_phenotypes(bfile, column: int = 1) -> np.ndarray:
    """.fam phenotype column (1-based, ``-9``/``NA`` -> NaN) (pipeline.py:240-293)."""
    if column < 1:
        raise ValueError(f"phenotype_column must be >= 1 (1-based), got {column}")
    rows = [line.split() for line in _lines(Path(f"{bfile}.fam"))]
    col = 4 + column
    if col >= len(rows[0]):
        raise ValueError(f"phenotype_column {column} exceeds available columns in .fam file")
    vals = np.array([r[col] for r in rows])
    miss = np.isin(vals, ["-9", "NA"])
    vals[miss] = "0"
    y = vals.astype(np.float64)
    y[miss] = np.nan
    if not np.any(~np.isnan(y) & (y != -9)):
        raise ValueError("No samples with valid phenotypes")
    return y


def read_covariate_file(path) -> tuple[np.ndarray, np.ndarray]:
    """GEMMA covariate file: whitespace table, ``NA`` -> NaN (covariate.py:19-95)."""
    rows = [line.split() for line in _lines(Path(path))]
    if not rows:
        raise ValueError(f"Covariate file is empty: {path}")
    k = len(rows[0])
    cov = np.zeros((len(rows), k))
    ind = np.ones(len(rows), dtype=np.int32)
    for i, r in enumerate(rows):
        if len(r) != k:
            raise ValueError(
                f"Covariate file row {i + 1} has {len(r)} columns but expected {k} "
                "(based on first row)"
            )
        for j, v in enumerate(r):
            if v == "NA":
                cov[i, j] = np.nan
                ind[i] = 0
            else:
                try:
                    cov[i, j] = float(v)
                except ValueError as e:
                    raise ValueError(f"Covariate file row {i + 1}: cannot parse {v!r}") from e
    return cov, ind


# ---------------------------------------------------------------- kinship text
def read_kinship_matrix(path, n_samples: int | None = None) -> np.ndarray:
    """``.cXX.txt`` reader with the square / size / symmetry checks of kinship/io.py:9-39."""
    k = np.loadtxt(path, dtype=np.float64)
    if k.ndim != 2 or k.shape[0] != k.shape[1]:
        raise ValueError(f"Kinship matrix must be square, got shape {k.shape}")
    if n_samples is not None and k.shape[0] != n_samples:
        raise ValueError(
            f"Kinship matrix dimension {k.shape[0]} does not match expected n_samples={n_samples}"
        )
    if not np.allclose(k, k.T, rtol=1e-10):
        raise ValueError("Kinship matrix is not symmetric")
    return k


def write_kinship_matrix(k: np.ndarray, path) -> None:
    """``%.10g``, tab separated, no header (kinship/io.py:43-67)."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        for row in k:
            f.write("\t".join(f"{v:.10g}" for v in row) + "\n")


# ---------------------------------------------------------------- association text
def write_eigenvalues(eigenvalues: np.ndarray, path) -> None:
    """GEMMA .eigenD.txt: one value per line, 10 significant digits
    (src/jamma/lmm/eigen_io.py WriteVector format)."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        f.writelines(f"{v:.10g}\n" for v in np.asarray(eigenvalues, dtype=np.float64))


def write_eigenvectors(eigenvectors: np.ndarray, path) -> None:
    """GEMMA .eigenU.txt: tab-separated rows (sample i = row i, eigenvector j = column j),
    10 significant digits, no header."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        for row in np.asarray(eigenvectors, dtype=np.float64):
            f.write("\t".join(f"{v:.10g}" for v in row) + "\n")


def write_eigen_files(eigenvalues, eigenvectors, output_dir, prefix: str = "result"):
    """Write {prefix}.eigenD.txt and {prefix}.eigenU.txt; returns both paths."""
    d = Path(output_dir) / f"{prefix}.eigenD.txt"
    u = Path(output_dir) / f"{prefix}.eigenU.txt"
    write_eigenvalues(eigenvalues, d)
    write_eigenvectors(eigenvectors, u)
    return d, u


def read_eigen_files(eigenD_path, eigenU_path, n_samples: int | None = None):
    """Read and cross-check a GEMMA eigen-file pair (counts, squareness, n_samples)."""
    evals = np.loadtxt(eigenD_path, dtype=np.float64, ndmin=1)
    evecs = np.loadtxt(eigenU_path, dtype=np.float64, ndmin=2)
    if evecs.shape[0] != evecs.shape[1]:
        raise ValueError(f"Eigenvector matrix must be square, got shape {evecs.shape} "
                         f"from {eigenU_path}")
    if evals.shape[0] != evecs.shape[0]:
        raise ValueError(f"Eigenvalue count ({evals.shape[0]}) does not match eigenvector "
                         f"dimensions {evecs.shape}. Files may be mismatched: "
                         f"{eigenD_path}, {eigenU_path}")
    if n_samples is not None and evals.shape[0] != n_samples:
        raise ValueError(f"Eigenvalue count ({evals.shape[0]}) does not match expected "
                         f"n_samples={n_samples}. Eigen files may be from a different dataset.")
    return evals, evecs


def write_gemma_log(output_dir, prefix: str, params: dict, timing: dict, command_line: str,
                    version: str | None = None) -> Path:
    """GEMMA-style ``{prefix}.log.txt`` with ``##`` section lines (the layout of
    ``write_gemma_log``, src/jamma/utils/logging.py:51-117): version and date, command
    line, one ``## key = value`` line per parameter, one ``## key time = s seconds`` line
    per timing entry."""
    from datetime import datetime

    if version is None:
        from jamma_b200 import __version__ as version
    out = Path(output_dir)
    out.mkdir(parents=True, exist_ok=True)
    path = out / f"{prefix}.log.txt"
    lines = ["##", f"## JAMMA Version = {version}", f"## Date = {datetime.now().isoformat()}",
             "##", f"## Command Line Input = {command_line}", "##", "## Summary Statistics:"]
    lines += [f"## {k} = {v}" for k, v in params.items()]
    lines += ["##", "## Computation Time:"]
    lines += [f"## {k} time = {v:.2f} seconds" if isinstance(v, float) else f"## {k} time = {v} seconds"
              for k, v in timing.items()]
    lines.append("##")
    path.write_text("\n".join(lines) + "\n")
    return path


@dataclass(slots=True)
class AssocResult:
    """One SNP's association record (``AssocResult``, src/jamma/lmm/stats.py:39-64)."""

    chr: str
    rs: str
    ps: int
    n_miss: int
    allele1: str
    allele0: str
    af: float
    beta: float
    se: float
    logl_H1: float | None = None
    l_remle: float | None = None
    p_wald: float | None = None
    p_score: float | None = None
    l_mle: float | None = None
    p_lrt: float | None = None


HEADER_WALD = "chr\trs\tps\tn_miss\tallele1\tallele0\taf\tbeta\tse\tlogl_H1\tl_remle\tp_wald"
HEADER_SCORE = "chr\trs\tps\tn_miss\tallele1\tallele0\taf\tbeta\tse\tp_score"
HEADER_LRT = "chr\trs\tps\tn_miss\tallele1\tallele0\taf\tl_mle\tp_lrt"
HEADER_ALL = (
    "chr\trs\tps\tn_miss\tallele1\tallele0\taf\t"
    "beta\tse\tlogl_H1\tl_remle\tl_mle\tp_wald\tp_lrt\tp_score"
)
_HEADERS = {"wald": HEADER_WALD, "score": HEADER_SCORE, "lrt": HEADER_LRT, "all": HEADER_ALL}
_STAT_FIELDS = {
    "wald": ("beta", "se", "logl_H1", "l_remle", "p_wald"),
    "score": ("beta", "se", "p_score"),
    "lrt": ("l_mle", "p_lrt"),
    "all": ("beta", "se", "logl_H1", "l_remle", "l_mle", "p_wald", "p_lrt", "p_score"),
}
MODE_TEST = {1: "wald", 2: "lrt", 3: "score", 4: "all"}


def format_assoc_line(r: AssocResult, test_type: str = "wald") -> str:
    """GEMMA line: meta, ``af:.3f``, statistics ``:.6e`` (lmm/io.py:12-135)."""
    head = [r.chr, r.rs, str(r.ps), str(r.n_miss), r.allele1, r.allele0, f"{r.af:.3f}"]
    return "\t".join(head + [f"{getattr(r, k):.6e}" for k in _STAT_FIELDS[test_type]])


def format_assoc_line_score(r: AssocResult) -> str:
    return format_assoc_line(r, "score")


def format_assoc_line_lrt(r: AssocResult) -> str:
    return format_assoc_line(r, "lrt")


def format_assoc_line_all(r: AssocResult) -> str:
    return format_assoc_line(r, "all")


def write_assoc_results(results: list[AssocResult], path, test_type: str = "wald") -> None:
    with IncrementalAssocWriter(path, test_type) as w:
        w.write_batch(results)


class IncrementalAssocWriter:
    """Streamed ``.assoc.txt`` writer (``IncrementalAssocWriter``, lmm/io.py:172-262)."""

    def __init__(self, path, test_type: str = "wald"):
        self.path = Path(path)
        self.test_type = test_type if test_type in _HEADERS else "wald"
        self._file = None
        self._count = 0

    def __enter__(self):
        self.path.parent.mkdir(parents=True, exist_ok=True)
        self._file = open(self.path, "w")
        self._file.write(_HEADERS[self.test_type] + "\n")
        return self

    def write(self, r: AssocResult) -> None:
        if self._file is None:
            raise RuntimeError("Writer not opened. Use as context manager.")
        self._file.write(format_assoc_line(r, self.test_type) + "\n")
        self._count += 1

    def write_batch(self, results) -> None:
        for r in results:
            self.write(r)

    def write_lines(self, lines: list[str]) -> None:
        if self._file is None:
            raise RuntimeError("Writer not opened. Use as context manager.")
        self._file.write("".join(s + "\n" for s in lines))
        self._count += len(lines)

    def __exit__(self, *exc) -> None:
        if self._file:
            self._file.close()
            self._file = None

    @property
    def count(self) -> int:
        return self._count


def pack_genotypes(genotypes: np.ndarray) -> np.ndarray:
    """(n, p) allele counts with NaN -> (p, ceil(n/4)) SNP-major .bed records.

    Inverse of the device decode (count-A1 codes 2 -> 00, missing -> 01, 1 -> 10,
    0 -> 11; padding samples -> 11).  Raises ValueError for other values.
    """
    g = np.asarray(genotypes)
    n, p = g.shape
    nan = np.isnan(g)
    if not np.all(nan | (g == 0) | (g == 1) | (g == 2)):
        raise ValueError("genotypes must be allele counts 0/1/2 or NaN for missing")
    bits = np.full((p, ((n + 3) // 4) * 4), 3, dtype=np.uint8)
    gt = g.T
    c = np.full(gt.shape, 3, dtype=np.uint8)
    c[gt == 2] = 0
    c[gt == 1] = 2
    c[nan.T] = 1
    bits[:, :n] = c
    packed = bits[:, 0::4] | (bits[:, 1::4] << 2) | (bits[:, 2::4] << 4) | (bits[:, 3::4] << 6)
    return np.ascontiguousarray(packed.astype(np.uint8))
