"""Centered (GEMMA -gk 1) and standardized (-gk 2) kinship on the GPU.

``compute_centered_kinship`` keeps jamma's signature and semantics
(src/jamma/kinship/compute.py:93-226): SNPs are filtered by MAF / missing rate /
monomorphism with statistics in the input dtype, each kept SNP is mean-imputed and
centred with its float64 mean over observed samples, and K = Xc Xc^T / p_kept.
Genotypes travel to the device as packed 2-bit records and are decoded there.
"""

from __future__ import annotations

import numpy as np
import torch

from jamma_b200 import _native
from jamma_b200.device import empty, ptr, require_cuda, stream_handle, workspace
from jamma_b200.engine import decode_packed, pass1_counts
from jamma_b200.io import BedFile, apply_snp_list_mask, pack_genotypes


def snp_stats_from_counts(counts: np.ndarray, n: int, dtype=np.float32):
    """(mean, miss, polymorphic) from device counts {n_obs, sum, n_het, n_hom2}.

    The mean is NumPy's ``nanmean`` in ``dtype``: the integer sum divided by the count
    in float64, then stored in ``dtype`` (0 for all-missing SNPs).  ``polymorphic`` is
    ``nanvar > 0``: at least two different observed genotypes.
    """
    n_obs = counts[:, 0].astype(np.int64)
    s = counts[:, 1].astype(np.float64)
    het = counts[:, 2].astype(np.int64)
    hom2 = counts[:, 3].astype(np.int64)
    hom0 = n_obs - het - hom2
    with np.errstate(invalid="ignore", divide="ignore"):
        mean = np.where(n_obs > 0, s / np.maximum(n_obs, 1), 0.0).astype(dtype)
    poly = ((hom0 > 0).astype(int) + (het > 0) + (hom2 > 0)) >= 2
    return mean, (n - n_obs).astype(np.int64), poly


def snp_sd_from_counts(counts: np.ndarray, n: int) -> np.ndarray:
    """Per-SNP standard deviation of the mean-imputed genotypes over all n samples, as
    ``impute_center_and_standardize`` forms it (src/jamma/kinship/missing.py:102-108):
    var = mean(x_imputed^2) - mean^2 with the float64 mean over observed samples."""
    n_obs = counts[:, 0].astype(np.float64)
    s = counts[:, 1].astype(np.float64)
    sq = counts[:, 2].astype(np.float64) + 4.0 * counts[:, 3].astype(np.float64)
    mu = np.where(n_obs > 0, s / np.maximum(n_obs, 1), 0.0)
    var = (sq + (n - n_obs) * mu * mu) / n - mu * mu
    return np.sqrt(np.maximum(var, 0.0))


def filter_mask(mean, miss, poly, n, maf_threshold, miss_threshold):
    """``compute_snp_filter_mask`` (src/jamma/core/snp_filter.py:59-91)."""
    af = np.asarray(mean, dtype=np.float64) / 2.0
    maf = np.minimum(af, 1.0 - af)
    keep = (maf >= maf_threshold) & ((miss / n) <= miss_threshold) & poly
    return keep, af


class _KinshipAccumulator:
    """FP64 centered (or, given per-SNP sd, standardized) Gram accumulated over SNP
    batches (``_accumulate_kinship``)."""

    def __init__(self, n: int, batch: int):
        self.n, self.batch = n, batch
        self.K = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        self.ws = workspace(_native.load().jb_kinship_f64_workspace_size(n, batch))
        self.p = 0

    def add(self, codes: torch.Tensor, means64: torch.Tensor, sd64: torch.Tensor | None = None) -> None:
        m, ld = codes.shape
        for s in range(0, m, self.batch):
            e = min(s + self.batch, m)
            if sd64 is None:
                _native.call("jb_kinship_accumulate_f64", ptr(codes[s:e]), ld, self.n, e - s,
                             ptr(means64[s:e]), ptr(self.K), self.n, ptr(self.ws), self.ws.numel(),
                             stream_handle())
            else:
                _native.call("jb_kinship_accumulate_std_f64", ptr(codes[s:e]), ld, self.n, e - s,
                             ptr(means64[s:e]), ptr(sd64[s:e]), ptr(self.K), self.n, ptr(self.ws),
                             self.ws.numel(), stream_handle())
        self.p += m

    def finish(self) -> torch.Tensor:
        _native.call("jb_kinship_finalize", ptr(self.K), self.n, self.n, 1.0 / self.p,
                     stream_handle())
        return self.K


# Missing-call density (fraction of a chunk's calls) above which the correction terms run
# on the INT8 tensor cores instead of the FP64 walk over each sample's missing SNPs.
TC_MISSING_DENSITY = 0.03


class _KinshipI8:
    """Exact INT8 tensor-core Gram + FP64 centring / missing-call corrections.

    MAX_CHUNK: SNPs per correction call (longer chunks are split).

    SNP chunks are transposed into the sample-major int8 operand (missing -> 0) and
    their correction vectors accumulated; ``finish`` runs the tcgen05 Gram once over all
    kept SNPs and combines the terms (see jb_gram.cu for the identity used).
    """

    MAX_CHUNK = 16384

    def __init__(self, n: int, p_kept: int):
        self.n, self.p = n, p_kept
        self.ldz = (p_kept + 127) // 128 * 128
        self.Zs = torch.zeros((n, self.ldz), dtype=torch.int8, device="cuda")
        self.a = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.b = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.RT = None
        self.sum_mu2 = 0.0
        self.col = 0
        self._status: list[torch.Tensor] = []
        self._density_scale = 1.0

    def add(self, codes: torch.Tensor, mu64: torch.Tensor, has_missing: bool,
            n_missing: int | None = None) -> None:
        """Add a chunk of decoded codes (m, ld).  ``n_missing``: the chunk's number of
        missing calls (from pass-1 counts; counted on the device when not given); chunks
        whose missing calls exceed TC_MISSING_DENSITY take the tensor-core correction."""
        m, ld = codes.shape
        if has_missing and n_missing is None:
            n_missing = int((codes[:, : self.n] == 3).sum())
        if m > self.MAX_CHUNK:  # the correction kernels take at most MAX_CHUNK SNPs per call
            for s in range(0, m, self.MAX_CHUNK):
                e = min(s + self.MAX_CHUNK, m)
                # the density test uses the whole chunk's average
                self._density_scale = m / (e - s)
                self.add(codes[s:e], mu64[s:e], has_missing, n_missing)
            self._density_scale = 1.0
            return
        st = stream_handle()
        if has_missing and self.RT is None:
            self.RT = torch.zeros((self.n, self.n), dtype=torch.float64, device="cuda")
        _native.call("jb_codes_to_sample_major", ptr(codes), ld, self.n, m, ptr(self.Zs), self.ldz,
                     self.col, None, 0, st)
        lib = _native.load()
        if has_missing and self.col % 16 == 0 and \
                n_missing > TC_MISSING_DENSITY * self.n * m * self._density_scale:
            ws = workspace(lib.jb_kinship_i8_tc_workspace_size(self.n, m))
            _native.call("jb_kinship_i8_corrections_tc", ptr(codes), ld, ptr(self.Zs), self.ldz,
                         self.col, self.n, m, ptr(mu64), ptr(self.a), ptr(self.b),
                         ptr(self.RT), self.n, ptr(ws), ws.numel(), st)
        else:
            ws = workspace(lib.jb_kinship_i8_corrections_workspace_size(self.n, m))
            _native.call("jb_kinship_i8_corrections", ptr(codes), ld, int(has_missing), self.n, m,
                         ptr(mu64), ptr(self.a), ptr(self.b), ptr(self.RT), self.n, ptr(ws),
                         ws.numel(), st)
        if has_missing:
            self._status.append(ws[:4].clone())  # status word, checked in finish()
        self.col += m

    def add_sum_mu2(self, mu64_host: np.ndarray) -> None:
        self.sum_mu2 += float(np.sum(np.asarray(mu64_host, dtype=np.float64) ** 2))

    def gram(self) -> torch.Tensor:
        """Exact int32 Gram of the accumulated calls (upper triangle, column-major)."""
        n = self.n
        st = stream_handle()
        C = torch.empty((n, n), dtype=torch.int32, device="cuda")
        ws = workspace(_native.load().jb_gram_i8_workspace_size(n))
        _native.call("jb_gram_i8", ptr(self.Zs), n, self.p, self.ldz, ptr(C), n, ptr(ws), ws.numel(), st)
        status = np.zeros(1, dtype=np.int32)
        _native.call("jb_gram_status", ptr(ws), status.ctypes.data, st)
        if status[0] != 0:
            raise RuntimeError(f"INT8 Gram pipeline reported status {int(status[0])}")
        self.Zs = None  # the operand is no longer needed
        return C

    def finish(self) -> torch.Tensor:
        n = self.n
        if self._status:
            st = torch.cat(self._status).view(torch.int32).cpu().numpy()
            if np.any(st != 0):
                raise RuntimeError(f"tensor-core kinship correction reported status {st[st != 0][0]}")
        C = self.gram()
        K = torch.empty((n, n), dtype=torch.float64, device="cuda")
        _native.call("jb_kinship_i8_finalize", ptr(C), n, n, ptr(self.a), ptr(self.b), self.sum_mu2,
                     ptr(self.RT), n, self.p, ptr(K), n, stream_handle())
        return K


def _kinship_from_packed(packed_dev: torch.Tensor, n: int, batch_size: int, maf_threshold: float,
                         miss_threshold: float, stat_dtype, precision: str = "fp64",
                         standardized: bool = False) -> tuple[torch.Tensor, int]:
    codes, counts = decode_packed(packed_dev, n, None, n)
    mean, miss, poly = snp_stats_from_counts(counts.cpu().numpy(), n, stat_dtype)
    keep, _ = filter_mask(mean, miss, poly, n, maf_threshold, miss_threshold)
    idx = np.where(keep)[0]
    if idx.size == 0:
        raise ValueError(
            f"No SNPs passed filtering (maf>={maf_threshold}, miss<={miss_threshold}, "
            f"polymorphic). Original SNP count: {packed_dev.shape[0]}"
        )
    c = counts.cpu().numpy()[idx]
    mu64 = torch.from_numpy(c[:, 1] / np.maximum(c[:, 0], 1)).to("cuda")  # float64 nanmean
    sel = torch.from_numpy(idx).to("cuda")
    if standardized:
        acc = _KinshipAccumulator(n, max(1, min(batch_size, 8192)))
        acc.add(codes.index_select(0, sel), mu64, torch.from_numpy(snp_sd_from_counts(c, n)).to("cuda"))
        return acc.finish(), idx.size
    if precision == "int8":
        acc = _KinshipI8(n, idx.size)
        acc.add(codes.index_select(0, sel), mu64, bool(np.any(c[:, 0] < n)),
                n_missing=int((n - c[:, 0]).sum()))
        acc.add_sum_mu2(c[:, 1] / np.maximum(c[:, 0], 1))
        return acc.finish(), idx.size
    acc = _KinshipAccumulator(n, max(1, min(batch_size, 8192)))
    acc.add(codes.index_select(0, sel), mu64)
    return acc.finish(), idx.size


def compute_standardized_kinship(genotypes: np.ndarray, batch_size: int = 10000,
                                 maf_threshold: float = 0.0, miss_threshold: float = 1.0,
                                 check_memory: bool = True) -> np.ndarray:
    """GEMMA -gk 2 relatedness matrix of an in-memory (n, p) genotype matrix.

    Keeps ``compute_standardized_kinship``'s signature and semantics
    (src/jamma/kinship/compute.py:229-360): the same SNP filter as -gk 1, then each kept
    SNP is mean-imputed, centred and divided by its standard deviation over all samples
    (``impute_center_and_standardize``, src/jamma/kinship/missing.py:64-119), and
    K = Z Z^T / p_kept.  FP64 on the device (per-SNP weights do not fit an exact integer
    Gram).
    """
    require_cuda()
    g = np.asarray(genotypes)
    n = g.shape[0]
    stat_dtype = np.float32 if g.dtype == np.float32 else np.float64
    packed = torch.from_numpy(pack_genotypes(g)).to("cuda")
    K, _ = _kinship_from_packed(packed, n, batch_size, maf_threshold, miss_threshold, stat_dtype,
                                "fp64", standardized=True)
    return K.cpu().numpy()


def compute_centered_kinship(genotypes: np.ndarray, batch_size: int = 10000,
                             maf_threshold: float = 0.0, miss_threshold: float = 1.0,
                             check_memory: bool = True, precision: str = "fp64") -> np.ndarray:
    """GEMMA -gk 1 relatedness matrix of an in-memory (n, p) genotype matrix.

    ``precision="fp64"`` accumulates the centred FP64 Gram (cuBLAS DSYRK);
    ``precision="int8"`` runs the exact INT8 tensor-core Gram with FP64 corrections.
    """
    if precision not in ("fp64", "int8"):
        raise ValueError("precision must be 'fp64' or 'int8'")
    require_cuda()
    g = np.asarray(genotypes)
    n = g.shape[0]
    stat_dtype = np.float32 if g.dtype == np.float32 else np.float64
    packed = torch.from_numpy(pack_genotypes(g)).to("cuda")
    K, _ = _kinship_from_packed(packed, n, batch_size, maf_threshold, miss_threshold, stat_dtype,
                                precision)
    return K.cpu().numpy()


def compute_kinship_from_bed(bfile, maf_threshold: float = 0.0, miss_threshold: float = 1.0,
                             chunk_size: int = 10000, sample_idx: np.ndarray | None = None,
                             as_device: bool = False, precision: str = "fp64",
                             kinship_mode: int = 1, ksnps_indices: np.ndarray | None = None):
    """Kinship streamed from a .bed file (``compute_kinship_streaming``,
    src/jamma/kinship/compute.py:502-690): pass 1 statistics, pass 2 accumulation,
    both decoded on the device.  Pass-1 means are float32 as in jamma's streaming path.

    ``kinship_mode`` 1 = centered (-gk 1), 2 = standardized (-gk 2, FP64 only);
    ``ksnps_indices`` restricts the kinship to those SNP columns (-ksnps).
    """
    if kinship_mode not in (1, 2):
        raise ValueError(f"invalid kinship mode {kinship_mode}; use 1 or 2")
    if kinship_mode == 2 and precision != "fp64":
        raise ValueError("standardized kinship (-gk 2) is computed in FP64 only")
    require_cuda()
    bed = BedFile(bfile)
    n = bed.n_samples if sample_idx is None else len(sample_idx)
    sidx = None if sample_idx is None else torch.from_numpy(
        np.asarray(sample_idx, dtype=np.int32)).to("cuda")
    counts = pass1_counts(bed, sidx, n, max(chunk_size, 16384))
    mean, miss, poly = snp_stats_from_counts(counts, n, np.float32)
    keep, _ = filter_mask(mean, miss, poly, n, maf_threshold, miss_threshold)
    if ksnps_indices is not None:
        apply_snp_list_mask(keep, ksnps_indices, keep.size, "Kinship SNP list")
    idx = np.where(keep)[0]
    if idx.size == 0:
        raise ValueError("No SNPs passed filtering")
    i8 = precision == "int8"
    acc = _KinshipI8(n, idx.size) if i8 else _KinshipAccumulator(n, min(chunk_size, 8192))
    for s in range(0, idx.size, chunk_size):
        sub = idx[s : s + chunk_size]
        rec = torch.from_numpy(bed.take(sub)).to("cuda")
        codes, _ = decode_packed(rec, bed.n_samples, sidx, n)
        c = counts[sub]
        mu64 = torch.from_numpy(c[:, 1] / np.maximum(c[:, 0], 1)).to("cuda")
        if i8:
            acc.add(codes, mu64, bool(np.any(c[:, 0] < n)), n_missing=int((n - c[:, 0]).sum()))
            acc.add_sum_mu2(c[:, 1] / np.maximum(c[:, 0], 1))
        elif kinship_mode == 2:
            acc.add(codes, mu64, torch.from_numpy(snp_sd_from_counts(c, n)).to("cuda"))
        else:
            acc.add(codes, mu64)
    K = acc.finish()
    return K if as_device else K.cpu().numpy()
