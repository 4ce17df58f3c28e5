"""Device-resident association engine.

A :class:`DeviceCohort` keeps one cohort on the GPU -- eigenvalues, eigenvectors,
rotated covariates and phenotypes, the per-phenotype null model and the prepared
lambda-grid tables -- so that any number of SNP chunks (and, in the serving loop,
new phenotypes or jobs) reuse them without another eigendecomposition.

Per chunk the pipeline is: packed .bed records -> ``jb_decode_bed`` (int8 codes +
per-SNP counts) -> ``jb_impute_f64`` (mean imputation, no centering) ->
``jb_rotate_f64`` (U^T G) -> ``jb_lmm_chunk`` (per-SNP search and statistics).
This restates ``run_lmm_association_streaming``'s device loop
(src/jamma/lmm/runner_streaming.py:412-586) with every step on the GPU.
"""

from __future__ import annotations

import numpy as np
import torch

from jamma_b200 import _native
from jamma_b200.device import colmajor, empty, ptr, require_cuda, stream_handle, workspace

OUT_KEYS = ("lambda_remle", "logl_h1", "beta", "se", "p_wald", "lambda_mle", "logl_mle",
            "p_lrt", "p_score")
MODE_KEYS = {
    1: ("lambda_remle", "logl_h1", "beta", "se", "p_wald"),
    2: ("lambda_mle", "logl_mle", "p_lrt"),
    3: ("beta", "se", "p_score"),
    4: OUT_KEYS,
}
MAX_CVT = 4

# The null model always runs with jamma's defaults: compute_null_model_mle is called
# without the user's lambda range (src/jamma/lmm/prepare.py:143).
NULL_L_MIN, NULL_L_MAX, NULL_N_GRID, NULL_N_ITER = 1e-5, 1e5, 50, 20
# log-lambda domain of the mixed form's series tables (jb_lmm_prepare precision 1)
SERIES_L_MIN, SERIES_L_MAX = 1e-5, 1e5


def eigh_device(K: torch.Tensor, threshold: float = 1e-10) -> tuple[torch.Tensor, torch.Tensor]:
    """In-place FP64 eigendecomposition of a device (n, n) symmetric matrix.

    Returns (eigenvalues (n,), eigenvectors as a column-major (n, n) tensor)."""
    require_cuda()
    n = K.shape[0]
    w = empty((n,))
    ws = workspace(_native.load().jb_eigh_workspace_size(n))
    _native.call("jb_eigh_f64", ptr(K), n, n, ptr(w), float(threshold), ptr(ws), ws.numel(),
                 stream_handle())
    return w, K


def rotate(U: torch.Tensor, B: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """U^T B for column-major U (n, n) and B (m, n) -> (m, n) column-major result."""
    n = U.shape[0]
    m = B.shape[0]
    if out is None:
        out = empty((m, n))
    _native.call("jb_rotate_f64", ptr(U), n, n, ptr(B), m, n, ptr(out), n, stream_handle())
    return out


def ozaki_split(U: torch.Tensor) -> torch.Tensor:
    """INT8 digit planes of column-major eigenvectors U (n, n) for the mixed rotation."""
    n = U.shape[0]
    oz = workspace(_native.load().jb_ozaki_workspace_size(n))
    _native.call("jb_ozaki_prepare", ptr(U), n, n, ptr(oz), oz.numel(), stream_handle())
    return oz


class DeviceCohort:
    """One cohort's resident state for association testing.

    Args:
        eigenvalues: (n,) thresholded eigenvalues (host array or device tensor).
        eigenvectors: (n, n) host array with eigenvectors as columns, or a device tensor
            already in column-major layout (as returned by :func:`eigh_device`).
        covariates: (n, c) host matrix W (c in 1..4), or None for an intercept.
        phenotypes: (n,) or (n, phi) host phenotypes (already restricted to analysed
            samples; every phenotype shares the sample set).
    """

    def __init__(self, eigenvalues, eigenvectors, covariates, phenotypes, lmm_mode=1,
                 l_min=1e-5, l_max=1e5, n_grid=50, n_refine=10, precision: str = "fp64",
                 ozaki: torch.Tensor | None = None):
        require_cuda()
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        if lmm_mode not in (1, 2, 3, 4):
            raise ValueError(f"lmm_mode must be 1, 2, 3 or 4, got {lmm_mode}")
        y = np.asarray(phenotypes, dtype=np.float64)
        if y.ndim == 1:
            y = y[:, None]
        n, phi = y.shape
        W = np.ones((n, 1)) if covariates is None else np.asarray(covariates, dtype=np.float64)
        if W.ndim == 1:
            W = W[:, None]
        c = W.shape[1]
        if n <= c + 1:
            raise ValueError(
                f"Over-parameterized model: {n} samples with {c} covariates leaves "
                f"df={n - c - 1} (need at least {c + 2} samples)"
            )
        if c > MAX_CVT:
            raise ValueError(f"at most {MAX_CVT} covariate columns are supported, got {c}")
        self.n, self.c, self.phi, self.mode = n, c, phi, lmm_mode
        self.l_min, self.l_max, self.n_grid = float(l_min), float(l_max), int(n_grid)
        self.n_iter = max(int(n_refine), 20)
        self.evals = (eigenvalues if isinstance(eigenvalues, torch.Tensor)
                      else colmajor(np.asarray(eigenvalues, dtype=np.float64)))
        self.U = (eigenvectors if isinstance(eigenvectors, torch.Tensor)
                  else colmajor(np.asarray(eigenvectors, dtype=np.float64)))
        if self.U.shape != (n, n) or self.evals.shape != (n,):
            raise ValueError("eigendecomposition does not match the number of samples")
        self.UtW = rotate(self.U, colmajor(W))
        self.Uty = rotate(self.U, colmajor(y))
        self.lam0 = self.logl0 = None
        st = stream_handle()
        if lmm_mode in (2, 3, 4):
            self.lam0 = empty((phi,))
            self.logl0 = empty((phi,))
            _native.call("jb_null_mle", n, c, phi, ptr(self.evals), ptr(self.UtW), n, ptr(self.Uty),
                         n, NULL_L_MIN, NULL_L_MAX, NULL_N_GRID, NULL_N_ITER, ptr(self.lam0),
                         ptr(self.logl0), st)
        self.ozaki = None
        if precision == "mixed":
            if ozaki is not None:  # digit planes shared with other users of the same cohort
                self.ozaki = ozaki
            else:
                self.ozaki = ozaki_split(self.U)
        self.code_ld = (n + 127) // 128 * 128 if precision == "mixed" else n
        self._rot_ws = None
        self._chunk_ws = None
        # The interpolated search expands 1/(lambda*eval + 1) in log lambda over the fixed
        # domain [1e-5, 1e5]: it needs the user's range inside that domain and no pole of
        # the weights near it; otherwise every probe is evaluated directly in FP64.
        ev_min = float(self.evals.min().item())
        self.search = 1 if (precision == "mixed" and 1.0 + SERIES_L_MAX * ev_min > 0.5
                            and self.l_min >= SERIES_L_MIN and self.l_max <= SERIES_L_MAX) else 0
        self.ws = workspace(_native.load().jb_lmm_workspace_size(n, c, phi, self.n_grid))
        _native.call("jb_lmm_prepare", lmm_mode, self.search, n, c, phi, ptr(self.evals), ptr(self.UtW), n,
                     ptr(self.Uty), n, ptr(self.lam0), self.l_min, self.l_max, self.n_grid,
                     ptr(self.ws), self.ws.numel(), st)
        # Mixed form with the series search: the linear genotype sums of each chunk come
        # from the int8 calls (basis U A_lin^T split into digit planes once per cohort).
        self.series_ws = None
        self._series_for = None
        series_rows = _native.load().jb_lmm_series_rows()  # ones row + series coefficients
        if self.search == 1 and series_rows * (c + phi) <= (n + 31) // 32 * 32:
            self.series_ws = workspace(_native.load().jb_lmm_series_workspace_size(n, c, phi))
            _native.call("jb_lmm_series_prepare", n, c, phi, self.n_grid, ptr(self.ws), self.ws.numel(),
                         ptr(self.U), n, ptr(self.series_ws), self.series_ws.numel(), st)

    # ------------------------------------------------------------ null model
    def null_model(self) -> tuple[np.ndarray | None, np.ndarray | None]:
        if self.lam0 is None:
            return None, None
        return self.lam0.cpu().numpy(), self.logl0.cpu().numpy()

    # ------------------------------------------------------------ per chunk
    def alloc_out(self, m: int) -> dict[str, torch.Tensor]:
        return {k: empty((self.phi, m)) for k in MODE_KEYS[self.mode]}

    def chunk_workspace(self, m: int) -> torch.Tensor:
        need = _native.load().jb_lmm_chunk_workspace_size(self.n, self.c, self.phi, self.n_grid, m)
        if self._chunk_ws is None or self._chunk_ws.numel() < need:
            self._chunk_ws = workspace(need)
        return self._chunk_ws

    def associate_rotated(self, UtG: torch.Tensor, out: dict | None = None) -> dict:
        """Statistics for a rotated chunk UtG (m, n) column-major; outputs (phi, m)."""
        m = UtG.shape[0]
        out = out if out is not None else self.alloc_out(m)
        o = _native.LmmOut(**{k: ptr(out.get(k)) for k in OUT_KEYS})
        cws = self.chunk_workspace(m)
        precision = self.search
        if self._series_for is not None and self._series_for == (m, UtG.data_ptr()):
            precision = 2  # linear sums already formed from this chunk's int8 calls
        self._series_for = None
        _native.call("jb_lmm_chunk", self.mode, precision, self.n, self.c, self.phi, m,
                     ptr(self.evals),
                     ptr(self.UtW), self.n, ptr(self.Uty), self.n, ptr(UtG), self.n,
                     ptr(self.lam0), ptr(self.logl0), self.l_min, self.l_max, self.n_grid,
                     self.n_iter, o, ptr(self.ws), self.ws.numel(), ptr(cws), cws.numel(),
                     stream_handle())
        return out

    def associate_genotypes(self, G: torch.Tensor, out: dict | None = None,
                            scratch: torch.Tensor | None = None) -> dict:
        """Rotate imputed genotypes G (m, n) and run the statistics."""
        UtG = rotate(self.U, G, out=scratch)
        return self.associate_rotated(UtG, out)

    def rotate_codes_i8(self, codes: torch.Tensor, means: torch.Tensor, has_missing: bool,
                        out: torch.Tensor | None = None, after_rotation=None) -> torch.Tensor:
        """Mixed form: INT8 tensor-core rotation of decoded codes -> U^T G (m, n) FP64.

        ``after_rotation`` (optional callable) runs between the rotation GEMM and the
        series-sum GEMM, e.g. to record a CUDA event that times the rotation alone."""
        m, ld = codes.shape
        need = _native.load().jb_rotate_i8_workspace_size(self.n, m)
        if self._rot_ws is None or self._rot_ws.numel() < need:
            self._rot_ws = workspace(need)
        out = out if out is not None else empty((m, self.n))
        _native.call("jb_rotate_i8", ptr(self.ozaki), self.n, ptr(codes), ld, m, ptr(means),
                     int(bool(has_missing)), ptr(out), self.n, ptr(self._rot_ws),
                     self._rot_ws.numel(), stream_handle())
        if after_rotation is not None:
            after_rotation()
        self._series_for = None
        if self.series_ws is not None:
            cws = self.chunk_workspace(m)
            _native.call("jb_lmm_chunk_series_i8", self.n, self.c, self.phi, self.n_grid, m,
                         ptr(self.series_ws), self.series_ws.numel(), ptr(codes), ld, ptr(means),
                         int(bool(has_missing)), ptr(self._rot_ws), self._rot_ws.numel(), ptr(cws),
                         cws.numel(), stream_handle())
            self._series_for = (m, out.data_ptr())
        return out

    def rotate_status(self) -> int:
        st = np.zeros(1, dtype=np.int32)
        if self._rot_ws is not None:
            _native.call("jb_rotate_status", ptr(self._rot_ws), st.ctypes.data, stream_handle())
        return int(st[0])

    def associate_codes(self, codes: torch.Tensor, means: torch.Tensor, out: dict | None = None,
                        bufs: dict | None = None, has_missing: bool = True) -> dict:
        """Decoded int8 codes (m, ld) + per-SNP imputation means (m,) -> statistics."""
        m, ld = codes.shape
        bufs = bufs if bufs is not None else {}
        if self.precision == "mixed":
            UtG = bufs.get("UtG")
            UtG = UtG[:m] if UtG is not None and UtG.shape[0] >= m else None
            return self.associate_rotated(self.rotate_codes_i8(codes, means, has_missing, UtG), out)
        G = bufs.get("G")
        if G is None or G.shape[0] < m:
            G = empty((m, self.n))
        G = G[:m]
        _native.call("jb_impute_f64", ptr(codes), ld, self.n, m, ptr(means), ptr(G), self.n,
                     stream_handle())
        UtG = bufs.get("UtG")
        UtG = UtG[:m] if UtG is not None and UtG.shape[0] >= m else None
        return self.associate_genotypes(G, out, UtG)


class ChunkGraph:
    """One chunk's device work captured as a CUDA graph over static buffers.

    The captured sequence is the whole per-chunk hot path of a cohort -- decode of the
    packed .bed records, rotation (INT8 tensor cores or FP64), the series sums and the
    per-SNP search with its statistics -- so a replay is one launch from the host instead
    of the eight to ten kernel and library launches of an eager chunk.  Fill ``packed``
    (m, bytes_per_snp) and ``means`` (m,) on the replaying stream (e.g. non-blocking
    copies from pinned host memory), call :meth:`replay`, read ``out``.  Work queued on one
    stream is ordered, so refilling the inputs for the next chunk right after a replay is
    safe; a chunk shorter than ``m`` uses the first rows and ignores the rest.

    Capture runs on a private stream without synchronising the device, with thread-local
    capture rules, so other streams and threads keep working meanwhile.  With
    ``capture=False`` the object keeps the same buffers and interface and replays by
    issuing the launches eagerly.  The graph keeps
    the cohort's workspaces alive; capture after any eager chunk larger than ``m`` so that
    no workspace is reallocated afterwards.  ``prefill(graph)``, if given, fills the input
    buffers (on the capture's private stream) before the eager warm-up run, whose results
    are then a real chunk's, left in ``out`` when the constructor returns.
    """

    def __init__(self, cohort: "DeviceCohort", m: int, n_file: int | None = None,
                 sample_idx: torch.Tensor | None = None, has_missing: bool = True,
                 prefill=None, capture: bool = True):
        n = cohort.n
        n_file = n if n_file is None else n_file
        self.cohort, self.m, self.n_file, self.sample_idx = cohort, m, n_file, sample_idx
        self.has_missing = bool(has_missing)
        self.packed = torch.zeros((m, (n_file + 3) // 4), dtype=torch.uint8, device="cuda")
        self.means = torch.zeros((m,), dtype=torch.float64, device="cuda")
        self.codes = torch.zeros((m, cohort.code_ld), dtype=torch.int8, device="cuda")
        self.counts = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
        self.out = cohort.alloc_out(m)
        self.bufs = {"UtG": empty((m, n))}
        if cohort.precision != "mixed":
            self.bufs["G"] = empty((m, n))
        caller = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        side.wait_stream(caller)
        with torch.cuda.stream(side):
            if prefill is not None:  # the warm-up computes a real first chunk
                prefill(self)
            self._run()  # eager warm-up: workspaces, library handles, kernel attributes
            self._keep = (cohort.ws, cohort._chunk_ws, cohort._rot_ws, cohort.series_ws,
                          cohort.ozaki)
            self.graph = None
            if capture:
                self.graph = torch.cuda.CUDAGraph()
                self.graph.capture_begin(capture_error_mode="thread_local")
                try:
                    self._run()
                finally:
                    self.graph.capture_end()
        caller.wait_stream(side)

    def _run(self) -> None:
        c = self.cohort
        _native.call("jb_decode_bed", ptr(self.packed), self.packed.shape[1], self.m,
                     ptr(self.sample_idx), c.n, ptr(self.codes), c.code_ld, ptr(self.counts),
                     stream_handle())
        c.associate_codes(self.codes, self.means, out=self.out, bufs=self.bufs,
                          has_missing=self.has_missing)

    def replay(self) -> dict:
        """Run the chunk on the current stream: the captured graph, or (``capture=False``)
        the same launches issued eagerly."""
        if self.graph is None:
            self._run()
        else:
            self.graph.replay()
        return self.out


def decode_packed(packed: torch.Tensor, n_file: int, sample_idx: torch.Tensor | None, n: int,
                  ld: int | None = None) -> tuple[torch.Tensor, torch.Tensor]:
    """Device decode of (m, bytes_per_snp) packed records -> codes (m, ld) + counts (m, 4)."""
    m, bps = packed.shape
    ld = n if ld is None else ld
    codes = torch.empty((m, ld), dtype=torch.int8, device="cuda")
    counts = torch.empty((m, 4), dtype=torch.int32, device="cuda")
    if sample_idx is None and n != n_file:
        raise ValueError("sample_idx is required when n differs from the file's sample count")
    _native.call("jb_decode_bed", ptr(packed), bps, m, ptr(sample_idx), n, ptr(codes), ld,
                 ptr(counts), stream_handle())
    return codes, counts


def pass1_counts(bed, sample_idx: torch.Tensor | None, n: int, chunk: int = 16384) -> np.ndarray:
    """Per-SNP counts {n_obs, sum, n_het, n_hom2} of every SNP of a .bed file over the
    analysed samples (jamma's pass-1 statistics loop, src/jamma/lmm/runner_streaming.py:
    224-284), pipelined: while the device decodes chunk k, the host reads chunk k+1 into the
    other pinned buffer; counts return by asynchronous copies collected one chunk behind."""
    p, bps = bed.n_snps, bed.bytes_per_snp
    out = np.empty((p, 4), dtype=np.int32)
    if p == 0:
        return out
    step = min(chunk, p)
    st = torch.cuda.current_stream()
    pin = [torch.empty((step, bps), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    pin_cnt = [torch.empty((step, 4), dtype=torch.int32, pin_memory=True) for _ in range(2)]
    dev = [torch.empty((step, bps), dtype=torch.uint8, device="cuda") for _ in range(2)]
    codes = torch.empty((step, n), dtype=torch.int8, device="cuda")
    cnt = torch.empty((step, 4), dtype=torch.int32, device="cuda")
    done = [None, None]   # counts of the chunk in buffer b are in pin_cnt[b]
    rng = [None, None]    # SNP range of the chunk in buffer b, not yet collected

    def collect(b: int) -> None:
        done[b].synchronize()
        s0, e0 = rng[b]
        out[s0:e0] = pin_cnt[b][: e0 - s0].numpy()
        rng[b] = None

    for ci, s in enumerate(range(0, p, step)):
        e = min(s + step, p)
        b = ci % 2
        if rng[b] is not None:
            collect(b)  # chunk ci-2: its upload has read pin[b], its counts are back
        bed.read_into(s, e, pin[b].numpy())
        dev[b][: e - s].copy_(pin[b][: e - s], non_blocking=True)
        _native.call("jb_decode_bed", ptr(dev[b]), bps, e - s, ptr(sample_idx), n, ptr(codes), n,
                     ptr(cnt), stream_handle())
        pin_cnt[b][: e - s].copy_(cnt[: e - s], non_blocking=True)
        done[b] = torch.cuda.Event()
        done[b].record(st)
        rng[b] = (s, e)
    for b in (0, 1):
        if rng[b] is not None:
            collect(b)
    return out
