"""Continuous-batching GWAS job server on one GPU.

Jobs of different sample and SNP counts arrive over time.  A job is admitted when its
device memory fits the HBM budget beside what is already resident; admitted jobs run
concurrently, each on its own CUDA stream, advancing one SNP chunk at a time, so their
kernels overlap on the device and a job that arrives while others run starts as soon as
memory frees up.  Cohorts (eigenvalues, eigenvectors and their INT8 digit planes) stay
resident and are shared: a job on a known cohort skips kinship and eigendecomposition.
A job's set-up (pass-1 counts, and for a new cohort the INT8 kinship and the
eigendecomposition, whose solver synchronises its stream) runs on a worker thread, so
the loop keeps feeding the other jobs' chunks meanwhile; jobs that need a cohort being
built wait for that one build.  Packed genotype records stream from pinned host memory
with asynchronous copies on the job's stream.  Every job's arithmetic is the library's ordinary association path with
per-job buffers and a fixed chunk width, so its results do not depend on what else runs.
"""

from __future__ import annotations

import functools
import threading
import time
from collections import OrderedDict, deque
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from jamma_b200 import _native
from jamma_b200 import engine as eng
from jamma_b200.device import empty, ptr, require_cuda, stream_handle
from jamma_b200.kinship import _KinshipI8, filter_mask, snp_stats_from_counts


@dataclass
class GwasJob:
    """One association request.

    ``packed``: (p, ceil(n/4)) count-A1 .bed records of the cohort's SNPs (host);
    ``phenotypes``: (n,) or (n, phi), no missing values (the serving path expects
    pre-filtered samples); ``cohort_id``: jobs naming a resident cohort reuse its
    eigendecomposition, otherwise the kinship is built from ``packed`` on the device.
    """

    job_id: str
    cohort_id: str
    packed: np.ndarray
    n_samples: int
    phenotypes: np.ndarray
    covariates: np.ndarray | None = None
    lmm_mode: int = 1
    maf_threshold: float = 0.01
    miss_threshold: float = 0.05
    arrival: float = 0.0
    admitted: float = 0.0  # left the queue (HBM budget and a slot free)
    ready: float = 0.0  # set-up done (statistics, cohort, chunk graph)
    new_cohort: bool = False  # this job built its cohort's kinship + eigendecomposition
    done: float = 0.0
    results: dict = field(default_factory=dict)
    snp_indices: np.ndarray | None = None


class _Resident:
    def __init__(self, evals: torch.Tensor, U: torch.Tensor, ozaki: torch.Tensor | None):
        self.evals, self.U, self.ozaki = evals, U, ozaki
        n = U.shape[0]
        self.bytes = 8 * n * n + 8 * n + (ozaki.numel() if ozaki is not None else 0)
        self.refs = 0


class _Building:
    """A cohort whose kinship + eigendecomposition one worker is computing; ``waiters``
    jobs (the builder included) will hold a reference to it."""

    def __init__(self):
        self.done = threading.Event()
        self.waiters = 1
        self.error: BaseException | None = None


class _Active:
    def __init__(self, job: GwasJob, stream: torch.cuda.Stream):
        self.job, self.stream = job, stream
        self.chunk_starts: list[int] = []
        self.next = 0
        self.inflight: list = []  # (event, host buffers, start, end)
        self.bytes = 0


@functools.lru_cache(maxsize=256)
def _eigh_workspace_bytes(n: int) -> int:
    return int(_native.load().jb_eigh_workspace_size(n))


def job_device_bytes(n: int, phi: int, n_cvt: int, chunk: int, resident: bool,
                     n_snps: int = 0) -> int:
    """Device bytes a job holds while it runs (cohort state counted when not resident).

    A job that builds its cohort also needs, at the peak of its set-up, the largest of the
    INT8 kinship's operands (n x p int8 calls + FP64 correction matrix + int32 Gram), the
    finalisation (correction + Gram + kinship) and the eigendecomposition (matrix +
    solver workspace), on top of the digit planes it keeps."""
    lib = _native.load()
    b = lib.jb_lmm_workspace_size(n, n_cvt, phi, 50) + lib.jb_lmm_chunk_workspace_size(
        n, n_cvt, phi, 50, chunk)
    b += lib.jb_rotate_i8_workspace_size(n, chunk) + chunk * n * 8 + chunk * ((n + 127) // 128 * 128)
    b += 9 * phi * chunk * 8 + 2 * n * (n_cvt + phi) * 8
    b += lib.jb_lmm_series_workspace_size(n, n_cvt, phi)
    if not resident:
        nn = n * n
        build = max(n * ((n_snps + 127) // 128 * 128) + 12 * nn, 20 * nn,
                    8 * nn + _eigh_workspace_bytes(n))
        b += build + lib.jb_ozaki_workspace_size(n) + n * 8
    return int(b)


def _release_cached(sync_lock: threading.Lock) -> bool:
    """Return the caching allocator's unused blocks to the device, unless a graph capture
    or an eigendecomposition holds ``sync_lock`` (freeing device memory synchronises the
    device, which neither may see, and would stall the caller behind a long solve).
    Returns whether it released."""
    if not sync_lock.acquire(blocking=False):
        return False
    try:
        torch.cuda.empty_cache()
    finally:
        sync_lock.release()
    return True


def _device_room(need: int, sync_lock: threading.Lock) -> bool:
    """True when the device has ``need`` bytes free, after returning the caching
    allocator's unused blocks if it does not at first (when that is possible now)."""
    if torch.cuda.mem_get_info()[0] >= need:
        return True
    return _release_cached(sync_lock) and torch.cuda.mem_get_info()[0] >= need


def _retry_out_of_memory(fn, sync_lock: threading.Lock, attempts: int = 3, pause_s: float = 0.5):
    """Run ``fn``; when the caching allocator cannot place one of its large transient
    buffers (the kinship operands, the eigensolver workspace), return the allocator's
    unused cached blocks to the device and try again, after a pause in which other jobs'
    chunks finish.  The budget accounting counts bytes in use, not how the allocator's
    cache is cut up, so one large request can fail while the budget still has room."""
    for attempt in range(attempts):
        try:
            return fn()
        except torch.OutOfMemoryError:
            if attempt == attempts - 1:
                raise
            time.sleep(pause_s * (attempt + 1))
            _release_cached(sync_lock)
    raise AssertionError("unreachable")


class GwasServer:
    """Continuous-batching job server (see the module docstring).

    A long-running server whose cohorts differ widely in size should keep PyTorch's caching
    allocator from splitting large blocks (``PYTORCH_CUDA_ALLOC_CONF=max_split_size_mb:256``,
    set before CUDA is first used): the budget counts bytes in use, and with splitting the
    freed multi-GB kinship and eigensolver buffers get cut up by smaller allocations until
    a large request fails while much memory sits cached but unused.  Admission of a job
    that builds a cohort also checks the device's free memory, returning the allocator's
    unused cached blocks first if needed.  ``capture_graphs=False`` issues each chunk's
    launches eagerly instead of replaying a captured graph (no capture under memory
    pressure).
    """

    def __init__(self, hbm_budget_bytes: int, max_active: int = 4, chunk: int = 4096,
                 precision: str = "mixed", setup_workers: int = 2, capture_graphs: bool = True):
        require_cuda()
        self._pool = ThreadPoolExecutor(max_workers=max(1, setup_workers),
                                        thread_name_prefix="jb-setup")
        self._lock = threading.Lock()  # cohorts / _building, shared with the workers
        # Graph captures and eigendecompositions never overlap: above ~23 000 samples the
        # solver synchronises the whole device, which a capture on another thread must not
        # see.
        self._device_sync_lock = threading.Lock()
        self.capture_graphs = capture_graphs
        self._building: dict[str, _Building] = {}
        self.preparing: list[tuple[_Active, Future]] = []
        self.budget = int(hbm_budget_bytes)
        self.max_active = max_active
        self.chunk = chunk
        self.precision = precision
        self.cohorts: OrderedDict[str, _Resident] = OrderedDict()
        self.queue: deque[GwasJob] = deque()
        self.active: list[_Active] = []
        self.finished: list[GwasJob] = []
        self.used = 0
        self.snps_done = 0
        self.t0 = None

    # ------------------------------------------------------------ admission
    def submit(self, job: GwasJob, now: float | None = None) -> None:
        job.arrival = time.perf_counter() if now is None else now
        self.queue.append(job)

    def _resident_bytes(self) -> int:
        return sum(r.bytes for r in self.cohorts.values())

    def _evict_for(self, need: int) -> None:
        for cid in list(self.cohorts):
            if self.used + self._resident_bytes() + need <= self.budget:
                return
            if self.cohorts[cid].refs == 0:
                del self.cohorts[cid]

    def _try_admit(self) -> None:
        while self.queue and len(self.active) + len(self.preparing) < self.max_active:
            job = self.queue[0]
            phi = 1 if np.ndim(job.phenotypes) == 1 else job.phenotypes.shape[1]
            c = 1 if job.covariates is None else job.covariates.shape[1]
            with self._lock:
                known = job.cohort_id in self.cohorts or job.cohort_id in self._building
                need = job_device_bytes(job.n_samples, phi, c, self.chunk, known,
                                        n_snps=int(np.shape(job.packed)[0]))
                self._evict_for(need)
                if self.used + self._resident_bytes() + need > self.budget:
                    if not self.active and not self.preparing:
                        raise MemoryError(f"job {job.job_id} needs {need} bytes, over the HBM budget")
                    return
                # a cohort build also needs the device to have that much free in fact: the
                # caching allocator may hold more than the bytes in use
                if not known and (self.active or self.preparing) and \
                        not _device_room(need, self._device_sync_lock):
                    return
                self.queue.popleft()
                # reserve the cohort now so that eviction cannot take it before set-up
                if job.cohort_id in self.cohorts:
                    self.cohorts[job.cohort_id].refs += 1
                    self.cohorts.move_to_end(job.cohort_id)
                    build = None
                elif job.cohort_id in self._building:
                    self._building[job.cohort_id].waiters += 1
                    build = False
                else:
                    self._building[job.cohort_id] = _Building()
                    build = True
            job.admitted = time.perf_counter()
            job.new_cohort = bool(build)
            act = _Active(job, torch.cuda.Stream())
            act.bytes = need
            self.used += need
            self.preparing.append((act, self._pool.submit(self._prepare, act, build)))

    def _cohort(self, job: GwasJob, build, codes, packed, cnt, poly) -> _Resident:
        """The job's resident cohort: already reserved (build None), built by this worker
        (True) or awaited from the worker building it (False)."""
        if build is None:
            with self._lock:
                return self.cohorts[job.cohort_id]
        if build is False:
            with self._lock:
                b = self._building.get(job.cohort_id)
            if b is not None:
                b.done.wait()
                if b.error is not None:
                    raise RuntimeError(f"cohort {job.cohort_id} set-up failed") from b.error
            with self._lock:
                return self.cohorts[job.cohort_id]
        with self._lock:
            b = self._building[job.cohort_id]
        def build_state():
            n = job.n_samples
            acc = _KinshipI8(n, int(poly.sum()))
            kidx = np.where(poly)[0]
            sel = torch.from_numpy(kidx).cuda()
            cc = cnt[kidx]
            acc.add(codes.index_select(0, sel), torch.from_numpy(cc[:, 1] / np.maximum(cc[:, 0], 1)).cuda(),
                    bool(np.any(cc[:, 0] < n)), n_missing=int((n - cc[:, 0]).sum()))
            acc.add_sum_mu2(cc[:, 1] / np.maximum(cc[:, 0], 1))
            K = acc.finish()
            del acc
            with self._device_sync_lock:  # the large-n solver synchronises the device
                evals, U = eng.eigh_device(K)
            oz = eng.ozaki_split(U) if self.precision == "mixed" else None
            torch.cuda.current_stream().synchronize()  # resident state complete for other streams
            return _Resident(evals, U, oz)

        try:  # new cohort: INT8 kinship + FP64 eigendecomposition on the device
            res = _retry_out_of_memory(build_state, self._device_sync_lock)
        except BaseException as e:
            with self._lock:
                b.error = e
                del self._building[job.cohort_id]
            b.done.set()
            raise
        with self._lock:
            res.refs = b.waiters
            self.cohorts[job.cohort_id] = res
            del self._building[job.cohort_id]
        b.done.set()
        return res

    def _prepare(self, act: _Active, build) -> _Active:
        """Worker thread: pass-1 statistics, the cohort, and the job's device state."""
        job = act.job
        n = job.n_samples
        with torch.cuda.stream(act.stream):
            packed = torch.from_numpy(job.packed).pin_memory().to("cuda", non_blocking=True)
            codes, counts = eng.decode_packed(packed, n, None, n)
            cnt = counts.cpu().numpy()  # pass 1: per-SNP statistics
            mean, miss, poly = snp_stats_from_counts(cnt, n, np.float32)
            keep, af = filter_mask(mean, miss, poly, n, job.maf_threshold, job.miss_threshold)
            idx = np.where(keep)[0]
            res = self._cohort(job, build, codes, packed, cnt, poly)
            act.cohort = eng.DeviceCohort(res.evals, res.U, job.covariates, job.phenotypes,
                                          job.lmm_mode, precision=self.precision, ozaki=res.ozaki)
            act.packed_host = torch.from_numpy(np.ascontiguousarray(job.packed[idx])).pin_memory()
            act.means = torch.from_numpy(mean[idx].astype(np.float64)).pin_memory()
            act.n_miss = miss[idx]
            # the job's chunk work as one CUDA graph, replayed for every chunk
            with self._device_sync_lock:  # no device synchronisation during capture
                act.graph = eng.ChunkGraph(act.cohort, min(self.chunk, max(1, idx.size)),
                                           has_missing=True, capture=self.capture_graphs)
        job.snp_indices = idx
        job.results = {k: np.empty((act.cohort.phi, idx.size)) for k in eng.MODE_KEYS[job.lmm_mode]}
        job.af, job.n_miss = af[idx], miss[idx]
        act.chunk_starts = list(range(0, idx.size, self.chunk))
        return act

    # ------------------------------------------------------------ execution
    def _launch_chunk(self, act: _Active) -> None:
        s = act.chunk_starts[act.next]
        e = min(s + self.chunk, act.job.snp_indices.size)
        act.next += 1
        g = act.graph
        with torch.cuda.stream(act.stream):
            # stream order: these copies wait for the previous replay to finish with the
            # static buffers, and the next chunk's copies wait for this replay
            g.packed[: e - s].copy_(act.packed_host[s:e], non_blocking=True)
            g.means[: e - s].copy_(act.means[s:e], non_blocking=True)
            out = g.replay()
            host = {k: torch.empty((v.shape[0], e - s), dtype=torch.float64).pin_memory()
                    for k, v in out.items()}
            for k, v in out.items():
                host[k].copy_(v[:, : e - s], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(act.stream)
        act.inflight.append((ev, host, s, e))

    def _poll(self, act: _Active) -> bool:
        """Collect finished chunks; returns True when the job is complete."""
        keep = []
        for item in act.inflight:
            ev, host, s, e = item[:4]
            if ev.query():
                for k, v in host.items():
                    act.job.results[k][:, s:e] = v.numpy()
                self.snps_done += (e - s) * act.cohort.phi
            else:
                keep.append(item)
        act.inflight = keep
        return act.next >= len(act.chunk_starts) and not act.inflight

    def step(self) -> bool:
        """One pass of the loop; returns False when it found nothing to do."""
        self._try_admit()
        busy = False
        for item in list(self.preparing):
            act, fut = item
            if fut.done():
                self.preparing.remove(item)
                try:
                    fut.result()  # re-raises a set-up failure here
                except BaseException:
                    # give back the job's reservation so that a server which catches the
                    # error and keeps running admits and evicts as before
                    self.used -= act.bytes
                    with self._lock:
                        res = self.cohorts.get(act.job.cohort_id)
                        if res is not None:
                            res.refs -= 1
                    raise
                act.job.ready = time.perf_counter()
                self.active.append(act)
                busy = True
        for act in list(self.active):
            if act.next < len(act.chunk_starts) and len(act.inflight) < 2:
                self._launch_chunk(act)
                busy = True
            if self._poll(act):
                act.job.done = time.perf_counter()
                self.finished.append(act.job)
                with self._lock:
                    self.cohorts[act.job.cohort_id].refs -= 1
                self.used -= act.bytes
                self.active.remove(act)
                busy = True
        return busy

    def run(self, arrivals: list[tuple[float, GwasJob]] | None = None) -> list[GwasJob]:
        """Drive the loop until every submitted (and, if given, scheduled) job is done.

        ``arrivals``: (offset seconds, job) pairs submitted when the wall clock reaches
        start + offset -- a job stream arriving while others run.
        """
        pending = deque(sorted(arrivals or [], key=lambda a: a[0]))
        self.t0 = time.perf_counter()
        while pending or self.queue or self.active or self.preparing:
            now = time.perf_counter()
            while pending and now - self.t0 >= pending[0][0]:
                self.submit(pending.popleft()[1], now)
            if not self.active and not self.queue and not self.preparing and pending:
                time.sleep(min(0.001, max(0.0, pending[0][0] - (now - self.t0))))
                continue
            if not self.step():
                time.sleep(0.0002)  # let the set-up workers run (they need the GIL between calls)
        torch.cuda.synchronize()
        return self.finished

    def latency_summary(self) -> dict:
        jobs = self.finished
        lat = np.array([j.done - j.arrival for j in jobs])
        span = max(j.done for j in jobs) - min(j.arrival for j in jobs)

        def pct(v):
            v = np.asarray(v, dtype=np.float64)
            return {"p50_s": float(np.percentile(v, 50)), "p99_s": float(np.percentile(v, 99))} \
                if v.size else None

        # where latency goes: queue wait, set-up (split by whether the job built its
        # cohort), and chunk execution after set-up
        phases = {
            "queue": pct([j.admitted - j.arrival for j in jobs]),
            "setup_new_cohort": pct([j.ready - j.admitted for j in jobs if j.new_cohort]),
            "setup_resident_cohort": pct([j.ready - j.admitted for j in jobs if not j.new_cohort]),
            "run": pct([j.done - j.ready for j in jobs]),
        }
        return {"jobs": len(jobs), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "snps_per_s": self.snps_done / span if span > 0 else None, "phases": phases}
