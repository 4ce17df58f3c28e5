"""The tensor-core pipelines' bounded waits end with an error status, not a hang.

Every mbarrier wait of the INT8 GEMM kernels has a deadline; when it passes, the kernel
records 100 + (the waiting role) in its status word, stops every role of the CTA and
frees its tensor memory.  The test shortens the deadline to 10 ms and turns off the
producer's tile loads through the library's test hook, so the first MMA wait runs out
with no copy and no MMA ever in flight -- no fault, no trap, no endless loop.  It checks
the status word of the Gram (workspace and allocation-free entry points) and of the
rotation, then restores the defaults and checks that the next launches on the same
context run normally and give exact results.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build, _native

    _build.build()
    return _native


def _gram(lib, Zd, n, p, ldz, noalloc=False):
    from jamma_b200.device import ptr, stream_handle, workspace

    st = stream_handle()
    C = torch.full((n, n), -1, dtype=torch.int32, device="cuda")
    status = np.full(1, -1, dtype=np.int32)
    if noalloc:
        lib.call("jb_gram_i8_noalloc", ptr(Zd), n, p, ldz, ptr(C), n, st)
        lib.call("jb_gram_i8_noalloc_status", status.ctypes.data, st)
    else:
        ws = workspace(lib.load().jb_gram_i8_workspace_size(n))
        lib.call("jb_gram_i8", ptr(Zd), n, p, ldz, ptr(C), n, ptr(ws), ws.numel(), st)
        lib.call("jb_gram_status", ptr(ws), status.ctypes.data, st)
    return int(status[0]), C


def test_pipeline_wait_deadline_reports_status_and_context_recovers(lib):
    from jamma_b200 import engine as eng

    n, p = 300, 1000
    rng = np.random.default_rng(1)
    Z = rng.integers(0, 3, size=(n, p), dtype=np.int8)
    ldz = (p + 127) // 128 * 128
    Zd = torch.zeros((n, ldz), dtype=torch.int8, device="cuda")
    Zd[:, :p] = torch.from_numpy(Z).cuda()
    exact = Z.astype(np.int64) @ Z.T.astype(np.int64)
    iu = np.triu_indices(n)

    g = synth.genotypes(n, 256, 0.02, seed=3)
    K = np.corrcoef(np.nan_to_num(g, nan=1.0))
    w, U = np.linalg.eigh(K)
    cohort = eng.DeviceCohort(np.where(np.abs(w) < 1e-10, 0.0, w), U, None, rng.normal(size=n),
                              lmm_mode=1, precision="mixed")
    from oracle import plink as OP

    packed = torch.from_numpy(OP.encode_genotypes(g)).cuda()
    codes, cnt = eng.decode_packed(packed, n, None, n, ld=cohort.code_ld)
    c = cnt.cpu().numpy()
    mu = torch.from_numpy(c[:, 1] / np.maximum(c[:, 0], 1)).cuda()

    prev_kernel = lib.load().jb_rotate_get_kernel()
    lib.call("jb_rotate_set_kernel", 0)  # the one-CTA kernel carries the test hook
    try:
        lib.call("jb_test_pipeline_timeout", 1, 10_000_000)  # no loads, 10 ms deadline
        for noalloc in (False, True):
            st, _ = _gram(lib, Zd, n, p, ldz, noalloc)
            assert 100 < st < 200, f"Gram (noalloc={noalloc}) status {st} after a timed-out wait"
        cohort.rotate_codes_i8(codes, mu, True)
        st = cohort.rotate_status()
        assert 100 < st < 200, f"rotation status {st} after a timed-out wait"
    finally:
        lib.call("jb_test_pipeline_timeout", 0, 2_000_000_000)
        lib.call("jb_rotate_set_kernel", prev_kernel)
    torch.cuda.synchronize()
    # the same context runs the next launches normally (tensor memory was released)
    for noalloc in (False, True):
        st, C = _gram(lib, Zd, n, p, ldz, noalloc)
        assert st == 0
        np.testing.assert_array_equal(C.cpu().numpy().T[iu], exact[iu])
    X = cohort.rotate_codes_i8(codes, mu, True)
    assert cohort.rotate_status() == 0
    gi = np.where(np.isnan(g), c[:, 1] / np.maximum(c[:, 0], 1), g)
    ref = U.T @ gi
    got = X.cpu().numpy().T
    assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()
