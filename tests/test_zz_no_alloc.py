"""The allocation-free INT8 Gram entry point agrees with the workspace entry point.

``jb_gram_i8_noalloc`` serves callers that cannot allocate device memory (their memory
pool already owns the GPU's free HBM, or they must avoid cudaMalloc's implicit device
synchronisation): it keeps its scratch in a static device array inside the library.
Both entry points compute an exact int32 Gram, so their outputs must be identical; the
check runs on two calls in a row with different inputs, because the shared static
scratch carries the previous call's contents into the next one.

This file is collected last so that a failure here cannot hide any other test result.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build, _native

    _build.build()
    return _native


def _operand(n, p, seed):
    rng = np.random.default_rng(seed)
    Z = rng.integers(0, 3, size=(n, p), dtype=np.int8)
    ldz = (p + 127) // 128 * 128
    Zd = torch.zeros((n, ldz), dtype=torch.int8, device="cuda")
    Zd[:, :p] = torch.from_numpy(Z).cuda()
    return Z, Zd, ldz


def test_noalloc_gram_matches_workspace_gram_on_consecutive_calls(lib):
    from jamma_b200.device import ptr, stream_handle, workspace

    st = stream_handle()
    for n, p, seed in ((300, 1000, 1), (515, 2200, 2)):
        Z, Zd, ldz = _operand(n, p, seed)
        ref = torch.zeros((n, n), dtype=torch.int32, device="cuda")
        ws = workspace(lib.load().jb_gram_i8_workspace_size(n))
        lib.call("jb_gram_i8", ptr(Zd), n, p, ldz, ptr(ref), n, ptr(ws), ws.numel(), st)
        got = torch.full((n, n), -1, dtype=torch.int32, device="cuda")
        lib.call("jb_gram_i8_noalloc", ptr(Zd), n, p, ldz, ptr(got), n, st)
        status = np.full(1, -1, dtype=np.int32)  # the pipeline status word in the static scratch
        lib.call("jb_gram_i8_noalloc_status", status.ctypes.data, st)
        assert status[0] == 0, f"no-alloc Gram pipeline status {status[0]}"
        torch.cuda.synchronize()
        iu = np.triu_indices(n)
        g = got.cpu().numpy().T  # column-major: (i, j), i <= j, at [j*n + i]
        r = ref.cpu().numpy().T
        np.testing.assert_array_equal(g[iu], r[iu])
        exact = Z.astype(np.int64) @ Z.T.astype(np.int64)
        np.testing.assert_array_equal(g[iu], exact[iu])


def test_noalloc_gram_rejects_sizes_beyond_its_scratch(lib):
    st = lib.load().jb_gram_i8_noalloc(None, 65409, 128, 128, None, 65409, 0)
    assert st == -1
    assert "scratch" in lib.last_error()
