"""Host-side pieces of the association runners and the server that need no GPU: the
column-wise AssocResult builder per test mode, and the server's out-of-memory retry and
cached-memory release rule."""

from __future__ import annotations

import threading

import numpy as np
import pytest
import torch

from jamma_b200 import engine as eng
from jamma_b200 import serve
from jamma_b200.io import AssocResult
from jamma_b200.lmm import _build_results


def _info(m):
    return [{"chr": "2", "rs": f"rs{j}", "pos": 100 + j, "a1": "A", "a0": "C"} for j in range(m)]


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_build_results_per_mode(mode):
    m = 6
    rng = np.random.default_rng(mode)
    arrays = {k: rng.random((2, m)) for k in eng.MODE_KEYS[mode]}
    idx = np.array([0, 2, 5])
    af, miss = rng.random(3), np.array([0, 3, 1])
    for f in (0, 1):
        res = _build_results(mode, idx, af, miss, _info(m), arrays, f=f)
        assert [r.rs for r in res] == ["rs0", "rs2", "rs5"]
        assert [r.ps for r in res] == [100, 102, 105]
        assert all(isinstance(r, AssocResult) for r in res)
        np.testing.assert_array_equal([r.n_miss for r in res], miss)
        np.testing.assert_array_equal([r.af for r in res], af)
        field = {"lambda_remle": "l_remle", "logl_h1": "logl_H1", "lambda_mle": "l_mle"}
        for key in eng.MODE_KEYS[mode]:
            name = field.get(key, key)
            if key == "logl_mle" or (mode == 2 and key in ("beta", "se")):
                continue
            # the builder takes one value per tested SNP in order (arrays are per kept SNP)
            np.testing.assert_array_equal([getattr(r, name) for r in res], arrays[key][f][:3])
        if mode == 2:  # no beta/se in the LRT-only row
            assert all(np.isnan(r.beta) and np.isnan(r.se) for r in res)
        if mode == 1:
            assert all(r.p_score is None and r.p_lrt is None and r.l_mle is None for r in res)
        if mode == 3:
            assert all(r.p_wald is None and r.l_remle is None for r in res)


def test_retry_out_of_memory_releases_and_retries(monkeypatch):
    released = []
    monkeypatch.setattr(torch.cuda, "empty_cache", lambda: released.append(1))
    calls = {"n": 0}

    def flaky():
        calls["n"] += 1
        if calls["n"] < 3:
            raise torch.OutOfMemoryError("no room")
        return "built"

    lock = threading.Lock()
    assert serve._retry_out_of_memory(flaky, lock, attempts=3, pause_s=0.0) == "built"
    assert calls["n"] == 3 and len(released) == 2

    def always():
        raise torch.OutOfMemoryError("no room")

    with pytest.raises(torch.OutOfMemoryError):
        serve._retry_out_of_memory(always, lock, attempts=2, pause_s=0.0)


def test_cached_memory_is_not_released_during_a_capture_or_solve(monkeypatch):
    released = []
    monkeypatch.setattr(torch.cuda, "empty_cache", lambda: released.append(1))
    lock = threading.Lock()
    with lock:  # a graph capture or an eigendecomposition in progress
        assert serve._release_cached(lock) is False
    assert released == []
    assert serve._release_cached(lock) is True and released == [1]
    assert not lock.locked()
