"""Autotuner: picks a chunk width and rotation schedule among the candidates, applies the
schedule, caches the result per GPU and shape, and the tuned schedule gives the same
statistics as the default one (the schedule only reorders whole output tiles)."""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from jamma_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


def test_tune_caches_and_schedule_keeps_results(tmp_path, monkeypatch):
    from jamma_b200 import autotune
    from jamma_b200 import engine as eng

    monkeypatch.setenv("JAMMA_B200_CACHE", str(tmp_path / "tune.json"))
    n = 700
    g = synth.genotypes(n, 400, 0.0, seed=3)
    w, U = np.linalg.eigh(np.corrcoef(g))
    y = synth.phenotypes(g, n_causal=5, h2=0.5, seed=4)
    cohort = eng.DeviceCohort(np.where(np.abs(w) < 1e-10, 0.0, w), U, None, y, lmm_mode=4,
                              precision="mixed")
    default, default_kernel = autotune.get_schedule(), autotune.get_kernel()
    codes, means = autotune._synthetic_chunk(n, 512, cohort.code_ld, seed=9)
    base = {k: v.cpu().numpy() for k, v in cohort.associate_codes(codes, means).items()}
    try:
        res = autotune.tune(cohort, chunks=(256, 512), reps=1)
        assert res["chunk"] in (256, 512) and res["kernel"] in autotune.KERNELS
        assert autotune.get_kernel() == res["kernel"]
        assert tuple(res["schedule"]) in autotune.SCHEDULES
        assert autotune.get_schedule() == tuple(res["schedule"])
        cached = json.loads((tmp_path / "tune.json").read_text())
        assert len(cached) == 1 and next(iter(cached.values()))["chunk"] == res["chunk"]
        autotune.set_schedule(*default)
        again = autotune.tune(cohort, chunks=(256, 512), reps=1)  # served from the cache
        assert again["trials"] == res["trials"]
        assert autotune.get_schedule() == tuple(res["schedule"])
        for kern, sched in ((0, (3, 64)), (0, (36, 4)), (1, (9, 16)), (1, (5, 32))):
            autotune.set_kernel(kern)
            autotune.set_schedule(*sched)
            got = {k: v.cpu().numpy() for k, v in cohort.associate_codes(codes, means).items()}
            for k in base:
                np.testing.assert_array_equal(got[k], base[k], err_msg=f"{kern} {sched} {k}")
        assert cohort.rotate_status() == 0
    finally:
        autotune.set_schedule(*default)
        autotune.set_kernel(default_kernel)


def test_schedule_rejects_bad_groups():
    from jamma_b200 import _native, autotune

    with pytest.raises(_native.NativeError, match="group sizes"):
        autotune.set_schedule(0, 16)
