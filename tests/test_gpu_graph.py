"""A chunk captured as a CUDA graph gives the same statistics as the eager chunk path.

The graph replays the same kernels and library calls on the same kind of buffers, so the
results are required to be bitwise equal, for two different chunks replayed through the
same graph (static input buffers refilled between replays)."""

from __future__ import annotations

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


@pytest.mark.parametrize("precision,n_cvt", [("mixed", 1), ("mixed", 2), ("fp64", 1)])
def test_graph_replay_equals_eager(precision, n_cvt):
    from jamma_b200 import engine as eng
    from oracle import plink as OP

    n, m = 520, 384
    g = synth.genotypes(n, 2 * m, 0.02, seed=11)
    K = np.corrcoef(np.nan_to_num(g, nan=1.0))
    w, U = np.linalg.eigh(K)
    y = synth.phenotypes(np.nan_to_num(g, nan=1.0), n_causal=6, h2=0.5, seed=12)
    cov = synth.covariates(n, n_cvt, seed=13)
    cohort = eng.DeviceCohort(np.where(np.abs(w) < 1e-10, 0.0, w), U, cov, y, lmm_mode=4,
                              precision=precision)
    packed = torch.from_numpy(OP.encode_genotypes(g)).cuda()
    mu = torch.from_numpy(np.nan_to_num(np.nanmean(g, axis=0)).astype(np.float32)
                          .astype(np.float64)).cuda()
    eager = []
    for s in (0, m):
        codes, _ = eng.decode_packed(packed[s:s + m], n, None, n, ld=cohort.code_ld)
        o = cohort.associate_codes(codes, mu[s:s + m], has_missing=True)
        eager.append({k: v.cpu().numpy() for k, v in o.items()})
    graph = eng.ChunkGraph(cohort, m, has_missing=True)
    for i, s in enumerate((0, m)):
        graph.packed.copy_(packed[s:s + m])
        graph.means.copy_(mu[s:s + m])
        got = {k: v.cpu().numpy() for k, v in graph.replay().items()}
        for k in eager[i]:
            np.testing.assert_array_equal(got[k], eager[i][k], err_msg=f"chunk {i} {k}")
    if precision == "mixed":
        assert cohort.rotate_status() == 0
