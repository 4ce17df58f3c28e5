"""The INT8 kinship's missing-call correction at shapes that reach its edge paths.

The correction walks each sample's missing SNPs for blocks of 4 096 samples, reads calls
as 16-sample words, and keeps per-SNP lists of missing samples per block.  These cases put
n across the 4 096-sample block boundary, make the last 16-sample word partial, take rows
that are and are not 16-byte aligned (vector and scalar loads), give one sample 60 % of its
calls missing (a long list) and one sample a single missing call, and compare with the
NumPy restatement of jamma's impute_and_center kinship (src/jamma/kinship/missing.py:22-61,
src/jamma/kinship/compute.py:93-226) within 1e-10 of the kinship's scale.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import kinship as OK

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


def _genotypes(n: int, p: int, seed: int) -> np.ndarray:
    g = synth.genotypes(n, p, 0.02, seed=seed)
    rng = np.random.default_rng(seed + 1)
    heavy = rng.choice(p, size=int(0.6 * p), replace=False)
    g[5, heavy] = np.nan  # one sample with 60 % of its calls missing
    g[n - 1, :] = np.nan_to_num(g[n - 1, :], nan=1.0)
    g[n - 1, 7] = np.nan  # the last sample (in the last partial word): one missing call
    return g


# 4 100: two blocks, a partial last word, rows not 16-byte aligned (scalar loads);
# 4 112: two blocks, 16-byte aligned rows (vector loads); SNP counts not multiples of 32
@pytest.mark.parametrize("n,p", [(4100, 1100), (4112, 1057)])
def test_sparse_correction_across_sample_blocks(n, p, monkeypatch):
    from jamma_b200 import kinship as KM

    g = _genotypes(n, p, seed=n + p)
    ref = OK.centered_kinship(g)
    scale = np.abs(ref).max()
    monkeypatch.setattr(KM, "TC_MISSING_DENSITY", 2.0)  # always the FP64 walk
    a = KM.compute_centered_kinship(g, batch_size=512, precision="int8")
    assert np.abs(a - ref).max() <= 1e-10 * scale
    np.testing.assert_array_equal(a, a.T)
    b = KM.compute_centered_kinship(g, batch_size=512, precision="int8")
    np.testing.assert_array_equal(a, b)  # bit-reproducible run to run
    monkeypatch.setattr(KM, "TC_MISSING_DENSITY", 0.0)  # the tensor-core form
    c = KM.compute_centered_kinship(g, batch_size=512, precision="int8")
    assert np.abs(c - ref).max() <= 1e-10 * scale
    assert np.abs(c - a).max() <= 5e-11 * scale
