"""Eigendecomposition above the single-GPU divide-and-conquer solver's size limit.

cuSOLVER's cusolverDnXsyevd rejects n above about 23 000 (its workspace, ~4 n^2 doubles,
passes 2^31 elements); jb_eigh_f64 then runs cusolverMgSyevd on a one-device grid.  jamma's
eigendecompose_kinship (src/jamma/lmm/eigen.py:28-128) returns ascending eigenvalues with
|lambda| < 1e-10 set to 0 and orthonormal eigenvectors; both are checked here on a
kinship-like matrix at n = 23 500 through the residual ||K U - U diag(w)|| and U^T U = I.
"""

from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


def test_large_n_eigendecomposition_takes_the_multi_device_solver_path():
    from jamma_b200 import _native
    from jamma_b200 import engine as eng

    n, p = 23500, 3000
    lib = _native.load()
    assert lib.jb_eigh_workspace_size(20000) > 0
    g = torch.Generator(device="cuda").manual_seed(3)
    G = torch.randn((n, p), dtype=torch.float64, device="cuda", generator=g)
    K = (G @ G.T) / p
    del G
    K0 = K.clone()
    w, U = eng.eigh_device(K)  # U: column-major (n, n), i.e. U.T holds the eigenvectors as rows
    V = U.T  # V[:, i] = i-th eigenvector
    assert bool(torch.all(w[1:] >= w[:-1]))
    assert bool(torch.all((w == 0) | (w.abs() >= 1e-10)))
    scale = K0.abs().max()
    R = K0 @ V - V * w
    assert float(R.abs().max() / scale) < 1e-10
    del R
    E = V.T @ V
    E.diagonal().sub_(1.0)
    assert float(E.abs().max()) < 1e-10
