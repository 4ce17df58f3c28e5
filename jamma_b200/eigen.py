"""FP64 eigendecomposition of the kinship matrix on the GPU.

``eigendecompose_kinship`` keeps jamma's contract (src/jamma/lmm/eigen.py:28-128):
ascending eigenvalues, eigenvectors as columns, |lambda| < threshold set to 0 (never
clamped), warnings for negative and repeated-zero eigenvalues.
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from jamma_b200.device import require_cuda
from jamma_b200.engine import eigh_device


def _warn(evals: np.ndarray, threshold: float) -> None:
    n_neg = int(np.sum(evals < -threshold))
    if n_neg > 0:
        warnings.warn(
            f"Kinship matrix has {n_neg} negative eigenvalue(s). "
            "Matrix may not be positive semi-definite.",
            stacklevel=3,
        )
    n_zero = int(np.sum(evals == 0.0))
    if n_zero > 1:
        warnings.warn(
            f"Kinship matrix has {n_zero} eigenvalues close to zero. "
            "Matrix may be rank-deficient.",
            stacklevel=3,
        )


def eigendecompose_kinship(K: np.ndarray, threshold: float = 1e-10, *,
                           check_memory: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """(eigenvalues ascending (n,), eigenvectors (n, n) as columns), FP64 on device."""
    K = np.asarray(K, dtype=np.float64)
    if K.ndim != 2 or K.shape[0] != K.shape[1]:
        raise ValueError(f"Kinship matrix must be square, got shape {K.shape}")
    require_cuda()
    # K is symmetric, so its row-major bytes are already the column-major layout.
    dk = torch.from_numpy(np.ascontiguousarray(K)).to("cuda")
    w, U = eigh_device(dk, threshold)
    evals = w.cpu().numpy()
    evecs = U.cpu().numpy().T
    _warn(evals, threshold)
    return evals, np.ascontiguousarray(evecs)


def eigendecompose_kinship_device(K: torch.Tensor, threshold: float = 1e-10):
    """Device-resident variant: returns (eigenvalues, column-major eigenvectors) tensors."""
    require_cuda()
    w, U = eigh_device(K, threshold)
    _warn(w.cpu().numpy(), threshold)
    return w, U
