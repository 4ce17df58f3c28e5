"""Device plumbing: CUDA availability, streams and column-major torch buffers.

PyTorch is used only to own device memory and streams; all arithmetic on the hot
path runs in libjamma_b200.so.  A column-major n x m matrix is stored as a
row-major torch tensor of shape (m, n) (row j = column j), so its device pointer and
leading dimension n can be handed straight to the C ABI.
"""

from __future__ import annotations

import numpy as np
import torch

from jamma_b200 import _native

_checked = False


def require_cuda() -> None:
    """Fail loudly unless a CUDA device and the native library are available."""
    global _checked
    if _checked:
        return
    if not torch.cuda.is_available():
        raise RuntimeError(
            "jamma_b200 runs its hot path on an NVIDIA GPU (built for B200, sm_100a); "
            "no CUDA device is visible and there is no CPU fallback"
        )
    _native.load()
    arch = _native.load().jb_device_arch()
    if arch < 100:
        raise RuntimeError(f"jamma_b200 is built for sm_100a; this device reports sm_{arch}")
    _checked = True


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def colmajor(a: np.ndarray, dtype=torch.float64) -> torch.Tensor:
    """Upload a host (n, m) matrix (or (n,) vector) as a column-major device buffer."""
    a = np.asarray(a)
    if a.ndim == 1:
        return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(device="cuda", dtype=dtype)


def to_host_colmajor(t: torch.Tensor) -> np.ndarray:
    """Inverse of :func:`colmajor` for matrices: (m, n) tensor -> (n, m) host array."""
    return t.detach().cpu().numpy().T


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else int(t.data_ptr())


def empty(shape, dtype=torch.float64) -> torch.Tensor:
    return torch.empty(shape, dtype=dtype, device="cuda")


def workspace(nbytes: int) -> torch.Tensor:
    """Byte buffer for a library workspace (256-byte aligned by the caching allocator)."""
    if nbytes < 0:
        from jamma_b200 import _native

        raise RuntimeError(f"workspace size query failed: {_native.last_error()}")
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")
