"""ctypes binding of libjamma_b200.so (the C ABI declared in include/jamma_b200.h).

The library is built in-tree by ``python -m jamma_b200._build``.  There is no
fallback: if the shared library is missing, or no CUDA device is visible, the
product path raises instead of computing anything on the CPU.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, Structure, c_char_p, c_double, c_int32, c_int64, c_size_t, c_uint8
from ctypes import c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libjamma_b200.so"

_u = ctypes.c_uint64  # uintptr_t stream
_p = c_void_p
_i64 = c_int64
_i32 = c_int32
_f64 = c_double


class LmmOut(Structure):
    """Mirror of ``jb_lmm_out``: nine phi x m double arrays (device pointers or NULL)."""

    _fields_ = [
        ("lambda_remle", _p),
        ("logl_h1", _p),
        ("beta", _p),
        ("se", _p),
        ("p_wald", _p),
        ("lambda_mle", _p),
        ("logl_mle", _p),
        ("p_lrt", _p),
        ("p_score", _p),
    ]


# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "jb_version": (_i32, []),
    "jb_last_error": (_i32, [c_char_p, c_size_t]),
    "jb_device_arch": (_i32, []),
    "jb_decode_bed": (_i32, [_p, _i64, _i64, _p, _i64, _p, _i64, _p, _u]),
    "jb_impute_f64": (_i32, [_p, _i64, _i64, _i64, _p, _p, _i64, _u]),
    "jb_pack_codes": (_i32, [_p, _i64, _i64, _i64, _p, _i64, _u]),
    "jb_kinship_f64_workspace_size": (_i64, [_i64, _i64]),
    "jb_kinship_accumulate_f64": (_i32, [_p, _i64, _i64, _i64, _p, _p, _i64, _p, _i64, _u]),
    "jb_kinship_accumulate_std_f64": (_i32, [_p, _i64, _i64, _i64, _p, _p, _p, _i64, _p, _i64, _u]),
    "jb_kinship_finalize": (_i32, [_p, _i64, _i64, _f64, _u]),
    "jb_eigh_workspace_size": (_i64, [_i64]),
    "jb_eigh_f64": (_i32, [_p, _i64, _i64, _p, _f64, _p, _i64, _u]),
    "jb_rotate_f64": (_i32, [_p, _i64, _i64, _p, _i64, _i64, _p, _i64, _u]),
    "jb_lmm_workspace_size": (_i64, [_i64, _i32, _i32, _i32]),
    "jb_lmm_prepare": (
        _i32,
        [_i32, _i32, _i64, _i32, _i32, _p, _p, _i64, _p, _i64, _p, _f64, _f64, _i32, _p, _i64, _u],
    ),
    "jb_lmm_chunk_workspace_size": (_i64, [_i64, _i32, _i32, _i32, _i64]),
    "jb_rotate_set_schedule": (_i32, [_i32, _i32]),
    "jb_rotate_get_schedule": (_i32, [_p, _p]),
    "jb_rotate_set_kernel": (_i32, [_i32]),
    "jb_rotate_get_kernel": (_i32, []),
    "jb_lmm_series_workspace_size": (_i64, [_i64, _i32, _i32]),
    "jb_lmm_series_rows": (_i32, []),
    "jb_lmm_series_prepare": (_i32, [_i64, _i32, _i32, _i32, _p, _i64, _p, _i64, _p, _i64, _u]),
    "jb_lmm_chunk_series_i8": (
        _i32, [_i64, _i32, _i32, _i32, _i64, _p, _i64, _p, _i64, _p, _i32, _p, _i64, _p, _i64, _u]),
    "jb_lmm_chunk": (
        _i32,
        [_i32, _i32, _i64, _i32, _i32, _i64, _p, _p, _i64, _p, _i64, _p, _i64, _p, _p, _f64,
         _f64, _i32, _i32, LmmOut, _p, _i64, _p, _i64, _u],
    ),
    "jb_gram_i8_workspace_size": (_i64, [_i64]),
    "jb_gram_i8": (_i32, [_p, _i64, _i64, _i64, _p, _i64, _p, _i64, _u]),
    "jb_gram_status": (_i32, [_p, _p, _u]),
    "jb_gram_i8_noalloc": (_i32, [_p, _i64, _i64, _i64, _p, _i64, _u]),
    "jb_gram_i8_noalloc_status": (_i32, [_p, _u]),
    "jb_test_pipeline_timeout": (_i32, [_i32, _i64]),
    "jb_kinship_i8_finalize_loco": (
        _i32, [_p, _p, _i64, _i64, _p, _p, _p, _p, _f64, _p, _p, _i64, _i64, _p, _i64, _u]),
    "jb_kinship_loco_f64": (_i32, [_p, _p, _i64, _i64, _i64, _p, _i64, _u]),
    "jb_codes_to_sample_major": (_i32, [_p, _i64, _i64, _i64, _p, _i64, _i64, _p, _i64, _u]),
    "jb_kinship_i8_corrections_workspace_size": (_i64, [_i64, _i64]),
    "jb_kinship_i8_tc_workspace_size": (_i64, [_i64, _i64]),
    "jb_kinship_i8_corrections_tc": (
        _i32, [_p, _i64, _p, _i64, _i64, _i64, _i64, _p, _p, _p, _p, _i64, _p, _i64, _u]),
    "jb_kinship_i8_corrections": (
        _i32, [_p, _i64, _i32, _i64, _i64, _p, _p, _p, _p, _i64, _p, _i64, _u]),
    "jb_kinship_i8_finalize": (_i32, [_p, _i64, _i64, _p, _p, _f64, _p, _i64, _i64, _p, _i64, _u]),
    "jb_ozaki_workspace_size": (_i64, [_i64]),
    "jb_ozaki_prepare": (_i32, [_p, _i64, _i64, _p, _i64, _u]),
    "jb_rotate_i8_workspace_size": (_i64, [_i64, _i64]),
    "jb_rotate_i8": (_i32, [_p, _i64, _p, _i64, _i64, _p, _i32, _p, _i64, _p, _i64, _u]),
    "jb_rotate_status": (_i32, [_p, _p, _u]),
    "jb_null_mle": (
        _i32,
        [_i64, _i32, _i32, _p, _p, _i64, _p, _i64, _f64, _f64, _i32, _i32, _p, _p, _u],
    ),
}

_lib = None


class NativeError(RuntimeError):
    """A libjamma_b200 entry point returned a non-zero status."""


def load(path: Path | None = None):
    """Load (once) and return the ctypes handle with all signatures bound."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build the CUDA library with `python -m jamma_b200._build` "
            "(there is no CPU fallback)"
        )
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().jb_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, what: str) -> None:
    if status != 0:
        raise NativeError(f"{what} failed (status {status}): {last_error()}")


def call(name: str, *args) -> int:
    """Call an entry point and raise NativeError on a non-zero status."""
    st = getattr(load(), name)(*args)
    check(st, name)
    return st


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def _ptr(x) -> int | None:
    if x is None:
        return None
    return int(x.data_ptr())


ptr = _ptr
__all__ = ["LmmOut", "NativeError", "call", "check", "load", "ptr", "exported_symbols", "c_uint8",
           "POINTER"]
