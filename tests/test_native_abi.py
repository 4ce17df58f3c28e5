"""The C-ABI library loads and exports every symbol include/jamma_b200.h declares (no GPU)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "jamma_b200.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from jamma_b200 import _build, _native

    _build.build()
    return _native.load()


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "jb_lmm_chunk" in names and "jb_decode_bed" in names and len(names) >= 14


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_bindings_cover_header():
    from jamma_b200 import _native

    assert set(declared_symbols()) <= set(_native.exported_symbols())


def test_version_and_error_text(lib):
    from jamma_b200 import _native

    assert lib.jb_version() >= 100
    buf = ctypes.create_string_buffer(8)
    assert lib.jb_last_error(buf, 8) == 0
    # shape validation fails before touching the device
    st = lib.jb_impute_f64(None, 1, 5, 1, None, None, 2, 0)  # ldg < n
    assert st == -1
    assert "bad shape" in _native.last_error()


def test_workspace_queries(lib):
    assert lib.jb_lmm_workspace_size(1000, 1, 1, 50) > 50 * 1000 * 8
    assert lib.jb_lmm_workspace_size(1000, 0, 1, 50) == -1
    assert lib.jb_kinship_f64_workspace_size(100, 10) == 8000
