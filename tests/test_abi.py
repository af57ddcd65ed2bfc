"""The C-ABI library loads and exports every entry point include/*.h declares
(no device calls, so this runs without a GPU)."""
import ctypes as ct
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(gc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    assert "gc_step" in names and "gc_ctx_create" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib_path = ROOT / "grasph.jl_b200" / "libgrasph_cuda.so"
    if not lib_path.exists():
        pytest.skip("libgrasph_cuda.so not built (run __graft_entry__.build())")
    lib = ct.CDLL(str(lib_path))
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_status_strings_without_device():
    lib_path = ROOT / "grasph.jl_b200" / "libgrasph_cuda.so"
    if not lib_path.exists():
        pytest.skip("libgrasph_cuda.so not built")
    lib = ct.CDLL(str(lib_path))
    lib.gc_status_string.restype = ct.c_char_p
    assert lib.gc_status_string(0) == b"GC_OK"
    assert lib.gc_status_string(4) == b"GC_ERR_NONFINITE"
