"""Integer constants of the C ABI, read from include/grasph_cuda.h so the
header stays the single definition of kinds, field ids and status codes."""
from __future__ import annotations

import re
from pathlib import Path

HEADER = Path(__file__).resolve().parents[2] / "include" / "grasph_cuda.h"


def _parse(text: str) -> dict:
    out = {}
    for m in re.finditer(r"\b(GC_[A-Z0-9_]+)\s*=\s*(-?\d+)", text):
        out[m.group(1)] = int(m.group(2))
    for m in re.finditer(r"#define\s+(GC_[A-Z0-9_]+)\s+(-?\d+)", text):
        out[m.group(1)] = int(m.group(2))
    return out


_VALUES = _parse(HEADER.read_text())
globals().update(_VALUES)

STATUS_NAMES = {v: k for k, v in _VALUES.items() if k.startswith("GC_ERR_") or k == "GC_OK"}
