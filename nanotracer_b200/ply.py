"""PLY in/out through the library's C++ reader/writer — the mirror of nano-splat's
read_ply / write_ply (crates/nano-splat/src/ply.rs:17-256) composed with
SplatBuffer::{from,to}_gaussians (splat_store.rs:60-94)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from ._lib import check, lib
from .splat_store import SplatBuffer


def write_ply(path: str | Path, splats: SplatBuffer) -> None:
    hs = splats.host_struct()
    check(lib().sc_write_ply(str(path).encode(), C.byref(hs)))


def read_ply(path: str | Path) -> SplatBuffer:
    n = C.c_uint32()
    check(lib().sc_read_ply(str(path).encode(), None, C.byref(n)))
    out = SplatBuffer.zeros(n.value)
    hs = out.host_struct()
    check(lib().sc_read_ply(str(path).encode(), C.byref(hs), C.byref(n)))
    return out
