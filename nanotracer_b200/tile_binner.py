"""Tile binning, radix sort and prefix scan — the mirror of TileBinner,
RadixSort and PrefixScan (crates/nano-optimize/src/tile_binner.rs:21-416,
radix_sort.rs:32-303, prefix_scan.rs:18-258).

TileBinner.bin keeps the reference's contract: it reads the pair count back
once (tile_binner.rs:243-245) and returns sorted keys, payloads and per-tile
[begin, end) ranges.  Keys are the reference's 32-bit (tile << 16 | depth16)
layout by default, or 64-bit (tile << 32 | depth bits) for scenes past 65536
tiles.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import SC_KEYS_NATIVE64, SC_KEYS_REF32, check, lib, sc_tiling
from .gpu import CudaCtx, DeviceBuffer


@dataclass
class TilingParams:
    width: int
    height: int
    tile_size: int = 16
    depth_max: float = 100.0
    tile_h_override: int | None = None  # non-square tiles (extension): tile_size is then the width

    @property
    def tile_w(self) -> int:
        return self.tile_size

    @property
    def tile_h(self) -> int:
        return self.tile_h_override or self.tile_size

    def tiles_x(self) -> int:
        return (self.width + self.tile_w - 1) // self.tile_w

    def tiles_y(self) -> int:
        return (self.height + self.tile_h - 1) // self.tile_h

    def num_tiles(self) -> int:
        return self.tiles_x() * self.tiles_y()

    def struct(self) -> sc_tiling:
        return sc_tiling(self.width, self.height, self.tile_w, self.tile_h, float(self.depth_max))


class TileBinningResult:
    """Device arrays owned by the library's bins object (valid until the next bin()).
    Holds its binner so the arrays outlive a temporary TileBinner(ctx).bin(...)."""

    def __init__(self, ctx: CudaCtx, handle, key_mode: int, owner=None):
        self.ctx = ctx
        self.handle = handle
        self.key_mode = key_mode
        self._owner = owner

    def _info(self):
        total, nt = C.c_uint64(), C.c_uint32()
        k, p, r = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().sc_bins_info(self.handle, C.byref(total), C.byref(nt), C.byref(k), C.byref(p), C.byref(r)))
        return total.value, nt.value, k.value, p.value, r.value

    @property
    def total_pairs(self) -> int:
        return self._info()[0]

    @property
    def num_tiles(self) -> int:
        return self._info()[1]

    def _read(self, addr: int, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype)
        if count:
            check(lib().sc_buffer_readback(self.ctx.handle, C.c_void_p(out.ctypes.data), C.c_void_p(addr), out.nbytes),
                  self.ctx.handle)
        return out

    def sorted_keys(self) -> np.ndarray:
        total, _, k, _, _ = self._info()
        return self._read(k, np.uint32 if self.key_mode == SC_KEYS_REF32 else np.uint64, total)

    def sorted_payloads(self) -> np.ndarray:
        total, _, _, p, _ = self._info()
        return self._read(p, np.uint32, total)

    def tile_ranges(self) -> np.ndarray:
        _, nt, _, _, r = self._info()
        return self._read(r, np.uint32, 2 * nt).reshape(nt, 2)


class TileBinner:
    def __init__(self, ctx: CudaCtx):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().sc_bins_create(ctx.handle, C.byref(h)), ctx.handle)
        self.handle = h

    def bin(self, projected: DeviceBuffer, n_splats: int, params: TilingParams, stride: int | None = None,
            n_views: int = 1, key_mode: int = SC_KEYS_REF32) -> TileBinningResult:
        t = params.struct()
        check(lib().sc_bin(self.ctx.handle, projected.cptr, int(n_splats), int(stride if stride is not None else n_splats),
                           int(n_views), C.byref(t), int(key_mode), self.handle), self.ctx.handle)
        return TileBinningResult(self.ctx, self.handle, key_mode, owner=self)

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                lib().sc_bins_free(self.ctx.handle, self.handle)
                self.handle = None
        except Exception:
            pass


class RadixSort:
    """Stable sort of (key, u32 payload) in place; keys u32 or u64."""

    def __init__(self, ctx: CudaCtx):
        self.ctx = ctx

    def sort(self, keys_a: DeviceBuffer, vals_a: DeviceBuffer, keys_b: DeviceBuffer, vals_b: DeviceBuffer, n: int,
             key_bits: int = 32, key_bytes: int = 4) -> None:
        f = lib().sc_radix_sort_u32 if key_bytes == 4 else lib().sc_radix_sort_u64
        check(f(self.ctx.handle, keys_a.cptr, vals_a.cptr, keys_b.cptr, vals_b.cptr, int(n), int(key_bits)),
              self.ctx.handle)


class PrefixScan:
    """Exclusive u32 scan in place (no 2^24 limit)."""

    def __init__(self, ctx: CudaCtx):
        self.ctx = ctx

    def scan(self, buf: DeviceBuffer, n: int, total: DeviceBuffer | None = None) -> None:
        check(lib().sc_exclusive_scan_u32(self.ctx.handle, buf.cptr, int(n), total.cptr if total is not None else None),
              self.ctx.handle)
