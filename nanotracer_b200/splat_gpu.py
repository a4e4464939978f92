"""Device parameter stores — the mirror of GpuSplatBuffer, GradSplatBuffers and
AdamMomentBuffers (crates/nano-optimize/src/splat_gpu.rs:29-423).

On the device each store is a coefficient-major slab (59 rows x capacity);
upload / readback convert from and to the SplatBuffer layout, so a round trip
is bit-exact (splat_gpu.rs:451-473).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import SC_MOMENTS_BF16, SC_SPLATS_BF16_REST, check, lib
from .gpu import CudaCtx
from .splat_store import SplatBuffer


class GpuSplatBuffer:
    def __init__(self, ctx: CudaCtx, handle: C.c_void_p):
        self.ctx = ctx
        self.handle = handle

    @classmethod
    def upload(cls, ctx: CudaCtx, src: SplatBuffer, capacity: int = 0, bf16_rest: bool = False) -> "GpuSplatBuffer":
        h = C.c_void_p()
        hs = src.host_struct()
        flags = SC_SPLATS_BF16_REST if bf16_rest else 0
        check(lib().sc_splats_upload(ctx.handle, C.byref(hs), int(capacity), flags, C.byref(h)), ctx.handle)
        return cls(ctx, h)

    @property
    def n(self) -> int:
        return int(lib().sc_splats_count(self.handle))

    @property
    def capacity(self) -> int:
        return int(lib().sc_splats_capacity(self.handle))

    def sync_from(self, src: SplatBuffer) -> None:
        hs = src.host_struct()
        check(lib().sc_splats_sync_from(self.ctx.handle, self.handle, C.byref(hs)), self.ctx.handle)

    def readback(self) -> SplatBuffer:
        out = SplatBuffer.zeros(self.n)
        hs = out.host_struct()
        check(lib().sc_splats_readback(self.ctx.handle, self.handle, C.byref(hs)), self.ctx.handle)
        return out

    def free(self) -> None:
        if self.handle:
            lib().sc_splats_free(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.free()
        except Exception:
            pass


class GradSplatBuffers:
    def __init__(self, ctx: CudaCtx, n: int):
        self.ctx = ctx
        self.n = int(n)
        h = C.c_void_p()
        check(lib().sc_grads_create(ctx.handle, max(self.n, 1), C.byref(h)), ctx.handle)
        self.handle = h

    def zero(self) -> None:
        check(lib().sc_grads_zero(self.ctx.handle, self.handle, self.n), self.ctx.handle)

    def upload(self, src: SplatBuffer) -> None:
        hs = src.host_struct()
        check(lib().sc_grads_upload(self.ctx.handle, self.handle, C.byref(hs)), self.ctx.handle)

    def readback(self, n: int | None = None) -> SplatBuffer:
        n = self.n if n is None else n
        out = SplatBuffer.zeros(n)
        hs = out.host_struct()
        check(lib().sc_grads_readback(self.ctx.handle, self.handle, n, C.byref(hs)), self.ctx.handle)
        return out

    def free(self) -> None:
        if self.handle:
            lib().sc_grads_free(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.free()
        except Exception:
            pass


class AdamMomentBuffers:
    def __init__(self, ctx: CudaCtx, n: int, bf16: bool = False):
        self.ctx = ctx
        self.n = int(n)
        h = C.c_void_p()
        check(lib().sc_moments_create(ctx.handle, max(self.n, 1), SC_MOMENTS_BF16 if bf16 else 0, C.byref(h)),
              ctx.handle)
        self.handle = h

    @classmethod
    def upload_from_cpu(cls, ctx: CudaCtx, m: SplatBuffer, v: SplatBuffer, capacity: int = 0,
                        bf16: bool = False) -> "AdamMomentBuffers":
        me = cls(ctx, max(len(m), capacity), bf16)
        hm, hv = m.host_struct(), v.host_struct()
        check(lib().sc_moments_upload(ctx.handle, me.handle, C.byref(hm), C.byref(hv)), ctx.handle)
        return me

    def download(self, n: int) -> tuple[SplatBuffer, SplatBuffer]:
        m, v = SplatBuffer.zeros(n), SplatBuffer.zeros(n)
        hm, hv = m.host_struct(), v.host_struct()
        check(lib().sc_moments_readback(self.ctx.handle, self.handle, n, C.byref(hm), C.byref(hv)), self.ctx.handle)
        return m, v

    def free(self) -> None:
        if self.handle:
            lib().sc_moments_free(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.free()
        except Exception:
            pass
