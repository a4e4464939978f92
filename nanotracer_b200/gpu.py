"""Device runtime — the mirror of WgpuCtx (crates/nano-optimize/src/gpu.rs:21-153).

CudaCtx owns one CUDA device and stream through the C ABI; DeviceBuffer is a
library-allocated device allocation (storage_buffer / storage_buffer_zeroed),
read back with a blocking copy (WgpuCtx::readback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr


class DeviceBuffer:
    def __init__(self, ctx: "CudaCtx", nbytes: int, label: str = ""):
        self.ctx = ctx
        self.nbytes = int(nbytes)
        self.label = label
        p = C.c_void_p()
        check(lib().sc_buffer_alloc(ctx.handle, max(self.nbytes, 16), C.byref(p)), ctx.handle)
        self.ptr = p.value

    @property
    def cptr(self) -> C.c_void_p:
        return C.c_void_p(self.ptr)

    def upload(self, arr: np.ndarray, offset: int = 0) -> None:
        a = np.ascontiguousarray(arr)
        assert a.nbytes + offset <= self.nbytes, "upload larger than the buffer"
        check(lib().sc_buffer_upload(self.ctx.handle, C.c_void_p(self.ptr + offset), ptr(a), a.nbytes), self.ctx.handle)

    def readback(self, dtype, count: int | None = None, offset: int = 0) -> np.ndarray:
        dt = np.dtype(dtype)
        if count is None:
            count = (self.nbytes - offset) // dt.itemsize
        out = np.empty(count, dt)
        check(lib().sc_buffer_readback(self.ctx.handle, ptr(out), C.c_void_p(self.ptr + offset), out.nbytes),
              self.ctx.handle)
        return out

    def copy_from(self, src: "DeviceBuffer", nbytes: int, dst_offset: int = 0, src_offset: int = 0) -> None:
        """Device-to-device copy on the context's stream (asynchronous)."""
        assert dst_offset + nbytes <= self.nbytes and src_offset + nbytes <= src.nbytes
        check(lib().sc_buffer_copy(self.ctx.handle, C.c_void_p(self.ptr + dst_offset), C.c_void_p(src.ptr + src_offset),
                                   nbytes), self.ctx.handle)

    def zero(self) -> None:
        check(lib().sc_buffer_zero(self.ctx.handle, self.cptr, self.nbytes), self.ctx.handle)

    def free(self) -> None:
        if self.ptr:
            lib().sc_buffer_free(self.ctx.handle, self.cptr)
            self.ptr = 0

    def __del__(self):
        try:
            if self.ptr and self.ctx.handle:
                self.free()
        except Exception:
            pass


class CudaCtx:
    """One device + stream (WgpuCtx::new returns Result; so does this)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().sc_ctx_create(int(device), C.byref(h)))
        self.handle = h
        self.device = device

    @classmethod
    def new(cls, device: int = 0) -> "CudaCtx":
        return cls(device)

    def storage_buffer(self, label: str, data: np.ndarray) -> DeviceBuffer:
        a = np.ascontiguousarray(data)
        b = DeviceBuffer(self, a.nbytes, label)
        if a.nbytes:
            b.upload(a)
        return b

    def storage_buffer_zeroed(self, label: str, nbytes: int) -> DeviceBuffer:
        return DeviceBuffer(self, nbytes, label)

    def readback(self, buf: DeviceBuffer, dtype, count: int | None = None) -> np.ndarray:
        return buf.readback(dtype, count)

    def write_buffer(self, buf: DeviceBuffer, data: np.ndarray, offset: int = 0) -> None:
        buf.upload(data, offset)

    def synchronize(self) -> None:
        check(lib().sc_ctx_synchronize(self.handle), self.handle)

    @property
    def stream(self) -> int:
        return lib().sc_ctx_stream(self.handle) or 0

    @property
    def launch_count(self) -> int:
        return int(lib().sc_ctx_launch_count(self.handle))

    def set_fp64_det(self, enabled: bool) -> None:
        """FP64 determinant and inverse of near-degenerate splats in
        project / project_backward (the reference computes them in f32,
        project_gaussians.wgsl:226-234)."""
        check(lib().sc_ctx_set_fp64_det(self.handle, 1 if enabled else 0), self.handle)

    def device_info(self) -> tuple[int, int, int]:
        sm, free, total = C.c_int(), C.c_size_t(), C.c_size_t()
        check(lib().sc_ctx_device_info(self.handle, C.byref(sm), C.byref(free), C.byref(total)), self.handle)
        return sm.value, free.value, total.value

    def close(self) -> None:
        if self.handle:
            lib().sc_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
