"""Rasteriser — the mirror of nano-optimize's Rasterizer and record types
(crates/nano-optimize/src/raster.rs:22-804) over the C ABI.

Calls keep the reference's argument meaning: the caller allocates the
projected / image / projected-grad buffers (alloc_*), composite_backward
accumulates into a projected-grad buffer the caller zeroed first
(raster.rs:647-651), project_backward overwrites the gradient store.  The
extensions are n_views (several cameras per call) and the exact backward mode.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import SC_BWD_EXACT, SC_BWD_REF, check, lib, ptr, sc_camera, sc_tiling
from .gpu import CudaCtx, DeviceBuffer
from .splat_gpu import GpuSplatBuffer, GradSplatBuffers
from .tile_binner import TileBinningResult, TilingParams

# ProjectedSplat (raster.rs:27-37) and ProjectedGrad (raster.rs:46-55), 48 bytes each
PROJECTED_DTYPE = np.dtype([("mean_xy", "<f4", 2), ("depth", "<f4"), ("radius", "<f4"), ("conic", "<f4", 3),
                            ("visible", "<f4"), ("color", "<f4", 3), ("opacity", "<f4")])
PROJECTED_GRAD_DTYPE = np.dtype([("dmean_opacity", "<f4", 4), ("dconic", "<f4", 4), ("dcolor", "<f4", 4)])
assert PROJECTED_DTYPE.itemsize == 48 and PROJECTED_GRAD_DTYPE.itemsize == 48


class CameraUniform:
    """CameraUniform (raster.rs:60-100); `.c` is the 96-byte C struct."""

    def __init__(self, c: sc_camera):
        self.c = c

    @classmethod
    def from_pose(cls, camera_pos, target, up, fov_y: float, width: int, height: int,
                  n_splats: int) -> "CameraUniform":
        e = (C.c_float * 3)(*map(float, camera_pos))
        t = (C.c_float * 3)(*map(float, target))
        u = (C.c_float * 3)(*map(float, up))
        c = sc_camera()
        lib().sc_camera_from_pose(e, t, u, float(fov_y), int(width), int(height), int(n_splats), C.byref(c))
        return cls(c)

    def as_array(self) -> np.ndarray:
        return np.frombuffer(bytes(self.c), dtype=np.uint8).copy()

    @property
    def view(self) -> np.ndarray:
        return np.array(self.c.view, np.float32).reshape(4, 4)  # [col][row]

    @property
    def focal(self) -> float:
        return float(self.c.focal)


def cameras_array(cams: list[CameraUniform]):
    arr = (sc_camera * len(cams))()
    for i, c in enumerate(cams):
        arr[i] = c.c
    return arr


def tiling_struct(p: TilingParams) -> sc_tiling:
    return sc_tiling(p.width, p.height, p.tile_w, p.tile_h, float(p.depth_max))


class Rasterizer:
    def __init__(self, ctx: CudaCtx):
        self.ctx = ctx

    # --- allocation helpers (raster.rs:460-552)
    def alloc_image(self, width: int, height: int, n_views: int = 1) -> DeviceBuffer:
        return self.ctx.storage_buffer_zeroed("predicted-image", n_views * width * height * 16)

    def alloc_aux(self, width: int, height: int, n_views: int = 1) -> DeviceBuffer:
        return self.ctx.storage_buffer_zeroed("forward-aux", n_views * width * height * 8)

    def alloc_projected(self, splats: GpuSplatBuffer, n_views: int = 1) -> DeviceBuffer:
        return self.ctx.storage_buffer_zeroed("projected", n_views * splats.capacity * 48)

    def alloc_projected_grad(self, splats: GpuSplatBuffer, n_views: int = 1) -> DeviceBuffer:
        return self.ctx.storage_buffer_zeroed("projected-grad", n_views * splats.capacity * 48)

    def zero_projected_grad(self, buf: DeviceBuffer) -> None:
        buf.zero()

    # --- passes
    def project(self, splats: GpuSplatBuffer, cameras, projected: DeviceBuffer) -> None:
        cams = cameras if isinstance(cameras, (list, tuple)) else [cameras]
        arr = cameras_array(cams)
        check(lib().sc_project(self.ctx.handle, splats.handle, arr, len(cams), projected.cptr), self.ctx.handle)

    def composite(self, projected: DeviceBuffer, bins: TileBinningResult, image: DeviceBuffer, params: TilingParams,
                  stride: int, n_views: int = 1, aux: DeviceBuffer | None = None) -> None:
        t = tiling_struct(params)
        check(lib().sc_composite(self.ctx.handle, projected.cptr, stride, n_views, bins.handle, C.byref(t), image.cptr,
                                 aux.cptr if aux is not None else None), self.ctx.handle)

    def composite_backward(self, projected: DeviceBuffer, bins: TileBinningResult, forward_out: DeviceBuffer,
                           dl_dc: DeviceBuffer, projected_grad: DeviceBuffer, params: TilingParams, stride: int,
                           n_views: int = 1, mode: int = SC_BWD_REF, aux: DeviceBuffer | None = None,
                           compensated: bool = False) -> None:
        """compensated: TwoSum-compensated per-(view, splat) totals across tiles
        (sc_composite_backward_ex with SC_BWD_FLAG_COMPENSATED)."""
        t = tiling_struct(params)
        check(lib().sc_composite_backward_ex(self.ctx.handle, projected.cptr, stride, n_views, bins.handle,
                                             C.byref(t), forward_out.cptr, dl_dc.cptr, int(mode),
                                             aux.cptr if aux is not None else None, projected_grad.cptr,
                                             1 if compensated else 0), self.ctx.handle)

    def project_backward(self, splats: GpuSplatBuffer, projected_grad: DeviceBuffer, camera: CameraUniform,
                         grads: GradSplatBuffers, accumulate: bool = False, view_offset: int = 0) -> None:
        pg = C.c_void_p(projected_grad.ptr + view_offset)
        check(lib().sc_project_backward(self.ctx.handle, splats.handle, pg, C.byref(camera.c), grads.handle,
                                        1 if accumulate else 0), self.ctx.handle)

    def mse_loss_grad(self, pred: DeviceBuffer, target: DeviceBuffer, params: TilingParams, dl_dc: DeviceBuffer,
                      n_views: int = 1, scale: float = 1.0) -> np.ndarray:
        t = tiling_struct(params)
        loss = self.ctx.storage_buffer_zeroed("loss", 8 * n_views)
        check(lib().sc_mse_loss_grad(self.ctx.handle, pred.cptr, target.cptr, n_views, C.byref(t), float(scale),
                                     dl_dc.cptr, loss.cptr), self.ctx.handle)
        sums = loss.readback(np.float64, n_views)
        return sums / (3.0 * params.width * params.height)

    def tonemap(self, image: DeviceBuffer, width: int, height: int, out: DeviceBuffer) -> None:
        check(lib().sc_tonemap(self.ctx.handle, image.cptr, width, height, out.cptr), self.ctx.handle)
