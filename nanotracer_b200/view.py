"""Headless forward path of the viewer: the compute pass of nano-view's frame
(crates/nano-view/src/lib.rs:762-795) — CameraUniform from the orbit pose,
project, bin with 16x16 tiles and depth_max = max(4 * orbit distance, 50),
composite, tonemap — into an RGBA8 device buffer instead of a swapchain
texture.  There is no window here; frame() returns the pixels."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._lib import SC_KEYS_REF32
from .gpu import CudaCtx
from .raster import CameraUniform, Rasterizer
from .splat_gpu import GpuSplatBuffer
from .splat_store import SplatBuffer
from .tile_binner import TileBinner, TilingParams


@dataclass
class OrbitCamera:
    """nano-view's OrbitCamera (lib.rs:152-169): spherical pose around a target."""

    target: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    distance: float = 4.0
    azimuth: float = 0.0
    elevation: float = 0.0
    fov_y: float = math.radians(50.0)

    def position(self) -> np.ndarray:
        # lib.rs:161-168, in f32
        ce = np.float32(math.cos(np.float32(self.elevation)))
        d = np.float32(self.distance)
        t = np.asarray(self.target, np.float32)
        return np.array([t[0] + d * ce * np.float32(math.cos(np.float32(self.azimuth))),
                         t[1] + d * np.float32(math.sin(np.float32(self.elevation))),
                         t[2] + d * ce * np.float32(math.sin(np.float32(self.azimuth)))], np.float32)


class HeadlessView:
    """One viewport: the device splat store plus the per-frame buffers."""

    TILE = 16

    def __init__(self, ctx: CudaCtx, splats: SplatBuffer | GpuSplatBuffer, width: int, height: int):
        self.ctx = ctx
        self.splats = splats if isinstance(splats, GpuSplatBuffer) else GpuSplatBuffer.upload(ctx, splats)
        self.width, self.height = int(width), int(height)
        self.rasterizer = Rasterizer(ctx)
        self.binner = TileBinner(ctx)
        self.projected = self.rasterizer.alloc_projected(self.splats, 1)
        self.image = self.rasterizer.alloc_image(self.width, self.height, 1)
        self.rgba8 = ctx.storage_buffer_zeroed("rgba8", 4 * self.width * self.height)

    def tiling(self, orbit: OrbitCamera) -> TilingParams:
        return TilingParams(self.width, self.height, self.TILE, max(orbit.distance * 4.0, 50.0))

    def frame(self, orbit: OrbitCamera) -> np.ndarray:
        """Render one frame; returns (height, width, 4) uint8 (sRGB, alpha = coverage)."""
        n = self.splats.n
        cam = CameraUniform.from_pose(orbit.position(), np.asarray(orbit.target, np.float32), (0.0, 1.0, 0.0),
                                      orbit.fov_y, self.width, self.height, n)
        self.rasterizer.project(self.splats, [cam], self.projected)
        params = self.tiling(orbit)
        bins = self.binner.bin(self.projected, n, params, stride=self.splats.capacity, n_views=1,
                               key_mode=SC_KEYS_REF32)
        self.rasterizer.composite(self.projected, bins, self.image, params, self.splats.capacity, 1)
        self.rasterizer.tonemap(self.image, self.width, self.height, self.rgba8)
        return self.rgba8.readback(np.uint8).reshape(self.height, self.width, 4)

    def hdr(self) -> np.ndarray:
        """The last frame before tonemapping: (height, width, 4) float32 (rgb, 1 - T)."""
        return self.image.readback(np.float32).reshape(self.height, self.width, 4)
