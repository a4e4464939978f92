"""Shared helpers for the GPU parity tests: run the device pipeline stage by
stage through the C ABI and feed the same intermediate arrays to the oracle."""
from __future__ import annotations

import math

import numpy as np

from nanotracer_b200 import CameraUniform, GpuSplatBuffer, Rasterizer, TileBinner, TilingParams
from nanotracer_b200._lib import SC_KEYS_NATIVE64, SC_KEYS_REF32
from nanotracer_b200.raster import PROJECTED_DTYPE
from nanotracer_b200.scene import FOV_Y, orbit_pose, random_scene

REC_FIELDS = ["mx", "my", "depth", "radius", "ca", "cb", "cc", "vis", "r", "g", "b", "op"]


def records_to_array(raw: np.ndarray) -> np.ndarray:
    """(n, 12) float32 view of ProjectedSplat records."""
    return np.ascontiguousarray(raw.view(np.float32).reshape(-1, 12))


def config1(n=5000, width=256, height=256, seed=0x5EED5EED):
    scene = random_scene(n, seed)
    eye, tgt, up = orbit_pose(0.0)
    cam = CameraUniform.from_pose(eye, tgt, up, FOV_Y, width, height, n)
    tl = TilingParams(width, height, 16, depth_max=8.0)
    return scene, cam, tl


class GpuPipe:
    """project -> bin -> composite -> backward on the device, keeping every
    intermediate for comparison."""

    def __init__(self, ctx, scene, cams, tl: TilingParams, key_mode=SC_KEYS_REF32, bf16=False):
        self.ctx, self.scene, self.tl = ctx, scene, tl
        self.cams = cams if isinstance(cams, list) else [cams]
        self.V = len(self.cams)
        self.g = GpuSplatBuffer.upload(ctx, scene, bf16_rest=bf16)
        self.r = Rasterizer(ctx)
        self.binner = TileBinner(ctx)
        self.key_mode = key_mode
        self.stride = self.g.capacity

    def project(self):
        self.proj = self.r.alloc_projected(self.g, self.V)
        self.r.project(self.g, self.cams, self.proj)
        raw = self.proj.readback(np.float32).reshape(self.V, self.stride, 12)
        return raw[:, : len(self.scene)]

    def bin(self):
        self.bins = self.binner.bin(self.proj, len(self.scene), self.tl, stride=self.stride, n_views=self.V,
                                    key_mode=self.key_mode)
        return self.bins.sorted_keys(), self.bins.sorted_payloads(), self.bins.tile_ranges()

    def composite(self):
        self.img = self.r.alloc_image(self.tl.width, self.tl.height, self.V)
        self.aux = self.r.alloc_aux(self.tl.width, self.tl.height, self.V)
        self.r.composite(self.proj, self.bins, self.img, self.tl, self.stride, self.V, aux=self.aux)
        img = self.img.readback(np.float32).reshape(self.V, self.tl.height, self.tl.width, 4)
        aux = self.aux.readback(np.uint32).reshape(self.V, self.tl.height, self.tl.width, 2)
        return img, aux

    def backward(self, dl_dc: np.ndarray, mode: int):
        self.dl = self.ctx.storage_buffer("dl_dc", np.ascontiguousarray(dl_dc, np.float32))
        self.pg = self.r.alloc_projected_grad(self.g, self.V)
        self.r.composite_backward(self.proj, self.bins, self.img, self.dl, self.pg, self.tl, self.stride, self.V,
                                  mode=mode, aux=self.aux)
        return self.pg.readback(np.float32).reshape(self.V, self.stride, 12)[:, : len(self.scene)]


def frac_close(a, b, atol, rtol=0.0):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return float(np.mean(d <= atol + rtol * np.abs(np.asarray(b, np.float64))))
