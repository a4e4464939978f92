"""The headless viewer frame (view.py, nano-view/src/lib.rs:762-795):
project -> bin (REF32 keys, depth_max = max(4 d, 50)) -> composite -> tonemap,
against the oracle's forward on the same projected records."""
import math

import numpy as np
import pytest

from nanotracer_b200.scene import random_scene
from nanotracer_b200.view import HeadlessView, OrbitCamera


def _tonemap(img):
    def srgb(c):
        c = np.clip(c, 0, 1)
        return np.where(c > 0.0031308, 1.055 * c ** (1 / 2.4) - 0.055, c * 12.92)
    rgb = img[..., :3] / (1 + np.maximum(img[..., :3], 0))
    return np.concatenate([np.round(np.clip(srgb(rgb), 0, 1) * 255), np.round(np.clip(img[..., 3:], 0, 1) * 255)], -1)


def test_orbit_camera_position():
    o = OrbitCamera(target=np.array([1, 2, 3], np.float32), distance=2.0, azimuth=0.0, elevation=math.pi / 2)
    assert np.allclose(o.position(), [1, 4, 3], atol=1e-6)
    o = OrbitCamera(distance=3.0, azimuth=math.pi / 2, elevation=0.0)
    assert np.allclose(o.position(), [0, 0, 3], atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("azimuth,elevation", [(0.3, 0.2), (2.0, -0.4)])
def test_frame_matches_oracle_forward(ctx, oracle, azimuth, elevation):
    W, H = 320, 200
    scene = random_scene(4000, 17)
    view = HeadlessView(ctx, scene, W, H)
    orbit = OrbitCamera(distance=4.0, azimuth=azimuth, elevation=elevation)
    px = view.frame(orbit)
    hdr = view.hdr()
    assert px.shape == (H, W, 4) and px.dtype == np.uint8
    assert np.abs(px.astype(int) - _tonemap(hdr).astype(int)).max() <= 1
    # the oracle composites the device's projected records with its own REF32 binning
    rec = view.projected.readback(np.float32).reshape(-1, 12)[: len(scene)]
    tl = oracle.tiling(W, H, 16, 16, max(4.0 * 4.0, 50.0))
    _, pay, ranges = oracle.bin_ref(rec, tl)
    want, _, _ = oracle.composite(rec, pay, ranges, tl)
    assert np.mean(np.abs(hdr - want) <= 1e-4) > 0.999
    assert (hdr[..., 3] > 0).mean() > 0.05  # something was drawn
