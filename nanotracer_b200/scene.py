"""Seeded synthetic scenes and cameras (no dataset, no network).

One seed drives every field: means U[-1,1]^3, log-scales N(ln 0.03, 0.3) per
axis, rotations normalise(N(0,1)^4) stored (w,x,y,z), opacity logits N(0,1),
SH DC N(0,0.3), SH rest (45, planar) N(0,0.05).  The target scene is a copy
with every field perturbed by N(0,0.05) and its quaternions renormalised.
Cameras are pinholes on a radius-4 orbit looking at the origin, up +Y,
50 degree vertical field of view.
"""
from __future__ import annotations

import math

import numpy as np

from .splat_store import SplatBuffer


def random_scene(n: int, seed: int = 0x5EED5EED) -> SplatBuffer:
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, (n, 3))
    scales = rng.normal(math.log(0.03), 0.3, (n, 3))
    q = rng.normal(0.0, 1.0, (n, 4))
    q /= np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
    op = rng.normal(0.0, 1.0, n)
    dc = rng.normal(0.0, 0.3, (n, 3))
    rest = rng.normal(0.0, 0.05, (n, 45))
    return SplatBuffer(pos, q, scales, op, dc, rest)


def perturbed(s: SplatBuffer, sigma: float = 0.05, seed: int = 0x7A56E7) -> SplatBuffer:
    rng = np.random.default_rng(seed)
    f = s.flat().astype(np.float64)
    f = f + rng.normal(0.0, sigma, f.shape)
    q = f[:, 3:7]
    q /= np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
    f[:, 3:7] = q
    return SplatBuffer.from_flat(f.astype(np.float32))


def orbit_pose(angle_deg: float, elevation_deg: float = 0.0, radius: float = 4.0):
    a, e = math.radians(angle_deg), math.radians(elevation_deg)
    eye = (radius * math.cos(e) * math.sin(a), radius * math.sin(e), radius * math.cos(e) * math.cos(a))
    return eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0)


def orbit_views(n_views: int, step: int = 0, jitter_deg: float = 10.0, seed: int = 0xCA3E7A):
    """n_views poses spread around the orbit, advanced 3 degrees per step, with
    seeded elevation jitter in [-jitter_deg, +jitter_deg]."""
    rng = np.random.default_rng(seed + step)
    poses = []
    for v in range(n_views):
        ang = 3.0 * step + 360.0 * v / n_views
        el = float(rng.uniform(-jitter_deg, jitter_deg)) if jitter_deg > 0 else 0.0
        poses.append(orbit_pose(ang, el))
    return poses


FOV_Y = math.radians(50.0)
