"""Host-side splat parameters — the mirror of nano-optimize's SplatBuffer
(crates/nano-optimize/src/splat_store.rs:20-133) and nano-splat's Gaussian
(crates/nano-splat/src/ply.rs:6-15).

SoA numpy arrays: positions (n,3), rotations (n,4) as (w,x,y,z), scales (n,3)
log-sigma, opacities (n,) logit, sh_dc (n,3), sh_rest (n,45) planar
R[15] G[15] B[15].  The same container holds gradients and Adam moments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import sc_host_splats

FIELDS = (("positions", 3), ("rotations", 4), ("scales", 3), ("opacities", 1), ("sh_dc", 3), ("sh_rest", 45))


@dataclass
class Gaussian:
    """One Inria 3DGS splat as PLY stores it (ply.rs:6-15)."""
    pos: np.ndarray
    normal: np.ndarray
    sh_dc: np.ndarray
    sh_rest: np.ndarray
    opacity: float
    scale: np.ndarray
    rotation: np.ndarray


def _empty(n: int) -> dict[str, np.ndarray]:
    return {name: np.zeros((n, w) if w > 1 else (n,), np.float32) for name, w in FIELDS}


@dataclass
class SplatBuffer:
    positions: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    rotations: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.float32))
    scales: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    opacities: np.ndarray = field(default_factory=lambda: np.zeros((0,), np.float32))
    sh_dc: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    sh_rest: np.ndarray = field(default_factory=lambda: np.zeros((0, 45), np.float32))

    def __post_init__(self):
        for name, w in FIELDS:
            a = np.ascontiguousarray(getattr(self, name), dtype=np.float32)
            setattr(self, name, a.reshape((-1, w)) if w > 1 else a.reshape(-1))

    @classmethod
    def zeros(cls, n: int) -> "SplatBuffer":
        return cls(**_empty(n))

    def __len__(self) -> int:
        return int(self.positions.shape[0])

    def copy(self) -> "SplatBuffer":
        return SplatBuffer(**{name: getattr(self, name).copy() for name, _ in FIELDS})

    # splat_store.rs:60-79
    @classmethod
    def from_gaussians(cls, gs: list[Gaussian]) -> "SplatBuffer":
        out = cls.zeros(len(gs))
        for i, g in enumerate(gs):
            out.positions[i] = g.pos
            out.rotations[i] = g.rotation
            out.scales[i] = g.scale
            out.opacities[i] = g.opacity
            out.sh_dc[i] = g.sh_dc
            rest = np.zeros(45, np.float32)
            r = np.asarray(g.sh_rest, np.float32)[:45]
            rest[: r.shape[0]] = r
            out.sh_rest[i] = rest
        return out

    # splat_store.rs:82-94
    def to_gaussians(self) -> list[Gaussian]:
        return [Gaussian(self.positions[i].copy(), np.array([0.0, 1.0, 0.0], np.float32), self.sh_dc[i].copy(),
                         self.sh_rest[i].copy(), float(self.opacities[i]), self.scales[i].copy(),
                         self.rotations[i].copy()) for i in range(len(self))]

    # splat_store.rs:99-113
    def swap_remove(self, i: int) -> None:
        last = len(self) - 1
        for name, _ in FIELDS:
            a = getattr(self, name)
            a[i] = a[last]
            setattr(self, name, a[:last].copy())

    # splat_store.rs:116-132
    def push_splat(self, pos, rotation, scale, opacity, sh_dc, sh_rest_45) -> None:
        vals = dict(positions=pos, rotations=rotation, scales=scale, opacities=[opacity], sh_dc=sh_dc,
                    sh_rest=sh_rest_45)
        for name, w in FIELDS:
            a = getattr(self, name)
            v = np.asarray(vals[name], np.float32).reshape((1, w) if w > 1 else (1,))
            setattr(self, name, np.concatenate([a, v]))

    def host_struct(self) -> sc_host_splats:
        """ctypes view for the C ABI; keeps no copy (arrays must stay alive)."""
        h = sc_host_splats()
        h.n = len(self)
        for name, _ in FIELDS:
            setattr(h, name, C.c_void_p(getattr(self, name).ctypes.data))
        return h

    def flat(self) -> np.ndarray:
        """All 59 parameters per splat, (n, 59), in slab row order."""
        return np.concatenate([self.positions, self.rotations, self.scales, self.opacities[:, None], self.sh_dc,
                               self.sh_rest], axis=1)

    @classmethod
    def from_flat(cls, a: np.ndarray) -> "SplatBuffer":
        a = np.asarray(a, np.float32)
        return cls(a[:, 0:3], a[:, 3:7], a[:, 7:10], a[:, 10], a[:, 11:14], a[:, 14:59])
