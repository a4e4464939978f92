"""Central finite differences in FP64 against the hand-written adjoint
(the uneven-batch workload's adjoint check): 64 random parameters of a 1000-splat scene at
64x64, h = 1e-3, MSE loss against a target rendered from a perturbed copy.

The loss is the oracle's FP64 instantiation end to end (projection, 64-bit
(tile, depth) binning, blend, MSE), evaluated at parameters perturbed in
their f32 storage: the difference quotient divides by the exact difference of
the two stored values.  Stated exceptions, each counted:
  * a parameter whose difference quotient at h and at h/2 disagree beyond
    1e-3 relative has a discontinuity (a pair crossing alpha = 1/255, a tile
    rectangle edge) inside [x - h, x + h]: no derivative to compare;
  * the reference adjoint omits the projection Jacobian's dependence on the
    position and the SH view direction's (project_backward.wgsl:18-24), so
    position gradients are compared at the reference FD test's relative
    tolerance (10 %, backward_finite_diff.rs:190-245) instead of 1e-3;
  * the adjoint does not gate the colour clamp max(c, 0)
    (project_gaussians.wgsl:150-154): SH parameters of a clamped channel have
    a zero difference quotient and are left out.
"""
from __future__ import annotations

import numpy as np

from nanotracer_b200.scene import FOV_Y, orbit_pose, perturbed, random_scene

N_SPLATS, W, H, TILE, H_FD = 1000, 64, 64, 16, 1e-3
# parameters drawn per group (64 in all): position, rotation, log-scale, opacity, SH DC, SH rest
DRAW = ((0, 3, 10), (3, 7, 14), (7, 10, 10), (10, 11, 8), (11, 14, 8), (14, 59, 14))
FD_RTOL = 1e-3
POS_RTOL = 0.10
SMOOTH_RTOL = 1e-3  # h vs h/2 agreement below which the quotient is a derivative


class Scene64:
    def __init__(self, oracle, seed=0xF64):
        self.O = oracle
        self.scene = random_scene(N_SPLATS, seed)
        eye, tgt, up = orbit_pose(0.0)
        self.cam = oracle.camera(eye, tgt, up, FOV_Y, W, H, N_SPLATS)
        self.tl = oracle.tiling(W, H, TILE, TILE, 8.0)
        t_img = self.render(oracle.OSplats.from_buffer(perturbed(self.scene)))[0]
        self.target = np.ascontiguousarray(t_img[..., :3], np.float32)

    def render(self, os_):
        O = self.O
        rec = O.project(os_, self.cam, "f64")
        _, pay, ranges = O.bin64(rec, 1, self.tl, "f64")
        img, ncon, tfin = O.composite(rec, pay, ranges.reshape(-1), self.tl, "f64")
        return img, rec, pay, ranges, ncon, tfin

    def loss(self, flat):
        os_ = self.O.OSplats.from_buffer(_from_flat(flat))
        img = self.render(os_)[0]
        loss, _ = self.O.mse(img, self.target, 1.0, "f64")
        return loss

    def adjoint_f64(self):
        O = self.O
        os_ = O.OSplats.from_buffer(self.scene)
        img, rec, pay, ranges, ncon, tfin = self.render(os_)
        _, dl = O.mse(img, self.target, 1.0, "f64")
        pg = O.composite_backward(rec, pay, ranges.reshape(-1), self.tl, img.reshape(-1, 4), dl, 1,
                                  ncon.reshape(-1), tfin.reshape(-1), "f64")
        return O.project_backward(os_, pg, self.cam, "f64"), rec

    def draw(self, grads, seed=0x5EED):
        """64 (splat, parameter) pairs among splats with a nonzero gradient."""
        rng = np.random.default_rng(seed)
        live = np.flatnonzero(np.abs(grads).sum(1) > 0)
        out = []
        for lo, hi, k in DRAW:
            splats = rng.choice(live, k, replace=False)
            cols = rng.integers(lo, hi, k)
            out += list(zip(splats.tolist(), cols.tolist()))
        return out

    def fd(self, i, c, h=H_FD):
        flat = self.scene.flat().astype(np.float32)
        lp, lm = flat.copy(), flat.copy()
        lp[i, c] = np.float32(float(flat[i, c]) + h)
        lm[i, c] = np.float32(float(flat[i, c]) - h)
        if 3 <= c < 7:  # a rotation stays a unit quaternion only to first order; the loss normalises it anyway
            pass
        return (self.loss(lp) - self.loss(lm)) / (float(lp[i, c]) - float(lm[i, c]))


def _from_flat(flat):
    from nanotracer_b200.splat_store import SplatBuffer
    return SplatBuffer.from_flat(np.asarray(flat, np.float32))


def clamped_channel(rec, i, c):
    """SH parameter c of splat i feeds a colour channel the projection clamped to 0."""
    if c < 11:
        return False
    ch = (c - 11) if c < 14 else (c - 14) // 15
    return rec[i, 8 + ch] == 0.0


def compare(scene64: Scene64, adjoint, params, rec):
    """Returns (rows, summary); asserts the bounds above."""
    rows = []
    for i, c in params:
        f1 = scene64.fd(i, c)
        f2 = scene64.fd(i, c, H_FD / 2)
        a = float(adjoint[i, c])
        smooth = abs(f1 - f2) <= SMOOTH_RTOL * max(abs(f1), abs(f2)) + 1e-12
        cause = None
        if not smooth:
            cause = "discontinuity within h"
        elif clamped_channel(rec, i, c):
            cause = "colour clamp (not gated by the reference adjoint)"
        tol = (POS_RTOL if c < 3 else FD_RTOL) * abs(f1) + 1e-9 * max(1.0, abs(f1))
        rows.append({"splat": i, "param": c, "adjoint": a, "fd": f1, "fd_half_h": f2, "cause": cause,
                     "ok": cause is not None or abs(a - f1) <= tol, "rel": abs(a - f1) / max(abs(f1), 1e-30)})
    bad = [r for r in rows if not r["ok"]]
    n_exc = sum(r["cause"] is not None for r in rows)
    checked = [r for r in rows if r["cause"] is None]
    summary = {"params": len(rows), "checked": len(checked), "excepted": n_exc,
               "rot_checked": sum(3 <= r["param"] < 7 for r in checked),
               "max_rel_nonpos": max([r["rel"] for r in checked if r["param"] >= 3] or [0.0]),
               "max_rel_pos": max([r["rel"] for r in checked if r["param"] < 3] or [0.0])}
    assert not bad, (summary, bad[:3])
    assert n_exc <= 16, (summary, [r for r in rows if r["cause"]][:5])
    assert summary["rot_checked"] >= 8, summary
    return rows, summary
