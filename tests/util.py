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


def small_scene(n=5000, width=256, height=256, seed=0x5EED5EED):
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

    def backward(self, dl_dc: np.ndarray, mode: int, compensated: bool = False):
        self.dl = self.ctx.storage_buffer("dl_dc", np.ascontiguousarray(dl_dc, np.float32))
        self.pg = self.r.alloc_projected_grad(self.g, self.V)
        self.r.composite_backward(self.proj, self.bins, self.img, self.dl, self.pg, self.tl, self.stride, self.V,
                                  mode=mode, aux=self.aux, compensated=compensated)
        return self.pg.readback(np.float32).reshape(self.V, self.stride, 12)[:, : len(self.scene)]


def frac_close(a, b, atol, rtol=0.0):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return float(np.mean(d <= atol + rtol * np.abs(np.asarray(b, np.float64))))


# ------------------------------------------------------------------ tolerances with stated causes
# Images: every pixel within IMG_ATOL of the oracle, except pixels whose
# forward walk passes near one of the blend's discontinuous tests: a pair test
# (alpha vs 1/255, alpha_raw vs 0.99, the quadratic form's sign) within THR_A
# (relative) of its threshold, or the transmittance stop (T vs 1e-4; in the
# reference backward also T vs 1.0001) within THR_T[mode].  There the GPU's
# ex2/rcp approximations (~1e-6 relative per pair, accumulated into T along a
# walk) may take the other branch.  Such exceptions are counted and bounded.
IMG_ATOL = 1e-4
THR_A = 1e-5
THR_T = {0: 3e-5, 1: 1e-4}    # by backward mode (0 = reference walk, 1 = exact)


def margins(oracle, rec, payloads, ranges, otl, mode):
    """(margin (H, W) in units of the tests' tolerances, bwd flags, fwd flags)."""
    return oracle.composite_margins(rec, payloads, np.asarray(ranges).reshape(-1), otl, mode, THR_A, THR_T[mode])


MAX_FLIP_FRAC = 1e-3          # at most this fraction of pixels may take the other branch
# Projected gradients: per component |gpu - oracle| <= GRAD_RTOL |oracle| +
# GRAD_ABS_REL A, A the oracle's sum over pixels of each term's magnitude
# before cancellation (oracle.composite_backward(want_abs=True)): the relative
# bar plus the rounding-error scale of a cancelling sum.  Splats in the walk
# of a near-threshold pixel are the stated exception.
GRAD_RTOL = 1e-3
GRAD_ABS_REL = 1e-4


def check_image_explained(gpu, ora, margin, atol=IMG_ATOL, max_frac=MAX_FLIP_FRAC, label=""):
    """gpu, ora (H, W, 4); margin (H, W) from margins().  Returns a summary
    dict (printed by the caller)."""
    d = np.abs(np.asarray(gpu, np.float64) - np.asarray(ora, np.float64)).reshape(-1, 4).max(axis=1)
    m = np.asarray(margin).reshape(-1)
    bad = d > atol
    unexplained = bad & (m >= 1.0)
    s = {"pixels": int(d.size), "beyond_atol": int(bad.sum()), "unexplained": int(unexplained.sum()),
         "near_threshold": int((m < 1.0).sum()), "max_err": float(d.max()),
         "max_err_explained_px": float(d[~bad].max()) if (~bad).any() else 0.0}
    if unexplained.any():
        i = int(np.flatnonzero(unexplained)[np.argmax(d[unexplained])])
        s["worst_unexplained"] = (i, float(d[i]), float(m[i]))
    assert not unexplained.any(), f"{label} pixels beyond {atol} with no near-threshold cause: {s}"
    assert bad.mean() <= max_frac, f"{label} too many near-threshold pixels: {s}"
    return s


PG_COLS = [0, 1, 2, 4, 5, 6, 8, 9, 10]  # dmean.xy, dopacity, dconic.abc, dcolor.rgb


def check_pg_explained(gpu, ora, absum, flags, rtol=GRAD_RTOL, arel=GRAD_ABS_REL, max_frac=MAX_FLIP_FRAC,
                       label=""):
    """Projected gradients (n, 12): per component within rtol |ora| + arel
    absum, except splats flagged by oracle.composite_margins."""
    g = np.asarray(gpu, np.float64)[:, PG_COLS]
    o = np.asarray(ora, np.float64)[:, PG_COLS]
    a = np.asarray(absum, np.float64)[:, PG_COLS]
    err = np.abs(g - o)
    ok_c = err <= rtol * np.abs(o) + arel * a
    bad = ~ok_c.all(axis=1)
    live = (np.abs(o) > 0).any(axis=1) | (np.abs(g) > 0).any(axis=1)
    unexplained = bad & ~np.asarray(flags, bool)
    pure = err <= rtol * np.abs(o)
    s = {"splats_with_grad": int(live.sum()), "beyond_bound": int(bad.sum()), "unexplained": int(unexplained.sum()),
         "flagged": int(np.asarray(flags, bool).sum()),
         "components_within_pure_rtol": float(pure[live].mean()) if live.any() else 1.0}
    if unexplained.any():
        i = int(np.flatnonzero(unexplained)[0])
        s["first_unexplained"] = (i, g[i].tolist(), o[i].tolist(), a[i].tolist())
    assert not unexplained.any(), f"{label} gradients beyond the bound with no near-threshold cause: {s}"
    assert bad.sum() <= max(1, max_frac * live.sum()), f"{label} too many flagged splats off the bound: {s}"
    return s


GROUPS = [(0, 3), (3, 7), (7, 10), (10, 11), (11, 14), (14, 59)]  # pos, rot, log-scale, logit, dc, rest


def check_param_grads(gpu, ora, rtol=GRAD_RTOL, label=""):
    """Per-splat parameter gradients (n, 59) from the same projected gradients:
    per parameter group |gpu - ora|_2 <= rtol |ora|_2 + 1e-6 |ora_splat|_2."""
    g, o = np.asarray(gpu, np.float64), np.asarray(ora, np.float64)
    tot = np.linalg.norm(o, axis=1)
    worst = 0.0
    for lo, hi in GROUPS:
        e = np.linalg.norm(g[:, lo:hi] - o[:, lo:hi], axis=1)
        r = np.linalg.norm(o[:, lo:hi], axis=1)
        bound = rtol * r + 1e-6 * tot
        bad = e > bound
        assert not bad.any(), f"{label} group {lo}:{hi}: {int(bad.sum())} splats, worst " \
                              f"{(e[bad] / np.maximum(r[bad], 1e-30)).max():.3g} relative"
        m = r > 0
        if m.any():
            worst = max(worst, float((e[m] / r[m]).max()))
    return {"worst_group_rel": worst}


def adam_first_step(theta, grads, lrs, b1=0.9, b2=0.999, eps=1e-15):
    """The oracle's Adam (t = 1, zero moments) over the six parameter groups,
    then the constraints: what the trainer's step does to the parameters."""
    from oracle import oracle as O
    th = np.array(theta, np.float32, copy=True)
    g = np.asarray(grads, np.float32)
    z = np.zeros_like(th[:, 0])
    for k, (lo, hi) in enumerate(GROUPS):
        p = np.ascontiguousarray(th[:, lo:hi])
        gg = np.ascontiguousarray(g[:, lo:hi])
        pn, _, _ = O.adam_step(p, gg, np.zeros_like(p), np.zeros_like(p), lrs[k], 1, b1, b2, eps)
        th[:, lo:hi] = pn.reshape(p.shape)
    rot, sc, op = O.apply_constraints(th[:, 3:7], th[:, 7:10], th[:, 10])
    th[:, 3:7], th[:, 7:10], th[:, 10] = rot.reshape(-1, 4), sc.reshape(-1, 3), op
    del z
    return th


def check_post_adam(gpu_theta, ora_theta, ora_grads, flags, alt_grads=None, unc=None, lrs=None, eps=1e-15,
                    label=""):
    """After one Adam step from zero moments a parameter moves by -lr sign(g):
    the trainer's parameters equal the oracle's except where a gradient's sign
    is not determined, i.e. in a (splat, group) with a component that is
    within GRAD_RTOL of the group's norm of zero (or below 1e-18, where FTZ
    differs), or whose oracle gradient differs in sign from alt_grads (the
    oracle's adjoint of the GPU's projected gradients, which the projected
    gradient bound certifies), or is within unc (the projected gradient
    bound's absolute term carried to the parameters: the rounding scale of
    the trainer's own sums), or a splat flagged near a threshold.  With lrs,
    a parameter whose gradient is of the order of Adam's eps moves by
    lr g / (|g| + eps), not lr sign(g): it is compared within that update's
    change under a GRAD_RTOL relative gradient error."""
    g, o, go = (np.asarray(x, np.float64) for x in (gpu_theta, ora_theta, ora_grads))
    tol = 1e-6 * np.abs(o) + 1e-7
    if lrs is not None:
        lr = np.zeros(o.shape[1])
        for k, (lo, hi) in enumerate(GROUPS):
            lr[lo:hi] = lrs[k]
        ag = np.abs(go)
        tol = tol + lr[None, :] * GRAD_RTOL * eps * ag / (ag + eps) ** 2
    close = np.abs(g - o) <= tol
    flags = np.asarray(flags, bool)
    ga = None if alt_grads is None else np.asarray(alt_grads, np.float64)
    n_bad, n_unexp = 0, 0
    for lo, hi in GROUPS:
        bad = ~close[:, lo:hi].all(axis=1)
        norm = np.linalg.norm(go[:, lo:hi], axis=1)
        near0 = (np.abs(go[:, lo:hi]) <= np.maximum(GRAD_RTOL * norm, 1e-18)[:, None]).any(axis=1)
        if ga is not None:  # the sign is open when the certified input difference reaches the gradient
            near0 |= (np.abs(go[:, lo:hi]) <= 1.01 * np.abs(ga[:, lo:hi] - go[:, lo:hi])).any(axis=1)
        if unc is not None:
            near0 |= (np.abs(go[:, lo:hi]) <= np.asarray(unc)[:, lo:hi]).any(axis=1)
        unexp = bad & ~near0 & ~flags
        if unexp.any():
            i = int(np.flatnonzero(unexp)[0])
            print({"unexplained_splat": i, "group": (lo, hi), "oracle_grad": go[i, lo:hi].tolist(),
                   "alt_grad": None if ga is None else ga[i, lo:hi].tolist(),
                   "unc": None if unc is None else np.asarray(unc)[i, lo:hi].tolist(),
                   "gpu_theta": g[i, lo:hi].tolist(), "oracle_theta": o[i, lo:hi].tolist()})
        n_bad += int(bad.sum())
        n_unexp += int(unexp.sum())
        assert not unexp.any(), f"{label} group {lo}:{hi}: {int(unexp.sum())} splats off with a determined sign " \
                                f"(first {int(np.flatnonzero(unexp)[0])})"
    s = {"groups_off": n_bad, "unexplained": n_unexp, "params": int(g.size),
         "params_equal_frac": float(close.mean())}
    assert n_bad <= max(1, 1e-3 * g.shape[0]), f"{label} too many groups off: {s}"
    return s


def check_same_first_step(a, b, lrs, max_frac=1e-4):
    """Parameters after one Adam step (zero moments) of two runs whose
    gradients differ only in float summation order: each parameter moved by
    -lr sign(g), so the runs agree to rounding except where a gradient's sign
    flipped, and there they differ by at most 2 lr of the parameter's group
    (the quaternion renormalisation spreads a flip over the splat's rotation).
    Such flips are counted and bounded."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.abs(a - b)
    same = d <= 1e-6 * np.abs(a) + 1e-7
    lr = np.zeros(a.shape[1])
    for k, (lo, hi) in enumerate(GROUPS):
        lr[lo:hi] = lrs[k]
    bound = 2.0 * lr[None, :] + 1e-5
    assert np.all(same | (d <= bound)), "a parameter moved further than a sign flip of its step"
    flipped = ~same
    assert flipped.mean() <= max_frac, f"{int(flipped.sum())} parameters differ"
    return {"params": int(a.size), "sign_flips": int(flipped.sum())}
