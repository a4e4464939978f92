"""Python face of the CPU oracle (oracle/splat_oracle.cpp) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm load this module, and only as the checker or the timed CPU baseline.  The
product library never links or calls it.

Parity status: the oracle restates the reference's WGSL kernels and Rust host
code (file:line citations in splat_oracle.cpp).  It is pinned against every
known-answer test the reference's own suite holds for this path (ported in
tests/test_oracle_kats.py and tests/golden/reference_kats.json); the reference
itself (Rust + wgpu) cannot be built or run here, so floating-point parity
beyond those tests' tolerances is "parity unpinned".
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libsplat_oracle.so"


class HostSplats(C.Structure):
    _fields_ = [("n", C.c_uint32), ("pos", C.c_void_p), ("rot", C.c_void_p), ("scale", C.c_void_p),
                ("opacity", C.c_void_p), ("sh_dc", C.c_void_p), ("sh_rest", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("cam_pos", C.c_float * 3), ("near_plane", C.c_float),
                ("focal", C.c_float), ("width", C.c_float), ("height", C.c_float), ("n_splats", C.c_uint32)]


class Tiling(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("tile_w", C.c_uint32), ("tile_h", C.c_uint32),
                ("depth_max", C.c_float)]


class AdamGroups(C.Structure):
    _fields_ = [("lr", C.c_float * 6), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


_lib = None


def build() -> Path:
    src = HERE / "splat_oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        P, U32, U64, F32, I32, D = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_int, C.c_double
        protos = {
            "oracle_set_threads": (None, [I32]),
            "oracle_max_threads": (I32, []),
            "oracle_camera_from_pose": (None, [P, P, P, F32, U32, U32, U32, C.POINTER(Camera)]),
            "oracle_powi_f32": (F32, [F32, I32]),
            "oracle_adam_step": (None, [U64, P, P, P, P, F32, F32, F32, F32, U64]),
            "oracle_apply_constraints": (None, [U32, P, P, P, F32, F32, F32]),
            "oracle_accumulate_grad": (None, [U32, P, P]),
            "oracle_prune": (U32, [C.POINTER(HostSplats), C.POINTER(HostSplats), C.POINTER(HostSplats), P, F32,
                                   C.POINTER(U32)]),
            "oracle_densify": (U32, [C.POINTER(HostSplats), C.POINTER(HostSplats), C.POINTER(HostSplats), P, U32,
                                     F32, F32, U32, U32, P]),
            "oracle_write_ply": (I32, [C.c_char_p, C.POINTER(HostSplats)]),
            "oracle_read_ply": (C.c_int64, [C.c_char_p, C.POINTER(HostSplats), U32]),
        }
        for sfx in ("f32", "f64"):
            protos.update({
                f"oracle_project_{sfx}": (None, [C.POINTER(HostSplats), C.POINTER(Camera), P]),
                f"oracle_bin_ref_{sfx}": (C.c_int64, [U32, P, C.POINTER(Tiling), P, P, U64, P]),
                f"oracle_bin64_{sfx}": (C.c_int64, [U32, U32, P, C.POINTER(Tiling), P, P, U64, P]),
                f"oracle_composite_{sfx}": (None, [P, P, P, C.POINTER(Tiling), P, P, P]),
                f"oracle_mse_{sfx}": (D, [U64, P, P, P, F32]),
                f"oracle_composite_backward_{sfx}": (None, [P, P, P, C.POINTER(Tiling), P, P, I32, P, P, P, P]),
                f"oracle_composite_margins_{sfx}": (None, [P, P, P, C.POINTER(Tiling), I32, D, D, P, P]),
                f"oracle_project_backward_{sfx}": (None, [C.POINTER(HostSplats), P, C.POINTER(Camera), P, P, P, P, P,
                                                          P, I32]),
                f"oracle_train_step_{sfx}": (D, [C.POINTER(HostSplats), C.POINTER(HostSplats), C.POINTER(HostSplats),
                                                 P, U32, P, P, C.POINTER(Tiling), I32, C.POINTER(AdamGroups), U64, P,
                                                 F32, P]),
                f"oracle_ssim_loss_grad_{sfx}": (D, [I32, I32, P, P, P, F32]),
                f"oracle_combined_loss_grad_{sfx}": (D, [I32, I32, P, P, P, F32, F32, P]),
            })
        for name, (res, args) in protos.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _dt(sfx):
    return np.float32 if sfx == "f32" else np.float64


class OSplats:
    """Flat host arrays with spare capacity (prune/densify grow in place)."""

    def __init__(self, pos, rot, scale, op, dc, rest, capacity=None):
        n = len(op)
        cap = max(n, capacity or n)
        self.arrays = []
        for a, w in ((pos, 3), (rot, 4), (scale, 3), (op, 1), (dc, 3), (rest, 45)):
            buf = np.zeros(cap * w, np.float32)
            buf[: n * w] = np.asarray(a, np.float32).reshape(-1)
            self.arrays.append(buf)
        self.h = HostSplats(n, *[C.c_void_p(b.ctypes.data) for b in self.arrays])

    @classmethod
    def from_buffer(cls, sb, capacity=None):
        return cls(sb.positions, sb.rotations, sb.scales, sb.opacities, sb.sh_dc, sb.sh_rest, capacity)

    @classmethod
    def zeros(cls, n, capacity=None):
        return cls(np.zeros((n, 3)), np.zeros((n, 4)), np.zeros((n, 3)), np.zeros(n), np.zeros((n, 3)),
                   np.zeros((n, 45)), capacity)

    @property
    def n(self):
        return self.h.n

    @property
    def capacity(self):
        return len(self.arrays[3])

    def reserve(self, cap):
        """Grow the backing arrays (the reference's Vecs grow on push)."""
        if cap <= self.capacity:
            return
        n = self.n
        for k, w in enumerate((3, 4, 3, 1, 3, 45)):
            buf = np.zeros(cap * w, np.float32)
            buf[: n * w] = self.arrays[k][: n * w]
            self.arrays[k] = buf
        self.h = HostSplats(n, *[C.c_void_p(b.ctypes.data) for b in self.arrays])

    def get(self):
        n = self.n
        w = (3, 4, 3, 1, 3, 45)
        out = [self.arrays[k][: n * w[k]].reshape(n, w[k]) if w[k] > 1 else self.arrays[k][:n] for k in range(6)]
        return out  # pos, rot, scale, op, dc, rest

    def flat(self):
        pos, rot, sc, op, dc, rest = self.get()
        return np.concatenate([pos, rot, sc, op[:, None], dc, rest], axis=1)


def camera(eye, target, up, fov_y, w, h, n=0) -> Camera:
    c = Camera()
    e = (C.c_float * 3)(*eye); t = (C.c_float * 3)(*target); u = (C.c_float * 3)(*up)
    lib().oracle_camera_from_pose(e, t, u, float(fov_y), int(w), int(h), int(n), C.byref(c))
    return c


def camera_from_struct(raw: bytes) -> Camera:
    c = Camera()
    C.memmove(C.byref(c), raw, C.sizeof(Camera))
    return c


def tiling(w, h, tw=16, th=None, depth_max=100.0) -> Tiling:
    return Tiling(int(w), int(h), int(tw), int(th or tw), float(depth_max))


def project(s: OSplats, cam: Camera, sfx="f32") -> np.ndarray:
    out = np.zeros(s.n * 12, _dt(sfx))
    getattr(lib(), f"oracle_project_{sfx}")(C.byref(s.h), C.byref(cam), _p(out))
    return out.reshape(s.n, 12)


def bin_ref(rec: np.ndarray, tl: Tiling, sfx="f32"):
    rec = np.ascontiguousarray(rec, _dt(sfx))
    n = rec.shape[0]
    nt = ((tl.width + tl.tile_w - 1) // tl.tile_w) * ((tl.height + tl.tile_h - 1) // tl.tile_h)
    ranges = np.zeros(2 * nt, np.uint32)
    f = getattr(lib(), f"oracle_bin_ref_{sfx}")
    K = f(n, _p(rec), C.byref(tl), None, None, 0, _p(ranges))
    K = -K if K < 0 else K
    keys = np.zeros(max(K, 1), np.uint32)
    pay = np.zeros(max(K, 1), np.uint32)
    K2 = f(n, _p(rec), C.byref(tl), _p(keys), _p(pay), K, _p(ranges))
    assert K2 == K
    return keys[:K], pay[:K], ranges.reshape(nt, 2)


def bin_ref_views(rec: np.ndarray, n_views: int, tl: Tiling, sfx="f32"):
    """bin_ref for each of n_views views (rec: the views' records one after
    another), laid out as sc_bin lays out the 32-bit keys of several views:
    key ((view * tiles + tile) << 16) | depth16, payloads view after view,
    ranges indexed by view * tiles + tile at positions in the whole array
    ((0, 0) for an empty tile)."""
    rec = np.asarray(rec).reshape(n_views, -1, 12)
    ks, ps, rs, base = [], [], [], 0
    for v in range(n_views):
        k, p, r = bin_ref(rec[v], tl, sfx)
        nt = r.shape[0]
        assert n_views * nt <= 1 << 16, "view * tiles + tile must fit 16 bits"
        ks.append(k.astype(np.uint32) + np.uint32((v * nt) << 16))
        ps.append(p)
        r = r.astype(np.uint64)
        full = r[:, 1] > r[:, 0]
        r[full] += base
        rs.append(r.astype(np.uint32))
        base += len(k)
    return np.concatenate(ks), np.concatenate(ps), np.concatenate(rs)


def bin64(rec: np.ndarray, n_views: int, tl: Tiling, sfx="f32"):
    rec = np.ascontiguousarray(rec, _dt(sfx))
    n = rec.shape[0] // n_views
    nt = ((tl.width + tl.tile_w - 1) // tl.tile_w) * ((tl.height + tl.tile_h - 1) // tl.tile_h)
    ranges = np.zeros(2 * nt * n_views, np.uint32)
    f = getattr(lib(), f"oracle_bin64_{sfx}")
    K = f(n_views, n, _p(rec), C.byref(tl), None, None, 0, _p(ranges))
    K = -K if K < 0 else K
    keys = np.zeros(max(K, 1), np.uint64)
    pay = np.zeros(max(K, 1), np.uint32)
    K2 = f(n_views, n, _p(rec), C.byref(tl), _p(keys), _p(pay), K, _p(ranges))
    assert K2 == K
    return keys[:K], pay[:K], ranges.reshape(nt * n_views, 2)


def composite(rec, payloads, ranges, tl: Tiling, sfx="f32"):
    rec = np.ascontiguousarray(rec, _dt(sfx))
    P = tl.width * tl.height
    out = np.zeros(P * 4, _dt(sfx))
    ncon = np.zeros(P, np.uint32)
    tfin = np.zeros(P, _dt(sfx))
    getattr(lib(), f"oracle_composite_{sfx}")(_p(rec), _p(np.ascontiguousarray(payloads, np.uint32)),
                                              _p(np.ascontiguousarray(ranges, np.uint32)), C.byref(tl), _p(out),
                                              _p(ncon), _p(tfin))
    return out.reshape(tl.height, tl.width, 4), ncon.reshape(tl.height, tl.width), tfin.reshape(tl.height, tl.width)


def mse(pred4, target3, scale=1.0, sfx="f32"):
    pred4 = np.ascontiguousarray(pred4, _dt(sfx)).reshape(-1)
    t = np.ascontiguousarray(target3, np.float32).reshape(-1)
    P = pred4.shape[0] // 4
    dl = np.zeros(P * 4, _dt(sfx))
    loss = getattr(lib(), f"oracle_mse_{sfx}")(P, _p(pred4), _p(t), _p(dl), float(scale))
    return loss, dl


def composite_backward(rec, payloads, ranges, tl: Tiling, fwd, dl_dc, mode=0, ncon=None, tfin=None, sfx="f32",
                       want_abs=False):
    """Projected gradients (n, 12); with want_abs also the per-component sums
    of the pixels' absolute terms (the scale of the sum's rounding error)."""
    rec = np.ascontiguousarray(rec, _dt(sfx))
    n = rec.shape[0]
    pg = np.zeros(n * 12, _dt(sfx))
    ab = np.zeros(n * 12, _dt(sfx)) if want_abs else None
    fwd = np.ascontiguousarray(fwd, _dt(sfx))
    dl = np.ascontiguousarray(dl_dc, _dt(sfx))
    nc = None if ncon is None else np.ascontiguousarray(ncon, np.uint32)
    tf = None if tfin is None else np.ascontiguousarray(tfin, _dt(sfx))
    getattr(lib(), f"oracle_composite_backward_{sfx}")(_p(rec), _p(np.ascontiguousarray(payloads, np.uint32)),
                                                       _p(np.ascontiguousarray(ranges, np.uint32)), C.byref(tl),
                                                       _p(fwd), _p(dl), int(mode), _p(nc), _p(tf), _p(pg), _p(ab))
    return (pg.reshape(n, 12), ab.reshape(n, 12)) if want_abs else pg.reshape(n, 12)


def composite_margins(rec, payloads, ranges, tl: Tiling, mode=1, thr_a=1e-5, thr_t=1e-4, sfx="f32"):
    """Near-threshold diagnostics of one view (test infrastructure; see
    composite_margins in splat_oracle.cpp).  Returns (margin (H, W): the
    forward walk's smallest distance to a blend threshold in units of the
    test's tolerance, below 1 = the pixel may render differently; bwd (n,)
    bool: splats whose gradient may differ when both sides differentiate the
    same forward; fwd (n,) bool: splats whose gradient may differ when each
    side differentiates its own forward)."""
    rec = np.ascontiguousarray(rec, _dt(sfx))
    n = rec.shape[0]
    margin = np.zeros(tl.width * tl.height, np.float32)
    flags = np.zeros(max(n, 1), np.uint8)
    getattr(lib(), f"oracle_composite_margins_{sfx}")(_p(rec), _p(np.ascontiguousarray(payloads, np.uint32)),
                                                      _p(np.ascontiguousarray(ranges, np.uint32)), C.byref(tl),
                                                      int(mode), float(thr_a), float(thr_t), _p(margin), _p(flags))
    f = flags[:n]
    return margin.reshape(tl.height, tl.width), (f & 1).astype(bool), (f & 2).astype(bool)


def project_backward(s: OSplats, pg, cam: Camera, sfx="f32"):
    n = s.n
    pg = np.ascontiguousarray(pg, _dt(sfx))
    outs = [np.zeros(n * w, _dt(sfx)) for w in (3, 4, 3, 1, 3, 45)]
    getattr(lib(), f"oracle_project_backward_{sfx}")(C.byref(s.h), _p(pg), C.byref(cam), *[_p(o) for o in outs], 0)
    return np.concatenate([outs[0].reshape(n, 3), outs[1].reshape(n, 4), outs[2].reshape(n, 3),
                           outs[3].reshape(n, 1), outs[4].reshape(n, 3), outs[5].reshape(n, 45)], axis=1)


def adam_step(p, g, m, v, lr, t, b1=0.9, b2=0.999, eps=1e-15):
    p, g, m, v = (np.ascontiguousarray(x, np.float32).copy() for x in (p, g, m, v))
    lib().oracle_adam_step(p.size, _p(p), _p(g), _p(m), _p(v), lr, b1, b2, eps, int(t))
    return p, m, v


def apply_constraints(rot, scale, op, lsmin=-10.0, lsmax=5.0, opmax=10.0):
    rot, scale, op = (np.ascontiguousarray(x, np.float32).copy() for x in (rot, scale, op))
    lib().oracle_apply_constraints(op.size, _p(rot), _p(scale), _p(op), lsmin, lsmax, opmax)
    return rot, scale, op


def accumulate_grad(dpos, acc):
    dpos, acc = np.ascontiguousarray(dpos, np.float32), np.ascontiguousarray(acc, np.float32).copy()
    lib().oracle_accumulate_grad(acc.size, _p(dpos), _p(acc))
    return acc


def prune(s: OSplats, m: OSplats | None, v: OSplats | None, acc, threshold):
    removed = C.c_uint32()
    n = lib().oracle_prune(C.byref(s.h), C.byref(m.h) if m else None, C.byref(v.h) if v else None, _p(acc),
                           float(threshold), C.byref(removed))
    if m: m.h.n = n
    if v: v.h.n = n
    return removed.value


def densify(s: OSplats, m, v, acc, grad_count, gthr, sthr, max_splats, it):
    """acc must hold n + 2 * max(0, max_splats - n) entries: children are
    appended before their parents are swap-removed (train.rs:486-546)."""
    counts = np.zeros(3, np.uint32)
    room = s.n + 2 * max(0, int(max_splats) - s.n)
    for b in (s, m, v):
        if b is not None:
            b.reserve(room)
    assert acc is None or len(acc) >= room, "grad_acc needs room for the transient children"
    n = lib().oracle_densify(C.byref(s.h), C.byref(m.h) if m else None, C.byref(v.h) if v else None, _p(acc),
                             int(grad_count), float(gthr), float(sthr), int(max_splats), int(it), _p(counts))
    if m: m.h.n = n
    if v: v.h.n = n
    return tuple(int(c) for c in counts)


def write_ply(path, s: OSplats):
    return lib().oracle_write_ply(str(path).encode(), C.byref(s.h))


def read_ply(path, cap):
    out = OSplats.zeros(0, cap)
    r = lib().oracle_read_ply(str(path).encode(), C.byref(out.h), int(cap))
    return r, out


def ssim(pred4, target3, w, h, scale=1.0, sfx="f32"):
    """loss.rs:340-375: (1 - mean SSIM over the three channels, scale * dL/dC as rgba)."""
    pred4 = np.ascontiguousarray(pred4, _dt(sfx)).reshape(-1)
    t = np.ascontiguousarray(target3, np.float32).reshape(-1)
    dl = np.zeros(w * h * 4, _dt(sfx))
    loss = getattr(lib(), f"oracle_ssim_loss_grad_{sfx}")(int(w), int(h), _p(pred4), _p(t), _p(dl), float(scale))
    return loss, dl


def combined(pred4, target3, w, h, lam, scale=1.0, sfx="f32"):
    """loss.rs:383-410: (total, mse, ssim, scale * dL/dC as rgba)."""
    pred4 = np.ascontiguousarray(pred4, _dt(sfx)).reshape(-1)
    t = np.ascontiguousarray(target3, np.float32).reshape(-1)
    dl = np.zeros(w * h * 4, _dt(sfx))
    parts = np.zeros(2, np.float64)
    total = getattr(lib(), f"oracle_combined_loss_grad_{sfx}")(int(w), int(h), _p(pred4), _p(t), _p(dl),
                                                               float(lam), float(scale), _p(parts))
    return total, parts[0], parts[1], dl


def train_step(s: OSplats, m: OSplats, v: OSplats, acc, cams: list, targets, tl: Tiling, mode: int, lrs, t: int,
               sfx="f32", want_images=False, ssim_lambda=0.0, grads_out=None):
    """One iteration in place; grads_out (float32 array of 59 * n, nullable)
    receives the iteration's gradient rows (pos 3n, rot 4n, scale 3n, opacity
    n, sh_dc 3n, sh_rest 45n)."""
    V = len(cams)
    arr = (Camera * V)(*cams)
    g = AdamGroups()
    for i, x in enumerate(lrs):
        g.lr[i] = x
    g.beta1, g.beta2, g.eps = 0.9, 0.999, 1e-15
    imgs = np.zeros(V * tl.width * tl.height * 4, np.float32) if want_images else None
    t3 = np.ascontiguousarray(targets, np.float32)
    loss = getattr(lib(), f"oracle_train_step_{sfx}")(C.byref(s.h), C.byref(m.h), C.byref(v.h), _p(acc), V, arr,
                                                      _p(t3), C.byref(tl), int(mode), C.byref(g), int(t), _p(imgs),
                                                      float(ssim_lambda), _p(grads_out))
    return loss, imgs


def set_threads(n: int):
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return lib().oracle_max_threads()
