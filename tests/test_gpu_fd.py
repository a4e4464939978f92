"""The device adjoint against FP64 central differences (the uneven-batch
workload's adjoint check): 64 random parameters of a 1000-splat 64x64 scene, h = 1e-3, the
gradient from the CUDA kernels (exact backward), the difference quotients
from the oracle's FP64 loss (tests/fd64.py states the bounds and the counted
exceptions)."""
import numpy as np
import pytest

from nanotracer_b200 import CameraUniform, GradSplatBuffers, TilingParams
from nanotracer_b200._lib import SC_BWD_EXACT, SC_KEYS_NATIVE64
from nanotracer_b200.scene import FOV_Y, orbit_pose

from tests.fd64 import H, N_SPLATS, TILE, W, Scene64, compare
from tests.util import GpuPipe

pytestmark = pytest.mark.gpu


def test_device_adjoint_matches_fp64_central_differences(ctx, oracle):
    s = Scene64(oracle)
    adj64, rec = s.adjoint_f64()
    params = s.draw(adj64)
    cam = CameraUniform.from_pose(*orbit_pose(0.0), FOV_Y, W, H, N_SPLATS)
    assert bytes(cam.c) == bytes(s.cam)
    pipe = GpuPipe(ctx, s.scene, cam, TilingParams(W, H, TILE, 8.0), key_mode=SC_KEYS_NATIVE64)
    pipe.project()
    pipe.bin()
    img, _ = pipe.composite()
    _, dl = oracle.mse(img[0], s.target)
    pipe.backward(dl.reshape(-1, 4), SC_BWD_EXACT)
    grads = GradSplatBuffers(ctx, N_SPLATS)
    pipe.r.project_backward(pipe.g, pipe.pg, cam, grads)
    dev = grads.readback(N_SPLATS).flat()
    rows, summary = compare(s, dev, params, rec)
    # the device adjoint and the FP64 adjoint agree on every drawn parameter without a stated exception
    for r in (r for r in rows if r["cause"] is None):
        a64 = float(adj64[r["splat"], r["param"]])
        assert abs(r["adjoint"] - a64) <= 1e-3 * abs(a64) + 1e-9, (r, a64)
    print(summary)
