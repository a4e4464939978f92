"""Parity with the oracle at the benchmark configurations' full sizes
(tests/parity.py states the checks and their tolerances).

  1M at 1080p: the benchmark's scene (1M splats, 1920x1080, 16x16
    tiles) seen from the first of its 8 orbit views (about 1.8e7 (tile, splat)
    pairs), one iteration stage by stage and through the captured step;
  200k at 1024x1024: 200k splats at 1024x1024, the same for its first iteration, then
    3 iterations of its orbit (3 degrees per iteration) against the oracle's.

The oracle runs on all host cores (its float atomics then vary the gradient
summation order between runs, which the bounds cover)."""
import numpy as np
import pytest

from nanotracer_b200 import AdamMomentBuffers, CameraUniform, GpuSplatBuffer, TilingParams, TrainConfig, Trainer
from nanotracer_b200._lib import SC_BWD_EXACT, SC_KEYS_REF32
from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
from nanotracer_b200.train import BENCH_LRS, render_targets

from tests.parity import iteration_parity
from tests.util import GpuPipe, check_image_explained, margins

pytestmark = pytest.mark.gpu

CONFIGS = {
    # name: (splats, width, height, orbit views, seed)
    "1M_1080p_view0": (1_000_000, 1920, 1080, 8, 5),
    "200k_1024_step0": (200_000, 1024, 1024, 1, 2),
}


@pytest.fixture
def all_cores(oracle):
    oracle.set_threads(oracle.max_threads())
    yield oracle
    oracle.set_threads(1)


@pytest.mark.parametrize("name", list(CONFIGS))
def test_full_size_iteration_parity(ctx, all_cores, name):
    n, W, H, n_orbit, seed = CONFIGS[name]
    scene = random_scene(n, seed)
    cam = CameraUniform.from_pose(*orbit_views(n_orbit, 0)[0], FOV_Y, W, H, n)
    report = iteration_parity(ctx, all_cores, scene, [cam], TilingParams(W, H, 16, 8.0), SC_BWD_EXACT, name)
    print(report)


def test_200k_orbit_iterations_track_the_oracle(ctx, all_cores):
    """The 200k-splat run (200k splats, 1024x1024, the camera advancing 3 degrees
    per iteration), 3 iterations from the same start: each iteration's loss
    within 1e-4 relative of the oracle's f32 iteration, and the trained
    parameters rendered by both within 1e-4 on all but near-threshold pixels
    (0.1 % at most)."""
    oracle = all_cores
    n, W, H = 200_000, 1024, 1024
    scene = random_scene(n, 2)
    tl = TilingParams(W, H, 16, 8.0)
    otl = oracle.tiling(W, H, 16, 16, 8.0)
    g = GpuSplatBuffer.upload(ctx, scene)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, TrainConfig(n_views=1, width=W, height=H, depth_max=8.0))
    target_scene = perturbed(scene)
    os_ = oracle.OSplats.from_buffer(scene)
    om, ov = oracle.OSplats.zeros(n), oracle.OSplats.zeros(n)
    oacc = np.zeros(n, np.float32)
    losses = []
    for t in range(1, 4):
        cam = CameraUniform.from_pose(*orbit_views(1, t - 1, jitter_deg=0.0)[0], FOV_Y, W, H, n)
        tgt = render_targets(ctx, target_scene, [cam], tl)
        tr.set_targets(ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32)))
        gl = tr.step(g, mo, acc, [cam], t)
        ol, _ = oracle.train_step(os_, om, ov, oacc, [oracle.camera_from_struct(bytes(cam.c))], tgt, otl, 1,
                                  BENCH_LRS, t)
        losses.append((gl, ol))
        assert abs(gl - ol) <= 1e-4 * ol, (t, gl, ol)
    # the trained parameters rendered by both, on the GPU's records and bins
    pipe = GpuPipe(ctx, g.readback(), cam, tl, key_mode=SC_KEYS_REF32)
    grec = pipe.project()[0]
    _, gpay, granges = pipe.bin()
    gimg, _ = pipe.composite()
    oimg, _, _ = oracle.composite(grec, gpay, granges.reshape(-1), otl)
    margin, _, _ = margins(oracle, grec, gpay, granges, otl, 1)
    s = check_image_explained(gimg[0], oimg, margin, label="200k after 3 iterations")
    print({"losses": losses, "image": s})
