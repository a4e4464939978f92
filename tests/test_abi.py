"""The C ABI without a GPU: the library loads, exports every function that
include/splat_cuda.h declares, and its host-side code (PLY I/O, camera
builder, status strings) matches the reference's behaviour."""
import ctypes as C
import json
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "splat_cuda.h"
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(sc_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from nanotracer_b200._lib import LIB_PATH, exported_symbols, lib
    L = lib()
    names = declared_functions()
    assert len(names) >= 50
    for n in names:
        assert hasattr(L, n), f"{n} declared in splat_cuda.h but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # every declared function has a ctypes prototype
    assert set(names) <= set(exported_symbols()), set(names) - set(exported_symbols())


def test_build_targets_sm100a_only():
    from nanotracer_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_status_strings_and_abi_version():
    from nanotracer_b200._lib import lib
    L = lib()
    assert L.sc_abi_version() == 1
    assert L.sc_status_string(0) == b"ok"
    assert L.sc_status_string(3) == b"capacity exceeded"


def test_camera_from_pose_matches_oracle_bitwise(oracle):
    """CameraUniform::from_pose (raster.rs:79-99): the library's host builder and
    the oracle's restatement of the RH look-at agree bit for bit."""
    from nanotracer_b200.raster import CameraUniform
    rng = np.random.default_rng(2)
    for _ in range(50):
        eye = rng.normal(size=3) * 4
        tgt = rng.normal(size=3)
        up = (0.0, 1.0, 0.0)
        fov = float(rng.uniform(0.3, 2.0))
        a = CameraUniform.from_pose(eye, tgt, up, fov, 1920, 1080, 7)
        b = oracle.camera(tuple(map(float, eye)), tuple(map(float, tgt)), up, fov, 1920, 1080, 7)
        assert bytes(a.c) == bytes(b)


def test_camera_standard_pose_kat():
    from nanotracer_b200.raster import CameraUniform
    c = CameraUniform.from_pose((0, 0, 0), (0, 0, -1), (0, 1, 0), math.pi / 2, 256, 256, 1)
    assert abs(c.focal - 128.0) < 1e-4
    v = c.view
    assert np.allclose(v, np.eye(4), atol=1e-7)


def test_ply_roundtrip_through_library(tmp_path):
    """ply.rs:262-287 through sc_write_ply / sc_read_ply."""
    from nanotracer_b200 import SplatBuffer, read_ply, write_ply
    g = KATS["ply_write_then_read_roundtrip"]["gaussian"]
    s = SplatBuffer([g["pos"]], [g["rotation"]], [g["scale"]], [g["opacity"]], [g["sh_dc"]],
                    [np.arange(45, dtype=np.float32) * np.float32(0.1)])
    p = tmp_path / "a.ply"
    write_ply(p, s)
    back = read_ply(p)
    assert len(back) == 1
    assert np.array_equal(back.flat(), s.flat())


def test_ply_library_and_oracle_files_identical(oracle, tmp_path):
    from nanotracer_b200 import write_ply
    from nanotracer_b200.scene import random_scene
    s = random_scene(333, seed=9)
    a, b = tmp_path / "lib.ply", tmp_path / "oracle.ply"
    write_ply(a, s)
    assert oracle.write_ply(b, oracle.OSplats.from_buffer(s)) == 0
    assert a.read_bytes() == b.read_bytes()
    assert a.stat().st_size == len(a.read_bytes()) and a.read_bytes().count(b"end_header\n") == 1


def test_ply_reader_by_name_missing_fields_and_errors(tmp_path):
    """read_ply matches properties by name (ply.rs:151-256): reordered fields,
    missing normals / f_rest read as absent / zero, missing required fields,
    ascii format and non-float properties are errors."""
    from nanotracer_b200 import read_ply
    from nanotracer_b200._lib import SplatCudaError
    props = ["rot_3", "rot_2", "rot_1", "rot_0", "opacity", "scale_2", "scale_1", "scale_0", "f_dc_2", "f_dc_1",
             "f_dc_0", "z", "y", "x", "f_rest_3"]
    vals = np.arange(len(props), dtype=np.float32) + 1
    hdr = "ply\nformat binary_little_endian 1.0\ncomment test\nelement vertex 1\n" + \
          "".join(f"property float {p}\n" for p in props) + "end_header\n"
    p = tmp_path / "r.ply"
    p.write_bytes(hdr.encode() + vals.tobytes())
    s = read_ply(p)
    d = dict(zip(props, vals))
    assert list(s.positions[0]) == [d["x"], d["y"], d["z"]]
    assert list(s.rotations[0]) == [d["rot_0"], d["rot_1"], d["rot_2"], d["rot_3"]]
    assert s.sh_rest[0, 3] == d["f_rest_3"] and s.sh_rest[0, 0] == 0.0
    # missing required property
    p2 = tmp_path / "m.ply"
    p2.write_bytes(hdr.replace("property float opacity\n", "").encode() + vals[:-1].tobytes())
    with pytest.raises(SplatCudaError):
        read_ply(p2)
    # ascii and non-float properties
    p3 = tmp_path / "a.ply"
    p3.write_bytes(hdr.replace("binary_little_endian", "ascii").encode())
    with pytest.raises(SplatCudaError):
        read_ply(p3)
    p4 = tmp_path / "u.ply"
    p4.write_bytes(hdr.replace("property float x", "property uchar x").encode())
    with pytest.raises(SplatCudaError):
        read_ply(p4)
    # empty file list
    p5 = tmp_path / "e.ply"
    p5.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 0\n" +
                   "".join(f"property float {q}\n" for q in props).encode() + b"end_header\n")
    assert len(read_ply(p5)) == 0


def test_splat_buffer_swap_remove_kat():
    """splat_store.rs:157-176."""
    from nanotracer_b200 import SplatBuffer
    b = SplatBuffer()
    for i in range(5):
        b.push_splat([i, i, i], [1, 0, 0, 0], [-1, -1, -1], 1.0, [0.1, 0.2, 0.3], np.zeros(45))
    b.swap_remove(1)
    assert len(b) == 4 and b.sh_rest.size == 4 * 45
    assert list(b.positions[1]) == [4.0, 4.0, 4.0]


def test_gaussians_roundtrip():
    """splat_store.rs:139-155."""
    from nanotracer_b200 import Gaussian, SplatBuffer
    g = Gaussian(np.array([1, 2, 3], np.float32), np.array([0, 1, 0], np.float32), np.array([0.1, 0.2, 0.3], np.float32),
                 np.zeros(45, np.float32), 1.5, np.array([-2, -2, -3], np.float32), np.array([1, 0, 0, 0], np.float32))
    buf = SplatBuffer.from_gaussians([g])
    back = buf.to_gaussians()
    assert len(back) == 1 and np.array_equal(back[0].pos, g.pos) and back[0].opacity == g.opacity


def test_compute_calls_fail_loudly_without_a_device():
    """No CPU fallback: without a usable GPU, creating a context raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nanotracer_b200 import CudaCtx, SplatCudaError
    with pytest.raises(SplatCudaError):
        CudaCtx(0)


def test_integration_ffi_block_binds_every_declared_function():
    """The Rust extern block a maintainer would add names every
    function include/splat_cuda.h declares."""
    import re
    root = Path(__file__).resolve().parent.parent
    header = (root / "include" / "splat_cuda.h").read_text()
    ffi = (root / "INTEGRATION.md").read_text()
    declared = sorted(set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", header)))
    assert declared
    assert [f for f in declared if f"fn {f}(" not in ffi] == []
