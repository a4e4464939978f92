"""ctypes binding of libsplatcuda.so (include/splat_cuda.h).

The library is loaded from nanotracer_b200/lib/libsplatcuda.so (built in-tree by
nanotracer_b200/build.py).  There is no CPU fallback: importing the compute API
without the library raises, and every call whose status is not SC_OK raises
SplatCudaError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libsplatcuda.so"

SC_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "capacity exceeded", 4: "CUDA error",
          5: "device wait timed out", 6: "non-finite values", 7: "I/O error", 8: "format error"}
SC_SPLATS_BF16_REST = 1
SC_MOMENTS_BF16 = 1
SC_BWD_REF = 0
SC_BWD_EXACT = 1
SC_KEYS_REF32 = 0
SC_KEYS_NATIVE64 = 1
SC_BWD_FLAG_COMPENSATED = 1


class SplatCudaError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


class sc_host_splats(C.Structure):
    _fields_ = [("n", C.c_uint32), ("positions", C.c_void_p), ("rotations", C.c_void_p), ("scales", C.c_void_p),
                ("opacities", C.c_void_p), ("sh_dc", C.c_void_p), ("sh_rest", C.c_void_p)]


class sc_camera(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("cam_pos", C.c_float * 3), ("near_plane", C.c_float),
                ("focal", C.c_float), ("width", C.c_float), ("height", C.c_float), ("n_splats", C.c_uint32)]


class sc_tiling(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("tile_w", C.c_uint32), ("tile_h", C.c_uint32),
                ("depth_max", C.c_float)]


class sc_adam_config(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class sc_adam_groups(C.Structure):
    _fields_ = [("lr", C.c_float * 6), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class sc_train_config(C.Structure):
    _fields_ = [("n_views", C.c_uint32), ("tiling", sc_tiling), ("adam", sc_adam_groups), ("bwd_mode", C.c_uint32),
                ("use_graph", C.c_uint32), ("blend_batch", C.c_uint32), ("sort_mode", C.c_uint32),
                ("tile_cull", C.c_uint32),
                ("log_scale_min", C.c_float), ("log_scale_max", C.c_float), ("opacity_logit_max", C.c_float),
                ("ssim_lambda", C.c_float), ("fp64_det", C.c_uint32), ("compensated_sums", C.c_uint32),
                ("sort_digit_bits", C.c_uint32)]


class sc_scenes_config(C.Structure):
    _fields_ = [("n_scenes", C.c_uint32), ("tiling", sc_tiling), ("adam", sc_adam_groups), ("use_graph", C.c_uint32),
                ("tile_cull", C.c_uint32), ("log_scale_min", C.c_float), ("log_scale_max", C.c_float),
                ("opacity_logit_max", C.c_float), ("fp64_det", C.c_uint32), ("compensated_sums", C.c_uint32)]


assert C.sizeof(sc_camera) == 96

P = C.c_void_p
U32 = C.c_uint32
U64 = C.c_uint64
F32 = C.c_float
I32 = C.c_int
ST = C.c_int

# name -> (restype, argtypes)
_PROTOS = {
    "sc_status_string": (C.c_char_p, [ST]),
    "sc_abi_version": (I32, []),
    "sc_ctx_create": (ST, [I32, C.POINTER(P)]),
    "sc_ctx_destroy": (None, [P]),
    "sc_last_error": (C.c_char_p, [P]),
    "sc_ctx_synchronize": (ST, [P]),
    "sc_ctx_stream": (P, [P]),
    "sc_ctx_set_stream": (ST, [P, P]),
    "sc_ctx_device_info": (ST, [P, C.POINTER(I32), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "sc_ctx_launch_count": (U64, [P]),
    "sc_ctx_set_fp64_det": (ST, [P, I32]),
    "sc_buffer_alloc": (ST, [P, C.c_size_t, C.POINTER(P)]),
    "sc_buffer_free": (ST, [P, P]),
    "sc_buffer_upload": (ST, [P, P, P, C.c_size_t]),
    "sc_buffer_readback": (ST, [P, P, P, C.c_size_t]),
    "sc_buffer_zero": (ST, [P, P, C.c_size_t]),
    "sc_buffer_copy": (ST, [P, P, P, C.c_size_t]),
    "sc_splats_upload": (ST, [P, C.POINTER(sc_host_splats), U32, U32, C.POINTER(P)]),
    "sc_splats_sync_from": (ST, [P, P, C.POINTER(sc_host_splats)]),
    "sc_splats_readback": (ST, [P, P, C.POINTER(sc_host_splats)]),
    "sc_splats_count": (U32, [P]),
    "sc_splats_capacity": (U32, [P]),
    "sc_splats_free": (None, [P, P]),
    "sc_grads_create": (ST, [P, U32, C.POINTER(P)]),
    "sc_grads_zero": (ST, [P, P, U32]),
    "sc_grads_upload": (ST, [P, P, C.POINTER(sc_host_splats)]),
    "sc_grads_readback": (ST, [P, P, U32, C.POINTER(sc_host_splats)]),
    "sc_grads_free": (None, [P, P]),
    "sc_moments_create": (ST, [P, U32, U32, C.POINTER(P)]),
    "sc_moments_upload": (ST, [P, P, C.POINTER(sc_host_splats), C.POINTER(sc_host_splats)]),
    "sc_moments_readback": (ST, [P, P, U32, C.POINTER(sc_host_splats), C.POINTER(sc_host_splats)]),
    "sc_moments_free": (None, [P, P]),
    "sc_camera_from_pose": (None, [P, P, P, F32, U32, U32, U32, C.POINTER(sc_camera)]),
    "sc_project": (ST, [P, P, P, U32, P]),
    "sc_bins_create": (ST, [P, C.POINTER(P)]),
    "sc_bins_free": (None, [P, P]),
    "sc_bin": (ST, [P, P, U32, U32, U32, C.POINTER(sc_tiling), I32, P]),
    "sc_bins_info": (ST, [P, C.POINTER(U64), C.POINTER(U32), C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "sc_radix_sort_u32": (ST, [P, P, P, P, P, U64, U32]),
    "sc_radix_sort_u64": (ST, [P, P, P, P, P, U64, U32]),
    "sc_exclusive_scan_u32": (ST, [P, P, U64, P]),
    "sc_exclusive_scan_u32_noalloc": (ST, [P, P, U64, P]),
    "sc_composite": (ST, [P, P, U32, U32, P, C.POINTER(sc_tiling), P, P]),
    "sc_mse_loss_grad": (ST, [P, P, P, U32, C.POINTER(sc_tiling), F32, P, P]),
    "sc_ssim_loss_grad": (ST, [P, P, P, U32, C.POINTER(sc_tiling), F32, P, P]),
    "sc_combined_loss_grad": (ST, [P, P, P, U32, C.POINTER(sc_tiling), F32, F32, P, P]),
    "sc_composite_backward": (ST, [P, P, U32, U32, P, C.POINTER(sc_tiling), P, P, I32, P, P]),
    "sc_composite_backward_ex": (ST, [P, P, U32, U32, P, C.POINTER(sc_tiling), P, P, I32, P, P, U32]),
    "sc_project_backward": (ST, [P, P, P, P, P, I32]),
    "sc_tonemap": (ST, [P, P, U32, U32, P]),
    "sc_adam_step": (ST, [P, P, P, P, P, U64, F32, U64, C.POINTER(sc_adam_config)]),
    "sc_adam_step_all": (ST, [P, P, P, P, U64, C.POINTER(sc_adam_groups)]),
    "sc_apply_constraints": (ST, [P, P, F32, F32, F32]),
    "sc_accumulate_grad": (ST, [P, P, P, U32]),
    "sc_prune_low_opacity": (ST, [P, P, P, P, F32, C.POINTER(U32)]),
    "sc_densify": (ST, [P, P, P, P, U32, F32, F32, U32, U32, C.POINTER(U32)]),
    "sc_write_ply": (ST, [C.c_char_p, C.POINTER(sc_host_splats)]),
    "sc_read_ply": (ST, [C.c_char_p, C.POINTER(sc_host_splats), C.POINTER(U32)]),
    "sc_trainer_create": (ST, [P, C.POINTER(sc_train_config), C.POINTER(P)]),
    "sc_trainer_free": (None, [P, P]),
    "sc_trainer_set_targets": (ST, [P, P]),
    "sc_trainer_set_host_targets": (ST, [P, P]),
    "sc_trainer_step": (ST, [P, P, P, P, P, U64, C.POINTER(C.c_double)]),
    "sc_trainer_images": (ST, [P, C.POINTER(P)]),
    "sc_trainer_stats": (ST, [P, C.POINTER(U64), C.POINTER(U32), P, P, C.POINTER(U64)]),
    "sc_trainer_set_profiling": (ST, [P, I32]),
    "sc_trainer_blend_work": (ST, [P, C.POINTER(U64)]),
    "sc_trainer_blend_pairs": (ST, [P, C.POINTER(U64)]),
    "sc_selftest_wait_timeout": (ST, [P]),
    "sc_scenes_trainer_create": (ST, [P, C.POINTER(sc_scenes_config), C.POINTER(P)]),
    "sc_scenes_trainer_free": (None, [P, P]),
    "sc_scenes_trainer_set_scene": (ST, [P, U32, P, P, P, U32, U32, P]),
    "sc_scenes_trainer_step": (ST, [P, P, U64, C.POINTER(C.c_double)]),
    "sc_scenes_trainer_images": (ST, [P, C.POINTER(P)]),
    "sc_scenes_trainer_stats": (ST, [P, C.POINTER(U64), C.POINTER(U32), C.POINTER(U64)]),
    "sc_trainer_step_grads": (ST, [P, P, P, F32, U32, U32, P, C.POINTER(C.c_double)]),
    "sc_adam_step_shard": (ST, [P, P, P, P, P, U32, U32, U32, U64, C.POINTER(sc_adam_groups), F32, F32, F32]),
    "sc_splats_pack_range": (ST, [P, P, U32, U32, U32, P]),
    "sc_splats_unpack_shards": (ST, [P, P, P, U32, U32]),
    "sc_moments_pack_range": (ST, [P, P, U32, U32, U32, P]),
    "sc_moments_unpack_shards": (ST, [P, P, U32, P, U32, U32]),
}

_lib = None


def lib():
    """Load libsplatcuda.so once.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        path = os.environ.get("SPLATCUDA_LIB", str(LIB_PATH))
        if not Path(path).exists():
            raise ImportError(f"libsplatcuda.so not found at {path}; build it with `python -m nanotracer_b200.build`")
        L = C.CDLL(path)
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_PROTOS)


def check(status: int, ctx=None) -> None:
    if status != SC_OK:
        msg = ""
        if ctx is not None:
            raw = lib().sc_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise SplatCudaError(status, msg)


def ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the library must be C-contiguous"
    return C.c_void_p(a.ctypes.data)
