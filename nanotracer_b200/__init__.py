"""nanotracer_b200 — B200-native (sm_100a) Gaussian-splat rasteriser and
optimiser step, a drop-in for ssoj13/nanotracer's nano-optimize hot path.

The compute lives in libsplatcuda.so (nanotracer_b200/csrc, C ABI in
include/splat_cuda.h); these modules mirror the reference's Rust API names
(CudaCtx ~ WgpuCtx, GpuSplatBuffer, Rasterizer, TileBinner, AdamGpu, train).
"""
from ._lib import SplatCudaError, lib  # noqa: F401
from .adam_gpu import AdamConfig, AdamGpu, densify, prune_low_opacity  # noqa: F401
from .gpu import CudaCtx, DeviceBuffer  # noqa: F401
from .ply import read_ply, write_ply  # noqa: F401
from .raster import PROJECTED_DTYPE, PROJECTED_GRAD_DTYPE, CameraUniform, Rasterizer  # noqa: F401
from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer, GradSplatBuffers  # noqa: F401
from .splat_store import Gaussian, SplatBuffer  # noqa: F401
from .tile_binner import PrefixScan, RadixSort, TileBinner, TilingParams  # noqa: F401
from .train import TrainConfig, Trainer, train  # noqa: F401
