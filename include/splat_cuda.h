/*
 * splat_cuda.h — C ABI of libsplatcuda.so, the sm_100a implementation of
 * nano-optimize's differentiable Gaussian-splat rasteriser and optimiser
 * step (ssoj13/nanotracer, crates/nano-optimize).
 *
 * Every entry point below names the reference interface it replaces
 * (file:line inside the reference project).  Conventions:
 *
 *   - Plain C types only: device memory is passed as `void*`/typed device
 *     pointers obtained from sc_buffer_alloc (or any cudaMalloc'd memory on
 *     the context's device), sizes are element counts, compound objects are
 *     opaque handles owned by the library.
 *   - Every call returns sc_status.  The reference panics or asserts where
 *     this ABI returns SC_ERR_INVALID_ARG / SC_ERR_CAPACITY; the one call that
 *     returned Result in the reference (WgpuCtx::new) maps to sc_ctx_create.
 *   - All calls are asynchronous on the context's stream except
 *     *_readback, sc_*_info, sc_ctx_synchronize and the PLY functions, which
 *     block — matching WgpuCtx::readback (gpu.rs:119-152).
 *   - A context is thread-compatible (one thread at a time), like one
 *     WgpuCtx per thread in the reference (docs/src/decisions.md:161-165).
 *   - Bounded device-side waits: kernels that spin on a flag (decoupled
 *     look-back) give up after a fixed iteration count and raise
 *     SC_ERR_TIMEOUT on the next status check instead of hanging.
 */
#ifndef SPLAT_CUDA_H
#define SPLAT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_ABI_VERSION 1

typedef enum sc_status {
  SC_OK = 0,
  SC_ERR_INVALID_ARG = 1,  /* a size, pointer or handle is invalid              */
  SC_ERR_OOM = 2,          /* device allocation failed                           */
  SC_ERR_CAPACITY = 3,     /* a device-side capacity overflowed (retry larger)   */
  SC_ERR_CUDA = 4,         /* a CUDA runtime error; sc_last_error() says which   */
  SC_ERR_TIMEOUT = 5,      /* a bounded device wait gave up                      */
  SC_ERR_NONFINITE = 6,    /* non-finite values where finite ones are required   */
  SC_ERR_IO = 7,           /* file could not be opened / read / written          */
  SC_ERR_FORMAT = 8        /* PLY header or record not understood                */
} sc_status;

typedef struct sc_ctx sc_ctx;          /* device + stream + scratch arena    */
typedef struct sc_splats sc_splats;    /* GpuSplatBuffer                     */
typedef struct sc_grads sc_grads;      /* GradSplatBuffers                   */
typedef struct sc_moments sc_moments;  /* AdamMomentBuffers                  */
typedef struct sc_bins sc_bins;        /* TileBinningResult                  */
typedef struct sc_trainer sc_trainer;  /* batched whole-iteration trainer    */

/* Host splat arrays, the flat layout of SplatBuffer (splat_store.rs:20-36):
 * positions n*3, rotations n*4 (w,x,y,z), scales n*3 (log sigma),
 * opacities n (logit), sh_dc n*3, sh_rest n*45 planar R[15] G[15] B[15].
 * The same struct carries gradients and Adam moments (AdamState slabs,
 * adam.rs:48-56, train.rs:84-89) in identical layout. */
typedef struct sc_host_splats {
  uint32_t n;
  float* positions;
  float* rotations;
  float* scales;
  float* opacities;
  float* sh_dc;
  float* sh_rest;
} sc_host_splats;

/* CameraUniform (raster.rs:60-77): 96 bytes, view is column-major. */
typedef struct sc_camera {
  float view[16];
  float cam_pos[3];
  float near_plane;
  float focal;
  float width;
  float height;
  uint32_t n_splats;
} sc_camera;

/* TilingParams (tile_binner.rs:21-42).  The reference's square tile_size is
 * tile_w == tile_h; non-square tiles (32x8) are an extension. */
typedef struct sc_tiling {
  uint32_t width;
  uint32_t height;
  uint32_t tile_w;
  uint32_t tile_h;
  float depth_max;
} sc_tiling;

/* ProjectedSplat (raster.rs:27-37), 48 bytes. */
typedef struct sc_projected_splat {
  float mean_xy[2];
  float depth;
  float radius;
  float conic[3];
  float visible;
  float color[3];
  float opacity;
} sc_projected_splat;

/* ProjectedGrad (raster.rs:46-55), 48 bytes. */
typedef struct sc_projected_grad {
  float dmean_opacity[4]; /* dmean.xy, dopacity, pad */
  float dconic[4];        /* a, b, c, pad            */
  float dcolor[4];        /* r, g, b, pad            */
} sc_projected_grad;

/* AdamConfig (adam.rs:22-39). */
typedef struct sc_adam_config {
  float lr;
  float beta1;
  float beta2;
  float eps;
} sc_adam_config;

/* Six learning-rate groups (pos, rot, scale, opacity, sh_dc, sh_rest).  The
 * reference's two groups (adam_gpu.rs:334-427: pos vs the rest) are
 * lr = {pos, attr, attr, attr, attr, attr}. */
typedef struct sc_adam_groups {
  float lr[6];
  float beta1;
  float beta2;
  float eps;
} sc_adam_groups;

/* Backward transmittance semantics.
 * SC_BWD_REF:   rasterize_backward.wgsl:73-210 — reverse walk over every
 *               entry of the tile from T = 1 - out.w, stopping at T > 1.0001.
 * SC_BWD_EXACT: reverse walk from each pixel's last contributor with the
 *               final transmittance recorded by the forward (aux buffer). */
typedef enum sc_bwd_mode { SC_BWD_REF = 0, SC_BWD_EXACT = 1 } sc_bwd_mode;

/* Key layouts for sc_bin.
 * SC_KEYS_REF32: (tile_id << 16) | u16(depth/depth_max * 65535), 32-bit keys,
 *                tile_emit.wgsl:54-61; at most 65536 tiles.
 * SC_KEYS_NATIVE64: (tile_id << 32) | float_bits(depth), 64-bit keys. */
typedef enum sc_key_mode { SC_KEYS_REF32 = 0, SC_KEYS_NATIVE64 = 1 } sc_key_mode;

#define SC_SPLATS_BF16_REST 1u   /* sh_rest stored as bf16 on the device    */
#define SC_MOMENTS_BF16 1u       /* Adam m and v stored as bf16             */

/* ------------------------------------------------------------------ runtime
 * replaces WgpuCtx (crates/nano-optimize/src/gpu.rs:21-153) */
const char* sc_status_string(sc_status s);
int sc_abi_version(void);
sc_status sc_ctx_create(int device, sc_ctx** out);                 /* WgpuCtx::new, gpu.rs:31-77 */
void sc_ctx_destroy(sc_ctx* ctx);
const char* sc_last_error(const sc_ctx* ctx);
sc_status sc_ctx_synchronize(sc_ctx* ctx);                         /* queue.poll(Wait), gpu.rs:140-146 */
void* sc_ctx_stream(sc_ctx* ctx);                                  /* the cudaStream_t calls run on */
sc_status sc_ctx_set_stream(sc_ctx* ctx, void* stream);
sc_status sc_ctx_device_info(sc_ctx* ctx, int* sm_count, size_t* free_bytes, size_t* total_bytes);
/* Number of kernels this context has launched so far (diagnostics / bench). */
uint64_t sc_ctx_launch_count(const sc_ctx* ctx);
sc_status sc_buffer_alloc(sc_ctx* ctx, size_t bytes, void** dptr);  /* storage_buffer_zeroed, gpu.rs:98-107 */
sc_status sc_buffer_free(sc_ctx* ctx, void* dptr);
sc_status sc_buffer_upload(sc_ctx* ctx, void* dst, const void* src, size_t bytes);   /* queue.write_buffer */
sc_status sc_buffer_readback(sc_ctx* ctx, void* dst, const void* src, size_t bytes); /* readback, gpu.rs:119-152 */
sc_status sc_buffer_zero(sc_ctx* ctx, void* dptr, size_t bytes);
/* device-to-device copy, asynchronous on the context's stream
 * (encoder.copy_buffer_to_buffer, as used by gpu.rs:119-152) */
sc_status sc_buffer_copy(sc_ctx* ctx, void* dst, const void* src, size_t bytes);

/* ------------------------------------------------------------- parameters
 * replaces GpuSplatBuffer / GradSplatBuffers / AdamMomentBuffers
 * (crates/nano-optimize/src/splat_gpu.rs:29-423) */
sc_status sc_splats_upload(sc_ctx* ctx, const sc_host_splats* src, uint32_t capacity, uint32_t flags,
                           sc_splats** out);                        /* GpuSplatBuffer::upload, splat_gpu.rs:94-120 */
sc_status sc_splats_sync_from(sc_ctx* ctx, sc_splats* dst, const sc_host_splats* src); /* sync_from, :126-152 */
sc_status sc_splats_readback(sc_ctx* ctx, const sc_splats* src, sc_host_splats* dst);  /* readback, :156-187 */
uint32_t sc_splats_count(const sc_splats* s);
uint32_t sc_splats_capacity(const sc_splats* s);
void sc_splats_free(sc_ctx* ctx, sc_splats* s);

sc_status sc_grads_create(sc_ctx* ctx, uint32_t capacity, sc_grads** out);  /* GradSplatBuffers::new, :36-57 */
sc_status sc_grads_zero(sc_ctx* ctx, sc_grads* g, uint32_t n);               /* GradSplatBuffers::zero, :62-75 */
sc_status sc_grads_upload(sc_ctx* ctx, sc_grads* g, const sc_host_splats* src);
sc_status sc_grads_readback(sc_ctx* ctx, const sc_grads* g, uint32_t n, sc_host_splats* dst);
void sc_grads_free(sc_ctx* ctx, sc_grads* g);

sc_status sc_moments_create(sc_ctx* ctx, uint32_t capacity, uint32_t flags, sc_moments** out); /* :202-240 */
sc_status sc_moments_upload(sc_ctx* ctx, sc_moments* mo, const sc_host_splats* m, const sc_host_splats* v); /* :246-300 */
sc_status sc_moments_readback(sc_ctx* ctx, const sc_moments* mo, uint32_t n, sc_host_splats* m,
                              sc_host_splats* v);                             /* download_to_cpu */
void sc_moments_free(sc_ctx* ctx, sc_moments* mo);

/* ------------------------------------------------------------- rasteriser
 * replaces Rasterizer (crates/nano-optimize/src/raster.rs:103-804) */
void sc_camera_from_pose(const float eye[3], const float target[3], const float up[3], float fov_y,
                         uint32_t width, uint32_t height, uint32_t n_splats,
                         sc_camera* out);                            /* CameraUniform::from_pose, raster.rs:79-99 */

/* project_gaussians.wgsl:156-259 for n_views cameras: projected holds
 * n_views * sc_splats_capacity() records, view-major.  The reference forms
 * det = s00 s11 - s01^2 in f32 and culls det <= 0 (:226-234); with
 * sc_ctx_set_fp64_det a near-degenerate splat (det < 2^-6 s00 s11 in f32)
 * gets its determinant and conic in FP64 instead. */
sc_status sc_project(sc_ctx* ctx, const sc_splats* s, const sc_camera* cams, uint32_t n_views,
                     sc_projected_splat* projected);                 /* Rasterizer::project, raster.rs:731-794 */

/* ----------------------------------------------------------- tile binner
 * replaces TileBinner / RadixSort / PrefixScan
 * (tile_binner.rs:21-416, radix_sort.rs:32-303, prefix_scan.rs:18-258) */
sc_status sc_bins_create(sc_ctx* ctx, sc_bins** out);
void sc_bins_free(sc_ctx* ctx, sc_bins* b);
/* Bins n_views * n_splats projected records (view-major, stride = stride_splats
 * records per view).  Tiles of view v are numbered v*num_tiles + tile.
 * Blocks once to read the pair count (tile_binner.rs:243-245 does the same). */
sc_status sc_bin(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t n_splats, uint32_t stride_splats,
                 uint32_t n_views, const sc_tiling* tiling, sc_key_mode mode, sc_bins* bins); /* TileBinner::bin */
/* total pairs, number of tiles (all views) and the device arrays of the last sc_bin:
 * sorted keys (uint32 for REF32, uint64 for NATIVE64), payloads (uint32 splat
 * index), tile ranges (2 x uint32 per tile, [begin, end), empty = (0,0)). */
sc_status sc_bins_info(const sc_bins* b, uint64_t* total_pairs, uint32_t* num_tiles, const void** sorted_keys,
                       const uint32_t** sorted_payloads, const uint32_t** tile_ranges);

/* Stable LSD radix sort (onesweep, decoupled look-back) of n (key, value)
 * pairs in place; keys_tmp / vals_tmp are ping-pong buffers of the same size.
 * key_bits: the pairs are ordered by the low key_bits bits of the key; any
 * higher bits travel with the key and keep their input order within equal
 * low bits (so key_bits = the width of the keys sorts them fully).  RadixSort::sort,
 * radix_sort.rs:144-303 (32 one-bit passes there; 8-bit digits here). */
sc_status sc_radix_sort_u32(sc_ctx* ctx, uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                            uint64_t n, uint32_t key_bits);
sc_status sc_radix_sort_u64(sc_ctx* ctx, uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                            uint64_t n, uint32_t key_bits);
/* Exclusive prefix sum of n uint32 in place (single pass, decoupled look-back);
 * total (device pointer, may be NULL) receives the sum.  PrefixScan::scan,
 * prefix_scan.rs:127-186 (limited to 2^24 elements there). */
sc_status sc_exclusive_scan_u32(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* total);
/* The same scan for callers that cannot allocate device memory: a host engine
 * that owns every device allocation through its own pool and forbids hidden
 * library allocations, or code on a latency-critical path where cudaMalloc's
 * implicit device synchronisation is not acceptable.  No counterpart in the
 * reference (its PrefixScan allocates its block sums per call,
 * prefix_scan.rs:127-186).
 * Its look-back scratch is a fixed file-scope device array of 128 KiB + 256 B
 * that every GPU loading the library holds until the process exits; n above
 * SC_NOALLOC_SCAN_MAX_N returns SC_ERR_INVALID_ARG without touching data.
 * The first call on a device looks the array's device address up (no
 * allocation) and keeps it until the process exits; make that first call
 * before any stream capture, and do not use the library on a device after a
 * cudaDeviceReset of it (the kept address would be stale).  All calls
 * share the array, which keeps the last call's contents (each call clears the
 * part it uses), so calls that overlap on the GPU — on different streams or
 * contexts of the same device — race and must be serialised by the caller.
 * It calls no cudaMalloc, cudaFree or allocating library routine. */
#define SC_NOALLOC_SCAN_MAX_N (1ull << 26)
sc_status sc_exclusive_scan_u32_noalloc(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* total);

/* rasterize.wgsl:48-118 over n_views views; image is n_views*W*H float4
 * (rgb, 1-T).  aux (nullable) receives per pixel {T_final bits, last
 * contributor count} for SC_BWD_EXACT. */
sc_status sc_composite(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t stride_splats, uint32_t n_views,
                       const sc_bins* bins, const sc_tiling* tiling, float* image,
                       uint32_t* aux);                               /* Rasterizer::composite, raster.rs:468-529 */

/* loss.rs:163-179 on the device: dl_dc = scale * 2 (p - t) / (3 W H) as float4,
 * loss_out (device double, nullable) receives per view the sum of (p-t)^2 over
 * pixels and channels (the loss is that sum / (3 W H)).
 * target is n_views*W*H float3. */
sc_status sc_mse_loss_grad(sc_ctx* ctx, const float* pred, const float* target, uint32_t n_views,
                           const sc_tiling* tiling, float scale, float* dl_dc, double* loss_out);

/* loss.rs:340-375 (ssim_loss_grad) on the device: dl_dc = scale * dL/dC of
 * L = 1 - mean SSIM over the pixels and the three channels (11-tap Gaussian
 * window, sigma 1.5, reflect-101 padding, C1 = 1e-4, C2 = 9e-4); loss_out
 * (device double per view, nullable) receives L.  Images of at least 6x6. */
sc_status sc_ssim_loss_grad(sc_ctx* ctx, const float* pred, const float* target, uint32_t n_views,
                            const sc_tiling* tiling, float scale, float* dl_dc, double* loss_out);

/* loss.rs:383-410 (combined_loss_grad): (1 - lambda) MSE + lambda (1 - SSIM),
 * lambda clamped to [0, 1]; lambda 0 is sc_mse_loss_grad exactly.  loss_out
 * (device double, nullable) receives per view {total, mse, ssim}. */
sc_status sc_combined_loss_grad(sc_ctx* ctx, const float* pred, const float* target, uint32_t n_views,
                                const sc_tiling* tiling, float lambda, float scale, float* dl_dc,
                                double* loss_out);

/* rasterize_backward.wgsl:73-210: accumulates into projected_grad, which the
 * caller zeroes first (raster.rs:647-651). */
sc_status sc_composite_backward(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t stride_splats,
                                uint32_t n_views, const sc_bins* bins, const sc_tiling* tiling,
                                const float* forward_out, const float* dl_dc, sc_bwd_mode mode,
                                const uint32_t* aux, sc_projected_grad* projected_grad); /* raster.rs:653-724 */

/* sc_composite_backward with options (flags):
 * SC_BWD_FLAG_COMPENSATED: the per-(view, splat) gradient totals across
 *   tiles are compensated sums.  The reference adds each (pixel, splat) term
 *   with a CAS float atomic in arrival order (rasterize_backward.wgsl:62-71,
 *   188-200), and plain float atomics here add one term per (tile, splat);
 *   with the flag every tile's term is added by an atomic that returns the
 *   old total, the exact rounding error of that addition (Knuth's TwoSum) is
 *   accumulated in a compensation record, and the two are added once at the
 *   end: the total is then within about one rounding of the exact sum of the
 *   tiles' terms, whatever their number and order.  Costs a second 48-byte
 *   record per (view, splat) (library scratch here) and 18 scalar atomics per
 *   (tile, splat) instead of 3 vector ones. */
#define SC_BWD_FLAG_COMPENSATED 1u
sc_status sc_composite_backward_ex(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t stride_splats,
                                   uint32_t n_views, const sc_bins* bins, const sc_tiling* tiling,
                                   const float* forward_out, const float* dl_dc, sc_bwd_mode mode,
                                   const uint32_t* aux, sc_projected_grad* projected_grad, uint32_t flags);

/* project_backward.wgsl:79-304 for one view; overwrites grads (accumulate = 0)
 * or adds into them (accumulate = 1, multi-view sums). */
sc_status sc_project_backward(sc_ctx* ctx, const sc_splats* s, const sc_projected_grad* projected_grad,
                              const sc_camera* cam, sc_grads* grads,
                              int accumulate);                       /* Rasterizer::project_backward, raster.rs:559-645 */

/* Precision option of sc_project and sc_project_backward (off by default,
 * which is the reference's f32 arithmetic): when enabled, a splat whose f32
 * 2x2 projected-covariance determinant keeps less than 2^-6 of s00 s11
 * (a needle-like splat, where cancellation has eaten the f32 determinant)
 * gets the determinant from Lagrange's identity det = |B0 x B1|^2 +
 * 0.3 (|B0|^2 + |B1|^2) + 0.09 (Sigma2D = B B^T + 0.3 I) and the inverse in
 * FP64; the adjoint recomputes the same FP64 conic.  No counterpart in the
 * reference (project_gaussians.wgsl:226-234, project_backward.wgsl:127-139). */
sc_status sc_ctx_set_fp64_det(sc_ctx* ctx, int enabled);

/* tonemap.wgsl:27-41 into a headless RGBA8 buffer (viewer path). */
sc_status sc_tonemap(sc_ctx* ctx, const float* image, uint32_t width, uint32_t height, uint8_t* rgba8);

/* ------------------------------------------------------------- optimiser
 * replaces AdamGpu (crates/nano-optimize/src/adam_gpu.rs:31-547) */
sc_status sc_adam_step(sc_ctx* ctx, float* params, const float* grads, float* m, float* v, uint64_t n,
                       float lr, uint64_t t, const sc_adam_config* cfg);   /* AdamGpu::step, :224-323 */
/* AdamGpu::step_all, :334-427.  With SC_SPLATS_BF16_REST storage the SH-rest
 * parameters are written back with stochastic rounding seeded by t (this call,
 * sc_adam_step_shard and sc_trainer_step alike), so updates smaller than half
 * a BF16 ulp survive in expectation; the same t gives the same bits. */
sc_status sc_adam_step_all(sc_ctx* ctx, sc_splats* s, const sc_grads* g, sc_moments* mo, uint64_t t,
                           const sc_adam_groups* groups);
sc_status sc_apply_constraints(sc_ctx* ctx, sc_splats* s, float log_scale_min, float log_scale_max,
                               float opacity_logit_max);                   /* :431-489 */
sc_status sc_accumulate_grad(sc_ctx* ctx, const sc_grads* g, float* grad_acc, uint32_t n); /* :492-541 */

/* ------------------------------------------------------- densify / prune
 * replaces train.rs:414-602 (CPU round trip there; stream compaction here).
 * The result order equals the reference's swap_remove order exactly. */
sc_status sc_prune_low_opacity(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* grad_acc, float threshold,
                               uint32_t* removed);                          /* prune_low_opacity, :572-602 */
sc_status sc_densify(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* grad_acc, uint32_t grad_count,
                     float grad_threshold, float split_log_scale_threshold, uint32_t max_splats, uint32_t iter,
                     uint32_t counts[3]);                                   /* densify, :414-549 */

/* ------------------------------------------------------------------ PLY
 * replaces nano-splat read_ply / write_ply (crates/nano-splat/src/ply.rs:17-256)
 * together with SplatBuffer::{from,to}_gaussians (splat_store.rs:60-94). */
sc_status sc_write_ply(const char* path, const sc_host_splats* s);
/* Reads the header; *n_out receives the vertex count.  When dst is non-NULL
 * and dst->n >= count, the records are decoded into dst and dst->n = count. */
sc_status sc_read_ply(const char* path, sc_host_splats* dst, uint32_t* n_out);

/* --------------------------------------------------------------- trainer
 * The batched whole iteration of train() (train.rs:155-250) for n_views
 * views per step: project -> bin -> composite + fused MSE -> backward ->
 * project backward summed over views -> accumulate -> Adam -> constraints,
 * replayed as one CUDA graph.  Loss is the mean of the per-view MSE. */
typedef struct sc_train_config {
  uint32_t n_views;            /* views per step                                 */
  sc_tiling tiling;            /* image size and tile shape                      */
  sc_adam_groups adam;         /* per-group learning rates                        */
  uint32_t bwd_mode;           /* sc_bwd_mode                                    */
  uint32_t use_graph;          /* capture the iteration as a CUDA graph          */
  uint32_t blend_batch;        /* blend batch depth: list positions the blend kernels stage per batch
                                  (a multiple of 32, capped at the tile's thread count); 0 = one per
                                  thread (tile pixels / 2 with two pixels per thread) */
  uint32_t sort_mode;          /* 0 = auto (two-level), 1 = depth presort + stable sort of the
                                  (tile, splat) pairs, 2 = depth presort + two-level binning
                                  (super tiles of 4x4 tiles, per-tile lists filled in depth order) */
  uint32_t tile_cull;          /* drop (tile, splat) pairs whose alpha stays below 1/255 over the
                                  whole tile (images unchanged: the blend skips those pairs) */
  float log_scale_min, log_scale_max, opacity_logit_max; /* train.rs:37-39 */
  float ssim_lambda;           /* loss = (1 - l) MSE + l (1 - SSIM), loss.rs:383-410 (TrainConfig::ssim_lambda,
                                  train.rs:52); 0 = MSE only, fused into the blend */
  uint32_t fp64_det;           /* FP64 determinant and inverse of near-degenerate splats in the projection
                                  and its adjoint (as sc_ctx_set_fp64_det) */
  uint32_t compensated_sums;   /* per-(view, splat) gradient totals across tiles as TwoSum-compensated
                                  atomic sums (as SC_BWD_FLAG_COMPENSATED) */
  uint32_t sort_digit_bits;    /* radix digit width of the binning sort (items or pairs): 8 or 9 bits per
                                  onesweep pass, 0 = fewer passes wins (radix_sort.rs:1-26 uses 1 bit) */
} sc_train_config;

sc_status sc_trainer_create(sc_ctx* ctx, const sc_train_config* cfg, sc_trainer** out);
void sc_trainer_free(sc_ctx* ctx, sc_trainer* tr);
/* targets: device array n_views*W*H float3 (rgb). */
sc_status sc_trainer_set_targets(sc_trainer* tr, const float* targets);
/* Targets in page-locked host memory (n_views*W*H float3): every step copies
 * them to a trainer-owned device buffer on a side stream, overlapped with the
 * projection, sorting and emission, and the blend waits for the copy (the
 * reference uploads its target before the iteration, train.rs:166-196).  The
 * caller may rewrite the host buffer between steps. */
sc_status sc_trainer_set_host_targets(sc_trainer* tr, const float* pinned_targets);
/* One training step with cameras cams[n_views] (host array); t is the new Adam
 * step count.  Blocks until the step has finished; loss_out (host, nullable)
 * receives the mean loss.  A step whose pair lists overflowed the device
 * capacity changes no parameter and is re-run with larger buffers. */
sc_status sc_trainer_step(sc_trainer* tr, sc_splats* s, sc_moments* mo, float* grad_acc, const sc_camera* cams,
                          uint64_t t, double* loss_out);
/* device array of the last step: images n_views*W*H float4 (rgb, 1-T) */
sc_status sc_trainer_images(const sc_trainer* tr, const float** images);
/* pairs: (tile, splat) pairs of the last step (all views); n_kernels: kernel
 * launches per step; names / avg_ms (arrays of SC_TRAINER_STAGES, nullable):
 * stage names and average device time per stage in ms over the steps since
 * profiling was enabled; items (nullable): two-level binning items of the last
 * step (0 on the pair-sort path). */
#define SC_TRAINER_STAGES 9
sc_status sc_trainer_stats(const sc_trainer* tr, uint64_t* pairs, uint32_t* n_kernels, const char** names,
                           float* avg_ms, uint64_t* items);
/* Record CUDA events between the stages of each step (also inside the graph)
 * and count the blends' work (sc_trainer_blend_work) when enabled is 1; 2
 * also counts contributing (pixel, entry) pairs (sc_trainer_blend_pairs),
 * which adds a few instructions per entry to the blends; 0 turns it off.
 * Each call resets the accumulated stage times and counters. */
sc_status sc_trainer_set_profiling(sc_trainer* tr, int enabled);
/* Blend work per step, averaged over the steps since profiling was enabled
 * (two-level binning only; zeros otherwise): out[0] list positions the
 * forward's batches covered, out[1] entries it blended, out[2], out[3] the
 * same for the backward.  No counterpart in the reference. */
sc_status sc_trainer_blend_work(const sc_trainer* tr, uint64_t out[4]);
/* Contributing (pixel, entry) pairs per step with profiling level 2, averaged
 * like sc_trainer_blend_work: out[0] pixels that took an entry's alpha in the
 * forward, out[1] the pixel-entry adjoints the backward formed.  With the
 * blends' warp instruction counts (from a profiler) they give the
 * instructions per pair.  No counterpart in the reference. */
sc_status sc_trainer_blend_pairs(const sc_trainer* tr, uint64_t out[2]);

/* ------------------------------------------------ many scenes in one launch per stage
 * No counterpart in the reference, which trains one scene per train() call
 * (train.rs:65-401).  n_scenes independent scenes, each with its own store,
 * Adam moments, densify statistic, camera, image size and target, step
 * together: every stage is one launch over all scenes (projection, depth sort,
 * two-level binning, blend forward and backward over one (scene, tile) grid,
 * projection backward, Adam), the whole step one CUDA graph.  Images of
 * different sizes share the tiling's tile grid (tiling.width x
 * tiling.height, the largest); a scene's pixels are those inside its own
 * width x height, and its loss is its own MSE (loss.rs:163-179).  Densify
 * and prune run per scene on its own store between steps (sc_densify,
 * sc_prune_low_opacity); a store whose capacity changes is set again. */
typedef struct sc_scenes_config {
  uint32_t n_scenes;           /* at most 64 */
  sc_tiling tiling;            /* the largest image and the tile shape */
  sc_adam_groups adam;
  uint32_t use_graph;
  uint32_t tile_cull;
  float log_scale_min, log_scale_max, opacity_logit_max;
  uint32_t fp64_det, compensated_sums;
} sc_scenes_config;
typedef struct sc_scenes_trainer sc_scenes_trainer;
sc_status sc_scenes_trainer_create(sc_ctx* ctx, const sc_scenes_config* cfg, sc_scenes_trainer** out);
void sc_scenes_trainer_free(sc_ctx* ctx, sc_scenes_trainer* st);
/* Scene i: its store, moments (capacity >= the store's), densify statistic
 * (device, one float per splat of capacity), image size (within the tiling)
 * and target (device, width * height float3, copied in by this call). */
sc_status sc_scenes_trainer_set_scene(sc_scenes_trainer* st, uint32_t i, sc_splats* s, sc_moments* mo,
                                      float* grad_acc, uint32_t width, uint32_t height, const float* target);
/* One step of every scene: cams[i] (host, its width/height = scene i's), the
 * shared Adam step count t; losses (host, nullable) receives each scene's
 * MSE.  Blocking, like sc_trainer_step. */
sc_status sc_scenes_trainer_step(sc_scenes_trainer* st, const sc_camera* cams, uint64_t t, double* losses);
/* device images of the last step: n_scenes x tiling.height x tiling.width float4 */
sc_status sc_scenes_trainer_images(const sc_scenes_trainer* st, const float** images);
sc_status sc_scenes_trainer_stats(const sc_scenes_trainer* st, uint64_t* pairs, uint32_t* n_kernels,
                                  uint64_t* items);

/* Failure-detection self-test (no counterpart in the reference): runs one
 * radix-sort pass whose look-back waits on a tile that is never processed.
 * The bounded wait gives up (about a second), the kernel ends, and the call
 * returns SC_ERR_TIMEOUT; the context stays usable.  Any other status means
 * the timeout path is broken. */
sc_status sc_selftest_wait_timeout(sc_ctx* ctx);

/* ------------------------------------------------ data-parallel views
 * No counterpart in the reference, which trains on one device (train.rs:155-250
 * renders the iteration's views one after another).  One iteration is split
 * across R ranks by views, ZeRO-1 style:
 *   1. every rank: sc_trainer_step_grads over its own views -> per-splat
 *      gradient summed over those views, written shard-major;
 *   2. the caller reduce-scatters that buffer (R chunks) over its communicator;
 *   3. every rank: sc_adam_step_shard on its chunk of splats [lo, lo+count);
 *   4. sc_splats_pack_range of that chunk, all-gather, sc_splats_unpack_shards.
 * Shard-major layout with chunks of `shard` splats: element (row r, splat i)
 * is at ((i / shard) * 59 + r) * shard + i % shard; rows 0-58 are the
 * parameter rows of sc_host_splats in slab order (pos 3, rot 4, log-scale 3,
 * opacity logit 1, sh_dc 3, sh_rest 45 planar). */
#define SC_PARAM_ROWS 59

/* Steps 1: the trainer's views rendered, dL/dC scaled by loss_weight (the
 * single-device step uses 1/n_views; a split iteration of V views in total
 * uses 1/V on every rank), and the per-splat gradient summed over the views
 * written to grads (n_shards * 59 * shard floats, n_shards * shard >= n;
 * rows of padding splats are zero).  loss_out = loss_weight * sum of the
 * views' MSE.  Parameters, moments and the densify statistic are untouched.
 * Blocking, like sc_trainer_step. */
sc_status sc_trainer_step_grads(sc_trainer* tr, sc_splats* s, const sc_camera* cams, float loss_weight,
                                uint32_t n_shards, uint32_t shard, float* grads, double* loss_out);
/* Step 3: Adam (shared t), densify statistic and constraints for splats
 * [lo, lo+count) from the reduced chunk shard_grads[r * shard + j]. */
sc_status sc_adam_step_shard(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* grad_acc, const float* shard_grads,
                             uint32_t lo, uint32_t count, uint32_t shard, uint64_t t, const sc_adam_groups* groups,
                             float log_scale_min, float log_scale_max, float opacity_logit_max);
/* Step 4: parameters of [lo, lo+count) as f32 rows out[r * shard + j], and the
 * inverse over n_shards gathered chunks (splats >= n are ignored; bf16 rows
 * round to nearest even, which reproduces the owner's stored value). */
sc_status sc_splats_pack_range(sc_ctx* ctx, const sc_splats* s, uint32_t lo, uint32_t count, uint32_t shard,
                               float* out);
sc_status sc_splats_unpack_shards(sc_ctx* ctx, sc_splats* s, const float* in, uint32_t n_shards, uint32_t shard);
/* The same for the Adam moments (chunks of 2 * 59 rows: m then v), used to
 * give every rank the full moments before a densify or prune. */
sc_status sc_moments_pack_range(sc_ctx* ctx, const sc_moments* mo, uint32_t lo, uint32_t count, uint32_t shard,
                                float* out);
sc_status sc_moments_unpack_shards(sc_ctx* ctx, sc_moments* mo, uint32_t n, const float* in, uint32_t n_shards,
                                   uint32_t shard);

#ifdef __cplusplus
}
#endif
#endif /* SPLAT_CUDA_H */
