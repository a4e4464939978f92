// k_blend.cu — per-tile alpha blending (forward + adjoint), MSE, tonemap.
//
// Forward (rasterize.wgsl:48-118): one CTA per (view, tile), one thread per
// pixel.  The tile's depth-sorted splat records are staged into shared memory
// in batches of blockDim records with cp.async (LDGSTS, 3 x 16 B per record),
// double-buffered so the gather of batch b+1 overlaps the blending of batch b.
// The CTA leaves as soon as every pixel is saturated (T < 1e-4).  The MSE of
// loss.rs:163-179 is fused into the epilogue: each pixel writes
// dL/dC = scale * 2 (C - target) / (3 W H) and its squared error, reduced per
// CTA in FP64 and added once per CTA.
//
// Backward (rasterize_backward.wgsl:73-210): same grid, reverse walk.  Per
// (pixel, splat) gradients (dmean.xy, dopacity, dconic.abc, dcolor.rgb) are
// summed across the warp with shuffles (skipped when no lane contributes),
// the warp sums are added into a per-batch shared-memory slot, and each
// batch slot goes to global memory with three float4 vector atomics — one set
// per (tile, splat) instead of the reference's nine CAS loops per
// (pixel, splat).
#include "sc_internal.cuh"

namespace sck {

struct BlendArgs {
  uint32_t width, height, tw, th, tiles_x, tiles_y, num_tiles, stride;
  uint64_t pixels;  // per view
};

static BlendArgs blend_args(const sc_tiling* tl, uint32_t stride) {
  BlendArgs a;
  a.width = tl->width; a.height = tl->height; a.tw = tl->tile_w; a.th = tl->tile_h;
  a.tiles_x = (tl->width + tl->tile_w - 1) / tl->tile_w;
  a.tiles_y = (tl->height + tl->tile_h - 1) / tl->tile_h;
  a.num_tiles = a.tiles_x * a.tiles_y;
  a.stride = stride;
  a.pixels = (uint64_t)tl->width * tl->height;
  return a;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

#define ALPHA_MIN (1.0f / 255.0f)
#define ALPHA_MAX 0.99f

// Gaussian weight and alpha of one (pixel, splat); returns false when the
// reference skips the pair (power > 0 or alpha < 1/255).  Shared by forward
// and backward so both make identical skip decisions.
__device__ __forceinline__ bool eval_alpha(float dx, float dy, const float4 rb, float op, float& g, float& alpha_raw,
                                           float& alpha) {
  const float power = -0.5f * (rb.x * dx * dx + 2.0f * rb.y * dx * dy + rb.z * dy * dy);
  if (power > 0.0f) return false;
  g = __expf(power);
  alpha_raw = op * g;
  alpha = fminf(alpha_raw, ALPHA_MAX);
  return alpha >= ALPHA_MIN;
}

template <typename T>
__device__ __forceinline__ T block_sum(T x, T* sred) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if (lane == 0) sred[warp] = x;
  __syncthreads();
  T r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sred[w];
  return r;  // valid in thread 0
}

// ---------------------------------------------------------------- forward
__global__ void __launch_bounds__(256) k_composite(const float4* __restrict__ rec, const uint32_t* __restrict__ payloads,
                                                   const uint2* __restrict__ ranges, BlendArgs a,
                                                   float4* __restrict__ image, uint2* __restrict__ aux,
                                                   const float* __restrict__ target, float gscale,
                                                   float4* __restrict__ dl_dc, double* __restrict__ loss,
                                                   const uint32_t* __restrict__ skip) {
  extern __shared__ float4 sbuf[];  // [2][B][3]
  __shared__ double sred[8];
  if (skip && (*skip & SC_DEVERR_CAPACITY)) return;  // pair lists of this step are incomplete
  const uint32_t B = blockDim.x;
  const uint32_t vt = blockIdx.x;
  const uint32_t v = vt / a.num_tiles, tile = vt - v * a.num_tiles;
  const uint32_t ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
  const uint32_t lx = threadIdx.x % a.tw, ly = threadIdx.x / a.tw;
  const uint32_t px = tx * a.tw + lx, py = ty * a.th + ly;
  const bool inb = px < a.width && py < a.height;
  const float pxf = (float)px + 0.5f, pyf = (float)py + 0.5f;
  const uint2 r = ranges[vt];
  const uint32_t begin = r.x, end = r.y > r.x ? r.y : r.x;
  const uint32_t nb = (end - begin + B - 1) / B;
  const float4* vrec = rec + (size_t)3 * v * a.stride;

  auto stage = [&](uint32_t b) {
    const uint32_t j = begin + b * B + threadIdx.x;
    if (j < end) {
      const float4* src = vrec + (size_t)3 * payloads[j];
      float4* dst = sbuf + (size_t)(b & 1) * 3 * B + 3 * threadIdx.x;
      cp_async16(dst, src);
      cp_async16(dst + 1, src + 1);
      cp_async16(dst + 2, src + 2);
    }
    cp_async_commit();
  };

  float T = 1.0f, cr = 0.f, cg = 0.f, cb = 0.f;
  uint32_t last = 0;
  bool done = !inb;
  if (nb > 0) stage(0);
  for (uint32_t b = 0; b < nb; ++b) {
    if (b + 1 < nb) { stage(b + 1); cp_async_wait_one(); } else { cp_async_wait_all(); }
    __syncthreads();
    const uint32_t cnt = min(B, end - (begin + b * B));
    if (!done) {
      const float4* sb = sbuf + (size_t)(b & 1) * 3 * B;
      for (uint32_t k = 0; k < cnt; ++k) {
        const float4 ra = sb[3 * k], rb = sb[3 * k + 1];
        float g, araw, alpha;
        if (!eval_alpha(pxf - ra.x, pyf - ra.y, rb, sb[3 * k + 2].w, g, araw, alpha)) continue;
        const float4 rc = sb[3 * k + 2];
        const float ta = T * alpha;
        cr += ta * rc.x; cg += ta * rc.y; cb += ta * rc.z;
        T = T * (1.0f - alpha);
        last = b * B + k + 1;
        if (T < 1e-4f) { done = true; break; }
      }
    }
    if (__syncthreads_count(done) == (int)B) break;
  }
  cp_async_wait_all();
  double sq = 0.0;
  if (inb) {
    const size_t pix = (size_t)v * a.pixels + (size_t)py * a.width + px;
    image[pix] = make_float4(cr, cg, cb, 1.0f - T);
    if (aux) aux[pix] = make_uint2(__float_as_uint(T), last);
    if (target) {
      const float dx = cr - target[3 * pix], dy = cg - target[3 * pix + 1], dz = cb - target[3 * pix + 2];
      dl_dc[pix] = make_float4(dx * gscale, dy * gscale, dz * gscale, 0.0f);
      sq = (double)(dx * dx + dy * dy + dz * dz);
    }
  }
  if (target && loss) {
    const double s = block_sum(sq, sred);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(&loss[v], s);
  }
}

sc_status launch_composite(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views, const uint32_t* payloads,
                           const uint32_t* ranges, const sc_tiling* tl, float4* image, uint2* aux, const float* target,
                           float mse_scale, float4* dl_dc, double* loss, const uint32_t* d_skip) {
  const BlendArgs a = blend_args(tl, stride);
  const uint32_t threads = tl->tile_w * tl->tile_h;
  if (threads > 256 || threads % 32 != 0) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile must hold 32..256 pixels, multiple of 32");
  const uint64_t grid = (uint64_t)n_views * a.num_tiles;
  if (grid == 0) return SC_OK;
  const float n_scalars = (float)tl->width * (float)tl->height * 3.0f;
  const float gscale = (2.0f / n_scalars) * mse_scale;
  const size_t smem = (size_t)2 * 3 * threads * sizeof(float4);
  k_composite<<<(unsigned)grid, threads, smem, ctx->stream>>>(rec, payloads, reinterpret_cast<const uint2*>(ranges), a,
                                                              image, aux, target, gscale, dl_dc, loss, d_skip);
  return sc_check_launch(ctx, "k_composite");
}

// ---------------------------------------------------------------- MSE (standalone)
__global__ void k_mse(const float4* __restrict__ pred, const float* __restrict__ target, uint64_t P, uint32_t n_views,
                      float gscale, float4* __restrict__ dl_dc, double* __restrict__ loss) {
  __shared__ double sred[8];
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t v = (uint32_t)(((uint64_t)blockIdx.x * blockDim.x) / P);  // blocks never straddle views
  double sq = 0.0;
  if (q < P * n_views) {
    const float4 p = pred[q];
    const float dx = p.x - target[3 * q], dy = p.y - target[3 * q + 1], dz = p.z - target[3 * q + 2];
    dl_dc[q] = make_float4(dx * gscale, dy * gscale, dz * gscale, 0.0f);
    sq = (double)(dx * dx + dy * dy + dz * dz);
  }
  if (loss) {
    const double s = block_sum(sq, sred);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(&loss[v], s);
  }
}

__global__ void k_mse_views(const float4* __restrict__ pred, const float* __restrict__ target, uint64_t P,
                            float gscale, float4* __restrict__ dl_dc, double* __restrict__ loss) {
  __shared__ double sred[8];
  const uint32_t v = blockIdx.y;
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (i < P) {
    const uint64_t q = (uint64_t)v * P + i;
    const float4 p = pred[q];
    const float dx = p.x - target[3 * q], dy = p.y - target[3 * q + 1], dz = p.z - target[3 * q + 2];
    dl_dc[q] = make_float4(dx * gscale, dy * gscale, dz * gscale, 0.0f);
    sq = (double)(dx * dx + dy * dy + dz * dz);
  }
  if (loss) {
    const double s = block_sum(sq, sred);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(&loss[v], s);
  }
}

sc_status launch_mse(sc_ctx* ctx, const float4* pred, const float* target, uint64_t P, uint32_t n_views, float scale,
                     float4* dl_dc, double* loss) {
  if (P == 0 || n_views == 0) return SC_OK;
  const float n_scalars = (float)P * 3.0f;
  const float gscale = (2.0f / n_scalars) * scale;
  dim3 grid((unsigned)sc_div_up(P, 256), n_views);
  k_mse_views<<<grid, 256, 0, ctx->stream>>>(pred, target, P, gscale, dl_dc, loss);
  return sc_check_launch(ctx, "k_mse");
}

// ---------------------------------------------------------------- backward
__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__global__ void __launch_bounds__(256) k_composite_backward(const float4* __restrict__ rec,
                                                            const uint32_t* __restrict__ payloads,
                                                            const uint2* __restrict__ ranges, BlendArgs a,
                                                            const float4* __restrict__ fwd,
                                                            const float4* __restrict__ dl_dc, int mode,
                                                            const uint2* __restrict__ aux,
                                                            float4* __restrict__ proj_grad,
                                                            const uint32_t* __restrict__ skip) {
  extern __shared__ float4 sbuf[];  // records [2][B][3], acc [B][3] (float4), ids [2][B]
  __shared__ uint32_t s_max;
  if (skip && (*skip & SC_DEVERR_CAPACITY)) return;
  const uint32_t B = blockDim.x;
  float4* sacc = sbuf + (size_t)6 * B;
  uint32_t* sids = reinterpret_cast<uint32_t*>(sbuf + (size_t)9 * B);
  const uint32_t vt = blockIdx.x;
  const uint32_t v = vt / a.num_tiles, tile = vt - v * a.num_tiles;
  const uint32_t ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
  const uint32_t lx = threadIdx.x % a.tw, ly = threadIdx.x / a.tw;
  const uint32_t px = tx * a.tw + lx, py = ty * a.th + ly;
  const bool inb = px < a.width && py < a.height;
  const float pxf = (float)px + 0.5f, pyf = (float)py + 0.5f;
  const uint2 r = ranges[vt];
  const uint32_t begin = r.x, end = r.y > r.x ? r.y : r.x;
  if (end <= begin) return;
  const float4* vrec = rec + (size_t)3 * v * a.stride;
  float4* vgrad = proj_grad + (size_t)3 * v * a.stride;

  float T = 1.0f, gr = 0.f, gg = 0.f, gb = 0.f;
  uint32_t stop = begin;
  if (inb) {
    const size_t pix = (size_t)v * a.pixels + (size_t)py * a.width + px;
    const float4 d = dl_dc[pix];
    gr = d.x; gg = d.y; gb = d.z;
    if (mode == SC_BWD_REF) {
      T = 1.0f - fwd[pix].w;
      stop = end;
    } else {
      const uint2 x = aux[pix];
      T = __uint_as_float(x.x);
      stop = begin + min(x.y, end - begin);
    }
  }
  bool done = !inb;
  if (threadIdx.x == 0) s_max = begin;
  __syncthreads();
  if (inb) atomicMax(&s_max, stop);
  for (uint32_t t = threadIdx.x; t < B; t += B) {
    sacc[3 * t] = make_float4(0, 0, 0, 0); sacc[3 * t + 1] = make_float4(0, 0, 0, 0); sacc[3 * t + 2] = make_float4(0, 0, 0, 0);
  }
  __syncthreads();
  const uint32_t hi0 = s_max;
  if (hi0 <= begin) return;
  const uint32_t nb = (hi0 - begin + B - 1) / B;
  auto lo_of = [&](uint32_t b) -> uint32_t { const uint32_t hi = hi0 - b * B; return hi - min(B, hi - begin); };
  auto stage = [&](uint32_t b) {
    const uint32_t hi = hi0 - b * B, lo = hi - min(B, hi - begin);
    const uint32_t j = lo + threadIdx.x;
    if (j < hi) {
      const uint32_t id = payloads[j];
      sids[(b & 1) * B + threadIdx.x] = id;
      const float4* src = vrec + (size_t)3 * id;
      float4* dst = sbuf + (size_t)(b & 1) * 3 * B + 3 * threadIdx.x;
      cp_async16(dst, src);
      cp_async16(dst + 1, src + 1);
      cp_async16(dst + 2, src + 2);
    }
    cp_async_commit();
  };

  float Sr = 0.f, Sg = 0.f, Sb = 0.f;
  const int lane = threadIdx.x & 31;
  stage(0);
  for (uint32_t b = 0; b < nb; ++b) {
    if (b + 1 < nb) { stage(b + 1); cp_async_wait_one(); } else { cp_async_wait_all(); }
    __syncthreads();
    const uint32_t lo = lo_of(b);
    const uint32_t cnt = (hi0 - b * B) - lo;
    const float4* sb = sbuf + (size_t)(b & 1) * 3 * B;
    if (!__all_sync(0xffffffffu, done)) {
      for (int k = (int)cnt - 1; k >= 0; --k) {
        const uint32_t j = lo + (uint32_t)k;
        float c0 = 0.f, c1 = 0.f, c2 = 0.f, c4 = 0.f, c5 = 0.f, c6 = 0.f, c8 = 0.f, c9 = 0.f, c10 = 0.f;
        bool contrib = false;
        if (!done && j < stop) {
          const float4 ra = sb[3 * k], rb = sb[3 * k + 1], rc = sb[3 * k + 2];
          const float dx = pxf - ra.x, dy = pyf - ra.y;
          float g, araw, alpha;
          if (eval_alpha(dx, dy, rb, rc.w, g, araw, alpha)) {
            const float oma = fmaxf(1.0f - alpha, 1e-4f);
            T = T / oma;
            if (mode == SC_BWD_REF && T > 1.0001f) {
              done = true;
            } else {
              const float ta = T * alpha;
              c8 = gr * ta; c9 = gg * ta; c10 = gb * ta;
              const float da_r = T * rc.x - Sr / oma, da_g = T * rc.y - Sg / oma, da_b = T * rc.z - Sb / oma;
              const float galpha = gr * da_r + gg * da_g + gb * da_b;
              const float gar = araw < ALPHA_MAX ? galpha : 0.0f;
              c2 = gar * g;
              const float gpow = gar * rc.w * g;
              c4 = gpow * -0.5f * (dx * dx);
              c5 = gpow * -0.5f * (2.0f * dx * dy);
              c6 = gpow * -0.5f * (dy * dy);
              c0 = gpow * (rb.x * dx + rb.y * dy);
              c1 = gpow * (rb.y * dx + rb.z * dy);
              Sr += ta * rc.x; Sg += ta * rc.y; Sb += ta * rc.z;
              contrib = true;
            }
          }
        }
        if (__any_sync(0xffffffffu, contrib)) {
          c0 = warp_sum(c0); c1 = warp_sum(c1); c2 = warp_sum(c2);
          c4 = warp_sum(c4); c5 = warp_sum(c5); c6 = warp_sum(c6);
          c8 = warp_sum(c8); c9 = warp_sum(c9); c10 = warp_sum(c10);
          if (lane == 0) {
            float* acc = reinterpret_cast<float*>(sacc + 3 * k);
            atomicAdd(acc + 0, c0); atomicAdd(acc + 1, c1); atomicAdd(acc + 2, c2);
            atomicAdd(acc + 4, c4); atomicAdd(acc + 5, c5); atomicAdd(acc + 6, c6);
            atomicAdd(acc + 8, c8); atomicAdd(acc + 9, c9); atomicAdd(acc + 10, c10);
          }
        }
        if (__all_sync(0xffffffffu, done)) break;
      }
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
      float4* acc = sacc + 3 * threadIdx.x;
      const float4 a0 = acc[0], a1 = acc[1], a2 = acc[2];
      const uint32_t id = sids[(b & 1) * B + threadIdx.x];
      float4* dst = vgrad + (size_t)3 * id;
      if (a0.x != 0.f || a0.y != 0.f || a0.z != 0.f) atomicAdd(dst, a0);
      if (a1.x != 0.f || a1.y != 0.f || a1.z != 0.f) atomicAdd(dst + 1, a1);
      if (a2.x != 0.f || a2.y != 0.f || a2.z != 0.f) atomicAdd(dst + 2, a2);
      acc[0] = make_float4(0, 0, 0, 0); acc[1] = acc[0]; acc[2] = acc[0];
    }
    if (__syncthreads_count(done) == (int)B) break;
  }
  cp_async_wait_all();
}

sc_status launch_composite_backward(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                    const uint32_t* payloads, const uint32_t* ranges, const sc_tiling* tl,
                                    const float4* fwd, const float4* dl_dc, int mode, const uint2* aux,
                                    float4* proj_grad, const uint32_t* d_skip) {
  const BlendArgs a = blend_args(tl, stride);
  const uint32_t threads = tl->tile_w * tl->tile_h;
  if (threads > 256 || threads % 32 != 0) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile must hold 32..256 pixels, multiple of 32");
  if (mode == SC_BWD_EXACT && !aux) return sc_fail(ctx, SC_ERR_INVALID_ARG, "exact backward needs the forward aux buffer");
  const uint64_t grid = (uint64_t)n_views * a.num_tiles;
  if (grid == 0) return SC_OK;
  const size_t smem = (size_t)9 * threads * sizeof(float4) + (size_t)2 * threads * sizeof(uint32_t);
  k_composite_backward<<<(unsigned)grid, threads, smem, ctx->stream>>>(
      rec, payloads, reinterpret_cast<const uint2*>(ranges), a, fwd, dl_dc, mode, aux, proj_grad, d_skip);
  return sc_check_launch(ctx, "k_composite_backward");
}

// ---------------------------------------------------------------- tonemap (tonemap.wgsl:27-41)
__device__ __forceinline__ float srgb(float c) {
  c = fminf(fmaxf(c, 0.0f), 1.0f);
  return c > 0.0031308f ? 1.055f * powf(c, 1.0f / 2.4f) - 0.055f : c * 12.92f;
}
__device__ __forceinline__ uint8_t unorm8(float x) {
  x = fminf(fmaxf(x, 0.0f), 1.0f);
  return (uint8_t)__float2int_rn(x * 255.0f);
}
__global__ void k_tonemap(const float4* __restrict__ img, uint32_t w, uint32_t h, uchar4* __restrict__ out) {
  const uint32_t x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
  if (x >= w || y >= h) return;
  const size_t i = (size_t)y * w + x;
  const float4 p = img[i];
  const float r = p.x / (1.0f + fmaxf(p.x, 0.0f)), g = p.y / (1.0f + fmaxf(p.y, 0.0f)), b = p.z / (1.0f + fmaxf(p.z, 0.0f));
  out[i] = make_uchar4(unorm8(srgb(r)), unorm8(srgb(g)), unorm8(srgb(b)), unorm8(p.w));
}

sc_status launch_tonemap(sc_ctx* ctx, const float4* img, uint32_t w, uint32_t h, uint8_t* out) {
  if (w == 0 || h == 0) return SC_OK;
  dim3 grid((w + 15) / 16, (h + 15) / 16), block(16, 16);
  k_tonemap<<<grid, block, 0, ctx->stream>>>(img, w, h, reinterpret_cast<uchar4*>(out));
  return sc_check_launch(ctx, "k_tonemap");
}

}  // namespace sck
