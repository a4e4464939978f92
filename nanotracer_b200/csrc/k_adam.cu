// k_adam.cu — Adam (adam_step.wgsl:24-36 / adam.rs:70-90), constraints
// (apply_constraints.wgsl:24-41), densify statistic (accumulate_grad_pos.wgsl:17-23),
// and GPU densify / prune by stream compaction (train.rs:414-602).
//
// Adam runs over the coefficient-major slab: one elementwise pass over the 59
// rows with the row's learning-rate group; bias corrections bc1/bc2 come from
// the host in f32 (adam_gpu.rs:275-276).  With bf16 storage the moments (and
// SH-rest parameters) are widened to f32 for the update and rounded back: the
// moments to nearest, the parameters stochastically (bf16_stochastic), since
// an update below half a BF16 ulp would otherwise be lost every step.
//
// Prune and densify reproduce the reference's swap_remove order exactly.
// Removing a set R of m indices from n by swap_remove in descending index
// order (train.rs:577-600) leaves every kept index below n-m in place.  The
// removal of descending rank k is processed when the array ends at n-k, so
// it receives the element then at position n-k: the original element if n-k
// was kept, or — when n-k is itself a removed slot, filled earlier — the
// element that filled it, which is the content of position n-m+excl[n-k]
// (excl = exclusive count of removals).  That chain strictly increases and
// stops at a kept index.  So the compaction is a scan of the removal flags
// and a move of one element into each hole below n-m; nothing else moves.
#include "sc_internal.cuh"

#include <cmath>
#include <vector>

namespace sck {

// ---------------------------------------------------------------- Adam
__global__ void k_adam_lanes(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                             float* __restrict__ v, uint64_t n, float lr, float b1, float b2, float eps, float bc1,
                             float bc2) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mn = b1 * m[i] + (1.0f - b1) * gi;
    const float vn = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mn;
    v[i] = vn;
    const float mh = mn / bc1, vh = vn / bc2;
    p[i] = p[i] - lr * mh / (sqrtf(vh) + eps);
  }
}

sc_status launch_adam_lanes(sc_ctx* ctx, float* p, const float* g, float* m, float* v, uint64_t n, float lr, float b1,
                            float b2, float eps, float bc1, float bc2) {
  if (n == 0) return SC_OK;
  const unsigned grid = (unsigned)std::min<uint64_t>(sc_div_up(n, 256), (uint64_t)ctx->sm_count * 32);
  k_adam_lanes<<<grid, 256, 0, ctx->stream>>>(p, g, m, v, n, lr, b1, b2, eps, bc1, bc2);
  return sc_check_launch(ctx, "k_adam_lanes");
}

// grid.y = row (59), grid.x covers splats
__global__ void k_adam_all(DSplats s, const float* __restrict__ g, uint32_t gcap, DMoments mo, AdamParams ap) {
  const int r = blockIdx.y;
  const float lr = ap.lr[adam_group(r)];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
    const float gi = g[(size_t)r * gcap + i];
    const size_t k = (size_t)r * mo.cap + i;
    const float m0 = mo.bf16 ? __bfloat162float(mo.m16[k]) : mo.m[k];
    const float v0 = mo.bf16 ? __bfloat162float(mo.v16[k]) : mo.v[k];
    const float mn = ap.beta1 * m0 + (1.0f - ap.beta1) * gi;
    const float vn = ap.beta2 * v0 + (1.0f - ap.beta2) * gi * gi;
    if (mo.bf16) { mo.m16[k] = __float2bfloat16_rn(mn); mo.v16[k] = __float2bfloat16_rn(vn); }
    else { mo.m[k] = mn; mo.v[k] = vn; }
    const float mh = mn / ap.bc1, vh = vn / ap.bc2;
    const float p = sp_row(s, r, i);
    sp_set_sr(s, r, i, p - lr * mh / (sqrtf(vh) + ap.eps), ap.seed);
  }
}

sc_status launch_adam_all(sc_ctx* ctx, const DSplats& s, const float* g, uint32_t gcap, const DMoments& mo,
                          const AdamParams& ap) {
  if (s.n == 0) return SC_OK;
  dim3 grid((unsigned)std::min<uint64_t>(sc_div_up(s.n, 256), 1024), SC_NROWS);
  k_adam_all<<<grid, 256, 0, ctx->stream>>>(s, g, gcap, mo, ap);
  return sc_check_launch(ctx, "k_adam_all");
}

__global__ void k_constraints(DSplats s, float lsmin, float lsmax, float opmax) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  float* q = s.slab + (size_t)SC_ROW_ROT * s.cap + i;
  const float w = q[0], x = q[(size_t)s.cap], y = q[2 * (size_t)s.cap], z = q[3 * (size_t)s.cap];
  const float n2 = w * w + x * x + y * y + z * z;
  const float nrm = fmaxf(sqrtf(n2), 1e-8f);
  q[0] = w / nrm; q[(size_t)s.cap] = x / nrm; q[2 * (size_t)s.cap] = y / nrm; q[3 * (size_t)s.cap] = z / nrm;
  for (int k = 0; k < 3; ++k) {
    float* p = s.slab + (size_t)(SC_ROW_SCALE + k) * s.cap + i;
    *p = fminf(fmaxf(*p, lsmin), lsmax);
  }
  float* o = s.slab + (size_t)SC_ROW_OP * s.cap + i;
  *o = fminf(fmaxf(*o, -opmax), opmax);
}

sc_status launch_constraints(sc_ctx* ctx, const DSplats& s, float lsmin, float lsmax, float opmax) {
  if (s.n == 0) return SC_OK;
  k_constraints<<<(unsigned)sc_div_up(s.n, 256), 256, 0, ctx->stream>>>(s, lsmin, lsmax, opmax);
  return sc_check_launch(ctx, "k_constraints");
}

__global__ void k_accumulate(const float* __restrict__ g, uint32_t gcap, float* __restrict__ acc, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  acc[i] = acc[i] + fabsf(g[i]) + fabsf(g[(size_t)gcap + i]) + fabsf(g[2 * (size_t)gcap + i]);
}

sc_status launch_accumulate(sc_ctx* ctx, const float* g, uint32_t gcap, float* acc, uint32_t n) {
  if (n == 0) return SC_OK;
  k_accumulate<<<(unsigned)sc_div_up(n, 256), 256, 0, ctx->stream>>>(g, gcap, acc, n);
  return sc_check_launch(ctx, "k_accumulate");
}

// ---------------------------------------------------------------- streaming Adam over gradient rows
// Adam + constraints + densify statistic over splats [lo, lo+count) from
// gradient rows g[r * gstride + j], j = i - lo (gstride and lo multiples of 8,
// as are the slab and moment capacities).  grid.y picks a row group — 0
// position rows (+ the statistic), 1 the rotation rows (normalised together),
// 2..4 log-scale rows (clamped), 5 opacity (clamped), 6..8 sh_dc, 9.. the 45
// sh_rest rows — and each thread updates 8 consecutive splats of it with
// 16-byte loads and stores, so the pass streams at the memory's pace instead
// of waiting on one splat's 59 rows at a time.  Same arithmetic as
// adam_scalar_fast and constrain_geometry.
constexpr int ADAM_SPT = 8;
constexpr int ADAM_GROUPS = 9 + (SC_NROWS - SC_ROW_REST);

__device__ __forceinline__ void ld8(const float* p, float* o) {
  const float4 a = reinterpret_cast<const float4*>(p)[0], b = reinterpret_cast<const float4*>(p)[1];
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}
__device__ __forceinline__ void ld8(const __nv_bfloat16* p, float* o) {
  const uint4 u = *reinterpret_cast<const uint4*>(p);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[k]));
    o[2 * k] = f.x; o[2 * k + 1] = f.y;
  }
}
__device__ __forceinline__ void st8(float* p, const float* o) {
  reinterpret_cast<float4*>(p)[0] = make_float4(o[0], o[1], o[2], o[3]);
  reinterpret_cast<float4*>(p)[1] = make_float4(o[4], o[5], o[6], o[7]);
}
__device__ __forceinline__ void st8(__nv_bfloat16* p, const float* o) {
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(o[2 * k], o[2 * k + 1]);
    w[k] = *reinterpret_cast<const uint32_t*>(&h);
  }
  *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
}

// BF16 parameters of splats i0 .. i0+7 of row r, stochastically rounded
__device__ __forceinline__ void st8_sr(__nv_bfloat16* p, const float* o, uint32_t seed, int r, uint32_t i0) {
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const __nv_bfloat16 lo = bf16_stochastic(o[2 * k], sr_bits(seed, r, i0 + 2 * k));
    const __nv_bfloat16 hi = bf16_stochastic(o[2 * k + 1], sr_bits(seed, r, i0 + 2 * k + 1));
    w[k] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
  }
  *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
}

// one row of 8 splats: parameters, moments and gradients widened to f32;
// `nv` < 8 loads (and later stores) only the first nv splats
struct Row8 {
  float p[8], m[8], v[8], g[8];
};
__device__ __forceinline__ void load_row8(const DSplats& s, const DMoments& mo, const float* __restrict__ g, int r,
                                          uint32_t i0, uint32_t j0, uint32_t gstride, int nv, Row8& x) {
  const size_t pk = (size_t)r * s.cap + i0, mk = (size_t)r * mo.cap + i0, gk = (size_t)r * gstride + j0;
  const bool rest16 = r >= SC_ROW_REST && s.bf16;
  if (nv == ADAM_SPT) {
    ld8(g + gk, x.g);
    if (rest16) ld8(s.rest16 + (size_t)(r - SC_ROW_REST) * s.cap + i0, x.p); else ld8(s.slab + pk, x.p);
    if (mo.bf16) { ld8(mo.m16 + mk, x.m); ld8(mo.v16 + mk, x.v); } else { ld8(mo.m + mk, x.m); ld8(mo.v + mk, x.v); }
    return;
  }
#pragma unroll
  for (int e = 0; e < ADAM_SPT; ++e) {
    x.g[e] = x.p[e] = x.m[e] = x.v[e] = 0.0f;
    if (e < nv) {
      x.g[e] = g[gk + e];
      x.p[e] = sp_row(s, r, i0 + e);
      x.m[e] = mo_ld(mo, mo.m, mo.m16, mk + e);
      x.v[e] = mo_ld(mo, mo.v, mo.v16, mk + e);
    }
  }
}
__device__ __forceinline__ void store_row8(const DSplats& s, const DMoments& mo, int r, uint32_t i0, int nv,
                                           const Row8& x, uint32_t seed) {
  const size_t pk = (size_t)r * s.cap + i0, mk = (size_t)r * mo.cap + i0;
  const bool rest16 = r >= SC_ROW_REST && s.bf16;
  if (nv == ADAM_SPT) {
    if (rest16) st8_sr(s.rest16 + (size_t)(r - SC_ROW_REST) * s.cap + i0, x.p, seed, r, i0);
    else st8(s.slab + pk, x.p);
    if (mo.bf16) { st8(mo.m16 + mk, x.m); st8(mo.v16 + mk, x.v); } else { st8(mo.m + mk, x.m); st8(mo.v + mk, x.v); }
    return;
  }
#pragma unroll
  for (int e = 0; e < ADAM_SPT; ++e) {
    if (e < nv) {
      sp_set_sr(s, r, i0 + e, x.p[e], seed);
      mo_st(mo, mo.m, mo.m16, mk + e, x.m[e]);
      mo_st(mo, mo.v, mo.v16, mk + e, x.v[e]);
    }
  }
}
// adam_scalar_fast on a row of 8
__device__ __forceinline__ void adam_row8(Row8& x, float a, float s2, const AdamParams& ap) {
#pragma unroll
  for (int e = 0; e < ADAM_SPT; ++e) {
    const float gr = x.g[e];
    const float m = ap.beta1 * x.m[e] + (1.0f - ap.beta1) * gr;
    const float v = ap.beta2 * x.v[e] + (1.0f - ap.beta2) * gr * gr;
    x.m[e] = m;
    x.v[e] = v;
    x.p[e] = x.p[e] - __fdividef(a * m, fmaf(sqrtf(v), s2, ap.eps));
  }
}

// GEOM: the 9 geometric row groups (grid.y 0..8); otherwise the 45 sh_rest
// rows (grid.y 0..44), a separate launch with its own, smaller register count.
// The geometric launch is held to 3 CTAs per SM (80 registers, a few bytes
// spilled in the rotation group): more rows in flight beat the spill.
template <bool GEOM>
__device__ __forceinline__ void adam_rows(const DSplats& s, const DMoments& mo, float* __restrict__ acc,
                                          const float* __restrict__ g, uint32_t lo, uint32_t count, uint32_t gstride,
                                          AdamParams ap, const float* __restrict__ d_bc,
                                          const uint32_t* __restrict__ skip) {
  const uint32_t j0 = (blockIdx.x * blockDim.x + threadIdx.x) * ADAM_SPT;
  if (j0 >= count) return;
  if (skip && (*skip & SC_DEVERR_CAPACITY)) return;  // a capacity overflow earlier in the step: leave parameters untouched
  if (d_bc) { ap.bc1 = d_bc[0]; ap.bc2 = d_bc[1]; ap.seed = __float_as_uint(d_bc[2]); }  // [2]: the step's bits
  const AdamFast af = adam_fast(ap);
  const int nv = (int)min((uint32_t)ADAM_SPT, count - j0);
  const uint32_t i0 = lo + j0;
  const int y = GEOM ? (int)blockIdx.y : 9 + (int)blockIdx.y;
  Row8 x;
  if (GEOM && y == 0) {  // position, and the densify statistic (accumulate_grad_pos.wgsl:17-23) from its gradients
    float st[ADAM_SPT];  // ((acc + |g0|) + |g1|) + |g2|, as the per-splat kernels add
#pragma unroll
    for (int e = 0; e < ADAM_SPT; ++e) st[e] = (acc && e < nv) ? acc[i0 + e] : 0.0f;
    for (int r = 0; r < 3; ++r) {
      load_row8(s, mo, g, r, i0, j0, gstride, nv, x);
#pragma unroll
      for (int e = 0; e < ADAM_SPT; ++e) st[e] = st[e] + fabsf(x.g[e]);
      adam_row8(x, af.a[0], af.s2, ap);
      store_row8(s, mo, r, i0, nv, x, ap.seed);
    }
    if (acc) {
#pragma unroll
      for (int e = 0; e < ADAM_SPT; ++e)
        if (e < nv) acc[i0 + e] = st[e];
    }
    return;
  }
  if (GEOM && y == 1) {  // rotation: update the four rows, then normalise each splat's quaternion from them
    for (int c = 0; c < 4; ++c) {
      load_row8(s, mo, g, SC_ROW_ROT + c, i0, j0, gstride, nv, x);
      adam_row8(x, af.a[1], af.s2, ap);
      store_row8(s, mo, SC_ROW_ROT + c, i0, nv, x, ap.seed);
    }
    float q[4][ADAM_SPT];
    for (int c = 0; c < 4; ++c) {
      const float* row = s.slab + (size_t)(SC_ROW_ROT + c) * s.cap + i0;
      if (nv == ADAM_SPT) {
        ld8(row, q[c]);
      } else {
#pragma unroll
        for (int e = 0; e < ADAM_SPT; ++e) q[c][e] = e < nv ? row[e] : 1.0f;
      }
    }
#pragma unroll
    for (int e = 0; e < ADAM_SPT; ++e) {
      const float n2 = q[0][e] * q[0][e] + q[1][e] * q[1][e] + q[2][e] * q[2][e] + q[3][e] * q[3][e];
      const float nrm = fmaxf(sqrtf(n2), 1e-8f);
      for (int c = 0; c < 4; ++c) q[c][e] /= nrm;
    }
    for (int c = 0; c < 4; ++c) {
      float* row = s.slab + (size_t)(SC_ROW_ROT + c) * s.cap + i0;
      if (nv == ADAM_SPT) {
        st8(row, q[c]);
      } else {
#pragma unroll
        for (int e = 0; e < ADAM_SPT; ++e)
          if (e < nv) row[e] = q[c][e];
      }
    }
    return;
  }
  // single rows: 7..9 log scale, 10 opacity, 11..13 sh_dc, 14.. sh_rest
  const int r = y <= 8 ? y + 5 : SC_ROW_REST + (y - 9);
  load_row8(s, mo, g, r, i0, j0, gstride, nv, x);
  adam_row8(x, af.a[adam_group(r)], af.s2, ap);
  if (r >= SC_ROW_SCALE && r < SC_ROW_SCALE + 3) {
#pragma unroll
    for (int e = 0; e < ADAM_SPT; ++e) x.p[e] = fminf(fmaxf(x.p[e], ap.log_scale_min), ap.log_scale_max);
  } else if (r == SC_ROW_OP) {
#pragma unroll
    for (int e = 0; e < ADAM_SPT; ++e) x.p[e] = fminf(fmaxf(x.p[e], -ap.opacity_logit_max), ap.opacity_logit_max);
  }
  store_row8(s, mo, r, i0, nv, x, ap.seed);
}

template <bool GEOM>
__global__ void __launch_bounds__(256, GEOM ? 3 : 4) k_adam_rows(DSplats s, DMoments mo, float* __restrict__ acc,
                                                   const float* __restrict__ g, uint32_t lo, uint32_t count,
                                                   uint32_t gstride, AdamParams ap, const float* __restrict__ d_bc,
                                                   const uint32_t* __restrict__ skip) {
  adam_rows<GEOM>(s, mo, acc, g, lo, count, gstride, ap, d_bc, skip);
}

// Many scenes: grid.z = scene, each with its own store, moments, statistic
// and gradient rows (all of its splats, the shared step t).
template <bool GEOM>
__global__ void __launch_bounds__(256, GEOM ? 3 : 4) k_adam_rows_scenes(const SceneDev* __restrict__ scenes,
                                                          AdamParams ap, const float* __restrict__ d_bc,
                                                          const uint32_t* __restrict__ skip) {
  const SceneDev sd = scenes[blockIdx.z];
  adam_rows<GEOM>(sd.s, sd.mo, sd.acc, sd.grads, 0, sd.s.n, sd.gstride, ap, d_bc, skip);
}

sc_status launch_adam_rows_scenes(sc_ctx* ctx, const SceneDev* d_scenes, uint32_t n_scenes, uint32_t max_count,
                                  const AdamParams& ap, const float* d_bc, const uint32_t* d_skip) {
  if (n_scenes == 0 || max_count == 0) return SC_OK;
  const unsigned gx = (unsigned)sc_div_up(sc_div_up(max_count, ADAM_SPT), 256);
  k_adam_rows_scenes<true><<<dim3(gx, 9, n_scenes), 256, 0, ctx->stream>>>(d_scenes, ap, d_bc, d_skip);
  SC_TRY(sc_check_launch(ctx, "k_adam_rows_scenes"));
  k_adam_rows_scenes<false><<<dim3(gx, ADAM_GROUPS - 9, n_scenes), 256, 0, ctx->stream>>>(d_scenes, ap, d_bc, d_skip);
  return sc_check_launch(ctx, "k_adam_rows_scenes");
}

sc_status launch_adam_rows(sc_ctx* ctx, const DSplats& s, const DMoments& mo, float* acc, const float* g, uint32_t lo,
                           uint32_t count, uint32_t gstride, const AdamParams& ap, const float* d_bc,
                           const uint32_t* d_skip) {
  if (count == 0) return SC_OK;
  if (lo % ADAM_SPT || gstride % ADAM_SPT || s.cap % ADAM_SPT || mo.cap % ADAM_SPT)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "Adam rows: offsets and strides must be multiples of 8");
  const unsigned gx = (unsigned)sc_div_up(sc_div_up(count, ADAM_SPT), 256);
  k_adam_rows<true><<<dim3(gx, 9), 256, 0, ctx->stream>>>(s, mo, acc, g, lo, count, gstride, ap, d_bc, d_skip);
  SC_TRY(sc_check_launch(ctx, "k_adam_rows"));
  k_adam_rows<false><<<dim3(gx, ADAM_GROUPS - 9), 256, 0, ctx->stream>>>(s, mo, acc, g, lo, count, gstride, ap, d_bc,
                                                                          d_skip);
  return sc_check_launch(ctx, "k_adam_rows");
}

// ---------------------------------------------------------------- data-parallel shards
// Adam + constraints + densify statistic on one reduce-scattered chunk
// g[r * shard + j] for splats [lo, lo+count): the streaming row kernel.
sc_status launch_adam_shard(sc_ctx* ctx, const DSplats& s, const DMoments& mo, float* acc, const float* g, uint32_t lo,
                            uint32_t count, uint32_t shard, const AdamParams& ap) {
  return launch_adam_rows(ctx, s, mo, acc, g, lo, count, shard, ap, nullptr, nullptr);
}

// grid.y = row
__global__ void k_pack_params(DSplats s, uint32_t lo, uint32_t count, uint32_t shard, float* __restrict__ out) {
  const int r = blockIdx.y;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
    out[(size_t)r * shard + j] = sp_row(s, r, lo + j);
}

// in = n_shards chunks of SC_NROWS rows x shard; splat i = q * shard + j
__global__ void k_unpack_params(DSplats s, const float* __restrict__ in, uint32_t n_shards, uint32_t shard) {
  const int r = blockIdx.y;
  const uint64_t total = std::min<uint64_t>((uint64_t)n_shards * shard, s.n);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t q = i / shard, j = i % shard;
    sp_set(s, r, (uint32_t)i, in[(q * SC_NROWS + r) * shard + j]);
  }
}

__global__ void k_pack_moments(DMoments mo, uint32_t lo, uint32_t count, uint32_t shard, float* __restrict__ out) {
  const int r = blockIdx.y >> 1, which = blockIdx.y & 1;  // m rows then v rows, interleaved by grid.y
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
    const size_t k = (size_t)r * mo.cap + lo + j;
    const float x = which ? mo_ld(mo, mo.v, mo.v16, k) : mo_ld(mo, mo.m, mo.m16, k);
    out[((size_t)which * SC_NROWS + r) * shard + j] = x;
  }
}

// in = n_shards chunks of 2 * SC_NROWS rows (m then v) x shard
__global__ void k_unpack_moments(DMoments mo, uint32_t n, const float* __restrict__ in, uint32_t n_shards,
                                 uint32_t shard) {
  const int r = blockIdx.y >> 1, which = blockIdx.y & 1;
  const uint64_t total = std::min<uint64_t>((uint64_t)n_shards * shard, n);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t q = i / shard, j = i % shard;
    const float x = in[((q * 2 + which) * SC_NROWS + r) * shard + j];
    const size_t k = (size_t)r * mo.cap + i;
    if (which) mo_st(mo, mo.v, mo.v16, k, x); else mo_st(mo, mo.m, mo.m16, k, x);
  }
}

static unsigned rows_grid_x(sc_ctx* ctx, uint64_t n) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(sc_div_up(n, 256), (uint64_t)ctx->sm_count * 4));
}

sc_status launch_pack_params(sc_ctx* ctx, const DSplats& s, uint32_t lo, uint32_t count, uint32_t shard, float* out) {
  if (count == 0) return SC_OK;
  k_pack_params<<<dim3(rows_grid_x(ctx, count), SC_NROWS), 256, 0, ctx->stream>>>(s, lo, count, shard, out);
  return sc_check_launch(ctx, "k_pack_params");
}
sc_status launch_unpack_params(sc_ctx* ctx, const DSplats& s, const float* in, uint32_t n_shards, uint32_t shard) {
  if (s.n == 0 || n_shards == 0 || shard == 0) return SC_OK;
  k_unpack_params<<<dim3(rows_grid_x(ctx, s.n), SC_NROWS), 256, 0, ctx->stream>>>(s, in, n_shards, shard);
  return sc_check_launch(ctx, "k_unpack_params");
}
sc_status launch_pack_moments(sc_ctx* ctx, const DMoments& mo, uint32_t lo, uint32_t count, uint32_t shard, float* out) {
  if (count == 0) return SC_OK;
  k_pack_moments<<<dim3(rows_grid_x(ctx, count), 2 * SC_NROWS), 256, 0, ctx->stream>>>(mo, lo, count, shard, out);
  return sc_check_launch(ctx, "k_pack_moments");
}
sc_status launch_unpack_moments(sc_ctx* ctx, const DMoments& mo, uint32_t n, const float* in, uint32_t n_shards,
                                uint32_t shard) {
  if (n == 0 || n_shards == 0 || shard == 0) return SC_OK;
  k_unpack_moments<<<dim3(rows_grid_x(ctx, n), 2 * SC_NROWS), 256, 0, ctx->stream>>>(mo, n, in, n_shards, shard);
  return sc_check_launch(ctx, "k_unpack_moments");
}

// ---------------------------------------------------------------- compaction helpers
// copy every parameter row, moment row and the statistic of splat `src` to `dst`
__device__ __forceinline__ void move_splat(const DSplats& s, const DMoments& mo, float* acc, uint32_t dst, uint32_t src) {
  const int frows = s.bf16 ? SC_ROW_REST : SC_NROWS;
  for (int r = 0; r < frows; ++r) s.slab[(size_t)r * s.cap + dst] = s.slab[(size_t)r * s.cap + src];
  if (s.bf16)
    for (int k = 0; k < 45; ++k) s.rest16[(size_t)k * s.cap + dst] = s.rest16[(size_t)k * s.cap + src];
  if (mo.m || mo.m16) {
    for (int r = 0; r < SC_NROWS; ++r) {
      const size_t a = (size_t)r * mo.cap + dst, b = (size_t)r * mo.cap + src;
      if (mo.bf16) { mo.m16[a] = mo.m16[b]; mo.v16[a] = mo.v16[b]; }
      else { mo.m[a] = mo.m[b]; mo.v[a] = mo.v[b]; }
    }
  }
  if (acc) acc[dst] = acc[src];
}

__device__ __forceinline__ void zero_moments(const DMoments& mo, uint32_t dst) {
  if (!(mo.m || mo.m16)) return;
  for (int r = 0; r < SC_NROWS; ++r) {
    const size_t a = (size_t)r * mo.cap + dst;
    if (mo.bf16) { mo.m16[a] = __float2bfloat16_rn(0.0f); mo.v16[a] = __float2bfloat16_rn(0.0f); }
    else { mo.m[a] = 0.0f; mo.v[a] = 0.0f; }
  }
}

// ---------------------------------------------------------------- prune (train.rs:572-602)
__global__ void k_prune_flags(const float* __restrict__ op, uint32_t n, float thr, uint32_t* __restrict__ flags) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flags[i] = op[i] < thr ? 1u : 0u;
}

// excl = exclusive count of removals, m = removals, holes are removed j < n - m.
// Sources are read only from positions >= n - m, which no thread writes.
__global__ void k_prune_move(DSplats s, DMoments mo, float* acc, uint32_t n, uint32_t m, float thr,
                             const uint32_t* __restrict__ excl) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t new_n = n - m;
  if (j >= new_n) return;
  const float* op = s.slab + (size_t)SC_ROW_OP * s.cap;
  if (!(op[j] < thr)) return;
  uint32_t q = n - (m - excl[j]);
  for (uint32_t guard = 0; guard <= m && op[q] < thr; ++guard) q = new_n + excl[q];  // strictly increasing chain
  move_splat(s, mo, acc, j, q);
}

sc_status prune(sc_ctx* ctx, sc_splats* sp, sc_moments* mo, float* acc, float thr, uint32_t* removed) {
  const uint32_t n = sp->n;
  *removed = 0;
  if (n == 0) return SC_OK;
  // scratch: excl (n+1 u32) | total (u64) | scan state
  const size_t scan_bytes = scan_scratch_bytes(n + 1);
  const size_t o_tot = (((size_t)(n + 1) * 4) + 255) & ~(size_t)255;
  const size_t o_scan = o_tot + 256;
  void* scr;
  SC_TRY(sc_scratch(ctx, o_scan + scan_bytes, &scr));
  uint32_t* excl = reinterpret_cast<uint32_t*>(scr);
  uint64_t* d_total = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(scr) + o_tot);
  void* sscr = reinterpret_cast<char*>(scr) + o_scan;
  const DSplats s = dview(sp);
  k_prune_flags<<<(unsigned)sc_div_up(n, 256), 256, 0, ctx->stream>>>(s.slab + (size_t)SC_ROW_OP * s.cap, n, thr, excl);
  SC_TRY(sc_check_launch(ctx, "k_prune_flags"));
  SC_CUDA_TRY(ctx, cudaMemsetAsync(excl + n, 0, 4, ctx->stream), "memset");
  SC_TRY(scan_u32(ctx, excl, n + 1, d_total, sscr, scan_bytes));
  uint64_t m = 0;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(&m, d_total, 8, cudaMemcpyDeviceToHost, ctx->stream), "readback");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  SC_TRY(sc_check_device_error(ctx));
  if (m == 0) return SC_OK;
  const uint32_t new_n = n - (uint32_t)m;
  const DMoments dm = mo ? dview(mo) : DMoments{nullptr, nullptr, nullptr, nullptr, 0, 0};
  if (new_n > 0) {
    k_prune_move<<<(unsigned)sc_div_up(new_n, 256), 256, 0, ctx->stream>>>(s, dm, acc, n, (uint32_t)m, thr, excl);
    SC_TRY(sc_check_launch(ctx, "k_prune_move"));
  }
  sp->n = new_n;
  *removed = (uint32_t)m;
  return SC_OK;
}

// ---------------------------------------------------------------- densify (train.rs:414-549)
// Affine LCG x -> a x + c (mod 2^32) advanced k steps by binary powering.
__device__ __forceinline__ uint32_t lcg_jump(uint32_t x, uint64_t k) {
  uint32_t A = 1u, C = 0u;               // accumulated map
  uint32_t a = 1664525u, c = 1013904223u;  // current power-of-two map
  while (k) {
    if (k & 1) { A = a * A; C = a * C + c; }
    c = a * c + c;
    a = a * a;
    k >>= 1;
  }
  return A * x + C;
}

// lcg01 / box_muller of train.rs:552-564 on draw index k (0-based) from state0
__device__ __forceinline__ float lcg01_at(uint32_t state0, uint64_t k) {
  const uint32_t st = lcg_jump(state0, k + 1);
  return (float)st / ((float)UINT32_MAX + 1.0f);
}
__device__ __forceinline__ float box_muller_at(uint32_t state0, uint64_t k) {
  const float u1 = fmaxf(lcg01_at(state0, k), 1e-8f);
  const float u2 = lcg01_at(state0, k + 1);
  const float two_pi = 2.0f * 3.14159265358979323846f;
  return sqrtf(-2.0f * logf(u1)) * cosf(two_pi * u2);
}

struct DensifyArgs {
  uint32_t n, budget, grad_count;
  float count_f, gthr, sthr, half, log_split;
  uint32_t state0;
};

// flags: cand (bit0), split-kind (bit1)
__global__ void k_densify_cand(DSplats s, const float* __restrict__ acc, DensifyArgs a, uint32_t* __restrict__ cand,
                               uint8_t* __restrict__ kind) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const float avg = acc[i] / a.count_f;
  const bool c = avg > a.gthr;
  float mx = -INFINITY;
  for (int k = 0; k < 3; ++k) mx = fmaxf(mx, s.slab[(size_t)(SC_ROW_SCALE + k) * s.cap + i]);
  cand[i] = c ? 1u : 0u;
  kind[i] = (mx > a.sthr) ? 1 : 0;
}

// after scanning cand: accepted = cand && rank < budget; write clone / split flags
__global__ void k_densify_accept(uint32_t n, uint32_t budget, const uint32_t* __restrict__ cand_excl,
                                 const uint32_t* __restrict__ cand_flag_src, const uint8_t* __restrict__ kind,
                                 uint32_t* __restrict__ clone_f, uint32_t* __restrict__ split_f) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool cand = cand_excl[i + 1] != cand_excl[i];
  const bool acc = cand && cand_excl[i] < budget;
  (void)cand_flag_src;
  clone_f[i] = (acc && !kind[i]) ? 1u : 0u;
  split_f[i] = (acc && kind[i]) ? 1u : 0u;
}

// record originals: clone rank -> index, split rank -> index
__global__ void k_densify_lists(uint32_t n, const uint32_t* __restrict__ clone_excl, const uint32_t* __restrict__ split_excl,
                                uint32_t* __restrict__ clone_list, uint32_t* __restrict__ split_list) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (clone_excl[i + 1] != clone_excl[i]) clone_list[clone_excl[i]] = i;
  if (split_excl[i + 1] != split_excl[i]) split_list[split_excl[i]] = i;
}

// clones: copy parent -> slot n + c with opacity + ln(1/2); parent opacity + ln(1/2)
__global__ void k_densify_clones(DSplats s, DMoments mo, float* acc, uint32_t n, uint32_t n_clone,
                                 const uint32_t* __restrict__ clone_list, float half) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_clone) return;
  const uint32_t i = clone_list[c], dst = n + c;
  const int frows = s.bf16 ? SC_ROW_REST : SC_NROWS;
  for (int r = 0; r < frows; ++r) s.slab[(size_t)r * s.cap + dst] = s.slab[(size_t)r * s.cap + i];
  if (s.bf16)
    for (int k = 0; k < 45; ++k) s.rest16[(size_t)k * s.cap + dst] = s.rest16[(size_t)k * s.cap + i];
  const float op_new = s.slab[(size_t)SC_ROW_OP * s.cap + i] + half;
  s.slab[(size_t)SC_ROW_OP * s.cap + dst] = op_new;
  s.slab[(size_t)SC_ROW_OP * s.cap + i] = op_new;
  zero_moments(mo, dst);
  if (acc) acc[dst] = 0.0f;
}

// children of split rank s into a staging area (2 per split), 59 fp32 rows each
__global__ void k_densify_children(DSplats s, uint32_t n_split, const uint32_t* __restrict__ split_list,
                                   DensifyArgs a, float* __restrict__ stage) {
  const uint32_t sr = blockIdx.x * blockDim.x + threadIdx.x;
  if (sr >= n_split) return;
  const uint32_t i = split_list[sr];
  float p[SC_NROWS];
  for (int r = 0; r < SC_NROWS; ++r) p[r] = sp_row(s, r, i);
  const float sig[3] = {expf(p[7]), expf(p[8]), expf(p[9])};
  // quaternion (x, y, z, w) from stored (w, x, y, z)
  const float bx = p[4], by = p[5], bz = p[6], w = p[3];
  for (int c = 0; c < 2; ++c) {
    const uint64_t k0 = (uint64_t)sr * 12 + (uint64_t)c * 6;
    const float o0 = box_muller_at(a.state0, k0) * sig[0];
    const float o1 = box_muller_at(a.state0, k0 + 2) * sig[1];
    const float o2 = box_muller_at(a.state0, k0 + 4) * sig[2];
    const float b2 = bx * bx + by * by + bz * bz;
    const float vb2 = (o0 * bx + o1 * by + o2 * bz) * 2.0f;
    const float ww = w * w - b2;
    const float cx = by * o2 - o1 * bz, cy = bz * o0 - o2 * bx, cz = bx * o1 - o0 * by;
    const float w2 = w * 2.0f;
    const float rx = (o0 * ww + bx * vb2) + cx * w2;
    const float ry = (o1 * ww + by * vb2) + cy * w2;
    const float rz = (o2 * ww + bz * vb2) + cz * w2;
    float* out = stage + (size_t)(2 * sr + c) * SC_NROWS;
    for (int r = 0; r < SC_NROWS; ++r) out[r] = p[r];
    out[0] = p[0] + rx; out[1] = p[1] + ry; out[2] = p[2] + rz;
    out[7] = p[7] + a.log_split; out[8] = p[8] + a.log_split; out[9] = p[9] + a.log_split;
  }
}

// child t (0 .. 2S-1) goes to slot n + n_clone + t when t < S, otherwise into the
// slot of the parent of split rank t - S (the swap_remove pairing)
__global__ void k_densify_place(DSplats s, DMoments mo, float* acc, uint32_t n, uint32_t n_clone, uint32_t n_split,
                                const uint32_t* __restrict__ split_list, const float* __restrict__ stage) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * n_split) return;
  const uint32_t dst = t < n_split ? n + n_clone + t : split_list[t - n_split];
  const float* src = stage + (size_t)t * SC_NROWS;
  for (int r = 0; r < SC_NROWS; ++r) sp_set(s, r, dst, src[r]);
  zero_moments(mo, dst);
  if (acc) acc[dst] = 0.0f;
}

sc_status densify(sc_ctx* ctx, sc_splats* sp, sc_moments* mo, float* acc, uint32_t grad_count, float gthr, float sthr,
                  uint32_t max_splats, uint32_t iter, uint32_t counts[3]) {
  counts[0] = counts[1] = counts[2] = 0;
  const uint32_t n = sp->n;
  if (n == 0) return SC_OK;
  DensifyArgs a;
  a.n = n;
  a.budget = max_splats > n ? max_splats - n : 0u;
  a.grad_count = grad_count;
  a.count_f = (float)(grad_count > 1 ? grad_count : 1u);
  a.gthr = gthr;
  a.sthr = sthr;
  a.half = -0.69314718055994530942f;
  a.log_split = -std::log(1.6f);
  a.state0 = iter * 1664525u + 1013904223u;
  const size_t n1 = (size_t)n + 1;
  const size_t scan_bytes = scan_scratch_bytes(n1);
  // layout: cand_excl | clone_excl | split_excl (n+1 each) | clone_list | split_list (n each) | kind (n) | totals | scan
  size_t off = 0;
  auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
  const size_t o_cand = take(n1 * 4), o_clone = take(n1 * 4), o_split = take(n1 * 4), o_cl = take((size_t)n * 4),
               o_sl = take((size_t)n * 4), o_kind = take(n), o_tot = take(32), o_scan = take(scan_bytes);
  void* scr;
  SC_TRY(sc_scratch(ctx, off, &scr));
  char* base = reinterpret_cast<char*>(scr);
  uint32_t* cand = reinterpret_cast<uint32_t*>(base + o_cand);
  uint32_t* clone_f = reinterpret_cast<uint32_t*>(base + o_clone);
  uint32_t* split_f = reinterpret_cast<uint32_t*>(base + o_split);
  uint32_t* clone_list = reinterpret_cast<uint32_t*>(base + o_cl);
  uint32_t* split_list = reinterpret_cast<uint32_t*>(base + o_sl);
  uint8_t* kind = reinterpret_cast<uint8_t*>(base + o_kind);
  uint64_t* tot = reinterpret_cast<uint64_t*>(base + o_tot);
  void* sscr = base + o_scan;
  const DSplats s = dview(sp);
  const unsigned g = (unsigned)sc_div_up(n, 256);
  SC_CUDA_TRY(ctx, cudaMemsetAsync(cand + n, 0, 4, ctx->stream), "memset");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(clone_f + n, 0, 4, ctx->stream), "memset");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(split_f + n, 0, 4, ctx->stream), "memset");
  k_densify_cand<<<g, 256, 0, ctx->stream>>>(s, acc, a, cand, kind);
  SC_TRY(sc_check_launch(ctx, "k_densify_cand"));
  SC_TRY(scan_u32(ctx, cand, n1, tot, sscr, scan_bytes));
  k_densify_accept<<<g, 256, 0, ctx->stream>>>(n, a.budget, cand, nullptr, kind, clone_f, split_f);
  SC_TRY(sc_check_launch(ctx, "k_densify_accept"));
  SC_TRY(scan_u32(ctx, clone_f, n1, tot + 1, sscr, scan_bytes));
  SC_TRY(scan_u32(ctx, split_f, n1, tot + 2, sscr, scan_bytes));
  k_densify_lists<<<g, 256, 0, ctx->stream>>>(n, clone_f, split_f, clone_list, split_list);
  SC_TRY(sc_check_launch(ctx, "k_densify_lists"));
  uint64_t h_tot[3];
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(h_tot, tot, 24, cudaMemcpyDeviceToHost, ctx->stream), "readback");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  SC_TRY(sc_check_device_error(ctx));
  const uint32_t n_clone = (uint32_t)h_tot[1], n_split = (uint32_t)h_tot[2];
  if (n_clone + n_split == 0) return SC_OK;
  const uint32_t new_n = n + n_clone + n_split;
  if (new_n > sp->cap || (mo && new_n > mo->cap))
    return sc_fail(ctx, SC_ERR_CAPACITY, "densify: splat / moment capacity below the grown count (reserve max_splats)");
  const DMoments dm = mo ? dview(mo) : DMoments{nullptr, nullptr, nullptr, nullptr, 0, 0};
  if (n_clone) {
    k_densify_clones<<<(unsigned)sc_div_up(n_clone, 128), 128, 0, ctx->stream>>>(s, dm, acc, n, n_clone, clone_list,
                                                                                 a.half);
    SC_TRY(sc_check_launch(ctx, "k_densify_clones"));
  }
  if (n_split) {
    float* stage;
    // separate allocation: the scan scratch above is still in use by the lists
    SC_CUDA_TRY(ctx, cudaMallocAsync(reinterpret_cast<void**>(&stage), (size_t)2 * n_split * SC_NROWS * 4, ctx->stream),
                "alloc densify stage");
    k_densify_children<<<(unsigned)sc_div_up(n_split, 64), 64, 0, ctx->stream>>>(s, n_split, split_list, a, stage);
    SC_TRY(sc_check_launch(ctx, "k_densify_children"));
    DSplats s2 = s;
    s2.n = new_n;
    k_densify_place<<<(unsigned)sc_div_up(2 * n_split, 128), 128, 0, ctx->stream>>>(s2, dm, acc, n, n_clone, n_split,
                                                                                    split_list, stage);
    SC_TRY(sc_check_launch(ctx, "k_densify_place"));
    SC_CUDA_TRY(ctx, cudaFreeAsync(stage, ctx->stream), "free densify stage");
  }
  sp->n = new_n;
  counts[0] = n_clone;
  counts[1] = 2 * n_split;
  counts[2] = n_split;
  return SC_OK;
}

}  // namespace sck
