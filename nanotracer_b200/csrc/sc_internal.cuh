// sc_internal.cuh — shared definitions of libsplatcuda (sm_100a).
//
// Device layout of the splat parameters ("slab", coefficient-major SoA):
//   row r of the 59 parameter rows lives at slab[r * cap + i] for splat i,
//   rows 0-2 position, 3-6 rotation (w,x,y,z), 7-9 log-sigma, 10 opacity
//   logit, 11-13 SH DC, 14-58 SH rest (planar R[15] G[15] B[15]).
// Every per-splat read or write of a row is a coalesced 4-byte access across
// a warp, the gather/scatter of densify is row-wise, and Adam is one
// elementwise pass over the slab.  With SC_SPLATS_BF16_REST the 45 rest rows
// live in a separate bf16 slab (rest16[k * cap + i]).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <string>

#include "../../include/splat_cuda.h"

#define SC_NROWS 59
#define SC_ROW_POS 0
#define SC_ROW_ROT 3
#define SC_ROW_SCALE 7
#define SC_ROW_OP 10
#define SC_ROW_DC 11
#define SC_ROW_REST 14
#define SC_MAX_VIEWS 64

// device error word bits
#define SC_DEVERR_TIMEOUT 1u
#define SC_DEVERR_CAPACITY 2u

// bounded spin limit for decoupled look-back waits (iterations of a poll loop
// with a nanosleep back-off; ~1 s worst case before giving up)
#define SC_SPIN_LIMIT (1u << 22)

struct sc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  std::string last_error;
  uint32_t* d_error = nullptr;    // device error word
  uint64_t* d_counters = nullptr; // scratch counters (tile ids, totals)
  uint32_t* h_error = nullptr;    // pinned mirror
  uint64_t launches = 0;
  // sc_ctx_set_fp64_det: near-degenerate splats get an FP64 determinant and
  // inverse in sc_project and sc_project_backward
  int fp64_det = 0;
  // grow-only scratch arena for temporaries of the reference-shaped calls
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
};

struct sc_splats {
  uint32_t n = 0, cap = 0, flags = 0;
  float* slab = nullptr;            // 14 or 59 rows x cap
  __nv_bfloat16* rest16 = nullptr;  // 45 rows x cap when bf16
};

struct sc_grads {
  uint32_t cap = 0;
  float* slab = nullptr;  // 59 rows x cap
};

struct sc_moments {
  uint32_t cap = 0, flags = 0;
  float* m = nullptr; float* v = nullptr;                  // fp32: 59 rows x cap
  __nv_bfloat16* m16 = nullptr; __nv_bfloat16* v16 = nullptr;  // bf16 form
};

// ---------------------------------------------------------------- views
struct DSplats {
  float* slab;
  __nv_bfloat16* rest16;
  uint32_t n, cap, bf16;
};

struct DMoments {
  float* m; float* v;
  __nv_bfloat16* m16; __nv_bfloat16* v16;
  uint32_t cap, bf16;
};

// One scene of a many-scene step (one view per scene): its parameter store,
// Adam state, densify statistic and gradient rows, its image size inside the
// step's common tile grid, and its MSE gradient scale 2 / (3 W H).
struct SceneDev {
  DSplats s;
  DMoments mo;
  float* acc;
  float* grads;  // SC_NROWS rows x gstride
  uint32_t gstride;
  uint32_t width, height;
  float gscale;
};

static inline DSplats dview(const sc_splats* s) {
  return DSplats{s->slab, s->rest16, s->n, s->cap, (s->flags & SC_SPLATS_BF16_REST) ? 1u : 0u};
}
static inline DMoments dview(const sc_moments* m) {
  return DMoments{m->m, m->v, m->m16, m->v16, m->cap, (m->flags & SC_MOMENTS_BF16) ? 1u : 0u};
}

__device__ __forceinline__ float sp_row(const DSplats& s, int r, uint32_t i) {
  if (r >= SC_ROW_REST && s.bf16) return __bfloat162float(s.rest16[(size_t)(r - SC_ROW_REST) * s.cap + i]);
  return s.slab[(size_t)r * s.cap + i];
}
__device__ __forceinline__ void sp_set(const DSplats& s, int r, uint32_t i, float v) {
  if (r >= SC_ROW_REST && s.bf16) { s.rest16[(size_t)(r - SC_ROW_REST) * s.cap + i] = __float2bfloat16_rn(v); return; }
  s.slab[(size_t)r * s.cap + i] = v;
}

// ---------------------------------------------------------------- tile culling
// A pixel reaches alpha = op exp(-q/2) >= 1/255 only inside the ellipse
// q(u, w) = a u^2 + 2 b u w + c w^2 <= L, L = 2 ln(255 op) (u, w: offsets from
// the mean, (a, b, c) the conic).  For a tile row (pixel-centre band
// w in [w0, w1]) the ellipse covers u in [u_min(w), u_max(w)] with
// u_max(w) = (-b w + sqrt(L a - det w^2)) / a concave and u_min convex, so
// their extremes over the band sit at the clamped extreme points of the
// ellipse (w = -/+ b xh / c, xh the half-width).  A tile whose pixel centres
// miss that interval holds no pixel the blend would accept, so the pair can be
// dropped without changing any image.  L is widened by 1e-3 relative + 1e-3
// and the interval by 1e-3 px, so float rounding in the blend can never
// accept a pixel this test rejects; the same margins cover the SFU
// approximations used here (relative errors near 1e-7, i.e. below 1e-5 px).
// Counting (projection) and emission call the same functions, so they agree.
__device__ __forceinline__ float cull_sqrt(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
struct CullShape {
  float mx, my, a, b, det, L, xh, yh, kx, inv_a;
  bool any;   // op > 1/255 and the conic is positive definite
  bool keep;  // not positive definite: keep the reference rectangle whole
};

__device__ __forceinline__ CullShape cull_shape(float mx, float my, float a, float b, float c, float op) {
  CullShape s;
  s.mx = mx; s.my = my; s.a = a; s.b = b;
  s.det = a * c - b * b;
  // An ill-conditioned conic (a needle-like splat: the determinant keeps less
  // than 2^-10 of a c) has lost too many bits to cancellation here for the
  // margins below, and the blend's own evaluation of the quadratic form is
  // noisy along the needle: such a splat keeps its whole rectangle.
  s.keep = !(a > 0.0f && c > 0.0f && s.det > 9.765625e-4f * a * c);
  s.any = op * 255.0f > 1.0f;
  const float q = 2.0f * __logf(fmaxf(op * 255.0f, 1.0f));
  s.L = q + 1e-3f * q + 1e-3f;
  s.xh = cull_sqrt(__fdividef(s.L * c, s.det));
  s.yh = cull_sqrt(__fdividef(s.L * a, s.det));
  s.kx = __fdividef(b * s.xh, c);
  s.inv_a = __fdividef(1.0f, a);
  return s;
}

// Tiles [tlo, thi] of row ty (tile width tw, height th) that the ellipse can
// reach; false when the row misses it.  Caller clamps to the 3-sigma rectangle.
__device__ __forceinline__ bool cull_row_span(const CullShape& s, int ty, uint32_t tw, uint32_t th, int& tlo,
                                              int& thi) {
  const float w0 = (float)(ty * (int)th) + 0.5f - s.my, w1 = (float)((ty + 1) * (int)th) - 0.5f - s.my;
  if (w1 < -s.yh || w0 > s.yh) return false;
  const float a0 = fmaxf(w0, -s.yh), a1 = fminf(w1, s.yh);
  const float wr = fminf(fmaxf(-s.kx, a0), a1), wl = fminf(fmaxf(s.kx, a0), a1);
  const float ur = (-s.b * wr + cull_sqrt(fmaxf(s.L * s.a - wr * wr * s.det, 0.0f))) * s.inv_a;
  const float ul = (-s.b * wl - cull_sqrt(fmaxf(s.L * s.a - wl * wl * s.det, 0.0f))) * s.inv_a;
  const float X0 = s.mx + ul - 1e-3f, X1 = s.mx + ur + 1e-3f;
  // tile tx's pixel centres span [tx*tw + 0.5, (tx+1)*tw - 0.5]
  const float inv_tw = __fdividef(1.0f, (float)tw);  // the 1e-3 px margin covers its rounding
  tlo = (int)ceilf((X0 + 0.5f) * inv_tw - 1.0f);
  thi = (int)floorf((X1 - 0.5f) * inv_tw);
  return thi >= tlo;
}

// Tiles [lo, hi] of row ty that a splat with 3-sigma tile rectangle
// [x0, x1] x [y0, y1] emits pairs for: the whole rectangle row, or with
// culling (test = culling on and the conic positive definite) the clamped
// cull_row_span.  false: the row emits nothing.  Counting, emission and the
// two-level binning all decide membership through this one function.
__device__ __forceinline__ bool splat_row_span(const CullShape& cs, bool test, int ty, int x0, int x1, uint32_t tw,
                                               uint32_t th, int& lo, int& hi) {
  lo = x0;
  hi = x1;
  if (test) {
    if (!cs.any || !cull_row_span(cs, ty, tw, th, lo, hi)) return false;
    lo = max(lo, x0);
    hi = min(hi, x1);
  }
  return hi >= lo;
}

// Two-level binning: super tiles of SC_SUPER x SC_SUPER tiles.
#define SC_SUPER 4

// The super columns [sx0, sx1] a splat emits items for in super row sy: the
// tiles that the ellipse can reach anywhere in the pixel-centre band from the
// first to the last of the super row's tile rows inside the splat's 3-sigma
// rectangle [x0, x1] x [y0, y1] (with culling; the rectangle's columns
// without).  One band instead of SC_SUPER tile rows: u_min is convex and u_max
// concave in w, so over the band their extremes sit at the clamped extreme
// points, two square roots per super row.  The band holds every tile row's
// band and the interval is widened by 1e-2 px (the tile rows' test uses
// 1e-3), so the hull holds every tile-row span that cull_row_span gives for
// the same rows, whatever the rounding: the member masks, taken from the tile
// rows, never reach outside it.  Counting (projection) and emission both call
// this, so they agree on the item count.
__device__ __forceinline__ bool super_row_hull(const CullShape& s, bool test, int sy, int x0, int y0, int x1, int y1,
                                               uint32_t tw, uint32_t th, int& sx0, int& sx1) {
  const int ty0 = max(sy * SC_SUPER, y0), ty1 = min(sy * SC_SUPER + SC_SUPER - 1, y1);
  if (ty1 < ty0) return false;
  int lo = x0, hi = x1;
  if (test) {
    if (!s.any) return false;
    const float w0 = (float)(ty0 * (int)th) + 0.5f - s.my, w1 = (float)((ty1 + 1) * (int)th) - 0.5f - s.my;
    if (w1 < -s.yh || w0 > s.yh) return false;
    const float a0 = fmaxf(w0, -s.yh), a1 = fminf(w1, s.yh);
    const float wr = fminf(fmaxf(-s.kx, a0), a1), wl = fminf(fmaxf(s.kx, a0), a1);
    const float ur = (-s.b * wr + cull_sqrt(fmaxf(s.L * s.a - wr * wr * s.det, 0.0f))) * s.inv_a;
    const float ul = (-s.b * wl - cull_sqrt(fmaxf(s.L * s.a - wl * wl * s.det, 0.0f))) * s.inv_a;
    const float X0 = s.mx + ul - 1e-2f, X1 = s.mx + ur + 1e-2f;
    const float inv_tw = __fdividef(1.0f, (float)tw);
    lo = max(lo, (int)ceilf((X0 + 0.5f) * inv_tw - 1.0f));
    hi = min(hi, (int)floorf((X1 - 0.5f) * inv_tw));
    if (hi < lo) return false;
  }
  sx0 = lo / SC_SUPER;
  sx1 = hi / SC_SUPER;
  return true;
}

// A splat's items, super row by super row: f gets the super row, the hull's
// super columns (super_row_hull) and the spans of the super row's tile rows
// (row c of the super row: tiles [lo[c], hi[c]], empty when lo > hi), from
// which each item's member mask is formed.
template <typename F>
__device__ __forceinline__ void for_each_super_span(const CullShape& cs, bool test, int x0, int y0, int x1, int y1,
                                                    uint32_t tw, uint32_t th, F&& f) {
  for (int sy = y0 / SC_SUPER; sy <= y1 / SC_SUPER; ++sy) {
    int sx0, sx1;
    if (!super_row_hull(cs, test, sy, x0, y0, x1, y1, tw, th, sx0, sx1)) continue;
    int rlo[SC_SUPER], rhi[SC_SUPER];
#pragma unroll
    for (int c = 0; c < SC_SUPER; ++c) {
      rlo[c] = 1;
      rhi[c] = 0;
      const int ty = sy * SC_SUPER + c;
      int lo, hi;
      if (ty >= y0 && ty <= y1 && splat_row_span(cs, test, ty, x0, x1, tw, th, lo, hi)) {
        rlo[c] = lo;
        rhi[c] = hi;
      }
    }
    f(sy, sx0, sx1, rlo, rhi);
  }
}

// member tiles of super column sx given the row spans: bit c * SC_SUPER + q
// for tile (sx * SC_SUPER + q, row c)
__device__ __forceinline__ uint32_t super_mask_of(int sx, const int* rlo, const int* rhi) {
  // row c's tiles [rlo, rhi] (empty when rlo > rhi) cover columns [lo, hi] of
  // super column sx: bits lo..hi of the row's nibble
  uint32_t m = 0;
  const int base = sx * SC_SUPER;
#pragma unroll
  for (int c = 0; c < SC_SUPER; ++c) {
    const int lo = max(rlo[c] - base, 0), hi = min(rhi[c] - base, SC_SUPER - 1);
    if (hi >= lo) m |= ((2u << hi) - (1u << lo)) << (c * SC_SUPER);
  }
  return m;
}

// ---------------------------------------------------------------- host helpers
sc_status sc_fail(sc_ctx* ctx, sc_status st, const std::string& msg);
sc_status sc_cuda_fail(sc_ctx* ctx, cudaError_t e, const char* what);
sc_status sc_check_launch(sc_ctx* ctx, const char* what);
// scratch arena: returns a device pointer to at least `bytes` (reused across calls
// on the same stream; contents undefined)
sc_status sc_scratch(sc_ctx* ctx, size_t bytes, void** out);
// read-and-clear the device error word (blocks)
sc_status sc_check_device_error(sc_ctx* ctx);

#define SC_TRY(expr)                      \
  do {                                    \
    sc_status _st = (expr);               \
    if (_st != SC_OK) return _st;         \
  } while (0)

#define SC_CUDA_TRY(ctx, expr, what)                      \
  do {                                                    \
    cudaError_t _e = (expr);                              \
    if (_e != cudaSuccess) return sc_cuda_fail(ctx, _e, what); \
  } while (0)

static inline uint64_t sc_div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------- kernel entry points
// (defined in the k_*.cu files, launched by the API layer)
namespace sck {

// projection: writes n_views*stride records; when depth_keys != nullptr also
// writes per (view, splat) a depth sort key (float bits, 0xFFFFFFFF when the
// splat emits no pairs; one segment of stride keys per view) and a count for
// the native pipeline: (tile, splat) pairs, or with bit 1 of `cull` two-level
// binning items.  Bit 0 of `cull`: exact tile culling.  zero_grad (nullable):
// per-(view, splat) gradient records of the same layout set to zero.
// scenes (nullable, n_views entries): view v projects scene v's own store
// (its first scene.s.n splats; the rest of the view's stride is culled).
sc_status launch_project(sc_ctx* ctx, const DSplats& s, const sc_camera* d_cams, uint32_t n_views,
                         uint32_t stride, float4* rec, const sc_tiling* tiling, uint32_t* depth_keys,
                         uint32_t* splat_ids, uint32_t* counts, int precise_det, int cull,
                         float4* zero_grad = nullptr, float4* zero_comp = nullptr,
                         const SceneDev* scenes = nullptr);

sc_status launch_project_backward(sc_ctx* ctx, const DSplats& s, const float4* proj_grad, const sc_camera* d_cam,
                                  float* grads, uint32_t gcap, int accumulate, int precise_det);

// Adam hyper-parameters, clamp limits and bias corrections of one step
struct AdamParams {
  float lr[6];
  float beta1, beta2, eps, bc1, bc2;
  float log_scale_min, log_scale_max, opacity_logit_max;
  uint32_t seed = 0;  // the step number: seeds the stochastic rounding of BF16 parameters
};

// BF16 parameters are written back with stochastic rounding.  An Adam step is
// about lr (1.25e-4 for the SH-rest group) while a BF16 ulp at the SH-rest
// coefficients' scale (~0.05) is 2.4e-4, so round-to-nearest would discard
// most updates; adding uniform bits below the BF16 mantissa before truncating
// rounds up or down with probabilities proportional to the distance, so the
// stored value equals the f32 update in expectation.  The bits come from a
// hash of (step, row, splat index): deterministic, and the same on every rank
// of the data-parallel path, which updates a splat with its global index.
__device__ __forceinline__ uint32_t sr_hash(uint32_t x) {
  // integer finaliser of Wellons' "lowbias32" (two xorshift-multiply rounds)
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t sr_bits(uint32_t seed, int row, uint32_t i) {
  return sr_hash(i * 0x9E3779B1u ^ sr_hash(seed * 0x85EBCA77u + (uint32_t)row));
}
__device__ __forceinline__ __nv_bfloat16 bf16_stochastic(float x, uint32_t rnd) {
  uint32_t b = __float_as_uint(x);
  // finite values: add 16 random bits to the magnitude below the kept 16 (the
  // sign bit is untouched, so negative values round symmetrically); Inf and NaN
  // pass through by truncation
  if ((b & 0x7F800000u) != 0x7F800000u) b += rnd & 0xFFFFu;
  return __ushort_as_bfloat16((unsigned short)(b >> 16));
}
// sp_set with stochastic rounding of BF16 rows
__device__ __forceinline__ void sp_set_sr(const DSplats& s, int r, uint32_t i, float v, uint32_t seed) {
  if (r >= SC_ROW_REST && s.bf16) {
    s.rest16[(size_t)(r - SC_ROW_REST) * s.cap + i] = bf16_stochastic(v, sr_bits(seed, r, i));
    return;
  }
  s.slab[(size_t)r * s.cap + i] = v;
}

// moments widened to / rounded from f32
__device__ __forceinline__ float mo_ld(const DMoments& mo, const float* f, const __nv_bfloat16* h, size_t k) {
  return mo.bf16 ? __bfloat162float(h[k]) : f[k];
}
__device__ __forceinline__ void mo_st(const DMoments& mo, float* f, __nv_bfloat16* h, size_t k, float x) {
  if (mo.bf16) h[k] = __float2bfloat16_rn(x); else f[k] = x;
}
// learning-rate group of parameter row r: pos, rot, scale, opacity, sh_dc, sh_rest
__device__ __forceinline__ int adam_group(int r) {
  return r < 3 ? 0 : (r < 7 ? 1 : (r < 10 ? 2 : (r < 11 ? 3 : (r < 14 ? 4 : 5))));
}
// Adam on one scalar (adam_step.wgsl:24-36), moments at flat index k
__device__ __forceinline__ float adam_scalar(const DMoments& mo, size_t k, float p, float gr, float lr,
                                             const AdamParams& ap) {
  const float m = ap.beta1 * mo_ld(mo, mo.m, mo.m16, k) + (1.0f - ap.beta1) * gr;
  const float v = ap.beta2 * mo_ld(mo, mo.v, mo.v16, k) + (1.0f - ap.beta2) * gr * gr;
  mo_st(mo, mo.m, mo.m16, k, m);
  mo_st(mo, mo.v, mo.v16, k, v);
  const float mh = m / ap.bc1, vh = v / ap.bc2;
  return p - lr * mh / (sqrtf(vh) + ap.eps);
}
// The same update with the bias corrections folded into per-group constants,
// a = lr / bc1 and s2 = 1 / sqrt(bc2): lr (m / bc1) / (sqrt(v / bc2) + eps)
// = a m / (sqrt(v) s2 + eps), with SFU reciprocals (a few ulp of the update,
// far below the parameters' own rounding).
struct AdamFast { float a[6]; float s2; };
__device__ __forceinline__ AdamFast adam_fast(const AdamParams& ap) {
  AdamFast f;
#pragma unroll
  for (int k = 0; k < 6; ++k) f.a[k] = __fdividef(ap.lr[k], ap.bc1);
  f.s2 = rsqrtf(ap.bc2);
  return f;
}
__device__ __forceinline__ float adam_scalar_fast(const DMoments& mo, size_t k, float p, float gr, float a, float s2,
                                                  const AdamParams& ap) {
  const float m = ap.beta1 * mo_ld(mo, mo.m, mo.m16, k) + (1.0f - ap.beta1) * gr;
  const float v = ap.beta2 * mo_ld(mo, mo.v, mo.v16, k) + (1.0f - ap.beta2) * gr * gr;
  mo_st(mo, mo.m, mo.m16, k, m);
  mo_st(mo, mo.v, mo.v16, k, v);
  return p - __fdividef(a * m, fmaf(sqrtf(v), s2, ap.eps));
}
// constraints on the updated geometric rows 0..13 (apply_constraints.wgsl:24-41)
__device__ __forceinline__ void constrain_geometry(float np[14], const AdamParams& ap) {
  const float n2 = np[3] * np[3] + np[4] * np[4] + np[5] * np[5] + np[6] * np[6];
  const float nrm = fmaxf(sqrtf(n2), 1e-8f);
  np[3] /= nrm; np[4] /= nrm; np[5] /= nrm; np[6] /= nrm;
  for (int k = 7; k < 10; ++k) np[k] = fminf(fmaxf(np[k], ap.log_scale_min), ap.log_scale_max);
  np[10] = fminf(fmaxf(np[10], -ap.opacity_logit_max), ap.opacity_logit_max);
}

// ---- many scenes in one step (one view per scene), each with its own store
// gradient rows of every scene from its view's records (grid.y = scene)
sc_status launch_project_backward_scenes(sc_ctx* ctx, const SceneDev* d_scenes, uint32_t n_scenes,
                                         uint32_t max_gstride, const float4* proj_grad, uint32_t stride,
                                         const sc_camera* d_cams, const uint32_t* d_skip, int precise_det,
                                         const float4* proj_comp);
// Adam + constraints + densify statistic of every scene's splats (grid.z = scene;
// gstride and the stores' capacities multiples of 8)
sc_status launch_adam_rows_scenes(sc_ctx* ctx, const SceneDev* d_scenes, uint32_t n_scenes, uint32_t max_count,
                                  const AdamParams& ap, const float* d_bc, const uint32_t* d_skip);

// ---- data-parallel views (one iteration split across ranks by views)
// Shard-major gradient layout: element (row r, splat i) of a buffer cut into
// chunks of `shard` splats sits at ((i / shard) * SC_NROWS + r) * shard + i % shard.
// Per-splat gradient summed over this rank's views, written shard-major; rows
// of splats in [n, n_shards*shard) are zero.
sc_status launch_project_backward_shards(sc_ctx* ctx, const DSplats& s, const float4* proj_grad, uint32_t stride,
                                         const sc_camera* d_cams, uint32_t n_views, float* grads, uint32_t n_shards,
                                         uint32_t shard, const uint32_t* d_skip_flag, int precise_det,
                                         const float4* proj_comp = nullptr);
// Adam + constraints + densify statistic for splats [lo, lo+count) from one
// reduce-scattered chunk g[r * shard + j]
// Adam + constraints + densify statistic over splats [lo, lo+count) from
// gradient rows g[r * gstride + j] (lo, gstride multiples of 8), streaming
// 8 splats of one row group per thread; bias corrections from d_bc when given
sc_status launch_adam_rows(sc_ctx* ctx, const DSplats& s, const DMoments& mo, float* grad_acc, const float* g,
                           uint32_t lo, uint32_t count, uint32_t gstride, const AdamParams& ap, const float* d_bc,
                           const uint32_t* d_skip_flag);
sc_status launch_adam_shard(sc_ctx* ctx, const DSplats& s, const DMoments& mo, float* grad_acc, const float* g,
                            uint32_t lo, uint32_t count, uint32_t shard, const AdamParams& ap);
// parameters / moments of [lo, lo+count) as f32 rows out[r * shard + j], and back
sc_status launch_pack_params(sc_ctx* ctx, const DSplats& s, uint32_t lo, uint32_t count, uint32_t shard, float* out);
sc_status launch_unpack_params(sc_ctx* ctx, const DSplats& s, const float* in, uint32_t n_shards, uint32_t shard);
sc_status launch_pack_moments(sc_ctx* ctx, const DMoments& mo, uint32_t lo, uint32_t count, uint32_t shard, float* out);
sc_status launch_unpack_moments(sc_ctx* ctx, const DMoments& mo, uint32_t n, const float* in, uint32_t n_shards,
                                uint32_t shard);

// scan / sort
sc_status scan_u32(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* d_total, void* scratch, size_t scratch_bytes);
// the same exclusive scan of out[0..n), out[i] = src[(i / seg) seg + idx[i]]
// for i < gn and 0 beyond (seg a multiple of 16), gathered as it is read
sc_status scan_u32_gather(sc_ctx* ctx, uint32_t* out, uint64_t n, const uint32_t* src, const uint32_t* idx,
                          uint32_t seg, uint64_t gn, uint64_t* d_total, void* scratch, size_t scratch_bytes);
size_t scan_scratch_bytes(uint64_t n);
template <typename K>
sc_status radix_sort(sc_ctx* ctx, K* keys, uint32_t* vals, K* keys_tmp, uint32_t* vals_tmp, uint64_t n,
                     uint32_t key_bits, const uint64_t* d_n, void* scratch, size_t scratch_bytes, bool* result_in_tmp,
                     int digit_bits = 0);
size_t radix_scratch_bytes(uint64_t n, uint32_t key_bytes);
// n_segs independent stable sorts of u32 keys, segment g = elements
// [g seg_len, (g + 1) seg_len); seg_len a multiple of RADIX_SEG_TILE
constexpr uint32_t RADIX_SEG_TILE = 4096;
sc_status radix_sort_segments(sc_ctx* ctx, uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                              uint32_t seg_len, uint32_t n_segs, uint32_t key_bits, void* scratch, size_t bytes,
                              bool* result_in_tmp);
size_t radix_seg_scratch_bytes(uint64_t seg_len, uint32_t n_segs);
// one look-back pass whose predecessor never publishes (bounded-wait self-test)
sc_status selftest_lookback_timeout(sc_ctx* ctx);

// binning
sc_status launch_tile_count(sc_ctx* ctx, const float4* rec, uint32_t n, uint32_t stride, uint32_t n_views,
                            const sc_tiling* tl, uint32_t* counts);
sc_status launch_tile_emit(sc_ctx* ctx, const float4* rec, uint32_t n, uint32_t stride, uint32_t n_views,
                           const sc_tiling* tl, const uint32_t* offsets, int key_mode, void* keys,
                           uint32_t* payloads, uint64_t cap);
// key_mode 2: presorted keys (view << tile_bits) | tile, tiles_per_view tiles
// per view; only the low key_bits bits of a key take part (the rest is payload,
// whose set bits are added to *high_popc when it is given)
sc_status launch_tile_ranges(sc_ctx* ctx, const void* keys, int key_mode, const uint64_t* d_total, uint64_t cap,
                             uint32_t num_tiles, uint32_t* ranges, uint32_t tiles_per_view = 0,
                             uint32_t tile_bits = 0, uint32_t key_bits = 32, uint64_t* high_popc = nullptr);
// depth-presorted emission for the native pipeline
sc_status launch_presorted_emit(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                const uint32_t* sorted_ids, const uint32_t* offsets, const uint32_t* counts_by_id,
                                const sc_tiling* tl, uint32_t* keys, uint32_t* payloads, uint64_t cap,
                                uint32_t* d_error, int cull);
// two-level binning (super tiles of SC_SUPER x SC_SUPER tiles):
// items (member mask << 16 | view << super_bits | super tile, splat) in depth
// order; bit (c * SC_SUPER + q) of the mask is tile (q, c) of the super tile.
// view << super_bits | super tile must fit in 16 bits.
sc_status launch_super_emit(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                            const uint32_t* sorted_ids, const uint32_t* offsets, const uint32_t* counts_by_id,
                            const sc_tiling* tl, uint32_t* keys, uint32_t* payloads, uint64_t cap, uint32_t* d_error,
                            int cull);
uint32_t super_tiles_per_view(const sc_tiling* tl);

// blending
sc_status launch_composite(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                           const uint32_t* payloads, const uint32_t* ranges, const sc_tiling* tl, float4* image,
                           uint2* aux, const float* target, float mse_scale, float4* dl_dc, double* loss,
                           const uint32_t* d_skip);
sc_status launch_mse(sc_ctx* ctx, const float4* pred, const float* target, uint64_t pixels_per_view,
                     uint32_t n_views, float scale, float4* dl_dc, double* loss);
// with a target, dL/dC of the MSE (mse_scale as in launch_composite) and its
// loss are formed from the image fwd instead of being read from dl_dc
sc_status launch_composite_backward(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                    const uint32_t* payloads, const uint32_t* ranges, const sc_tiling* tl,
                                    const float4* fwd, const float4* dl_dc, int mode, const uint2* aux,
                                    float4* proj_grad, const uint32_t* d_skip, const float* target = nullptr,
                                    float mse_scale = 0.0f, double* loss = nullptr, float4* proj_comp = nullptr);
// proj_comp (nullable, same layout as proj_grad, zeroed by the caller): the
// per-(view, splat) totals across tiles are then TwoSum-compensated atomic sums,
// their rounding errors accumulated in proj_comp (the total is grad + comp)
sc_status launch_fold_comp(sc_ctx* ctx, float4* proj_grad, const float4* proj_comp, uint64_t n_float4);
// the same two passes over super-tile item lists (launch_super_emit's items
// sorted by super tile, item_ranges per (view, super tile)): each tile blends
// the items whose member mask holds it, in list order; aux then holds
// positions within the super tile's list.  batch: list positions staged per
// batch (0 = one per thread).  scenes (nullable): view v's pixels are those
// inside scene v's width x height (the images keep the tiling's row pitch) and
// its MSE scale is the scene's.  work (nullable, 3 BLEND_WORK_SLOTS u64,
// accumulated): BLEND_WORK_SLOTS (scanned, staged) pairs — the list positions
// the CTAs' batches covered and the entries they staged — then, with
// count_pairs, as many counts of contributing (pixel, entry) pairs.
constexpr uint32_t BLEND_WORK_SLOTS = 64;
sc_status launch_composite_items(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                 const uint32_t* item_keys, const uint32_t* item_ids, const uint32_t* item_ranges,
                                 const sc_tiling* tl, float4* image, uint2* aux, const float* target, float mse_scale,
                                 float4* dl_dc, double* loss, const uint32_t* d_skip, uint64_t* work = nullptr,
                                 uint32_t batch = 0, const SceneDev* scenes = nullptr, bool count_pairs = false);
sc_status launch_composite_backward_items(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                          const uint32_t* item_keys, const uint32_t* item_ids,
                                          const uint32_t* item_ranges, const sc_tiling* tl, const float4* fwd,
                                          const float4* dl_dc, int mode, const uint2* aux, float4* proj_grad,
                                          const uint32_t* d_skip, const float* target = nullptr,
                                          float mse_scale = 0.0f, double* loss = nullptr, uint64_t* work = nullptr,
                                          float4* proj_comp = nullptr, uint32_t batch = 0,
                                          const SceneDev* scenes = nullptr, bool count_pairs = false);
sc_status launch_tonemap(sc_ctx* ctx, const float4* img, uint32_t w, uint32_t h, uint8_t* out);

// SSIM (loss.rs:22-375): scale * dL_ssim/dC added into dl_dc, per-view sum of
// the SSIM map added into ssim_sum; terms = ssim_terms_bytes() of scratch
void ssim_window(float g[11]);
size_t ssim_terms_bytes(uint64_t pixels_per_view, uint32_t n_views);
sc_status launch_ssim(sc_ctx* ctx, const float4* pred, const float* target, uint32_t w, uint32_t h, uint32_t n_views,
                      float scale, float4* dl_dc, double* ssim_sum, float* terms);
// per view {total, mse, ssim} from the squared-error sums and SSIM-map sums (loss.rs:383-410)
sc_status launch_loss_parts(sc_ctx* ctx, const double* mse, const double* ssim_sum, uint32_t n_views, uint64_t P,
                            float lambda, double* out);

// optimiser
sc_status launch_adam_lanes(sc_ctx* ctx, float* p, const float* g, float* m, float* v, uint64_t n, float lr,
                            float b1, float b2, float eps, float bc1, float bc2);
sc_status launch_adam_all(sc_ctx* ctx, const DSplats& s, const float* g, uint32_t gcap, const DMoments& mo,
                          const AdamParams& ap);
sc_status launch_constraints(sc_ctx* ctx, const DSplats& s, float lsmin, float lsmax, float opmax);
sc_status launch_accumulate(sc_ctx* ctx, const float* g, uint32_t gcap, float* acc, uint32_t n);

// densify / prune (compaction through a source map)
sc_status prune(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* acc, float thr, uint32_t* removed);
sc_status densify(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* acc, uint32_t grad_count, float gthr,
                  float sthr, uint32_t max_splats, uint32_t iter, uint32_t counts[3]);

}  // namespace sck

// host-side f32 x^t by square-and-multiply (the algorithm behind f32::powi,
// used for Adam's bias corrections, adam_gpu.rs:275-276)
static inline float sc_powi_f32(float a, int b) {
  const bool recip = b < 0;
  float r = 1.0f;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0f / r : r;
}
