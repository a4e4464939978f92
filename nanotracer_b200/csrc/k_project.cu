// k_project.cu — per-splat projection (forward) and its adjoint.
//
// Forward: the arithmetic of project_gaussians.wgsl:156-259 (pinhole, RH view,
// Sigma2D + 0.3 I low-pass, 3-sigma radius, frustum cull, order-3 SH,
// sigmoid opacity).  The 2D covariance is formed as B B^T with
// B = J W R diag(sigma) (2x3), which is algebraically the reference's
// J (W R S^2 R^T W^T) J^T with fewer operations.  One thread per (splat,
// view), consecutive CTAs taking the views of one 128-splat chunk: 64
// registers instead of the 128 of a thread looping over the views, and a
// splat's parameters are read from L2 by its views after the first (0.56 ms
// at 1M splats and 8 views; 0.62 ms with the views on the grid's slow axis,
// each view streaming the parameters from DRAM).  Each CTA stages its chunk's
// parameter rows in shared memory with cp.async, all copies in flight at once,
// and counts a splat's items with one band hull per super row (0.355 ms).
//
// Backward: project_backward.wgsl:79-304, with the same omissions as the
// reference (no dJ/dt in the position gradient, no SH view-direction
// gradient, no colour-clamp gate).  With the FP64 determinant option the
// adjoint recomputes the same FP64 conic as the forward, so dSigma2D =
// -C dConic C differentiates the conic the blend used.  One thread per splat
// sums the per-view gradients (geometric sums in registers, the 45 SH-rest
// sums in a shared-memory column) and writes the splat's 59 gradient rows once
// (coefficient-major, cut into shards for the data-parallel path); Adam then
// streams over those rows (k_adam.cu).  A single kernel doing both held 59
// gradients and the Adam state of one splat per thread at 128 registers and
// waited on memory; the split moves 2 x 236 bytes more per splat and ran the
// pair in 0.49 ms instead of 0.83 ms at 1M splats and 8 views.
#include "sc_internal.cuh"

namespace sck {

// SH constants, project_gaussians.wgsl:47-61
#define SH_C0 0.2820948f
#define SH_C1 0.488602f
#define SH_C2_0 1.0925485f
#define SH_C2_1 -1.0925485f
#define SH_C2_2 0.31539157f
#define SH_C2_3 -1.0925485f
#define SH_C2_4 0.54627424f
#define SH_C3_0 -0.5900436f
#define SH_C3_1 2.8906114f
#define SH_C3_2 -0.4570458f
#define SH_C3_3 0.37317634f
#define SH_C3_4 -0.4570458f
#define SH_C3_5 1.4453057f
#define SH_C3_6 -0.5900436f

struct Cam {
  float v[16];
  float cp[3];
  float near_plane, focal, width, height;
};

__device__ __forceinline__ Cam load_cam(const sc_camera* c) {
  Cam k;
  const float4* p = reinterpret_cast<const float4*>(c);
  float4 a = __ldg(p + 0), b = __ldg(p + 1), cc = __ldg(p + 2), d = __ldg(p + 3), e = __ldg(p + 4), f = __ldg(p + 5);
  k.v[0] = a.x; k.v[1] = a.y; k.v[2] = a.z; k.v[3] = a.w;
  k.v[4] = b.x; k.v[5] = b.y; k.v[6] = b.z; k.v[7] = b.w;
  k.v[8] = cc.x; k.v[9] = cc.y; k.v[10] = cc.z; k.v[11] = cc.w;
  k.v[12] = d.x; k.v[13] = d.y; k.v[14] = d.z; k.v[15] = d.w;
  k.cp[0] = e.x; k.cp[1] = e.y; k.cp[2] = e.z; k.near_plane = e.w;
  k.focal = f.x; k.width = f.y; k.height = f.z;
  return k;
}

__device__ __forceinline__ void sh_basis15(float x, float y, float z, float b[15]) {
  const float xx = x * x, yy = y * y, zz = z * z;
  b[0] = -SH_C1 * y; b[1] = SH_C1 * z; b[2] = -SH_C1 * x;
  b[3] = SH_C2_0 * x * y;
  b[4] = SH_C2_1 * y * z;
  b[5] = SH_C2_2 * (2.0f * zz - xx - yy);
  b[6] = SH_C2_3 * x * z;
  b[7] = SH_C2_4 * (xx - yy);
  b[8] = SH_C3_0 * y * (3.0f * xx - yy);
  b[9] = SH_C3_1 * x * y * z;
  b[10] = SH_C3_2 * y * (4.0f * zz - xx - yy);
  b[11] = SH_C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
  b[12] = SH_C3_4 * x * (4.0f * zz - xx - yy);
  b[13] = SH_C3_5 * z * (xx - yy);
  b[14] = SH_C3_6 * x * (xx - 3.0f * yy);
}

// rotation matrix (row r, column c) of quaternion (w, x, y, z), project_gaussians.wgsl:68-80
// In the IEEE geometry (X = true: the forward and sc_project_backward) every
// rounding step of the rotation and of geometry() below is written out
// (__fmaf_rn / __fmul_rn / __fadd_rn), so the compiler has no contraction left
// to choose and the two form bit-identical covariances: they agree on which
// needle-like splats the f32 determinant test culls.  The trainer's adjoint
// (X = false) leaves the contraction to the compiler.
template <bool X> __device__ __forceinline__ float mul_(float a, float b) { return X ? __fmul_rn(a, b) : a * b; }
template <bool X> __device__ __forceinline__ float fma_(float a, float b, float c) {
  return X ? __fmaf_rn(a, b, c) : a * b + c;
}
template <bool X> __device__ __forceinline__ float sum_sq2(float a, float b) { return fma_<X>(a, a, mul_<X>(b, b)); }
template <bool X> __device__ __forceinline__ float dot2(float a, float b, float c, float d) {
  return fma_<X>(a, b, mul_<X>(c, d));
}
template <bool X>
__device__ __forceinline__ void quat_rot(float w, float x, float y, float z, float R[3][3]) {
  R[0][0] = fma_<X>(-2.0f, sum_sq2<X>(y, z), 1.0f); R[1][0] = mul_<X>(2.0f, dot2<X>(x, y, w, z));
  R[2][0] = mul_<X>(2.0f, dot2<X>(x, z, -w, y));
  R[0][1] = mul_<X>(2.0f, dot2<X>(x, y, -w, z)); R[1][1] = fma_<X>(-2.0f, sum_sq2<X>(x, z), 1.0f);
  R[2][1] = mul_<X>(2.0f, dot2<X>(y, z, w, x));
  R[0][2] = mul_<X>(2.0f, dot2<X>(x, z, w, y)); R[1][2] = mul_<X>(2.0f, dot2<X>(y, z, -w, x));
  R[2][2] = fma_<X>(-2.0f, sum_sq2<X>(x, y), 1.0f);
}

// Geometry shared by forward and backward for one (splat, view).
struct Geo {
  float tx, ty, tz;         // camera-space x, y and positive depth
  float R[3][3];            // rotation, R[row][col]
  float W[3][3];            // view rotation, W[row][col]
  float sig[3];             // exp(log-sigma)
  float j0[3], j1[3];       // projection Jacobian rows
  float s00, s01, s11, det; // dilated 2D covariance
  float ca, cb, cc;         // conic
};

// Division and exp for the geometry: IEEE-rounded in the forward (its radius
// and tile rectangle must match the reference's float arithmetic) and in
// sc_project_backward, the SFU approximations (a few ulp) in the trainer's
// adjoint, whose gradients are compared by tolerance.
template <bool FAST> __device__ __forceinline__ float gdiv(float a, float b) { return FAST ? __fdividef(a, b) : a / b; }
template <bool FAST> __device__ __forceinline__ float gexp(float a) { return FAST ? __expf(a) : expf(a); }

// returns false when culled by the near plane or a non-positive determinant
template <bool FAST>
__device__ __forceinline__ bool geometry(const Cam& c, float px, float py, float pz, float qw, float qx, float qy,
                                         float qz, float l0, float l1, float l2, int precise, Geo& g) {
  const float vx = fma_<!FAST>(c.v[8], pz, fma_<!FAST>(c.v[4], py, fma_<!FAST>(c.v[0], px, c.v[12])));
  const float vy = fma_<!FAST>(c.v[9], pz, fma_<!FAST>(c.v[5], py, fma_<!FAST>(c.v[1], px, c.v[13])));
  const float vz = fma_<!FAST>(c.v[10], pz, fma_<!FAST>(c.v[6], py, fma_<!FAST>(c.v[2], px, c.v[14])));
  const float vw = fma_<!FAST>(c.v[11], pz, fma_<!FAST>(c.v[7], py, fma_<!FAST>(c.v[3], px, c.v[15])));
  const float depth = -gdiv<FAST>(vz, vw);
  if (!(depth >= c.near_plane)) return false;
  g.tx = gdiv<FAST>(vx, vw); g.ty = gdiv<FAST>(vy, vw); g.tz = depth;
  quat_rot<!FAST>(qw, qx, qy, qz, g.R);
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) g.W[r][k] = c.v[4 * k + r];
  g.sig[0] = gexp<FAST>(l0); g.sig[1] = gexp<FAST>(l1); g.sig[2] = gexp<FAST>(l2);
  const float f = c.focal;
  const float iz = gdiv<FAST>(1.0f, g.tz), iz2 = mul_<!FAST>(iz, iz);
  g.j0[0] = mul_<!FAST>(f, iz); g.j0[1] = 0.0f; g.j0[2] = mul_<!FAST>(mul_<!FAST>(-f, g.tx), iz2);
  g.j1[0] = 0.0f; g.j1[1] = mul_<!FAST>(-f, iz); g.j1[2] = mul_<!FAST>(mul_<!FAST>(f, g.ty), iz2);
  // B = J W R S (2x3)
  float JW0[3], JW1[3];
  for (int k = 0; k < 3; ++k) {
    JW0[k] = dot2<!FAST>(g.j0[2], g.W[2][k], g.j0[0], g.W[0][k]);
    JW1[k] = dot2<!FAST>(g.j1[2], g.W[2][k], g.j1[1], g.W[1][k]);
  }
  float B0[3], B1[3];
  for (int k = 0; k < 3; ++k) {
    B0[k] = mul_<!FAST>(fma_<!FAST>(JW0[2], g.R[2][k], dot2<!FAST>(JW0[1], g.R[1][k], JW0[0], g.R[0][k])), g.sig[k]);
    B1[k] = mul_<!FAST>(fma_<!FAST>(JW1[2], g.R[2][k], dot2<!FAST>(JW1[1], g.R[1][k], JW1[0], g.R[0][k])), g.sig[k]);
  }
  const float a = fma_<!FAST>(B0[2], B0[2], dot2<!FAST>(B0[1], B0[1], B0[0], B0[0]));
  const float b = fma_<!FAST>(B0[2], B1[2], dot2<!FAST>(B0[1], B1[1], B0[0], B1[0]));
  const float d = fma_<!FAST>(B1[2], B1[2], dot2<!FAST>(B1[1], B1[1], B1[0], B1[0]));
  g.s00 = (FAST ? a + 0.3f : __fadd_rn(a, 0.3f)); g.s01 = b; g.s11 = (FAST ? d + 0.3f : __fadd_rn(d, 0.3f));
  g.det = (FAST ? g.s00 * g.s11 - g.s01 * g.s01 : __fsub_rn(__fmul_rn(g.s00, g.s11), __fmul_rn(g.s01, g.s01)));
  if (precise && g.det < mul_<!FAST>(mul_<!FAST>(0.015625f, g.s00), g.s11)) {
    // near-degenerate (needle-like) splat: the f32 determinant has lost more
    // than 6 bits to cancellation.  Re-form it in FP64 through Lagrange's
    // identity |B0|^2 |B1|^2 - (B0.B1)^2 = |B0 x B1|^2, which has no
    // cancellation, and invert in FP64.
    const double c0 = (double)B0[1] * B1[2] - (double)B0[2] * B1[1];
    const double c1 = (double)B0[2] * B1[0] - (double)B0[0] * B1[2];
    const double c2 = (double)B0[0] * B1[1] - (double)B0[1] * B1[0];
    const double ad = (double)B0[0] * B0[0] + (double)B0[1] * B0[1] + (double)B0[2] * B0[2];
    const double dd = (double)B1[0] * B1[0] + (double)B1[1] * B1[1] + (double)B1[2] * B1[2];
    const double bd = (double)B0[0] * B1[0] + (double)B0[1] * B1[1] + (double)B0[2] * B1[2];
    const double detd = (c0 * c0 + c1 * c1 + c2 * c2) + 0.3 * (ad + dd) + 0.09;
    const double inv = 1.0 / detd;
    g.det = (float)detd;
    g.ca = (float)((dd + 0.3) * inv); g.cb = (float)(-bd * inv); g.cc = (float)((ad + 0.3) * inv);
    return true;
  }
  if (!(g.det > 0.0f)) return false;
  const float inv = gdiv<FAST>(1.0f, g.det);
  g.ca = mul_<!FAST>(g.s11, inv); g.cb = mul_<!FAST>(-g.s01, inv); g.cc = mul_<!FAST>(g.s00, inv);
  return true;
}

// tile rectangle of a projected record, tile_count.wgsl:40-50 (same float ops)
__device__ __forceinline__ bool tile_rect(float mx, float my, float r, float vis, uint32_t tw, uint32_t th,
                                          uint32_t tiles_x, uint32_t tiles_y, int& x0, int& y0, int& x1, int& y1) {
  if (vis == 0.0f) return false;
  const float tsw = (float)tw, tsh = (float)th;
  x0 = max((int)floorf(__fdiv_rn(mx - r, tsw)), 0);
  y0 = max((int)floorf(__fdiv_rn(my - r, tsh)), 0);
  x1 = min((int)floorf(__fdiv_rn(mx + r, tsw)), (int)tiles_x - 1);
  y1 = min((int)floorf(__fdiv_rn(my + r, tsh)), (int)tiles_y - 1);
  return !(x1 < x0 || y1 < y0);
}

// cull: exact tile culling; super: count two-level binning items (super tiles
// reached) instead of (tile, splat) pairs; depth_max: the depth quantisation
// of the reference's 32-bit pair keys
struct TileArgs { uint32_t tw, th, tiles_x, tiles_y, cull, super; float depth_max; };

// One thread per (splat, view).  Consecutive CTAs take the views of one chunk
// of splats (view = block % n_views), so the views after the first read the
// chunk's parameters from L2 while each view plane of the outputs is still
// written with coalesced stores (the per-view work — rotation, scales, SH —
// does not share between views anyway).
// scenes (nullable): view v projects scene v's own store.
constexpr uint32_t PROJ_THREADS = 128;
__device__ __forceinline__ void proj_cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}

__global__ void __launch_bounds__(PROJ_THREADS, 8) k_project(DSplats s_all, const sc_camera* __restrict__ cams, uint32_t n_views,
                                                 uint32_t stride, float4* __restrict__ rec, TileArgs ta,
                                                 uint32_t* __restrict__ depth_keys, uint32_t* __restrict__ ids,
                                                 uint32_t* __restrict__ counts, int precise,
                                                 float4* __restrict__ zero_grad, float4* __restrict__ zero_comp,
                                                 const SceneDev* __restrict__ scenes) {
  // the chunk's 14 geometric / opacity / DC rows (and, in the BF16 form, its 45
  // SH-rest rows) are staged in shared memory by 16-byte cp.async copies issued
  // together at the start, so their latency is paid once, not once per
  // dependent load batch
  __shared__ __align__(16) float s_par[14 * PROJ_THREADS];
  __shared__ __align__(16) __nv_bfloat16 s_rest[45 * PROJ_THREADS];
  const uint32_t chunk = blockIdx.x / n_views;
  const uint32_t v = blockIdx.x - chunk * n_views;
  const uint32_t i0 = chunk * PROJ_THREADS;
  const uint32_t i = i0 + threadIdx.x;
  const DSplats s = scenes ? scenes[v].s : s_all;
  // a chunk lies wholly inside the store's capacity or wholly outside (cap is a
  // multiple of 256, chunks are 128 splats): only whole chunks are copied
  const bool staged = i0 < s.cap && i0 < s.n;
  if (staged) {
    for (uint32_t c = threadIdx.x; c < 14 * (PROJ_THREADS / 4); c += PROJ_THREADS) {
      const uint32_t r = c / (PROJ_THREADS / 4), q = c % (PROJ_THREADS / 4);
      proj_cp_async16(s_par + r * PROJ_THREADS + q * 4, s.slab + (size_t)r * s.cap + i0 + q * 4);
    }
    if (s.bf16) {
      for (uint32_t c = threadIdx.x; c < 45 * (PROJ_THREADS / 8); c += PROJ_THREADS) {
        const uint32_t r = c / (PROJ_THREADS / 8), q = c % (PROJ_THREADS / 8);
        proj_cp_async16(s_rest + r * PROJ_THREADS + q * 8, s.rest16 + (size_t)r * s.cap + i0 + q * 8);
      }
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
  }
  __syncthreads();
  if (i >= stride) return;
  const bool live = i < s.n;
  float px = 0, py = 0, pz = 0, qw = 1, qx = 0, qy = 0, qz = 0, l0 = 0, l1 = 0, l2 = 0, op = 0, d0 = 0, d1 = 0, d2 = 0;
  if (live) {
    const float* pr = s_par + threadIdx.x;
    px = pr[0 * PROJ_THREADS]; py = pr[1 * PROJ_THREADS]; pz = pr[2 * PROJ_THREADS];
    qw = pr[3 * PROJ_THREADS]; qx = pr[4 * PROJ_THREADS]; qy = pr[5 * PROJ_THREADS]; qz = pr[6 * PROJ_THREADS];
    l0 = pr[7 * PROJ_THREADS]; l1 = pr[8 * PROJ_THREADS]; l2 = pr[9 * PROJ_THREADS];
    op = pr[10 * PROJ_THREADS];
    d0 = pr[11 * PROJ_THREADS]; d1 = pr[12 * PROJ_THREADS]; d2 = pr[13 * PROJ_THREADS];
  }
  const float opacity = 1.0f / (1.0f + expf(-op));
  {
    float4 ra = make_float4(0, 0, 0, 0), rb = ra, rc = ra;
    // a splat that emits no pair sorts last (the sort reads the low 16 bits: it
    // ties only with splats at or beyond depth_max, and emits nothing)
    uint32_t key = 0xFFFFFFFFu, cnt = 0;
    if (live) {
      const Cam c = load_cam(cams + v);
      Geo g;
      if (geometry<false>(c, px, py, pz, qw, qx, qy, qz, l0, l1, l2, precise, g)) {
        const float f = c.focal;
        const float mx = c.width * 0.5f + (f * g.tx) / g.tz;
        const float my = c.height * 0.5f - (f * g.ty) / g.tz;
        const float mid = 0.5f * (g.s00 + g.s11);
        const float lambda = mid + sqrtf(fmaxf(mid * mid - g.det, 0.0f));
        const float radius = ceilf(3.0f * sqrtf(lambda));
        const float maxp = fmaxf(c.width, c.height) + radius;
        if (!(mx < -radius || mx >= c.width + radius || my < -radius || my >= c.height + radius || radius >= maxp)) {
          float dx = c.cp[0] - px, dy = c.cp[1] - py, dz = c.cp[2] - pz;
          const float len = sqrtf(dx * dx + dy * dy + dz * dz);
          dx /= len; dy /= len; dz /= len;
          float b[15];
          sh_basis15(dx, dy, dz, b);
          // the storage form decided once for the 45 loads (sp_row tests it per load)
          float ar = 0.f, ag = 0.f, ab = 0.f;
          const size_t pitch = s.cap;
          if (s.bf16) {
            const __nv_bfloat16* p = s_rest + threadIdx.x;
#pragma unroll
            for (int k = 0; k < 15; ++k) {
              ar += __bfloat162float(p[k * PROJ_THREADS]) * b[k];
              ag += __bfloat162float(p[(15 + k) * PROJ_THREADS]) * b[k];
              ab += __bfloat162float(p[(30 + k) * PROJ_THREADS]) * b[k];
            }
          } else {
            const float* p = s.slab + (size_t)SC_ROW_REST * pitch + i;
#pragma unroll
            for (int k = 0; k < 15; ++k) {
              ar += p[(size_t)k * pitch] * b[k];
              ag += p[(size_t)(15 + k) * pitch] * b[k];
              ab += p[(size_t)(30 + k) * pitch] * b[k];
            }
          }
          const float cr = fmaxf(SH_C0 * d0 + ar + 0.5f, 0.0f);
          const float cg = fmaxf(SH_C0 * d1 + ag + 0.5f, 0.0f);
          const float cb = fmaxf(SH_C0 * d2 + ab + 0.5f, 0.0f);
          ra = make_float4(mx, my, g.tz, radius);
          rb = make_float4(g.ca, g.cb, g.cc, 1.0f);
          rc = make_float4(cr, cg, cb, opacity);
          if (depth_keys) {
            int x0, y0, x1, y1;
            if (tile_rect(mx, my, radius, 1.0f, ta.tw, ta.th, ta.tiles_x, ta.tiles_y, x0, y0, x1, y1)) {
              const CullShape cs = cull_shape(mx, my, g.ca, g.cb, g.cc, opacity);
              const bool test = ta.cull && !cs.keep;
              if (ta.super) {
                for (int sy = y0 / SC_SUPER; sy <= y1 / SC_SUPER; ++sy) {
                  int sx0, sx1;
                  if (super_row_hull(cs, test, sy, x0, y0, x1, y1, ta.tw, ta.th, sx0, sx1))
                    cnt += (uint32_t)(sx1 - sx0 + 1);
                }
              } else if (!test) {
                cnt = (uint32_t)(x1 - x0 + 1) * (uint32_t)(y1 - y0 + 1);
              } else {
                for (int ty = y0; ty <= y1; ++ty) {
                  int lo, hi;
                  if (splat_row_span(cs, test, ty, x0, x1, ta.tw, ta.th, lo, hi)) cnt += (uint32_t)(hi - lo + 1);
                }
              }
              // the depth presort's key: the reference's 16-bit depth
              // (tile_emit.wgsl:54-55, the same float operations as the REF32
              // pair keys), so that a stable sort of the splats in index order
              // gives each tile the reference's (depth, splat index) order
              if (cnt) {
                const float dn = fminf(fmaxf(__fdiv_rn(g.tz, ta.depth_max), 0.0f), 1.0f);
                key = (uint32_t)(dn * 65535.0f);
              }
            }
          }
        }
      }
    }
    const size_t o = (size_t)v * stride + i;
    rec[3 * o + 0] = ra; rec[3 * o + 1] = rb; rec[3 * o + 2] = rc;
    if (zero_grad) {  // the blend backward's per-(view, splat) gradient records start at zero
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      zero_grad[3 * o + 0] = z; zero_grad[3 * o + 1] = z; zero_grad[3 * o + 2] = z;
    }
    if (zero_comp) {  // and their compensation records (compensated sums)
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      zero_comp[3 * o + 0] = z; zero_comp[3 * o + 1] = z; zero_comp[3 * o + 2] = z;
    }
    if (depth_keys) {
      depth_keys[o] = key;
      ids[o] = i;
      counts[o] = cnt;
    }
  }
}

sc_status launch_project(sc_ctx* ctx, const DSplats& s, const sc_camera* d_cams, uint32_t n_views, uint32_t stride,
                         float4* rec, const sc_tiling* tl, uint32_t* depth_keys, uint32_t* ids, uint32_t* counts,
                         int precise, int cull, float4* zero_grad, float4* zero_comp, const SceneDev* scenes) {
  if (stride == 0 || n_views == 0) return SC_OK;
  TileArgs ta{1, 1, 1, 1, 0, 0, 1.0f};
  if (tl) ta = TileArgs{tl->tile_w, tl->tile_h, (tl->width + tl->tile_w - 1) / tl->tile_w,
                        (tl->height + tl->tile_h - 1) / tl->tile_h, (cull & 1) ? 1u : 0u, (cull & 2) ? 1u : 0u,
                        tl->depth_max};
  const uint32_t bs = PROJ_THREADS;  // grid: (splats / bs) x views CTAs, views innermost
  const uint64_t blocks = sc_div_up(stride, bs) * (uint64_t)n_views;
  if (blocks > 0x7FFFFFFFull) return sc_fail(ctx, SC_ERR_INVALID_ARG, "too many splat views for one launch");
  k_project<<<(unsigned)blocks, bs, 0, ctx->stream>>>(s, d_cams, n_views, stride, rec, ta, depth_keys, ids, counts,
                                                      precise, zero_grad, zero_comp, scenes);
  return sc_check_launch(ctx, "k_project");
}

// ---------------------------------------------------------------- backward
// Per-view gradient of one splat (project_backward.wgsl:79-304).  Writes the
// 11 geometric gradients into gpos/grot/gsc/gop and returns the colour
// gradient and SH basis for the caller to form the 48 SH gradients.
template <bool FAST>
__device__ __forceinline__ bool splat_backward_view(const Cam& c, float px, float py, float pz, float qw, float qx,
                                                    float qy, float qz, float l0, float l1, float l2, float opacity,
                                                    const float4 pg0, const float4 pg1, const float4 pg2,
                                                    float gpos[3], float grot[4], float gsc[3], float& gop,
                                                    float basis[15], int precise) {
  // FAST = false (sc_project_backward) forms the geometry exactly as the
  // forward does, so it keeps exactly the splats the forward kept; the
  // trainer's FAST adjoint can differ from the forward only for a needle whose
  // f32 determinant is within rounding of zero (the FP64 option decides those
  // robustly)
  Geo g;
  if (!geometry<FAST>(c, px, py, pz, qw, qx, qy, qz, l0, l1, l2, precise, g)) return false;
  const float f = c.focal;
  const float iz = gdiv<FAST>(1.0f, g.tz), iz2 = iz * iz;
  // opacity logit
  gop += pg0.z * opacity * (1.0f - opacity);
  // SH basis at the view direction
  float dx = c.cp[0] - px, dy = c.cp[1] - py, dz = c.cp[2] - pz;
  if (FAST) {
    const float il = rsqrtf(dx * dx + dy * dy + dz * dz);
    sh_basis15(dx * il, dy * il, dz * il, basis);
  } else {
    const float len = sqrtf(dx * dx + dy * dy + dz * dz);
    sh_basis15(dx / len, dy / len, dz / len, basis);
  }
  // dSigma2D = -C dConic C with the off-diagonal conic gradient halved
  const float C00 = g.ca, C01 = g.cb, C11 = g.cc;
  const float D00 = pg1.x, D01 = 0.5f * pg1.y, D11 = pg1.z;
  const float P00 = C00 * D00 + C01 * D01, P10 = C01 * D00 + C11 * D01;
  const float P01 = C00 * D01 + C01 * D11, P11 = C01 * D01 + C11 * D11;
  const float ds00 = -(P00 * C00 + P01 * C01);
  const float ds11 = -(P10 * C01 + P11 * C11);
  const float ds01 = -(P00 * C01 + P01 * C11) - (P10 * C00 + P11 * C01);
  const float h = 0.5f * ds01;
  // dSigma_cam = J^T dS J (3x3 symmetric); J rows j0 = (j0x, 0, j0z), j1 = (0, j1y, j1z)
  float dC[3][3];
  {
    const float a0[3] = {g.j0[0], g.j0[1], g.j0[2]}, a1[3] = {g.j1[0], g.j1[1], g.j1[2]};
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k)
        dC[r][k] = a0[r] * ds00 * a0[k] + a0[r] * h * a1[k] + a1[r] * h * a0[k] + a1[r] * ds11 * a1[k];
  }
  // dSigma_world = W^T dC W
  float T1[3][3], dW[3][3];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) T1[r][k] = dC[r][0] * g.W[0][k] + dC[r][1] * g.W[1][k] + dC[r][2] * g.W[2][k];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) dW[r][k] = g.W[0][r] * T1[0][k] + g.W[1][r] * T1[1][k] + g.W[2][r] * T1[2][k];
  // dR = (dW + dW^T) R S^2 ; G[row][col]
  const float s2[3] = {g.sig[0] * g.sig[0], g.sig[1] * g.sig[1], g.sig[2] * g.sig[2]};
  float G[3][3];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) {
      float acc = 0.f;
      for (int m = 0; m < 3; ++m) acc += (dW[r][m] + dW[m][r]) * g.R[m][k];
      G[r][k] = acc * s2[k];
    }
  // log-sigma: dL/d(s_k^2) = R_k^T dW R_k, times 2 s_k^2
  for (int k = 0; k < 3; ++k) {
    float acc = 0.f;
    for (int r = 0; r < 3; ++r) {
      float row = dW[r][0] * g.R[0][k] + dW[r][1] * g.R[1][k] + dW[r][2] * g.R[2][k];
      acc += g.R[r][k] * row;
    }
    gsc[k] += acc * 2.0f * s2[k];
  }
  // quaternion, project_backward.wgsl:280-286
  grot[0] += 2.0f * (qz * (G[1][0] - G[0][1]) + qy * (G[0][2] - G[2][0]) + qx * (G[2][1] - G[1][2]));
  grot[1] += 2.0f * (qy * (G[0][1] + G[1][0]) + qz * (G[0][2] + G[2][0]) + qw * (G[2][1] - G[1][2])) -
             4.0f * qx * (G[1][1] + G[2][2]);
  grot[2] += -4.0f * qy * (G[0][0] + G[2][2]) +
             2.0f * (qx * (G[0][1] + G[1][0]) + qw * (G[0][2] - G[2][0]) + qz * (G[1][2] + G[2][1]));
  grot[3] += -4.0f * qz * (G[0][0] + G[1][1]) +
             2.0f * (qw * (G[1][0] - G[0][1]) + qx * (G[0][2] + G[2][0]) + qy * (G[1][2] + G[2][1]));
  // position, project_backward.wgsl:288-303
  const float dtx = f * iz * pg0.x;
  const float dty = -f * iz * pg0.y;
  const float dtz = -f * g.tx * iz2 * pg0.x + f * g.ty * iz2 * pg0.y;
  const float cx = dtx, cy = dty, cz = -dtz;
  for (int k = 0; k < 3; ++k) gpos[k] += g.W[0][k] * cx + g.W[1][k] * cy + g.W[2][k] * cz;
  return true;
}

__global__ void __launch_bounds__(128) k_project_backward(DSplats s, const float4* __restrict__ pg,
                                                          const sc_camera* __restrict__ cam, float* __restrict__ out,
                                                          uint32_t gcap, int accumulate, int precise) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const Cam c = load_cam(cam);
  float gpos[3] = {0, 0, 0}, grot[4] = {0, 0, 0, 0}, gsc[3] = {0, 0, 0}, gop = 0, basis[15];
  const float4 p0 = pg[3 * (size_t)i], p1 = pg[3 * (size_t)i + 1], p2 = pg[3 * (size_t)i + 2];
  const float op = 1.0f / (1.0f + expf(-sp_row(s, 10, i)));
  const bool ok = splat_backward_view<false>(c, sp_row(s, 0, i), sp_row(s, 1, i), sp_row(s, 2, i), sp_row(s, 3, i),
                                      sp_row(s, 4, i), sp_row(s, 5, i), sp_row(s, 6, i), sp_row(s, 7, i),
                                      sp_row(s, 8, i), sp_row(s, 9, i), op, p0, p1, p2, gpos, grot, gsc, gop, basis,
                                      precise);
  float row[SC_NROWS];
#pragma unroll
  for (int r = 0; r < SC_NROWS; ++r) row[r] = 0.f;
  if (ok) {
    row[0] = gpos[0]; row[1] = gpos[1]; row[2] = gpos[2];
    row[3] = grot[0]; row[4] = grot[1]; row[5] = grot[2]; row[6] = grot[3];
    row[7] = gsc[0]; row[8] = gsc[1]; row[9] = gsc[2];
    row[10] = gop;
    row[11] = p2.x * SH_C0; row[12] = p2.y * SH_C0; row[13] = p2.z * SH_C0;
#pragma unroll
    for (int k = 0; k < 15; ++k) {
      row[14 + k] = p2.x * basis[k]; row[29 + k] = p2.y * basis[k]; row[44 + k] = p2.z * basis[k];
    }
  }
#pragma unroll
  for (int r = 0; r < SC_NROWS; ++r) {
    float* dst = out + (size_t)r * gcap + i;
    *dst = accumulate ? *dst + row[r] : row[r];
  }
}

sc_status launch_project_backward(sc_ctx* ctx, const DSplats& s, const float4* pg, const sc_camera* d_cam,
                                  float* grads, uint32_t gcap, int accumulate, int precise_det) {
  if (s.n == 0) return SC_OK;
  k_project_backward<<<(unsigned)sc_div_up(s.n, 128), 128, 0, ctx->stream>>>(s, pg, d_cam, grads, gcap, accumulate,
                                                                             precise_det);
  return sc_check_launch(ctx, "k_project_backward");
}

// ---------------------------------------------------------------- per-splat gradient rows
// Sum of splat i's parameter gradients over n_views views, in the order of the
// views (project_backward.wgsl:79-304 per view, accumulated like the
// reference's per-view passes into one gradient buffer), written as its 59
// gradient rows.  The views are taken in groups of 32, in two phases per group
// so that the geometric adjoint and the 45 SH-rest sums are never live
// together: phase 1 runs the geometric adjoint of each view (14 sums in
// registers) and marks the views it accepts; phase 2 forms the SH-rest sums of
// the marked views (colour gradient times the basis at the view direction,
// the same arithmetic as the adjoint's basis) and adds them into this thread's
// column of a shared-memory block.  Peak register use is that of the larger
// phase, not of both.
__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

constexpr int PB_THREADS = 128;
constexpr int PB_GROUP = 32;  // views per group: one validity bit each

__device__ __forceinline__ void project_backward_rows(const DSplats& s, const float4* __restrict__ pg,
                                                      uint32_t stride, const sc_camera* __restrict__ cams,
                                                      uint32_t n_views, float* __restrict__ out, uint32_t n_shards,
                                                      uint32_t shard, const uint32_t* __restrict__ skip, int precise,
                                                      const float4* __restrict__ pc) {
  __shared__ float s_rest[45 * PB_THREADS];
  const uint64_t i = (uint64_t)blockIdx.x * PB_THREADS + threadIdx.x;
  if (i >= (uint64_t)n_shards * shard) return;
  float* dst = out + (i / shard) * SC_NROWS * (uint64_t)shard + i % shard;
  float* srest = s_rest + threadIdx.x;  // this thread's column: sum k at srest[k * PB_THREADS]
#pragma unroll
  for (int k = 0; k < 45; ++k) srest[k * PB_THREADS] = 0.f;
  float gpos[3] = {0.f, 0.f, 0.f}, grot[4] = {0.f, 0.f, 0.f, 0.f}, gsc[3] = {0.f, 0.f, 0.f}, gop = 0.f;
  float gdc[3] = {0.f, 0.f, 0.f};
  // padding splats, or a step whose emission overflowed, contribute nothing
  if (i < s.n && !(skip && (*skip & SC_DEVERR_CAPACITY))) {
    const uint32_t si = (uint32_t)i;
    const float px = sp_row(s, 0, si), py = sp_row(s, 1, si), pz = sp_row(s, 2, si);
    const float qw = sp_row(s, 3, si), qx = sp_row(s, 4, si), qy = sp_row(s, 5, si), qz = sp_row(s, 6, si);
    const float l0 = sp_row(s, 7, si), l1 = sp_row(s, 8, si), l2 = sp_row(s, 9, si);
    const float opacity = __fdividef(1.0f, 1.0f + __expf(-sp_row(s, 10, si)));
    for (uint32_t g0 = 0; g0 < n_views; g0 += PB_GROUP) {
      const uint32_t g1 = min(n_views, g0 + (uint32_t)PB_GROUP);
      uint32_t accepted = 0;
      for (uint32_t v = g0; v < g1; ++v) {
        const size_t o = (size_t)v * stride + si;
        float4 p2 = pg[3 * o + 2];
        float4 p0 = pg[3 * o], p1 = pg[3 * o + 1];
        if (pc) {  // compensated sums: the total is the sum plus its accumulated rounding errors
          p0 = f4add(p0, pc[3 * o]); p1 = f4add(p1, pc[3 * o + 1]); p2 = f4add(p2, pc[3 * o + 2]);
        }
        if (p0.x == 0.f && p0.y == 0.f && p0.z == 0.f && p1.x == 0.f && p1.y == 0.f && p1.z == 0.f && p2.x == 0.f &&
            p2.y == 0.f && p2.z == 0.f)
          continue;  // splat untouched in this view: every gradient term is zero
        const Cam c = load_cam(cams + v);
        float basis[15];  // formed again in phase 2
        if (!splat_backward_view<true>(c, px, py, pz, qw, qx, qy, qz, l0, l1, l2, opacity, p0, p1, p2, gpos, grot,
                                       gsc, gop, basis, precise))
          continue;
        accepted |= 1u << (v - g0);
        gdc[0] += p2.x * SH_C0; gdc[1] += p2.y * SH_C0; gdc[2] += p2.z * SH_C0;
      }
      if (!accepted) continue;
      float grest[45];
#pragma unroll
      for (int k = 0; k < 45; ++k) grest[k] = 0.f;
      while (accepted) {
        const uint32_t v = g0 + (uint32_t)(__ffs(accepted) - 1);
        accepted &= accepted - 1u;
        float4 p2 = pg[3 * ((size_t)v * stride + si) + 2];
        if (pc) p2 = f4add(p2, pc[3 * ((size_t)v * stride + si) + 2]);
        const float4 e = __ldg(reinterpret_cast<const float4*>(cams + v) + 4);  // camera position
        // the view direction and basis exactly as splat_backward_view<true> forms them
        const float dx = e.x - px, dy = e.y - py, dz = e.z - pz;
        const float il = rsqrtf(dx * dx + dy * dy + dz * dz);
        float basis[15];
        sh_basis15(dx * il, dy * il, dz * il, basis);
#pragma unroll
        for (int k = 0; k < 15; ++k) {
          grest[k] += p2.x * basis[k]; grest[15 + k] += p2.y * basis[k]; grest[30 + k] += p2.z * basis[k];
        }
      }
#pragma unroll
      for (int k = 0; k < 45; ++k) srest[k * PB_THREADS] += grest[k];
    }
  }
  const float gg[14] = {gpos[0], gpos[1], gpos[2], grot[0], grot[1], grot[2], grot[3],
                        gsc[0],  gsc[1],  gsc[2],  gop,     gdc[0],  gdc[1],  gdc[2]};
#pragma unroll
  for (int r = 0; r < 14; ++r) dst[(size_t)r * shard] = gg[r];
#pragma unroll
  for (int k = 0; k < 45; ++k) dst[(size_t)(SC_ROW_REST + k) * shard] = srest[k * PB_THREADS];
}

__global__ void __launch_bounds__(PB_THREADS, 5) k_project_backward_shards(DSplats s, const float4* __restrict__ pg,
                                                                     uint32_t stride,
                                                                     const sc_camera* __restrict__ cams,
                                                                     uint32_t n_views, float* __restrict__ out,
                                                                     uint32_t n_shards, uint32_t shard,
                                                                     const uint32_t* __restrict__ skip, int precise,
                                                                     const float4* __restrict__ pc) {
  project_backward_rows(s, pg, stride, cams, n_views, out, n_shards, shard, skip, precise, pc);
}

// Many scenes, one view each: grid.y = scene; scene v's gradient rows from
// its view's records (pg + 3 v stride) into its own rows (grads, gstride).
__global__ void __launch_bounds__(PB_THREADS, 5) k_project_backward_scenes(const SceneDev* __restrict__ scenes,
                                                                     const float4* __restrict__ pg, uint32_t stride,
                                                                     const sc_camera* __restrict__ cams,
                                                                     const uint32_t* __restrict__ skip, int precise,
                                                                     const float4* __restrict__ pc) {
  const uint32_t v = blockIdx.y;
  const SceneDev sd = scenes[v];
  const size_t off = (size_t)3 * v * stride;
  project_backward_rows(sd.s, pg + off, stride, cams + v, 1, sd.grads, 1, sd.gstride, skip, precise,
                        pc ? pc + off : nullptr);
}

sc_status launch_project_backward_scenes(sc_ctx* ctx, const SceneDev* d_scenes, uint32_t n_scenes,
                                         uint32_t max_gstride, const float4* pg, uint32_t stride,
                                         const sc_camera* d_cams, const uint32_t* d_skip, int precise_det,
                                         const float4* pc) {
  if (n_scenes == 0 || max_gstride == 0) return SC_OK;
  const dim3 grid((unsigned)sc_div_up(max_gstride, PB_THREADS), n_scenes);
  k_project_backward_scenes<<<grid, PB_THREADS, 0, ctx->stream>>>(d_scenes, pg, stride, d_cams, d_skip, precise_det,
                                                                  pc);
  return sc_check_launch(ctx, "k_project_backward_scenes");
}

sc_status launch_project_backward_shards(sc_ctx* ctx, const DSplats& s, const float4* pg, uint32_t stride,
                                         const sc_camera* d_cams, uint32_t n_views, float* grads, uint32_t n_shards,
                                         uint32_t shard, const uint32_t* d_skip, int precise_det,
                                         const float4* pc) {
  const uint64_t total = (uint64_t)n_shards * shard;
  if (total == 0) return SC_OK;
  k_project_backward_shards<<<(unsigned)sc_div_up(total, PB_THREADS), PB_THREADS, 0, ctx->stream>>>(
      s, pg, stride, d_cams, n_views, grads, n_shards, shard, d_skip, precise_det, pc);
  return sc_check_launch(ctx, "k_project_backward_shards");
}

}  // namespace sck
