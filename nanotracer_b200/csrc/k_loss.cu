// k_loss.cu — SSIM loss and gradient on the device (loss.rs:22-375; the
// reference computes it on the CPU after reading the image back,
// train.rs:180-196).
//
// SSIM (Wang et al. 2004) over an 11-tap separable Gaussian window (sigma 1.5)
// with reflect-101 padding, C1 = 1e-4, C2 = 9e-4, per rgb channel; the loss is
// 1 - mean SSIM and its gradient is the reference's analytic form: coefficient
// planes P = dSSIM/dmu_x, Q = dSSIM/dsigma_x^2, R = dSSIM/dsigma_xy (and
// mu_x*Q, mu_y*R) pulled back through the adjoint of the blur.
//
// Two kernels per call, each one CTA per 32x8 pixel tile of one view:
//   k_ssim_terms  stage the tile plus a 5-pixel reflected halo of prediction and
//                 target in shared memory, blur (horizontal then vertical, the
//                 reference's order and f32 rounding: no contraction) the five
//                 moments of the three channels, write the 15 coefficient planes
//                 and add the tile's SSIM-map sum to the view's f64 total;
//   k_ssim_grad   stage the coefficient planes with a 5-pixel halo (zero outside
//                 the image), apply the transposed blur as a gather (vertical
//                 then horizontal; near the border the reflected taps add their
//                 mirrored sources), combine with the prediction and target and
//                 add scale * dL/dC into dl_dc.
// Reflect-101 with a 5-pixel radius folds at most once for images of 6 or more
// pixels per side, which the host requires.
#include "sc_internal.cuh"

#include <cmath>

namespace sck {

namespace {

constexpr int SS_W = 11, SS_R = 5;
constexpr int SS_TW = 32, SS_TH = 8;
constexpr int SS_RW = SS_TW + 2 * SS_R, SS_RH = SS_TH + 2 * SS_R;  // 42 x 18
constexpr int SS_PLANES = 15;                                        // 5 per channel
constexpr float SS_C1 = 0.0001f, SS_C2 = 0.0009f;

struct SsimArgs {
  float g[SS_W];
  uint32_t w, h;
  uint64_t P;
  float scale;
  float inv_n;  // 1 / (w h) in f32
};

__device__ __forceinline__ int reflect101(int i, int n) {
  // single fold: i in [-(n-1), 2(n-1)]
  if (i < 0) i = -i;
  if (i >= n) i = 2 * (n - 1) - i;
  return i;
}

// reference rounding: every product and sum rounded separately
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

struct TermsSmem {
  float X[3][SS_RH][SS_RW];
  float Y[3][SS_RH][SS_RW];
  float Hs[SS_PLANES][SS_RH][SS_TW];
};

__global__ void __launch_bounds__(256) k_ssim_terms(const float4* __restrict__ pred, const float* __restrict__ target,
                                                    SsimArgs a, float* __restrict__ terms,
                                                    double* __restrict__ ssim_sum) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TermsSmem& sm = *reinterpret_cast<TermsSmem*>(smem_raw);
  __shared__ double red[8];
  const uint32_t v = blockIdx.z;
  const int x0 = blockIdx.x * SS_TW, y0 = blockIdx.y * SS_TH;
  const int W = (int)a.w, H = (int)a.h;
  const float4* pv = pred + (uint64_t)v * a.P;
  const float* tv = target + (uint64_t)v * a.P * 3;
  for (int idx = threadIdx.x; idx < SS_RH * SS_RW; idx += blockDim.x) {
    const int ry = idx / SS_RW, rx = idx % SS_RW;
    // clamp to the blur footprint of the image first (columns past it feed no output pixel)
    const int gy = reflect101(min(y0 - SS_R + ry, H - 1 + SS_R), H);
    const int gx = reflect101(min(x0 - SS_R + rx, W - 1 + SS_R), W);
    const uint64_t p = (uint64_t)gy * W + gx;
    const float4 c = pv[p];
    sm.X[0][ry][rx] = c.x; sm.X[1][ry][rx] = c.y; sm.X[2][ry][rx] = c.z;
    sm.Y[0][ry][rx] = tv[3 * p]; sm.Y[1][ry][rx] = tv[3 * p + 1]; sm.Y[2][ry][rx] = tv[3 * p + 2];
  }
  __syncthreads();
  // horizontal pass over every staged row, output columns only
  for (int idx = threadIdx.x; idx < 3 * SS_RH * SS_TW; idx += blockDim.x) {
    const int c = idx / (SS_RH * SS_TW), rem = idx % (SS_RH * SS_TW);
    const int ry = rem / SS_TW, tx = rem % SS_TW;
    float sx = 0.f, sy = 0.f, sxx = 0.f, syy = 0.f, sxy = 0.f;
#pragma unroll
    for (int k = 0; k < SS_W; ++k) {
      const float x = sm.X[c][ry][tx + k], y = sm.Y[c][ry][tx + k], g = a.g[k];
      sx = add(sx, mul(x, g));
      sy = add(sy, mul(y, g));
      sxx = add(sxx, mul(mul(x, x), g));
      syy = add(syy, mul(mul(y, y), g));
      sxy = add(sxy, mul(mul(x, y), g));
    }
    sm.Hs[c * 5 + 0][ry][tx] = sx; sm.Hs[c * 5 + 1][ry][tx] = sy; sm.Hs[c * 5 + 2][ry][tx] = sxx;
    sm.Hs[c * 5 + 3][ry][tx] = syy; sm.Hs[c * 5 + 4][ry][tx] = sxy;
  }
  __syncthreads();
  // vertical pass, SSIM map and coefficient planes: one pixel per thread
  double local = 0.0;
  {
    const int ty = threadIdx.x / SS_TW, tx = threadIdx.x % SS_TW;
    const int x = x0 + tx, y = y0 + ty;
    if (x < W && y < H) {
      const uint64_t p = (uint64_t)y * W + x;
      for (int c = 0; c < 3; ++c) {
        float m[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < SS_W; ++k)
#pragma unroll
          for (int q = 0; q < 5; ++q) m[q] = add(m[q], mul(sm.Hs[c * 5 + q][ty + k][tx], a.g[k]));
        const float mux = m[0], muy = m[1];
        const float mux2 = mul(mux, mux), muy2 = mul(muy, muy);
        const float sxx = sub(m[2], mux2), syy = sub(m[3], muy2), sxy = sub(m[4], mul(mux, muy));
        const float av = add(mul(mul(2.0f, mux), muy), SS_C1);
        const float bv = add(mul(2.0f, sxy), SS_C2);
        const float cv = add(add(mux2, muy2), SS_C1);
        const float dv = add(add(sxx, syy), SS_C2);
        local += (double)__fdiv_rn(mul(av, bv), mul(cv, dv));
        const float cd = mul(cv, dv);
        const float pp = __fdiv_rn(mul(mul(2.0f, bv), sub(mul(muy, cv), mul(mux, av))), mul(cv, cd));
        const float qq = __fdiv_rn(mul(-av, bv), mul(mul(cv, dv), dv));
        const float rr = __fdiv_rn(mul(2.0f, av), cd);
        float* t = terms + ((uint64_t)v * SS_PLANES + c * 5) * a.P + p;
        t[0] = pp;
        t[a.P] = qq;
        t[2 * a.P] = rr;
        t[3 * a.P] = mul(mux, qq);
        t[4 * a.P] = mul(muy, rr);
      }
    }
  }
  // block sum of the SSIM map -> one f64 atomic per block
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    atomicAdd(ssim_sum + v, s);
  }
}

struct GradSmem {
  float F[SS_PLANES][SS_RH][SS_RW];
  float Vt[SS_PLANES][SS_TH][SS_RW];
};

// transposed 1-D blur at global index i along an axis of length n, reading
// src[j] for the sources j of i staged at local index j - base
template <int STRIDE>
__device__ __forceinline__ float blur_adjoint_1d(const float* src, int i, int n, int base, const float* g) {
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < SS_W; ++k) acc += g[k] * src[(i - k + SS_R - base) * STRIDE] * ((unsigned)(i - k + SS_R) < (unsigned)n);
  if (i <= SS_R && i >= 1) {  // taps whose source index reflected below 0 onto i
    for (int k = 0; k < SS_W; ++k) {
      const int j = -i - k + SS_R;
      if (j >= 0) acc += g[k] * src[(j - base) * STRIDE];
    }
  }
  if (i >= n - 1 - SS_R && i <= n - 2) {  // taps that reflected beyond n-1 onto i
    for (int k = 0; k < SS_W; ++k) {
      const int j = 2 * (n - 1) - i - k + SS_R;
      if (j <= n - 1) acc += g[k] * src[(j - base) * STRIDE];
    }
  }
  return acc;
}

__global__ void __launch_bounds__(256) k_ssim_grad(const float4* __restrict__ pred, const float* __restrict__ target,
                                                   SsimArgs a, const float* __restrict__ terms,
                                                   float4* __restrict__ dl_dc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradSmem& sm = *reinterpret_cast<GradSmem*>(smem_raw);
  const uint32_t v = blockIdx.z;
  const int x0 = blockIdx.x * SS_TW, y0 = blockIdx.y * SS_TH;
  const int W = (int)a.w, H = (int)a.h;
  const float* tv = terms + (uint64_t)v * SS_PLANES * a.P;
  for (int idx = threadIdx.x; idx < SS_PLANES * SS_RH * SS_RW; idx += blockDim.x) {
    const int pl = idx / (SS_RH * SS_RW), rem = idx % (SS_RH * SS_RW);
    const int ry = rem / SS_RW, rx = rem % SS_RW;
    const int gy = y0 - SS_R + ry, gx = x0 - SS_R + rx;
    float val = 0.f;
    if (gy >= 0 && gy < H && gx >= 0 && gx < W) val = tv[(uint64_t)pl * a.P + (uint64_t)gy * W + gx];
    sm.F[pl][ry][rx] = val;
  }
  __syncthreads();
  // vertical adjoint: the tile's rows, every staged column
  for (int idx = threadIdx.x; idx < SS_PLANES * SS_TH * SS_RW; idx += blockDim.x) {
    const int pl = idx / (SS_TH * SS_RW), rem = idx % (SS_TH * SS_RW);
    const int ty = rem / SS_RW, rx = rem % SS_RW;
    const int i = y0 + ty;
    float r = 0.f;
    if (i < H) r = blur_adjoint_1d<SS_RW>(&sm.F[pl][0][rx], i, H, y0 - SS_R, a.g);
    sm.Vt[pl][ty][rx] = r;
  }
  __syncthreads();
  // horizontal adjoint and the per-pixel gradient
  const int ty = threadIdx.x / SS_TW, tx = threadIdx.x % SS_TW;
  const int x = x0 + tx, y = y0 + ty;
  if (x >= W || y >= H) return;
  const uint64_t p = (uint64_t)y * W + x;
  const float4 pr = pred[(uint64_t)v * a.P + p];
  const float* tg = target + ((uint64_t)v * a.P + p) * 3;
  const float xs[3] = {pr.x, pr.y, pr.z};
  float gout[3];
  for (int c = 0; c < 3; ++c) {
    float s[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) s[q] = blur_adjoint_1d<1>(&sm.Vt[c * 5 + q][ty][0], x, W, x0 - SS_R, a.g);
    const float dssim = s[0] + 2.0f * (xs[c] * s[1] - s[3]) + (tg[c] * s[2] - s[4]);
    gout[c] = (-a.inv_n * dssim) / 3.0f * a.scale;
  }
  float4 d = dl_dc[(uint64_t)v * a.P + p];
  d.x += gout[0]; d.y += gout[1]; d.z += gout[2];
  dl_dc[(uint64_t)v * a.P + p] = d;
}

__global__ void k_loss_parts(const double* __restrict__ mse, const double* __restrict__ ssim_sum, uint32_t n_views,
                             double inv_3p, float lambda, double* __restrict__ out) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_views) return;
  const double m = mse ? mse[v] * inv_3p : 0.0;
  const double s = ssim_sum ? 1.0 - ssim_sum[v] * inv_3p : 0.0;
  const double l = (double)lambda;
  out[3 * v] = lambda == 0.0f ? m : (lambda == 1.0f ? s : (1.0 - l) * m + l * s);
  out[3 * v + 1] = lambda == 1.0f ? 0.0 : m;
  out[3 * v + 2] = lambda == 0.0f ? 0.0 : s;
}

}  // namespace

sc_status launch_loss_parts(sc_ctx* ctx, const double* mse, const double* ssim_sum, uint32_t n_views, uint64_t P,
                            float lambda, double* out) {
  if (n_views == 0) return SC_OK;
  k_loss_parts<<<(n_views + 63) / 64, 64, 0, ctx->stream>>>(mse, ssim_sum, n_views, 1.0 / (3.0 * (double)P), lambda,
                                                             out);
  return sc_check_launch(ctx, "k_loss_parts");
}

void ssim_window(float g[11]) {
  // loss.rs:36-51, in f32 like the reference
  const float centre = 5.0f, two_sigma_sq = 2.0f * 1.5f * 1.5f;
  float sum = 0.0f;
  for (int i = 0; i < SS_W; ++i) {
    const float d = (float)i - centre;
    g[i] = std::exp(-d * d / two_sigma_sq);
    sum += g[i];
  }
  for (int i = 0; i < SS_W; ++i) g[i] /= sum;
}

size_t ssim_terms_bytes(uint64_t pixels_per_view, uint32_t n_views) {
  return (size_t)n_views * SS_PLANES * pixels_per_view * sizeof(float);
}

sc_status launch_ssim(sc_ctx* ctx, const float4* pred, const float* target, uint32_t w, uint32_t h, uint32_t n_views,
                      float scale, float4* dl_dc, double* ssim_sum, float* terms) {
  if (n_views == 0) return SC_OK;
  if (w < 6 || h < 6) return sc_fail(ctx, SC_ERR_INVALID_ARG, "SSIM needs images of at least 6x6 pixels");
  SsimArgs a;
  ssim_window(a.g);
  a.w = w; a.h = h; a.P = (uint64_t)w * h; a.scale = scale;
  a.inv_n = 1.0f / (float)a.P;
  static bool attr_set[64] = {};
  const int dev = ctx->device & 63;
  if (!attr_set[dev]) {
    SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ssim_terms, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(TermsSmem)), "ssim smem");
    SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ssim_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(GradSmem)), "ssim smem");
    attr_set[dev] = true;
  }
  const dim3 grid((w + SS_TW - 1) / SS_TW, (h + SS_TH - 1) / SS_TH, n_views);
  k_ssim_terms<<<grid, 256, sizeof(TermsSmem), ctx->stream>>>(pred, target, a, terms, ssim_sum);
  SC_TRY(sc_check_launch(ctx, "k_ssim_terms"));
  k_ssim_grad<<<grid, 256, sizeof(GradSmem), ctx->stream>>>(pred, target, a, terms, dl_dc);
  return sc_check_launch(ctx, "k_ssim_grad");
}

}  // namespace sck
