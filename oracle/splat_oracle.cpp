// splat_oracle.cpp — CPU restatement of nano-optimize's Gaussian-splat
// training path, used ONLY as test infrastructure: the parity tests, the
// smoke check and the CPU-baseline leg of the benchmark load it as the
// checker.  Nothing in the product library links or calls this file.
//
// It restates, in plain scalar C++ (templated on float / double), the
// arithmetic of the reference's WGSL kernels and Rust host code:
//
//   camera          crates/nano-optimize/src/raster.rs:79-99 (CameraUniform::from_pose,
//                   glam 0.33.12 look_at_mat4 RH — third-party, restated from the
//                   standard right-handed look-at definition)
//   projection      crates/nano-optimize/src/shaders/project_gaussians.wgsl:156-259
//                   (+ eval_sh :88-154, quat_to_mat3 :68-80)
//   binning         shaders/tile_count.wgsl:28-55, shaders/tile_emit.wgsl:36-67,
//                   shaders/tile_ranges.wgsl:22-41; the sort is a stable sort by key
//                   from emission order, which is what radix_sort.rs:1-26 produces
//   composite       shaders/rasterize.wgsl:48-118
//   MSE             crates/nano-optimize/src/loss.rs:163-179
//   SSIM, combined  crates/nano-optimize/src/loss.rs:22-152, 193-410
//   backward        shaders/rasterize_backward.wgsl:73-210
//   project bwd     shaders/project_backward.wgsl:79-304
//   Adam            crates/nano-optimize/src/adam.rs:70-90, adam_gpu.rs:262-323
//   constraints     shaders/apply_constraints.wgsl:24-41
//   grad acc        shaders/accumulate_grad_pos.wgsl:17-23
//   prune/densify   crates/nano-optimize/src/train.rs:414-602 (swap-remove order, LCG)
//   PLY             crates/nano-splat/src/ply.rs:17-256
//
// Compiled with -ffp-contract=off so every float operation rounds where the
// reference's source rounds.  Two documented extensions beyond the
// reference, each flagged where used:
//   * "exact" backward mode (per-pixel last-contributor count and final
//     transmittance recorded by the forward), next to the reference's
//     "ref" mode that reverse-walks the whole tile list;
//   * 64-bit (view, tile, depth-bits) keys next to the reference's
//     32-bit (tile << 16 | depth16) keys, and multi-view pipelines.
// And test diagnostics with no reference counterpart: near-threshold
// margins of the blend's discontinuous tests (composite_margins), the
// absolute-value sums that bound a gradient sum's rounding error, and the
// iteration's gradient rows as an output of train_step.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

// ---------------------------------------------------------------- types
struct HostSplats {          // mirrors SplatBuffer (splat_store.rs:20-36)
  uint32_t n;
  float* pos;                // n*3
  float* rot;                // n*4 (w, x, y, z)
  float* scale;              // n*3 log-sigma
  float* opacity;            // n   logit
  float* sh_dc;              // n*3
  float* sh_rest;            // n*45 planar R[15] G[15] B[15]
};

template <typename T>
struct HostGrads {           // same layout as HostSplats, element type T
  T* pos; T* rot; T* scale; T* opacity; T* sh_dc; T* sh_rest;
};

struct Camera {              // CameraUniform (raster.rs:60-77), 96 bytes
  float view[16];            // column-major
  float cam_pos[3];
  float near_plane;
  float focal;
  float width;
  float height;
  uint32_t n_splats;
};
static_assert(sizeof(Camera) == 96, "camera layout");

struct Tiling {              // TilingParams (tile_binner.rs:21-42), tiles may be non-square
  uint32_t width, height, tile_w, tile_h;
  float depth_max;
  uint32_t tiles_x() const { return (width + tile_w - 1) / tile_w; }
  uint32_t tiles_y() const { return (height + tile_h - 1) / tile_h; }
  uint32_t num_tiles() const { return tiles_x() * tiles_y(); }
};

// Projected record, 12 scalars: mean.xy, depth, radius | conic.abc, visible | rgb, opacity
// (ProjectedSplat, raster.rs:27-37).  Projected grad, 12 scalars: dmean.xy, dopacity, pad |
// dconic.abc, pad | dcolor.rgb, pad (ProjectedGrad, raster.rs:46-55).
enum { R_MX = 0, R_MY, R_DEPTH, R_RADIUS, R_CA, R_CB, R_CC, R_VIS, R_R, R_G, R_B, R_OP };
enum { G_MX = 0, G_MY = 1, G_OP = 2, G_CA = 4, G_CB = 5, G_CC = 6, G_R = 8, G_G = 9, G_B = 10 };

// SH constants, project_gaussians.wgsl:47-61 (f32 literals)
static const float SH_C0 = 0.2820948f;
static const float SH_C1 = 0.488602f;
static const float SH_C2_0 = 1.0925485f, SH_C2_1 = -1.0925485f, SH_C2_2 = 0.31539157f,
                   SH_C2_3 = -1.0925485f, SH_C2_4 = 0.54627424f;
static const float SH_C3_0 = -0.5900436f, SH_C3_1 = 2.8906114f, SH_C3_2 = -0.4570458f,
                   SH_C3_3 = 0.37317634f, SH_C3_4 = -0.4570458f, SH_C3_5 = 1.4453057f,
                   SH_C3_6 = -0.5900436f;

template <typename T> struct V3 { T x, y, z; };
template <typename T> static inline V3<T> v3(T x, T y, T z) { return {x, y, z}; }
template <typename T> static inline T dot3(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// column-major 3x3: c[col] is a column
template <typename T> struct M3 { V3<T> c[3]; };
template <typename T> static inline V3<T> add3(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> static inline V3<T> mul3s(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> static inline T comp(V3<T> a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
template <typename T> static inline V3<T> mat_vec(const M3<T>& m, V3<T> v) {
  // WGSL m * v = m[0]*v.x + m[1]*v.y + m[2]*v.z
  return add3(add3(mul3s(m.c[0], v.x), mul3s(m.c[1], v.y)), mul3s(m.c[2], v.z));
}
template <typename T> static inline M3<T> mat_mul(const M3<T>& a, const M3<T>& b) {
  M3<T> r; for (int j = 0; j < 3; ++j) r.c[j] = mat_vec(a, b.c[j]); return r;
}
template <typename T> static inline M3<T> transpose(const M3<T>& m) {
  M3<T> r;
  r.c[0] = {m.c[0].x, m.c[1].x, m.c[2].x};
  r.c[1] = {m.c[0].y, m.c[1].y, m.c[2].y};
  r.c[2] = {m.c[0].z, m.c[1].z, m.c[2].z};
  return r;
}
template <typename T> static inline M3<T> mat_add(const M3<T>& a, const M3<T>& b) {
  M3<T> r; for (int j = 0; j < 3; ++j) r.c[j] = add3(a.c[j], b.c[j]); return r;
}
template <typename T> static inline T elem(const M3<T>& m, int col, int row) { return comp(m.c[col], row); }

// quat (w,x,y,z) -> column-major rotation, project_gaussians.wgsl:68-80
template <typename T> static M3<T> quat_to_mat3(T w, T x, T y, T z) {
  const T one = T(1), two = T(2);
  M3<T> m;
  m.c[0] = {one - two * (y * y + z * z), two * (x * y + w * z), two * (x * z - w * y)};
  m.c[1] = {two * (x * y - w * z), one - two * (x * x + z * z), two * (y * z + w * x)};
  m.c[2] = {two * (x * z + w * y), two * (y * z - w * x), one - two * (x * x + y * y)};
  return m;
}

template <typename T> static inline T sigmoid(T x) { return T(1) / (T(1) + std::exp(-x)); }

template <typename T> static void sh_basis(V3<T> d, T b[15]) {
  const T x = d.x, y = d.y, z = d.z;
  const T xx = x * x, yy = y * y, zz = z * z;
  b[0] = -T(SH_C1) * y;  b[1] = T(SH_C1) * z;  b[2] = -T(SH_C1) * x;
  b[3] = T(SH_C2_0) * x * y;
  b[4] = T(SH_C2_1) * y * z;
  b[5] = T(SH_C2_2) * (T(2) * zz - xx - yy);
  b[6] = T(SH_C2_3) * x * z;
  b[7] = T(SH_C2_4) * (xx - yy);
  b[8] = T(SH_C3_0) * y * (T(3) * xx - yy);
  b[9] = T(SH_C3_1) * x * y * z;
  b[10] = T(SH_C3_2) * y * (T(4) * zz - xx - yy);
  b[11] = T(SH_C3_3) * z * (T(2) * zz - T(3) * xx - T(3) * yy);
  b[12] = T(SH_C3_4) * x * (T(4) * zz - xx - yy);
  b[13] = T(SH_C3_5) * z * (xx - yy);
  b[14] = T(SH_C3_6) * x * (xx - T(3) * yy);
}

// eval_sh, project_gaussians.wgsl:88-154
template <typename T> static V3<T> eval_sh(const float* dc, const float* rest, V3<T> dir) {
  V3<T> rgb = {T(SH_C0) * T(dc[0]), T(SH_C0) * T(dc[1]), T(SH_C0) * T(dc[2])};
  T b[15]; sh_basis(dir, b);
  T ar = 0, ag = 0, ab = 0;
  for (int i = 0; i < 3; ++i) { ar = ar + T(rest[i]) * b[i]; ag = ag + T(rest[15 + i]) * b[i]; ab = ab + T(rest[30 + i]) * b[i]; }
  for (int i = 0; i < 5; ++i) { ar = ar + T(rest[3 + i]) * b[3 + i]; ag = ag + T(rest[18 + i]) * b[3 + i]; ab = ab + T(rest[33 + i]) * b[3 + i]; }
  for (int i = 0; i < 7; ++i) { ar = ar + T(rest[8 + i]) * b[8 + i]; ag = ag + T(rest[23 + i]) * b[8 + i]; ab = ab + T(rest[38 + i]) * b[8 + i]; }
  rgb = {rgb.x + ar, rgb.y + ag, rgb.z + ab};
  return {std::max(rgb.x + T(0.5), T(0)), std::max(rgb.y + T(0.5), T(0)), std::max(rgb.z + T(0.5), T(0))};
}

// Shared forward intermediates of project_gaussians.wgsl / project_backward.wgsl.
template <typename T> struct ProjState {
  bool culled;
  V3<T> t;            // (cam.x, cam.y, depth)
  M3<T> R, W;
  V3<T> s2;
  V3<T> j0, j1;
  T s00, s01, s11, det;
  T ca, cb, cc;
};

template <typename T>
static ProjState<T> project_state(const HostSplats& s, uint32_t i, const Camera& cam) {
  ProjState<T> st{};
  const float* V = cam.view;
  const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
  // view * vec4(p, 1): columns V[0..3], V[4..7], V[8..11], V[12..15]
  T vx = T(V[0]) * px + T(V[4]) * py + T(V[8]) * pz + T(V[12]);
  T vy = T(V[1]) * px + T(V[5]) * py + T(V[9]) * pz + T(V[13]);
  T vz = T(V[2]) * px + T(V[6]) * py + T(V[10]) * pz + T(V[14]);
  T vw = T(V[3]) * px + T(V[7]) * py + T(V[11]) * pz + T(V[15]);
  V3<T> cam_xyz = {vx / vw, vy / vw, vz / vw};
  const T depth = -cam_xyz.z;
  if (depth < T(cam.near_plane)) { st.culled = true; return st; }
  st.t = {cam_xyz.x, cam_xyz.y, depth};
  st.R = quat_to_mat3<T>(s.rot[4 * i], s.rot[4 * i + 1], s.rot[4 * i + 2], s.rot[4 * i + 3]);
  V3<T> sigma = {std::exp(T(s.scale[3 * i])), std::exp(T(s.scale[3 * i + 1])), std::exp(T(s.scale[3 * i + 2]))};
  st.s2 = {sigma.x * sigma.x, sigma.y * sigma.y, sigma.z * sigma.z};
  M3<T> M; M.c[0] = mul3s(st.R.c[0], st.s2.x); M.c[1] = mul3s(st.R.c[1], st.s2.y); M.c[2] = mul3s(st.R.c[2], st.s2.z);
  M3<T> cov_w = mat_mul(M, transpose(st.R));
  st.W.c[0] = {T(V[0]), T(V[1]), T(V[2])};
  st.W.c[1] = {T(V[4]), T(V[5]), T(V[6])};
  st.W.c[2] = {T(V[8]), T(V[9]), T(V[10])};
  M3<T> cov_c = mat_mul(mat_mul(st.W, cov_w), transpose(st.W));
  const T inv_z = T(1) / st.t.z;
  const T inv_z2 = inv_z * inv_z;
  const T f = T(cam.focal);
  st.j0 = {f * inv_z, T(0), -f * st.t.x * inv_z2};
  st.j1 = {T(0), -f * inv_z, f * st.t.y * inv_z2};
  V3<T> r0 = mat_vec(cov_c, st.j0);
  V3<T> r1 = mat_vec(cov_c, st.j1);
  T s00 = dot3(r0, st.j0), s01 = dot3(r0, st.j1), s11 = dot3(r1, st.j1);
  s00 = s00 + T(0.3f);
  s11 = s11 + T(0.3f);
  st.s00 = s00; st.s01 = s01; st.s11 = s11;
  st.det = s00 * s11 - s01 * s01;
  if (st.det <= T(0)) { st.culled = true; return st; }
  const T inv_det = T(1) / st.det;
  st.ca = s11 * inv_det; st.cb = -s01 * inv_det; st.cc = s00 * inv_det;
  st.culled = false;
  return st;
}

// project_gaussians.wgsl:156-259, one splat
template <typename T>
static void project_one(const HostSplats& s, uint32_t i, const Camera& cam, T* out) {
  for (int k = 0; k < 12; ++k) out[k] = T(0);
  ProjState<T> st = project_state<T>(s, i, cam);
  if (st.culled) return;
  const T cx = T(cam.width) * T(0.5), cy = T(cam.height) * T(0.5);
  const T f = T(cam.focal);
  const T mx = cx + (f * st.t.x) / st.t.z;
  const T my = cy - (f * st.t.y) / st.t.z;
  const T mid = T(0.5) * (st.s00 + st.s11);
  const T lambda = mid + std::sqrt(std::max(mid * mid - st.det, T(0)));
  const T radius = std::ceil(T(3) * std::sqrt(lambda));
  const T W_ = T(cam.width), H_ = T(cam.height);
  const T max_pixel = std::max(W_, H_) + radius;
  if (mx < -radius || mx >= W_ + radius || my < -radius || my >= H_ + radius || radius >= max_pixel) return;
  V3<T> d = {T(cam.cam_pos[0]) - T(s.pos[3 * i]), T(cam.cam_pos[1]) - T(s.pos[3 * i + 1]),
             T(cam.cam_pos[2]) - T(s.pos[3 * i + 2])};
  const T len = std::sqrt(dot3(d, d));
  V3<T> dir = {d.x / len, d.y / len, d.z / len};
  V3<T> rgb = eval_sh<T>(s.sh_dc + 3 * i, s.sh_rest + 45 * i, dir);
  out[R_MX] = mx; out[R_MY] = my; out[R_DEPTH] = st.t.z; out[R_RADIUS] = radius;
  out[R_CA] = st.ca; out[R_CB] = st.cb; out[R_CC] = st.cc; out[R_VIS] = T(1);
  out[R_R] = rgb.x; out[R_G] = rgb.y; out[R_B] = rgb.z;
  out[R_OP] = sigmoid<T>(T(s.opacity[i]));
}

template <typename T>
static void project_all(const HostSplats& s, const Camera& cam, T* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)s.n; ++i) project_one<T>(s, (uint32_t)i, cam, out + 12 * i);
}

// ---------------------------------------------------------------- binning
struct TileRect { int32_t x0, y0, x1, y1; bool empty; };

// tile bbox, tile_count.wgsl:40-50 / tile_emit.wgsl:47-52 (tile_w / tile_h generalise ts)
template <typename T> static TileRect tile_rect(const T* rec, const Tiling& tl) {
  TileRect r{0, 0, -1, -1, true};
  if (rec[R_VIS] == T(0)) return r;
  const float mx = (float)rec[R_MX], my = (float)rec[R_MY], rad = (float)rec[R_RADIUS];
  const float tw = (float)tl.tile_w, th = (float)tl.tile_h;
  r.x0 = std::max((int32_t)std::floor((mx - rad) / tw), 0);
  r.y0 = std::max((int32_t)std::floor((my - rad) / th), 0);
  r.x1 = std::min((int32_t)std::floor((mx + rad) / tw), (int32_t)tl.tiles_x() - 1);
  r.y1 = std::min((int32_t)std::floor((my + rad) / th), (int32_t)tl.tiles_y() - 1);
  r.empty = (r.x1 < r.x0 || r.y1 < r.y0);
  return r;
}

// depth quantisation, tile_emit.wgsl:54-55
template <typename T> static uint32_t depth16(const T* rec, float depth_max) {
  float d = (float)rec[R_DEPTH] / depth_max;
  d = std::min(std::max(d, 0.0f), 1.0f);
  return (uint32_t)(d * 65535.0f);
}

static inline uint32_t float_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// Reference binning: count -> exclusive scan -> emit (splat, ty, tx) -> stable sort by
// 32-bit key -> ranges.  Returns total pairs, or -(needed) when cap is too small.
template <typename T>
static int64_t bin_ref(uint32_t n, const T* rec, const Tiling& tl, uint32_t* keys, uint32_t* payloads,
                       uint64_t cap, uint32_t* ranges) {
  const uint32_t ntiles = tl.num_tiles();
  std::vector<uint64_t> offs(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i) {
    TileRect r = tile_rect(rec + 12 * i, tl);
    uint64_t c = r.empty ? 0 : (uint64_t)(r.x1 - r.x0 + 1) * (uint64_t)(r.y1 - r.y0 + 1);
    offs[i + 1] = offs[i] + c;
  }
  const uint64_t K = offs[n];
  for (uint32_t t = 0; t < 2 * ntiles; ++t) ranges[t] = 0;
  if (K > cap) return -(int64_t)K;
  std::vector<uint32_t> k0(K), p0(K);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    TileRect r = tile_rect(rec + 12 * i, tl);
    if (r.empty) continue;
    const uint32_t d = depth16(rec + 12 * i, tl.depth_max);
    uint64_t w = offs[i];
    for (int32_t ty = r.y0; ty <= r.y1; ++ty)
      for (int32_t tx = r.x0; tx <= r.x1; ++tx) {
        const uint32_t tile = (uint32_t)ty * tl.tiles_x() + (uint32_t)tx;
        k0[w] = (tile << 16) | d; p0[w] = (uint32_t)i; ++w;
      }
  }
  std::vector<uint32_t> idx(K);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return k0[a] < k0[b]; });
  for (uint64_t j = 0; j < K; ++j) { keys[j] = k0[idx[j]]; payloads[j] = p0[idx[j]]; }
  // tile_ranges.wgsl:27-40
  for (uint64_t j = 0; j < K; ++j) {
    const uint32_t tile = keys[j] >> 16;
    const bool starts = (j == 0) || ((keys[j - 1] >> 16) != tile);
    const bool ends = (j + 1 == K) || ((keys[j + 1] >> 16) != tile);
    if (tile >= ntiles) continue;
    if (starts) ranges[2 * tile] = (uint32_t)j;
    if (ends) ranges[2 * tile + 1] = (uint32_t)(j + 1);
  }
  return (int64_t)K;
}

// Native binning (extension): keys = ((view*T + tile) << 32) | float_bits(depth), emitted in
// (view, splat, ty, tx) order and stably sorted.  Ranges are indexed by view*T + tile.
template <typename T>
static int64_t bin64(uint32_t n_views, uint32_t n, const T* rec, const Tiling& tl, uint64_t* keys,
                     uint32_t* payloads, uint64_t cap, uint32_t* ranges) {
  const uint32_t ntiles = tl.num_tiles();
  const uint64_t NV = (uint64_t)n_views * n;
  std::vector<uint64_t> offs(NV + 1, 0);
  for (uint64_t q = 0; q < NV; ++q) {
    TileRect r = tile_rect(rec + 12 * q, tl);
    uint64_t c = r.empty ? 0 : (uint64_t)(r.x1 - r.x0 + 1) * (uint64_t)(r.y1 - r.y0 + 1);
    offs[q + 1] = offs[q] + c;
  }
  const uint64_t K = offs[NV];
  for (uint64_t t = 0; t < 2ull * ntiles * n_views; ++t) ranges[t] = 0;
  if (K > cap) return -(int64_t)K;
  std::vector<uint64_t> k0(K);
  std::vector<uint32_t> p0(K);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t q = 0; q < (int64_t)NV; ++q) {
    TileRect r = tile_rect(rec + 12 * q, tl);
    if (r.empty) continue;
    const uint64_t view = (uint64_t)q / n;
    const uint32_t i = (uint32_t)((uint64_t)q % n);
    const uint32_t db = float_bits((float)rec[12 * q + R_DEPTH]);
    uint64_t w = offs[q];
    for (int32_t ty = r.y0; ty <= r.y1; ++ty)
      for (int32_t tx = r.x0; tx <= r.x1; ++tx) {
        const uint64_t tile = view * ntiles + (uint64_t)ty * tl.tiles_x() + (uint64_t)tx;
        k0[w] = (tile << 32) | db; p0[w] = i; ++w;
      }
  }
  std::vector<uint32_t> idx(K);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return k0[a] < k0[b]; });
  for (uint64_t j = 0; j < K; ++j) { keys[j] = k0[idx[j]]; payloads[j] = p0[idx[j]]; }
  for (uint64_t j = 0; j < K; ++j) {
    const uint64_t tile = keys[j] >> 32;
    const bool starts = (j == 0) || ((keys[j - 1] >> 32) != tile);
    const bool ends = (j + 1 == K) || ((keys[j + 1] >> 32) != tile);
    if (starts) ranges[2 * tile] = (uint32_t)j;
    if (ends) ranges[2 * tile + 1] = (uint32_t)(j + 1);
  }
  return (int64_t)K;
}

// ---------------------------------------------------------------- composite
static const float ALPHA_MIN = 1.0f / 255.0f;
static const float ALPHA_MAX = 0.99f;

// rasterize.wgsl:48-118.  One view; ranges indexed by tile.  n_contrib / t_final are the
// "exact" extension (nullable).
template <typename T>
static void composite(const T* rec, const uint32_t* payloads, const uint32_t* ranges, const Tiling& tl,
                      T* out, uint32_t* n_contrib, T* t_final) {
  const uint32_t tx_n = tl.tiles_x(), ty_n = tl.tiles_y();
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int64_t ty = 0; ty < (int64_t)ty_n; ++ty)
    for (int64_t tx = 0; tx < (int64_t)tx_n; ++tx) {
      const uint32_t tile = (uint32_t)ty * tx_n + (uint32_t)tx;
      const uint32_t begin = ranges[2 * tile], end = ranges[2 * tile + 1];
      for (uint32_t ly = 0; ly < tl.tile_h; ++ly)
        for (uint32_t lx = 0; lx < tl.tile_w; ++lx) {
          const uint32_t px = (uint32_t)tx * tl.tile_w + lx, py = (uint32_t)ty * tl.tile_h + ly;
          if (px >= tl.width || py >= tl.height) continue;
          const T pix_x = T((float)px + 0.5f), pix_y = T((float)py + 0.5f);
          T cr = 0, cg = 0, cb = 0, Tr = 1;
          uint32_t last = 0;
          for (uint32_t j = begin; j < end; ++j) {
            const T* p = rec + 12 * (size_t)payloads[j];
            const T dx = pix_x - p[R_MX], dy = pix_y - p[R_MY];
            const T power = T(-0.5) * (p[R_CA] * dx * dx + T(2) * p[R_CB] * dx * dy + p[R_CC] * dy * dy);
            if (power > T(0)) continue;
            const T g = std::exp(power);
            const T alpha_raw = p[R_OP] * g;
            const T alpha = std::min(alpha_raw, T(ALPHA_MAX));
            if (alpha < T(ALPHA_MIN)) continue;
            const T ta = Tr * alpha;
            cr = cr + ta * p[R_R]; cg = cg + ta * p[R_G]; cb = cb + ta * p[R_B];
            Tr = Tr * (T(1) - alpha);
            last = j - begin + 1;
            if (Tr < T(1e-4f)) break;
          }
          const size_t pi = (size_t)py * tl.width + px;
          out[4 * pi] = cr; out[4 * pi + 1] = cg; out[4 * pi + 2] = cb; out[4 * pi + 3] = T(1) - Tr;
          if (n_contrib) n_contrib[pi] = last;
          if (t_final) t_final[pi] = Tr;
        }
    }
}

// loss.rs:163-179 — dL/dC = 2 (p - t) / (3 W H); loss with an f64 accumulator.  scale multiplies
// the gradient (1/V for a V-view mean loss; 1 reproduces the reference).
template <typename T>
static double mse(uint64_t P, const T* pred4, const float* target3, T* dl_dc4, float scale) {
  const float n_scalars = (float)P * 3.0f;  // (width as f32) * (height as f32) * 3.0
  const T inv_n = T(2.0f / n_scalars) * T(scale);
  double sum = 0.0;
  for (uint64_t i = 0; i < P; ++i) {
    const T dx = pred4[4 * i] - T(target3[3 * i]);
    const T dy = pred4[4 * i + 1] - T(target3[3 * i + 1]);
    const T dz = pred4[4 * i + 2] - T(target3[3 * i + 2]);
    sum += (double)(dx * dx + dy * dy + dz * dz);
    dl_dc4[4 * i] = dx * inv_n; dl_dc4[4 * i + 1] = dy * inv_n; dl_dc4[4 * i + 2] = dz * inv_n; dl_dc4[4 * i + 3] = T(0);
  }
  return sum / ((double)P * 3.0);
}

// ---------------------------------------------------------------- SSIM (loss.rs:22-375)
// Wang et al. 2004 structural similarity over an 11-tap separable Gaussian
// window (sigma 1.5) with reflect-101 padding, C1 = 1e-4, C2 = 9e-4, and the
// reference's analytic gradient: three quotient-rule coefficient planes
// P = dSSIM/dmu_x, Q = dSSIM/dsigma_x^2, R = dSSIM/dsigma_xy pulled back
// through the adjoint of the blur (loss.rs:193-335).
static const int SSIM_WIN = 11;
static const int SSIM_RAD = 5;
static const float SSIM_C1 = 0.0001f;
static const float SSIM_C2 = 0.0009f;

// loss.rs:36-51, in f32 like the reference
static void ssim_window(float g[SSIM_WIN]) {
  const float centre = (float)(SSIM_WIN - 1) * 0.5f;
  const float two_sigma_sq = 2.0f * 1.5f * 1.5f;
  float sum = 0.0f;
  for (int i = 0; i < SSIM_WIN; ++i) {
    const float d = (float)i - centre;
    g[i] = std::exp(-d * d / two_sigma_sq);
    sum += g[i];
  }
  for (int i = 0; i < SSIM_WIN; ++i) g[i] /= sum;
}

// loss.rs:56-67: reflect-101 index into [0, n)
static inline int reflect101(int i, int n) {
  if (n == 1) return 0;
  const int period = 2 * (n - 1);
  int x = ((i % period) + period) % period;
  if (x >= n) x = period - x;
  return x;
}

// loss.rs:73-100: horizontal then vertical gather pass
template <typename T>
static void ssim_blur(const T* src, int w, int h, const float* g, T* dst) {
  std::vector<T> tmp((size_t)w * h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      T acc = T(0);
      for (int k = 0; k < SSIM_WIN; ++k) acc += src[(size_t)y * w + reflect101(x + k - SSIM_RAD, w)] * T(g[k]);
      tmp[(size_t)y * w + x] = acc;
    }
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      T acc = T(0);
      for (int k = 0; k < SSIM_WIN; ++k) acc += tmp[(size_t)reflect101(y + k - SSIM_RAD, h) * w + x] * T(g[k]);
      dst[(size_t)y * w + x] = acc;
    }
}

// loss.rs:122-152: transpose of ssim_blur, vertical scatter then horizontal scatter
template <typename T>
static void ssim_blur_adjoint(const T* src, int w, int h, const float* g, T* dst) {
  std::vector<T> tmp((size_t)w * h, T(0));
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const T s = src[(size_t)y * w + x];
      for (int k = 0; k < SSIM_WIN; ++k) tmp[(size_t)reflect101(y + k - SSIM_RAD, h) * w + x] += s * T(g[k]);
    }
  std::fill(dst, dst + (size_t)w * h, T(0));
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const T s = tmp[(size_t)y * w + x];
      for (int k = 0; k < SSIM_WIN; ++k) dst[(size_t)y * w + reflect101(x + k - SSIM_RAD, w)] += s * T(g[k]);
    }
}

// loss.rs:193-335 for one channel plane: returns sum of the SSIM map (f64)
// and writes dSSIM/dx (before the -1/N and channel-average factors).
template <typename T>
static double ssim_channel(const T* x, const T* y, int w, int h, const float* g, T* dssim) {
  const size_t n = (size_t)w * h;
  std::vector<T> xx(n), yy(n), xy(n), mx(n), my(n), gxx(n), gyy(n), gxy(n);
  for (size_t i = 0; i < n; ++i) { xx[i] = x[i] * x[i]; yy[i] = y[i] * y[i]; xy[i] = x[i] * y[i]; }
  ssim_blur(x, w, h, g, mx.data());
  ssim_blur(y, w, h, g, my.data());
  ssim_blur(xx.data(), w, h, g, gxx.data());
  ssim_blur(yy.data(), w, h, g, gyy.data());
  ssim_blur(xy.data(), w, h, g, gxy.data());
  std::vector<T> p(n), q(n), r(n), mq(n), mr(n);
  double sum = 0.0;
  const T c1 = T(SSIM_C1), c2 = T(SSIM_C2);
  for (size_t i = 0; i < n; ++i) {
    const T mux = mx[i], muy = my[i];
    const T mux2 = mux * mux, muy2 = muy * muy;
    const T sxx = gxx[i] - mux2, syy = gyy[i] - muy2, sxy = gxy[i] - mux * muy;
    const T a = T(2) * mux * muy + c1, b = T(2) * sxy + c2;
    const T c = mux2 + muy2 + c1, d = sxx + syy + c2;
    sum += (double)((a * b) / (c * d));
    const T cd = c * d;
    p[i] = T(2) * b * (muy * c - mux * a) / (c * cd);
    q[i] = -a * b / (c * d * d);
    r[i] = T(2) * a / cd;
    mq[i] = mux * q[i];
    mr[i] = muy * r[i];
  }
  std::vector<T> sp(n), sq(n), sr(n), smq(n), smr(n);
  ssim_blur_adjoint(p.data(), w, h, g, sp.data());
  ssim_blur_adjoint(q.data(), w, h, g, sq.data());
  ssim_blur_adjoint(r.data(), w, h, g, sr.data());
  ssim_blur_adjoint(mq.data(), w, h, g, smq.data());
  ssim_blur_adjoint(mr.data(), w, h, g, smr.data());
  for (size_t i = 0; i < n; ++i)
    dssim[i] = sp[i] + T(2) * (x[i] * sq[i] - smq[i]) + (y[i] * sr[i] - smr[i]);
  return sum;
}

// loss.rs:340-375 on an rgba prediction and rgb target: loss = 1 - mean of the
// three channel SSIMs; dl_dc4 = scale * dL/dC (alpha lane zero).
template <typename T>
static double ssim_loss_grad(int w, int h, const T* pred4, const float* target3, T* dl_dc4, float scale) {
  float g[SSIM_WIN];
  ssim_window(g);
  const size_t n = (size_t)w * h;
  std::vector<T> xc(n), yc(n), ds(n);
  T lc[3];
  const T inv_n = T(1.0f / (float)n);
  for (int ch = 0; ch < 3; ++ch) {
    for (size_t i = 0; i < n; ++i) { xc[i] = pred4[4 * i + ch]; yc[i] = T(target3[3 * i + ch]); }
    const double sum = ssim_channel(xc.data(), yc.data(), w, h, g, ds.data());
    lc[ch] = T(1) - (T)(sum / (double)n);
    for (size_t i = 0; i < n; ++i) dl_dc4[4 * i + ch] = (-inv_n * ds[i]) / T(3) * T(scale);
  }
  for (size_t i = 0; i < n; ++i) dl_dc4[4 * i + 3] = T(0);
  return (double)((lc[0] + lc[1] + lc[2]) / T(3));
}

// loss.rs:383-410: (1 - lambda) MSE + lambda (1 - SSIM); lambda 0 is the pure
// MSE path bit for bit, lambda 1 the pure SSIM path.  scale multiplies the
// gradient (1/V for a V-view mean).  parts (nullable) = {mse, ssim}.
template <typename T>
static double combined_loss_grad(int w, int h, const T* pred4, const float* target3, T* dl_dc4, float lambda,
                                 float scale, double* parts) {
  lambda = std::min(std::max(lambda, 0.0f), 1.0f);
  const uint64_t P = (uint64_t)w * h;
  if (lambda == 0.0f) {
    const double m = mse<T>(P, pred4, target3, dl_dc4, scale);
    if (parts) { parts[0] = m; parts[1] = 0.0; }
    return m;
  }
  if (lambda == 1.0f) {
    const double sv = ssim_loss_grad<T>(w, h, pred4, target3, dl_dc4, scale);
    if (parts) { parts[0] = 0.0; parts[1] = sv; }
    return sv;
  }
  std::vector<T> gm(4 * P), gs(4 * P);
  const double m = mse<T>(P, pred4, target3, gm.data(), 1.0f);
  const double sv = ssim_loss_grad<T>(w, h, pred4, target3, gs.data(), 1.0f);
  const T om = T(1.0f - lambda), l = T(lambda);
  for (uint64_t k = 0; k < 4 * P; ++k) dl_dc4[k] = (gm[k] * om + gs[k] * l) * T(scale);
  if (parts) { parts[0] = m; parts[1] = sv; }
  return (double)(om * (T)m + l * (T)sv);
}

template <typename T> static inline void atomic_add(T* p, T v) {
#pragma omp atomic
  *p += v;
}

// rasterize_backward.wgsl:73-210 ("ref" mode, mode == 0) and the exact extension (mode == 1:
// start at the forward's last contributor with the recorded final transmittance, no T bail).
// abs_grad (nullable, test diagnostics): receives per component the sum over pixels of the
// magnitude of each pixel's term taken before any cancellation (every product and sum that
// forms the term replaced by its absolute value), the scale that bounds the rounding error
// of the gradient sum, including the cancellation in T c - S / (1 - alpha).
template <typename T>
static void composite_backward(const T* rec, const uint32_t* payloads, const uint32_t* ranges,
                               const Tiling& tl, const T* fwd_out, const T* dl_dc, int mode,
                               const uint32_t* n_contrib, const T* t_final, T* proj_grad, T* abs_grad = nullptr) {
  const uint32_t tx_n = tl.tiles_x(), ty_n = tl.tiles_y();
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int64_t ty = 0; ty < (int64_t)ty_n; ++ty)
    for (int64_t tx = 0; tx < (int64_t)tx_n; ++tx) {
      const uint32_t tile = (uint32_t)ty * tx_n + (uint32_t)tx;
      const uint32_t begin = ranges[2 * tile], end = ranges[2 * tile + 1];
      if (end <= begin) continue;
      for (uint32_t ly = 0; ly < tl.tile_h; ++ly)
        for (uint32_t lx = 0; lx < tl.tile_w; ++lx) {
          const uint32_t px = (uint32_t)tx * tl.tile_w + lx, py = (uint32_t)ty * tl.tile_h + ly;
          if (px >= tl.width || py >= tl.height) continue;
          const size_t pi = (size_t)py * tl.width + px;
          const T pix_x = T((float)px + 0.5f), pix_y = T((float)py + 0.5f);
          T Tr;
          uint32_t stop = end;
          if (mode == 0) {
            Tr = T(1) - fwd_out[4 * pi + 3];
          } else {
            Tr = t_final[pi];
            stop = begin + n_contrib[pi];
          }
          const T gr = dl_dc[4 * pi], gg = dl_dc[4 * pi + 1], gb = dl_dc[4 * pi + 2];
          T Sr = 0, Sg = 0, Sb = 0;
          for (uint32_t jj = stop; jj > begin; --jj) {
            const uint32_t j = jj - 1;
            const uint32_t sidx = payloads[j];
            const T* p = rec + 12 * (size_t)sidx;
            const T dx = pix_x - p[R_MX], dy = pix_y - p[R_MY];
            const T power = T(-0.5) * (p[R_CA] * dx * dx + T(2) * p[R_CB] * dx * dy + p[R_CC] * dy * dy);
            if (power > T(0)) continue;
            const T g = std::exp(power);
            const T sigma = p[R_OP];
            const T alpha_raw = sigma * g;
            const T alpha = std::min(alpha_raw, T(ALPHA_MAX));
            if (alpha < T(ALPHA_MIN)) continue;
            const T oma = std::max(T(1) - alpha, T(1e-4f));
            Tr = Tr / oma;
            if (mode == 0 && Tr > T(1.0001f)) break;
            const T ta = Tr * alpha;
            const T cr = ta * p[R_R], cg = ta * p[R_G], cb = ta * p[R_B];
            const T dCr = gr * ta, dCg = gg * ta, dCb = gb * ta;
            const T da_r = Tr * p[R_R] - Sr / oma, da_g = Tr * p[R_G] - Sg / oma, da_b = Tr * p[R_B] - Sb / oma;
            const T grad_alpha = gr * da_r + gg * da_g + gb * da_b;
            const T sat = alpha_raw < T(ALPHA_MAX) ? T(1) : T(0);
            const T gar = grad_alpha * sat;
            const T gsig = gar * g;
            const T gpow = gar * sigma * g;
            const T ga = gpow * T(-0.5) * (dx * dx);
            const T gbb = gpow * T(-0.5) * (T(2) * dx * dy);
            const T gc = gpow * T(-0.5) * (dy * dy);
            const T gmx = gpow * (p[R_CA] * dx + p[R_CB] * dy);
            const T gmy = gpow * (p[R_CB] * dx + p[R_CC] * dy);
            T* o = proj_grad + 12 * (size_t)sidx;
            atomic_add(&o[G_MX], gmx); atomic_add(&o[G_MY], gmy); atomic_add(&o[G_OP], gsig);
            atomic_add(&o[G_CA], ga); atomic_add(&o[G_CB], gbb); atomic_add(&o[G_CC], gc);
            atomic_add(&o[G_R], dCr); atomic_add(&o[G_G], dCg); atomic_add(&o[G_B], dCb);
            if (abs_grad) {
              const T gabs = sat * (std::abs(gr) * (std::abs(Tr * p[R_R]) + std::abs(Sr / oma)) +
                                    std::abs(gg) * (std::abs(Tr * p[R_G]) + std::abs(Sg / oma)) +
                                    std::abs(gb) * (std::abs(Tr * p[R_B]) + std::abs(Sb / oma)));
              const T pabs = gabs * sigma * g;
              T* q = abs_grad + 12 * (size_t)sidx;
              atomic_add(&q[G_MX], pabs * (std::abs(p[R_CA] * dx) + std::abs(p[R_CB] * dy)));
              atomic_add(&q[G_MY], pabs * (std::abs(p[R_CB] * dx) + std::abs(p[R_CC] * dy)));
              atomic_add(&q[G_OP], gabs * g);
              atomic_add(&q[G_CA], pabs * T(0.5) * (dx * dx));
              atomic_add(&q[G_CB], pabs * std::abs(dx * dy));
              atomic_add(&q[G_CC], pabs * T(0.5) * (dy * dy));
              atomic_add(&q[G_R], std::abs(dCr)); atomic_add(&q[G_G], std::abs(dCg));
              atomic_add(&q[G_B], std::abs(dCb));
            }
            Sr = Sr + cr; Sg = Sg + cg; Sb = Sb + cb;
          }
        }
    }
}

// ---------------------------------------------------------------- near-threshold diagnostics
// Test infrastructure with no counterpart in the reference.  The blend makes
// discontinuous decisions: skip a pair when the quadratic form is negative
// (power > 0) or alpha < 1/255, gate the opacity gradient at alpha_raw < 0.99,
// stop a pixel when T < 1e-4 after a blend (forward) or when the recomputed T
// exceeds 1.0001 (the reference backward, mode 0).  Arithmetic that differs
// from this oracle's only by rounding (another exp, another operation order)
// can take the other branch of such a test only where the compared quantity
// lies within its rounding error of the threshold: thr_a (relative) for the
// per-pair tests, thr_t for the transmittance tests, whose errors accumulate
// along a walk.
//
// margin[pixel]: the smallest distance of the pixel's forward walk to a
// threshold, in units of that test's thr (below 1: the pixel may render
// differently).  flags[splat] bit 0: the splat is in a pixel's walk at or
// before a near-threshold pair test (or, mode 0, a near-threshold backward
// stop), so its gradient from that pixel may differ even when the backward
// gets the same forward image and aux; bit 1: the splat is in the walk of a
// pixel whose forward may differ (any near test, a near stop extended to the
// next pair the pixel would blend), so its gradient may differ when each side
// differentiates its own forward.
template <typename T>
static void composite_margins(const T* rec, const uint32_t* payloads, const uint32_t* ranges, const Tiling& tl,
                              int mode, double thr_a, double thr_t, float* margin, uint8_t* flags) {
  const uint32_t tx_n = tl.tiles_x(), ty_n = tl.tiles_y();
  const double amin = (double)ALPHA_MIN, amax = (double)ALPHA_MAX;
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int64_t ty = 0; ty < (int64_t)ty_n; ++ty)
    for (int64_t tx = 0; tx < (int64_t)tx_n; ++tx) {
      const uint32_t tile = (uint32_t)ty * tx_n + (uint32_t)tx;
      const uint32_t begin = ranges[2 * tile], end = std::max(ranges[2 * tile + 1], begin);
      for (uint32_t ly = 0; ly < tl.tile_h; ++ly)
        for (uint32_t lx = 0; lx < tl.tile_w; ++lx) {
          const uint32_t px = (uint32_t)tx * tl.tile_w + lx, py = (uint32_t)ty * tl.tile_h + ly;
          if (px >= tl.width || py >= tl.height) continue;
          const T pix_x = T((float)px + 0.5f), pix_y = T((float)py + 0.5f);
          // the alpha of position j (-1 when the sign test skips it) and the
          // pair tests' distances in units of thr_a: da (skip tests), dg (0.99 gate)
          auto pair_at = [&](uint32_t j, double& da, double& dg) -> T {
            const T* p = rec + 12 * (size_t)payloads[j];
            const T dx = pix_x - p[R_MX], dy = pix_y - p[R_MY];
            const T quad = p[R_CA] * dx * dx + T(2) * p[R_CB] * dx * dy + p[R_CC] * dy * dy;
            const double qabs = std::abs((double)p[R_CA] * dx * dx) + std::abs(2.0 * (double)p[R_CB] * dx * dy) +
                                std::abs((double)p[R_CC] * dy * dy);
            da = qabs > 0.0 ? std::abs((double)quad) / qabs / thr_a : 1e30;
            dg = 1e30;
            const T power = T(-0.5) * quad;
            if (power > T(0)) return T(-1);
            const T araw = p[R_OP] * std::exp(power);
            const T alpha = std::min(araw, T(ALPHA_MAX));
            da = std::min(da, std::abs((double)alpha - amin) / amin / thr_a);
            if (alpha >= T(ALPHA_MIN)) dg = std::abs((double)araw - amax) / amax / thr_a;
            return alpha;
          };
          double m = 1e30;         // forward walk, any test
          int64_t k_pair = -1;     // last position with a near pair test (the gate: itself only)
          std::vector<uint32_t> gate_near;
          T Tr = 1;
          bool t_near = false;
          uint32_t j = begin;
          for (; j < end; ++j) {
            double da, dg;
            const T alpha = pair_at(j, da, dg);
            m = std::min(m, std::min(da, dg));
            if (da < 1.0) k_pair = j;
            if (dg < 1.0) gate_near.push_back(j);
            if (alpha < T(ALPHA_MIN)) continue;
            Tr = Tr * (T(1) - alpha);
            const double dt = std::abs((double)Tr - 1e-4) / 1e-4 / thr_t;
            m = std::min(m, dt);
            if (Tr < T(1e-4f)) {
              t_near = dt < 1.0;
              break;
            }
          }
          uint32_t walk_end = j < end ? j + 1 : end;  // one past the forward's last position
          if (t_near)  // the stop may move to the next pair this pixel would blend
            for (uint32_t k = walk_end; k < end; ++k) {
              double da, dg;
              walk_end = k + 1;
              if (pair_at(k, da, dg) >= T(ALPHA_MIN)) break;
            }
          if (mode == 0) {  // the reference backward walks every entry from the end of the list
            T Tb = T(1) - (T(1) - Tr);
            for (uint32_t jj = end; jj > begin; --jj) {
              double da, dg;
              const T alpha = pair_at(jj - 1, da, dg);
              if (da < 1.0) k_pair = std::max<int64_t>(k_pair, (int64_t)jj - 1);
              if (dg < 1.0) gate_near.push_back(jj - 1);
              if (alpha < T(ALPHA_MIN)) continue;
              Tb = Tb / std::max(T(1) - alpha, T(1e-4f));
              const double db = std::abs((double)Tb - 1.0001) / 1.0001 / thr_t;
              if (db < 1.0) k_pair = std::max<int64_t>(k_pair, (int64_t)jj - 1);
              if (Tb > T(1.0001f)) break;
            }
          }
          margin[(size_t)py * tl.width + px] = (float)std::min(m, 1e30);
          if (!flags) continue;
          for (int64_t k = begin; k <= k_pair; ++k) {
#pragma omp atomic update
            flags[payloads[k]] |= (uint8_t)1;
          }
          for (uint32_t k : gate_near) {
#pragma omp atomic update
            flags[payloads[k]] |= (uint8_t)1;
          }
          if (m < 1.0)
            for (uint32_t k = begin; k < walk_end; ++k) {
#pragma omp atomic update
              flags[payloads[k]] |= (uint8_t)2;
            }
        }
    }
}

// project_backward.wgsl:79-304.  accumulate != 0 adds into grads (multi-view sum), otherwise
// overwrites like the reference.
template <typename T>
static void project_backward_one(const HostSplats& s, uint32_t i, const T* pg, const Camera& cam,
                                 HostGrads<T>& g, int accumulate) {
  T dpos[3] = {0, 0, 0}, drot[4] = {0, 0, 0, 0}, dsc[3] = {0, 0, 0}, dop = 0, ddc[3] = {0, 0, 0}, drest[45];
  for (int k = 0; k < 45; ++k) drest[k] = 0;
  ProjState<T> st = project_state<T>(s, i, cam);
  if (!st.culled) {
    const T f = T(cam.focal);
    const T inv_z = T(1) / st.t.z, inv_z2 = inv_z * inv_z;
    const T dmx = pg[G_MX], dmy = pg[G_MY], dsig = pg[G_OP];
    const T dca = pg[G_CA], dcb = pg[G_CB], dcc = pg[G_CC];
    const T dcr = pg[G_R], dcg = pg[G_G], dcbl = pg[G_B];
    const T os = sigmoid<T>(T(s.opacity[i]));
    dop = dsig * os * (T(1) - os);
    V3<T> d = {T(cam.cam_pos[0]) - T(s.pos[3 * i]), T(cam.cam_pos[1]) - T(s.pos[3 * i + 1]),
               T(cam.cam_pos[2]) - T(s.pos[3 * i + 2])};
    const T len = std::sqrt(dot3(d, d));
    V3<T> dir = {d.x / len, d.y / len, d.z / len};
    ddc[0] = dcr * T(SH_C0); ddc[1] = dcg * T(SH_C0); ddc[2] = dcbl * T(SH_C0);
    T b[15]; sh_basis(dir, b);
    for (int k = 0; k < 15; ++k) { drest[k] = dcr * b[k]; drest[15 + k] = dcg * b[k]; drest[30 + k] = dcbl * b[k]; }
    // dSigma2D = -(C * dconic_mat * C), dconic_mat off-diagonal halved (:203-217)
    const T C00 = st.ca, C01 = st.cb, C11 = st.cc;
    const T D00 = dca, D01 = dcb * T(0.5), D11 = dcc;
    // (C * D): column-major 2x2 products
    const T P00 = C00 * D00 + C01 * D01, P10 = C01 * D00 + C11 * D01;   // col 0 of C*D (rows 0,1)
    const T P01 = C00 * D01 + C01 * D11, P11 = C01 * D01 + C11 * D11;   // col 1
    // (C*D) * C
    const T Q00 = P00 * C00 + P01 * C01, Q10 = P10 * C00 + P11 * C01;
    const T Q01 = P00 * C01 + P01 * C11, Q11 = P10 * C01 + P11 * C11;
    const T ds00 = T(-1) * Q00, ds11 = T(-1) * Q11;
    const T ds01 = (T(-1) * Q01) + (T(-1) * Q10);
    // dsigma_2d matrix, element (row a, col b)
    T dS[2][2] = {{ds00, ds01 * T(0.5)}, {ds01 * T(0.5), ds11}};
    T dcc00 = 0, dcc01 = 0, dcc02 = 0, dcc11 = 0, dcc12 = 0, dcc22 = 0;
    for (int a = 0; a < 2; ++a)
      for (int bb = 0; bb < 2; ++bb) {
        const T coef = dS[a][bb];
        const V3<T> ja = a == 0 ? st.j0 : st.j1;
        const V3<T> jb = bb == 0 ? st.j0 : st.j1;
        dcc00 = dcc00 + ja.x * coef * jb.x;
        dcc01 = dcc01 + ja.x * coef * jb.y;
        dcc02 = dcc02 + ja.x * coef * jb.z;
        dcc11 = dcc11 + ja.y * coef * jb.y;
        dcc12 = dcc12 + ja.y * coef * jb.z;
        dcc22 = dcc22 + ja.z * coef * jb.z;
      }
    M3<T> dcov_cam;
    dcov_cam.c[0] = {dcc00, dcc01, dcc02};
    dcov_cam.c[1] = {dcc01, dcc11, dcc12};
    dcov_cam.c[2] = {dcc02, dcc12, dcc22};
    M3<T> dcw = mat_mul(mat_mul(transpose(st.W), dcov_cam), st.W);
    M3<T> RS2; RS2.c[0] = mul3s(st.R.c[0], st.s2.x); RS2.c[1] = mul3s(st.R.c[1], st.s2.y); RS2.c[2] = mul3s(st.R.c[2], st.s2.z);
    M3<T> dR = mat_mul(mat_add(dcw, transpose(dcw)), RS2);
    // G[row][col] = dR[col][row]
    const T G00 = elem(dR, 0, 0), G10 = elem(dR, 0, 1), G20 = elem(dR, 0, 2);
    const T G01 = elem(dR, 1, 0), G11 = elem(dR, 1, 1), G21 = elem(dR, 1, 2);
    const T G02 = elem(dR, 2, 0), G12 = elem(dR, 2, 1), G22 = elem(dR, 2, 2);
    const T d_s2_x = dot3(st.R.c[0], mat_vec(dcw, st.R.c[0]));
    const T d_s2_y = dot3(st.R.c[1], mat_vec(dcw, st.R.c[1]));
    const T d_s2_z = dot3(st.R.c[2], mat_vec(dcw, st.R.c[2]));
    dsc[0] = d_s2_x * T(2) * st.s2.x; dsc[1] = d_s2_y * T(2) * st.s2.y; dsc[2] = d_s2_z * T(2) * st.s2.z;
    const T qw = s.rot[4 * i], qx = s.rot[4 * i + 1], qy = s.rot[4 * i + 2], qz = s.rot[4 * i + 3];
    drot[0] = T(2) * (qz * (G10 - G01) + qy * (G02 - G20) + qx * (G21 - G12));
    drot[1] = T(2) * (qy * (G01 + G10) + qz * (G02 + G20) + qw * (G21 - G12)) - T(4) * qx * (G11 + G22);
    drot[2] = T(-4) * qy * (G00 + G22) + T(2) * (qx * (G01 + G10) + qw * (G02 - G20) + qz * (G12 + G21));
    drot[3] = T(-4) * qz * (G00 + G11) + T(2) * (qw * (G10 - G01) + qx * (G02 + G20) + qy * (G12 + G21));
    // position (:288-303)
    const V3<T> dtx = {f * inv_z, T(0), -f * st.t.x * inv_z2};
    const V3<T> dty = {T(0), -f * inv_z, f * st.t.y * inv_z2};
    const V3<T> dLdt = add3(mul3s(dtx, dmx), mul3s(dty, dmy));
    const V3<T> dLdcam = {dLdt.x, dLdt.y, -dLdt.z};
    const V3<T> dp = mat_vec(transpose(st.W), dLdcam);
    dpos[0] = dp.x; dpos[1] = dp.y; dpos[2] = dp.z;
  }
  auto put = [&](T* dst, const T* src, int cnt) {
    for (int k = 0; k < cnt; ++k) dst[k] = accumulate ? dst[k] + src[k] : src[k];
  };
  put(g.pos + 3 * (size_t)i, dpos, 3);
  put(g.rot + 4 * (size_t)i, drot, 4);
  put(g.scale + 3 * (size_t)i, dsc, 3);
  put(g.opacity + i, &dop, 1);
  put(g.sh_dc + 3 * (size_t)i, ddc, 3);
  put(g.sh_rest + 45 * (size_t)i, drest, 45);
}

template <typename T>
static void project_backward_all(const HostSplats& s, const T* pg, const Camera& cam, HostGrads<T>& g, int accumulate) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)s.n; ++i) project_backward_one<T>(s, (uint32_t)i, pg + 12 * i, cam, g, accumulate);
}

// ---------------------------------------------------------------- Adam & friends (f32)
// compiler-rt style square-and-multiply, the algorithm behind Rust's f32::powi
static float powi_f32(float a, int b) {
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

// adam.rs:70-90 (bias corrections from the host, adam_gpu.rs:275-276)
static void adam_lanes(uint64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                       float eps, uint64_t t) {
  const float bc1 = 1.0f - powi_f32(b1, (int)t);
  const float bc2 = 1.0f - powi_f32(b2, (int)t);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.0f - b1) * gi;
    v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
    const float m_hat = m[i] / bc1;
    const float v_hat = v[i] / bc2;
    p[i] -= lr * m_hat / (std::sqrt(v_hat) + eps);
  }
}

// apply_constraints.wgsl:24-41
static void apply_constraints(uint32_t n, float* rot, float* scale, float* op, float lsmin, float lsmax, float opmax) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    float* q = rot + 4 * i;
    const float n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    const float nrm = std::max(std::sqrt(n2), 1e-8f);
    for (int k = 0; k < 4; ++k) q[k] = q[k] / nrm;
    for (int k = 0; k < 3; ++k) scale[3 * i + k] = std::min(std::max(scale[3 * i + k], lsmin), lsmax);
    op[i] = std::min(std::max(op[i], -opmax), opmax);
  }
}

// accumulate_grad_pos.wgsl:17-23
static void accumulate_grad(uint32_t n, const float* dpos, float* acc) {
  for (uint32_t i = 0; i < n; ++i)
    acc[i] = acc[i] + std::fabs(dpos[3 * i]) + std::fabs(dpos[3 * i + 1]) + std::fabs(dpos[3 * i + 2]);
}

// ---------------------------------------------------------------- prune / densify
// A SoA vector view over HostSplats with capacity, supporting the reference's swap_remove /
// push_splat (splat_store.rs:99-132) and AdamState::grow / swap_remove_range (adam.rs:94-112).
struct Slabs {
  HostSplats* s; HostSplats* m; HostSplats* v; float* acc; uint32_t n;
  static void swap_attr(HostSplats* h, uint32_t i, uint32_t last) {
    auto sw = [&](float* a, int w) { for (int k = 0; k < w; ++k) std::swap(a[(size_t)w * i + k], a[(size_t)w * last + k]); };
    sw(h->pos, 3); sw(h->rot, 4); sw(h->scale, 3); sw(h->opacity, 1); sw(h->sh_dc, 3); sw(h->sh_rest, 45);
  }
  void swap_remove(uint32_t i) {
    const uint32_t last = n - 1;
    swap_attr(s, i, last);
    if (m) swap_attr(m, i, last);
    if (v) swap_attr(v, i, last);
    if (acc) std::swap(acc[i], acc[last]);
    n -= 1;
  }
  static void copy_from(HostSplats* h, uint32_t dst, const float* pos, const float* rot, const float* sc, float op,
                        const float* dc, const float* rest) {
    std::memcpy(h->pos + 3 * (size_t)dst, pos, 12); std::memcpy(h->rot + 4 * (size_t)dst, rot, 16);
    std::memcpy(h->scale + 3 * (size_t)dst, sc, 12); h->opacity[dst] = op;
    std::memcpy(h->sh_dc + 3 * (size_t)dst, dc, 12); std::memcpy(h->sh_rest + 45 * (size_t)dst, rest, 180);
  }
  static void zero_at(HostSplats* h, uint32_t dst) {
    static const float z[45] = {0};
    copy_from(h, dst, z, z, z, 0.0f, z, z);
  }
  void push(const float* pos, const float* rot, const float* sc, float op, const float* dc, const float* rest) {
    copy_from(s, n, pos, rot, sc, op, dc, rest);
    if (m) zero_at(m, n);
    if (v) zero_at(v, n);
    if (acc) acc[n] = 0.0f;
    n += 1;
  }
};

// train.rs:572-602
static uint32_t prune_low_opacity(Slabs& sl, float threshold) {
  std::vector<uint32_t> rm;
  for (uint32_t i = 0; i < sl.n; ++i) if (sl.s->opacity[i] < threshold) rm.push_back(i);
  std::sort(rm.begin(), rm.end(), [](uint32_t a, uint32_t b) { return a > b; });
  for (uint32_t i : rm) sl.swap_remove(i);
  return (uint32_t)rm.size();
}

// train.rs:552-564
static float lcg01(uint32_t* state) {
  *state = *state * 1664525u + 1013904223u;
  return (float)(*state) / ((float)UINT32_MAX + 1.0f);
}
static float box_muller(uint32_t* state) {
  const float u1 = std::max(lcg01(state), 1e-8f);
  const float u2 = lcg01(state);
  const float two_pi = 2.0f * 3.14159265358979323846f;
  return std::sqrt(-2.0f * std::log(u1)) * std::cos(two_pi * u2);
}

// quaternion (x,y,z,w) applied to a vector: v (w^2 - b.b) + b (2 b.v) + (b x v)(2w)
static void quat_rotate(const float q_xyzw[4], const float v[3], float out[3]) {
  const float bx = q_xyzw[0], by = q_xyzw[1], bz = q_xyzw[2], w = q_xyzw[3];
  const float b2 = bx * bx + by * by + bz * bz;
  const float vb2 = (v[0] * bx + v[1] * by + v[2] * bz) * 2.0f;
  const float ww = w * w - b2;
  const float cx = by * v[2] - v[1] * bz, cy = bz * v[0] - v[2] * bx, cz = bx * v[1] - v[0] * by;
  const float w2 = w * 2.0f;
  out[0] = (v[0] * ww + bx * vb2) + cx * w2;
  out[1] = (v[1] * ww + by * vb2) + cy * w2;
  out[2] = (v[2] * ww + bz * vb2) + cz * w2;
}

// train.rs:414-549
static void densify(Slabs& sl, uint32_t grad_count, float grad_threshold, float split_thr, uint32_t max_splats,
                    uint32_t iter, uint32_t out_counts[3]) {
  const uint32_t n_before = sl.n;
  const float count_f = (float)std::max(grad_count, 1u);
  std::vector<uint32_t> to_clone, to_split;
  uint64_t projected = n_before;
  for (uint32_t i = 0; i < n_before; ++i) {
    const float avg = sl.acc[i] / count_f;
    if (avg <= grad_threshold) continue;
    float mx = -std::numeric_limits<float>::infinity();
    for (int k = 0; k < 3; ++k) mx = std::fmax(mx, sl.s->scale[3 * i + k]);
    if (mx > split_thr) {
      if (projected < max_splats) { to_split.push_back(i); projected += 1; }
    } else if (projected < max_splats) {
      to_clone.push_back(i); projected += 1;
    }
  }
  uint32_t rng = iter * 1664525u + 1013904223u;
  const float half = -0.69314718055994530942f;       // -LN_2 as f32
  const float log_split = -std::log(1.6f);
  for (uint32_t i : to_clone) {
    float pos[3], rot[4], sc[3], dc[3], rest[45];
    std::memcpy(pos, sl.s->pos + 3 * (size_t)i, 12); std::memcpy(rot, sl.s->rot + 4 * (size_t)i, 16);
    std::memcpy(sc, sl.s->scale + 3 * (size_t)i, 12); std::memcpy(dc, sl.s->sh_dc + 3 * (size_t)i, 12);
    std::memcpy(rest, sl.s->sh_rest + 45 * (size_t)i, 180);
    const float op_new = sl.s->opacity[i] + half;
    sl.push(pos, rot, sc, op_new, dc, rest);
    sl.s->opacity[i] = op_new;
  }
  std::vector<uint32_t> parents;
  for (uint32_t i : to_split) {
    float pos[3], rot[4], sc[3], dc[3], rest[45];
    std::memcpy(pos, sl.s->pos + 3 * (size_t)i, 12); std::memcpy(rot, sl.s->rot + 4 * (size_t)i, 16);
    std::memcpy(sc, sl.s->scale + 3 * (size_t)i, 12); std::memcpy(dc, sl.s->sh_dc + 3 * (size_t)i, 12);
    std::memcpy(rest, sl.s->sh_rest + 45 * (size_t)i, 180);
    const float op = sl.s->opacity[i];
    const float nls[3] = {sc[0] + log_split, sc[1] + log_split, sc[2] + log_split};
    const float sig[3] = {std::exp(sc[0]), std::exp(sc[1]), std::exp(sc[2])};
    const float q[4] = {rot[1], rot[2], rot[3], rot[0]};
    for (int c = 0; c < 2; ++c) {
      float off[3];
      off[0] = box_muller(&rng) * sig[0];
      off[1] = box_muller(&rng) * sig[1];
      off[2] = box_muller(&rng) * sig[2];
      float r[3]; quat_rotate(q, off, r);
      const float np[3] = {pos[0] + r[0], pos[1] + r[1], pos[2] + r[2]};
      sl.push(np, rot, nls, op, dc, rest);
    }
    parents.push_back(i);
  }
  std::sort(parents.begin(), parents.end(), [](uint32_t a, uint32_t b) { return a > b; });
  for (uint32_t i : parents) sl.swap_remove(i);
  out_counts[0] = (uint32_t)to_clone.size();
  out_counts[1] = (uint32_t)to_split.size() * 2;
  out_counts[2] = (uint32_t)parents.size();
}

// ---------------------------------------------------------------- camera (raster.rs:79-99)
static void camera_from_pose(const float eye[3], const float target[3], const float up[3], float fov_y,
                             uint32_t w, uint32_t h, uint32_t n, Camera* out) {
  auto norm = [](float v[3]) {
    const float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const float r = 1.0f / len;
    v[0] *= r; v[1] *= r; v[2] *= r;
  };
  auto cross = [](const float a[3], const float b[3], float o[3]) {
    o[0] = a[1] * b[2] - b[1] * a[2];
    o[1] = a[2] * b[0] - b[2] * a[0];
    o[2] = a[0] * b[1] - b[0] * a[1];
  };
  float f[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
  norm(f);
  float s[3]; cross(f, up, s); norm(s);
  float u[3]; cross(s, f, u);
  auto d = [](const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  float* V = out->view;
  V[0] = s[0]; V[1] = u[0]; V[2] = -f[0]; V[3] = 0.0f;
  V[4] = s[1]; V[5] = u[1]; V[6] = -f[1]; V[7] = 0.0f;
  V[8] = s[2]; V[9] = u[2]; V[10] = -f[2]; V[11] = 0.0f;
  V[12] = -d(eye, s); V[13] = -d(eye, u); V[14] = d(eye, f); V[15] = 1.0f;
  out->cam_pos[0] = eye[0]; out->cam_pos[1] = eye[1]; out->cam_pos[2] = eye[2];
  out->near_plane = 0.01f;
  out->focal = (float)h / (2.0f * std::tan(fov_y * 0.5f));
  out->width = (float)w;
  out->height = (float)h;
  out->n_splats = n;
}

// ---------------------------------------------------------------- PLY (ply.rs)
static const char* kPlyProps[] = {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"};

static int write_ply(const char* path, const HostSplats& s) {
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return -1;
  std::string hdr = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(s.n) + "\n";
  for (const char* p : kPlyProps) hdr += std::string("property float ") + p + "\n";
  for (int i = 0; i < 45; ++i) hdr += "property float f_rest_" + std::to_string(i) + "\n";
  hdr += "property float opacity\n";
  for (int i = 0; i < 3; ++i) hdr += "property float scale_" + std::to_string(i) + "\n";
  for (int i = 0; i < 4; ++i) hdr += "property float rot_" + std::to_string(i) + "\n";
  hdr += "end_header\n";
  std::fwrite(hdr.data(), 1, hdr.size(), fp);
  std::vector<float> rec(62);
  for (uint32_t i = 0; i < s.n; ++i) {
    int k = 0;
    for (int c = 0; c < 3; ++c) rec[k++] = s.pos[3 * (size_t)i + c];
    rec[k++] = 0.0f; rec[k++] = 1.0f; rec[k++] = 0.0f;          // normal = +Y (splat_store.rs:85)
    for (int c = 0; c < 3; ++c) rec[k++] = s.sh_dc[3 * (size_t)i + c];
    for (int c = 0; c < 45; ++c) rec[k++] = s.sh_rest[45 * (size_t)i + c];
    rec[k++] = s.opacity[i];
    for (int c = 0; c < 3; ++c) rec[k++] = s.scale[3 * (size_t)i + c];
    for (int c = 0; c < 4; ++c) rec[k++] = s.rot[4 * (size_t)i + c];
    std::fwrite(rec.data(), 4, 62, fp);
  }
  std::fclose(fp);
  return 0;
}

// returns vertex count (>= 0) and fills `out` when its capacity suffices; -1 I/O, -2 format,
// -3 missing required property, -(1000 + count) when capacity is too small.
static int64_t read_ply(const char* path, HostSplats* out, uint32_t cap) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return -1;
  char line[512];
  if (!std::fgets(line, sizeof line, fp) || std::string(line).substr(0, 3) != "ply") { std::fclose(fp); return -2; }
  bool ble = false; uint64_t count = 0; std::vector<std::string> props;
  for (;;) {
    if (!std::fgets(line, sizeof line, fp)) { std::fclose(fp); return -2; }
    std::string t(line);
    while (!t.empty() && (t.back() == '\n' || t.back() == '\r' || t.back() == ' ')) t.pop_back();
    size_t a = t.find_first_not_of(' ');
    t = a == std::string::npos ? "" : t.substr(a);
    if (t.empty() || t.rfind("comment ", 0) == 0) continue;
    if (t == "end_header") break;
    if (t.rfind("format ", 0) == 0) { ble = t.rfind("format binary_little_endian", 0) == 0; continue; }
    if (t.rfind("element vertex ", 0) == 0) { count = std::strtoull(t.c_str() + 15, nullptr, 10); continue; }
    if (t.rfind("property float ", 0) == 0) { std::string nm = t.substr(15); while (!nm.empty() && nm.back() == ' ') nm.pop_back(); props.push_back(nm); continue; }
    if (t.rfind("element ", 0) == 0) continue;
    if (t.rfind("property ", 0) == 0) { std::fclose(fp); return -2; }
  }
  if (!ble) { std::fclose(fp); return -2; }
  auto off = [&](const std::string& nm) -> int { for (size_t i = 0; i < props.size(); ++i) if (props[i] == nm) return (int)i; return -1; };
  const char* req[] = {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
                       "rot_0", "rot_1", "rot_2", "rot_3"};
  for (const char* r : req) if (off(r) < 0) { std::fclose(fp); return -3; }
  if (count > cap) { std::fclose(fp); return -(int64_t)(1000 + count); }
  int rest_off[45];
  for (int i = 0; i < 45; ++i) rest_off[i] = off("f_rest_" + std::to_string(i));
  std::vector<float> rec(props.size());
  for (uint64_t i = 0; i < count; ++i) {
    if (std::fread(rec.data(), 4, props.size(), fp) != props.size()) { std::fclose(fp); return -1; }
    for (int c = 0; c < 3; ++c) out->pos[3 * i + c] = rec[off(std::string(1, "xyz"[c]))];
    for (int c = 0; c < 3; ++c) out->sh_dc[3 * i + c] = rec[off("f_dc_" + std::to_string(c))];
    for (int c = 0; c < 45; ++c) out->sh_rest[45 * i + c] = rest_off[c] >= 0 ? rec[rest_off[c]] : 0.0f;
    out->opacity[i] = rec[off("opacity")];
    for (int c = 0; c < 3; ++c) out->scale[3 * i + c] = rec[off("scale_" + std::to_string(c))];
    for (int c = 0; c < 4; ++c) out->rot[4 * i + c] = rec[off("rot_" + std::to_string(c))];
  }
  std::fclose(fp);
  out->n = (uint32_t)count;
  return (int64_t)count;
}

// ---------------------------------------------------------------- whole iteration
// One training iteration over n_views views (extension of train.rs:155-250 to several views
// per step with a mean loss): project -> bin_ref (the reference's 32-bit keys and order) ->
// composite -> MSE -> backward -> project backward (summed over views) -> accumulate ->
// Adam (6 lr groups) -> constraints.
struct AdamGroups { float lr[6]; float beta1, beta2, eps; };

template <typename T>
static double train_step(HostSplats& s, HostSplats& m, HostSplats& v, float* grad_acc, uint32_t n_views,
                         const Camera* cams, const float* targets, const Tiling& tl, int mode,
                         const AdamGroups& ag, uint64_t t, float* out_images /* nullable, V*P*4 f32 */,
                         float ssim_lambda, float* grads_out = nullptr /* nullable, 59*n f32 slab */) {
  const uint32_t n = s.n;
  const uint64_t P = (uint64_t)tl.width * tl.height;
  const uint32_t ntiles = tl.num_tiles();
  std::vector<T> rec((size_t)12 * n), img(4 * P), dl(4 * P), tfin(P), pg;
  std::vector<uint32_t> ncon(P);
  std::vector<T> gbuf((size_t)59 * n, T(0));
  HostGrads<T> g{gbuf.data(), gbuf.data() + 3 * (size_t)n, gbuf.data() + 7 * (size_t)n, gbuf.data() + 10 * (size_t)n,
                 gbuf.data() + 11 * (size_t)n, gbuf.data() + 14 * (size_t)n};
  double loss = 0.0;
  for (uint32_t vi = 0; vi < n_views; ++vi) {
    project_all<T>(s, cams[vi], rec.data());
    // count pairs first to size the key buffers
    uint64_t K = 0;
    for (uint32_t i = 0; i < n; ++i) { TileRect r = tile_rect(rec.data() + 12 * (size_t)i, tl); if (!r.empty) K += (uint64_t)(r.x1 - r.x0 + 1) * (r.y1 - r.y0 + 1); }
    std::vector<uint32_t> keys(K), pay(K), ranges(2 * (size_t)ntiles);
    bin_ref<T>(n, rec.data(), tl, keys.data(), pay.data(), K, ranges.data());
    composite<T>(rec.data(), pay.data(), ranges.data(), tl, img.data(), ncon.data(), tfin.data());
    loss += combined_loss_grad<T>((int)tl.width, (int)tl.height, img.data(), targets + 3 * P * vi, dl.data(),
                                  ssim_lambda, 1.0f / (float)n_views, nullptr) /
            (double)n_views;
    if (out_images) for (uint64_t k = 0; k < 4 * P; ++k) out_images[4 * P * vi + k] = (float)img[k];
    pg.assign((size_t)12 * n, T(0));
    composite_backward<T>(rec.data(), pay.data(), ranges.data(), tl, img.data(), dl.data(), mode, ncon.data(), tfin.data(), pg.data());
    project_backward_all<T>(s, pg.data(), cams[vi], g, 1);
  }
  std::vector<float> gf((size_t)59 * n);
  for (size_t k = 0; k < gf.size(); ++k) gf[k] = (float)gbuf[k];
  if (grads_out) std::copy(gf.begin(), gf.end(), grads_out);
  accumulate_grad(n, gf.data(), grad_acc);
  float* gp = gf.data();
  const size_t off[7] = {0, 3 * (size_t)n, 7 * (size_t)n, 10 * (size_t)n, 11 * (size_t)n, 14 * (size_t)n, 59 * (size_t)n};
  float* pp[6] = {s.pos, s.rot, s.scale, s.opacity, s.sh_dc, s.sh_rest};
  float* mp[6] = {m.pos, m.rot, m.scale, m.opacity, m.sh_dc, m.sh_rest};
  float* vp[6] = {v.pos, v.rot, v.scale, v.opacity, v.sh_dc, v.sh_rest};
  for (int k = 0; k < 6; ++k)
    adam_lanes(off[k + 1] - off[k], pp[k], gp + off[k], mp[k], vp[k], ag.lr[k], ag.beta1, ag.beta2, ag.eps, t);
  apply_constraints(n, s.rot, s.scale, s.opacity, -10.0f, 5.0f, 10.0f);
  return loss;
}

}  // namespace oracle

// ================================================================ C ABI for ctypes
using namespace oracle;

extern "C" {

void oracle_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}
int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_camera_from_pose(const float* eye, const float* target, const float* up, float fov_y, uint32_t w,
                             uint32_t h, uint32_t n, Camera* out) {
  camera_from_pose(eye, target, up, fov_y, w, h, n, out);
}

#define ORACLE_FLOAT_API(T, SFX)                                                                                   \
  void oracle_project_##SFX(const HostSplats* s, const Camera* cam, T* out) { project_all<T>(*s, *cam, out); }   \
  int64_t oracle_bin_ref_##SFX(uint32_t n, const T* rec, const Tiling* tl, uint32_t* keys, uint32_t* pay,        \
                               uint64_t cap, uint32_t* ranges) {                                                 \
    return bin_ref<T>(n, rec, *tl, keys, pay, cap, ranges);                                                      \
  }                                                                                                              \
  int64_t oracle_bin64_##SFX(uint32_t nv, uint32_t n, const T* rec, const Tiling* tl, uint64_t* keys,            \
                             uint32_t* pay, uint64_t cap, uint32_t* ranges) {                                    \
    return bin64<T>(nv, n, rec, *tl, keys, pay, cap, ranges);                                                    \
  }                                                                                                              \
  void oracle_composite_##SFX(const T* rec, const uint32_t* pay, const uint32_t* ranges, const Tiling* tl,       \
                              T* out, uint32_t* ncon, T* tfin) {                                                 \
    composite<T>(rec, pay, ranges, *tl, out, ncon, tfin);                                                        \
  }                                                                                                              \
  double oracle_mse_##SFX(uint64_t P, const T* pred, const float* target, T* dl, float scale) {                  \
    return mse<T>(P, pred, target, dl, scale);                                                                   \
  }                                                                                                              \
  void oracle_composite_backward_##SFX(const T* rec, const uint32_t* pay, const uint32_t* ranges,                \
                                       const Tiling* tl, const T* fwd, const T* dl, int mode,                    \
                                       const uint32_t* ncon, const T* tfin, T* pg, T* abs_pg) {                  \
    composite_backward<T>(rec, pay, ranges, *tl, fwd, dl, mode, ncon, tfin, pg, abs_pg);                         \
  }                                                                                                              \
  void oracle_composite_margins_##SFX(const T* rec, const uint32_t* pay, const uint32_t* ranges,                 \
                                      const Tiling* tl, int mode, double thr_a, double thr_t, float* margin,     \
                                      uint8_t* flags) {                                                          \
    composite_margins<T>(rec, pay, ranges, *tl, mode, thr_a, thr_t, margin, flags);                              \
  }                                                                                                              \
  void oracle_project_backward_##SFX(const HostSplats* s, const T* pg, const Camera* cam, T* gpos, T* grot,      \
                                     T* gsc, T* gop, T* gdc, T* grest, int accumulate) {                         \
    HostGrads<T> g{gpos, grot, gsc, gop, gdc, grest};                                                            \
    project_backward_all<T>(*s, pg, *cam, g, accumulate);                                                        \
  }                                                                                                              \
  double oracle_train_step_##SFX(HostSplats* s, HostSplats* m, HostSplats* v, float* acc, uint32_t nv,          \
                                 const Camera* cams, const float* targets, const Tiling* tl, int mode,           \
                                 const AdamGroups* ag, uint64_t t, float* out_images, float ssim_lambda,         \
                                 float* grads_out) {                                                             \
    return train_step<T>(*s, *m, *v, acc, nv, cams, targets, *tl, mode, *ag, t, out_images, ssim_lambda,         \
                         grads_out);                                                                             \
  }                                                                                                              \
  double oracle_ssim_loss_grad_##SFX(int w, int h, const T* pred, const float* target, T* dl, float scale) {     \
    return ssim_loss_grad<T>(w, h, pred, target, dl, scale);                                                     \
  }                                                                                                              \
  double oracle_combined_loss_grad_##SFX(int w, int h, const T* pred, const float* target, T* dl, float lambda,  \
                                         float scale, double* parts) {                                           \
    return combined_loss_grad<T>(w, h, pred, target, dl, lambda, scale, parts);                                  \
  }

ORACLE_FLOAT_API(float, f32)
ORACLE_FLOAT_API(double, f64)

float oracle_powi_f32(float a, int b) { return powi_f32(a, b); }

void oracle_adam_step(uint64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                      float eps, uint64_t t) {
  adam_lanes(n, p, g, m, v, lr, b1, b2, eps, t);
}

void oracle_apply_constraints(uint32_t n, float* rot, float* scale, float* op, float lsmin, float lsmax,
                              float opmax) {
  apply_constraints(n, rot, scale, op, lsmin, lsmax, opmax);
}

void oracle_accumulate_grad(uint32_t n, const float* dpos, float* acc) { accumulate_grad(n, dpos, acc); }

// s/m/v/acc must have room for the grown count; m, v, acc may be null.  Returns the new count.
uint32_t oracle_prune(HostSplats* s, HostSplats* m, HostSplats* v, float* acc, float threshold, uint32_t* removed) {
  Slabs sl{s, m, v, acc, s->n};
  *removed = prune_low_opacity(sl, threshold);
  s->n = sl.n;
  return sl.n;
}

uint32_t oracle_densify(HostSplats* s, HostSplats* m, HostSplats* v, float* acc, uint32_t grad_count,
                        float grad_thr, float split_thr, uint32_t max_splats, uint32_t iter, uint32_t* counts) {
  Slabs sl{s, m, v, acc, s->n};
  densify(sl, grad_count, grad_thr, split_thr, max_splats, iter, counts);
  s->n = sl.n;
  return sl.n;
}

int oracle_write_ply(const char* path, const HostSplats* s) { return write_ply(path, *s); }
int64_t oracle_read_ply(const char* path, HostSplats* out, uint32_t cap) { return read_ply(path, out, cap); }

}  // extern "C"
