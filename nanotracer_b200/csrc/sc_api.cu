// sc_api.cu — the extern "C" boundary of libsplatcuda (include/splat_cuda.h):
// context and buffers (WgpuCtx, gpu.rs), parameter stores (splat_gpu.rs),
// the reference-shaped rasteriser / binner / optimiser calls, densify/prune,
// and the host-side camera builder.  No CPU fallback: every compute call
// launches a kernel of this library on the context's stream.
#include "sc_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

// ================================================================ helpers
sc_status sc_fail(sc_ctx* ctx, sc_status st, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return st;
}

sc_status sc_cuda_fail(sc_ctx* ctx, cudaError_t e, const char* what) {
  if (ctx) ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? SC_ERR_OOM : SC_ERR_CUDA;
}

sc_status sc_check_launch(sc_ctx* ctx, const char* what) {
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return sc_cuda_fail(ctx, e, what);
  return SC_OK;
}

sc_status sc_scratch(sc_ctx* ctx, size_t bytes, void** out) {
  if (bytes <= ctx->scratch_bytes && ctx->scratch) { *out = ctx->scratch; return SC_OK; }
  size_t want = std::max(bytes, ctx->scratch_bytes + ctx->scratch_bytes / 2);
  want = (want + 4095) & ~(size_t)4095;
  if (ctx->scratch) {
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync before scratch growth");
    cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
  }
  SC_CUDA_TRY(ctx, cudaMalloc(&ctx->scratch, want), "scratch alloc");
  ctx->scratch_bytes = want;
  *out = ctx->scratch;
  return SC_OK;
}

sc_status sc_check_device_error(sc_ctx* ctx) {
  uint32_t e = 0;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(&e, ctx->d_error, 4, cudaMemcpyDeviceToHost, ctx->stream), "read error word");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  if (e) {
    SC_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream), "clear error word");
    if (e & SC_DEVERR_TIMEOUT) return sc_fail(ctx, SC_ERR_TIMEOUT, "a bounded device wait gave up");
    if (e & SC_DEVERR_CAPACITY) return sc_fail(ctx, SC_ERR_CAPACITY, "a device-side capacity overflowed");
  }
  return SC_OK;
}

static uint32_t bits_for(uint64_t max_value) {
  uint32_t b = 0;
  while (b < 64 && (max_value >> b) != 0) ++b;
  return b;
}

// ================================================================ runtime
extern "C" {

const char* sc_status_string(sc_status s) {
  switch (s) {
    case SC_OK: return "ok";
    case SC_ERR_INVALID_ARG: return "invalid argument";
    case SC_ERR_OOM: return "out of device memory";
    case SC_ERR_CAPACITY: return "capacity exceeded";
    case SC_ERR_CUDA: return "CUDA error";
    case SC_ERR_TIMEOUT: return "device wait timed out";
    case SC_ERR_NONFINITE: return "non-finite values";
    case SC_ERR_IO: return "I/O error";
    case SC_ERR_FORMAT: return "format error";
  }
  return "unknown status";
}

int sc_abi_version(void) { return SC_ABI_VERSION; }

sc_status sc_ctx_create(int device, sc_ctx** out) {
  if (!out) return SC_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return SC_ERR_CUDA;
  if (device < 0 || device >= count) return SC_ERR_INVALID_ARG;
  sc_ctx* ctx = new sc_ctx();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_error, 256);
  if (e == cudaSuccess) e = cudaMemset(ctx->d_error, 0, 256);
  if (e != cudaSuccess) {
    sc_ctx_destroy(ctx);
    return SC_ERR_CUDA;
  }
  ctx->own_stream = true;
  *out = ctx;
  return SC_OK;
}

void sc_ctx_destroy(sc_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->d_error) cudaFree(ctx->d_error);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* sc_last_error(const sc_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

sc_status sc_ctx_synchronize(sc_ctx* ctx) {
  if (!ctx) return SC_ERR_INVALID_ARG;
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
  return sc_check_device_error(ctx);
}

void* sc_ctx_stream(sc_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

sc_status sc_ctx_set_stream(sc_ctx* ctx, void* stream) {
  if (!ctx) return SC_ERR_INVALID_ARG;
  if (ctx->own_stream && ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  ctx->stream = (cudaStream_t)stream;
  ctx->own_stream = false;
  return SC_OK;
}

sc_status sc_ctx_device_info(sc_ctx* ctx, int* sm_count, size_t* free_b, size_t* total_b) {
  if (!ctx) return SC_ERR_INVALID_ARG;
  if (sm_count) *sm_count = ctx->sm_count;
  size_t f = 0, t = 0;
  SC_CUDA_TRY(ctx, cudaMemGetInfo(&f, &t), "mem info");
  if (free_b) *free_b = f;
  if (total_b) *total_b = t;
  return SC_OK;
}

uint64_t sc_ctx_launch_count(const sc_ctx* ctx) { return ctx ? ctx->launches : 0; }

sc_status sc_ctx_set_fp64_det(sc_ctx* ctx, int enabled) {
  if (!ctx) return SC_ERR_INVALID_ARG;
  ctx->fp64_det = enabled ? 1 : 0;
  return SC_OK;
}

sc_status sc_buffer_alloc(sc_ctx* ctx, size_t bytes, void** dptr) {
  if (!ctx || !dptr) return SC_ERR_INVALID_ARG;
  *dptr = nullptr;
  if (bytes == 0) bytes = 16;
  SC_CUDA_TRY(ctx, cudaMalloc(dptr, bytes), "buffer alloc");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(*dptr, 0, bytes, ctx->stream), "buffer zero");
  return SC_OK;
}

sc_status sc_buffer_free(sc_ctx* ctx, void* dptr) {
  if (!ctx) return SC_ERR_INVALID_ARG;
  if (!dptr) return SC_OK;
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync before free");
  SC_CUDA_TRY(ctx, cudaFree(dptr), "buffer free");
  return SC_OK;
}

sc_status sc_buffer_upload(sc_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx || (bytes && (!dst || !src))) return SC_ERR_INVALID_ARG;
  if (!bytes) return SC_OK;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "upload sync");
  return SC_OK;
}

sc_status sc_buffer_readback(sc_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx || (bytes && (!dst || !src))) return SC_ERR_INVALID_ARG;
  if (!bytes) return SC_OK;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream), "readback");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "readback sync");
  return sc_check_device_error(ctx);
}

sc_status sc_buffer_copy(sc_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx || (bytes && (!dst || !src))) return SC_ERR_INVALID_ARG;
  if (!bytes) return SC_OK;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
  return SC_OK;
}

sc_status sc_buffer_zero(sc_ctx* ctx, void* dptr, size_t bytes) {
  if (!ctx || (bytes && !dptr)) return SC_ERR_INVALID_ARG;
  if (!bytes) return SC_OK;
  SC_CUDA_TRY(ctx, cudaMemsetAsync(dptr, 0, bytes, ctx->stream), "zero");
  return SC_OK;
}

// ================================================================ parameter stores
static uint32_t round_cap(uint32_t n) { return std::max<uint32_t>(256u, (n + 255u) & ~255u); }

// host SoA (per-splat interleaved attributes) <-> device rows
static void host_to_rows(const sc_host_splats* h, uint32_t cap, std::vector<float>& rows) {
  const uint32_t n = h->n;
  rows.assign((size_t)SC_NROWS * cap, 0.0f);
  auto put = [&](int row0, const float* src, int w) {
    for (uint32_t i = 0; i < n; ++i)
      for (int k = 0; k < w; ++k) rows[(size_t)(row0 + k) * cap + i] = src[(size_t)w * i + k];
  };
  put(SC_ROW_POS, h->positions, 3);
  put(SC_ROW_ROT, h->rotations, 4);
  put(SC_ROW_SCALE, h->scales, 3);
  put(SC_ROW_OP, h->opacities, 1);
  put(SC_ROW_DC, h->sh_dc, 3);
  put(SC_ROW_REST, h->sh_rest, 45);
}

static void rows_to_host(const std::vector<float>& rows, uint32_t cap, uint32_t n, sc_host_splats* h) {
  auto get = [&](int row0, float* dst, int w) {
    if (!dst) return;
    for (uint32_t i = 0; i < n; ++i)
      for (int k = 0; k < w; ++k) dst[(size_t)w * i + k] = rows[(size_t)(row0 + k) * cap + i];
  };
  get(SC_ROW_POS, h->positions, 3);
  get(SC_ROW_ROT, h->rotations, 4);
  get(SC_ROW_SCALE, h->scales, 3);
  get(SC_ROW_OP, h->opacities, 1);
  get(SC_ROW_DC, h->sh_dc, 3);
  get(SC_ROW_REST, h->sh_rest, 45);
}

static bool host_valid(const sc_host_splats* h) {
  return h && (h->n == 0 || (h->positions && h->rotations && h->scales && h->opacities && h->sh_dc && h->sh_rest));
}

static void f32_to_bf16_rows(const float* src, size_t count, std::vector<__nv_bfloat16>& dst) {
  dst.resize(count);
  for (size_t k = 0; k < count; ++k) dst[k] = __float2bfloat16_rn(src[k]);
}

static sc_status upload_rows(sc_ctx* ctx, sc_splats* s, const std::vector<float>& rows) {
  const uint32_t cap = s->cap;
  const bool bf = (s->flags & SC_SPLATS_BF16_REST) != 0;
  const size_t frows = bf ? SC_ROW_REST : SC_NROWS;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(s->slab, rows.data(), frows * cap * 4, cudaMemcpyHostToDevice, ctx->stream), "upload");
  if (bf) {
    std::vector<__nv_bfloat16> h16;
    f32_to_bf16_rows(rows.data() + (size_t)SC_ROW_REST * cap, (size_t)45 * cap, h16);
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(s->rest16, h16.data(), h16.size() * 2, cudaMemcpyHostToDevice, ctx->stream), "upload");
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "upload sync");
  } else {
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "upload sync");
  }
  return SC_OK;
}

sc_status sc_splats_upload(sc_ctx* ctx, const sc_host_splats* src, uint32_t capacity, uint32_t flags, sc_splats** out) {
  if (!ctx || !out || !host_valid(src)) return SC_ERR_INVALID_ARG;
  *out = nullptr;
  sc_splats* s = new sc_splats();
  s->n = src->n;
  s->cap = round_cap(std::max(capacity, src->n));
  s->flags = flags;
  const bool bf = (flags & SC_SPLATS_BF16_REST) != 0;
  const size_t frows = bf ? SC_ROW_REST : SC_NROWS;
  cudaError_t e = cudaMalloc(&s->slab, frows * s->cap * 4);
  if (e == cudaSuccess && bf) e = cudaMalloc(&s->rest16, (size_t)45 * s->cap * 2);
  if (e != cudaSuccess) {
    sc_splats_free(ctx, s);
    return sc_cuda_fail(ctx, e, "splat alloc");
  }
  std::vector<float> rows;
  host_to_rows(src, s->cap, rows);
  sc_status st = upload_rows(ctx, s, rows);
  if (st != SC_OK) { sc_splats_free(ctx, s); return st; }
  *out = s;
  return SC_OK;
}

sc_status sc_splats_sync_from(sc_ctx* ctx, sc_splats* dst, const sc_host_splats* src) {
  if (!ctx || !dst || !host_valid(src)) return SC_ERR_INVALID_ARG;
  if (src->n > dst->cap) return sc_fail(ctx, SC_ERR_CAPACITY, "sync_from: more splats than capacity");
  std::vector<float> rows;
  host_to_rows(src, dst->cap, rows);
  dst->n = src->n;
  return upload_rows(ctx, dst, rows);
}

sc_status sc_splats_readback(sc_ctx* ctx, const sc_splats* s, sc_host_splats* dst) {
  if (!ctx || !s || !dst) return SC_ERR_INVALID_ARG;
  const uint32_t cap = s->cap;
  std::vector<float> rows((size_t)SC_NROWS * cap);
  const bool bf = (s->flags & SC_SPLATS_BF16_REST) != 0;
  const size_t frows = bf ? SC_ROW_REST : SC_NROWS;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(rows.data(), s->slab, frows * cap * 4, cudaMemcpyDeviceToHost, ctx->stream), "readback");
  std::vector<__nv_bfloat16> h16;
  if (bf) {
    h16.resize((size_t)45 * cap);
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(h16.data(), s->rest16, h16.size() * 2, cudaMemcpyDeviceToHost, ctx->stream), "readback");
  }
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "readback sync");
  if (bf)
    for (size_t k = 0; k < h16.size(); ++k) rows[(size_t)SC_ROW_REST * cap + k] = __bfloat162float(h16[k]);
  rows_to_host(rows, cap, s->n, dst);
  dst->n = s->n;
  return sc_check_device_error(ctx);
}

uint32_t sc_splats_count(const sc_splats* s) { return s ? s->n : 0; }
uint32_t sc_splats_capacity(const sc_splats* s) { return s ? s->cap : 0; }

void sc_splats_free(sc_ctx* ctx, sc_splats* s) {
  if (!s) return;
  if (ctx) cudaStreamSynchronize(ctx->stream);
  if (s->slab) cudaFree(s->slab);
  if (s->rest16) cudaFree(s->rest16);
  delete s;
}

sc_status sc_grads_create(sc_ctx* ctx, uint32_t capacity, sc_grads** out) {
  if (!ctx || !out) return SC_ERR_INVALID_ARG;
  sc_grads* g = new sc_grads();
  g->cap = round_cap(capacity);
  cudaError_t e = cudaMalloc(&g->slab, (size_t)SC_NROWS * g->cap * 4);
  if (e != cudaSuccess) { delete g; return sc_cuda_fail(ctx, e, "grad alloc"); }
  e = cudaMemsetAsync(g->slab, 0, (size_t)SC_NROWS * g->cap * 4, ctx->stream);
  if (e != cudaSuccess) { cudaFree(g->slab); delete g; return sc_cuda_fail(ctx, e, "grad zero"); }
  *out = g;
  return SC_OK;
}

sc_status sc_grads_zero(sc_ctx* ctx, sc_grads* g, uint32_t n) {
  if (!ctx || !g) return SC_ERR_INVALID_ARG;
  (void)n;
  SC_CUDA_TRY(ctx, cudaMemsetAsync(g->slab, 0, (size_t)SC_NROWS * g->cap * 4, ctx->stream), "grad zero");
  return SC_OK;
}

sc_status sc_grads_upload(sc_ctx* ctx, sc_grads* g, const sc_host_splats* src) {
  if (!ctx || !g || !host_valid(src)) return SC_ERR_INVALID_ARG;
  if (src->n > g->cap) return sc_fail(ctx, SC_ERR_CAPACITY, "grads: more splats than capacity");
  std::vector<float> rows;
  host_to_rows(src, g->cap, rows);
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(g->slab, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "upload");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "upload sync");
  return SC_OK;
}

sc_status sc_grads_readback(sc_ctx* ctx, const sc_grads* g, uint32_t n, sc_host_splats* dst) {
  if (!ctx || !g || !dst || n > g->cap) return SC_ERR_INVALID_ARG;
  std::vector<float> rows((size_t)SC_NROWS * g->cap);
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(rows.data(), g->slab, rows.size() * 4, cudaMemcpyDeviceToHost, ctx->stream), "readback");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "readback sync");
  rows_to_host(rows, g->cap, n, dst);
  dst->n = n;
  return sc_check_device_error(ctx);
}

void sc_grads_free(sc_ctx* ctx, sc_grads* g) {
  if (!g) return;
  if (ctx) cudaStreamSynchronize(ctx->stream);
  if (g->slab) cudaFree(g->slab);
  delete g;
}

sc_status sc_moments_create(sc_ctx* ctx, uint32_t capacity, uint32_t flags, sc_moments** out) {
  if (!ctx || !out) return SC_ERR_INVALID_ARG;
  sc_moments* m = new sc_moments();
  m->cap = round_cap(capacity);
  m->flags = flags;
  const size_t cnt = (size_t)SC_NROWS * m->cap;
  cudaError_t e;
  if (flags & SC_MOMENTS_BF16) {
    e = cudaMalloc(&m->m16, cnt * 2);
    if (e == cudaSuccess) e = cudaMalloc(&m->v16, cnt * 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->m16, 0, cnt * 2, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->v16, 0, cnt * 2, ctx->stream);
  } else {
    e = cudaMalloc(&m->m, cnt * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->v, cnt * 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->m, 0, cnt * 4, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->v, 0, cnt * 4, ctx->stream);
  }
  if (e != cudaSuccess) { sc_moments_free(ctx, m); return sc_cuda_fail(ctx, e, "moment alloc"); }
  *out = m;
  return SC_OK;
}

static sc_status moments_put(sc_ctx* ctx, sc_moments* mo, const sc_host_splats* h, bool is_v) {
  std::vector<float> rows;
  host_to_rows(h, mo->cap, rows);
  if (mo->flags & SC_MOMENTS_BF16) {
    std::vector<__nv_bfloat16> r16;
    f32_to_bf16_rows(rows.data(), rows.size(), r16);
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(is_v ? mo->v16 : mo->m16, r16.data(), r16.size() * 2, cudaMemcpyHostToDevice, ctx->stream), "upload");
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  } else {
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(is_v ? mo->v : mo->m, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "upload");
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  }
  return SC_OK;
}

sc_status sc_moments_upload(sc_ctx* ctx, sc_moments* mo, const sc_host_splats* m, const sc_host_splats* v) {
  if (!ctx || !mo || !host_valid(m) || !host_valid(v)) return SC_ERR_INVALID_ARG;
  if (m->n > mo->cap || v->n > mo->cap) return sc_fail(ctx, SC_ERR_CAPACITY, "moments: more splats than capacity");
  SC_TRY(moments_put(ctx, mo, m, false));
  return moments_put(ctx, mo, v, true);
}

sc_status sc_moments_readback(sc_ctx* ctx, const sc_moments* mo, uint32_t n, sc_host_splats* m, sc_host_splats* v) {
  if (!ctx || !mo || n > mo->cap) return SC_ERR_INVALID_ARG;
  const size_t cnt = (size_t)SC_NROWS * mo->cap;
  for (int which = 0; which < 2; ++which) {
    sc_host_splats* dst = which ? v : m;
    if (!dst) continue;
    std::vector<float> rows(cnt);
    if (mo->flags & SC_MOMENTS_BF16) {
      std::vector<__nv_bfloat16> r16(cnt);
      SC_CUDA_TRY(ctx, cudaMemcpyAsync(r16.data(), which ? mo->v16 : mo->m16, cnt * 2, cudaMemcpyDeviceToHost, ctx->stream), "readback");
      SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
      for (size_t k = 0; k < cnt; ++k) rows[k] = __bfloat162float(r16[k]);
    } else {
      SC_CUDA_TRY(ctx, cudaMemcpyAsync(rows.data(), which ? mo->v : mo->m, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream), "readback");
      SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    }
    rows_to_host(rows, mo->cap, n, dst);
    dst->n = n;
  }
  return sc_check_device_error(ctx);
}

void sc_moments_free(sc_ctx* ctx, sc_moments* mo) {
  if (!mo) return;
  if (ctx) cudaStreamSynchronize(ctx->stream);
  if (mo->m) cudaFree(mo->m);
  if (mo->v) cudaFree(mo->v);
  if (mo->m16) cudaFree(mo->m16);
  if (mo->v16) cudaFree(mo->v16);
  delete mo;
}

// ================================================================ camera (raster.rs:79-99)
// Right-handed look-at (glam look_at_mat4): f = normalize(target - eye),
// s = normalize(f x up), u = s x f; columns (s.x, u.x, -f.x, 0), (s.y, u.y,
// -f.y, 0), (s.z, u.z, -f.z, 0), (-s.eye, -u.eye, f.eye, 1).
void sc_camera_from_pose(const float eye[3], const float target[3], const float up[3], float fov_y, uint32_t width,
                         uint32_t height, uint32_t n_splats, sc_camera* out) {
  auto normalize = [](float v[3]) {
    const float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const float r = 1.0f / len;
    v[0] *= r; v[1] *= r; v[2] *= r;
  };
  float f[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
  normalize(f);
  float s[3] = {f[1] * up[2] - up[1] * f[2], f[2] * up[0] - up[2] * f[0], f[0] * up[1] - up[0] * f[1]};
  normalize(s);
  const float u[3] = {s[1] * f[2] - f[1] * s[2], s[2] * f[0] - f[2] * s[0], s[0] * f[1] - f[0] * s[1]};
  float* v = out->view;
  v[0] = s[0]; v[1] = u[0]; v[2] = -f[0]; v[3] = 0.0f;
  v[4] = s[1]; v[5] = u[1]; v[6] = -f[1]; v[7] = 0.0f;
  v[8] = s[2]; v[9] = u[2]; v[10] = -f[2]; v[11] = 0.0f;
  v[12] = -(eye[0] * s[0] + eye[1] * s[1] + eye[2] * s[2]);
  v[13] = -(eye[0] * u[0] + eye[1] * u[1] + eye[2] * u[2]);
  v[14] = eye[0] * f[0] + eye[1] * f[1] + eye[2] * f[2];
  v[15] = 1.0f;
  out->cam_pos[0] = eye[0]; out->cam_pos[1] = eye[1]; out->cam_pos[2] = eye[2];
  out->near_plane = 0.01f;
  out->focal = (float)height / (2.0f * std::tan(fov_y * 0.5f));
  out->width = (float)width;
  out->height = (float)height;
  out->n_splats = n_splats;
}

// cameras are staged through the scratch-independent error buffer page
static sc_status stage_cams(sc_ctx* ctx, const sc_camera* cams, uint32_t n_views, sc_camera** d_cams) {
  // cameras live in a small dedicated slice right after the error word page
  static_assert(sizeof(sc_camera) == 96, "camera layout");
  if (n_views > SC_MAX_VIEWS) return sc_fail(ctx, SC_ERR_INVALID_ARG, "too many views");
  void* p;
  SC_CUDA_TRY(ctx, cudaMallocAsync(&p, (size_t)n_views * sizeof(sc_camera), ctx->stream), "camera alloc");
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(p, cams, (size_t)n_views * sizeof(sc_camera), cudaMemcpyHostToDevice, ctx->stream), "camera upload");
  *d_cams = reinterpret_cast<sc_camera*>(p);
  return SC_OK;
}

static bool tiling_ok(const sc_tiling* t) {
  return t && t->width > 0 && t->height > 0 && t->tile_w > 0 && t->tile_h > 0;
}

// ================================================================ rasteriser
sc_status sc_project(sc_ctx* ctx, const sc_splats* s, const sc_camera* cams, uint32_t n_views,
                     sc_projected_splat* projected) {
  if (!ctx || !s || !cams || (!projected && s->n)) return SC_ERR_INVALID_ARG;
  if (n_views == 0) return SC_OK;
  sc_camera* d_cams;
  SC_TRY(stage_cams(ctx, cams, n_views, &d_cams));
  sc_status st = sck::launch_project(ctx, dview(s), d_cams, n_views, s->cap, reinterpret_cast<float4*>(projected),
                                     nullptr, nullptr, nullptr, nullptr, ctx->fp64_det, 0);
  cudaFreeAsync(d_cams, ctx->stream);
  return st;
}

}  // extern "C"

// ================================================================ bins
struct sc_bins {
  uint64_t cap = 0;
  void* keys = nullptr; void* keys_tmp = nullptr;
  uint32_t* vals = nullptr; uint32_t* vals_tmp = nullptr;
  uint32_t* ranges = nullptr; uint64_t ranges_cap = 0;
  uint32_t* counts = nullptr; uint64_t counts_cap = 0;
  uint64_t* d_total = nullptr;
  uint64_t total = 0;
  uint32_t num_tiles = 0, n_views = 0;
  int key_mode = 0;
  size_t kbytes = 0;  // width of the allocated key buffers
};

static void bins_release(sc_bins* b) {
  if (b->keys) cudaFree(b->keys);
  if (b->keys_tmp) cudaFree(b->keys_tmp);
  if (b->vals) cudaFree(b->vals);
  if (b->vals_tmp) cudaFree(b->vals_tmp);
  b->keys = b->keys_tmp = nullptr;
  b->vals = b->vals_tmp = nullptr;
  b->cap = 0;
}

extern "C" {

sc_status sc_bins_create(sc_ctx* ctx, sc_bins** out) {
  if (!ctx || !out) return SC_ERR_INVALID_ARG;
  sc_bins* b = new sc_bins();
  cudaError_t e = cudaMalloc(&b->d_total, 64);
  if (e != cudaSuccess) { delete b; return sc_cuda_fail(ctx, e, "bins alloc"); }
  *out = b;
  return SC_OK;
}

void sc_bins_free(sc_ctx* ctx, sc_bins* b) {
  if (!b) return;
  if (ctx) cudaStreamSynchronize(ctx->stream);
  bins_release(b);
  if (b->ranges) cudaFree(b->ranges);
  if (b->counts) cudaFree(b->counts);
  if (b->d_total) cudaFree(b->d_total);
  delete b;
}

sc_status sc_bin(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t n, uint32_t stride, uint32_t n_views,
                 const sc_tiling* tl, sc_key_mode mode, sc_bins* b) {
  if (!ctx || !b || !tiling_ok(tl) || (n && !projected) || stride < n) return SC_ERR_INVALID_ARG;
  const uint32_t tiles_x = (tl->width + tl->tile_w - 1) / tl->tile_w;
  const uint32_t tiles_y = (tl->height + tl->tile_h - 1) / tl->tile_h;
  const uint64_t all_tiles = (uint64_t)tiles_x * tiles_y * std::max(n_views, 1u);
  if (mode == SC_KEYS_REF32 && all_tiles > 65536)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "REF32 keys hold at most 65536 tiles (tile_emit.wgsl key layout)");
  if (all_tiles > 0xFFFFFFFFull) return sc_fail(ctx, SC_ERR_INVALID_ARG, "too many tiles");
  b->num_tiles = (uint32_t)all_tiles;
  b->n_views = n_views;
  b->key_mode = mode;
  const uint64_t items = (uint64_t)n * n_views;
  // ranges
  if (b->ranges_cap < all_tiles) {
    if (b->ranges) cudaFree(b->ranges);
    b->ranges = nullptr;
    SC_CUDA_TRY(ctx, cudaMalloc(&b->ranges, all_tiles * 8), "ranges alloc");
    b->ranges_cap = all_tiles;
  }
  if (items == 0) {
    b->total = 0;
    SC_CUDA_TRY(ctx, cudaMemsetAsync(b->ranges, 0, all_tiles * 8, ctx->stream), "ranges zero");
    SC_CUDA_TRY(ctx, cudaMemsetAsync(b->d_total, 0, 8, ctx->stream), "total zero");
    return SC_OK;
  }
  if (b->counts_cap < items + 1) {
    if (b->counts) cudaFree(b->counts);
    b->counts = nullptr;
    SC_CUDA_TRY(ctx, cudaMalloc(&b->counts, (items + 1) * 4), "counts alloc");
    b->counts_cap = items + 1;
  }
  const float4* rec = reinterpret_cast<const float4*>(projected);
  // 1. count (tile_count.wgsl)
  SC_TRY(sck::launch_tile_count(ctx, rec, n, stride, n_views, tl, b->counts));
  SC_CUDA_TRY(ctx, cudaMemsetAsync(b->counts + items, 0, 4, ctx->stream), "memset");
  // 2. exclusive scan -> offsets, total
  void* scr;
  const size_t scan_bytes = sck::scan_scratch_bytes(items + 1);
  SC_TRY(sc_scratch(ctx, scan_bytes, &scr));
  SC_TRY(sck::scan_u32(ctx, b->counts, items + 1, b->d_total, scr, scan_bytes));
  // 3. read the pair count (the reference reads it back too, tile_binner.rs:243-245)
  uint64_t K = 0;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(&K, b->d_total, 8, cudaMemcpyDeviceToHost, ctx->stream), "total readback");
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  SC_TRY(sc_check_device_error(ctx));
  if (K >= (1ull << 31)) return sc_fail(ctx, SC_ERR_CAPACITY, "more than 2^31 tile/splat pairs");
  b->total = K;
  const size_t kb = mode == SC_KEYS_REF32 ? 4 : 8;
  if (K > b->cap || kb > b->kbytes) {
    bins_release(b);
    b->kbytes = kb;
    const uint64_t cap = K + K / 8 + 1024;
    SC_CUDA_TRY(ctx, cudaMalloc(&b->keys, cap * kb), "keys alloc");
    SC_CUDA_TRY(ctx, cudaMalloc(&b->keys_tmp, cap * kb), "keys alloc");
    SC_CUDA_TRY(ctx, cudaMalloc(&b->vals, cap * 4), "vals alloc");
    SC_CUDA_TRY(ctx, cudaMalloc(&b->vals_tmp, cap * 4), "vals alloc");
    b->cap = cap;
  }
  if (K == 0) {
    SC_CUDA_TRY(ctx, cudaMemsetAsync(b->ranges, 0, all_tiles * 8, ctx->stream), "ranges zero");
    return SC_OK;
  }
  // 4. emit (tile_emit.wgsl)
  SC_TRY(sck::launch_tile_emit(ctx, rec, n, stride, n_views, tl, b->counts, mode, b->keys, b->vals, K));
  // 5. sort
  const uint32_t tile_bits = bits_for(all_tiles - 1);
  bool in_tmp = false;
  if (mode == SC_KEYS_REF32) {
    const uint32_t key_bits = 16 + tile_bits;
    const size_t rb = sck::radix_scratch_bytes(K, 4);
    SC_TRY(sc_scratch(ctx, rb, &scr));
    SC_TRY(sck::radix_sort<uint32_t>(ctx, (uint32_t*)b->keys, b->vals, (uint32_t*)b->keys_tmp, b->vals_tmp, K, key_bits,
                                     nullptr, scr, rb, &in_tmp));
  } else {
    const uint32_t key_bits = 32 + tile_bits;
    const size_t rb = sck::radix_scratch_bytes(K, 8);
    SC_TRY(sc_scratch(ctx, rb, &scr));
    SC_TRY(sck::radix_sort<uint64_t>(ctx, (uint64_t*)b->keys, b->vals, (uint64_t*)b->keys_tmp, b->vals_tmp, K, key_bits,
                                     nullptr, scr, rb, &in_tmp));
  }
  if (in_tmp) {
    std::swap(b->keys, b->keys_tmp);
    std::swap(b->vals, b->vals_tmp);
  }
  // 6. ranges (tile_ranges.wgsl)
  return sck::launch_tile_ranges(ctx, b->keys, mode == SC_KEYS_REF32 ? 0 : 1, b->d_total, K, b->num_tiles, b->ranges);
}

sc_status sc_bins_info(const sc_bins* b, uint64_t* total, uint32_t* num_tiles, const void** keys,
                       const uint32_t** payloads, const uint32_t** ranges) {
  if (!b) return SC_ERR_INVALID_ARG;
  if (total) *total = b->total;
  if (num_tiles) *num_tiles = b->num_tiles;
  if (keys) *keys = b->keys;
  if (payloads) *payloads = b->vals;
  if (ranges) *ranges = b->ranges;
  return SC_OK;
}

sc_status sc_radix_sort_u32(sc_ctx* ctx, uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                            uint64_t n, uint32_t key_bits) {
  if (!ctx || (n && (!keys || !vals || !keys_tmp || !vals_tmp)) || key_bits > 32) return SC_ERR_INVALID_ARG;
  if (n == 0) return SC_OK;
  const size_t rb = sck::radix_scratch_bytes(n, 4);
  void* scr;
  SC_TRY(sc_scratch(ctx, rb, &scr));
  bool in_tmp = false;
  SC_TRY(sck::radix_sort<uint32_t>(ctx, keys, vals, keys_tmp, vals_tmp, n, key_bits, nullptr, scr, rb, &in_tmp));
  if (in_tmp) {
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(keys, keys_tmp, n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy back");
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(vals, vals_tmp, n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy back");
  }
  return SC_OK;
}

sc_status sc_radix_sort_u64(sc_ctx* ctx, uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                            uint64_t n, uint32_t key_bits) {
  if (!ctx || (n && (!keys || !vals || !keys_tmp || !vals_tmp)) || key_bits > 64) return SC_ERR_INVALID_ARG;
  if (n == 0) return SC_OK;
  const size_t rb = sck::radix_scratch_bytes(n, 8);
  void* scr;
  SC_TRY(sc_scratch(ctx, rb, &scr));
  bool in_tmp = false;
  SC_TRY(sck::radix_sort<uint64_t>(ctx, keys, vals, keys_tmp, vals_tmp, n, key_bits, nullptr, scr, rb, &in_tmp));
  if (in_tmp) {
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(keys, keys_tmp, n * 8, cudaMemcpyDeviceToDevice, ctx->stream), "copy back");
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(vals, vals_tmp, n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy back");
  }
  return SC_OK;
}

sc_status sc_exclusive_scan_u32(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* total) {
  if (!ctx || (n && !data)) return SC_ERR_INVALID_ARG;
  const size_t sb = sck::scan_scratch_bytes(n);
  void* scr;
  SC_TRY(sc_scratch(ctx, sb, &scr));
  return sck::scan_u32(ctx, data, n, total, scr, sb);
}

sc_status sc_composite(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t stride, uint32_t n_views,
                       const sc_bins* b, const sc_tiling* tl, float* image, uint32_t* aux) {
  if (!ctx || !b || !tiling_ok(tl) || !image) return SC_ERR_INVALID_ARG;
  if (b->key_mode == SC_KEYS_REF32 && b->n_views > 1 && b->n_views != n_views) return SC_ERR_INVALID_ARG;
  if (b->total > 0 && (!b->vals || !projected)) return SC_ERR_INVALID_ARG;
  return sck::launch_composite(ctx, reinterpret_cast<const float4*>(projected), stride, n_views, b->vals, b->ranges, tl,
                               reinterpret_cast<float4*>(image), reinterpret_cast<uint2*>(aux), nullptr, 1.0f, nullptr,
                               nullptr, nullptr);
}

sc_status sc_mse_loss_grad(sc_ctx* ctx, const float* pred, const float* target, uint32_t n_views, const sc_tiling* tl,
                           float scale, float* dl_dc, double* loss_out) {
  if (!ctx || !pred || !target || !dl_dc || !tiling_ok(tl)) return SC_ERR_INVALID_ARG;
  const uint64_t P = (uint64_t)tl->width * tl->height;
  if (loss_out) SC_CUDA_TRY(ctx, cudaMemsetAsync(loss_out, 0, (size_t)n_views * 8, ctx->stream), "memset loss");
  return sck::launch_mse(ctx, reinterpret_cast<const float4*>(pred), target, P, n_views, scale,
                         reinterpret_cast<float4*>(dl_dc), loss_out);
}

// scratch for the SSIM coefficient planes plus 2 doubles per view (MSE means, SSIM sums)
static sc_status ssim_scratch(sc_ctx* ctx, uint64_t P, uint32_t n_views, float** terms, double** sums) {
  const size_t tb = (sck::ssim_terms_bytes(P, n_views) + 255) & ~(size_t)255;
  void* scr = nullptr;
  SC_TRY(sc_scratch(ctx, tb + 16 * (size_t)n_views, &scr));
  *terms = reinterpret_cast<float*>(scr);
  *sums = reinterpret_cast<double*>(reinterpret_cast<char*>(scr) + tb);
  SC_CUDA_TRY(ctx, cudaMemsetAsync(*sums, 0, 16 * (size_t)n_views, ctx->stream), "zero sums");
  return SC_OK;
}

sc_status sc_ssim_loss_grad(sc_ctx* ctx, const float* pred, const float* target, uint32_t n_views, const sc_tiling* tl,
                            float scale, float* dl_dc, double* loss_out) {
  if (!ctx || !pred || !target || !dl_dc || !tiling_ok(tl)) return SC_ERR_INVALID_ARG;
  if (n_views == 0) return SC_OK;
  const uint64_t P = (uint64_t)tl->width * tl->height;
  float* terms; double* sums;
  SC_TRY(ssim_scratch(ctx, P, n_views, &terms, &sums));
  SC_CUDA_TRY(ctx, cudaMemsetAsync(dl_dc, 0, (size_t)n_views * P * 16, ctx->stream), "zero dl_dc");
  SC_TRY(sck::launch_ssim(ctx, reinterpret_cast<const float4*>(pred), target, tl->width, tl->height, n_views, scale,
                          reinterpret_cast<float4*>(dl_dc), sums + n_views, terms));
  if (!loss_out) return SC_OK;
  // {total, mse, ssim} triples into the scratch's MSE slot region is too small; write L directly
  double* parts = nullptr;
  SC_CUDA_TRY(ctx, cudaMallocAsync(&parts, 24 * (size_t)n_views, ctx->stream), "loss parts");
  sc_status st = sck::launch_loss_parts(ctx, nullptr, sums + n_views, n_views, P, 1.0f, parts);
  if (st == SC_OK)
    st = cudaMemcpy2DAsync(loss_out, 8, parts, 24, 8, n_views, cudaMemcpyDeviceToDevice, ctx->stream) == cudaSuccess
             ? SC_OK
             : sc_fail(ctx, SC_ERR_CUDA, "loss copy");
  cudaFreeAsync(parts, ctx->stream);
  return st;
}

sc_status sc_combined_loss_grad(sc_ctx* ctx, const float* pred, const float* target, uint32_t n_views,
                                const sc_tiling* tl, float lambda, float scale, float* dl_dc, double* loss_out) {
  if (!ctx || !pred || !target || !dl_dc || !tiling_ok(tl)) return SC_ERR_INVALID_ARG;
  if (n_views == 0) return SC_OK;
  if (!(lambda >= 0.0f)) lambda = 0.0f;  // also maps NaN to 0
  if (lambda > 1.0f) lambda = 1.0f;
  const uint64_t P = (uint64_t)tl->width * tl->height;
  float* terms = nullptr; double* sums = nullptr;
  if (lambda > 0.0f) SC_TRY(ssim_scratch(ctx, P, n_views, &terms, &sums));
  double* mse = nullptr;
  if (lambda < 1.0f) {
    SC_CUDA_TRY(ctx, cudaMallocAsync(&mse, 8 * (size_t)n_views, ctx->stream), "mse sums");
    SC_CUDA_TRY(ctx, cudaMemsetAsync(mse, 0, 8 * (size_t)n_views, ctx->stream), "zero mse");
    SC_TRY(sck::launch_mse(ctx, reinterpret_cast<const float4*>(pred), target, P, n_views, scale * (1.0f - lambda),
                           reinterpret_cast<float4*>(dl_dc), mse));
  } else {
    SC_CUDA_TRY(ctx, cudaMemsetAsync(dl_dc, 0, (size_t)n_views * P * 16, ctx->stream), "zero dl_dc");
  }
  sc_status st = SC_OK;
  if (lambda > 0.0f)
    st = sck::launch_ssim(ctx, reinterpret_cast<const float4*>(pred), target, tl->width, tl->height, n_views,
                          scale * lambda, reinterpret_cast<float4*>(dl_dc), sums, terms);
  if (st == SC_OK && loss_out) st = sck::launch_loss_parts(ctx, mse, sums, n_views, P, lambda, loss_out);
  if (mse) cudaFreeAsync(mse, ctx->stream);
  return st;
}

sc_status sc_composite_backward(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t stride, uint32_t n_views,
                                const sc_bins* b, const sc_tiling* tl, const float* fwd, const float* dl_dc,
                                sc_bwd_mode mode, const uint32_t* aux, sc_projected_grad* pg) {
  if (!ctx || !b || !tiling_ok(tl) || !fwd || !dl_dc || !pg) return SC_ERR_INVALID_ARG;
  if (mode != SC_BWD_REF && mode != SC_BWD_EXACT) return SC_ERR_INVALID_ARG;
  if (b->total > 0 && (!b->vals || !projected)) return SC_ERR_INVALID_ARG;
  return sck::launch_composite_backward(ctx, reinterpret_cast<const float4*>(projected), stride, n_views, b->vals,
                                        b->ranges, tl, reinterpret_cast<const float4*>(fwd),
                                        reinterpret_cast<const float4*>(dl_dc), (int)mode,
                                        reinterpret_cast<const uint2*>(aux), reinterpret_cast<float4*>(pg), nullptr);
}

sc_status sc_composite_backward_ex(sc_ctx* ctx, const sc_projected_splat* projected, uint32_t stride,
                                   uint32_t n_views, const sc_bins* b, const sc_tiling* tl, const float* fwd,
                                   const float* dl_dc, sc_bwd_mode mode, const uint32_t* aux, sc_projected_grad* pg,
                                   uint32_t flags) {
  if (!(flags & SC_BWD_FLAG_COMPENSATED))
    return sc_composite_backward(ctx, projected, stride, n_views, b, tl, fwd, dl_dc, mode, aux, pg);
  if (flags & ~SC_BWD_FLAG_COMPENSATED) return sc_fail(ctx, SC_ERR_INVALID_ARG, "unknown backward flag");
  if (!ctx || !b || !tiling_ok(tl) || !fwd || !dl_dc || !pg) return SC_ERR_INVALID_ARG;
  if (mode != SC_BWD_REF && mode != SC_BWD_EXACT) return SC_ERR_INVALID_ARG;
  if (b->total > 0 && (!b->vals || !projected)) return SC_ERR_INVALID_ARG;
  const uint64_t n4 = (uint64_t)n_views * stride * 3;  // float4 records of the gradient buffer
  void* comp = nullptr;
  SC_CUDA_TRY(ctx, cudaMallocAsync(&comp, std::max<uint64_t>(n4, 1) * 16, ctx->stream), "compensation records");
  sc_status st = SC_OK;
  if (cudaMemsetAsync(comp, 0, n4 * 16, ctx->stream) != cudaSuccess) st = sc_fail(ctx, SC_ERR_CUDA, "zero");
  if (st == SC_OK)
    st = sck::launch_composite_backward(ctx, reinterpret_cast<const float4*>(projected), stride, n_views, b->vals,
                                        b->ranges, tl, reinterpret_cast<const float4*>(fwd),
                                        reinterpret_cast<const float4*>(dl_dc), (int)mode,
                                        reinterpret_cast<const uint2*>(aux), reinterpret_cast<float4*>(pg), nullptr,
                                        nullptr, 0.0f, nullptr, reinterpret_cast<float4*>(comp));
  if (st == SC_OK)
    st = sck::launch_fold_comp(ctx, reinterpret_cast<float4*>(pg), reinterpret_cast<const float4*>(comp), n4);
  cudaFreeAsync(comp, ctx->stream);
  return st;
}

sc_status sc_project_backward(sc_ctx* ctx, const sc_splats* s, const sc_projected_grad* pg, const sc_camera* cam,
                              sc_grads* g, int accumulate) {
  if (!ctx || !s || !pg || !cam || !g) return SC_ERR_INVALID_ARG;
  if (g->cap < s->n) return sc_fail(ctx, SC_ERR_CAPACITY, "grads smaller than the splat count");
  sc_camera* d_cam;
  SC_TRY(stage_cams(ctx, cam, 1, &d_cam));
  sc_status st = sck::launch_project_backward(ctx, dview(s), reinterpret_cast<const float4*>(pg), d_cam, g->slab,
                                              g->cap, accumulate, ctx->fp64_det);
  cudaFreeAsync(d_cam, ctx->stream);
  return st;
}

sc_status sc_tonemap(sc_ctx* ctx, const float* image, uint32_t w, uint32_t h, uint8_t* rgba8) {
  if (!ctx || !image || !rgba8) return SC_ERR_INVALID_ARG;
  return sck::launch_tonemap(ctx, reinterpret_cast<const float4*>(image), w, h, rgba8);
}

// ================================================================ optimiser
sc_status sc_adam_step(sc_ctx* ctx, float* params, const float* grads, float* m, float* v, uint64_t n, float lr,
                       uint64_t t, const sc_adam_config* cfg) {
  if (!ctx || !cfg || (n && (!params || !grads || !m || !v)) || t == 0) return SC_ERR_INVALID_ARG;
  const float bc1 = 1.0f - sc_powi_f32(cfg->beta1, (int)t);
  const float bc2 = 1.0f - sc_powi_f32(cfg->beta2, (int)t);
  return sck::launch_adam_lanes(ctx, params, grads, m, v, n, lr, cfg->beta1, cfg->beta2, cfg->eps, bc1, bc2);
}

sc_status sc_adam_step_all(sc_ctx* ctx, sc_splats* s, const sc_grads* g, sc_moments* mo, uint64_t t,
                           const sc_adam_groups* gr) {
  if (!ctx || !s || !g || !mo || !gr || t == 0) return SC_ERR_INVALID_ARG;
  if (g->cap < s->n || mo->cap < s->n) return sc_fail(ctx, SC_ERR_CAPACITY, "grads/moments smaller than the splat count");
  sck::AdamParams ap;
  for (int k = 0; k < 6; ++k) ap.lr[k] = gr->lr[k];
  ap.beta1 = gr->beta1; ap.beta2 = gr->beta2; ap.eps = gr->eps;
  ap.bc1 = 1.0f - sc_powi_f32(gr->beta1, (int)t);
  ap.bc2 = 1.0f - sc_powi_f32(gr->beta2, (int)t);
  ap.log_scale_min = ap.log_scale_max = ap.opacity_logit_max = 0.0f;
  ap.seed = (uint32_t)t;
  return sck::launch_adam_all(ctx, dview(s), g->slab, g->cap, dview(mo), ap);
}

sc_status sc_selftest_wait_timeout(sc_ctx* ctx) {
  if (!ctx) return SC_ERR_INVALID_ARG;
  return sck::selftest_lookback_timeout(ctx);
}

sc_status sc_adam_step_shard(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* acc, const float* g, uint32_t lo,
                             uint32_t count, uint32_t shard, uint64_t t, const sc_adam_groups* gr, float lsmin,
                             float lsmax, float opmax) {
  if (!ctx || !s || !mo || !gr || t == 0 || (count && !g)) return SC_ERR_INVALID_ARG;
  if (count > shard || (uint64_t)lo + count > s->n)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "shard range outside the splat count or wider than the chunk");
  if (mo->cap < s->n) return sc_fail(ctx, SC_ERR_CAPACITY, "moments smaller than the splat count");
  sck::AdamParams ap;
  for (int k = 0; k < 6; ++k) ap.lr[k] = gr->lr[k];
  ap.beta1 = gr->beta1; ap.beta2 = gr->beta2; ap.eps = gr->eps;
  ap.bc1 = 1.0f - sc_powi_f32(gr->beta1, (int)t);
  ap.bc2 = 1.0f - sc_powi_f32(gr->beta2, (int)t);
  ap.log_scale_min = lsmin; ap.log_scale_max = lsmax; ap.opacity_logit_max = opmax;
  ap.seed = (uint32_t)t;
  return sck::launch_adam_shard(ctx, dview(s), dview(mo), acc, g, lo, count, shard, ap);
}

sc_status sc_splats_pack_range(sc_ctx* ctx, const sc_splats* s, uint32_t lo, uint32_t count, uint32_t shard,
                               float* out) {
  if (!ctx || !s || (count && !out)) return SC_ERR_INVALID_ARG;
  if (count > shard || (uint64_t)lo + count > s->n)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "pack range outside the splat count or wider than the chunk");
  return sck::launch_pack_params(ctx, dview(s), lo, count, shard, out);
}

sc_status sc_splats_unpack_shards(sc_ctx* ctx, sc_splats* s, const float* in, uint32_t n_shards, uint32_t shard) {
  if (!ctx || !s || (n_shards && shard && !in)) return SC_ERR_INVALID_ARG;
  if ((uint64_t)n_shards * shard < s->n)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "gathered chunks cover fewer splats than the store holds");
  return sck::launch_unpack_params(ctx, dview(s), in, n_shards, shard);
}

sc_status sc_moments_pack_range(sc_ctx* ctx, const sc_moments* mo, uint32_t lo, uint32_t count, uint32_t shard,
                                float* out) {
  if (!ctx || !mo || (count && !out)) return SC_ERR_INVALID_ARG;
  if (count > shard || (uint64_t)lo + count > mo->cap)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "pack range outside the moments or wider than the chunk");
  return sck::launch_pack_moments(ctx, dview(mo), lo, count, shard, out);
}

sc_status sc_moments_unpack_shards(sc_ctx* ctx, sc_moments* mo, uint32_t n, const float* in, uint32_t n_shards,
                                   uint32_t shard) {
  if (!ctx || !mo || (n_shards && shard && !in)) return SC_ERR_INVALID_ARG;
  if (n > mo->cap || (uint64_t)n_shards * shard < n)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "moments unpack: n beyond capacity or not covered by the chunks");
  return sck::launch_unpack_moments(ctx, dview(mo), n, in, n_shards, shard);
}

sc_status sc_apply_constraints(sc_ctx* ctx, sc_splats* s, float lsmin, float lsmax, float opmax) {
  if (!ctx || !s) return SC_ERR_INVALID_ARG;
  return sck::launch_constraints(ctx, dview(s), lsmin, lsmax, opmax);
}

sc_status sc_accumulate_grad(sc_ctx* ctx, const sc_grads* g, float* acc, uint32_t n) {
  if (!ctx || !g || (n && !acc) || n > g->cap) return SC_ERR_INVALID_ARG;
  return sck::launch_accumulate(ctx, g->slab, g->cap, acc, n);
}

sc_status sc_prune_low_opacity(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* acc, float thr, uint32_t* removed) {
  if (!ctx || !s || !removed) return SC_ERR_INVALID_ARG;
  if (mo && mo->cap < s->n) return SC_ERR_INVALID_ARG;
  return sck::prune(ctx, s, mo, acc, thr, removed);
}

sc_status sc_densify(sc_ctx* ctx, sc_splats* s, sc_moments* mo, float* acc, uint32_t grad_count, float gthr,
                     float sthr, uint32_t max_splats, uint32_t iter, uint32_t counts[3]) {
  if (!ctx || !s || !acc || !counts) return SC_ERR_INVALID_ARG;
  if (mo && mo->cap < s->n) return SC_ERR_INVALID_ARG;
  return sck::densify(ctx, s, mo, acc, grad_count, gthr, sthr, max_splats, iter, counts);
}

}  // extern "C"
