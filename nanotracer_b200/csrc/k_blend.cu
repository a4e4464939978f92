// k_blend.cu — per-tile alpha blending (forward + adjoint), MSE, tonemap.
//
// Forward (rasterize.wgsl:48-118): one CTA per (view, tile); each thread owns
// PPT vertically adjacent pixels (a warp covers an 8 x 4 PPT block of the
// tile), two of them in packed f32x2 arithmetic.  The tile's depth-ordered
// list — its own pair list, or its super tile's item list filtered by the
// member masks — is staged into shared memory in batches of B list positions
// (the blend batch depth: one per thread by default, fewer when configured)
// with cp.async (3 x 16 B per record), double buffered so the gather
// of batch b+1 overlaps the blending of batch b, and the CTA leaves as soon as
// every pixel is saturated (T < 1e-4).  The MSE of loss.rs:163-179 — dL/dC =
// scale * 2 (C - target) / (3 W H) per pixel, squared errors reduced per CTA
// in FP64 — runs in the forward's epilogue or in the backward's prologue.
//
// Backward (rasterize_backward.wgsl:73-210): same grid, reverse walk from each
// pixel's last contributor (exact mode) or from the list's end (the
// reference's mode).  Per (pixel, splat) a thread forms the raw sums of the
// opacity gradient h and its moments (h, h dx, h dy, h dx^2, h dx dy, h dy^2)
// and the colour gradient over its pixels; two entries' 18 sums are reduced
// over the warp together by a recursive-halving reduce-scatter (20 shuffles)
// that leaves each total on one lane, which adds it to the entry's
// shared-memory slot; after each batch the slots become the splats' gradients
// (dmean.xy, dopacity, dconic.abc, dcolor.rgb, with the conic and opacity
// applied once per entry) and go to global memory with three float4 vector
// atomics per (tile, splat) — the reference issues nine CAS loops per (pixel,
// splat).  The transmittance reconstruction T_i = T_{i+1} / (1 - alpha_i) uses
// one approximate reciprocal per (pixel, splat).
#include "sc_internal.cuh"

namespace sck {

struct BlendArgs {
  uint32_t width, height, tw, th, tiles_x, tiles_y, num_tiles, stride;
  uint64_t pixels;  // per view
  uint32_t batch;   // list positions staged per batch, at most the block's threads
  const SceneDev* scenes;  // per-view image sizes and MSE scales (many-scene steps), or null
  bool count_pairs;        // with work counters: also count contributing (pixel, entry) pairs
};

static BlendArgs blend_args(const sc_tiling* tl, uint32_t stride) {
  BlendArgs a;
  a.width = tl->width; a.height = tl->height; a.tw = tl->tile_w; a.th = tl->tile_h;
  a.tiles_x = (tl->width + tl->tile_w - 1) / tl->tile_w;
  a.tiles_y = (tl->height + tl->tile_h - 1) / tl->tile_h;
  a.num_tiles = a.tiles_x * a.tiles_y;
  a.stride = stride;
  a.pixels = (uint64_t)tl->width * tl->height;
  a.batch = 0;
  a.scenes = nullptr;
  a.count_pairs = false;
  return a;
}

// a view's image size and MSE scale: the scene's in a many-scene step
__device__ __forceinline__ void view_dims(const BlendArgs& a, uint32_t v, float gscale, uint32_t& W, uint32_t& H,
                                          float& gs) {
  W = a.width; H = a.height; gs = gscale;
  if (a.scenes) {
    const SceneDev& sd = a.scenes[v];
    W = sd.width; H = sd.height; gs = sd.gscale;
  }
}

// The pixels of thread threadIdx.x in tile (tx, ty): PPT vertically adjacent
// pixels from (px, py0).  Where the tile splits that way (tile_w a multiple of
// 8, tile_h / PPT of 4) a warp takes an 8 x 4 PPT block, else whole rows of the
// tile.  The compact block leaves more entries that no pixel of a warp takes
// (the backward skips their reduction) and lets a warp's pixels saturate
// together (1M splats, 8 views of 1920x1080, 16 x 16 tiles: forward 1.016 ->
// 0.985 ms, backward 2.563 -> 2.515 ms against warps of 16 x 4 pixels).
template <int PPT>
__device__ __forceinline__ void tile_pixel(const BlendArgs& a, uint32_t tx, uint32_t ty, uint32_t& px,
                                           uint32_t& py0) {
  const uint32_t wl = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const bool blk = (a.tw & 7) == 0 && ((a.th / PPT) & 3) == 0;
  const uint32_t lx = blk ? (wl % (a.tw >> 3)) * 8 + (ln & 7) : threadIdx.x % a.tw;
  const uint32_t lr = blk ? (wl / (a.tw >> 3)) * 4 + (ln >> 3) : threadIdx.x / a.tw;
  px = tx * a.tw + lx;
  py0 = ty * a.th + PPT * lr;
}

// the batch depth for a launch of `threads` threads: `batch` rounded down to
// whole warps and capped at the threads (each stages one position), 0 = threads
static uint32_t batch_depth(uint32_t batch, uint32_t threads) {
  batch &= ~31u;
  return (batch == 0 || batch > threads) ? threads : batch;
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
#define FULL_MASK 0xffffffffu

// e^(-q/2) = 2^(q * NEG_HALF_LOG2E), log2 e = 1 / ln 2
#define NEG_HALF_LOG2E (-0.72134752044448170368f)

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }

// The conic's quadratic form at (dx, dy) is A + B dy + c dy^2 with A = a dx^2
// and B = 2 b dx, shared by a thread's pixels in one column; per pixel it is
// evaluated as (c dy + B) dy + A.  Every rounding step is written out (no
// contraction left to the compiler), so the one-pixel path and the packed
// two-pixel path (sm_100 f32x2 instructions) produce the same bits.
struct EntryGeom {
  float dx, A, B;
};
__device__ __forceinline__ EntryGeom entry_geom(float fx, const float4 ra, const float4 rb) {
  EntryGeom e;
  e.dx = __fadd_rn(fx, -ra.x);
  e.A = __fmul_rn(__fmul_rn(rb.x, e.dx), e.dx);
  e.B = __fmul_rn(2.0f * rb.y, e.dx);
  return e;
}

// Gaussian weight and alpha of one (pixel, splat); false when the reference
// skips the pair (power = -quad/2 > 0, or alpha < 1/255).  Shared by forward
// and backward so both make identical skip decisions.
__device__ __forceinline__ bool eval_alpha(const EntryGeom& e, float c, float dy, float op, float& g,
                                           float& alpha_raw, float& alpha) {
  const float quad = __fmaf_rn(__fmaf_rn(c, dy, e.B), dy, e.A);
  g = ex2_approx(__fmul_rn(quad, NEG_HALF_LOG2E));
  alpha_raw = __fmul_rn(op, g);
  alpha = fminf(alpha_raw, ALPHA_MAX);
  return quad >= 0.0f && alpha >= ALPHA_MIN;
}

// The same for a thread's two pixels (rows fy.x, fy.y of one column) with
// packed arithmetic; v0, v1 are the per-pixel results of eval_alpha.
__device__ __forceinline__ void eval_alpha2(const EntryGeom& e, float c, float2 fy, float ry, float op, float2& dy,
                                            float2& g, float2& alpha_raw, float2& alpha, bool& v0, bool& v1) {
  dy = __fadd2_rn(fy, f2(-ry));
  const float2 quad = __ffma2_rn(__ffma2_rn(f2(c), dy, f2(e.B)), dy, f2(e.A));
  const float2 ex = __fmul2_rn(quad, f2(NEG_HALF_LOG2E));
  g = make_float2(ex2_approx(ex.x), ex2_approx(ex.y));
  alpha_raw = __fmul2_rn(f2(op), g);
  alpha = make_float2(fminf(alpha_raw.x, ALPHA_MAX), fminf(alpha_raw.y, ALPHA_MAX));
  v0 = quad.x >= 0.0f && alpha.x >= ALPHA_MIN;
  v1 = quad.y >= 0.0f && alpha.y >= ALPHA_MIN;
}

template <typename T>
__device__ __forceinline__ T block_sum(T x, T* sred) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
  if (lane == 0) sred[warp] = x;
  __syncthreads();
  T r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sred[w];
  return r;  // valid in thread 0
}

// MSE term of one pixel (loss.rs:163-179): returns dL/dC = gscale (C - target)
// and adds the squared error to sq.  The forward epilogue and the backward
// prologue both use it, so either pass can own the loss.
__device__ __forceinline__ float3 mse_pixel(float cr, float cg, float cb, const float* __restrict__ tgt, float gscale,
                                            double& sq) {
  const float dx = __fadd_rn(cr, -tgt[0]), dy = __fadd_rn(cg, -tgt[1]), dz = __fadd_rn(cb, -tgt[2]);
  sq += (double)__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
  return make_float3(__fmul_rn(dx, gscale), __fmul_rn(dy, gscale), __fmul_rn(dz, gscale));
}

// Work counters of one blend launch (when given): per CTA, the list positions
// its batches covered and the entries it staged, added into one of
// BLEND_WORK_SLOTS (scanned, staged) pairs so that the atomics spread.
__device__ __forceinline__ void add_work(unsigned long long* work, uint32_t scanned, uint32_t staged) {
  if (work && threadIdx.x == 0 && scanned) {
    unsigned long long* w = work + 2 * (blockIdx.x % BLEND_WORK_SLOTS);
    atomicAdd(w, (unsigned long long)scanned);
    atomicAdd(w + 1, (unsigned long long)staged);
  }
}

// With COUNT, a blend launch also counts its contributing (pixel, entry)
// pairs (a pixel that takes an entry's alpha): the CTA's sum goes to the slot
// after the BLEND_WORK_SLOTS (scanned, staged) pairs.  Every thread of the CTA
// calls it; it ends with a barrier, so sred can be reused right after.
__device__ __forceinline__ void add_pixel_pairs(unsigned long long* work, uint32_t n, double* sred) {
  const double tot = block_sum((double)n, sred);
  if (threadIdx.x == 0 && tot > 0.0)
    atomicAdd(work + 2 * BLEND_WORK_SLOTS + blockIdx.x % BLEND_WORK_SLOTS, (unsigned long long)tot);
  __syncthreads();
}

// Pixel placement: thread t owns column t % tw and rows PPT*(t / tw) + k.

// Where a CTA's depth-ordered splat list comes from.  LIST_PAIRS: the tile's
// pair list, ids[ranges[view * tiles + tile]].  LIST_ITEMS: its super tile's
// item list, ids[ranges[view * super tiles + super tile]], of which the CTA
// keeps the items whose member mask (bits 16..31 of keys; bit (ty % 4) * 4 +
// tx % 4 is tile (tx, ty)) holds its tile.  Both lists are in depth order, so
// a tile blends the same splats in the same order either way.
enum { LIST_PAIRS = 0, LIST_ITEMS = 1 };
struct ListArgs {
  const uint32_t* ids;
  const uint2* ranges;
  const uint32_t* keys;  // LIST_ITEMS
  uint32_t super_x, super_per_view;
};

template <int LIST>
__device__ __forceinline__ uint2 list_range(const ListArgs& l, const BlendArgs& a, uint32_t v, uint32_t tx,
                                            uint32_t ty, uint32_t tile, uint32_t& bit) {
  if (LIST == LIST_PAIRS) {
    bit = 0;
    return l.ranges[(size_t)v * a.num_tiles + tile];
  }
  bit = (ty % SC_SUPER) * SC_SUPER + tx % SC_SUPER;
  return l.ranges[(size_t)v * l.super_per_view + (ty / SC_SUPER) * l.super_x + tx / SC_SUPER];
}

// Staging a batch of list positions [p0, p1) (at most B <= blockDim of them) as
// entries takes two calls, so that a batch's list words are loaded one batch
// ahead of their use: fetch_list loads this thread's position (the id and, for
// item lists, the key); place_list then stages the entries — each one's record
// (3 float4) into rbuf by cp.async, its id into ids_out (when given) and, for
// item lists, its position relative to `base` into pos.  Pair lists stage
// every position (entry k = position p0 + k); item lists keep the items of the
// CTA's tile in list order (a ballot per warp, then a prefix over the warps'
// counts in wcnt).  place_list returns the entry count; every thread of the
// CTA calls it.
struct ListWord {
  uint32_t key, id, j;
  bool valid;
};

template <int LIST>
__device__ __forceinline__ ListWord fetch_list(const ListArgs& l, uint32_t p0, uint32_t p1) {
  ListWord f;
  f.j = p0 + threadIdx.x;
  f.valid = f.j < p1;
  f.key = 0;
  f.id = 0;
  if (f.valid) {
    if (LIST == LIST_ITEMS) f.key = l.keys[f.j];
    f.id = l.ids[f.j];
  }
  return f;
}

template <int LIST>
__device__ __forceinline__ uint32_t place_list(const ListWord& f, uint32_t count, const float4* vrec, uint32_t bit,
                                               uint32_t base, float4* rbuf, uint32_t* pos, uint32_t* ids_out,
                                               uint32_t* wcnt) {
  const uint32_t t = threadIdx.x;
  bool keep = f.valid;
  uint32_t slot = t, total = count;
  if (LIST == LIST_ITEMS) {
    keep = keep && ((f.key >> (16u + bit)) & 1u);
    const uint32_t bal = __ballot_sync(FULL_MASK, keep);
    const uint32_t lane = t & 31u, warp = t >> 5;
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) {
      const uint32_t c = wcnt[w];
      before += w < warp ? c : 0u;
      total += c;
    }
    slot = before + __popc(bal & ((1u << lane) - 1u));
  }
  if (keep) {
    const float4* src = vrec + (size_t)3 * f.id;
    float4* dst = rbuf + 3 * slot;
    cp_async16(dst, src);
    cp_async16(dst + 1, src + 1);
    cp_async16(dst + 2, src + 2);
    if (LIST == LIST_ITEMS) pos[slot] = f.j - base;
    if (ids_out) ids_out[slot] = f.id;
  }
  cp_async_commit();
  return total;
}

// ---------------------------------------------------------------- forward
template <int PPT, int LIST, bool COUNT>
__global__ void __launch_bounds__(256) k_composite(const float4* __restrict__ rec, ListArgs l, BlendArgs a,
                                                   float4* __restrict__ image, uint2* __restrict__ aux,
                                                   const float* __restrict__ target, float gscale,
                                                   float4* __restrict__ dl_dc, double* __restrict__ loss,
                                                   const uint32_t* __restrict__ skip,
                                                   unsigned long long* __restrict__ work) {
  extern __shared__ float4 sbuf[];  // records [2][B][3], item positions [2][B] (u32)
  __shared__ double sred[8];
  __shared__ uint32_t s_wcnt[2][8];
  if (skip && (*skip & SC_DEVERR_CAPACITY)) return;  // the lists of this step are incomplete
  const uint32_t B = a.batch;
  uint32_t* spos = reinterpret_cast<uint32_t*>(sbuf + (size_t)6 * B);
  const uint32_t vt = blockIdx.x;
  const uint32_t v = vt / a.num_tiles, tile = vt - v * a.num_tiles;
  const uint32_t ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
  uint32_t px, py0;
  tile_pixel<PPT>(a, tx, ty, px, py0);
  const float fx = (float)px + 0.5f;
  uint32_t W, H;
  float gs;
  view_dims(a, v, gscale, W, H, gs);
  uint32_t bit;
  const uint2 r = list_range<LIST>(l, a, v, tx, ty, tile, bit);
  const uint32_t begin = r.x, end = r.y > r.x ? r.y : r.x;
  const uint32_t nb = (end - begin + B - 1) / B;
  const float4* vrec = rec + (size_t)3 * v * a.stride;

  auto fetch = [&](uint32_t b) -> ListWord {
    const uint32_t p0 = begin + b * B;
    return fetch_list<LIST>(l, p0, min(end, p0 + B));
  };
  auto place = [&](uint32_t b, const ListWord& f) -> uint32_t {
    return place_list<LIST>(f, min(B, end - (begin + b * B)), vrec, bit, begin, sbuf + (size_t)(b & 1) * 3 * B,
                            spos + (b & 1) * B, nullptr, s_wcnt[b & 1]);
  };
  // list position (relative to begin) of entry k of batch b
  auto position = [&](uint32_t b, uint32_t k) -> uint32_t {
    return LIST == LIST_PAIRS ? b * B + k : spos[(b & 1) * B + k];
  };

  float T[PPT], cr[PPT], cg[PPT], cb[PPT], fy[PPT];
  uint32_t last[PPT];
  bool done[PPT];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    T[k] = 1.0f; cr[k] = cg[k] = cb[k] = 0.f; last[k] = 0;
    fy[k] = (float)(py0 + k) + 0.5f;
    done[k] = !(px < W && py0 + k < H);
    all_done &= done[k];
  }
  ListWord f = fetch(0);
  uint32_t cnt_next = nb > 0 ? place(0, f) : 0u;
  if (nb > 1) f = fetch(1);
  uint32_t w_scan = 0, w_staged = 0, w_pix = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint32_t cnt = cnt_next;
    w_scan += min(B, end - (begin + b * B));
    w_staged += cnt;
    if (b + 1 < nb) {
      cnt_next = place(b + 1, f);
      if (b + 2 < nb) f = fetch(b + 2);
      cp_async_wait_one();
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    if (!all_done) {
      const float4* sb = sbuf + (size_t)(b & 1) * 3 * B;
      if constexpr (PPT == 2) {
        // both pixels in packed arithmetic; a pixel that skips the splat gets
        // alpha 0, which leaves its colour and T bit for bit unchanged.  A
        // pixel is done exactly when its T < 1e-4 (a pixel outside the image,
        // never written, runs with T = 0).
        const bool in0 = px < W && py0 < H, in1 = px < W && py0 + 1 < H;
        float2 T2 = make_float2(in0 ? T[0] : 0.0f, in1 ? T[1] : 0.0f);
        float2 R2 = make_float2(cr[0], cr[1]), G2 = make_float2(cg[0], cg[1]), B2 = make_float2(cb[0], cb[1]);
        const float2 fy2 = make_float2(fy[0], fy[1]);
        int lk0 = -1, lk1 = -1;  // this batch's last contributing entries, as list positions below
        auto blend1 = [&](uint32_t k) {
          const float4 ra = sb[3 * k], rb = sb[3 * k + 1], rc = sb[3 * k + 2];
          const EntryGeom e = entry_geom(fx, ra, rb);
          float2 dy, g, araw, al;
          bool v0, v1;
          eval_alpha2(e, rb.z, fy2, ra.y, rc.w, dy, g, araw, al, v0, v1);
          v0 &= T2.x >= 1e-4f;
          v1 &= T2.y >= 1e-4f;
          // without a branch: a pixel that skips gets alpha 0, which changes no bit
          const float2 am = make_float2(v0 ? al.x : 0.0f, v1 ? al.y : 0.0f);
          const float2 ta = __fmul2_rn(T2, am);
          R2 = __ffma2_rn(ta, f2(rc.x), R2);
          G2 = __ffma2_rn(ta, f2(rc.y), G2);
          B2 = __ffma2_rn(ta, f2(rc.z), B2);
          T2 = __fmul2_rn(T2, __fadd2_rn(f2(1.0f), make_float2(-am.x, -am.y)));
          if constexpr (COUNT) w_pix += (uint32_t)v0 + (uint32_t)v1;
          lk0 = v0 ? (int)k : lk0;
          lk1 = v1 ? (int)k : lk1;
        };
        // one saturation test per four entries (1M splats, 8 views of 1920x1080:
        // 0.986 ms with a test per entry, 0.928 per two, 0.893 per four, no
        // gain per eight at 69 registers): an entry past a pixel's saturation
        // gives it alpha 0 and changes nothing
        uint32_t k = 0;
        bool sat = false;
        for (; k + 3 < cnt; k += 4) {
          blend1(k);
          blend1(k + 1);
          blend1(k + 2);
          blend1(k + 3);
          if (T2.x < 1e-4f && T2.y < 1e-4f) { sat = true; break; }
        }
        if (!sat)
          for (; k < cnt; ++k) blend1(k);
        if (lk0 >= 0) last[0] = position(b, (uint32_t)lk0) + 1;
        if (lk1 >= 0) last[1] = position(b, (uint32_t)lk1) + 1;
        done[0] = T2.x < 1e-4f;
        done[1] = T2.y < 1e-4f;
        T[0] = T2.x; T[1] = T2.y; cr[0] = R2.x; cr[1] = R2.y;
        cg[0] = G2.x; cg[1] = G2.y; cb[0] = B2.x; cb[1] = B2.y;
        all_done = done[0] && done[1];
      } else {
        for (uint32_t k = 0; k < cnt; ++k) {
          const float4 ra = sb[3 * k], rb = sb[3 * k + 1], rc = sb[3 * k + 2];
          const EntryGeom e = entry_geom(fx, ra, rb);
          all_done = true;
#pragma unroll
          for (int q = 0; q < PPT; ++q) {
            if (!done[q]) {
              float g, araw, alpha;
              if (eval_alpha(e, rb.z, __fadd_rn(fy[q], -ra.y), rc.w, g, araw, alpha)) {
                const float ta = __fmul_rn(T[q], alpha);
                cr[q] = __fmaf_rn(ta, rc.x, cr[q]);
                cg[q] = __fmaf_rn(ta, rc.y, cg[q]);
                cb[q] = __fmaf_rn(ta, rc.z, cb[q]);
                T[q] = __fmul_rn(T[q], __fadd_rn(1.0f, -alpha));
                if constexpr (COUNT) ++w_pix;
                last[q] = position(b, k) + 1;
                if (T[q] < 1e-4f) done[q] = true;
              }
            }
            all_done &= done[q];
          }
          if (all_done) break;
        }
      }
    }
    if (__syncthreads_count(all_done) == (int)blockDim.x) break;
  }
  cp_async_wait_all();
  add_work(work, w_scan, w_staged);
  if constexpr (COUNT) add_pixel_pairs(work, w_pix, sred);
  double sq = 0.0;
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const uint32_t py = py0 + q;
    if (px < W && py < H) {
      const size_t pix = (size_t)v * a.pixels + (size_t)py * a.width + px;
      image[pix] = make_float4(cr[q], cg[q], cb[q], 1.0f - T[q]);
      if (aux) aux[pix] = make_uint2(__float_as_uint(T[q]), last[q]);
      if (target) {
        const float3 d = mse_pixel(cr[q], cg[q], cb[q], target + 3 * pix, gs, sq);
        dl_dc[pix] = make_float4(d.x, d.y, d.z, 0.0f);
      }
    }
  }
  if (target && loss) {
    const double s = block_sum(sq, sred);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(&loss[v], s);
  }
}

template <int PPT, int LIST>
static sc_status composite_ppt(sc_ctx* ctx, const BlendArgs& a, uint32_t grid, uint32_t threads, const float4* rec,
                               const ListArgs& l, float4* image, uint2* aux, const float* target, float gscale,
                               float4* dl_dc, double* loss, const uint32_t* d_skip, uint64_t* work) {
  const size_t smem = (size_t)2 * 3 * threads * sizeof(float4) + (size_t)2 * threads * sizeof(uint32_t);
  BlendArgs ab = a;
  ab.batch = batch_depth(a.batch, threads);
  unsigned long long* w = reinterpret_cast<unsigned long long*>(work);
  if (work && a.count_pairs)
    k_composite<PPT, LIST, true><<<grid, threads, smem, ctx->stream>>>(rec, l, ab, image, aux, target, gscale, dl_dc,
                                                                       loss, d_skip, w);
  else
    k_composite<PPT, LIST, false><<<grid, threads, smem, ctx->stream>>>(rec, l, ab, image, aux, target, gscale, dl_dc,
                                                                        loss, d_skip, w);
  return sc_check_launch(ctx, "k_composite");
}

// pixels per thread: 2 when the tile splits into whole warps that way (4 per
// thread measured slower in both kernels at 16x16 tiles: fewer warps per tile
// to hide the entry loop's latency, more registers)
static int pick_ppt(const sc_tiling* tl) {
  const uint32_t px = tl->tile_w * tl->tile_h;
  return (tl->tile_h % 2 == 0 && (px / 2) % 32 == 0) ? 2 : 1;
}

template <int LIST>
static sc_status composite_list(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views, const ListArgs& l,
                                const sc_tiling* tl, float4* image, uint2* aux, const float* target, float mse_scale,
                                float4* dl_dc, double* loss, const uint32_t* d_skip, uint64_t* work,
                                uint32_t batch, const SceneDev* scenes, bool count_pairs) {
  BlendArgs a = blend_args(tl, stride);
  a.batch = batch;
  a.scenes = scenes;
  a.count_pairs = count_pairs;
  const uint32_t pixels = tl->tile_w * tl->tile_h;
  if (pixels > 512 || pixels % 32 != 0) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile must hold 32..512 pixels, multiple of 32");
  const uint64_t grid = (uint64_t)n_views * a.num_tiles;
  if (grid == 0) return SC_OK;
  const float n_scalars = (float)tl->width * (float)tl->height * 3.0f;
  const float gscale = (2.0f / n_scalars) * mse_scale;
  const int ppt = pick_ppt(tl);
  if (ppt == 1 && pixels > 256) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile too large for one pixel per thread");
  if (ppt == 2)
    return composite_ppt<2, LIST>(ctx, a, (uint32_t)grid, pixels / 2, rec, l, image, aux, target, gscale, dl_dc, loss,
                                  d_skip, work);
  return composite_ppt<1, LIST>(ctx, a, (uint32_t)grid, pixels, rec, l, image, aux, target, gscale, dl_dc, loss,
                                d_skip, work);
}

sc_status launch_composite(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views, const uint32_t* payloads,
                           const uint32_t* ranges, const sc_tiling* tl, float4* image, uint2* aux, const float* target,
                           float mse_scale, float4* dl_dc, double* loss, const uint32_t* d_skip) {
  ListArgs l{payloads, reinterpret_cast<const uint2*>(ranges), nullptr, 0, 0};
  return composite_list<LIST_PAIRS>(ctx, rec, stride, n_views, l, tl, image, aux, target, mse_scale, dl_dc, loss,
                                    d_skip, nullptr, 0, nullptr, false);
}

sc_status launch_composite_items(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                 const uint32_t* item_keys, const uint32_t* item_ids, const uint32_t* item_ranges,
                                 const sc_tiling* tl, float4* image, uint2* aux, const float* target, float mse_scale,
                                 float4* dl_dc, double* loss, const uint32_t* d_skip, uint64_t* work,
                                 uint32_t batch, const SceneDev* scenes, bool count_pairs) {
  const BlendArgs a = blend_args(tl, stride);
  ListArgs l{item_ids, reinterpret_cast<const uint2*>(item_ranges), item_keys, (a.tiles_x + SC_SUPER - 1) / SC_SUPER,
             super_tiles_per_view(tl)};
  return composite_list<LIST_ITEMS>(ctx, rec, stride, n_views, l, tl, image, aux, target, mse_scale, dl_dc, loss,
                                    d_skip, work, batch, scenes, count_pairs);
}

// ---------------------------------------------------------------- MSE (standalone)
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
  return sc_check_launch(ctx, "k_mse_views");
}

// ---------------------------------------------------------------- backward
// Reduce-scatter of N values over the warp by recursive halving: at the level
// of lane bit O a lane keeps one half of its slots and sends the other half to
// lane ^ O, which keeps the opposite half (2 selects and 1 shuffle per slot
// pair, ceil(n / 2) slots left; the adds go two at a time as packed f32x2
// adds, the same roundings); after the 5 levels every lane holds one slot.
// rs_owner<N>(lane) is the value index that slot totals (-1: a padding
// slot).  N = 9: 12 shuffles; N = 18: 20.
template <int N, int O>
__device__ __forceinline__ float rs_level(const float* x, int lane) {
  constexpr int M = (N + 1) / 2;
  float y[M], kp[M], rv[M];
  const bool bit = lane & O;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const float lo = x[i];
    const float hi = i + M < N ? x[i + M] : 0.0f;
    const float send = bit ? lo : hi;
    kp[i] = bit ? hi : lo;
    rv[i] = __shfl_xor_sync(FULL_MASK, send, O);
  }
#pragma unroll
  for (int i = 0; i + 1 < M; i += 2) {
    const float2 t = __fadd2_rn(make_float2(kp[i], kp[i + 1]), make_float2(rv[i], rv[i + 1]));
    y[i] = t.x; y[i + 1] = t.y;
  }
  if constexpr (M & 1) y[M - 1] = kp[M - 1] + rv[M - 1];
  if constexpr (O == 1) {
    static_assert(M == 1, "at most 32 values");
    return y[0];
  } else {
    return rs_level<M, O / 2>(y, lane);
  }
}
template <int N>
__device__ __forceinline__ float warp_reduce_scatter(const float (&x)[N], int lane) {
  return rs_level<N, 16>(x, lane);
}
template <int N>
__device__ __forceinline__ int rs_owner(int lane) {
  int lo = 0, len = N, n = N;
  for (int o = 16; o >= 1; o >>= 1) {
    const int m = (n + 1) / 2;
    if (lane & o) { lo += m; len = max(len - m, 0); } else { len = min(len, m); }
    n = m;
  }
  return len >= 1 ? lo : -1;
}

// Entries per warp reduction: 2 (an 18-value reduce-scatter, 20 shuffles for
// two entries).  3 entries (27 values, 28 shuffles) measured slower at 80
// registers; more than 3 do not fit the 32 lanes.
constexpr int RS_E = 2;

// Compensated accumulation of x into the sum *s, the rounding error of the
// addition going to *c: the atomic returns the old sum, the device forms the
// same rounded sum again (an atomic float add rounds to nearest) and Knuth's
// TwoSum gives the exact error of that addition.  *s + *c then carries the
// total to within about one rounding of the final value, whatever the number
// and the order of the tiles that add to it (plain float atomics: an error
// growing with the number of additions and their magnitudes).
__device__ __forceinline__ void twosum_atomic_add(float* s, float* c, float x) {
  if (x == 0.0f) return;
  const float old = atomicAdd(s, x);
  const float sum = __fadd_rn(old, x);
  const float bp = __fsub_rn(sum, old);
  const float err = __fadd_rn(__fsub_rn(old, __fsub_rn(sum, bp)), __fsub_rn(x, bp));
  if (err != 0.0f) atomicAdd(c, err);
}
__device__ __forceinline__ void twosum_atomic_add4(float4* s, float4* c, float4 x) {
  float* sp = reinterpret_cast<float*>(s);
  float* cp = reinterpret_cast<float*>(c);
  twosum_atomic_add(sp, cp, x.x);
  twosum_atomic_add(sp + 1, cp + 1, x.y);
  twosum_atomic_add(sp + 2, cp + 2, x.z);
}

// MODE is the sc_bwd_mode.  In exact mode a pixel takes part from its last
// contributor down to the start of the tile's list and never stops early, so
// the early-exit bookkeeping exists only in reference mode.
// With a target, the MSE's dL/dC (and the loss, added to loss[view]) is formed
// here from the forward image instead of being read from dl_dc.
// COMP: the per-(view, splat) totals across tiles are accumulated with
// twosum_atomic_add into proj_grad and the compensation records proj_comp.
template <int PPT, int MODE, int LIST, bool COMP, bool COUNT>
__global__ void __launch_bounds__(256) k_composite_backward(const float4* __restrict__ rec, ListArgs l, BlendArgs a,
                                                            const float4* __restrict__ fwd,
                                                            const float4* __restrict__ dl_dc,
                                                            const float* __restrict__ target, float gscale,
                                                            double* __restrict__ loss,
                                                            const uint2* __restrict__ aux,
                                                            float4* __restrict__ proj_grad,
                                                            const uint32_t* __restrict__ skip,
                                                            unsigned long long* __restrict__ work,
                                                            float4* __restrict__ proj_comp) {
  // records [2][B][3], acc [B][3] (float4), ids [2][B], item positions [2][B] (u32)
  extern __shared__ float4 sbuf[];
  __shared__ uint32_t s_max;
  __shared__ double s_red[8];
  __shared__ uint32_t s_wcnt[2][8];
  if (skip && (*skip & SC_DEVERR_CAPACITY)) return;
  const uint32_t B = a.batch;
  float4* sacc = sbuf + (size_t)6 * B;
  uint32_t* sids = reinterpret_cast<uint32_t*>(sbuf + (size_t)9 * B);
  uint32_t* spos = sids + 2 * B;
  const uint32_t vt = blockIdx.x;
  const uint32_t v = vt / a.num_tiles, tile = vt - v * a.num_tiles;
  const uint32_t ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
  uint32_t px, py0;
  tile_pixel<PPT>(a, tx, ty, px, py0);
  const float fx = (float)px + 0.5f;
  uint32_t W, H;
  float gs;
  view_dims(a, v, gscale, W, H, gs);
  uint32_t bit;
  const uint2 r = list_range<LIST>(l, a, v, tx, ty, tile, bit);
  const uint32_t begin = r.x, end = r.y > r.x ? r.y : r.x;
  const float4* vrec = rec + (size_t)3 * v * a.stride;
  float4* vgrad = proj_grad + (size_t)3 * v * a.stride;

  // GS = dL/dC . S, the accumulated colour behind the pixel dotted with its
  // colour gradient: dL/dalpha_i = (T_{i+1} (dL/dC . c_i) - GS) / (1 - alpha_i)
  float T[PPT], gr[PPT], gg[PPT], gb[PPT], GS[PPT], fy[PPT];
  uint32_t stop[PPT];
  bool done[PPT];
  uint32_t tstop = begin;
  bool all_done = true;
  double sq = 0.0;
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const uint32_t py = py0 + q;
    fy[q] = (float)py + 0.5f;
    T[q] = 1.0f; gr[q] = gg[q] = gb[q] = 0.f; GS[q] = 0.f;
    stop[q] = begin;
    done[q] = !(px < W && py < H);
    if (!done[q]) {
      const size_t pix = (size_t)v * a.pixels + (size_t)py * a.width + px;
      float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
      if (target || MODE == SC_BWD_REF) c = fwd[pix];
      if (target) {
        const float3 d = mse_pixel(c.x, c.y, c.z, target + 3 * pix, gs, sq);
        gr[q] = d.x; gg[q] = d.y; gb[q] = d.z;
      } else {
        const float4 d = dl_dc[pix];
        gr[q] = d.x; gg[q] = d.y; gb[q] = d.z;
      }
      if (MODE == SC_BWD_REF) {
        T[q] = 1.0f - c.w;
        stop[q] = end;
      } else {
        const uint2 x = aux[pix];
        T[q] = __uint_as_float(x.x);
        stop[q] = begin + min(x.y, end - begin);
      }
      tstop = max(tstop, stop[q]);
    }
    all_done &= done[q];
  }
  if (target && loss) {  // every CTA, the ones with an empty list too
    const double sum = block_sum(sq, s_red);
    if (threadIdx.x == 0 && sum != 0.0) atomicAdd(&loss[v], sum);
  }
  if (end <= begin) return;
  if (threadIdx.x == 0) s_max = begin;
  if (threadIdx.x < B) {
    sacc[3 * threadIdx.x] = make_float4(0, 0, 0, 0);
    sacc[3 * threadIdx.x + 1] = make_float4(0, 0, 0, 0);
    sacc[3 * threadIdx.x + 2] = make_float4(0, 0, 0, 0);
  }
  __syncthreads();
  if (tstop > begin) atomicMax(&s_max, tstop);
  __syncthreads();
  const uint32_t hi0 = s_max;
  if (hi0 <= begin) return;
  const uint32_t nb = (hi0 - begin + B - 1) / B;
  // batch b: list positions [hi - min(B, hi - begin), hi), hi = hi0 - b B
  auto fetch = [&](uint32_t b) -> ListWord {
    const uint32_t hi = hi0 - b * B, lo = hi - min(B, hi - begin);
    return fetch_list<LIST>(l, lo, hi);
  };
  auto place = [&](uint32_t b, const ListWord& f) -> uint32_t {
    const uint32_t hi = hi0 - b * B, lo = hi - min(B, hi - begin);
    return place_list<LIST>(f, hi - lo, vrec, bit, begin, sbuf + (size_t)(b & 1) * 3 * B, spos + (b & 1) * B,
                            sids + (b & 1) * B, s_wcnt[b & 1]);
  };

  const int lane = threadIdx.x & 31;
  // after the 18-value reduce-scatter of entries (k, k - 1) this lane adds one
  // value: of entry k - rs_ent, at float rs_off of its 3 float4 slot (w unused)
  const int rs_idx = rs_owner<9 * RS_E>(lane);
  const int rs_ent = rs_idx / 9;
  const int rs_off = rs_idx >= 0 ? rs_idx % 9 + (rs_idx % 9) / 3 : -1;
  ListWord f = fetch(0);
  uint32_t cnt_next = place(0, f);
  if (nb > 1) f = fetch(1);
  uint32_t w_staged = 0, w_pix = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint32_t cnt = cnt_next;
    w_staged += cnt;
    if (b + 1 < nb) {
      cnt_next = place(b + 1, f);
      if (b + 2 < nb) f = fetch(b + 2);
      cp_async_wait_one();
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    const uint32_t hi = hi0 - b * B;
    const uint32_t lo = hi - min(B, hi - begin);
    const uint32_t* bpos = spos + (b & 1) * B;
    const float4* sb = sbuf + (size_t)(b & 1) * 3 * B;
    if (!__all_sync(FULL_MASK, all_done)) {
      float2 T2 = make_float2(T[0], T[PPT - 1]), GS2 = make_float2(GS[0], GS[PPT - 1]);
      const float2 gr2 = make_float2(gr[0], gr[PPT - 1]), gg2 = make_float2(gg[0], gg[PPT - 1]);
      const float2 gb2 = make_float2(gb[0], gb[PPT - 1]), fy2 = make_float2(fy[0], fy[PPT - 1]);
      // one entry: this thread's raw sums of it into c[0..8] (zeros when none of
      // its pixels takes part); returns whether one does
      auto entry = [&](int k, float* c) -> bool {
          const uint32_t j = LIST == LIST_PAIRS ? lo + (uint32_t)k : begin + bpos[k];
          // this thread's sums over its pixels: h = dL/dalpha * gauss (the opacity
          // gradient), its first and second moments in (dx, dy), and the colour
          // gradient; the per-splat terms are formed from them once per entry
          float sh = 0.f, shx = 0.f, shy = 0.f, shxx = 0.f, shxy = 0.f, shyy = 0.f;
          float scr = 0.f, scg = 0.f, scb = 0.f;
          bool contrib = false;
          const float4 ra = sb[3 * k], rb = sb[3 * k + 1], rc = sb[3 * k + 2];
          const EntryGeom e = entry_geom(fx, ra, rb);
          if constexpr (PPT == 2) {
            // both pixels in packed arithmetic; a pixel that skips the splat gets
            // zero alpha and weight, so it adds nothing and keeps its T
            float2 dy, g, araw, al;
            bool v0, v1;
            eval_alpha2(e, rb.z, fy2, ra.y, rc.w, dy, g, araw, al, v0, v1);
            v0 &= (MODE == SC_BWD_EXACT || !done[0]) && j < stop[0];
            v1 &= (MODE == SC_BWD_EXACT || !done[1]) && j < stop[1];
            // the exact mode takes no branch here: with both pixels skipping, every
            // sum below is zero and T and GS keep their values
            if (MODE == SC_BWD_REF ? (v0 || v1) : true) {
              const float2 oma = __fadd2_rn(f2(1.0f), make_float2(-al.x, -al.y));
              const float2 inv = make_float2(rcp_approx(oma.x), rcp_approx(oma.y));
              const float2 Tn = __fmul2_rn(T2, inv);  // T_i = T_{i+1} / (1 - alpha_i)
              if (MODE == SC_BWD_REF) {
                if (v0 && Tn.x > 1.0001f) { done[0] = true; v0 = false; }
                if (v1 && Tn.y > 1.0001f) { done[1] = true; v1 = false; }
              }
              if (MODE == SC_BWD_REF ? (v0 || v1) : true) {
                const float2 am = make_float2(v0 ? al.x : 0.0f, v1 ? al.y : 0.0f);
                const float2 gm = make_float2(v0 && araw.x < ALPHA_MAX ? g.x : 0.0f,
                                              v1 && araw.y < ALPHA_MAX ? g.y : 0.0f);
                const float2 ta = __fmul2_rn(Tn, am);
                const float2 p = __fmul2_rn(ta, gr2), q = __fmul2_rn(ta, gg2), w = __fmul2_rn(ta, gb2);
                scr = p.x + p.y; scg = q.x + q.y; scb = w.x + w.y;
                // dC/dalpha = T_i c - S / (1 - alpha) = (T_{i+1} c - S) / (1 - alpha)
                const float2 dc = __ffma2_rn(gb2, f2(rc.z), __ffma2_rn(gg2, f2(rc.y), __fmul2_rn(gr2, f2(rc.x))));
                const float2 galpha = __fmul2_rn(inv, __ffma2_rn(T2, dc, make_float2(-GS2.x, -GS2.y)));
                const float2 h = __fmul2_rn(galpha, gm);
                const float2 hy = __fmul2_rn(h, dy);
                sh = h.x + h.y;
                shy = hy.x + hy.y;
                shyy = fmaf(hy.x, dy.x, hy.y * dy.y);
                shx = sh * e.dx;  // both pixels share dx
                shxx = shx * e.dx;
                shxy = shy * e.dx;
                GS2 = __ffma2_rn(ta, dc, GS2);
                T2 = make_float2(v0 ? Tn.x : T2.x, v1 ? Tn.y : T2.y);
                if constexpr (COUNT) w_pix += (uint32_t)v0 + (uint32_t)v1;
                contrib = v0 || v1;
              }
            }
            if (MODE == SC_BWD_REF) all_done = (done[0] || j <= begin) && (done[1] || j <= begin);
          } else {
            all_done = true;
  #pragma unroll
            for (int q = 0; q < PPT; ++q) {
              if ((MODE == SC_BWD_EXACT || !done[q]) && j < stop[q]) {
                const float dy = __fadd_rn(fy[q], -ra.y);
                float g, araw, alpha;
                if (eval_alpha(e, rb.z, dy, rc.w, g, araw, alpha)) {
                  const float inv = rcp_approx(__fadd_rn(1.0f, -alpha));
                  const float Tn = __fmul_rn(T[q], inv);  // T_i = T_{i+1} / (1 - alpha_i)
                  if (MODE == SC_BWD_REF && Tn > 1.0001f) {
                    done[q] = true;
                  } else {
                    const float ta = __fmul_rn(Tn, alpha);
                    scr += gr[q] * ta; scg += gg[q] * ta; scb += gb[q] * ta;
                    const float dc = gr[q] * rc.x + gg[q] * rc.y + gb[q] * rc.z;
                    const float galpha = inv * (T[q] * dc - GS[q]);
                    const float h = araw < ALPHA_MAX ? galpha * g : 0.0f;
                    const float hx = h * e.dx, hy = h * dy;
                    sh += h;
                    shx += hx; shy += hy;
                    shxx += hx * e.dx; shxy += hx * dy; shyy += hy * dy;
                    GS[q] += ta * dc;
                    T[q] = Tn;
                    if constexpr (COUNT) ++w_pix;
                    contrib = true;
                  }
                }
              }
              if (MODE == SC_BWD_REF) all_done &= done[q] || j <= begin;
            }
          }
        c[0] = shx; c[1] = shy; c[2] = sh; c[3] = shxx; c[4] = shxy; c[5] = shyy;
        c[6] = scr; c[7] = scg; c[8] = scb;
        return contrib;
      };
      // entries k .. k - RS_E + 1 together: one 9 RS_E-value reduce-scatter
      for (int k = (int)cnt - 1; k >= 0; k -= RS_E) {
        float c[9 * RS_E];
        bool any = false;
#pragma unroll
        for (int q = 0; q < RS_E; ++q) {
          if (k - q >= 0) {
            any |= entry(k - q, c + 9 * q);
          } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) c[9 * q + i] = 0.0f;
          }
        }
        if (MODE == SC_BWD_EXACT) all_done = false;
        if (__any_sync(FULL_MASK, any)) {
          // the splats' raw sums; the flush turns them into their gradients
          const float w = warp_reduce_scatter<9 * RS_E>(c, lane);
          if (rs_off >= 0 && k >= rs_ent) atomicAdd(reinterpret_cast<float*>(sacc + 3 * (k - rs_ent)) + rs_off, w);
        }
        if (MODE == SC_BWD_REF && __all_sync(FULL_MASK, all_done)) break;
      }
      if constexpr (PPT == 2) {
        T[0] = T2.x; T[1] = T2.y; GS[0] = GS2.x; GS[1] = GS2.y;
      }
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
      // the entry's sums over the CTA's pixels of h = dL/dalpha * gauss and its
      // moments in (dx, dy) become, with the splat's opacity and conic (a, b, c)
      // (rasterize_backward.wgsl:174-185): dpower = op h, dmean = dpower (a dx +
      // b dy, b dx + c dy), dconic = dpower (-1/2)(dx^2, 2 dx dy, dy^2); the
      // opacity and colour gradients are the sums themselves
      float4* acc = sacc + 3 * threadIdx.x;
      const float4 m0 = acc[0], m1 = acc[1], a2 = acc[2];  // (SHX, SHY, SH), (SHXX, SHXY, SHYY), colour
      const float4 cb = sb[3 * threadIdx.x + 1];
      const float op = sb[3 * threadIdx.x + 2].w;
      const float4 a0 = make_float4(op * (cb.x * m0.x + cb.y * m0.y), op * (cb.y * m0.x + cb.z * m0.y), m0.z, 0.0f);
      const float4 a1 = make_float4(-0.5f * op * m1.x, -op * m1.y, -0.5f * op * m1.z, 0.0f);
      const uint32_t id = sids[(b & 1) * B + threadIdx.x];
      float4* dst = vgrad + (size_t)3 * id;
      if constexpr (COMP) {
        float4* cdst = proj_comp + (size_t)3 * v * a.stride + (size_t)3 * id;
        twosum_atomic_add4(dst, cdst, a0);
        twosum_atomic_add4(dst + 1, cdst + 1, a1);
        twosum_atomic_add4(dst + 2, cdst + 2, a2);
      } else {
        if (a0.x != 0.f || a0.y != 0.f || a0.z != 0.f) atomicAdd(dst, a0);
        if (a1.x != 0.f || a1.y != 0.f || a1.z != 0.f) atomicAdd(dst + 1, a1);
        if (a2.x != 0.f || a2.y != 0.f || a2.z != 0.f) atomicAdd(dst + 2, a2);
      }
      acc[0] = make_float4(0, 0, 0, 0); acc[1] = acc[0]; acc[2] = acc[0];
    }
    if (__syncthreads_count(all_done) == (int)blockDim.x) break;
  }
  cp_async_wait_all();
  add_work(work, hi0 - begin, w_staged);
  if constexpr (COUNT) add_pixel_pairs(work, w_pix, s_red);
}

template <int PPT, int LIST, int MODE>
static void backward_launch(const BlendArgs& a, uint32_t grid, uint32_t threads, size_t smem, cudaStream_t st,
                            const float4* rec, const ListArgs& l, const float4* fwd, const float4* dl_dc,
                            const float* target, float gscale, double* loss, const uint2* aux, float4* proj_grad,
                            const uint32_t* d_skip, unsigned long long* w, float4* proj_comp) {
  const bool count = w && a.count_pairs;
  if (proj_comp && count)
    k_composite_backward<PPT, MODE, LIST, true, true><<<grid, threads, smem, st>>>(
        rec, l, a, fwd, dl_dc, target, gscale, loss, aux, proj_grad, d_skip, w, proj_comp);
  else if (proj_comp)
    k_composite_backward<PPT, MODE, LIST, true, false><<<grid, threads, smem, st>>>(
        rec, l, a, fwd, dl_dc, target, gscale, loss, aux, proj_grad, d_skip, w, proj_comp);
  else if (count)
    k_composite_backward<PPT, MODE, LIST, false, true><<<grid, threads, smem, st>>>(
        rec, l, a, fwd, dl_dc, target, gscale, loss, aux, proj_grad, d_skip, w, nullptr);
  else
    k_composite_backward<PPT, MODE, LIST, false, false><<<grid, threads, smem, st>>>(
        rec, l, a, fwd, dl_dc, target, gscale, loss, aux, proj_grad, d_skip, w, nullptr);
}

template <int PPT, int LIST>
static sc_status backward_ppt(sc_ctx* ctx, const BlendArgs& a, uint32_t grid, uint32_t threads, const float4* rec,
                              const ListArgs& l, const float4* fwd, const float4* dl_dc, const float* target,
                              float gscale, double* loss, int mode, const uint2* aux, float4* proj_grad,
                              const uint32_t* d_skip, uint64_t* work, float4* proj_comp) {
  const size_t smem = (size_t)9 * threads * sizeof(float4) + (size_t)4 * threads * sizeof(uint32_t);
  unsigned long long* w = reinterpret_cast<unsigned long long*>(work);
  BlendArgs ab = a;
  ab.batch = batch_depth(a.batch, threads);
  if (mode == SC_BWD_EXACT)
    backward_launch<PPT, LIST, SC_BWD_EXACT>(ab, grid, threads, smem, ctx->stream, rec, l, fwd, dl_dc, target, gscale,
                                             loss, aux, proj_grad, d_skip, w, proj_comp);
  else
    backward_launch<PPT, LIST, SC_BWD_REF>(ab, grid, threads, smem, ctx->stream, rec, l, fwd, dl_dc, target, gscale,
                                           loss, aux, proj_grad, d_skip, w, proj_comp);
  return sc_check_launch(ctx, "k_composite_backward");
}

template <int LIST>
static sc_status backward_list(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views, const ListArgs& l,
                               const sc_tiling* tl, const float4* fwd, const float4* dl_dc, const float* target,
                               float mse_scale, double* loss, int mode, const uint2* aux, float4* proj_grad,
                               const uint32_t* d_skip, uint64_t* work, float4* proj_comp, uint32_t batch,
                               const SceneDev* scenes, bool count_pairs) {
  BlendArgs a = blend_args(tl, stride);
  a.batch = batch;
  a.scenes = scenes;
  a.count_pairs = count_pairs;
  const float gscale = (2.0f / ((float)tl->width * (float)tl->height * 3.0f)) * mse_scale;
  const uint32_t pixels = tl->tile_w * tl->tile_h;
  if (pixels > 512 || pixels % 32 != 0) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile must hold 32..512 pixels, multiple of 32");
  if (mode == SC_BWD_EXACT && !aux) return sc_fail(ctx, SC_ERR_INVALID_ARG, "exact backward needs the forward aux buffer");
  const uint64_t grid = (uint64_t)n_views * a.num_tiles;
  if (grid == 0) return SC_OK;
  const int ppt = pick_ppt(tl);
  if (ppt == 1 && pixels > 256) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile too large for one pixel per thread");
  if (ppt == 2)
    return backward_ppt<2, LIST>(ctx, a, (uint32_t)grid, pixels / 2, rec, l, fwd, dl_dc, target, gscale, loss, mode,
                                 aux, proj_grad, d_skip, work, proj_comp);
  return backward_ppt<1, LIST>(ctx, a, (uint32_t)grid, pixels, rec, l, fwd, dl_dc, target, gscale, loss, mode, aux,
                               proj_grad, d_skip, work, proj_comp);
}

sc_status launch_composite_backward(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                    const uint32_t* payloads, const uint32_t* ranges, const sc_tiling* tl,
                                    const float4* fwd, const float4* dl_dc, int mode, const uint2* aux,
                                    float4* proj_grad, const uint32_t* d_skip, const float* target,
                                    float mse_scale, double* loss, float4* proj_comp) {
  ListArgs l{payloads, reinterpret_cast<const uint2*>(ranges), nullptr, 0, 0};
  return backward_list<LIST_PAIRS>(ctx, rec, stride, n_views, l, tl, fwd, dl_dc, target, mse_scale, loss, mode, aux,
                                   proj_grad, d_skip, nullptr, proj_comp, 0, nullptr, false);
}

sc_status launch_composite_backward_items(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                          const uint32_t* item_keys, const uint32_t* item_ids,
                                          const uint32_t* item_ranges, const sc_tiling* tl, const float4* fwd,
                                          const float4* dl_dc, int mode, const uint2* aux, float4* proj_grad,
                                          const uint32_t* d_skip, const float* target, float mse_scale,
                                          double* loss, uint64_t* work, float4* proj_comp, uint32_t batch,
                                          const SceneDev* scenes, bool count_pairs) {
  const BlendArgs a = blend_args(tl, stride);
  ListArgs l{item_ids, reinterpret_cast<const uint2*>(item_ranges), item_keys, (a.tiles_x + SC_SUPER - 1) / SC_SUPER,
             super_tiles_per_view(tl)};
  return backward_list<LIST_ITEMS>(ctx, rec, stride, n_views, l, tl, fwd, dl_dc, target, mse_scale, loss, mode, aux,
                                   proj_grad, d_skip, work, proj_comp, batch, scenes, count_pairs);
}

// proj_grad += proj_comp over n float4 (the compensated totals rounded once)
__global__ void k_fold_comp(float4* __restrict__ g, const float4* __restrict__ c, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 x = g[i], y = c[i];
  g[i] = make_float4(x.x + y.x, x.y + y.y, x.z + y.z, x.w + y.w);
}

sc_status launch_fold_comp(sc_ctx* ctx, float4* proj_grad, const float4* proj_comp, uint64_t n_float4) {
  if (n_float4 == 0) return SC_OK;
  k_fold_comp<<<(unsigned)sc_div_up(n_float4, 256), 256, 0, ctx->stream>>>(proj_grad, proj_comp, n_float4);
  return sc_check_launch(ctx, "k_fold_comp");
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
