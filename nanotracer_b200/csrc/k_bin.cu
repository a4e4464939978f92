// k_bin.cu — tile binning: per-splat tile counts, pair emission, per-tile ranges.
//
// Reference-shaped path (sc_bin):  tile_count.wgsl:28-55 -> scan ->
// tile_emit.wgsl:36-67 -> radix sort -> tile_ranges.wgsl:22-41, extended to
// n_views views (tile ids view*num_tiles + tile) and two key layouts:
//   REF32   (tile << 16) | u16(clamp(depth / depth_max, 0, 1) * 65535)
//   NATIVE  ((view*num_tiles + tile) << 32) | float_bits(depth)   (u64)
// Emission order is (view, splat, ty, tx), so a stable key sort reproduces
// the reference's order exactly (ties resolve to ascending splat index).
//
// Trainer path: the splats of each view are first sorted, stably in index
// order, on the reference's 16-bit quantised depth (one segmented sort over
// the views), so every later stable sort keeps each tile's (depth16, splat
// index) order, the order of the REF32 keys.  Then either (sort_mode 1) pairs
// are emitted in that order with a u32 key (view << tile_bits) | tile and
// sorted on the tile bits alone, or (the default, two-level binning) one item
// per (view, super tile of 4 x 4 tiles, splat) is emitted with the tiles it
// reaches as a 16-bit member mask in the key, sorted on the super-tile bits in
// one pass, and each tile's blend keeps its super tile's items whose mask
// holds it.
#include "sc_internal.cuh"

namespace sck {

struct BinArgs {
  uint32_t tw, th, tiles_x, tiles_y, num_tiles;
  float depth_max;
  uint32_t tile_bits;  // presorted pipeline: pair key = (view << tile_bits) | tile
};

static BinArgs bin_args(const sc_tiling* tl) {
  BinArgs a;
  a.tw = tl->tile_w; a.th = tl->tile_h;
  a.tiles_x = (tl->width + tl->tile_w - 1) / tl->tile_w;
  a.tiles_y = (tl->height + tl->tile_h - 1) / tl->tile_h;
  a.num_tiles = a.tiles_x * a.tiles_y;
  a.depth_max = tl->depth_max;
  a.tile_bits = 0;
  while ((1u << a.tile_bits) <= a.num_tiles) ++a.tile_bits;  // 2^tile_bits > num_tiles
  return a;
}

__device__ __forceinline__ bool rect_of(const float4 ra, const float4 rb, const BinArgs& a, int& x0, int& y0, int& x1,
                                        int& y1) {
  if (rb.w == 0.0f) return false;
  const float tsw = (float)a.tw, tsh = (float)a.th;
  x0 = max((int)floorf(__fdiv_rn(ra.x - ra.w, tsw)), 0);
  y0 = max((int)floorf(__fdiv_rn(ra.y - ra.w, tsh)), 0);
  x1 = min((int)floorf(__fdiv_rn(ra.x + ra.w, tsw)), (int)a.tiles_x - 1);
  y1 = min((int)floorf(__fdiv_rn(ra.y + ra.w, tsh)), (int)a.tiles_y - 1);
  return !(x1 < x0 || y1 < y0);
}

__global__ void k_tile_count(const float4* __restrict__ rec, uint32_t n, uint32_t stride, uint32_t n_views, BinArgs a,
                             uint32_t* __restrict__ counts) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (uint64_t)n_views * n) return;
  const uint32_t v = (uint32_t)(q / n), i = (uint32_t)(q % n);
  const size_t o = (size_t)v * stride + i;
  int x0, y0, x1, y1;
  uint32_t c = 0;
  if (rect_of(rec[3 * o], rec[3 * o + 1], a, x0, y0, x1, y1)) c = (uint32_t)(x1 - x0 + 1) * (uint32_t)(y1 - y0 + 1);
  counts[q] = c;
}

sc_status launch_tile_count(sc_ctx* ctx, const float4* rec, uint32_t n, uint32_t stride, uint32_t n_views,
                            const sc_tiling* tl, uint32_t* counts) {
  const uint64_t total = (uint64_t)n * n_views;
  if (total == 0) return SC_OK;
  k_tile_count<<<(unsigned)sc_div_up(total, 256), 256, 0, ctx->stream>>>(rec, n, stride, n_views, bin_args(tl), counts);
  return sc_check_launch(ctx, "k_tile_count");
}

template <int MODE>
__global__ void k_tile_emit(const float4* __restrict__ rec, uint32_t n, uint32_t stride, uint32_t n_views, BinArgs a,
                            const uint32_t* __restrict__ offsets, void* __restrict__ keys_v,
                            uint32_t* __restrict__ payloads, uint64_t cap) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (uint64_t)n_views * n) return;
  const uint32_t v = (uint32_t)(q / n), i = (uint32_t)(q % n);
  const size_t o = (size_t)v * stride + i;
  const float4 ra = rec[3 * o], rb = rec[3 * o + 1];
  int x0, y0, x1, y1;
  if (!rect_of(ra, rb, a, x0, y0, x1, y1)) return;
  uint64_t w = offsets[q];
  if (MODE == 0) {
    // tile_emit.wgsl:54-55
    const float dn = fminf(fmaxf(__fdiv_rn(ra.z, a.depth_max), 0.0f), 1.0f);
    const uint32_t d16 = (uint32_t)(dn * 65535.0f);
    uint32_t* keys = reinterpret_cast<uint32_t*>(keys_v);
    const uint32_t vbase = v * a.num_tiles;
    for (int ty = y0; ty <= y1; ++ty)
      for (int tx = x0; tx <= x1; ++tx) {
        if (w >= cap) return;
        keys[w] = ((vbase + (uint32_t)ty * a.tiles_x + (uint32_t)tx) << 16) | d16;
        payloads[w] = i;
        ++w;
      }
  } else {
    const uint64_t db = __float_as_uint(ra.z);
    uint64_t* keys = reinterpret_cast<uint64_t*>(keys_v);
    const uint64_t vbase = (uint64_t)v * a.num_tiles;
    for (int ty = y0; ty <= y1; ++ty)
      for (int tx = x0; tx <= x1; ++tx) {
        if (w >= cap) return;
        keys[w] = ((vbase + (uint64_t)ty * a.tiles_x + (uint64_t)tx) << 32) | db;
        payloads[w] = i;
        ++w;
      }
  }
}

sc_status launch_tile_emit(sc_ctx* ctx, const float4* rec, uint32_t n, uint32_t stride, uint32_t n_views,
                           const sc_tiling* tl, const uint32_t* offsets, int key_mode, void* keys, uint32_t* payloads,
                           uint64_t cap) {
  const uint64_t total = (uint64_t)n * n_views;
  if (total == 0) return SC_OK;
  const unsigned g = (unsigned)sc_div_up(total, 256);
  if (key_mode == SC_KEYS_REF32)
    k_tile_emit<0><<<g, 256, 0, ctx->stream>>>(rec, n, stride, n_views, bin_args(tl), offsets, keys, payloads, cap);
  else
    k_tile_emit<1><<<g, 256, 0, ctx->stream>>>(rec, n, stride, n_views, bin_args(tl), offsets, keys, payloads, cap);
  return sc_check_launch(ctx, "k_tile_emit");
}

// tile_ranges.wgsl:22-41.  tile of a key: REF32 key >> 16, NATIVE key >> 32;
// presorted u32 key (mode 2) (view << tile_bits) | tile, range index
// view * tiles_per_view + tile.  Boundaries are changes of the whole key.
template <int MODE>
__global__ void k_tile_ranges(const void* __restrict__ keys_v, const uint64_t* __restrict__ d_total, uint64_t cap,
                              uint32_t num_tiles, uint32_t tiles_per_view, uint32_t tile_bits, uint32_t key_mask,
                              uint32_t* __restrict__ ranges, unsigned long long* __restrict__ high_popc) {
  const uint64_t K = min(*d_total, cap);
  uint32_t pc = 0;  // set bits above key_mask (mode 2)
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < K; j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t t, tp = ~0ull, tn = ~0ull;
    if (MODE == 0) {
      const uint32_t* k = reinterpret_cast<const uint32_t*>(keys_v);
      t = k[j] >> 16;
      if (j > 0) tp = k[j - 1] >> 16;
      if (j + 1 < K) tn = k[j + 1] >> 16;
    } else if (MODE == 1) {
      const uint64_t* k = reinterpret_cast<const uint64_t*>(keys_v);
      t = k[j] >> 32;
      if (j > 0) tp = k[j - 1] >> 32;
      if (j + 1 < K) tn = k[j + 1] >> 32;
    } else {
      const uint32_t* k = reinterpret_cast<const uint32_t*>(keys_v);
      t = k[j] & key_mask;
      pc += __popc(k[j] & ~key_mask);
      if (j > 0) tp = k[j - 1] & key_mask;
      if (j + 1 < K) tn = k[j + 1] & key_mask;
    }
    uint64_t idx = t;
    if (MODE == 2) {
      const uint32_t tile = (uint32_t)t & ((1u << tile_bits) - 1u);
      if (tile >= tiles_per_view) continue;
      idx = (uint64_t)(t >> tile_bits) * tiles_per_view + tile;
    }
    if (idx >= num_tiles) continue;
    if (tp != t) ranges[2 * idx] = (uint32_t)j;
    if (tn != t) ranges[2 * idx + 1] = (uint32_t)(j + 1);
  }
  if (MODE == 2 && high_popc) {
    __shared__ uint32_t s_pc[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pc += __shfl_xor_sync(0xffffffffu, pc, o);
    if ((threadIdx.x & 31) == 0) s_pc[threadIdx.x >> 5] = pc;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long tot = 0;
      for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) tot += s_pc[w];
      if (tot) atomicAdd(high_popc, tot);
    }
  }
}

// The same for presorted u32 keys (mode 2) read four at a time: a thread
// loads keys [4q, 4q + 4) with one 16-byte access and takes the key before and
// after its four from the neighbouring lanes (lanes 0 and 31 load theirs), so
// every key is read once instead of three times.  The warp walks the quads
// together (the loop condition is the warp's first quad), which the shuffles
// need.
__global__ void __launch_bounds__(256) k_tile_ranges_u32x4(const uint32_t* __restrict__ k,
                                                           const uint64_t* __restrict__ d_total, uint64_t cap,
                                                           uint32_t num_tiles, uint32_t tiles_per_view,
                                                           uint32_t tile_bits, uint32_t key_mask,
                                                           uint32_t* __restrict__ ranges,
                                                           unsigned long long* __restrict__ high_popc) {
  const uint64_t K = min(*d_total, cap);
  const uint64_t nq = (K + 3) >> 2;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  constexpr uint64_t NONE = ~0ull;  // no neighbour: differs from every masked key
  uint32_t pc = 0;
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q - lane < nq; q += step) {
    const uint64_t j0 = q << 2;
    uint32_t x[4] = {0u, 0u, 0u, 0u};
    if (j0 + 3 < K) {
      const uint4 v = *reinterpret_cast<const uint4*>(k + j0);
      x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (j0 + i < K) x[i] = k[j0 + i];
    }
    // the keys either side of this thread's four
    uint32_t before = __shfl_up_sync(0xffffffffu, x[3], 1);
    uint32_t after = __shfl_down_sync(0xffffffffu, x[0], 1);
    if (lane == 0 && j0 > 0 && j0 - 1 < K) before = k[j0 - 1];
    if (lane == 31 && j0 + 4 < K) after = k[j0 + 4];
    uint64_t m[6];
    m[0] = j0 > 0 ? (uint64_t)(before & key_mask) : NONE;
#pragma unroll
    for (int i = 0; i < 4; ++i) m[i + 1] = j0 + i < K ? (uint64_t)(x[i] & key_mask) : NONE;
    m[5] = j0 + 4 < K ? (uint64_t)(after & key_mask) : NONE;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint64_t j = j0 + i;
      if (j >= K) break;
      pc += __popc(x[i] & ~key_mask);
      const uint64_t t = m[i + 1];
      const uint32_t tile = (uint32_t)t & ((1u << tile_bits) - 1u);
      if (tile >= tiles_per_view) continue;
      const uint64_t idx = (t >> tile_bits) * tiles_per_view + tile;
      if (idx >= num_tiles) continue;
      if (m[i] != t) ranges[2 * idx] = (uint32_t)j;
      if (m[i + 2] != t) ranges[2 * idx + 1] = (uint32_t)(j + 1);
    }
  }
  if (high_popc) {
    __shared__ uint32_t s_pc[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pc += __shfl_xor_sync(0xffffffffu, pc, o);
    if (lane == 0) s_pc[threadIdx.x >> 5] = pc;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long tot = 0;
      for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) tot += s_pc[w];
      if (tot) atomicAdd(high_popc, tot);
    }
  }
}

sc_status launch_tile_ranges(sc_ctx* ctx, const void* keys, int key_mode, const uint64_t* d_total, uint64_t cap,
                             uint32_t num_tiles, uint32_t* ranges, uint32_t tiles_per_view, uint32_t tile_bits,
                             uint32_t key_bits, uint64_t* high_popc) {
  SC_CUDA_TRY(ctx, cudaMemsetAsync(ranges, 0, (size_t)num_tiles * 8, ctx->stream), "memset ranges");
  if (cap == 0) return SC_OK;
  const unsigned g = (unsigned)std::min<uint64_t>(sc_div_up(cap, 256), (uint64_t)ctx->sm_count * 16);
  if (key_mode == 0)
    k_tile_ranges<0><<<g, 256, 0, ctx->stream>>>(keys, d_total, cap, num_tiles, 0, 0, ~0u, ranges, nullptr);
  else if (key_mode == 1)
    k_tile_ranges<1><<<g, 256, 0, ctx->stream>>>(keys, d_total, cap, num_tiles, 0, 0, ~0u, ranges, nullptr);
  else if (reinterpret_cast<uintptr_t>(keys) % 16 != 0)  // the 16-byte loads need an aligned array
    k_tile_ranges<2><<<g, 256, 0, ctx->stream>>>(keys, d_total, cap, num_tiles, tiles_per_view, tile_bits,
                                                 key_bits >= 32 ? ~0u : (1u << key_bits) - 1u, ranges,
                                                 reinterpret_cast<unsigned long long*>(high_popc));
  else
    k_tile_ranges_u32x4<<<(unsigned)std::min<uint64_t>(sc_div_up(sc_div_up(cap, 4), 256), (uint64_t)ctx->sm_count * 8),
                          256, 0, ctx->stream>>>(static_cast<const uint32_t*>(keys), d_total, cap, num_tiles,
                                                 tiles_per_view, tile_bits,
                                                 key_bits >= 32 ? ~0u : (1u << key_bits) - 1u, ranges,
                                                 reinterpret_cast<unsigned long long*>(high_popc));
  return sc_check_launch(ctx, "k_tile_ranges");
}

// ---------------------------------------------------------------- depth-presorted path
// sorted_ids[v*stride + r] is the splat of depth rank r in view v.

// One thread generates the pairs of one depth-ranked splat, row by row.  With
// culling, each row keeps the span of tiles that cull_row_span returns — the
// function the projection counted with — clamped to the 3-sigma rectangle.
// Exactly `count` pairs are written per splat; should a row span ever differ
// from the count, surplus tiles are dropped and missing slots get an
// out-of-range key that sorts last and that the range kernel ignores.
//
// A warp's 32 consecutive ranked splats own one contiguous output range
// [offsets[j0], offsets[j0 + 32]).  The warp walks it in chunks of
// EMIT_WCHUNK pairs: every lane writes the pairs of its splat that fall in the
// chunk into the warp's shared-memory buffer (resuming its row walk where the
// previous chunk stopped, one run of a row at a time), then the warp stores
// the chunk with coalesced 4-byte stores.  Warps never wait for each other.
constexpr int EMIT_WARPS = 8;
constexpr int EMIT_WCHUNK = 512;

__global__ void __launch_bounds__(EMIT_WARPS * 32) k_presorted_emit(
    const float4* __restrict__ rec, uint32_t stride, uint32_t n_views, const uint32_t* __restrict__ sorted_ids,
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ counts_by_id, BinArgs a,
    uint32_t* __restrict__ keys, uint32_t* __restrict__ payloads, uint64_t cap, uint32_t* __restrict__ err, int cull) {
  __shared__ uint32_t sk[EMIT_WARPS][EMIT_WCHUNK], sp[EMIT_WARPS][EMIT_WCHUNK];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t total = (uint64_t)n_views * stride;
  const uint64_t jw = (uint64_t)blockIdx.x * blockDim.x + (uint64_t)warp * 32;
  if (jw >= total) return;
  const uint64_t j = jw + lane;
  const uint64_t jend = jw + 32 < total ? jw + 32 : total;
  const uint64_t wlo = offsets[jw], whi = offsets[jend];  // offsets holds total + 1 entries
  if (lane == 0 && whi > cap) atomicOr(err, SC_DEVERR_CAPACITY);
  // this lane's splat and its row walk
  uint32_t cnt = 0, id = 0, vbase = 0;
  uint64_t off = 0;
  int x0 = 0, y0 = 0, x1 = -1, y1 = -1;
  CullShape cs{};
  bool test = false;
  if (j < total) {
    const uint32_t v = (uint32_t)(j / stride);
    id = sorted_ids[j];
    const size_t o = (size_t)v * stride + id;
    cnt = counts_by_id[o];
    if (cnt) {
      off = offsets[j];
      const float4 ra = rec[3 * o], rb = rec[3 * o + 1], rc = rec[3 * o + 2];
      if (!rect_of(ra, rb, a, x0, y0, x1, y1)) { x0 = 0; y0 = 0; x1 = -1; y1 = -1; }
      cs = cull_shape(ra.x, ra.y, rb.x, rb.y, rb.z, rc.w);
      test = cull && !cs.keep;
      vbase = v << a.tile_bits;
    }
  }
  uint32_t* wk = sk[warp];
  uint32_t* wp = sp[warp];
  int ty = y0 - 1, tx = 0, hi = -1;  // tx > hi: the next pair starts a new row
  bool rows_done = cnt == 0;
  uint32_t w = 0, rowbase = 0;
  for (uint64_t cb = wlo; cb < whi; cb += EMIT_WCHUNK) {
    const uint64_t ce = cb + EMIT_WCHUNK < whi ? cb + EMIT_WCHUNK : whi;
    const int64_t room = (int64_t)ce - (int64_t)off;  // this lane's pairs with index < ce
    const uint32_t wend = room <= (int64_t)w ? w : (uint32_t)(room < (int64_t)cnt ? room : (int64_t)cnt);
    int slot = (int)((int64_t)off - (int64_t)cb) + (int)w;
    while (w < wend) {
      if (tx > hi) {  // next row whose span is not empty
        bool found = false;
        while (!rows_done) {
          ++ty;
          if (ty > y1) { rows_done = true; break; }
          int lo = x0, h = x1;
          if (test) {
            if (!cs.any || !cull_row_span(cs, ty, a.tw, a.th, lo, h)) continue;
            lo = max(lo, x0);
            h = min(h, x1);
            if (h < lo) continue;
          }
          tx = lo;
          hi = h;
          found = true;
          break;
        }
        if (!found) {  // count and emission disagreed: pad
          for (; w < wend; ++w, ++slot) { wk[slot] = 0xFFFFFFFFu; wp[slot] = 0; }
          break;
        }
        rowbase = vbase + (uint32_t)ty * a.tiles_x;
      }
      const uint32_t run = min((uint32_t)(hi - tx + 1), wend - w);
      for (uint32_t q = 0; q < run; ++q) {
        wk[slot + q] = rowbase + (uint32_t)tx + q;
        wp[slot + q] = id;
      }
      tx += (int)run;
      w += run;
      slot += (int)run;
    }
    __syncwarp();
    const uint32_t n = (uint32_t)(ce - cb);
    for (uint32_t t = lane; t < n; t += 32) {
      const uint64_t g = cb + t;
      if (g < cap) {
        keys[g] = wk[t];
        payloads[g] = wp[t];
      }
    }
    __syncwarp();
  }
}

sc_status launch_presorted_emit(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                                const uint32_t* sorted_ids, const uint32_t* offsets, const uint32_t* counts_by_id,
                                const sc_tiling* tl, uint32_t* keys, uint32_t* payloads, uint64_t cap,
                                uint32_t* d_error, int cull) {
  const uint64_t total = (uint64_t)n_views * stride;
  if (total == 0) return SC_OK;
  k_presorted_emit<<<(unsigned)sc_div_up(total, EMIT_WARPS * 32), EMIT_WARPS * 32, 0, ctx->stream>>>(
      rec, stride, n_views, sorted_ids, offsets, counts_by_id, bin_args(tl), keys, payloads, cap, d_error, cull);
  return sc_check_launch(ctx, "k_presorted_emit");
}

// ---------------------------------------------------------------- two-level binning
// Super tiles of SC_SUPER x SC_SUPER tiles.  Items (super tile, splat) are
// emitted in depth order and grouped per super tile by a short stable sort;
// then one CTA per super tile decides for each of its items which of the 16
// tiles it covers (the same splat_row_span test as the pair counting) and
// appends the splat to those tiles' lists in item order, so every tile's list
// is the depth-ordered list of the pair pipeline without sorting the pairs.
uint32_t super_tiles_per_view(const sc_tiling* tl) {
  const BinArgs a = bin_args(tl);
  return ((a.tiles_x + SC_SUPER - 1) / SC_SUPER) * ((a.tiles_y + SC_SUPER - 1) / SC_SUPER);
}

static uint32_t super_bits_for(uint32_t n) {  // 2^b > n
  uint32_t b = 0;
  while ((1ull << b) <= n) ++b;
  return b;
}

constexpr int SUPER_MASK_SHIFT = 16;  // item key: member mask << 16 | view << super_bits | super tile

// One CTA per 256 consecutive depth-ranked (view, splat) entries, whose items
// form one contiguous output range.  A lane walks one splat's super rows, so a
// warp takes as long as its largest splat: the CTA first sorts its splats into
// classes by item count (a shared-memory counting sort, order within a class
// arbitrary) and hands them to the lanes in class order, so that a warp's
// lanes carry splats of about the same size.  The items are staged in shared
// memory in chunks of SE_CHUNK positions and stored coalesced; a lane
// regenerates its items for every chunk that holds some of them.  The output
// does not depend on which lane takes which splat (each item's position is
// its splat's offset plus its rank among the splat's items).
constexpr int SE_THREADS = 256;
constexpr int SE_CHUNK = 2048;
constexpr int SE_CLASSES = 32;  // item counts 0..30, and 31 or more

__global__ void __launch_bounds__(SE_THREADS) k_super_emit(
    const float4* __restrict__ rec, uint32_t stride, uint32_t n_views, const uint32_t* __restrict__ sorted_ids,
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ counts_by_id, BinArgs a, uint32_t super_x,
    uint32_t super_bits, uint32_t* __restrict__ keys, uint32_t* __restrict__ payloads, uint64_t cap,
    uint32_t* __restrict__ err, int cull) {
  __shared__ uint32_t sk[SE_CHUNK], sp[SE_CHUNK];
  __shared__ uint32_t s_class[SE_CLASSES];
  __shared__ uint16_t s_perm[SE_THREADS];
  const uint64_t total = (uint64_t)n_views * stride;
  const uint64_t j0 = (uint64_t)blockIdx.x * SE_THREADS;
  const uint64_t jend = j0 + SE_THREADS < total ? j0 + SE_THREADS : total;
  // item offsets are 32-bit (the scan of the counts), so is the chunk walk
  const uint32_t clo = offsets[j0], chi = offsets[jend];
  if (threadIdx.x == 0 && chi > cap) atomicOr(err, SC_DEVERR_CAPACITY);
  // this thread's entry's item count decides its class
  uint32_t own = 0;
  {
    const uint64_t jt = j0 + threadIdx.x;
    if (jt < total) {
      const uint32_t v = (uint32_t)(jt / stride);
      own = counts_by_id[(size_t)v * stride + sorted_ids[jt]];
    }
  }
  const uint32_t cls = own < SE_CLASSES - 1 ? own : SE_CLASSES - 1;
  if (threadIdx.x < SE_CLASSES) s_class[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t rank = atomicAdd(&s_class[cls], 1u);
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive scan of the class sizes
    const uint32_t c = s_class[threadIdx.x];
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if ((int)threadIdx.x >= o) x += y;
    }
    s_class[threadIdx.x] = x - c;
  }
  __syncthreads();
  s_perm[s_class[cls] + rank] = (uint16_t)threadIdx.x;
  __syncthreads();
  // the splat this lane walks
  const uint64_t j = j0 + s_perm[threadIdx.x];
  uint32_t cnt = 0, id = 0, vkey = 0, off = 0;
  int x0 = 0, y0 = 0, x1 = -1, y1 = -1;
  CullShape cs{};
  bool test = false;
  if (j < total) {
    const uint32_t v = (uint32_t)(j / stride);
    id = sorted_ids[j];
    const size_t o = (size_t)v * stride + id;
    cnt = counts_by_id[o];
    if (cnt) {
      off = offsets[j];
      const float4 ra = rec[3 * o], rb = rec[3 * o + 1], rc = rec[3 * o + 2];
      if (!rect_of(ra, rb, a, x0, y0, x1, y1)) { x0 = 0; y0 = 0; x1 = -1; y1 = -1; }
      cs = cull_shape(ra.x, ra.y, rb.x, rb.y, rb.z, rc.w);
      test = (cull & 1) && !cs.keep;
      vkey = v << super_bits;
    }
  }
  for (uint32_t cb = clo; cb < chi; cb += SE_CHUNK) {
    const uint32_t ce = min(cb + (uint32_t)SE_CHUNK, chi);
    if (cnt && off < ce && off + cnt > cb) {
      uint32_t w = 0;
      for_each_super_span(cs, test, x0, y0, x1, y1, a.tw, a.th,
                          [&](int sy, int sx0, int sx1, const int* rlo, const int* rhi) {
        for (int sx = sx0; sx <= sx1; ++sx, ++w) {
          const uint32_t g = off + w;
          if (w < cnt && g >= cb && g < ce) {
            sk[g - cb] = (super_mask_of(sx, rlo, rhi) << SUPER_MASK_SHIFT) | vkey |
                         ((uint32_t)sy * super_x + (uint32_t)sx);
            sp[g - cb] = id;
          }
        }
      });
      for (; w < cnt; ++w) {  // count and emission disagreed: pad with a key that sorts last
        const uint32_t g = off + w;
        if (g >= cb && g < ce) { sk[g - cb] = 0xFFFFFFFFu; sp[g - cb] = 0; }
      }
    }
    __syncthreads();
    const uint32_t n = ce - cb;
    for (uint32_t t = threadIdx.x; t < n; t += SE_THREADS) {
      const uint32_t g = cb + t;
      if (g < cap) {
        keys[g] = sk[t];
        payloads[g] = sp[t];
      }
    }
    __syncthreads();
  }
}

sc_status launch_super_emit(sc_ctx* ctx, const float4* rec, uint32_t stride, uint32_t n_views,
                            const uint32_t* sorted_ids, const uint32_t* offsets, const uint32_t* counts_by_id,
                            const sc_tiling* tl, uint32_t* keys, uint32_t* payloads, uint64_t cap, uint32_t* d_error,
                            int cull) {
  const uint64_t total = (uint64_t)n_views * stride;
  if (total == 0) return SC_OK;
  const BinArgs a = bin_args(tl);
  const uint32_t sx = (a.tiles_x + SC_SUPER - 1) / SC_SUPER;
  const uint32_t bits = super_bits_for(super_tiles_per_view(tl));
  k_super_emit<<<(unsigned)sc_div_up(total, SE_THREADS), SE_THREADS, 0, ctx->stream>>>(
      rec, stride, n_views, sorted_ids, offsets, counts_by_id, a, sx, bits, keys, payloads, cap, d_error, cull);
  return sc_check_launch(ctx, "k_super_emit");
}

}  // namespace sck
