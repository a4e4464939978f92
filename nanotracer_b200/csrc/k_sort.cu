// k_sort.cu — single-pass exclusive scan and onesweep LSD radix sort, both
// with decoupled look-back (Merrill & Garland 2016; Adinets & Merrill 2022).
//
// Replaces the reference's 3-level Hillis-Steele scan (prefix_scan.rs:127-186,
// n <= 2^24) and its 32 one-bit split passes (radix_sort.rs:144-303, ~160
// dispatches per sort).  Here one sort is one histogram kernel plus one kernel
// per 8- or 9-bit digit.  Both are stable and deterministic: tiles take their
// position from an atomic ticket, rank their items warp-by-warp in input
// order (ballot-based peer masks), and obtain the running digit offsets from
// their predecessors' published aggregates.
//
// Every look-back wait is bounded: after SC_SPIN_LIMIT polls the block sets
// SC_DEVERR_TIMEOUT in the context's error word and proceeds with what it has
// (the output is then garbage, the host reports SC_ERR_TIMEOUT) instead of
// hanging the GPU.
#include "sc_internal.cuh"

namespace sck {

// ---------------------------------------------------------------- memory-order helpers
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------- exclusive scan
#define SCAN_THREADS 256
#define SCAN_IPT 16
#define SCAN_TILE (SCAN_THREADS * SCAN_IPT)
#define SCAN_FLAG_AGG (1ull << 62)
#define SCAN_FLAG_PRE (2ull << 62)
#define SCAN_VAL_MASK ((1ull << 62) - 1)

__device__ __forceinline__ unsigned long long warp_incl_scan_u64(unsigned long long x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Gather of the scanned values (when src is given): element i < gn is
// src[(i / seg) seg + idx[i]] — the value of the idx[i]-th element of its
// segment (a view's counts by splat, read in depth order) — and 0 beyond gn.
static_assert(SCAN_IPT == 16, "the scan's vector accesses move 16 elements per thread");
// 16 consecutive u32 through four 16-byte accesses (p 16-byte aligned)
__device__ __forceinline__ void load_u32x16(const uint32_t* p, uint32_t v[16]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint4 t = reinterpret_cast<const uint4*>(p)[q];
    v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
  }
}
__device__ __forceinline__ void store_u32x16(uint32_t* p, const uint32_t v[16]) {
#pragma unroll
  for (int q = 0; q < 4; ++q)
    reinterpret_cast<uint4*>(p)[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

struct ScanGather {
  const uint32_t* src;
  const uint32_t* idx;
  uint32_t seg;
  uint64_t n;
};

__global__ void __launch_bounds__(SCAN_THREADS) k_scan(uint32_t* __restrict__ data, uint64_t n,
                                                       unsigned long long* __restrict__ status,
                                                       unsigned* __restrict__ ticket, uint64_t* __restrict__ total,
                                                       uint32_t* __restrict__ err, ScanGather gather) {
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_warp[SCAN_THREADS / 32];
  __shared__ unsigned long long s_excl;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const unsigned tile = s_tile;
  const uint64_t base = (uint64_t)tile * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_IPT;
  uint32_t x[SCAN_IPT];
  unsigned long long tsum = 0;
  if (gather.src) {
    // a thread's SCAN_IPT indices with 16-byte loads when they are all in range
    // and the array is 16-byte aligned (base is a multiple of SCAN_IPT)
    uint32_t ix[SCAN_IPT];
    if (base + SCAN_IPT <= gather.n && (reinterpret_cast<uintptr_t>(gather.idx) & 15) == 0) {
      load_u32x16(gather.idx + base, ix);
    } else {
#pragma unroll
      for (int k = 0; k < SCAN_IPT; ++k) ix[k] = base + k < gather.n ? gather.idx[base + k] : 0u;
    }
    uint32_t g = base < gather.n ? (uint32_t)(base / gather.seg) : 0u;  // the segment of element base
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
      const uint64_t i = base + k;
      if (i >= (uint64_t)(g + 1) * gather.seg) ++g;  // a thread's elements cross at most one segment end
      x[k] = i < gather.n ? gather.src[(size_t)g * gather.seg + ix[k]] : 0u;
      tsum += x[k];
    }
  } else {
    if (base + SCAN_IPT <= n && (reinterpret_cast<uintptr_t>(data) & 15) == 0) {
      load_u32x16(data + base, x);
    } else {
#pragma unroll
      for (int k = 0; k < SCAN_IPT; ++k) x[k] = (base + k < n) ? data[base + k] : 0u;
    }
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) tsum += x[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long incl = warp_incl_scan_u64(tsum);
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned long long w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0ull;
    w = warp_incl_scan_u64(w);
    if (lane < SCAN_THREADS / 32) s_warp[lane] = w;  // inclusive per warp
    // look-back by warp 0
    const unsigned long long agg = __shfl_sync(0xffffffffu, w, SCAN_THREADS / 32 - 1);
    if (lane == 0) st_release_u64(&status[tile], (tile == 0 ? SCAN_FLAG_PRE : SCAN_FLAG_AGG) | agg);
    unsigned long long excl = 0;
    if (tile > 0) {
      // warp-wide look-back: lane l inspects predecessor pred - l; indices below
      // zero read as an inclusive prefix of 0, so the walk always terminates.
      long long pred = (long long)tile - 1;
      unsigned spins = 0;
      bool gave_up = false;
      for (;;) {
        const long long idx = pred - lane;
        unsigned long long st = 0;
        for (;;) {
          st = idx >= 0 ? ld_acquire_u64(&status[idx]) : SCAN_FLAG_PRE;
          if (__all_sync(0xffffffffu, (st >> 62) != 0ull)) break;
          if (++spins > SC_SPIN_LIMIT) { gave_up = true; break; }
          __nanosleep(32);
        }
        if (gave_up) break;
        const unsigned pre = __ballot_sync(0xffffffffu, (st >> 62) == 2ull);
        const int first = pre ? __ffs(pre) - 1 : 32;  // nearest predecessor holding an inclusive prefix
        unsigned long long val = (lane <= first) ? (st & SCAN_VAL_MASK) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        excl += val;
        if (pre) break;
        pred -= 32;
      }
      if (gave_up && lane == 0) atomicOr(err, SC_DEVERR_TIMEOUT);
      if (lane == 0) st_release_u64(&status[tile], SCAN_FLAG_PRE | ((excl + agg) & SCAN_VAL_MASK));
    }
    if (lane == 0) s_excl = excl;
  }
  __syncthreads();
  unsigned long long run = s_excl + (warp > 0 ? s_warp[warp - 1] : 0ull) + (incl - tsum);
  if (base + SCAN_IPT <= n && (reinterpret_cast<uintptr_t>(data) & 15) == 0) {
    uint32_t o[SCAN_IPT];
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
      o[k] = (uint32_t)run;
      run += x[k];
    }
    store_u32x16(data + base, o);
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
      if (base + k < n) data[base + k] = (uint32_t)run;
      run += x[k];
    }
  }
  // the thread holding the last element publishes the total
  if (total && n > 0 && base <= n - 1 && n - 1 < base + SCAN_IPT) *total = run;
}

size_t scan_scratch_bytes(uint64_t n) {
  const uint64_t tiles = sc_div_up(n, SCAN_TILE);
  return 256 + tiles * 8;
}

static sc_status scan_u32_impl(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* d_total, void* scratch,
                               size_t bytes, ScanGather gather) {
  if (n == 0) {
    if (d_total) SC_CUDA_TRY(ctx, cudaMemsetAsync(d_total, 0, 8, ctx->stream), "memset total");
    return SC_OK;
  }
  const uint64_t tiles = sc_div_up(n, SCAN_TILE);
  if (bytes < scan_scratch_bytes(n)) return sc_fail(ctx, SC_ERR_INVALID_ARG, "scan scratch too small");
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
  unsigned long long* status = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(scratch) + 256);
  SC_CUDA_TRY(ctx, cudaMemsetAsync(scratch, 0, scan_scratch_bytes(n), ctx->stream), "memset scan status");
  k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, ctx->stream>>>(data, n, status, ticket, d_total, ctx->d_error, gather);
  return sc_check_launch(ctx, "k_scan");
}

sc_status scan_u32(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* d_total, void* scratch, size_t bytes) {
  return scan_u32_impl(ctx, data, n, d_total, scratch, bytes, ScanGather{nullptr, nullptr, 1, 0});
}

sc_status scan_u32_gather(sc_ctx* ctx, uint32_t* out, uint64_t n, const uint32_t* src, const uint32_t* idx,
                          uint32_t seg, uint64_t gn, uint64_t* d_total, void* scratch, size_t bytes) {
  if (seg == 0 || seg % SCAN_IPT) return sc_fail(ctx, SC_ERR_INVALID_ARG, "gather segment must be a multiple of 16");
  return scan_u32_impl(ctx, out, n, d_total, scratch, bytes, ScanGather{src, idx, seg, gn});
}

// ---------------------------------------------------------------- allocation-free scan
// Scratch of sc_exclusive_scan_u32_noalloc: a 256-byte ticket area followed by
// one 8-byte look-back status word per 4096-element tile, for at most
// SC_NOALLOC_SCAN_MAX_N elements (128 KiB + 256 B).  It is a file-scope device
// array, so every GPU that loads this library holds it until the process
// exits, and every call shares it.
static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[256 + (SC_NOALLOC_SCAN_MAX_N / SCAN_TILE) * 8];

static_assert(SC_NOALLOC_SCAN_MAX_N % SCAN_TILE == 0, "maximum must be a whole number of scan tiles");

}  // namespace sck

#include <mutex>

namespace {
// Device address of the scratch array, per device.  Host code cannot use the
// array's name as a device pointer: it is a host-side stand-in.
constexpr int kMaxDevices = 64;
void* g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mu;
}  // namespace

extern "C" sc_status sc_exclusive_scan_u32_noalloc(sc_ctx* ctx, uint32_t* data, uint64_t n, uint64_t* total) {
  if (!ctx || (n && !data)) return SC_ERR_INVALID_ARG;
  if (n > SC_NOALLOC_SCAN_MAX_N)
    return sc_fail(ctx, SC_ERR_INVALID_ARG,
                   "sc_exclusive_scan_u32_noalloc: n exceeds SC_NOALLOC_SCAN_MAX_N (67108864 elements)");
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return SC_ERR_INVALID_ARG;
  void* scratch = nullptr;
  {
    // one-time set-up per device, with that device current: look up the
    // array's device address (a query, not an allocation)
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    scratch = g_noalloc_ptr[ctx->device];
    if (!scratch) {
      int cur = -1;
      SC_CUDA_TRY(ctx, cudaGetDevice(&cur), "get device");
      if (cur != ctx->device) SC_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "set device");
      const cudaError_t e = cudaGetSymbolAddress(&scratch, sck::g_noalloc_scan_scratch);
      if (cur != ctx->device) cudaSetDevice(cur);
      if (e != cudaSuccess || !scratch) return sc_cuda_fail(ctx, e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                                           "scratch symbol address");
      g_noalloc_ptr[ctx->device] = scratch;
    }
  }
  if (n == 0) {
    if (total) SC_CUDA_TRY(ctx, cudaMemsetAsync(total, 0, 8, ctx->stream), "memset total");
    return SC_OK;
  }
  const uint64_t tiles = sc_div_up(n, SCAN_TILE);
  // the ticket and the look-back flags of this call's tiles must start at zero
  // (the array keeps the previous call's contents)
  SC_CUDA_TRY(ctx, cudaMemsetAsync(scratch, 0, 256 + tiles * 8, ctx->stream), "clear scan scratch");
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
  unsigned long long* status = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(scratch) + 256);
  sck::k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, ctx->stream>>>(data, n, status, ticket, total, ctx->d_error,
                                                                 sck::ScanGather{nullptr, nullptr, 1, 0});
  return sc_check_launch(ctx, "k_scan");
}

namespace sck {

// ---------------------------------------------------------------- onesweep radix sort
#define RS_THREADS 256
#define RS_WARPS (RS_THREADS / 32)
#define RS_FLAG_AGG (1u << 30)
#define RS_FLAG_PRE (2u << 30)
#define RS_VAL_MASK ((1u << 30) - 1)
#define RS_HIST_BLOCKS_PER_SM 4
#define RS_HIST_UNROLL 8  // keys each histogram thread loads before counting them
#define RS_MAX_PASSES 8         // 64-bit keys at 8 or 9 bits per pass
#define RS_HIST_BYTES (RS_MAX_PASSES * 512 * 4)

template <typename K> struct RsCfg;
template <> struct RsCfg<uint32_t> { static constexpr int IPT = 16; };
template <> struct RsCfg<uint64_t> { static constexpr int IPT = 12; };

// A sort uses RB = 8 or 9 bits per pass (RADIX digits), whichever needs
// fewer passes for its key_bits; each of the 256 threads owns DPT = RADIX /
// 256 consecutive digits in a pass's per-digit work.
template <int RB> struct Rdx {
  static constexpr int RADIX = 1 << RB;
  static constexpr int DPT = RADIX / RS_THREADS;
};

// digit mask of pass p when only the low key_bits bits are sorted
__host__ __device__ __forceinline__ uint32_t rs_digit_mask(uint32_t key_bits, int p, int rb) {
  const int rem = (int)key_bits - rb * p;
  return rem >= rb ? (1u << rb) - 1u : (rem <= 0 ? 0u : (1u << rem) - 1u);
}

// Global digit histograms of all passes in one read of the keys.
template <typename K, int RB>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const K* __restrict__ keys, uint64_t n_cap,
                                                        const uint64_t* __restrict__ d_n, int passes,
                                                        uint32_t key_bits, uint32_t* __restrict__ hist /* passes x RADIX */) {
  constexpr int RADIX = Rdx<RB>::RADIX;
  __shared__ uint32_t sh[RS_MAX_PASSES * RADIX];
  for (int t = threadIdx.x; t < passes * RADIX; t += RS_THREADS) sh[t] = 0;
  __syncthreads();
  const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
  // RS_HIST_UNROLL independent coalesced loads in flight per thread before
  // their shared-memory counts: one load per iteration left the kernel bound
  // on memory latency, not bandwidth
  const uint64_t step = (uint64_t)gridDim.x * RS_THREADS;
  for (uint64_t i0 = (uint64_t)blockIdx.x * RS_THREADS + threadIdx.x; i0 < n; i0 += step * RS_HIST_UNROLL) {
    K k[RS_HIST_UNROLL];
#pragma unroll
    for (int u = 0; u < RS_HIST_UNROLL; ++u) {
      const uint64_t i = i0 + u * step;
      k[u] = i < n ? keys[i] : K(0);
    }
#pragma unroll
    for (int u = 0; u < RS_HIST_UNROLL; ++u) {
      if (i0 + u * step < n) {
        for (int p = 0; p < passes; ++p)
          atomicAdd(&sh[p * RADIX + ((uint32_t)(k[u] >> (RB * p)) & rs_digit_mask(key_bits, p, RB))], 1u);
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < passes * RADIX; t += RS_THREADS) {
    const uint32_t c = sh[t];
    if (c) atomicAdd(&hist[t], c);
  }
}

// exclusive scan of each pass's RADIX bins (one block of RADIX threads per pass)
template <int RB>
__global__ void __launch_bounds__(1 << RB) k_rs_hist_scan(uint32_t* __restrict__ hist) {
  constexpr int RADIX = Rdx<RB>::RADIX;
  __shared__ uint32_t s[RADIX];
  uint32_t* h = hist + blockIdx.x * RADIX;
  const uint32_t v = h[threadIdx.x];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < RADIX; o <<= 1) {
    uint32_t y = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
    __syncthreads();
    s[threadIdx.x] += y;
    __syncthreads();
  }
  h[threadIdx.x] = s[threadIdx.x] - v;
}

template <typename K, int RB>
struct RsSmem {
  static constexpr int IPT = RsCfg<K>::IPT;
  static constexpr int TILE = RS_THREADS * IPT;
  static constexpr int RADIX = Rdx<RB>::RADIX;
  K keys[TILE];                       // keys in digit order (scatter staging)
  uint32_t vals[TILE];                // payloads in input (warp-striped) order, prefetched with cp.async
  uint16_t src[TILE];                 // digit-order slot -> input slot of its payload
  uint32_t warp_hist[RS_WARPS][RADIX];
  uint32_t tile_excl[RADIX];
  int out_base[RADIX];                // global position of digit d's first slot, minus its tile offset
  uint32_t tile_id;
};

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The work of one tile once its index is known.  FULL: the tile lies wholly
// below n, so no per-key bounds test is needed.  NARROW: this pass's digit has
// dbits < RB bits (the last pass of a short key), so fewer ballots rank it.
template <typename K, bool FULL, bool NARROW, int RB>
__device__ __forceinline__ void rs_pass_tile(RsSmem<K, RB>& sm, const K* __restrict__ kin,
                                             const uint32_t* __restrict__ vin, K* __restrict__ kout,
                                             uint32_t* __restrict__ vout, uint64_t n, int shift,
                                             const uint32_t* __restrict__ digit_base, unsigned* __restrict__ lookback,
                                             uint32_t* __restrict__ err, uint32_t tile, uint64_t tbase, int dbits) {
  constexpr int IPT = RsCfg<K>::IPT;
  constexpr int TILE = RS_THREADS * IPT;
  constexpr int RADIX = Rdx<RB>::RADIX, DPT = Rdx<RB>::DPT;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (!NARROW) dbits = RB;
  const uint32_t dmask = (1u << dbits) - 1u;
  // warp-striped layout: item k of lane l in warp w is input slot w*32*IPT + k*32 + l
  const uint32_t wslot = (uint32_t)warp * 32 * IPT;
  const uint64_t wbase = tbase + wslot;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const uint64_t i = wbase + (uint64_t)k * 32 + lane;
    if (FULL || i < n) cp_async4(&sm.vals[wslot + k * 32 + lane], vin + i);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  K key[IPT];
  uint32_t rank[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const uint64_t i = wbase + (uint64_t)k * 32 + lane;
    key[k] = (FULL || i < n) ? kin[i] : (K)0;
  }
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const bool valid = FULL || wbase + (uint64_t)k * 32 + lane < n;
    const uint32_t d = (uint32_t)(key[k] >> shift) & dmask;
    unsigned peers = FULL ? 0xffffffffu : __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      if (!NARROW || b < dbits) {
        const bool bit = (d >> b) & 1u;
        const unsigned m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
      }
    }
    const int leader = valid ? 31 - __clz(peers) : lane;
    uint32_t old = 0;
    if (valid && lane == leader) {
      old = sm.warp_hist[warp][d];
      sm.warp_hist[warp][d] = old + __popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader);
    rank[k] = old + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  // per digit (DPT consecutive digits per thread): exclusive prefix over warps, tile count
  uint32_t cnt[DPT];
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    const int d = threadIdx.x * DPT + j;
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
      const uint32_t x = sm.warp_hist[w][d];
      sm.warp_hist[w][d] = c;
      c += x;
    }
    cnt[j] = c;
  }
  // publish this tile's counts, then look back for the running prefixes
  unsigned* lb = lookback + (size_t)tile * RADIX;
#pragma unroll
  for (int j = 0; j < DPT; ++j)
    st_relaxed_u32(&lb[threadIdx.x * DPT + j], (tile == 0 ? RS_FLAG_PRE : RS_FLAG_AGG) | cnt[j]);
  // with several digits per thread the digits walk back in lockstep, so their
  // status loads are in flight together instead of one chain after another
  uint32_t excl[DPT];
#pragma unroll
  for (int j = 0; j < DPT; ++j) excl[j] = 0;
  if (DPT == 1 && tile > 0) {
    const int d = threadIdx.x;
    long long pred = (long long)tile - 1;
    unsigned spins = 0;
    while (pred >= 0) {
      const unsigned st = ld_relaxed_u32(&lookback[(size_t)pred * RADIX + d]);
      const unsigned flag = st & ~RS_VAL_MASK;
      if (flag == 0u) {
        if (++spins > SC_SPIN_LIMIT) { atomicOr(err, SC_DEVERR_TIMEOUT); break; }
        __nanosleep(20);
        continue;
      }
      excl[0] += st & RS_VAL_MASK;
      if (flag == RS_FLAG_PRE) break;
      --pred;
    }
    st_relaxed_u32(&lb[d], RS_FLAG_PRE | ((excl[0] + cnt[0]) & RS_VAL_MASK));
  } else if (DPT > 1 && tile > 0) {
    long long pred[DPT];
    bool open[DPT];
#pragma unroll
    for (int j = 0; j < DPT; ++j) { pred[j] = (long long)tile - 1; open[j] = true; }
    unsigned spins = 0;
    for (;;) {
      unsigned st[DPT];
#pragma unroll
      for (int j = 0; j < DPT; ++j)
        st[j] = open[j] ? ld_relaxed_u32(&lookback[(size_t)pred[j] * RADIX + threadIdx.x * DPT + j]) : 0u;
      bool waiting = false, any_open = false;
#pragma unroll
      for (int j = 0; j < DPT; ++j) {
        if (!open[j]) continue;
        const unsigned flag = st[j] & ~RS_VAL_MASK;
        if (flag == 0u) {  // predecessor not published yet: poll it again
          waiting = true;
          any_open = true;
          continue;
        }
        excl[j] += st[j] & RS_VAL_MASK;
        if (flag == RS_FLAG_PRE || --pred[j] < 0) open[j] = false;
        else any_open = true;
      }
      if (!any_open) break;
      if (waiting) {
        if (++spins > SC_SPIN_LIMIT) { atomicOr(err, SC_DEVERR_TIMEOUT); break; }
        __nanosleep(20);
      }
    }
#pragma unroll
    for (int j = 0; j < DPT; ++j)
      st_relaxed_u32(&lb[threadIdx.x * DPT + j], RS_FLAG_PRE | ((excl[j] + cnt[j]) & RS_VAL_MASK));
  }
  // tile-local exclusive scan of the digit counts (DPT consecutive digits per thread)
  {
    uint32_t tsum = 0;
#pragma unroll
    for (int j = 0; j < DPT; ++j) tsum += cnt[j];
    uint32_t x = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    __shared__ uint32_t s_w[RS_WARPS];
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < RS_WARPS ? s_w[lane] : 0u;
#pragma unroll
      for (int o = 1; o < RS_WARPS; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < RS_WARPS) s_w[lane] = w;
    }
    __syncthreads();
    uint32_t te = x - tsum + (warp > 0 ? s_w[warp - 1] : 0u);
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      const int d = threadIdx.x * DPT + j;
      sm.tile_excl[d] = te;
      sm.out_base[d] = (int)(digit_base[d] + excl[j]) - (int)te;
      te += cnt[j];
    }
  }
  __syncthreads();
  // keys to digit order in shared memory, with the input slot of each payload
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    if (FULL || wbase + (uint64_t)k * 32 + lane < n) {
      const uint32_t dd = (uint32_t)(key[k] >> shift) & dmask;
      const uint32_t pos = sm.tile_excl[dd] + sm.warp_hist[warp][dd] + rank[k];
      sm.keys[pos] = key[k];
      sm.src[pos] = (uint16_t)(wslot + k * 32 + lane);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  const uint32_t valid = FULL ? (uint32_t)TILE : (uint32_t)min((uint64_t)TILE, n - tbase);
  for (uint32_t idx = threadIdx.x; idx < valid; idx += RS_THREADS) {
    const K kk = sm.keys[idx];
    const uint32_t dd = (uint32_t)(kk >> shift) & dmask;
    const long long g = (long long)sm.out_base[dd] + (long long)idx;
    if (g < 0 || (uint64_t)g >= n) {  // only after a look-back gave up: keep the write in bounds
      atomicOr(err, SC_DEVERR_TIMEOUT);
      continue;
    }
    kout[g] = kk;
    vout[g] = sm.vals[sm.src[idx]];
  }
}

// One onesweep pass.  Ranking: the lanes of a warp holding the same digit are
// found with RB ballots (one per digit bit), a fixed cost independent of how
// many distinct digits the warp holds; lanes are ranked in input order, so the
// pass is stable.  Look-back status words carry their own value (flag in the
// top 2 bits, count below), so relaxed loads and stores suffice.
template <typename K, bool NARROW, int RB>
__global__ void __launch_bounds__(RS_THREADS, RB == 8 ? 4 : 3) k_rs_pass(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                        K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                        uint64_t n_cap, const uint64_t* __restrict__ d_n, int shift,
                                                        const uint32_t* __restrict__ digit_base,
                                                        unsigned* __restrict__ lookback, unsigned* __restrict__ ticket,
                                                        uint32_t* __restrict__ err, int dbits) {
  constexpr int IPT = RsCfg<K>::IPT;
  constexpr int TILE = RS_THREADS * IPT;
  constexpr int RADIX = Rdx<RB>::RADIX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsSmem<K, RB>& sm = *reinterpret_cast<RsSmem<K, RB>*>(smem_raw);
  if (threadIdx.x == 0) sm.tile_id = atomicAdd(ticket, 1u);
  for (int t = threadIdx.x; t < RS_WARPS * RADIX; t += RS_THREADS) (&sm.warp_hist[0][0])[t] = 0;
  __syncthreads();
  const uint32_t tile = sm.tile_id;
  const uint64_t n = d_n ? min(*d_n, n_cap) : n_cap;
  const uint64_t tbase = (uint64_t)tile * TILE;
  if (tbase >= n) return;  // every later ticket is beyond n as well: nobody waits on this tile
  if (tbase + TILE <= n)
    rs_pass_tile<K, true, NARROW, RB>(sm, kin, vin, kout, vout, n, shift, digit_base, lookback, err, tile, tbase,
                                      dbits);
  else
    rs_pass_tile<K, false, NARROW, RB>(sm, kin, vin, kout, vout, n, shift, digit_base, lookback, err, tile, tbase,
                                       dbits);
}

size_t radix_scratch_bytes(uint64_t n, uint32_t key_bytes) {
  const int tile = RS_THREADS * (key_bytes == 4 ? RsCfg<uint32_t>::IPT : RsCfg<uint64_t>::IPT);
  const uint64_t tiles = sc_div_up(n > 0 ? n : 1, tile);
  // [hist passes x RADIX u32][tickets 16 u32][lookback passes x tiles x RADIX u32]; 9-bit digits bound both
  const int max_passes = (int)((key_bytes * 8 + 8) / 9);
  return RS_HIST_BYTES + 64 + (size_t)max_passes * tiles * 512 * 4;
}

template <typename K, int RB>
static sc_status radix_passes(sc_ctx* ctx, K* keys, uint32_t* vals, K* keys_tmp, uint32_t* vals_tmp, uint64_t n_cap,
                              uint32_t key_bits, const uint64_t* d_n, void* scratch, size_t bytes,
                              bool* result_in_tmp) {
  constexpr int RADIX = Rdx<RB>::RADIX;
  const int passes = (int)((key_bits + RB - 1) / RB);
  constexpr int TILE = RS_THREADS * RsCfg<K>::IPT;
  const uint64_t tiles = sc_div_up(n_cap, TILE);
  const size_t need = RS_HIST_BYTES + 64 + (size_t)passes * tiles * RADIX * 4;
  if (bytes < need) return sc_fail(ctx, SC_ERR_INVALID_ARG, "radix scratch too small");
  uint32_t* hist = reinterpret_cast<uint32_t*>(scratch);
  unsigned* tickets = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(scratch) + RS_HIST_BYTES);
  unsigned* lookback = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(scratch) + RS_HIST_BYTES + 64);
  SC_CUDA_TRY(ctx, cudaMemsetAsync(scratch, 0, need, ctx->stream), "memset radix scratch");
  const unsigned hist_blocks = (unsigned)std::min<uint64_t>(sc_div_up(n_cap, RS_THREADS),
                                                            (uint64_t)ctx->sm_count * RS_HIST_BLOCKS_PER_SM);
  k_rs_hist<K, RB><<<hist_blocks, RS_THREADS, 0, ctx->stream>>>(keys, n_cap, d_n, passes, key_bits, hist);
  SC_TRY(sc_check_launch(ctx, "k_rs_hist"));
  k_rs_hist_scan<RB><<<passes, RADIX, 0, ctx->stream>>>(hist);
  SC_TRY(sc_check_launch(ctx, "k_rs_hist_scan"));
  const size_t smem = sizeof(RsSmem<K, RB>);
  static bool attr_set = false;
  if (!attr_set) {
    SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_rs_pass<K, false, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem), "smem attr");
    SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_rs_pass<K, true, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem), "smem attr");
    attr_set = true;
  }
  K* kin = keys; uint32_t* vin = vals; K* kout = keys_tmp; uint32_t* vout = vals_tmp;
  for (int p = 0; p < passes; ++p) {
    const int dbits = std::min(RB, (int)key_bits - RB * p);
    if (dbits == RB)
      k_rs_pass<K, false, RB><<<(unsigned)tiles, RS_THREADS, smem, ctx->stream>>>(
          kin, vin, kout, vout, n_cap, d_n, RB * p, hist + p * RADIX, lookback + (size_t)p * tiles * RADIX,
          tickets + p, ctx->d_error, RB);
    else
      k_rs_pass<K, true, RB><<<(unsigned)tiles, RS_THREADS, smem, ctx->stream>>>(
          kin, vin, kout, vout, n_cap, d_n, RB * p, hist + p * RADIX, lookback + (size_t)p * tiles * RADIX,
          tickets + p, ctx->d_error, dbits);
    SC_TRY(sc_check_launch(ctx, "k_rs_pass"));
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  *result_in_tmp = (passes & 1) != 0;
  return SC_OK;
}

// 8 or 9 bits per pass: a 9-bit pass costs about 1.5 8-bit passes (3 instead
// of 4 blocks per SM, one ballot more, two digits per thread in the look-back;
// measured on 8M 64-bit keys: 4 passes 0.59 ms, 5 passes 0.49 ms), so 9 bits
// are taken only when they save a third of the passes — in practice a 9-bit
// key, one pass instead of an 8-bit and a 1-bit pass (2.8e7 items: 0.44 ms
// instead of 0.57 ms, with the histogram).
// digit_bits 8 or 9 forces the digit width (the autotuner's radix-width axis).
template <typename K>
sc_status radix_sort(sc_ctx* ctx, K* keys, uint32_t* vals, K* keys_tmp, uint32_t* vals_tmp, uint64_t n_cap,
                     uint32_t key_bits, const uint64_t* d_n, void* scratch, size_t bytes, bool* result_in_tmp,
                     int digit_bits) {
  *result_in_tmp = false;
  if (n_cap == 0) return SC_OK;
  if (n_cap > RS_VAL_MASK) return sc_fail(ctx, SC_ERR_CAPACITY, "radix sort limited to 2^30 - 1 elements");
  if (key_bits > sizeof(K) * 8) return sc_fail(ctx, SC_ERR_INVALID_ARG, "key_bits larger than the key type");
  if (digit_bits != 0 && digit_bits != 8 && digit_bits != 9)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "radix digits are 8 or 9 bits (0 = chosen by pass count)");
  if (key_bits == 0) return SC_OK;
  if (digit_bits == 9 || (digit_bits == 0 && 3 * ((key_bits + 8) / 9) < 2 * ((key_bits + 7) / 8)))
    return radix_passes<K, 9>(ctx, keys, vals, keys_tmp, vals_tmp, n_cap, key_bits, d_n, scratch, bytes,
                              result_in_tmp);
  return radix_passes<K, 8>(ctx, keys, vals, keys_tmp, vals_tmp, n_cap, key_bits, d_n, scratch, bytes,
                            result_in_tmp);
}

// ---------------------------------------------------------------- segmented sort
// n_segs independent sorts of u32 keys (with u32 payloads), segment g holding
// elements [g seg_len, (g + 1) seg_len), seg_len a multiple of the tile
// (RS_SEG_TILE).  Every tile lies in one segment; the passes keep one digit
// histogram per segment (its base includes the segment's offset) and a tile's
// look-back stops at the first tile of its segment, so one launch per pass
// sorts every segment.  The trainer sorts each view's depth keys this way: 32
// bits in 4 passes instead of (view << 32 | depth) keys in 5.
#define RS_SEG_TILE (RS_THREADS * 16)

template <int RB>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist_seg(const uint32_t* __restrict__ keys, uint32_t seg_len,
                                                            uint32_t n_segs, int passes, uint32_t key_bits,
                                                            uint32_t* __restrict__ hist /* [passes][n_segs][RADIX] */) {
  constexpr int RADIX = Rdx<RB>::RADIX;
  __shared__ uint32_t sh[4 * RADIX];
  for (int t = threadIdx.x; t < passes * RADIX; t += RS_THREADS) sh[t] = 0;
  __syncthreads();
  const uint32_t g = blockIdx.y;
  const uint32_t* k0 = keys + (size_t)g * seg_len;
  const uint64_t step = (uint64_t)gridDim.x * RS_THREADS;
  for (uint64_t i0 = (uint64_t)blockIdx.x * RS_THREADS + threadIdx.x; i0 < seg_len; i0 += step * RS_HIST_UNROLL) {
    uint32_t k[RS_HIST_UNROLL];
#pragma unroll
    for (int u = 0; u < RS_HIST_UNROLL; ++u) {
      const uint64_t i = i0 + u * step;
      k[u] = i < seg_len ? k0[i] : 0u;
    }
#pragma unroll
    for (int u = 0; u < RS_HIST_UNROLL; ++u) {
      if (i0 + u * step < seg_len) {
        for (int p = 0; p < passes; ++p)
          atomicAdd(&sh[p * RADIX + ((k[u] >> (RB * p)) & rs_digit_mask(key_bits, p, RB))], 1u);
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < passes * RADIX; t += RS_THREADS) {
    const uint32_t c = sh[t];
    if (c) atomicAdd(&hist[((size_t)(t / RADIX) * n_segs + g) * RADIX + t % RADIX], c);
  }
}

// exclusive scan of each (pass, segment) histogram plus the segment's base
template <int RB>
__global__ void __launch_bounds__(1 << RB) k_rs_hist_scan_seg(uint32_t* __restrict__ hist, uint32_t n_segs,
                                                              uint32_t seg_len) {
  constexpr int RADIX = Rdx<RB>::RADIX;
  __shared__ uint32_t s[RADIX];
  uint32_t* h = hist + (size_t)blockIdx.x * RADIX;
  const uint32_t base = (blockIdx.x % n_segs) * seg_len;
  const uint32_t v = h[threadIdx.x];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < RADIX; o <<= 1) {
    uint32_t y = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
    __syncthreads();
    s[threadIdx.x] += y;
    __syncthreads();
  }
  h[threadIdx.x] = base + s[threadIdx.x] - v;
}

template <bool NARROW>
__global__ void __launch_bounds__(RS_THREADS, 4) k_rs_pass_seg(const uint32_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
                                                            uint32_t* __restrict__ vout, uint64_t n, uint32_t tiles_per_seg,
                                                            int shift, const uint32_t* __restrict__ digit_base,
                                                            unsigned* __restrict__ lookback,
                                                            unsigned* __restrict__ ticket, uint32_t* __restrict__ err,
                                                            int dbits) {
  constexpr int RADIX = Rdx<8>::RADIX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsSmem<uint32_t, 8>& sm = *reinterpret_cast<RsSmem<uint32_t, 8>*>(smem_raw);
  if (threadIdx.x == 0) sm.tile_id = atomicAdd(ticket, 1u);
  for (int t = threadIdx.x; t < RS_WARPS * RADIX; t += RS_THREADS) (&sm.warp_hist[0][0])[t] = 0;
  __syncthreads();
  const uint32_t tile = sm.tile_id;
  const uint64_t tbase = (uint64_t)tile * RS_SEG_TILE;
  if (tbase >= n) return;
  const uint32_t g = tile / tiles_per_seg, local = tile - g * tiles_per_seg;
  // tiles of segment g look back only on their own segment's tiles, which hold
  // earlier tickets
  rs_pass_tile<uint32_t, true, NARROW, 8>(sm, kin, vin, kout, vout, n, shift, digit_base + (size_t)g * RADIX,
                                          lookback + (size_t)g * tiles_per_seg * RADIX, err, local, tbase, dbits);
}

size_t radix_seg_scratch_bytes(uint64_t seg_len, uint32_t n_segs) {
  const uint64_t tiles = sc_div_up(seg_len, RS_SEG_TILE) * n_segs;
  return (size_t)4 * n_segs * 256 * 4 + 64 + (size_t)4 * tiles * 256 * 4;
}

sc_status radix_sort_segments(sc_ctx* ctx, uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                              uint32_t seg_len, uint32_t n_segs, uint32_t key_bits, void* scratch, size_t bytes,
                              bool* result_in_tmp) {
  constexpr int RB = 8, RADIX = 256;
  *result_in_tmp = false;
  const uint64_t n = (uint64_t)seg_len * n_segs;
  if (n == 0 || key_bits == 0) return SC_OK;
  if (seg_len % RS_SEG_TILE) return sc_fail(ctx, SC_ERR_INVALID_ARG, "segment length must be a multiple of the sort tile");
  if (n > RS_VAL_MASK) return sc_fail(ctx, SC_ERR_CAPACITY, "radix sort limited to 2^30 - 1 elements");
  if (key_bits > 32) return sc_fail(ctx, SC_ERR_INVALID_ARG, "key_bits larger than the key type");
  const int passes = (int)((key_bits + RB - 1) / RB);
  const uint32_t tps = seg_len / RS_SEG_TILE;
  const uint64_t tiles = (uint64_t)tps * n_segs;
  const size_t hist_bytes = (size_t)passes * n_segs * RADIX * 4;
  const size_t need = hist_bytes + 64 + (size_t)passes * tiles * RADIX * 4;
  if (bytes < need) return sc_fail(ctx, SC_ERR_INVALID_ARG, "radix scratch too small");
  uint32_t* hist = reinterpret_cast<uint32_t*>(scratch);
  unsigned* tickets = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(scratch) + hist_bytes);
  unsigned* lookback = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(scratch) + hist_bytes + 64);
  SC_CUDA_TRY(ctx, cudaMemsetAsync(scratch, 0, need, ctx->stream), "memset radix scratch");
  const unsigned bx = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>(sc_div_up(seg_len, RS_THREADS), (uint64_t)ctx->sm_count * RS_HIST_BLOCKS_PER_SM / n_segs));
  k_rs_hist_seg<RB><<<dim3(bx, n_segs), RS_THREADS, 0, ctx->stream>>>(keys, seg_len, n_segs, passes, key_bits, hist);
  SC_TRY(sc_check_launch(ctx, "k_rs_hist_seg"));
  k_rs_hist_scan_seg<RB><<<(unsigned)(passes * n_segs), RADIX, 0, ctx->stream>>>(hist, n_segs, seg_len);
  SC_TRY(sc_check_launch(ctx, "k_rs_hist_scan_seg"));
  const size_t smem = sizeof(RsSmem<uint32_t, RB>);
  static bool attr_set = false;
  if (!attr_set) {
    SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_rs_pass_seg<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem), "smem attr");
    SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_rs_pass_seg<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem), "smem attr");
    attr_set = true;
  }
  uint32_t* kin = keys; uint32_t* vin = vals; uint32_t* kout = keys_tmp; uint32_t* vout = vals_tmp;
  for (int p = 0; p < passes; ++p) {
    const int dbits = std::min(RB, (int)key_bits - RB * p);
    const uint32_t* db = hist + (size_t)p * n_segs * RADIX;
    unsigned* lb = lookback + (size_t)p * tiles * RADIX;
    if (dbits == RB)
      k_rs_pass_seg<false><<<(unsigned)tiles, RS_THREADS, smem, ctx->stream>>>(kin, vin, kout, vout, n, tps, RB * p,
                                                                             db, lb, tickets + p, ctx->d_error, RB);
    else
      k_rs_pass_seg<true><<<(unsigned)tiles, RS_THREADS, smem, ctx->stream>>>(kin, vin, kout, vout, n, tps, RB * p,
                                                                            db, lb, tickets + p, ctx->d_error, dbits);
    SC_TRY(sc_check_launch(ctx, "k_rs_pass_seg"));
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  *result_in_tmp = (passes & 1) != 0;
  return SC_OK;
}

template sc_status radix_sort<uint32_t>(sc_ctx*, uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint64_t, uint32_t,
                                        const uint64_t*, void*, size_t, bool*, int);

// Failure-detection self-test: one onesweep pass over two tiles whose ticket
// counter starts at 1, so the first tile to run looks back on tile 0, which no
// block ever processes.  Its bounded wait gives up after SC_SPIN_LIMIT polls,
// raises SC_DEVERR_TIMEOUT and skips every out-of-range write; the kernel
// ends and the host reads the error word.
sc_status selftest_lookback_timeout(sc_ctx* ctx) {
  using K = uint32_t;
  constexpr int TILE = RS_THREADS * RsCfg<K>::IPT;
  const uint64_t n = 2 * (uint64_t)TILE;
  const size_t data = (size_t)n * 4;
  const size_t need = 4 * data + RS_HIST_BYTES + 64 + (size_t)2 * 256 * 4;
  void* buf = nullptr;
  SC_TRY(sc_scratch(ctx, need, &buf));
  char* p = reinterpret_cast<char*>(buf);
  K* keys = reinterpret_cast<K*>(p);
  uint32_t* vals = reinterpret_cast<uint32_t*>(p + data);
  K* kout = reinterpret_cast<K*>(p + 2 * data);
  uint32_t* vout = reinterpret_cast<uint32_t*>(p + 3 * data);
  uint32_t* hist = reinterpret_cast<uint32_t*>(p + 4 * data);
  unsigned* ticket = reinterpret_cast<unsigned*>(p + 4 * data + RS_HIST_BYTES);
  unsigned* lookback = reinterpret_cast<unsigned*>(p + 4 * data + RS_HIST_BYTES + 64);
  SC_CUDA_TRY(ctx, cudaMemsetAsync(p, 0, need, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(ticket, 1, 1, ctx->stream), "ticket = 1");  // tile 0 is never handed out
  const size_t smem = sizeof(RsSmem<K, 8>);
  SC_CUDA_TRY(ctx, cudaFuncSetAttribute(k_rs_pass<K, false, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem), "smem attr");
  k_rs_pass<K, false, 8><<<2, RS_THREADS, smem, ctx->stream>>>(keys, vals, kout, vout, n, nullptr, 0, hist, lookback,
                                                               ticket, ctx->d_error, 8);
  SC_TRY(sc_check_launch(ctx, "k_rs_pass (timeout self-test)"));
  return sc_check_device_error(ctx);
}
template sc_status radix_sort<uint64_t>(sc_ctx*, uint64_t*, uint32_t*, uint64_t*, uint32_t*, uint64_t, uint32_t,
                                        const uint64_t*, void*, size_t, bool*, int);

}  // namespace sck
