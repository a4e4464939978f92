// trainer.cu — the batched training iteration (train.rs:155-250 for n_views
// views per step) as one stream of kernels, replayed as a CUDA graph.
//
//   H2D step params (cameras, Adam bias corrections)         memcpy node
//   project + SH for all views, per-view depth keys, counts  k_project
//   per-view depth sort of the splats                        segmented onesweep u32, 16-bit depth
//     (the reference's quantised depth: a stable sort in splat order gives each tile the
//     (depth16, splat index) order of the reference's 32-bit pair keys)
//   item counts in depth order -> offsets                    gather + decoupled-look-back scan
//   items (mask | view, super tile; splat) in depth order    k_super_emit (two-level binning)
//   stable sort of the items by super tile                   onesweep u32 (super tile bits)
//   per-super-tile ranges (+ pair count from the masks)      k_tile_ranges_u32x4
//   alpha-blend forward over the super-tile item lists       k_composite (item lists)
//   alpha-blend backward, MSE dL/dC in its prologue          k_composite_backward (item lists)
//   project backward over all views -> gradient rows         k_project_backward_shards (one shard)
//   Adam + constraints + densify statistic over the rows     k_adam_rows
//   loss / pair count / error word -> pinned host            finalize + memcpy node
// (sort_mode 1 keeps the pair path: emission of (view*T + tile, splat) pairs,
// their stable tile sort, per-tile ranges and pair-list blends.)
//
// The item (or pair) buffers have a device-side capacity.  When a step emits
// more than fit, the emit kernel raises SC_DEVERR_CAPACITY, the blend and Adam
// kernels of that step skip their work (parameters are untouched), and the host
// grows the buffers and runs the step again.
#include "sc_internal.cuh"

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>


namespace {

struct StepParams {
  sc_camera cams[SC_MAX_VIEWS];
  float bc[4];  // bc1, bc2, the step number's bits (stochastic-rounding seed)
};

struct StepOut {
  double loss;
  unsigned long long pairs;
  unsigned long long items;  // two-level binning items
  uint32_t err;
  uint32_t pad;
};

// loss = mean over the views, or (weight > 0) weight * sum over the views, of
// (1 - lambda) MSE + lambda (1 - SSIM) (loss.rs:383-410; MSE alone without SSIM sums)
__global__ void k_finalize(const double* __restrict__ loss_sums, const double* __restrict__ ssim_sums, float lambda,
                           uint32_t n_views, double inv_count, double weight, const uint64_t* __restrict__ d_total,
                           const uint32_t* __restrict__ err, StepOut* __restrict__ out) {
  double acc = 0.0;
  for (uint32_t v = 0; v < n_views; ++v) {
    const double m = loss_sums[v] * inv_count;
    if (!ssim_sums) { acc += m; continue; }
    const double sv = 1.0 - ssim_sums[v] * inv_count;
    acc += lambda == 1.0f ? sv : (1.0 - (double)lambda) * m + (double)lambda * sv;
  }
  out->loss = weight > 0.0 ? acc * weight : acc / (double)n_views;
  out->pairs = d_total[0];
  out->items = d_total[1];
  out->err = *err;
}

// stage names of the two-level binning step (the pair-sort step uses kStageNames)
const char* kStageNames2[] = {"project", "depth_sort", "count_scan", "item_emit", "item_sort", "item_ranges",
                              "blend_fwd", "blend_bwd", "bwd_adam"};
const char* kStageNames[] = {"project", "depth_sort", "count_scan", "emit", "tile_sort", "ranges",
                             "blend_fwd", "blend_bwd", "bwd_adam"};
constexpr int kStages = 9;

uint32_t bits_for(uint64_t max_value) {
  uint32_t b = 0;
  while (b < 64 && (max_value >> b) != 0) ++b;
  return b;
}

}  // namespace

struct sc_trainer {
  sc_ctx* ctx = nullptr;
  sc_train_config cfg{};
  uint32_t V = 0, tiles_x = 0, tiles_y = 0, T = 0;
  uint64_t P = 0;
  uint32_t stride = 0;
  StepParams* h_params = nullptr;
  StepParams* d_params = nullptr;
  StepOut* h_out = nullptr;
  StepOut* d_out = nullptr;
  // per (view, splat)
  float4* rec = nullptr; float4* pgrad = nullptr;
  float4* pcomp = nullptr;  // compensation records of pgrad (cfg.compensated_sums)
  float* grads = nullptr;  // [SC_NROWS][grad_stride] per-splat gradient rows (one GPU)
  uint32_t grad_stride = 0;
  uint32_t* dkeys = nullptr; uint32_t* dkeys_tmp = nullptr;  // per view, a segment of stride depth keys
  uint32_t* ids = nullptr; uint32_t* ids_tmp = nullptr;
  uint32_t* counts_by_id = nullptr; uint32_t* counts = nullptr;
  // pairs (the pair-sort path uses all four; two-level binning writes vals only)
  uint64_t kcap = 0;
  uint32_t* keys = nullptr; uint32_t* keys_tmp = nullptr; uint32_t* vals = nullptr; uint32_t* vals_tmp = nullptr;
  // two-level binning: (member mask | super tile, splat) items, per-tile counts -> offsets
  bool two_level = false;
  uint32_t ST = 0, super_bits = 0;
  uint64_t icap = 0;
  uint32_t* ikeys = nullptr; uint32_t* ikeys_tmp = nullptr; uint32_t* ivals = nullptr; uint32_t* ivals_tmp = nullptr;
  uint32_t* iranges = nullptr;  // [V * ST] (begin, end) of each super tile's items
  // per (view, tile) / pixel
  uint32_t* ranges = nullptr;
  float4* image = nullptr; uint2* aux = nullptr; float4* dl_dc = nullptr;
  // SSIM term of the loss (cfg.ssim_lambda > 0): coefficient planes and per-view map sums
  float* ssim_terms = nullptr; double* d_ssim = nullptr;
  const float* targets = nullptr;
  // targets in pinned host memory: copied every step on a side stream, in
  // parallel with projection, sorting and emission, into d_host_targets
  const float* h_targets = nullptr;
  float* d_host_targets = nullptr;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_fwd = nullptr;
  cudaEvent_t ev_view[SC_MAX_VIEWS] = {};  // view v's targets copied
  cudaStream_t bwd_stream[SC_MAX_VIEWS] = {};  // view v's blend backward (host targets)
  cudaEvent_t ev_bwd[SC_MAX_VIEWS] = {};
  double* d_loss = nullptr;
  uint64_t* d_total = nullptr;
  void* scratch = nullptr; size_t scratch_bytes = 0;
  // gradient-only steps (data-parallel views): shard-major output
  bool grads_mode = false;
  float loss_weight = 0.0f;
  float* gout = nullptr;
  uint32_t g_shards = 0, g_shard = 0;
  // many scenes (sc_scenes_trainer): view v is scene v, with its own store,
  // moments, statistic, gradient rows and image size; the table is copied to
  // the device by the step's first node
  bool scenes_mode = false;
  struct SceneHost {
    sc_splats* s = nullptr; sc_moments* mo = nullptr; float* acc = nullptr;
    uint32_t width = 0, height = 0;
    float* grads = nullptr; uint32_t gstride = 0;
  } scene[SC_MAX_VIEWS];
  SceneDev* h_scenes = nullptr;  // pinned
  SceneDev* d_scenes = nullptr;
  double* h_losses = nullptr;    // pinned: per-view squared-error sums of the last step
  uint32_t scene_max_cap = 0, scene_max_gstride = 0;
  // graph
  cudaGraphExec_t exec = nullptr;
  const void* g_key[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  uint64_t g_key_n = 0, g_key_kcap = 0, g_key_icap = 0;
  bool g_key_grads = false;
  float g_key_w = 0.0f;
  uint32_t g_key_shards = 0, g_key_shard = 0;
  // results of the last step
  uint64_t last_pairs = 0, last_items = 0;
  uint32_t kernels_per_step = 0;
  // profiling: 0 off, 1 stage events + blend work counters, 2 also (pixel, entry) pair counts
  int profiling = 0;
  cudaEvent_t ev[kStages + 1] = {};
  double acc_ms[kStages] = {};
  uint64_t prof_steps = 0;
  float avg_ms_out[kStages] = {};
  // blend work counters while profiling: forward then backward slots
  uint64_t* d_work = nullptr;
  uint64_t work_acc[6] = {};  // fwd scanned, staged; bwd scanned, staged; fwd, bwd (pixel, entry) pairs
};

static void trainer_free_splat_arrays(sc_trainer* tr) {
  cudaFree(tr->rec); cudaFree(tr->pgrad); cudaFree(tr->pcomp); cudaFree(tr->grads); cudaFree(tr->dkeys);
  cudaFree(tr->dkeys_tmp);
  tr->pcomp = nullptr;
  cudaFree(tr->ids); cudaFree(tr->ids_tmp); cudaFree(tr->counts_by_id); cudaFree(tr->counts);
  tr->rec = tr->pgrad = nullptr; tr->dkeys = tr->dkeys_tmp = nullptr;
  tr->ids = tr->ids_tmp = tr->counts_by_id = tr->counts = nullptr;
  tr->stride = 0;
}

static void trainer_free_pairs(sc_trainer* tr) {
  cudaFree(tr->keys); cudaFree(tr->keys_tmp); cudaFree(tr->vals); cudaFree(tr->vals_tmp);
  tr->keys = tr->keys_tmp = tr->vals = tr->vals_tmp = nullptr;
  tr->kcap = 0;
}

static void trainer_free_items(sc_trainer* tr) {
  cudaFree(tr->ikeys); cudaFree(tr->ikeys_tmp); cudaFree(tr->ivals); cudaFree(tr->ivals_tmp);
  tr->ikeys = tr->ikeys_tmp = tr->ivals = tr->ivals_tmp = nullptr;
  tr->icap = 0;
}

static void trainer_drop_graph(sc_trainer* tr) {
  if (tr->exec) cudaGraphExecDestroy(tr->exec);
  tr->exec = nullptr;
}

static sc_status ensure_scratch(sc_trainer* tr) {
  sc_ctx* ctx = tr->ctx;
  const uint64_t nsp = (uint64_t)tr->V * tr->stride;
  size_t need = std::max({sck::radix_seg_scratch_bytes(tr->stride, tr->V),
                          sck::radix_scratch_bytes(std::max<uint64_t>(tr->kcap, 1), 4),
                          sck::radix_scratch_bytes(std::max<uint64_t>(tr->icap, 1), 4), sck::scan_scratch_bytes(nsp + 1),
                          sck::scan_scratch_bytes((uint64_t)tr->V * tr->T + 1)});
  if (need <= tr->scratch_bytes) return SC_OK;
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  cudaFree(tr->scratch);
  tr->scratch = nullptr;
  need = need + need / 4;
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->scratch, need), "trainer scratch");
  tr->scratch_bytes = need;
  trainer_drop_graph(tr);
  return SC_OK;
}

// Per-view arrays hold stride = cap rounded up to whole sort tiles, so each
// view's depth keys are one segment of the segmented depth sort.
static sc_status ensure_splat_arrays(sc_trainer* tr, uint32_t cap) {
  cap = (uint32_t)sc_div_up(cap, sck::RADIX_SEG_TILE) * sck::RADIX_SEG_TILE;
  if (tr->stride == cap) return SC_OK;
  sc_ctx* ctx = tr->ctx;
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  trainer_free_splat_arrays(tr);
  const size_t nv = (size_t)tr->V * cap;
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->rec, nv * 48), "rec");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->pgrad, nv * 48), "pgrad");
  if (tr->cfg.compensated_sums) SC_CUDA_TRY(ctx, cudaMalloc(&tr->pcomp, nv * 48), "pcomp");
  tr->grad_stride = (cap + 63u) & ~63u;
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->grads, (size_t)SC_NROWS * tr->grad_stride * 4), "grads");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->dkeys, nv * 4), "dkeys");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->dkeys_tmp, nv * 4), "dkeys");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->ids, nv * 4), "ids");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->ids_tmp, nv * 4), "ids");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->counts_by_id, nv * 4), "counts");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->counts, (nv + 1) * 4), "counts");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->rec, 0, nv * 48, ctx->stream), "zero");
  tr->stride = cap;
  trainer_drop_graph(tr);
  return ensure_scratch(tr);
}

static sc_status ensure_items(sc_trainer* tr, uint64_t I) {
  if (!tr->two_level || (I <= tr->icap && tr->icap)) return SC_OK;
  sc_ctx* ctx = tr->ctx;
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  trainer_free_items(tr);
  uint64_t cap = I + I / 4 + 65536;
  if (cap > (1ull << 30) - 1) cap = (1ull << 30) - 1;
  if (I > cap) return sc_fail(ctx, SC_ERR_CAPACITY, "more than 2^30 binning items in one step");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->ikeys, cap * 4), "items");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->ikeys_tmp, cap * 4), "items");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->ivals, cap * 4), "items");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->ivals_tmp, cap * 4), "items");
  // zero-filled so a step whose emission overflowed still reads valid ids
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->ivals, 0, cap * 4, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->ivals_tmp, 0, cap * 4, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->ikeys, 0, cap * 4, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->ikeys_tmp, 0, cap * 4, ctx->stream), "zero");
  tr->icap = cap;
  trainer_drop_graph(tr);
  return ensure_scratch(tr);
}

static sc_status ensure_pairs(sc_trainer* tr, uint64_t K) {
  if (tr->two_level || (K <= tr->kcap && tr->kcap)) return SC_OK;  // two-level blends the item lists
  sc_ctx* ctx = tr->ctx;
  SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  trainer_free_pairs(tr);
  uint64_t cap = K + K / 4 + 65536;
  if (cap > (1ull << 30) - 1) cap = (1ull << 30) - 1;
  if (K > cap) return sc_fail(ctx, SC_ERR_CAPACITY, "more than 2^30 tile/splat pairs in one step");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->vals, cap * 4), "vals");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->keys, cap * 4), "keys");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->keys_tmp, cap * 4), "keys");
  SC_CUDA_TRY(ctx, cudaMalloc(&tr->vals_tmp, cap * 4), "vals");
  // zero-filled so a step whose emission overflowed still reads valid ids
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->vals, 0, cap * 4, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->keys, 0, cap * 4, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->keys_tmp, 0, cap * 4, ctx->stream), "zero");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->vals_tmp, 0, cap * 4, ctx->stream), "zero");
  tr->kcap = cap;
  trainer_drop_graph(tr);
  return ensure_scratch(tr);
}

static void mark(sc_trainer* tr, int i, bool capturing) {
  if (!tr->profiling) return;
  if (capturing)
    cudaEventRecordWithFlags(tr->ev[i], tr->ctx->stream, cudaEventRecordExternal);
  else
    cudaEventRecord(tr->ev[i], tr->ctx->stream);
}

// Enqueue one step.  sizing: stop after the scan, read the pair count and
// (re)size the pair buffers before emitting (eager runs only).
static sc_status enqueue_step(sc_trainer* tr, sc_splats* s, sc_moments* mo, float* acc, bool capturing, bool sizing) {
  sc_ctx* ctx = tr->ctx;
  const sc_camera* d_cams = reinterpret_cast<const sc_camera*>(tr->d_params);  // cams is the first member
  const float* d_bc = reinterpret_cast<const float*>(reinterpret_cast<const char*>(tr->d_params) +
                                                     offsetof(StepParams, bc));
  const uint32_t V = tr->V;
  const uint64_t nsp = (uint64_t)V * tr->stride;
  const DSplats ds = s ? dview(s) : DSplats{};
  const DMoments dm = mo ? dview(mo) : DMoments{};
  const uint64_t launches0 = ctx->launches;
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(tr->d_params, tr->h_params, sizeof(StepParams), cudaMemcpyHostToDevice, ctx->stream),
              "params H2D");
  if (tr->scenes_mode)
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(tr->d_scenes, tr->h_scenes, sizeof(SceneDev) * V, cudaMemcpyHostToDevice,
                                     ctx->stream), "scene table H2D");
  const SceneDev* scenes = tr->scenes_mode ? tr->d_scenes : nullptr;
  if (tr->h_targets) {  // host targets: this step's copy runs beside the stages that do not read them, view by view
    SC_CUDA_TRY(ctx, cudaEventRecord(tr->ev_fork, ctx->stream), "fork");
    SC_CUDA_TRY(ctx, cudaStreamWaitEvent(tr->copy_stream, tr->ev_fork, 0), "fork wait");
    const size_t vb = (size_t)tr->P * 3;
    for (uint32_t v = 0; v < V; ++v) {
      SC_CUDA_TRY(ctx, cudaMemcpyAsync(tr->d_host_targets + v * vb, tr->h_targets + v * vb, vb * sizeof(float),
                                       cudaMemcpyHostToDevice, tr->copy_stream), "targets H2D");
      SC_CUDA_TRY(ctx, cudaEventRecord(tr->ev_view[v], tr->copy_stream), "copied");
    }
  }
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->d_loss, 0, 8 * (size_t)V, ctx->stream), "zero loss");
  uint64_t* work_fwd = tr->profiling ? tr->d_work : nullptr;
  uint64_t* work_bwd = tr->profiling ? tr->d_work + 3 * sck::BLEND_WORK_SLOTS : nullptr;
  if (tr->profiling)
    SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->d_work, 0, 6 * sck::BLEND_WORK_SLOTS * 8, ctx->stream), "zero work");
  SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->counts + nsp, 0, 4, ctx->stream), "zero count tail");
  mark(tr, 0, capturing);
  SC_TRY(sck::launch_project(ctx, ds, d_cams, V, tr->stride, tr->rec, &tr->cfg.tiling, tr->dkeys, tr->ids,
                             tr->counts_by_id, tr->cfg.fp64_det ? 1 : 0,
                             (tr->cfg.tile_cull ? 1 : 0) | (tr->two_level ? 2 : 0), tr->pgrad, tr->pcomp,
                             tr->scenes_mode ? tr->d_scenes : nullptr));
  mark(tr, 1, capturing);
  bool in_tmp = false;
  SC_TRY(sck::radix_sort_segments(ctx, tr->dkeys, tr->ids, tr->dkeys_tmp, tr->ids_tmp, tr->stride, V, 16, tr->scratch,
                                  tr->scratch_bytes, &in_tmp));
  const uint32_t* sorted_ids = in_tmp ? tr->ids_tmp : tr->ids;
  mark(tr, 2, capturing);
  const uint32_t all_tiles = V * tr->T;
  const uint32_t* svals = nullptr;
  const uint32_t* item_keys = nullptr;
  const uint32_t* item_ids = nullptr;
  if (tr->two_level) {
    // items (member mask | view, super tile; splat) in depth order, grouped
    // per super tile by a stable sort; each tile then blends the items of its
    // super tile whose mask holds it
    const int cull = tr->cfg.tile_cull ? 1 : 0;
    uint64_t* d_items = tr->d_total + 1;
    // item counts in depth order (gathered through the sorted ids) -> offsets
    SC_TRY(sck::scan_u32_gather(ctx, tr->counts, nsp + 1, tr->counts_by_id, sorted_ids, tr->stride, nsp, d_items,
                                tr->scratch, tr->scratch_bytes));
    if (sizing) {
      uint64_t I = 0;
      SC_CUDA_TRY(ctx, cudaMemcpyAsync(&I, d_items, 8, cudaMemcpyDeviceToHost, ctx->stream), "items");
      SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
      SC_TRY(ensure_items(tr, I));
    }
    mark(tr, 3, capturing);
    SC_TRY(sck::launch_super_emit(ctx, tr->rec, tr->stride, V, sorted_ids, tr->counts, tr->counts_by_id,
                                  &tr->cfg.tiling, tr->ikeys, tr->ivals, tr->icap, ctx->d_error, cull));
    mark(tr, 4, capturing);
    SC_TRY(sck::radix_sort<uint32_t>(ctx, tr->ikeys, tr->ivals, tr->ikeys_tmp, tr->ivals_tmp, tr->icap, tr->super_bits,
                                     d_items, tr->scratch, tr->scratch_bytes, &in_tmp, (int)tr->cfg.sort_digit_bits));
    item_keys = in_tmp ? tr->ikeys_tmp : tr->ikeys;
    item_ids = in_tmp ? tr->ivals_tmp : tr->ivals;
    mark(tr, 5, capturing);
    // the super tiles' ranges; the member bits of the masks add up to the pair count
    SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->d_total, 0, 8, ctx->stream), "zero pairs");
    SC_TRY(sck::launch_tile_ranges(ctx, item_keys, 2, d_items, tr->icap, V * tr->ST, tr->iranges, tr->ST,
                                   tr->super_bits, tr->super_bits + bits_for(V - 1), tr->d_total));
  } else {
  SC_TRY(sck::scan_u32_gather(ctx, tr->counts, nsp + 1, tr->counts_by_id, sorted_ids, tr->stride, nsp, tr->d_total,
                              tr->scratch, tr->scratch_bytes));
  if (sizing) {
    uint64_t K = 0;
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(&K, tr->d_total, 8, cudaMemcpyDeviceToHost, ctx->stream), "K");
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    SC_TRY(ensure_pairs(tr, K));
  }
  mark(tr, 3, capturing);
  SC_TRY(sck::launch_presorted_emit(ctx, tr->rec, tr->stride, V, sorted_ids, tr->counts, tr->counts_by_id,
                                    &tr->cfg.tiling, tr->keys, tr->vals, tr->kcap, ctx->d_error,
                                    (int)tr->cfg.tile_cull));
  mark(tr, 4, capturing);
  // keys are (view << tile_bits) | tile: the stable sort on the tile bits alone
  // groups the pairs by tile, then view (the emission is view-major), then depth
  const uint32_t tile_bits = bits_for(tr->T);
  SC_TRY(sck::radix_sort<uint32_t>(ctx, tr->keys, tr->vals, tr->keys_tmp, tr->vals_tmp, tr->kcap, tile_bits,
                                   tr->d_total, tr->scratch, tr->scratch_bytes, &in_tmp, (int)tr->cfg.sort_digit_bits));
  const uint32_t* skeys = in_tmp ? tr->keys_tmp : tr->keys;
  svals = in_tmp ? tr->vals_tmp : tr->vals;
  mark(tr, 5, capturing);
  SC_TRY(sck::launch_tile_ranges(ctx, skeys, 2, tr->d_total, tr->kcap, all_tiles, tr->ranges, tr->T, tile_bits));
  }
  mark(tr, 6, capturing);
  const float weight = tr->grads_mode ? tr->loss_weight : 1.0f / (float)V;
  const float lam = tr->cfg.ssim_lambda;
  const float mse_w = lam > 0.0f ? weight * (1.0f - lam) : weight;
  // with the MSE alone, the backward forms dL/dC from the image, so the targets
  // are needed only from the backward on (a host upload overlaps the forward)
  const bool mse_in_bwd = lam == 0.0f;
  const float* fwd_target = mse_in_bwd ? nullptr : tr->targets;
  if (tr->h_targets && !mse_in_bwd)  // the copies run in order: the last view's event covers all
    SC_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, tr->ev_view[V - 1], 0), "join");
  if (tr->two_level)
    SC_TRY(sck::launch_composite_items(ctx, tr->rec, tr->stride, V, item_keys, item_ids, tr->iranges, &tr->cfg.tiling,
                                       tr->image, tr->aux, fwd_target, mse_w, tr->dl_dc, tr->d_loss, ctx->d_error,
                                       work_fwd, tr->cfg.blend_batch, scenes, tr->profiling >= 2));
  else
    SC_TRY(sck::launch_composite(ctx, tr->rec, tr->stride, V, svals, tr->ranges, &tr->cfg.tiling, tr->image, tr->aux,
                                 fwd_target, mse_w, tr->dl_dc, tr->d_loss, ctx->d_error));
  if (lam > 0.0f) {
    SC_CUDA_TRY(ctx, cudaMemsetAsync(tr->d_ssim, 0, 8 * (size_t)V, ctx->stream), "zero ssim");
    SC_TRY(sck::launch_ssim(ctx, tr->image, tr->targets, tr->cfg.tiling.width, tr->cfg.tiling.height, V,
                            weight * lam, tr->dl_dc, tr->d_ssim, tr->ssim_terms));
  }
  mark(tr, 7, capturing);
  const float* bwd_target = mse_in_bwd ? tr->targets : nullptr;
  // with host targets and the MSE formed here, one launch per view on its own
  // stream, each after the forward and its own view's copy: the backward of
  // the first views overlaps the upload of the last ones, and the views' tails
  // (tiles with long lists) overlap each other
  const bool per_view = tr->h_targets && mse_in_bwd;
  if (per_view) SC_CUDA_TRY(ctx, cudaEventRecord(tr->ev_fwd, ctx->stream), "forward done");
  for (uint32_t v0 = 0; v0 < V; v0 += per_view ? 1 : V) {
    const uint32_t nv = per_view ? 1 : V;
    cudaStream_t main_stream = ctx->stream;
    if (per_view) {
      SC_CUDA_TRY(ctx, cudaStreamWaitEvent(tr->bwd_stream[v0], tr->ev_fwd, 0), "fork");
      SC_CUDA_TRY(ctx, cudaStreamWaitEvent(tr->bwd_stream[v0], tr->ev_view[v0], 0), "copied");
      ctx->stream = tr->bwd_stream[v0];  // the launch helpers enqueue on the context's stream
    }
    const size_t so = (size_t)3 * v0 * tr->stride, po = (size_t)v0 * tr->P;
    const float* tg = bwd_target ? bwd_target + 3 * po : nullptr;
    sc_status st;
    if (tr->two_level)
      st = (sck::launch_composite_backward_items(ctx, tr->rec + so, tr->stride, nv, item_keys, item_ids,
                                                  tr->iranges + (size_t)2 * v0 * tr->ST, &tr->cfg.tiling,
                                                  tr->image + po, tr->dl_dc ? tr->dl_dc + po : nullptr,
                                                  (int)tr->cfg.bwd_mode, tr->aux + po,
                                                  tr->pgrad + so, ctx->d_error, tg, mse_w, tr->d_loss + v0, work_bwd,
                                                  tr->pcomp ? tr->pcomp + so : nullptr, tr->cfg.blend_batch,
                                                  scenes ? scenes + v0 : nullptr, tr->profiling >= 2));
    else
      st = (sck::launch_composite_backward(ctx, tr->rec + so, tr->stride, nv, svals, tr->ranges + (size_t)2 * v0 * tr->T,
                                            &tr->cfg.tiling, tr->image + po, tr->dl_dc ? tr->dl_dc + po : nullptr,
                                            (int)tr->cfg.bwd_mode,
                                            tr->aux + po, tr->pgrad + so, ctx->d_error, tg, mse_w, tr->d_loss + v0,
                                            tr->pcomp ? tr->pcomp + so : nullptr));
    ctx->stream = main_stream;
    SC_TRY(st);
    if (per_view) SC_CUDA_TRY(ctx, cudaEventRecord(tr->ev_bwd[v0], tr->bwd_stream[v0]), "view done");
  }
  if (per_view)
    for (uint32_t v = 0; v < V; ++v) SC_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, tr->ev_bwd[v], 0), "join");
  mark(tr, 8, capturing);
  sck::AdamParams ap;
  for (int k = 0; k < 6; ++k) ap.lr[k] = tr->cfg.adam.lr[k];
  ap.beta1 = tr->cfg.adam.beta1; ap.beta2 = tr->cfg.adam.beta2; ap.eps = tr->cfg.adam.eps;
  ap.bc1 = ap.bc2 = 1.0f;
  ap.log_scale_min = tr->cfg.log_scale_min; ap.log_scale_max = tr->cfg.log_scale_max;
  ap.opacity_logit_max = tr->cfg.opacity_logit_max;
  if (tr->scenes_mode) {
    // every scene's gradient rows from its own view, then every scene's Adam step
    SC_TRY(sck::launch_project_backward_scenes(ctx, tr->d_scenes, V, tr->scene_max_gstride, tr->pgrad, tr->stride,
                                               d_cams, ctx->d_error, tr->cfg.fp64_det ? 1 : 0, tr->pcomp));
    SC_TRY(sck::launch_adam_rows_scenes(ctx, tr->d_scenes, V, tr->scene_max_cap, ap, d_bc, ctx->d_error));
  } else if (tr->grads_mode)
    SC_TRY(sck::launch_project_backward_shards(ctx, ds, tr->pgrad, tr->stride, d_cams, V, tr->gout, tr->g_shards,
                                               tr->g_shard, ctx->d_error, tr->cfg.fp64_det ? 1 : 0, tr->pcomp));
  else {
    // per-splat gradient rows summed over the views, then Adam streamed over the rows
    SC_TRY(sck::launch_project_backward_shards(ctx, ds, tr->pgrad, tr->stride, d_cams, V, tr->grads, 1,
                                               tr->grad_stride, ctx->d_error, tr->cfg.fp64_det ? 1 : 0, tr->pcomp));
    SC_TRY(sck::launch_adam_rows(ctx, ds, dm, acc, tr->grads, 0, ds.n, tr->grad_stride, ap, d_bc, ctx->d_error));
  }
  mark(tr, 9, capturing);
  k_finalize<<<1, 1, 0, ctx->stream>>>(tr->d_loss, lam > 0.0f ? tr->d_ssim : nullptr, lam, V,
                                       1.0 / (3.0 * (double)tr->P), tr->grads_mode ? (double)tr->loss_weight : 0.0,
                                       tr->d_total, ctx->d_error, tr->d_out);
  SC_TRY(sc_check_launch(ctx, "k_finalize"));
  SC_CUDA_TRY(ctx, cudaMemcpyAsync(tr->h_out, tr->d_out, sizeof(StepOut), cudaMemcpyDeviceToHost, ctx->stream), "out D2H");
  if (tr->scenes_mode)
    SC_CUDA_TRY(ctx, cudaMemcpyAsync(tr->h_losses, tr->d_loss, 8 * (size_t)V, cudaMemcpyDeviceToHost, ctx->stream),
                "losses D2H");
  tr->kernels_per_step = (uint32_t)(ctx->launches - launches0);
  return SC_OK;
}

extern "C" {

sc_status sc_trainer_create(sc_ctx* ctx, const sc_train_config* cfg, sc_trainer** out) {
  if (!ctx || !cfg || !out) return SC_ERR_INVALID_ARG;
  if (cfg->n_views == 0 || cfg->n_views > SC_MAX_VIEWS) return sc_fail(ctx, SC_ERR_INVALID_ARG, "n_views out of range");
  const sc_tiling& t = cfg->tiling;
  if (!t.width || !t.height || !t.tile_w || !t.tile_h) return SC_ERR_INVALID_ARG;
  const uint32_t threads = t.tile_w * t.tile_h;
  if (threads > 256 || threads % 32) return sc_fail(ctx, SC_ERR_INVALID_ARG, "tile must hold 32..256 pixels, multiple of 32");
  if (cfg->bwd_mode != SC_BWD_REF && cfg->bwd_mode != SC_BWD_EXACT) return SC_ERR_INVALID_ARG;
  if (!(cfg->ssim_lambda >= 0.0f && cfg->ssim_lambda <= 1.0f))
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "ssim_lambda must lie in [0, 1]");
  if (cfg->ssim_lambda > 0.0f && (t.width < 6 || t.height < 6))
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "the SSIM loss needs images of at least 6x6 pixels");
  sc_trainer* tr = new sc_trainer();
  tr->ctx = ctx;
  tr->cfg = *cfg;
  tr->V = cfg->n_views;
  tr->tiles_x = (t.width + t.tile_w - 1) / t.tile_w;
  tr->tiles_y = (t.height + t.tile_h - 1) / t.tile_h;
  tr->T = tr->tiles_x * tr->tiles_y;
  if (bits_for(tr->T) + bits_for(tr->V - 1) > 32) {
    delete tr;
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "too many tiles x views for 32-bit pair keys");
  }
  // sort_mode 0 (auto) and 2: two-level binning; 1: depth presort + sort of the (tile, splat) pairs
  if (cfg->sort_mode > 2) {
    delete tr;
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "sort_mode must be 0, 1 or 2");
  }
  if (cfg->sort_digit_bits != 0 && cfg->sort_digit_bits != 8 && cfg->sort_digit_bits != 9) {
    delete tr;
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "sort_digit_bits must be 0, 8 or 9");
  }
  if (cfg->blend_batch != 0 && (cfg->blend_batch % 32 || cfg->blend_batch < 32)) {
    delete tr;
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "blend_batch must be 0 or a multiple of 32");
  }
  tr->ST = sck::super_tiles_per_view(&t);
  tr->super_bits = bits_for(tr->ST);
  // the item key holds view << super_bits | super tile in 16 bits, the member mask above
  tr->two_level = cfg->sort_mode != 1 && tr->super_bits + bits_for(tr->V - 1) <= 16;
  tr->P = (uint64_t)t.width * t.height;
  const size_t pix = (size_t)tr->V * tr->P;
  cudaError_t e = cudaMallocHost(&tr->h_params, sizeof(StepParams));
  if (e == cudaSuccess) e = cudaMallocHost(&tr->h_out, sizeof(StepOut));
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_params, sizeof(StepParams));
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_out, sizeof(StepOut));
  if (e == cudaSuccess) e = cudaMalloc(&tr->ranges, (size_t)tr->V * tr->T * 8);
  if (e == cudaSuccess) e = cudaMalloc(&tr->image, pix * 16);
  if (e == cudaSuccess) e = cudaMalloc(&tr->aux, pix * 8);
  if (e == cudaSuccess) e = cudaMalloc(&tr->dl_dc, pix * 16);
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_loss, 8 * (size_t)tr->V);
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_work, 6 * sck::BLEND_WORK_SLOTS * 8);
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_total, 64);
  if (e == cudaSuccess) e = cudaMemset(tr->d_total, 0, 64);
  if (e == cudaSuccess && tr->two_level) e = cudaMalloc(&tr->iranges, (size_t)tr->V * tr->ST * 8);
  if (e == cudaSuccess && cfg->ssim_lambda > 0.0f) e = cudaMalloc(&tr->ssim_terms, sck::ssim_terms_bytes(tr->P, tr->V));
  if (e == cudaSuccess && cfg->ssim_lambda > 0.0f) e = cudaMalloc(&tr->d_ssim, 8 * (size_t)tr->V);
  for (int i = 0; i <= kStages && e == cudaSuccess; ++i) e = cudaEventCreate(&tr->ev[i]);
  if (e != cudaSuccess) {
    sc_trainer_free(ctx, tr);
    return sc_cuda_fail(ctx, e, "trainer alloc");
  }
  std::memset(tr->h_params, 0, sizeof(StepParams));
  *out = tr;
  return SC_OK;
}

void sc_trainer_free(sc_ctx* ctx, sc_trainer* tr) {
  if (!tr) return;
  if (ctx) cudaStreamSynchronize(ctx->stream);
  trainer_drop_graph(tr);
  trainer_free_splat_arrays(tr);
  trainer_free_pairs(tr);
  trainer_free_items(tr);
  cudaFree(tr->iranges);
  cudaFree(tr->ranges); cudaFree(tr->image); cudaFree(tr->aux); cudaFree(tr->dl_dc);
  cudaFree(tr->d_loss); cudaFree(tr->d_work); cudaFree(tr->d_total); cudaFree(tr->d_params); cudaFree(tr->d_out);
  cudaFree(tr->ssim_terms); cudaFree(tr->d_ssim);
  cudaFree(tr->d_host_targets);
  if (tr->copy_stream) cudaStreamDestroy(tr->copy_stream);
  if (tr->ev_fork) cudaEventDestroy(tr->ev_fork);
  if (tr->ev_fwd) cudaEventDestroy(tr->ev_fwd);
  for (uint32_t v = 0; v < SC_MAX_VIEWS; ++v) {
    if (tr->ev_view[v]) cudaEventDestroy(tr->ev_view[v]);
    if (tr->ev_bwd[v]) cudaEventDestroy(tr->ev_bwd[v]);
    if (tr->bwd_stream[v]) cudaStreamDestroy(tr->bwd_stream[v]);
  }
  cudaFree(tr->scratch);
  for (uint32_t v = 0; v < SC_MAX_VIEWS; ++v) cudaFree(tr->scene[v].grads);
  cudaFree(tr->d_scenes);
  if (tr->h_scenes) cudaFreeHost(tr->h_scenes);
  if (tr->h_losses) cudaFreeHost(tr->h_losses);
  if (tr->h_params) cudaFreeHost(tr->h_params);
  if (tr->h_out) cudaFreeHost(tr->h_out);
  for (int i = 0; i <= kStages; ++i)
    if (tr->ev[i]) cudaEventDestroy(tr->ev[i]);
  delete tr;
}

sc_status sc_trainer_set_targets(sc_trainer* tr, const float* targets) {
  if (!tr || !targets) return SC_ERR_INVALID_ARG;
  if (tr->targets != targets || tr->h_targets) trainer_drop_graph(tr);
  tr->targets = targets;
  tr->h_targets = nullptr;
  return SC_OK;
}

sc_status sc_trainer_set_host_targets(sc_trainer* tr, const float* pinned_targets) {
  if (!tr || !pinned_targets) return SC_ERR_INVALID_ARG;
  sc_ctx* ctx = tr->ctx;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, pinned_targets) != cudaSuccess || at.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "host targets must be page-locked (cudaMallocHost / pinned) memory");
  }
  if (!tr->d_host_targets) {
    SC_CUDA_TRY(ctx, cudaMalloc(&tr->d_host_targets, (size_t)tr->V * tr->P * 3 * sizeof(float)), "targets");
    SC_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&tr->copy_stream, cudaStreamNonBlocking), "copy stream");
    SC_CUDA_TRY(ctx, cudaEventCreateWithFlags(&tr->ev_fork, cudaEventDisableTiming), "event");
    SC_CUDA_TRY(ctx, cudaEventCreateWithFlags(&tr->ev_fwd, cudaEventDisableTiming), "event");
    for (uint32_t v = 0; v < tr->V; ++v) {
      SC_CUDA_TRY(ctx, cudaEventCreateWithFlags(&tr->ev_view[v], cudaEventDisableTiming), "event");
      SC_CUDA_TRY(ctx, cudaEventCreateWithFlags(&tr->ev_bwd[v], cudaEventDisableTiming), "event");
      SC_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&tr->bwd_stream[v], cudaStreamNonBlocking), "stream");
    }
  }
  if (tr->h_targets != pinned_targets) trainer_drop_graph(tr);
  tr->h_targets = pinned_targets;
  tr->targets = tr->d_host_targets;
  return SC_OK;
}

sc_status sc_trainer_set_profiling(sc_trainer* tr, int enabled) {
  if (!tr) return SC_ERR_INVALID_ARG;
  const int level = enabled <= 0 ? 0 : (enabled >= 2 ? 2 : 1);
  if (tr->profiling != level) trainer_drop_graph(tr);
  tr->profiling = level;
  for (int i = 0; i < kStages; ++i) tr->acc_ms[i] = 0.0;
  for (int i = 0; i < 6; ++i) tr->work_acc[i] = 0;
  tr->prof_steps = 0;
  return SC_OK;
}

}  // extern "C"

// Run one step (full, or gradient-only per tr->grads_mode) with the step
// parameters already in pinned memory: graph capture/replay, capacity retry.
static sc_status run_step(sc_trainer* tr, sc_splats* s, sc_moments* mo, float* acc, double* loss_out) {
  sc_ctx* ctx = tr->ctx;
  // many scenes: the table (stores, counts, rows) is copied by the step's first
  // node, so the graph depends only on the capacities that size its grids
  SC_TRY(ensure_splat_arrays(tr, tr->scenes_mode ? tr->scene_max_cap : s->cap));
  for (int attempt = 0; attempt < 4; ++attempt) {
    const bool sizing = tr->kcap == 0 || (tr->two_level && tr->icap == 0);
    const void* mkey = mo ? (mo->m ? (const void*)mo->m : (const void*)mo->m16) : nullptr;
    const void* key[8] = {s ? s->slab : nullptr, s ? s->rest16 : nullptr, mkey, acc, tr->targets, tr->scratch,
                          tr->gout, tr->h_targets};
    const uint64_t key_n = s ? s->n : ((uint64_t)tr->scene_max_cap << 32 | tr->scene_max_gstride);
    const bool key_ok = tr->exec && std::equal(key, key + 8, tr->g_key) && tr->g_key_n == key_n &&
                        tr->g_key_kcap == tr->kcap && tr->g_key_icap == tr->icap && tr->g_key_grads == tr->grads_mode &&
                        tr->g_key_w == tr->loss_weight && tr->g_key_shards == tr->g_shards &&
                        tr->g_key_shard == tr->g_shard;
    if (!key_ok) trainer_drop_graph(tr);
    if (tr->cfg.use_graph && !sizing) {
      if (!tr->exec) {
        cudaGraph_t g = nullptr;
        SC_CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed), "begin capture");
        sc_status st = enqueue_step(tr, s, mo, acc, true, false);
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
        if (st != SC_OK) { if (g) cudaGraphDestroy(g); return st; }
        if (ce != cudaSuccess) return sc_cuda_fail(ctx, ce, "end capture");
        ce = cudaGraphInstantiate(&tr->exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { tr->exec = nullptr; return sc_cuda_fail(ctx, ce, "graph instantiate"); }
        std::copy(key, key + 8, tr->g_key);
        tr->g_key_n = key_n;
        tr->g_key_kcap = tr->kcap;
        tr->g_key_icap = tr->icap;
        tr->g_key_grads = tr->grads_mode;
        tr->g_key_w = tr->loss_weight;
        tr->g_key_shards = tr->g_shards;
        tr->g_key_shard = tr->g_shard;
      }
      SC_CUDA_TRY(ctx, cudaGraphLaunch(tr->exec, ctx->stream), "graph launch");
      ctx->launches += tr->kernels_per_step;
    } else {
      SC_TRY(enqueue_step(tr, s, mo, acc, false, sizing));
    }
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "step sync");
    const StepOut o = *tr->h_out;
    tr->last_pairs = o.pairs;
    tr->last_items = o.items;
    if (o.err & SC_DEVERR_TIMEOUT) {
      cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream);
      return sc_fail(ctx, SC_ERR_TIMEOUT, "a bounded device wait gave up during the step");
    }
    if (o.err & SC_DEVERR_CAPACITY) {
      // the blend and Adam kernels skipped this step; grow and run it again
      SC_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream), "clear error");
      SC_TRY(ensure_items(tr, o.items));
      SC_TRY(ensure_pairs(tr, o.pairs));
      continue;
    }
    if (tr->profiling) {
      for (int i = 0; i < kStages; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, tr->ev[i], tr->ev[i + 1]) == cudaSuccess) tr->acc_ms[i] += ms;
      }
      // per pass (forward, backward): BLEND_WORK_SLOTS (scanned, staged) pairs, then as many pixel-pair counts
      constexpr uint32_t S = sck::BLEND_WORK_SLOTS;
      uint64_t w[6 * S];
      SC_CUDA_TRY(ctx, cudaMemcpy(w, tr->d_work, sizeof(w), cudaMemcpyDeviceToHost), "work D2H");
      for (uint32_t k = 0; k < 2; ++k)
        for (uint32_t i = 0; i < S; ++i) {
          tr->work_acc[2 * k] += w[3 * S * k + 2 * i];
          tr->work_acc[2 * k + 1] += w[3 * S * k + 2 * i + 1];
          tr->work_acc[4 + k] += w[3 * S * k + 2 * S + i];
        }
      tr->prof_steps++;
    }
    if (loss_out) *loss_out = o.loss;
    return SC_OK;
  }
  return sc_fail(ctx, SC_ERR_CAPACITY, "pair capacity kept overflowing");
}

extern "C" {

sc_status sc_trainer_step(sc_trainer* tr, sc_splats* s, sc_moments* mo, float* acc, const sc_camera* cams, uint64_t t,
                          double* loss_out) {
  if (!tr || !s || !mo || !acc || !cams || t == 0) return SC_ERR_INVALID_ARG;
  if (!tr->targets) return sc_fail(tr->ctx, SC_ERR_INVALID_ARG, "trainer has no targets");
  if (mo->cap < s->n) return SC_ERR_INVALID_ARG;
  // step parameters into pinned memory (the graph's first node copies them)
  std::memcpy(tr->h_params->cams, cams, sizeof(sc_camera) * tr->V);
  tr->h_params->bc[0] = 1.0f - sc_powi_f32(tr->cfg.adam.beta1, (int)t);
  tr->h_params->bc[1] = 1.0f - sc_powi_f32(tr->cfg.adam.beta2, (int)t);
  const uint32_t seed = (uint32_t)t;  // the stochastic rounding's seed, read by the Adam kernel as bits
  std::memcpy(&tr->h_params->bc[2], &seed, sizeof(seed));
  tr->grads_mode = false;
  tr->loss_weight = 0.0f;
  tr->gout = nullptr;
  tr->g_shards = tr->g_shard = 0;
  return run_step(tr, s, mo, acc, loss_out);
}

sc_status sc_trainer_step_grads(sc_trainer* tr, sc_splats* s, const sc_camera* cams, float loss_weight,
                                uint32_t n_shards, uint32_t shard, float* grads, double* loss_out) {
  if (!tr || !s || !cams || !grads || !(loss_weight > 0.0f) || n_shards == 0 || shard == 0)
    return SC_ERR_INVALID_ARG;
  if (!tr->targets) return sc_fail(tr->ctx, SC_ERR_INVALID_ARG, "trainer has no targets");
  if ((uint64_t)n_shards * shard < s->n)
    return sc_fail(tr->ctx, SC_ERR_INVALID_ARG, "n_shards * shard must cover the splat count");
  std::memcpy(tr->h_params->cams, cams, sizeof(sc_camera) * tr->V);
  tr->h_params->bc[0] = tr->h_params->bc[1] = 1.0f;
  tr->grads_mode = true;
  tr->loss_weight = loss_weight;
  tr->gout = grads;
  tr->g_shards = n_shards;
  tr->g_shard = shard;
  return run_step(tr, s, nullptr, nullptr, loss_out);
}

sc_status sc_trainer_images(const sc_trainer* tr, const float** images) {
  if (!tr || !images) return SC_ERR_INVALID_ARG;
  *images = reinterpret_cast<const float*>(tr->image);
  return SC_OK;
}

sc_status sc_trainer_stats(const sc_trainer* tr, uint64_t* pairs, uint32_t* n_kernels, const char** names,
                           float* avg_ms, uint64_t* items) {
  if (!tr) return SC_ERR_INVALID_ARG;
  if (pairs) *pairs = tr->last_pairs;
  if (items) *items = tr->last_items;
  if (n_kernels) *n_kernels = tr->kernels_per_step;
  for (int i = 0; i < kStages; ++i) {
    if (names) names[i] = tr->two_level ? kStageNames2[i] : kStageNames[i];
    if (avg_ms) avg_ms[i] = tr->prof_steps ? (float)(tr->acc_ms[i] / (double)tr->prof_steps) : 0.0f;
  }
  return SC_OK;
}

sc_status sc_trainer_blend_work(const sc_trainer* tr, uint64_t out[4]) {
  if (!tr || !out) return SC_ERR_INVALID_ARG;
  for (int i = 0; i < 4; ++i) out[i] = tr->prof_steps ? tr->work_acc[i] / tr->prof_steps : 0;
  return SC_OK;
}

sc_status sc_trainer_blend_pairs(const sc_trainer* tr, uint64_t out[2]) {
  if (!tr || !out) return SC_ERR_INVALID_ARG;
  for (int i = 0; i < 2; ++i) out[i] = tr->prof_steps ? tr->work_acc[4 + i] / tr->prof_steps : 0;
  return SC_OK;
}

}  // extern "C"

// ================================================================ many scenes
struct sc_scenes_trainer {
  sc_trainer* tr = nullptr;
  uint32_t n = 0;
  bool set[SC_MAX_VIEWS] = {};
};

extern "C" {

sc_status sc_scenes_trainer_create(sc_ctx* ctx, const sc_scenes_config* cfg, sc_scenes_trainer** out) {
  if (!ctx || !cfg || !out) return SC_ERR_INVALID_ARG;
  if (cfg->n_scenes == 0 || cfg->n_scenes > SC_MAX_VIEWS) return sc_fail(ctx, SC_ERR_INVALID_ARG, "n_scenes out of range");
  sc_train_config tc{};
  tc.n_views = cfg->n_scenes;
  tc.tiling = cfg->tiling;
  tc.adam = cfg->adam;
  tc.bwd_mode = SC_BWD_EXACT;
  tc.use_graph = cfg->use_graph;
  tc.sort_mode = 2;
  tc.tile_cull = cfg->tile_cull;
  tc.log_scale_min = cfg->log_scale_min; tc.log_scale_max = cfg->log_scale_max;
  tc.opacity_logit_max = cfg->opacity_logit_max;
  tc.fp64_det = cfg->fp64_det;
  tc.compensated_sums = cfg->compensated_sums;
  sc_trainer* tr = nullptr;
  SC_TRY(sc_trainer_create(ctx, &tc, &tr));
  if (!tr->two_level) {
    sc_trainer_free(ctx, tr);
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "too many scenes x super tiles for the 16-bit item keys");
  }
  tr->scenes_mode = true;
  cudaError_t e = cudaMallocHost(&tr->h_scenes, sizeof(SceneDev) * cfg->n_scenes);
  if (e == cudaSuccess) e = cudaMallocHost(&tr->h_losses, 8 * (size_t)cfg->n_scenes);
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_scenes, sizeof(SceneDev) * cfg->n_scenes);
  if (e == cudaSuccess) e = cudaMalloc(&tr->d_host_targets, (size_t)tr->V * tr->P * 3 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(tr->d_host_targets, 0, (size_t)tr->V * tr->P * 3 * sizeof(float));
  if (e != cudaSuccess) {
    sc_trainer_free(ctx, tr);
    return sc_cuda_fail(ctx, e, "scenes trainer alloc");
  }
  std::memset(tr->h_scenes, 0, sizeof(SceneDev) * cfg->n_scenes);
  tr->targets = tr->d_host_targets;  // the scenes' targets, copied in at the tiling's row pitch
  sc_scenes_trainer* st = new sc_scenes_trainer();
  st->tr = tr;
  st->n = cfg->n_scenes;
  *out = st;
  return SC_OK;
}

void sc_scenes_trainer_free(sc_ctx* ctx, sc_scenes_trainer* st) {
  if (!st) return;
  sc_trainer_free(ctx, st->tr);
  delete st;
}

sc_status sc_scenes_trainer_set_scene(sc_scenes_trainer* st, uint32_t i, sc_splats* s, sc_moments* mo, float* grad_acc,
                                      uint32_t width, uint32_t height, const float* target) {
  if (!st || i >= st->n || !s || !mo || !grad_acc || !target) return SC_ERR_INVALID_ARG;
  sc_trainer* tr = st->tr;
  sc_ctx* ctx = tr->ctx;
  if (width == 0 || height == 0 || width > tr->cfg.tiling.width || height > tr->cfg.tiling.height)
    return sc_fail(ctx, SC_ERR_INVALID_ARG, "a scene's image must fit the trainer's tiling");
  if (mo->cap < s->cap) return sc_fail(ctx, SC_ERR_INVALID_ARG, "moments smaller than the scene's store");
  if (s->cap % 8 || mo->cap % 8) return sc_fail(ctx, SC_ERR_INVALID_ARG, "store capacities must be multiples of 8");
  auto& h = tr->scene[i];
  const uint32_t gstride = (s->cap + 63u) & ~63u;
  if (h.gstride != gstride) {
    SC_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    cudaFree(h.grads);
    h.grads = nullptr;
    SC_CUDA_TRY(ctx, cudaMalloc(&h.grads, (size_t)SC_NROWS * gstride * 4), "scene gradient rows");
    h.gstride = gstride;
  }
  h.s = s; h.mo = mo; h.acc = grad_acc; h.width = width; h.height = height;
  // the target at the tiling's row pitch (pixels outside the scene's image stay zero and unused)
  const size_t pitch = (size_t)tr->cfg.tiling.width * 3 * sizeof(float);
  SC_CUDA_TRY(ctx, cudaMemcpy2DAsync(tr->d_host_targets + (size_t)i * tr->P * 3, pitch, target,
                                     (size_t)width * 3 * sizeof(float), (size_t)width * 3 * sizeof(float), height,
                                     cudaMemcpyDeviceToDevice, ctx->stream), "scene target");
  st->set[i] = true;
  uint32_t mc = 0, mg = 0;
  for (uint32_t k = 0; k < st->n; ++k)
    if (st->set[k]) { mc = std::max(mc, tr->scene[k].s->cap); mg = std::max(mg, tr->scene[k].gstride); }
  if (mc != tr->scene_max_cap || mg != tr->scene_max_gstride) trainer_drop_graph(tr);
  tr->scene_max_cap = mc;
  tr->scene_max_gstride = mg;
  return SC_OK;
}

sc_status sc_scenes_trainer_step(sc_scenes_trainer* st, const sc_camera* cams, uint64_t t, double* losses) {
  if (!st || !cams || t == 0) return SC_ERR_INVALID_ARG;
  sc_trainer* tr = st->tr;
  for (uint32_t i = 0; i < st->n; ++i)
    if (!st->set[i]) return sc_fail(tr->ctx, SC_ERR_INVALID_ARG, "every scene needs sc_scenes_trainer_set_scene first");
  for (uint32_t i = 0; i < st->n; ++i) {
    const auto& h = tr->scene[i];
    if (h.s->cap > tr->scene_max_cap || h.gstride != ((h.s->cap + 63u) & ~63u))
      return sc_fail(tr->ctx, SC_ERR_INVALID_ARG, "a scene's store changed capacity: set the scene again");
    if ((uint32_t)cams[i].width != h.width || (uint32_t)cams[i].height != h.height)
      return sc_fail(tr->ctx, SC_ERR_INVALID_ARG, "a camera's image size differs from its scene's");
    SceneDev& d = tr->h_scenes[i];
    d.s = dview(h.s);
    d.mo = dview(h.mo);
    d.acc = h.acc;
    d.grads = h.grads;
    d.gstride = h.gstride;
    d.width = h.width;
    d.height = h.height;
    d.gscale = 2.0f / ((float)h.width * (float)h.height * 3.0f);  // loss.rs:163-179, one scene's own MSE
  }
  std::memcpy(tr->h_params->cams, cams, sizeof(sc_camera) * tr->V);
  tr->h_params->bc[0] = 1.0f - sc_powi_f32(tr->cfg.adam.beta1, (int)t);
  tr->h_params->bc[1] = 1.0f - sc_powi_f32(tr->cfg.adam.beta2, (int)t);
  const uint32_t seed = (uint32_t)t;
  std::memcpy(&tr->h_params->bc[2], &seed, sizeof(seed));
  tr->grads_mode = false;
  tr->loss_weight = 0.0f;
  tr->gout = nullptr;
  tr->g_shards = tr->g_shard = 0;
  SC_TRY(run_step(tr, nullptr, nullptr, nullptr, nullptr));
  if (losses)
    for (uint32_t i = 0; i < st->n; ++i)
      losses[i] = tr->h_losses[i] / (3.0 * (double)tr->scene[i].width * (double)tr->scene[i].height);
  return SC_OK;
}

sc_status sc_scenes_trainer_images(const sc_scenes_trainer* st, const float** images) {
  if (!st) return SC_ERR_INVALID_ARG;
  return sc_trainer_images(st->tr, images);
}

sc_status sc_scenes_trainer_stats(const sc_scenes_trainer* st, uint64_t* pairs, uint32_t* n_kernels, uint64_t* items) {
  if (!st) return SC_ERR_INVALID_ARG;
  return sc_trainer_stats(st->tr, pairs, n_kernels, nullptr, nullptr, items);
}

}  // extern "C"
