// Batched form (pimdal_group_batch_create, pimdal_hash_join_batch_create,
// pimdal_batch_run, pimdal_batch_autotune): plans of many independent
// operator instances.  The reference runs one operator instance per DPU
// launch (host loops over dpu_launch in pimdal/main/*/host); here a plan packs
// any number of instances into one persistent launch per phase, fed by a
// device work queue of (instance, row block) items in instance-major order.
//
// A plan is built once on the host: instance descriptors with their table
// regions, the work items and the scratch, all in one device allocation.
// pimdal_batch_run launches a fixed kernel sequence that reads nothing from
// the host (queue counters reset themselves, the hash join's look-back epoch
// advances on the device), so a run can be captured in a CUDA graph and the
// graph replayed.
#include <algorithm>
#include <vector>

#include "batch.cuh"

struct pimdal_batch {
  int kind = 0;
  int device = 0;
  uint32_t count = 0;
  void *mem = nullptr;
  size_t bytes = 0;
  pd_gb_batch gb{};
  pd_hj_batch hj{};
};

namespace {

struct Carve {  // sequential 256-byte aligned sub-allocations of one block
  size_t off = 0;
  size_t take(size_t n) {
    const size_t o = off;
    off += pd_align_up(std::max<size_t>(n, 1), 256);
    return o;
  }
};

uint32_t ceil_log2(uint64_t v) {
  uint32_t b = 0;
  while ((1ull << b) < v) ++b;
  return b;
}

int upload(void *dst, const void *src, size_t n) {
  if (!n) return PIMDAL_OK;
  return cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice) == cudaSuccess ? PIMDAL_OK : PIMDAL_ERR_CUDA;
}

int alloc_plan(pimdal_ctx *ctx, int kind, uint32_t count, size_t bytes, pimdal_batch **out) {
  auto *b = new (std::nothrow) pimdal_batch;
  if (!b) return PIMDAL_ERR_OOM;
  b->kind = kind;
  b->device = ctx->device;
  b->count = count;
  b->bytes = bytes;
  if (cudaMalloc(&b->mem, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return PIMDAL_ERR_OOM;
  }
  if (cudaMemset(b->mem, 0, std::min<size_t>(bytes, 512)) != cudaSuccess) {
    cudaFree(b->mem);
    delete b;
    return PIMDAL_ERR_CUDA;
  }
  *out = b;
  return PIMDAL_OK;
}

uint32_t item_rows(const pimdal_batch_tuning_t *t) {
  uint32_t r = (t && t->rows_per_item) ? t->rows_per_item : 65536u;
  return std::max<uint32_t>(128, r / 128 * 128);
}

uint32_t load_pct(const pimdal_batch_tuning_t *t) {
  return (t && t->load_factor_pct) ? t->load_factor_pct : 50u;
}

bool tuning_ok(const pimdal_batch_tuning_t *t) {
  if (!t) return true;
  if (t->load_factor_pct && (t->load_factor_pct < 10 || t->load_factor_pct > 90)) return false;
  if (t->rows_per_item && (t->rows_per_item < 128 || t->rows_per_item > (1u << 30))) return false;
  return true;
}

}  // namespace

extern "C" int pimdal_group_batch_create(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *args,
                                         uint32_t count, const pimdal_batch_tuning_t *tuning,
                                         pimdal_aggr_results_t *d_results, pimdal_batch_t **plan) {
  if (!ctx || !plan || (count && (!args || !d_results)) || !tuning_ok(tuning)) return PIMDAL_ERR_ARG;
  *plan = nullptr;
  cudaSetDevice(ctx->device);
  const uint32_t R = item_rows(tuning);
  const uint32_t lf = load_pct(tuning);
  std::vector<pd_gb_inst> inst(count);
  std::vector<uint2> items;
  std::vector<uint64_t> slot0(count + 1, 0);
  for (uint32_t i = 0; i < count; ++i) {
    const pimdal_aggr_arguments_t &a = args[i];
    if (a.key_dtype != PIMDAL_I32 && a.key_dtype != PIMDAL_U32) return PIMDAL_ERR_ARG;
    if (a.method != PIMDAL_GROUP_AUTO && a.method != PIMDAL_GROUP_HASH && a.method != PIMDAL_GROUP_SORT)
      return PIMDAL_ERR_ARG;
    if ((a.size && !a.in) || a.size >= (1ull << 30)) return PIMDAL_ERR_ARG;
    pd_gb_inst &g = inst[i];
    g.key = (const uint32_t *)a.in;
    g.val = a.in_val;
    g.n = a.size;
    g.out_key = (uint32_t *)a.out;
    g.out_sum = a.out_sum;
    g.out_count = a.out_count;
    g.out_min = a.out_min;
    g.out_max = a.out_max;
    g.out_cap = a.out_capacity;
    g.d_count = &d_results[i].t_count;
    g.flip = a.key_dtype == PIMDAL_I32 ? 0x80000000u : 0u;
    const uint64_t expect = std::max<uint64_t>(
        1, a.expected_groups ? a.expected_groups : std::min<uint64_t>(a.size, 1ull << 22));
    pd_gb_mode(expect, &g.mode, &g.wrep);
    const uint64_t slots = std::max<uint64_t>(256, pd_ceil_div(expect * 100, lf));
    if (slots >= (1ull << 31)) return PIMDAL_ERR_ARG;
    g.slots = (uint32_t)slots;
    g.slot0 = slot0[i];
    slot0[i + 1] = slot0[i] + slots;
    for (uint64_t r = 0; r < a.size; r += R) items.push_back(make_uint2(i, (uint32_t)r));
  }
  const uint64_t total = slot0[count];
  if (total >= (1ull << 32) || items.size() >= (1ull << 32)) return PIMDAL_ERR_ARG;
  pimdal_sort_arguments_t sa{};
  sa.nr_elements = std::max<uint64_t>(total, 1);
  size_t sort_ws = 0;
  if (pimdal_sort_workspace_size(&sa, &sort_ws)) return PIMDAL_ERR_ARG;
  Carve c;  // control words first: alloc_plan zeroes the start of the block
  const size_t o_ctr = c.take(256);
  const size_t o_ngroups = c.take(256);
  const size_t o_inst = c.take(sizeof(pd_gb_inst) * count);
  const size_t o_items = c.take(sizeof(uint2) * items.size());
  const size_t o_slot0 = c.take(8ull * (count + 1));
  const size_t o_igroups = c.take(4ull * count);
  const size_t o_istart = c.take(8ull * count);
  const size_t o_gtab = c.take(32 * total);
  size_t o_buf[6];
  for (auto &o : o_buf) o = c.take(4 * total);
  const size_t o_sort = c.take(sort_ws);
  pimdal_batch *b;
  int st = alloc_plan(ctx, PIMDAL_BATCH_GROUP, count, c.off, &b);
  if (st) return st;
  char *m = (char *)b->mem;
  pd_gb_batch &d = b->gb;
  d.inst = (const pd_gb_inst *)(m + o_inst);
  d.count = count;
  d.items = (const uint2 *)(m + o_items);
  d.nitems = (uint32_t)items.size();
  d.rows_per_item = R;
  d.gtab = (unsigned long long *)(m + o_gtab);
  d.total_slots = total;
  d.slot0 = (const uint64_t *)(m + o_slot0);
  d.counters = (uint32_t *)(m + o_ctr);
  d.ngroups = (unsigned long long *)(m + o_ngroups);
  d.inst_groups = (uint32_t *)(m + o_igroups);
  d.inst_start = (uint64_t *)(m + o_istart);
  uint32_t **bufs[6] = {&d.ckey, &d.cslot, &d.skey, &d.sslot, &d.ikey, &d.islot};
  for (int k = 0; k < 6; ++k) *bufs[k] = (uint32_t *)(m + o_buf[k]);
  d.sort_ws = m + o_sort;
  d.inst_bits = std::max<uint32_t>(1, ceil_log2(count));
  d.d_error = ctx->d_error;
  if ((st = upload(m + o_inst, inst.data(), sizeof(pd_gb_inst) * count)) ||
      (st = upload(m + o_items, items.data(), sizeof(uint2) * items.size())) ||
      (st = upload(m + o_slot0, slot0.data(), 8ull * (count + 1)))) {
    pimdal_batch_destroy(b);
    return st;
  }
  *plan = b;
  return PIMDAL_OK;
}

extern "C" int pimdal_hash_join_batch_create(pimdal_ctx_t *ctx,
                                             const pimdal_hash_join_arguments_t *args,
                                             uint32_t count, const pimdal_batch_tuning_t *tuning,
                                             pimdal_merge_results_t *d_results,
                                             pimdal_batch_t **plan) {
  if (!ctx || !plan || (count && (!args || !d_results)) || !tuning_ok(tuning)) return PIMDAL_ERR_ARG;
  *plan = nullptr;
  cudaSetDevice(ctx->device);
  const uint32_t R = item_rows(tuning);
  const uint32_t lf = load_pct(tuning);
  const uint32_t T = pd_hj_tile_rows();
  std::vector<pd_hj_inst> inst(count);
  std::vector<uint2> bitems;
  std::vector<uint64_t> tile0(count + 1, 0);
  uint64_t words = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const pimdal_hash_join_arguments_t &a = args[i];
    if ((a.size_build && !a.build_key) || (a.size_probe && !a.probe_key)) return PIMDAL_ERR_ARG;
    if (a.out_capacity && (!a.out_build_payload || !a.out_probe_ptr)) return PIMDAL_ERR_ARG;
    if (a.size_build >= (1ull << 31) || a.size_probe >= (1ull << 30)) return PIMDAL_ERR_ARG;
    pd_hj_inst &h = inst[i];
    h.bkey = (const uint32_t *)a.build_key;
    h.bpay = a.build_payload;
    h.nb = a.size_build;
    h.pkey = (const uint32_t *)a.probe_key;
    h.prow = a.probe_ptr;
    // an instance without build rows has no matches: it probes nothing
    h.np = a.size_build ? a.size_probe : 0;
    h.out_pay = a.out_build_payload;
    h.out_row = a.out_probe_ptr;
    h.cap = a.out_capacity;
    h.d_count = &d_results[i].t_count;
    h.bits = pd_hj_table_bits(a.size_build, lf);
    if (h.bits > 32) return PIMDAL_ERR_ARG;  // at most 2^32 slots per table
    h.tile0 = tile0[i];
    tile0[i + 1] = tile0[i] + pd_ceil_div(h.np, T);
    words += 1ull << h.bits;
    for (uint64_t r = 0; r < a.size_build; r += R) bitems.push_back(make_uint2(i, (uint32_t)r));
  }
  if (bitems.size() >= (1ull << 32)) return PIMDAL_ERR_ARG;
  Carve c;  // control words first: alloc_plan zeroes the start of the block
  const size_t o_ctr = c.take(256);
  const size_t o_epoch = c.take(256);
  const size_t o_inst = c.take(sizeof(pd_hj_inst) * count);
  const size_t o_tile0 = c.take(8ull * (count + 1));
  const size_t o_items = c.take(sizeof(uint2) * bitems.size());
  const size_t o_head = c.take(32ull * count);
  const size_t o_status = c.take(8 * tile0[count]);
  const size_t o_tab = c.take(8 * words);
  pimdal_batch *b;
  int st = alloc_plan(ctx, PIMDAL_BATCH_HASH_JOIN, count, c.off, &b);
  if (st) return st;
  char *m = (char *)b->mem;
  if (cudaMemset(m + o_status, 0, 8 * tile0[count]) != cudaSuccess) {
    pimdal_batch_destroy(b);
    return PIMDAL_ERR_CUDA;
  }
  uint64_t w = 0;
  for (uint32_t i = 0; i < count; ++i) {
    inst[i].table = (unsigned long long *)(m + o_tab) + w;
    inst[i].header = (uint32_t *)(m + o_head) + 8ull * i;
    w += 1ull << inst[i].bits;
  }
  pd_hj_batch &d = b->hj;
  d.inst = (const pd_hj_inst *)(m + o_inst);
  d.count = count;
  d.tile0 = (const uint64_t *)(m + o_tile0);
  d.total_tiles = tile0[count];
  d.bitems = (const uint2 *)(m + o_items);
  d.nbitems = (uint32_t)bitems.size();
  d.build_rows_per_item = R;
  d.tables = (unsigned long long *)(m + o_tab);
  d.table_words = words;
  d.headers = (uint32_t *)(m + o_head);
  d.status = (uint64_t *)(m + o_status);
  d.epoch = (uint32_t *)(m + o_epoch);
  d.counters = (uint32_t *)(m + o_ctr);
  d.d_error = ctx->d_error;
  if ((st = upload(m + o_inst, inst.data(), sizeof(pd_hj_inst) * count)) ||
      (st = upload(m + o_tile0, tile0.data(), 8ull * (count + 1))) ||
      (st = upload(m + o_items, bitems.data(), sizeof(uint2) * bitems.size()))) {
    pimdal_batch_destroy(b);
    return st;
  }
  *plan = b;
  return PIMDAL_OK;
}

extern "C" int pimdal_batch_run(pimdal_ctx_t *ctx, pimdal_batch_t *plan, pimdal_stream_t stream) {
  if (!ctx || !plan || plan->device != ctx->device) return PIMDAL_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (plan->count == 0) return PIMDAL_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return plan->kind == PIMDAL_BATCH_GROUP ? pd_gb_batch_run(ctx, plan->gb, s)
                                          : pd_hj_batch_run(ctx, plan->hj, s);
}

extern "C" int pimdal_batch_device_bytes(const pimdal_batch_t *plan, size_t *bytes) {
  if (!plan || !bytes) return PIMDAL_ERR_ARG;
  *bytes = plan->bytes;
  return PIMDAL_OK;
}

extern "C" int pimdal_batch_destroy(pimdal_batch_t *plan) {
  if (!plan) return PIMDAL_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaSetDevice(plan->device);
  cudaDeviceSynchronize();
  cudaFree(plan->mem);
  cudaSetDevice(dev);
  delete plan;
  return PIMDAL_OK;
}

namespace {

// Shape of a batch for the tuning cache: kind, count, total and largest row
// counts and expected groups, and the instances' log2 size histogram.
std::vector<uint64_t> batch_shape(int kind, const void *args, uint32_t count) {
  std::vector<uint64_t> k{(uint64_t)kind, count, 0, 0, 0, 0};
  k.resize(6 + 32, 0);
  for (uint32_t i = 0; i < count; ++i) {
    uint64_t rows, groups;
    if (kind == PIMDAL_BATCH_GROUP) {
      const auto &a = ((const pimdal_aggr_arguments_t *)args)[i];
      rows = a.size;
      groups = a.expected_groups;
    } else {
      const auto &a = ((const pimdal_hash_join_arguments_t *)args)[i];
      rows = a.size_probe;
      groups = a.size_build;
    }
    k[2] += rows;
    k[3] = std::max(k[3], rows);
    k[4] += groups;
    k[5] = std::max(k[5], groups);
    ++k[6 + std::min<uint32_t>(31, ceil_log2(rows + 1))];
  }
  return k;
}

}  // namespace

extern "C" int pimdal_batch_autotune(pimdal_ctx_t *ctx, int kind, const void *args, uint32_t count,
                                     void *d_results, pimdal_batch_tuning_t *best, int *cached,
                                     pimdal_stream_t stream) {
  if (!ctx || !best || (count && (!args || !d_results))) return PIMDAL_ERR_ARG;
  if (kind != PIMDAL_BATCH_GROUP && kind != PIMDAL_BATCH_HASH_JOIN) return PIMDAL_ERR_ARG;
  const std::vector<uint64_t> shape = batch_shape(kind, args, count);
  auto hit = ctx->tune_cache.find(shape);
  if (hit != ctx->tune_cache.end()) {
    *best = hit->second;
    if (cached) *cached = 1;
    return PIMDAL_OK;
  }
  if (cached) *cached = 0;
  cudaSetDevice(ctx->device);
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t rows_c[] = {16384, 65536, 262144};
  const uint32_t load_c[] = {35, 50, 70};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return PIMDAL_ERR_CUDA;
  float best_ms = -1.f;
  int st = PIMDAL_OK;
  for (uint32_t r : rows_c) {
    for (uint32_t lf : load_c) {
      pimdal_batch_tuning_t t{};
      t.rows_per_item = r;
      t.load_factor_pct = lf;
      pimdal_batch_t *plan = nullptr;
      st = kind == PIMDAL_BATCH_GROUP
               ? pimdal_group_batch_create(ctx, (const pimdal_aggr_arguments_t *)args, count, &t,
                                           (pimdal_aggr_results_t *)d_results, &plan)
               : pimdal_hash_join_batch_create(ctx, (const pimdal_hash_join_arguments_t *)args, count,
                                               &t, (pimdal_merge_results_t *)d_results, &plan);
      if (st == PIMDAL_ERR_OOM) continue;  // a candidate that does not fit is skipped
      if (st) break;
      float ms = 0.f;
      st = pimdal_batch_run(ctx, plan, stream);  // warm-up
      if (!st) {
        cudaEventRecord(e0, s);
        st = pimdal_batch_run(ctx, plan, stream);
        cudaEventRecord(e1, s);
      }
      if (!st) st = pimdal_ctx_sync_status(ctx, stream);
      if (!st) cudaEventElapsedTime(&ms, e0, e1);
      pimdal_batch_destroy(plan);
      if (st) break;
      if (best_ms < 0.f || ms < best_ms) {
        best_ms = ms;
        *best = t;
      }
    }
    if (st) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  if (best_ms < 0.f) return PIMDAL_ERR_OOM;
  ctx->tune_cache[shape] = *best;
  return PIMDAL_OK;
}
