// K-HGB / K-SGB: hash and sort group-by with exact int64 SUM / COUNT / MIN / MAX
// (pimdal_group_kernel).
//
// Reference behaviour: group_kernel of pimdal/aggregate/aggregate_hash.c:123-194
// inserts key_ptr pairs into a shared WRAM table of AGG_TABLE_SIZE slots under
// a mutex pool (hash_insert :43-82), spills rows whose bucket is full and
// re-aggregates them in later rounds; group_kernel of
// pimdal/aggregate/aggregate.c:82-158 run-length-aggregates sorted pairs.  The
// aggregation function is a function pointer (aggregate.h:11); the host then
// merges per-DPU partials and orders by key (host_aggregate_sync.cpp:71-95).
// The CPU operator reference/db_operators/aggregate.cpp:40-83 aggregates into
// thread-local absl::flat_hash_maps merged under omp critical.
//
// This operator returns, ordered by key, every group's key and any of SUM,
// COUNT, MIN, MAX of int64 values (all exact, int64 wrap-around sums).
//
// B200 design, hash method:
//  1. persistent CTAs aggregate their rows into a 2048-group shared-memory
//     table (64-bit atomicCAS on the tagged key, 64-bit shared atomics on the
//     aggregates); a row whose group finds no slot within 16 probes goes to
//     the global table directly; at the end each CTA merges its table into
//     the global one (64-bit global atomics);
//  2. the occupied global slots are compacted, sorted by key with K-SORT
//     (element count read on the device) and gathered into the outputs.
// Sort method: K-SORT of (key, row id), then a reduce-by-key over the sorted
// rows (see k_gb_segreduce).
#include <algorithm>

#include "common.cuh"

namespace {

constexpr int GB_THREADS = 512;
constexpr uint32_t GB_SMEM_SLOTS = 2048;
constexpr uint32_t GB_SMEM_PROBES = 16;
constexpr unsigned long long GB_TAG = 1ull << 32;  // occupied marker above the key

struct GbParams {
  const uint32_t *key;
  const int64_t *val;  // NULL: every value is 1
  uint64_t n;
  // global table (capacity 2^bits)
  unsigned long long *gkey;
  long long *gsum;
  unsigned long long *gcnt;
  long long *gmin, *gmax;
  uint32_t bits;
  unsigned long long *ngroups;  // compacted group count (device)
  uint32_t *ckey, *cslot;
  uint32_t *d_error;
};

__device__ __forceinline__ uint32_t gb_hash(uint32_t key, uint32_t bits) {
  return (uint32_t)(((uint64_t)key * PD_GOLDEN64) >> (64 - bits));
}

__global__ void __launch_bounds__(256) k_gb_init(GbParams p) {
  const uint64_t cap = 1ull << p.bits;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += stride) {
    p.gkey[i] = 0;
    p.gsum[i] = 0;
    p.gcnt[i] = 0;
    p.gmin[i] = INT64_MAX;
    p.gmax[i] = INT64_MIN;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *p.ngroups = 0;
}

__device__ __forceinline__ void global_add(const GbParams &p, uint32_t key, long long sum,
                                           unsigned long long cnt, long long mn, long long mx) {
  const uint64_t mask = (1ull << p.bits) - 1;
  const unsigned long long tagged = GB_TAG | key;
  uint64_t s = gb_hash(key, p.bits);
  for (uint64_t t = 0; t <= mask; ++t) {
    unsigned long long cur = p.gkey[s];
    if (cur == 0) cur = atomicCAS(p.gkey + s, 0ull, tagged);
    if (cur == 0 || cur == tagged) {
      atomicAdd((unsigned long long *)(p.gsum + s), (unsigned long long)sum);
      atomicAdd(p.gcnt + s, cnt);
      atomicMin(p.gmin + s, mn);
      atomicMax(p.gmax + s, mx);
      return;
    }
    s = (s + 1) & mask;
  }
  atomicOr(p.d_error, PD_DEVERR_TABLE_FULL);
}

constexpr size_t GB_SMEM_BYTES = 40ull * GB_SMEM_SLOTS;

__global__ void __launch_bounds__(GB_THREADS) k_gb_aggregate(GbParams p) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  unsigned long long *s_key = reinterpret_cast<unsigned long long *>(gb_smem);
  long long *s_sum = reinterpret_cast<long long *>(s_key + GB_SMEM_SLOTS);
  unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(s_sum + GB_SMEM_SLOTS);
  long long *s_min = reinterpret_cast<long long *>(s_cnt + GB_SMEM_SLOTS);
  long long *s_max = s_min + GB_SMEM_SLOTS;
  for (uint32_t i = threadIdx.x; i < GB_SMEM_SLOTS; i += GB_THREADS) {
    s_key[i] = 0;
    s_sum[i] = 0;
    s_cnt[i] = 0;
    s_min[i] = INT64_MAX;
    s_max[i] = INT64_MIN;
  }
  __syncthreads();
  constexpr uint32_t SBITS = 11;  // log2(GB_SMEM_SLOTS)
  const uint64_t stride = (uint64_t)gridDim.x * GB_THREADS;
  for (uint64_t i = (uint64_t)blockIdx.x * GB_THREADS + threadIdx.x; i < p.n; i += stride) {
    const uint32_t k = __ldcs(p.key + i);
    const long long v = p.val ? (long long)__ldcs(p.val + i) : 1ll;
    const unsigned long long tagged = GB_TAG | k;
    uint32_t s = gb_hash(k, SBITS);
    bool done = false;
    for (uint32_t t = 0; t < GB_SMEM_PROBES; ++t) {
      unsigned long long cur = s_key[s];
      if (cur == 0) cur = atomicCAS(s_key + s, 0ull, tagged);
      if (cur == 0 || cur == tagged) {
        atomicAdd((unsigned long long *)(s_sum + s), (unsigned long long)v);
        atomicAdd(s_cnt + s, 1ull);
        atomicMin(s_min + s, v);
        atomicMax(s_max + s, v);
        done = true;
        break;
      }
      s = (s + 1) & (GB_SMEM_SLOTS - 1);
    }
    if (!done) global_add(p, k, v, 1ull, v, v);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < GB_SMEM_SLOTS; i += GB_THREADS) {
    if (s_key[i])
      global_add(p, (uint32_t)s_key[i], s_sum[i], s_cnt[i], s_min[i], s_max[i]);
  }
}

// Occupied slots -> (key, slot) list (order is restored by the sort that follows).
__global__ void __launch_bounds__(256) k_gb_compact(GbParams p) {
  const uint64_t cap = 1ull << p.bits;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < cap; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const unsigned long long k = i < cap ? p.gkey[i] : 0ull;
    const unsigned m = __ballot_sync(0xffffffffu, k != 0);
    if (!m) continue;
    uint32_t pos = 0;
    if (lane == 0) pos = (uint32_t)atomicAdd(p.ngroups, (unsigned long long)__popc(m));
    pos = __shfl_sync(0xffffffffu, pos, 0) + __popc(m & ((1u << lane) - 1u));
    if (k) {
      p.ckey[pos] = (uint32_t)k;
      p.cslot[pos] = (uint32_t)i;
    }
  }
}

struct GatherParams {
  const uint32_t *skey, *sslot;
  const unsigned long long *ngroups;
  const long long *gsum, *gmin, *gmax;
  const unsigned long long *gcnt;
  uint32_t *out_key;
  int64_t *out_sum, *out_count, *out_min, *out_max;
  uint64_t cap;
  uint64_t *d_count;
  uint32_t *d_error;
};

__global__ void __launch_bounds__(256) k_gb_gather(GatherParams g) {
  const uint64_t n = *g.ngroups;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *g.d_count = n;
    if (n > g.cap) atomicOr(g.d_error, PD_DEVERR_CAPACITY);
  }
  const uint64_t lim = min(n, g.cap);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += stride) {
    const uint32_t s = g.sslot[i];
    if (g.out_key) g.out_key[i] = g.skey[i];
    if (g.out_sum) g.out_sum[i] = g.gsum[s];
    if (g.out_count) g.out_count[i] = (int64_t)g.gcnt[s];
    if (g.out_min) g.out_min[i] = g.gmin[s];
    if (g.out_max) g.out_max[i] = g.gmax[s];
  }
}

// ---------------------------------------------------------------------------
// Sort method: reduce-by-key over (sorted key, row id), values gathered by
// row id.  Tiles of 4096 sorted rows; a thread owns 16 consecutive rows.
//  1. k_sr_heads: group heads per tile;
//  2. k_sr_scan (one block): exclusive head prefix per tile, group count G;
//  3. k_sr_init: outputs 0..G-1 set to the aggregate identities;
//  4. k_gb_segreduce: a group inside one thread's rows is stored directly; a
//     group cut by a thread boundary is merged with 64-bit global atomics.
// ---------------------------------------------------------------------------
constexpr int SR_THREADS = 256;
constexpr int SR_ITEMS = 16;
constexpr int SR_TILE = SR_THREADS * SR_ITEMS;

struct SegParams {
  const uint32_t *skey, *sidx;
  const int64_t *val;
  uint64_t n;
  uint32_t *out_key;
  long long *out_sum, *out_min, *out_max;
  unsigned long long *out_cnt;
  uint64_t cap;
  uint64_t *tile_heads;  // per tile: heads, then the exclusive prefix
  uint64_t tiles;
  uint32_t *d_error;
  uint64_t *d_count;     // G
};

__device__ __forceinline__ bool sr_head(const SegParams &p, uint64_t i) {
  return i < p.n && (i == 0 || p.skey[i] != p.skey[i - 1]);
}

__global__ void __launch_bounds__(SR_THREADS) k_sr_heads(SegParams p) {
  __shared__ uint32_t s_red[SR_THREADS / 32];
  const uint64_t r0 = (uint64_t)blockIdx.x * SR_TILE + threadIdx.x;
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < SR_ITEMS; ++j) c += sr_head(p, r0 + (uint64_t)j * SR_THREADS);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < SR_THREADS / 32; ++w) t += s_red[w];
    p.tile_heads[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(1024) k_sr_scan(SegParams p) {
  __shared__ uint64_t s_w[32];
  __shared__ uint64_t s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (uint64_t base = 0; base < p.tiles; base += 1024) {
    const uint64_t i = base + tid;
    const uint64_t v = i < p.tiles ? p.tile_heads[i] : 0;
    uint64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    uint64_t pre = 0, tot = 0;
    for (int w = 0; w < 32; ++w) {
      if (w < warp) pre += s_w[w];
      tot += s_w[w];
    }
    if (i < p.tiles) p.tile_heads[i] = s_carry + pre + inc - v;
    __syncthreads();
    if (tid == 0) s_carry += tot;
    __syncthreads();
  }
  if (tid == 0) {
    *p.d_count = s_carry;
    if (s_carry > p.cap) atomicOr(p.d_error, PD_DEVERR_CAPACITY);
  }
}

__global__ void __launch_bounds__(256) k_sr_init(SegParams p) {
  const uint64_t lim = min(*p.d_count, p.cap);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += stride) {
    if (p.out_sum) p.out_sum[i] = 0;
    if (p.out_cnt) p.out_cnt[i] = 0;
    if (p.out_min) p.out_min[i] = INT64_MAX;
    if (p.out_max) p.out_max[i] = INT64_MIN;
  }
}

__device__ __forceinline__ void sr_flush(const SegParams &p, uint64_t g, uint32_t key, bool whole,
                                         long long sum, unsigned long long cnt, long long mn,
                                         long long mx) {
  if (g >= p.cap) return;  // reported by k_sr_scan
  if (whole) {
    if (p.out_key) p.out_key[g] = key;
    if (p.out_sum) p.out_sum[g] = sum;
    if (p.out_cnt) p.out_cnt[g] = cnt;
    if (p.out_min) p.out_min[g] = mn;
    if (p.out_max) p.out_max[g] = mx;
  } else {
    if (p.out_key) p.out_key[g] = key;  // every writer stores the same key
    if (p.out_sum) atomicAdd((unsigned long long *)(p.out_sum + g), (unsigned long long)sum);
    if (p.out_cnt) atomicAdd(p.out_cnt + g, cnt);
    if (p.out_min) atomicMin(p.out_min + g, mn);
    if (p.out_max) atomicMax(p.out_max + g, mx);
  }
}

__global__ void __launch_bounds__(SR_THREADS) k_gb_segreduce(SegParams p) {
  __shared__ uint32_t s_warp[SR_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t tile = blockIdx.x;
  const uint64_t r0 = tile * SR_TILE + (uint64_t)tid * SR_ITEMS;
  uint32_t key[SR_ITEMS];
  uint32_t heads = 0, nh = 0;
  const uint32_t before = (r0 > 0 && r0 - 1 < p.n) ? p.skey[r0 - 1] : 0u;
#pragma unroll
  for (int j = 0; j < SR_ITEMS; ++j) {
    key[j] = (r0 + j < p.n) ? p.skey[r0 + j] : 0u;
    const uint32_t prev = j ? key[j - 1] : before;
    const bool h = (r0 + j < p.n) && (r0 + j == 0 || key[j] != prev);
    heads |= (uint32_t)h << j;
    nh += h;
  }
  uint32_t inc = nh;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  uint32_t wpre = 0;
#pragma unroll
  for (int w = 0; w < SR_THREADS / 32; ++w)
    if (w < warp) wpre += s_warp[w];
  // heads strictly before this thread's first row
  uint64_t g = p.tile_heads[tile] + wpre + inc - nh;
  bool open_whole = false;  // the current segment began at a head in this thread
  long long sum = 0, mn = INT64_MAX, mx = INT64_MIN;
  unsigned long long cnt = 0;
  bool have = false;
  uint32_t cur_key = 0;
  uint64_t cur_g = 0;
#pragma unroll
  for (int j = 0; j < SR_ITEMS; ++j) {
    if (r0 + j >= p.n) break;
    if ((heads >> j) & 1u) {
      if (have) sr_flush(p, cur_g, cur_key, open_whole, sum, cnt, mn, mx);
      cur_g = g;
      ++g;
      cur_key = key[j];
      open_whole = true;
      sum = 0; cnt = 0; mn = INT64_MAX; mx = INT64_MIN;
      have = true;
    } else if (!have) {
      cur_g = g - 1;  // continues the group of the previous rows
      cur_key = key[j];
      open_whole = false;
      have = true;
    }
    const long long v = p.val ? (long long)p.val[p.sidx[r0 + j]] : 1ll;
    sum = (long long)((unsigned long long)sum + (unsigned long long)v);
    ++cnt;
    mn = min(mn, v);
    mx = max(mx, v);
  }
  if (have) {
    // the last segment is whole only if the next row starts a new group
    const uint64_t nx = r0 + SR_ITEMS;
    const bool ends = nx >= p.n || p.skey[nx] != cur_key;
    sr_flush(p, cur_g, cur_key, open_whole && ends, sum, cnt, mn, mx);
  }
}

struct GbLayout {
  uint32_t bits;
  size_t gkey, gsum, gcnt, gmin, gmax, ngroups, ckey, cslot, skey, sslot, sort_ws, total;
};

bool gb_layout(const pimdal_aggr_arguments_t *a, GbLayout *l) {
  const bool sort = a->method == PIMDAL_GROUP_SORT;
  size_t o = 0;
  pimdal_sort_arguments_t sa{};
  size_t w = 0;
  if (sort) {
    sa.nr_elements = a->size;
    if (pimdal_sort_workspace_size(&sa, &w)) return false;
    l->bits = 0;
    l->ngroups = o; o += pd_align_up(8 * (pd_ceil_div(a->size, SR_TILE) + 1), 256);
    l->skey = o; o += pd_align_up(4 * a->size, 256);
    l->sslot = o; o += pd_align_up(4 * a->size, 256);
    l->sort_ws = o; o += w;
    l->total = o;
    return true;
  }
  uint64_t expect = a->expected_groups ? a->expected_groups : std::min<uint64_t>(a->size, 1ull << 22);
  uint64_t cap = 2048;
  while (cap < 2 * expect) cap <<= 1;
  uint32_t bits = 0;
  while ((1ull << bits) < cap) ++bits;
  l->bits = bits;
  l->gkey = o; o += pd_align_up(8 * cap, 256);
  l->gsum = o; o += pd_align_up(8 * cap, 256);
  l->gcnt = o; o += pd_align_up(8 * cap, 256);
  l->gmin = o; o += pd_align_up(8 * cap, 256);
  l->gmax = o; o += pd_align_up(8 * cap, 256);
  l->ngroups = o; o += 256;
  l->ckey = o; o += pd_align_up(4 * cap, 256);
  l->cslot = o; o += pd_align_up(4 * cap, 256);
  l->skey = o; o += pd_align_up(4 * cap, 256);
  l->sslot = o; o += pd_align_up(4 * cap, 256);
  sa.nr_elements = cap;
  if (pimdal_sort_workspace_size(&sa, &w)) return false;
  l->sort_ws = o; o += w;
  l->total = o;
  return true;
}

}  // namespace

extern "C" int pimdal_group_workspace_size(const pimdal_aggr_arguments_t *a, size_t *bytes) {
  if (!a || !bytes) return PIMDAL_ERR_ARG;
  GbLayout l;
  if (!gb_layout(a, &l)) return PIMDAL_ERR_ARG;
  *bytes = l.total;
  return PIMDAL_OK;
}

extern "C" int pimdal_group_kernel(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *a,
                                   pimdal_aggr_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result) return PIMDAL_ERR_ARG;
  if (a->key_dtype != PIMDAL_I32 && a->key_dtype != PIMDAL_U32) return PIMDAL_ERR_ARG;
  if (a->method != PIMDAL_GROUP_AUTO && a->method != PIMDAL_GROUP_HASH &&
      a->method != PIMDAL_GROUP_SORT)
    return PIMDAL_ERR_ARG;
  if (a->size && !a->in) return PIMDAL_ERR_ARG;
  if (a->size >= (1ull << 30)) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  if (a->size == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d_result, 0, sizeof(uint64_t), s));
    return PIMDAL_OK;
  }
  GbLayout l;
  if (!gb_layout(a, &l)) return PIMDAL_ERR_ARG;
  int st;
  char *ws = (char *)pd_workspace(ctx, l.total, s, &st);
  if (!ws) return st;
  pimdal_sort_arguments_t sa{};
  sa.key_dtype = a->key_dtype;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;

  if (a->method == PIMDAL_GROUP_SORT) {
    sa.nr_elements = a->size;
    sa.in = a->in;
    sa.in_ptr = nullptr;  // row ids
    sa.out = ws + l.skey;
    sa.out_ptr = (uint32_t *)(ws + l.sslot);
    if ((st = pd_sort_with_workspace(ctx, &sa, ws + l.sort_ws, s))) return st;
    SegParams p{};
    p.skey = (const uint32_t *)(ws + l.skey);
    p.sidx = (const uint32_t *)(ws + l.sslot);
    p.val = a->in_val;
    p.n = a->size;
    p.out_key = (uint32_t *)a->out;
    p.out_sum = (long long *)a->out_sum;
    p.out_cnt = (unsigned long long *)a->out_count;
    p.out_min = (long long *)a->out_min;
    p.out_max = (long long *)a->out_max;
    p.cap = a->out_capacity;
    p.tile_heads = (uint64_t *)(ws + l.ngroups);
    p.tiles = pd_ceil_div(a->size, SR_TILE);
    p.d_error = ctx->d_error;
    p.d_count = &d_result->t_count;
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_sr_heads<<<(unsigned)p.tiles, SR_THREADS, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_sr_scan<<<1, 1024, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_sr_init<<<ctx->sm_count * 8, 256, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_SEGREDUCE, s);
      k_gb_segreduce<<<(unsigned)p.tiles, SR_THREADS, 0, s>>>(p);
    }
    return pd_launch_status(ctx);
  }

  GbParams p{};
  p.key = (const uint32_t *)a->in;
  p.val = a->in_val;
  p.n = a->size;
  p.gkey = (unsigned long long *)(ws + l.gkey);
  p.gsum = (long long *)(ws + l.gsum);
  p.gcnt = (unsigned long long *)(ws + l.gcnt);
  p.gmin = (long long *)(ws + l.gmin);
  p.gmax = (long long *)(ws + l.gmax);
  p.bits = l.bits;
  p.ngroups = (unsigned long long *)(ws + l.ngroups);
  p.ckey = (uint32_t *)(ws + l.ckey);
  p.cslot = (uint32_t *)(ws + l.cslot);
  p.d_error = ctx->d_error;
  const uint64_t cap = 1ull << l.bits;
  const unsigned init_grid = (unsigned)std::min<uint64_t>(pd_ceil_div(cap, 256), ctx->sm_count * 8ull);
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gb_init<<<init_grid, 256, 0, s>>>(p);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_GROUP, s);
    const unsigned grid = (unsigned)std::min<uint64_t>(pd_ceil_div(a->size, GB_THREADS * 8ull),
                                                       (uint64_t)ctx->sm_count * 2);
    PD_CHECK_CUDA(cudaFuncSetAttribute(k_gb_aggregate, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)GB_SMEM_BYTES));
    k_gb_aggregate<<<grid ? grid : 1, GB_THREADS, GB_SMEM_BYTES, s>>>(p);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gb_compact<<<init_grid, 256, 0, s>>>(p);
  }
  sa.nr_elements = cap;  // upper bound; the real count is read on the device
  sa.in = p.ckey;
  sa.in_ptr = p.cslot;
  sa.out = ws + l.skey;
  sa.out_ptr = (uint32_t *)(ws + l.sslot);
  if ((st = pd_sort_ex2(ctx, &sa, PD_KEY_PLAIN, ws + l.sort_ws, s, nullptr,
                        (const uint64_t *)p.ngroups)))
    return st;
  GatherParams g{};
  g.skey = (const uint32_t *)(ws + l.skey);
  g.sslot = (const uint32_t *)(ws + l.sslot);
  g.ngroups = p.ngroups;
  g.gsum = p.gsum;
  g.gmin = p.gmin;
  g.gmax = p.gmax;
  g.gcnt = p.gcnt;
  g.out_key = (uint32_t *)a->out;
  g.out_sum = a->out_sum;
  g.out_count = a->out_count;
  g.out_min = a->out_min;
  g.out_max = a->out_max;
  g.cap = a->out_capacity;
  g.d_count = &d_result->t_count;
  g.d_error = ctx->d_error;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gb_gather<<<init_grid, 256, 0, s>>>(g);
  }
  return pd_launch_status(ctx);
}
