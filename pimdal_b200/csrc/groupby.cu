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
// B200 design, hash method.  A group lives in one 32-byte slot
// {count << 32 | key, sum, min, max}: the claiming compare-and-swap carries
// the first rows' count, and every later update of the group touches the same
// sector.  Three aggregation modes, chosen from the expected group count:
//  - GB_WARP (a few dozen groups): each warp owns a private shared-memory
//    table of 192 slots (split in up to 4 replicas, each for a subset of the
//    lanes), so only a few lanes of one warp ever contend;
//  - GB_SMEM (up to a few thousand groups): every row updates the CTA's
//    shared-memory table (6144 slots, 192 KB, one 1024-thread CTA per SM);
//  - GB_PART (many groups): the rows (key and value) are first radix-
//    partitioned by the top bits of a multiplicative hash of the key, in
//    stable passes of at most 6 bits, into 2^b partitions of about 1024
//    groups each.  Persistent CTAs then take chunks of consecutive rows (a
//    chunk spans one or two partitions), aggregate each chunk in the
//    shared-memory table and flush the slots it claimed into the global
//    table -- about one global merge per group instead of global atomics
//    per row.  This is the single-pass form of the reference's spill rounds
//    (aggregate_hash.c:145-188), which re-aggregate the rows that did not
//    fit the DPU's table;
//  - GB_DIRECT (the batched form's many-group instances, or
//    PIMDAL_GROUP_DIRECT=1): rows update the global table directly.  When
//    the table is larger than an L2 budget it can be split into K sub-tables
//    by the high hash bits and aggregated in K launches, each touching an
//    L2-sized sub-table (PIMDAL_GROUP_L2_BUDGET_MB; one pass by default).
// Shared tables probe 4-slot buckets of 32-bit keys with one 16-byte load.
// A row whose group finds no shared slot within 16 buckets goes to the global
// table; shared tables are merged into the global table at the end of each
// CTA.  A global update reads the slot's sector once (two 16-byte loads
// issued together), claims an empty slot with one compare-and-swap, and adds
// the count and sum with fire-and-forget reductions; min/max reductions are
// issued only when the loaded value shows they change the slot.
// The occupied global slots are then compacted, sorted by key with K-SORT
// (element count read on the device) and gathered into the outputs.
// Sort method: K-SORT of (key, row id), then a reduce-by-key over the sorted
// rows (see k_gb_segreduce).
#include <algorithm>

#include "batch.cuh"

namespace {

constexpr int GB_THREADS = 1024;
constexpr int GB_WARPS = GB_THREADS / 32;
constexpr uint32_t GB_SMEM_SLOTS = 6144;
constexpr uint32_t GB_WARP_SLOTS = GB_SMEM_SLOTS / GB_WARPS;  // 192 per warp
constexpr uint32_t GB_SMEM_PROBES = 16;  // buckets
constexpr size_t GB_SMEM_BYTES = 32ull * GB_SMEM_SLOTS;      // 192 KB
constexpr uint64_t GB_WARP_MAX_GROUPS = 64;                  // GB_WARP at or below
constexpr uint64_t GB_SMEM_MAX_GROUPS = 4608;                // GB_SMEM at or below (load 3/4)
constexpr uint64_t GB_L2_BUDGET = 1ull << 40;                // one pass unless overridden
enum { GB_WARP = 0, GB_SMEM = 1, GB_DIRECT = 2, GB_PART = 3 };
constexpr uint64_t GB_PART_GROUPS = 1024;   // groups per hash partition
constexpr uint32_t GB_PART_MAX_BITS = 12;

struct GbParams {
  const uint32_t *key;
  const int64_t *val;  // NULL: every value is 1
  uint64_t n;
  int vec;             // key and val 16-byte aligned: 4 rows per vector load
  // global table: npasses sub-tables of sub_cap 32-byte slots
  unsigned long long *gtab;
  uint32_t sub_cap, npasses;
  uint32_t wrep;       // GB_WARP: private replicas per warp (1, 2 or 4)
  unsigned long long *ngroups;  // compacted group count (device)
  uint32_t *ckey, *cslot;
  uint32_t *d_error;
};

__device__ __forceinline__ uint64_t gb_h(uint32_t key) { return pd_mix64(key); }
__device__ __forceinline__ uint32_t gb_pass(uint64_t h, uint32_t k) {
  return (uint32_t)(((h >> 32) * k) >> 32);
}
__device__ __forceinline__ uint32_t gb_slot(uint64_t h, uint32_t cap) {
  return (uint32_t)(((h & 0xffffffffull) * cap) >> 32);
}

__global__ void __launch_bounds__(256) k_gb_init(GbParams p) {
  const uint64_t slots = (uint64_t)p.sub_cap * p.npasses;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  ulonglong2 *t = reinterpret_cast<ulonglong2 *>(p.gtab);
  const ulonglong2 lo = make_ulonglong2(0ull, 0ull);
  const ulonglong2 hi = make_ulonglong2((unsigned long long)INT64_MAX, (unsigned long long)INT64_MIN);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += stride) {
    t[2 * i] = lo;
    t[2 * i + 1] = hi;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *p.ngroups = 0;
}

// Adds a partial aggregate of `key` to sub-table `pass` of the global table,
// starting at slot s whose sector (a, b) the caller may already have loaded.
__device__ void global_add_from(const GbParams &p, uint32_t key, uint32_t pass, uint32_t s,
                                ulonglong2 a, ulonglong2 b, bool loaded, uint32_t cnt,
                                long long sum, long long mn, long long mx) {
  const uint32_t cap = p.sub_cap;
  unsigned long long *base = p.gtab + (uint64_t)pass * cap * 4;
  const unsigned long long mine = ((unsigned long long)cnt << 32) | key;
  for (uint32_t t = 0; t < cap; ++t) {
    unsigned long long *slot = base + (uint64_t)s * 4;
    if (!loaded) {
      a = __ldcg(reinterpret_cast<const ulonglong2 *>(slot));
      b = __ldcg(reinterpret_cast<const ulonglong2 *>(slot) + 1);
    }
    loaded = false;
    unsigned long long w = a.x;
    bool claimed = false;
    if (w == 0) {
      w = atomicCAS(slot, 0ull, mine);
      claimed = w == 0;
    }
    if (claimed || (uint32_t)w == key) {
      if (!claimed) atomicAdd(slot, (unsigned long long)cnt << 32);
      atomicAdd(slot + 1, (unsigned long long)sum);
      // min/max only move one way: a stale value can only cause a redundant reduction
      if (mn < (long long)b.x) atomicMin(reinterpret_cast<long long *>(slot) + 2, mn);
      if (mx > (long long)b.y) atomicMax(reinterpret_cast<long long *>(slot) + 3, mx);
      return;
    }
    s = (s + 1 == cap) ? 0 : s + 1;
  }
  atomicOr(p.d_error, PD_DEVERR_TABLE_FULL);
}

__device__ __forceinline__ void global_add(const GbParams &p, uint32_t key, uint64_t h, uint32_t pass,
                                           uint32_t cnt, long long sum, long long mn, long long mx) {
  global_add_from(p, key, pass, gb_slot(h, p.sub_cap), ulonglong2{}, ulonglong2{}, false, cnt, sum,
                  mn, mx);
}

// Shared table: 4-slot buckets of 32-bit keys (empty = all ones), one 16-byte
// load probes a bucket.  The all-ones key itself bypasses shared tables.
constexpr uint32_t GB_EMPTY = 0xFFFFFFFFu;

struct SmemTable {
  uint32_t *key;
  uint32_t *cnt;
  long long *sum;
  longlong2 *mm;     // (min, max)
  uint16_t *list;    // batched runs: slots claimed since the last flush
  uint32_t *nlist;
};

__device__ __forceinline__ int bucket_match(const uint4 &q, uint32_t key) {
  return q.x == key ? 0 : q.y == key ? 1 : q.z == key ? 2 : q.w == key ? 3 : -1;
}

// Slot of `key` in buckets [base, base + nb) of a shared table, claiming an
// empty slot when the key is absent; -1 when no bucket within the probe limit
// has room (the row then goes to the global table).
__device__ __noinline__ int smem_find(const SmemTable &t, uint32_t base, uint32_t nb, uint32_t key,
                                      uint32_t b) {
  for (uint32_t i = 0; i < GB_SMEM_PROBES;) {
    const uint32_t s0 = 4 * (base + b);
    // plain loads: a key never changes once set, so a stale bucket costs at
    // most a failed compare-and-swap and another look
    const uint4 q = *reinterpret_cast<const uint4 *>(t.key + s0);
    const int hit = bucket_match(q, key);
    if (hit >= 0) return (int)s0 + hit;
    const int e = bucket_match(q, GB_EMPTY);
    if (e < 0) {  // full bucket without the key: next bucket
      b = (b + 1 == nb) ? 0 : b + 1;
      ++i;
      continue;
    }
    const uint32_t old = atomicCAS(t.key + s0 + e, GB_EMPTY, key);
    if (old == GB_EMPTY && t.list) t.list[atomicAdd(t.nlist, 1u)] = (uint16_t)(s0 + e);
    if (old == GB_EMPTY || old == key) return (int)s0 + e;
    // lost the slot to another key: look at the bucket again
  }
  return -1;
}

// Four rows of one lane: (A) bucket lookups with all four loads in flight,
// the rare claims and full buckets on a slow path; (B) the updates as
// straight-line predicated shared atomics.
template <int MODE>
__device__ __forceinline__ void gb_rows4(const GbParams &p, const SmemTable &t, uint32_t pass,
                                         const uint32_t (&k)[4], const long long (&v)[4],
                                         uint32_t valid, uint32_t base, uint32_t nb) {
  if constexpr (MODE == GB_DIRECT) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (!((valid >> r) & 1u)) continue;
      const uint64_t h = gb_h(k[r]);
      if (p.npasses > 1 && gb_pass(h, p.npasses) != pass) continue;
      global_add(p, k[r], h, pass, 1u, v[r], v[r], v[r]);
    }
  } else {
    // home and next bucket of every row, all eight loads in flight together
    uint32_t b[4];
    uint4 q[4], q2[4];
    int slot[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      b[r] = gb_slot(gb_h(k[r]), nb);
      const uint32_t b2 = b[r] + 1 == nb ? 0 : b[r] + 1;
      q[r] = *reinterpret_cast<const uint4 *>(t.key + 4 * (base + b[r]));
      q2[r] = *reinterpret_cast<const uint4 *>(t.key + 4 * (base + b2));
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      // the all-ones key equals the empty marker: it always takes the global path
      const int hit = bucket_match(q[r], k[r]);
      const bool home_full = bucket_match(q[r], GB_EMPTY) < 0;
      const int hit2 = home_full ? bucket_match(q2[r], k[r]) : -1;
      const uint32_t b2 = b[r] + 1 == nb ? 0 : b[r] + 1;
      slot[r] = k[r] == GB_EMPTY ? -1
              : hit >= 0         ? (int)(4 * (base + b[r])) + hit
              : hit2 >= 0        ? (int)(4 * (base + b2)) + hit2
                                 : -2;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (!((valid >> r) & 1u)) slot[r] = -3;
      else if (slot[r] == -2) slot[r] = smem_find(t, base, nb, k[r], b[r]);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (slot[r] >= 0) {
        atomicAdd(t.cnt + slot[r], 1u);
        atomicAdd(reinterpret_cast<unsigned long long *>(t.sum) + slot[r], (unsigned long long)v[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (slot[r] >= 0) {
        const longlong2 m = t.mm[slot[r]];
        if (v[r] < m.x) atomicMin(&t.mm[slot[r]].x, v[r]);
        if (v[r] > m.y) atomicMax(&t.mm[slot[r]].y, v[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (slot[r] == -1) global_add(p, k[r], gb_h(k[r]), 0, 1u, v[r], v[r], v[r]);
  }
}

// Rows [r0, r1) of p by `warps` warps (this one is number gw): 128
// consecutive rows per warp step, 4 per lane (one 16-byte key load and two
// 16-byte value loads when aligned), then the unaligned rest.
template <int MODE>
__device__ __forceinline__ void gb_range(const GbParams &p, const SmemTable &t, uint32_t pass,
                                         uint64_t r0, uint64_t r1, uint64_t gw, uint64_t warps,
                                         int lane, uint32_t base, uint32_t nb) {
  uint64_t done = r0;
  if (p.vec && (r0 & 3u) == 0) {
    const uint64_t q1 = r1 / 4;  // quads of rows
    const uint4 *k4 = reinterpret_cast<const uint4 *>(p.key);
    const longlong2 *v2 = reinterpret_cast<const longlong2 *>(p.val);
    for (uint64_t b = r0 / 4 + gw * 32; b < q1; b += warps * 32) {
      const uint64_t q = b + lane;
      const bool ok = q < q1;
      uint4 k = make_uint4(0, 0, 0, 0);
      longlong2 va = make_longlong2(1, 1), vb = make_longlong2(1, 1);
      if (ok) {
        k = __ldcs(k4 + q);
        bool need = true;
        if (MODE == GB_DIRECT && p.npasses > 1) {
          need = gb_pass(gb_h(k.x), p.npasses) == pass || gb_pass(gb_h(k.y), p.npasses) == pass ||
                 gb_pass(gb_h(k.z), p.npasses) == pass || gb_pass(gb_h(k.w), p.npasses) == pass;
        }
        if (p.val && need) {
          va = __ldcs(v2 + 2 * q);
          vb = __ldcs(v2 + 2 * q + 1);
        }
      }
      const uint32_t kk[4] = {k.x, k.y, k.z, k.w};
      const long long vv[4] = {va.x, va.y, vb.x, vb.y};
      gb_rows4<MODE>(p, t, pass, kk, vv, ok ? 0xFu : 0u, base, nb);
    }
    done = q1 * 4;
  }
  // unaligned input or the last rows: lane-striped groups of four rows
  for (uint64_t b = done + gw * 128; b < r1; b += warps * 128) {
    uint32_t kk[4];
    long long vv[4];
    uint32_t valid = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint64_t i = b + 32 * r + lane;
      const bool in = i < r1;
      valid |= (uint32_t)in << r;
      kk[r] = in ? p.key[i] : 0u;
      vv[r] = (in && p.val) ? (long long)p.val[i] : 1ll;
    }
    gb_rows4<MODE>(p, t, pass, kk, vv, valid, base, nb);
  }
}

__device__ __forceinline__ SmemTable gb_smem_table(unsigned char *smem) {
  SmemTable t;
  t.key = reinterpret_cast<uint32_t *>(smem);
  t.cnt = t.key + GB_SMEM_SLOTS;
  t.sum = reinterpret_cast<long long *>(t.cnt + GB_SMEM_SLOTS);
  t.mm = reinterpret_cast<longlong2 *>(t.sum + GB_SMEM_SLOTS);
  t.list = nullptr;
  t.nlist = nullptr;
  return t;
}

__device__ __forceinline__ void gb_clear_slot(const SmemTable &t, uint32_t i) {
  t.key[i] = GB_EMPTY;
  t.cnt[i] = 0;
  t.sum[i] = 0;
  t.mm[i] = make_longlong2(INT64_MAX, INT64_MIN);
}

// Shared buckets of this lane: its warp's replica (GB_WARP) or the CTA table.
__device__ __forceinline__ void gb_buckets(int mode, uint32_t wrep, uint32_t *base, uint32_t *nb) {
  *base = 0;
  *nb = GB_SMEM_SLOTS / 4;
  if (mode == GB_WARP) {
    const int lane = threadIdx.x & 31;
    *nb = GB_WARP_SLOTS / 4 / wrep;
    *base = (threadIdx.x >> 5) * (GB_WARP_SLOTS / 4) + (lane / (32 / wrep)) * *nb;
  }
}

// Persistent CTAs over all rows.  In GB_WARP mode each warp's 192 slots form
// p.wrep private replicas, one per group of 32 / p.wrep lanes.
template <int MODE>
__global__ void __launch_bounds__(GB_THREADS, MODE == GB_DIRECT ? 2 : 1)
k_gb_aggregate(GbParams p, uint32_t pass) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  const SmemTable t = gb_smem_table(gb_smem);
  if (MODE != GB_DIRECT) {
    for (uint32_t i = threadIdx.x; i < GB_SMEM_SLOTS; i += GB_THREADS) gb_clear_slot(t, i);
    __syncthreads();
  }
  uint32_t base, nb;
  gb_buckets(MODE, p.wrep, &base, &nb);
  const uint64_t warps = (uint64_t)gridDim.x * GB_WARPS;
  const uint64_t gw = (uint64_t)blockIdx.x * GB_WARPS + (threadIdx.x >> 5);
  gb_range<MODE>(p, t, pass, 0, p.n, gw, warps, threadIdx.x & 31, base, nb);
  if (MODE != GB_DIRECT) {
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < GB_SMEM_SLOTS; i += GB_THREADS) {
      const uint32_t k = t.key[i];
      if (k != GB_EMPTY)
        global_add(p, k, gb_h(k), 0, t.cnt[i], t.sum[i], t.mm[i].x, t.mm[i].y);
    }
  }
}

// GB_PART: rows grouped by a hash digit.  Persistent CTAs claim chunks of
// `chunk` consecutive rows; a chunk goes through the shared table and the
// slots it claimed are flushed to the global table and reset.
__global__ void __launch_bounds__(GB_THREADS, 1) k_gb_chunks(GbParams p, uint64_t chunk,
                                                             uint32_t *claim) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  __shared__ uint32_t s_item, s_nlist;
  SmemTable t = gb_smem_table(gb_smem);
  t.list = reinterpret_cast<uint16_t *>(gb_smem + GB_SMEM_BYTES);
  t.nlist = &s_nlist;
  for (uint32_t i = threadIdx.x; i < GB_SMEM_SLOTS; i += GB_THREADS) gb_clear_slot(t, i);
  if (threadIdx.x == 0) s_nlist = 0;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = threadIdx.x >> 5;
  const uint64_t nchunks = pd_ceil_div(p.n, chunk);
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t it = atomicAdd(claim, 1u);
      if (it >= nchunks && atomicAdd(claim + 1, 1u) == gridDim.x - 1) {
        claim[0] = 0;  // the last claimer of the launch resets the counters
        claim[1] = 0;
      }
      s_item = it;
    }
    __syncthreads();
    const uint64_t it = s_item;
    if (it >= nchunks) break;
    const uint64_t r0 = it * chunk, r1 = min(r0 + chunk, p.n);
    gb_range<GB_SMEM>(p, t, 0, r0, r1, warp, GB_WARPS, lane, 0, GB_SMEM_SLOTS / 4);
    __syncthreads();
    const uint32_t nl = s_nlist;
    for (uint32_t i = threadIdx.x; i < nl; i += GB_THREADS) {
      const uint32_t j = t.list[i];
      const uint32_t k = t.key[j];
      global_add(p, k, gb_h(k), 0, t.cnt[j], t.sum[j], t.mm[j].x, t.mm[j].y);
      gb_clear_slot(t, j);
    }
    __syncthreads();
    if (threadIdx.x == 0) s_nlist = 0;
  }
}

// ---------------------------------------------------------------------------
// Batched group-by (pd_gb_batch): persistent CTAs take (instance, row block)
// work items from a device queue in instance-major order.  An item's rows go
// through the CTA's shared table in the instance's mode; at the end of the
// item the slots it claimed are merged into the instance's global table and
// reset.  The instances' tables are then compacted together, sorted by key
// and stably by instance, and gathered into each instance's outputs.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t gbb_inst_of_slot(const pd_gb_batch &b, uint64_t slot) {
  uint32_t lo = 0, hi = b.count;  // last instance whose slot0 <= slot
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (b.slot0[m] <= slot) lo = m; else hi = m;
  }
  return lo;
}

__device__ __forceinline__ GbParams gbb_params(const pd_gb_batch &b, const pd_gb_inst &in) {
  GbParams p{};
  p.key = in.key;
  p.val = in.val;
  p.n = in.n;
  p.vec = ((uintptr_t)in.key & 15u) == 0 && ((uintptr_t)in.val & 15u) == 0;
  p.gtab = b.gtab + 4 * in.slot0;
  p.sub_cap = in.slots;
  p.npasses = 1;
  p.wrep = in.wrep;
  p.d_error = b.d_error;
  return p;
}

__global__ void __launch_bounds__(256) k_gbb_init(pd_gb_batch b) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  ulonglong2 *t = reinterpret_cast<ulonglong2 *>(b.gtab);
  const ulonglong2 lo = make_ulonglong2(0ull, 0ull);
  const ulonglong2 hi = make_ulonglong2((unsigned long long)INT64_MAX, (unsigned long long)INT64_MIN);
  const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t i = i0; i < b.total_slots; i += stride) {
    t[2 * i] = lo;
    t[2 * i + 1] = hi;
  }
  for (uint64_t i = i0; i < b.count; i += stride) b.inst_groups[i] = 0;
  if (i0 == 0) *b.ngroups = 0;
}

__global__ void __launch_bounds__(GB_THREADS, 1) k_gbb_aggregate(pd_gb_batch b) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  __shared__ uint32_t s_item, s_nlist;
  SmemTable t = gb_smem_table(gb_smem);
  t.list = reinterpret_cast<uint16_t *>(gb_smem + GB_SMEM_BYTES);
  t.nlist = &s_nlist;
  for (uint32_t i = threadIdx.x; i < GB_SMEM_SLOTS; i += GB_THREADS) gb_clear_slot(t, i);
  if (threadIdx.x == 0) s_nlist = 0;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = threadIdx.x >> 5;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t it = atomicAdd(b.counters, 1u);
      if (it >= b.nitems && atomicAdd(b.counters + 1, 1u) == gridDim.x - 1) {
        b.counters[0] = 0;  // the last claimer of the launch resets the queue
        b.counters[1] = 0;
      }
      s_item = it;
    }
    __syncthreads();
    const uint32_t it = s_item;
    if (it >= b.nitems) break;
    const uint2 item = b.items[it];
    const pd_gb_inst &in = b.inst[item.x];
    const GbParams p = gbb_params(b, in);
    const uint64_t r0 = item.y, r1 = min((uint64_t)item.y + b.rows_per_item, in.n);
    const int mode = (int)in.mode;
    uint32_t base, nb;
    gb_buckets(mode, in.wrep, &base, &nb);
    if (mode == GB_WARP) gb_range<GB_WARP>(p, t, 0, r0, r1, warp, GB_WARPS, lane, base, nb);
    else if (mode == GB_SMEM) gb_range<GB_SMEM>(p, t, 0, r0, r1, warp, GB_WARPS, lane, base, nb);
    else gb_range<GB_DIRECT>(p, t, 0, r0, r1, warp, GB_WARPS, lane, base, nb);
    if (mode != GB_DIRECT) {
      __syncthreads();
      const uint32_t nl = s_nlist;
      for (uint32_t i = threadIdx.x; i < nl; i += GB_THREADS) {
        const uint32_t j = t.list[i];
        const uint32_t k = t.key[j];
        global_add(p, k, gb_h(k), 0, t.cnt[j], t.sum[j], t.mm[j].x, t.mm[j].y);
        gb_clear_slot(t, j);
      }
      __syncthreads();
      if (threadIdx.x == 0) s_nlist = 0;
    }
  }
}

// Occupied slots of every instance -> (order-transformed key, slot).
__global__ void __launch_bounds__(256) k_gbb_compact(pd_gb_batch b) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < b.total_slots; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const unsigned long long w = i < b.total_slots ? __ldcs(b.gtab + 4 * i) : 0ull;
    const unsigned m = __ballot_sync(0xffffffffu, w != 0);
    if (!m) continue;
    uint32_t pos = 0;
    if (lane == 0) pos = (uint32_t)atomicAdd(b.ngroups, (unsigned long long)__popc(m));
    pos = __shfl_sync(0xffffffffu, pos, 0) + __popc(m & ((1u << lane) - 1u));
    if (w) {
      const uint32_t inst = gbb_inst_of_slot(b, i);
      atomicAdd(b.inst_groups + inst, 1u);
      b.ckey[pos] = (uint32_t)w ^ b.inst[inst].flip;
      b.cslot[pos] = (uint32_t)i;
    }
  }
}

// Key-ordered (key, slot) -> (instance, slot) for the stable sort by instance.
__global__ void __launch_bounds__(256) k_gbb_inst(pd_gb_batch b) {
  const uint64_t n = *b.ngroups;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t slot = b.sslot[i];
    b.ikey[i] = gbb_inst_of_slot(b, slot);
    b.islot[i] = slot;
  }
}

// Per-instance first position and group count (one block).
__global__ void __launch_bounds__(1024) k_gbb_start(pd_gb_batch b) {
  __shared__ uint64_t s_w[32];
  __shared__ uint64_t s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < b.count; base += 1024) {
    const uint32_t i = base + tid;
    const uint64_t v = i < b.count ? b.inst_groups[i] : 0;
    uint64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    uint64_t pre = 0, tot = 0;
    for (int w = 0; w < 32; ++w) {
      if (w < warp) pre += s_w[w];
      tot += s_w[w];
    }
    if (i < b.count) {
      b.inst_start[i] = s_carry + pre + inc - v;
      const pd_gb_inst &in = b.inst[i];
      *in.d_count = v;
      if (v > in.out_cap) atomicOr(b.d_error, PD_DEVERR_CAPACITY);
    }
    __syncthreads();
    if (tid == 0) s_carry += tot;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_gbb_gather(pd_gb_batch b) {
  const uint64_t n = *b.ngroups;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const ulonglong2 *t = reinterpret_cast<const ulonglong2 *>(b.gtab);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t inst = b.ckey[i];
    const uint64_t s = b.cslot[i];
    const pd_gb_inst &in = b.inst[inst];
    const uint64_t j = i - b.inst_start[inst];
    if (j >= in.out_cap) continue;
    const ulonglong2 x = t[2 * s], y = t[2 * s + 1];
    if (in.out_key) in.out_key[j] = (uint32_t)x.x;
    if (in.out_sum) in.out_sum[j] = (int64_t)x.y;
    if (in.out_count) in.out_count[j] = (int64_t)(x.x >> 32);
    if (in.out_min) in.out_min[j] = (int64_t)y.x;
    if (in.out_max) in.out_max[j] = (int64_t)y.y;
  }
}

// Occupied slots -> (key, slot) list (order is restored by the sort that follows).
__global__ void __launch_bounds__(256) k_gb_compact(GbParams p) {
  const uint64_t slots = (uint64_t)p.sub_cap * p.npasses;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < slots; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const unsigned long long w = i < slots ? __ldcs(p.gtab + 4 * i) : 0ull;
    const unsigned m = __ballot_sync(0xffffffffu, w != 0);
    if (!m) continue;
    uint32_t pos = 0;
    if (lane == 0) pos = (uint32_t)atomicAdd(p.ngroups, (unsigned long long)__popc(m));
    pos = __shfl_sync(0xffffffffu, pos, 0) + __popc(m & ((1u << lane) - 1u));
    if (w) {
      p.ckey[pos] = (uint32_t)w;
      p.cslot[pos] = (uint32_t)i;
    }
  }
}

struct GatherParams {
  const uint32_t *skey, *sslot;
  const unsigned long long *ngroups;
  const unsigned long long *gtab;
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
  const ulonglong2 *t = reinterpret_cast<const ulonglong2 *>(g.gtab);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += stride) {
    const uint64_t s = g.sslot[i];
    const ulonglong2 a = t[2 * s], b = t[2 * s + 1];
    if (g.out_key) g.out_key[i] = g.skey[i];
    if (g.out_sum) g.out_sum[i] = (int64_t)a.y;
    if (g.out_count) g.out_count[i] = (int64_t)(a.x >> 32);
    if (g.out_min) g.out_min[i] = (int64_t)b.x;
    if (g.out_max) g.out_max[i] = (int64_t)b.y;
  }
}

// ---------------------------------------------------------------------------
// Sort method.  When the values' range fits 32 bits (checked on the device:
// k_vrange), each row's value - min travels through the sort as its payload
// and the reduce-by-key reads the values from the sorted stream; otherwise
// the sort carries row ids and the reduce gathers the values by row id.
// Both paths are enqueued; the device sets one path's row count to n and
// the other's to 0, and a path with no rows does nothing -- so the choice
// needs no host round trip.  Without values (COUNT only) keys are sorted
// alone.  Tiles of 4096 sorted rows; a thread owns 16 consecutive rows.
//  1. k_sr_heads: group heads per tile;
//  2. k_sr_scan (one block): exclusive head prefix per tile, group count G;
//  3. k_sr_init: outputs 0..G-1 set to the aggregate identities;
//  4. k_gb_segreduce: a group inside one thread's rows is stored directly;
//     groups cut by thread boundaries are joined by a block-wide segmented
//     scan and stored directly too; only the (at most two) groups of a tile
//     that cross the tile's edges are merged with 64-bit global atomics.
// ---------------------------------------------------------------------------
constexpr int SR_THREADS = 256;
constexpr int SR_ITEMS = 16;
constexpr int SR_TILE = SR_THREADS * SR_ITEMS;

struct SegParams {
  const uint32_t *skey, *sidx;  // sidx: row ids, or payloads (pay_min set); NULL: no values
  const int64_t *val;           // gathered by row id (row-id path)
  const long long *pay_min;     // payload path: value = *pay_min + payload
  const uint64_t *n_dev;        // rows of this path (0: the path is not taken)
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

// The path's row count; false when the path is not taken.
__device__ __forceinline__ bool sr_active(SegParams &p) {
  if (p.n_dev) p.n = *p.n_dev;
  return p.n != 0;
}

__global__ void __launch_bounds__(SR_THREADS) k_sr_heads(SegParams p) {
  __shared__ uint32_t s_red[SR_THREADS / 32];
  if (!sr_active(p)) return;
  for (uint64_t tile = blockIdx.x; tile < p.tiles; tile += gridDim.x) {
    const uint64_t r0 = tile * SR_TILE + threadIdx.x;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < SR_ITEMS; ++j) c += sr_head(p, r0 + (uint64_t)j * SR_THREADS);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __syncthreads();  // s_red of the previous tile has been read
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < SR_THREADS / 32; ++w) t += s_red[w];
      p.tile_heads[tile] = t;
    }
  }
}

__global__ void __launch_bounds__(1024) k_sr_scan(SegParams p) {
  __shared__ uint64_t s_w[32];
  __shared__ uint64_t s_carry;
  if (!sr_active(p)) return;
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
  if (!sr_active(p)) return;
  const uint64_t lim = min(*p.d_count, p.cap);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += stride) {
    if (p.out_sum) p.out_sum[i] = 0;
    if (p.out_cnt) p.out_cnt[i] = 0;
    if (p.out_min) p.out_min[i] = INT64_MAX;
    if (p.out_max) p.out_max[i] = INT64_MIN;
  }
}

struct SrAgg {
  uint32_t cnt;  // rows inside one tile
  long long sum, mn, mx;
};

__device__ __forceinline__ SrAgg sr_empty() { return SrAgg{0u, 0ll, INT64_MAX, INT64_MIN}; }

__device__ __forceinline__ void sr_acc(SrAgg &a, long long v) {
  ++a.cnt;
  a.sum = (long long)((unsigned long long)a.sum + (unsigned long long)v);
  a.mn = min(a.mn, v);
  a.mx = max(a.mx, v);
}

__device__ __forceinline__ SrAgg sr_join(const SrAgg &a, const SrAgg &b) {
  return SrAgg{a.cnt + b.cnt, (long long)((unsigned long long)a.sum + (unsigned long long)b.sum),
               min(a.mn, b.mn), max(a.mx, b.mx)};
}

// Segmented-scan element: f = a group head lies in the covered rows; key and
// agg describe the rows from the last such head (or all rows when f = 0).
struct SrSeg {
  uint32_t f, key;
  SrAgg a;
};

__device__ __forceinline__ SrSeg sr_combine(const SrSeg &l, const SrSeg &r) {
  if (r.f) return r;
  return SrSeg{l.f, l.key, sr_join(l.a, r.a)};
}

__device__ __forceinline__ SrSeg sr_shfl_up(const SrSeg &x, int o) {
  SrSeg y;
  y.f = __shfl_up_sync(0xffffffffu, x.f, o);
  y.key = __shfl_up_sync(0xffffffffu, x.key, o);
  y.a.cnt = __shfl_up_sync(0xffffffffu, x.a.cnt, o);
  y.a.sum = __shfl_up_sync(0xffffffffu, x.a.sum, o);
  y.a.mn = __shfl_up_sync(0xffffffffu, x.a.mn, o);
  y.a.mx = __shfl_up_sync(0xffffffffu, x.a.mx, o);
  return y;
}

__device__ __forceinline__ void sr_store(const SegParams &p, uint64_t g, uint32_t key, bool whole,
                                         const SrAgg &a) {
  if (g >= p.cap || a.cnt == 0) return;  // overflow is reported by k_sr_scan
  if (p.out_key) p.out_key[g] = key;     // every writer of a group stores the same key
  if (whole) {
    if (p.out_sum) p.out_sum[g] = a.sum;
    if (p.out_cnt) p.out_cnt[g] = a.cnt;
    if (p.out_min) p.out_min[g] = a.mn;
    if (p.out_max) p.out_max[g] = a.mx;
  } else {
    if (p.out_sum) atomicAdd((unsigned long long *)(p.out_sum + g), (unsigned long long)a.sum);
    if (p.out_cnt) atomicAdd(p.out_cnt + g, (unsigned long long)a.cnt);
    if (p.out_min) atomicMin(p.out_min + g, a.mn);
    if (p.out_max) atomicMax(p.out_max + g, a.mx);
  }
}

// 3 CTAs per SM (80 registers, a 28-byte spill) instead of 2 at 126:
// 1.26 -> 1.10 ms over 2^28 sorted rows (4 CTAs at 64 spilled more, 1.22).
__global__ void __launch_bounds__(SR_THREADS, 3) k_gb_segreduce(SegParams p) {
  __shared__ uint32_t s_heads[SR_THREADS / 32];
  __shared__ SrSeg s_seg[SR_THREADS / 32];
  if (!sr_active(p)) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (uint64_t tile = blockIdx.x; tile < p.tiles; tile += gridDim.x) {
  __syncthreads();  // the previous tile's readers of shared memory are done
  const uint64_t t0 = tile * SR_TILE;
  const uint64_t r0 = t0 + (uint64_t)tid * SR_ITEMS;
  const bool full = t0 + SR_TILE <= p.n;
  uint32_t key[SR_ITEMS], idx[SR_ITEMS];
  const bool has_idx = p.sidx != nullptr;
  if (full) {
    const uint4 *k4 = reinterpret_cast<const uint4 *>(p.skey + r0);
    const uint4 *i4 = reinterpret_cast<const uint4 *>(p.sidx + r0);
#pragma unroll
    for (int j = 0; j < SR_ITEMS / 4; ++j) {
      const uint4 a = __ldcs(k4 + j);
      const uint4 b = has_idx ? __ldcs(i4 + j) : make_uint4(0, 0, 0, 0);
      key[4 * j] = a.x; key[4 * j + 1] = a.y; key[4 * j + 2] = a.z; key[4 * j + 3] = a.w;
      idx[4 * j] = b.x; idx[4 * j + 1] = b.y; idx[4 * j + 2] = b.z; idx[4 * j + 3] = b.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < SR_ITEMS; ++j) {
      key[j] = (r0 + j < p.n) ? p.skey[r0 + j] : 0u;
      idx[j] = (has_idx && r0 + j < p.n) ? p.sidx[r0 + j] : 0u;
    }
  }
  long long val[SR_ITEMS];
  if (p.pay_min) {
    const long long pmin = *p.pay_min;
#pragma unroll
    for (int j = 0; j < SR_ITEMS; ++j) val[j] = pmin + (long long)idx[j];
  } else {
#pragma unroll
    for (int j = 0; j < SR_ITEMS; ++j)
      val[j] = (p.val && (full || r0 + j < p.n)) ? (long long)__ldg(p.val + idx[j]) : 1ll;
  }
  const uint32_t before = (r0 > 0 && r0 - 1 < p.n) ? p.skey[r0 - 1] : 0u;
  uint32_t heads = 0, nh = 0;
#pragma unroll
  for (int j = 0; j < SR_ITEMS; ++j) {
    const uint32_t prev = j ? key[j - 1] : before;
    const bool h = (full || r0 + j < p.n) && (r0 + j == 0 || key[j] != prev);
    heads |= (uint32_t)h << j;
    nh += h;
  }
  // heads strictly before this thread's first row (global group index)
  uint32_t inc = nh;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_heads[warp] = inc;
  // rows: lead (before the first head), whole groups, tail (from the last head)
  SrAgg lead = sr_empty(), cur = sr_empty();
  __syncthreads();
  uint32_t wpre = 0, btot = 0;
#pragma unroll
  for (int w = 0; w < SR_THREADS / 32; ++w) {
    if (w < warp) wpre += s_heads[w];
    btot += s_heads[w];
  }
  const uint64_t gfirst = p.tile_heads[tile] + wpre + inc - nh;
  uint64_t g = gfirst;
  bool have = false;
  uint32_t cur_key = 0;
#pragma unroll
  for (int j = 0; j < SR_ITEMS; ++j) {
    if (!full && r0 + j >= p.n) break;
    if ((heads >> j) & 1u) {
      if (have) sr_store(p, g - 1, cur_key, true, cur);
      else lead = cur;
      have = true;
      cur = sr_empty();
      cur_key = key[j];
      ++g;
    }
    sr_acc(cur, val[j]);
  }
  if (!have) lead = cur;
  // block-wide inclusive segmented scan of (have, tail)
  SrSeg x{have ? 1u : 0u, have ? cur_key : key[0], have ? cur : lead};
  SrSeg incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const SrSeg y = sr_shfl_up(incl, o);
    if (lane >= o) incl = sr_combine(y, incl);
  }
  SrSeg wex = sr_shfl_up(incl, 1);
  if (lane == 0) wex = SrSeg{0u, 0u, sr_empty()};
  if (lane == 31) s_seg[warp] = incl;
  __syncthreads();
  SrSeg pre{0u, 0u, sr_empty()};
  for (int w = 0; w < warp; ++w) pre = sr_combine(pre, s_seg[w]);
  const SrSeg ex = sr_combine(pre, wex);
  if (have) {
    // the group that ends just before this thread's first head
    const SrAgg tot = sr_join(ex.a, lead);
    const uint32_t k = ex.f ? ex.key : (lead.cnt ? key[0] : before);
    sr_store(p, gfirst - 1, k, ex.f != 0, tot);
  }
  if (tid == SR_THREADS - 1) {
    const SrSeg all = sr_combine(pre, incl);
    const uint64_t nx = t0 + SR_TILE;  // first row of the next tile
    const bool ends = nx >= p.n || p.skey[nx] != p.skey[nx - 1];
    if (all.f) {
      sr_store(p, p.tile_heads[tile] + btot - 1, all.key, ends, all.a);
    } else {
      sr_store(p, p.tile_heads[tile] - 1, p.skey[t0], false, all.a);
    }
  }
  }
}

// Minimum and maximum of the values (mm[0], mm[1]).
__global__ void k_vrange_init(long long *mm) {
  mm[0] = INT64_MAX;
  mm[1] = INT64_MIN;
}

__global__ void __launch_bounds__(256) k_vrange(const long long *v, uint64_t n, long long *mm) {
  long long lo = INT64_MAX, hi = INT64_MIN;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t done = 0;
  if (((uintptr_t)v & 15u) == 0) {
    // four 16-byte loads of a thread in flight together (one at a time left
    // the read latency-bound)
    constexpr int U = 4;
    const longlong2 *v2 = reinterpret_cast<const longlong2 *>(v);
    const uint64_t n2 = n / 2;
    uint64_t i = i0;
    for (; i + (U - 1) * stride < n2; i += U * stride) {
      longlong2 x[U];
#pragma unroll
      for (int u = 0; u < U; ++u) x[u] = __ldcs(v2 + i + u * stride);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        lo = min(lo, min(x[u].x, x[u].y));
        hi = max(hi, max(x[u].x, x[u].y));
      }
    }
    for (; i < n2; i += stride) {
      const longlong2 x = __ldcs(v2 + i);
      lo = min(lo, min(x.x, x.y));
      hi = max(hi, max(x.x, x.y));
    }
    done = n2 * 2;
  }
  for (uint64_t i = done + i0; i < n; i += stride) {
    const long long x = v[i];
    lo = min(lo, x);
    hi = max(hi, x);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}

// The payload path takes the rows when max - min fits 32 bits, else the
// row-id path does.
__global__ void k_vrange_pick(const long long *mm, uint64_t n, uint64_t *n_pay, uint64_t *n_idx) {
  const bool fits = (unsigned long long)mm[1] - (unsigned long long)mm[0] <= 0xFFFFFFFFull;
  *n_pay = fits ? n : 0;
  *n_idx = fits ? 0 : n;
}

struct GbLayout {
  int mode;
  uint32_t sub_cap, npasses, wrep;
  uint32_t part_bits;   // GB_PART: hash partitions 2^part_bits
  size_t gtab, ngroups, ckey, cslot, skey, sslot, sort_ws, pkey, pval, vrange, total;
};

bool gb_force_direct() {
  static const bool d = [] {
    const char *e = getenv("PIMDAL_GROUP_DIRECT");
    return e && atoi(e) != 0;
  }();
  return d;
}

// The partition request of GB_PART (keys only; the values travel as 64-bit
// words beside them).
pimdal_sort_arguments_t gb_part_args(const pimdal_aggr_arguments_t *a, uint32_t bits) {
  pimdal_sort_arguments_t sa{};
  sa.nr_elements = a->size;
  sa.key_dtype = PIMDAL_U32;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;
  sa.begin_bit = 32 - bits;
  sa.end_bit = 32;
  return sa;
}

// Bytes of one global sub-table (an L2-sized slice of the table that one
// aggregation launch updates); PIMDAL_GROUP_L2_BUDGET_MB overrides it.
uint64_t gb_l2_budget() {
  static const uint64_t b = [] {
    const char *e = getenv("PIMDAL_GROUP_L2_BUDGET_MB");
    const long long mb = e ? atoll(e) : 0;
    return mb > 0 ? (uint64_t)mb << 20 : GB_L2_BUDGET;
  }();
  return b;
}

// An autotuned choice for the high-cardinality hash modes: mode GB_PART with
// 2^part_bits partitions, or GB_DIRECT; mode < 0 keeps the library's choice.
struct GbTune {
  int mode = -1;
  uint32_t part_bits = 0;
};

bool gb_layout(const pimdal_aggr_arguments_t *a, GbLayout *l, const GbTune *tune = nullptr) {
  const bool sort = a->method == PIMDAL_GROUP_SORT;
  size_t o = 0;
  pimdal_sort_arguments_t sa{};
  size_t w = 0;
  if (sort) {
    sa.nr_elements = a->size;
    if (pimdal_sort_workspace_size(&sa, &w)) return false;
    l->mode = -1;
    l->sub_cap = l->npasses = l->wrep = 0;
    l->vrange = o; o += 256;  // min, max, rows of the payload and row-id paths
    l->ngroups = o; o += pd_align_up(8 * (pd_ceil_div(a->size, SR_TILE) + 1), 256);
    l->skey = o; o += pd_align_up(4 * a->size, 256);
    l->sslot = o; o += pd_align_up(4 * a->size, 256);
    l->sort_ws = o; o += w;
    l->total = o;
    return true;
  }
  uint64_t expect = a->expected_groups ? a->expected_groups : std::min<uint64_t>(a->size, 1ull << 22);
  expect = std::max<uint64_t>(expect, 1);
  l->mode = expect <= GB_WARP_MAX_GROUPS ? GB_WARP : expect <= GB_SMEM_MAX_GROUPS ? GB_SMEM
          : gb_force_direct() ? GB_DIRECT : GB_PART;
  if (tune && tune->mode >= 0 && l->mode >= GB_DIRECT) l->mode = tune->mode;
  l->part_bits = 0;
  l->pkey = l->pval = 0;
  if (l->mode == GB_PART) {
    uint32_t b = 1;
    while (b < GB_PART_MAX_BITS && (expect >> b) > GB_PART_GROUPS) ++b;
    if (tune && tune->mode == GB_PART && tune->part_bits >= 1 && tune->part_bits <= GB_PART_MAX_BITS)
      b = tune->part_bits;
    l->part_bits = b;
  }
  // GB_WARP replicas: keep each replica's load at or below 1/3
  l->wrep = expect <= 16 ? 4 : expect <= 32 ? 2 : 1;
  // load factor 1/2 for the small tables, 3/4 for the large ones
  uint64_t slots = l->mode >= GB_DIRECT ? expect + expect / 3 + 1 : 2 * expect;
  slots = std::max<uint64_t>(slots, 2048);
  if (slots >= (1ull << 31)) return false;
  uint64_t np = 1;
  if (l->mode == GB_DIRECT) np = std::max<uint64_t>(1, pd_ceil_div(32 * slots, gb_l2_budget()));
  l->npasses = (uint32_t)np;
  l->sub_cap = (uint32_t)pd_ceil_div(slots, np);
  const uint64_t cap = (uint64_t)l->sub_cap * np;
  l->gtab = o; o += pd_align_up(32 * cap, 256);
  l->ngroups = o; o += 256;
  l->ckey = o; o += pd_align_up(4 * cap, 256);
  l->cslot = o; o += pd_align_up(4 * cap, 256);
  l->skey = o; o += pd_align_up(4 * cap, 256);
  l->sslot = o; o += pd_align_up(4 * cap, 256);
  sa.nr_elements = cap;
  if (pimdal_sort_workspace_size(&sa, &w)) return false;
  if (l->mode == GB_PART) {
    // the partition's scratch and the final sort's run one after the other
    const pimdal_sort_arguments_t pa = gb_part_args(a, l->part_bits);
    const size_t pw = pd_partition_workspace(&pa, a->in_val != nullptr);
    if (!pw) return false;
    w = std::max(w, pw);
    l->pkey = o; o += pd_align_up(4 * a->size, 256);
    if (a->in_val) { l->pval = o; o += pd_align_up(8 * a->size, 256); }
  }
  l->sort_ws = o; o += w;
  l->total = o;
  return true;
}

}  // namespace

void pd_gb_mode(uint64_t expect, uint32_t *mode, uint32_t *wrep) {
  expect = std::max<uint64_t>(expect, 1);
  *mode = expect <= GB_WARP_MAX_GROUPS ? GB_WARP : expect <= GB_SMEM_MAX_GROUPS ? GB_SMEM : GB_DIRECT;
  *wrep = expect <= 16 ? 4 : expect <= 32 ? 2 : 1;
}

size_t pd_gb_batch_shared_bytes() { return GB_SMEM_BYTES + 2 * GB_SMEM_SLOTS; }

int pd_gb_batch_run(pimdal_ctx *ctx, const pd_gb_batch &b, cudaStream_t s) {
  const unsigned grid = (unsigned)std::min<uint64_t>(pd_ceil_div(std::max<uint64_t>(b.total_slots, 1), 256),
                                                     ctx->sm_count * 8ull);
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gbb_init<<<grid, 256, 0, s>>>(b);
  }
  if (b.nitems) {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_GROUP, s);
    const size_t smem = pd_gb_batch_shared_bytes();
    PD_CHECK_CUDA(cudaFuncSetAttribute(k_gbb_aggregate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gbb_aggregate<<<std::min<unsigned>(ctx->sm_count, b.nitems), GB_THREADS, smem, s>>>(b);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gbb_compact<<<grid, 256, 0, s>>>(b);
  }
  int st;
  pimdal_sort_arguments_t sa{};
  sa.key_dtype = PIMDAL_U32;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;
  sa.nr_elements = std::max<uint64_t>(b.total_slots, 1);
  sa.in = b.ckey;
  sa.in_ptr = b.cslot;
  sa.out = b.skey;
  sa.out_ptr = b.sslot;
  if ((st = pd_sort_ex2(ctx, &sa, PD_KEY_PLAIN, b.sort_ws, s, nullptr, (const uint64_t *)b.ngroups)))
    return st;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gbb_inst<<<grid, 256, 0, s>>>(b);
  }
  sa.in = b.ikey;
  sa.in_ptr = b.islot;
  sa.out = b.ckey;
  sa.out_ptr = b.cslot;
  sa.begin_bit = 0;
  sa.end_bit = b.inst_bits;
  if ((st = pd_sort_ex2(ctx, &sa, PD_KEY_PLAIN, b.sort_ws, s, nullptr, (const uint64_t *)b.ngroups)))
    return st;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gbb_start<<<1, 1024, 0, s>>>(b);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gbb_gather<<<grid, 256, 0, s>>>(b);
  }
  return pd_launch_status(ctx);
}

namespace {
// The autotuner's candidates for a high-cardinality hash group-by: the
// partitioned mode at the suggested partition count and its neighbours, and
// the direct global table.  Empty when there is nothing to choose.
std::vector<GbTune> gb_candidates(const pimdal_aggr_arguments_t *a) {
  std::vector<GbTune> c;
  GbLayout l;
  if (a->method == PIMDAL_GROUP_SORT || !gb_layout(a, &l) || l.mode < GB_DIRECT) return c;
  GbLayout p;
  GbTune t;
  t.mode = GB_PART;
  if (!gb_layout(a, &p, &t)) return c;
  for (int d = -1; d <= 1; ++d) {
    const int b = (int)p.part_bits + d;
    if (b < 1 || b > (int)GB_PART_MAX_BITS) continue;
    t.part_bits = (uint32_t)b;
    c.push_back(t);
  }
  t.mode = GB_DIRECT;
  t.part_bits = 0;
  c.push_back(t);
  return c;
}

std::vector<uint64_t> gb_shape(const pimdal_aggr_arguments_t *a) {
  const uint64_t outs = (a->out_sum != nullptr) | (a->out_count != nullptr) << 1 |
                        (a->out_min != nullptr) << 2 | (a->out_max != nullptr) << 3;
  return {2, pd_log2_ceil(a->size), pd_log2_ceil(a->expected_groups), a->in_val != nullptr, outs};
}

GbTune gb_cached(const pimdal_ctx *ctx, const pimdal_aggr_arguments_t *a) {
  GbTune t;
  if (a->method == PIMDAL_GROUP_SORT) return t;
  const auto it = ctx->op_tune.find(gb_shape(a));
  if (it != ctx->op_tune.end() && it->second.group_mode) {
    t.mode = it->second.group_mode == 1 ? GB_PART : GB_DIRECT;
    t.part_bits = it->second.group_part_bits;
  }
  return t;
}
}  // namespace

extern "C" int pimdal_group_workspace_size(const pimdal_aggr_arguments_t *a, size_t *bytes) {
  if (!a || !bytes) return PIMDAL_ERR_ARG;
  GbLayout l;
  if (!gb_layout(a, &l)) return PIMDAL_ERR_ARG;
  *bytes = l.total;
  for (const auto &t : gb_candidates(a)) {  // a tuned choice may be used instead
    GbLayout m;
    if (gb_layout(a, &m, &t)) *bytes = std::max(*bytes, m.total);
  }
  return PIMDAL_OK;
}

namespace {
int group_kernel_tuned(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *a,
                       pimdal_aggr_results_t *d_result, pimdal_stream_t stream,
                       const GbTune &tune);
}  // namespace

extern "C" int pimdal_group_kernel(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *a,
                                   pimdal_aggr_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result) return PIMDAL_ERR_ARG;
  return group_kernel_tuned(ctx, a, d_result, stream, gb_cached(ctx, a));
}

extern "C" int pimdal_group_autotune(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *a,
                                     pimdal_aggr_results_t *d_result, pimdal_tuning_t *best,
                                     int *cached, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result || !best) return PIMDAL_ERR_ARG;
  if (cached) *cached = 0;
  *best = pimdal_tuning_t{};
  const auto cands = gb_candidates(a);
  if (cands.empty())  // nothing to choose: the library's choice
    return pimdal_group_kernel(ctx, a, d_result, stream);
  const auto key = gb_shape(a);
  const auto it = ctx->op_tune.find(key);
  if (it != ctx->op_tune.end()) {
    *best = it->second;
    best->candidates = 0;
    if (cached) *cached = 1;
    return PIMDAL_OK;
  }
  cudaStream_t s = (cudaStream_t)stream;
  float best_ms = -1.f;
  size_t best_i = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    auto run = [&] { return group_kernel_tuned(ctx, a, d_result, stream, cands[i]); };
    if (pd_time_call(ctx, s, run) < 0.f) continue;  // warm-up
    const float ms = pd_time_call(ctx, s, run);
    if (ms >= 0.f && (best_ms < 0.f || ms < best_ms)) {
      best_ms = ms;
      best_i = i;
    }
  }
  if (best_ms < 0.f) return PIMDAL_ERR_CUDA;
  pimdal_tuning_t t{};
  t.group_mode = cands[best_i].mode == GB_PART ? 1 : 2;
  t.group_part_bits = cands[best_i].part_bits;
  t.ms = best_ms;
  t.candidates = (uint32_t)cands.size();
  ctx->op_tune[key] = t;
  *best = t;
  return group_kernel_tuned(ctx, a, d_result, stream, cands[best_i]);
}

namespace {
int group_kernel_tuned(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *a,
                       pimdal_aggr_results_t *d_result, pimdal_stream_t stream,
                       const GbTune &tune) {
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
  if (!gb_layout(a, &l, &tune)) return PIMDAL_ERR_ARG;
  int st;
  char *ws = (char *)pd_workspace(ctx, l.total, s, &st);
  if (!ws) return st;
  pimdal_sort_arguments_t sa{};
  sa.key_dtype = a->key_dtype;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;

  if (a->method == PIMDAL_GROUP_SORT) {
    long long *mm = (long long *)(ws + l.vrange);
    uint64_t *n_pay = (uint64_t *)(mm + 2), *n_idx = n_pay + 1;
    sa.nr_elements = a->size;
    sa.in = a->in;
    sa.in_ptr = nullptr;
    sa.out = ws + l.skey;
    SegParams p{};
    p.skey = (const uint32_t *)(ws + l.skey);
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
    auto reduce = [&](const SegParams &q) -> int {
      const unsigned sr_grid = (unsigned)std::min<uint64_t>(q.tiles, ctx->sm_count * 8ull);
      {
        pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
        k_sr_heads<<<sr_grid, SR_THREADS, 0, s>>>(q);
      }
      {
        pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
        k_sr_scan<<<1, 1024, 0, s>>>(q);
      }
      {
        pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
        k_sr_init<<<ctx->sm_count * 8, 256, 0, s>>>(q);
      }
      {
        pd_launch_scope sc(ctx, PIMDAL_KERNEL_SEGREDUCE, s);
        k_gb_segreduce<<<sr_grid, SR_THREADS, 0, s>>>(q);
      }
      return pd_launch_status(ctx);
    };
    if (!a->in_val) {  // COUNT only: the keys alone
      sa.out_ptr = nullptr;
      if ((st = pd_sort_with_workspace(ctx, &sa, ws + l.sort_ws, s))) return st;
      return reduce(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_vrange_init<<<1, 1, 0, s>>>(mm);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      const unsigned g = (unsigned)std::min<uint64_t>(pd_ceil_div(a->size, 512), ctx->sm_count * 8ull);
      k_vrange<<<g, 256, 0, s>>>((const long long *)a->in_val, a->size, mm);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_vrange_pick<<<1, 1, 0, s>>>(mm, a->size, n_pay, n_idx);
    }
    sa.out_ptr = (uint32_t *)(ws + l.sslot);
    p.sidx = (const uint32_t *)(ws + l.sslot);
    // payload path: value - min sorted beside the key
    if ((st = pd_sort_pay64(ctx, &sa, ws + l.sort_ws, s, n_pay, a->in_val, (const int64_t *)mm)))
      return st;
    SegParams q = p;
    q.pay_min = mm;
    q.n_dev = n_pay;
    if ((st = reduce(q))) return st;
    // row-id path: values gathered by row id
    if ((st = pd_sort_ex2(ctx, &sa, PD_KEY_PLAIN, ws + l.sort_ws, s, nullptr, n_idx))) return st;
    q = p;
    q.val = a->in_val;
    q.n_dev = n_idx;
    return reduce(q);
  }

  GbParams p{};
  p.key = (const uint32_t *)a->in;
  p.val = a->in_val;
  p.n = a->size;
  p.vec = ((uintptr_t)a->in & 15u) == 0 && ((uintptr_t)a->in_val & 15u) == 0;
  p.gtab = (unsigned long long *)(ws + l.gtab);
  p.sub_cap = l.sub_cap;
  p.npasses = l.npasses;
  p.wrep = l.wrep;
  p.ngroups = (unsigned long long *)(ws + l.ngroups);
  p.ckey = (uint32_t *)(ws + l.ckey);
  p.cslot = (uint32_t *)(ws + l.cslot);
  p.d_error = ctx->d_error;
  const uint64_t cap = (uint64_t)l.sub_cap * l.npasses;
  const unsigned init_grid = (unsigned)std::min<uint64_t>(pd_ceil_div(cap, 256), ctx->sm_count * 8ull);
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gb_init<<<init_grid, 256, 0, s>>>(p);
  }
  const uint64_t want = pd_ceil_div(a->size, (uint64_t)GB_THREADS * 4);
  if (l.mode == GB_PART) {
    // rows grouped by the top part_bits of the key's multiplicative hash
    pimdal_sort_arguments_t pa = gb_part_args(a, l.part_bits);
    pa.in = a->in;
    pa.out = ws + l.pkey;
    int64_t *pval = a->in_val ? (int64_t *)(ws + l.pval) : nullptr;
    if ((st = pd_partition(ctx, &pa, PD_KEY_MULHASH, ws + l.sort_ws, s, (const uint64_t *)a->in_val,
                           (uint64_t *)pval)))
      return st;
    p.key = (const uint32_t *)(ws + l.pkey);
    p.val = pval;
    p.vec = 1;
    // a chunk holds at most about one partition's rows, so at most about
    // 2 * GB_PART_GROUPS groups; with few partitions it is cut further so
    // that every SM gets several chunks
    const uint64_t per_sm = pd_ceil_div(a->size, 8ull * ctx->sm_count);
    const uint64_t chunk = std::max<uint64_t>(
        4096, pd_align_up(std::min<uint64_t>(a->size >> l.part_bits, per_sm), 1024));
    const unsigned grid = (unsigned)std::min<uint64_t>(pd_ceil_div(a->size, chunk), ctx->sm_count);
    const size_t smem = pd_gb_batch_shared_bytes();
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_GROUP, s);
    PD_CHECK_CUDA(cudaFuncSetAttribute(k_gb_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gb_chunks<<<grid ? grid : 1, GB_THREADS, smem, s>>>(p, chunk, ctx->d_counters + PD_COUNTER_GROUP);
  } else if (l.mode == GB_DIRECT) {
    const unsigned grid = (unsigned)std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 2);
    for (uint32_t q = 0; q < l.npasses; ++q) {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_GROUP, s);
      k_gb_aggregate<GB_DIRECT><<<grid ? grid : 1, GB_THREADS, 0, s>>>(p, q);
    }
  } else {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_GROUP, s);
    const unsigned grid = (unsigned)std::min<uint64_t>(want, (uint64_t)ctx->sm_count);
    auto k = l.mode == GB_WARP ? k_gb_aggregate<GB_WARP> : k_gb_aggregate<GB_SMEM>;
    PD_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GB_SMEM_BYTES));
    k<<<grid ? grid : 1, GB_THREADS, GB_SMEM_BYTES, s>>>(p, 0);
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
  g.gtab = p.gtab;
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
}  // namespace
