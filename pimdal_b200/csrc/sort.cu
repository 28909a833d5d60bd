// K-SORT: stable onesweep LSD radix sort of (uint32/int32 key, uint32 row id)
// (pimdal_sort_kernel).
//
// Reference behaviour: sort_kernel / sort_part_kernel (pimdal/sort/sort.h:7-25,
// sort_keyval.c:37-179) range-partition key_ptr pairs and quicksort each
// bucket (not stable); the CPU operator reference/db_operators/sort.cpp:30-40
// sorts one key column ascending.  This operator returns the stable
// ascending order of (key, row id) pairs, row ids fused in from the index
// when no row-id column is given (the create_ptr glue of
// pimdal/main/sort/dpu/kernel_sort.c).
//
// B200 design (HBM-bound, no tensor cores):
//  1. k_sort_hist: one read of the keys builds the 256-bin histograms of all
//     digit positions (warp-private shared-memory counters).
//  2. k_sort_plan (one CTA): exclusive scans of the histograms; a pass whose
//     digit is the same for every key (count == n) is skipped; buffers are
//     routed so the last active pass writes the caller's output.  Computed on
//     the device, so the whole sort is stream-ordered and capturable.
//  3. k_sort_pass, once per digit: a CTA takes the next tile of RS_TILE keys
//     (atomic tile counter, so tiles are processed in input order), counts
//     its digits and publishes the counts early, ranks keys per warp
//     (shared-memory lane masks group the lanes of one digit), resolves the
//     digits' global offsets with a per-digit decoupled look-back, stages the
//     tile in shared memory in digit order and writes each digit run
//     contiguously.
#include <algorithm>

#include "common.cuh"

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
#ifndef PD_RS_ITEMS
#define PD_RS_ITEMS 20  // keys per thread of a digit-pass tile (measured best with 3 CTAs per SM)
#endif
#ifndef PD_RS_MIN_CTAS
#define PD_RS_MIN_CTAS 3  // CTAs per SM the pass is compiled for (register budget)
#endif
#ifndef PD_RS_MATCH
// lanes sharing a digit in full tiles: 0 one ballot per digit bit, 1
// shared-memory atomicOr masks
#define PD_RS_MATCH 1
#endif
#ifndef PD_RS_WFULL
#define PD_RS_WFULL 1  // 1: full tiles write their staged keys in a fully unrolled loop
#endif
constexpr int RS_ITEMS = PD_RS_ITEMS;
constexpr int RS_WARP_TILE = 32 * RS_ITEMS;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_MIN_CTAS = PD_RS_MIN_CTAS;
static_assert(RS_ITEMS % 2 == 0 && RS_TILE <= 65536, "16-bit packed staged positions");
constexpr int RS_RADIX_BITS = 8;
constexpr int RS_RADIX = 1 << RS_RADIX_BITS;       // 256 (== RS_THREADS)
constexpr int RS_MAX_PASSES = 4;
constexpr uint32_t RS_FLAG_AGG = 1u << 30, RS_FLAG_INC = 2u << 30, RS_COUNT_MASK = (1u << 30) - 1;
static_assert(RS_RADIX == RS_THREADS, "one thread per digit");
// The atomicOr masks (two per warp and digit) borrow the staging buffer
// during the ranking; it must hold them even for keys alone.
constexpr int RS_MATCH_WORDS = 2 * RS_WARPS * RS_RADIX;
static_assert(PD_RS_MATCH == 0 || RS_MATCH_WORDS <= RS_TILE, "match masks fit the key staging");

enum : uint32_t { BUF_IN = 0, BUF_OUT = 1, BUF_ALT = 2 };

struct SortPlan {
  uint32_t active[RS_MAX_PASSES];
  uint32_t src[RS_MAX_PASSES];
  uint32_t dst[RS_MAX_PASSES];
  uint32_t first[RS_MAX_PASSES];  // first active pass (reads the input row ids)
  uint32_t n_active;
};

struct SortParams {
  const void *in;
  const uint32_t *in_ptr;  // NULL: row id = ptr_base + index
  uint64_t ptr_base;
  void *out;
  uint32_t *out_ptr;
  uint32_t *alt_key, *alt_ptr;
  // 64-bit values carried beside the keys (the small-radix pass only)
  const unsigned long long *in_v64;
  unsigned long long *out_v64, *alt_v64;
  uint32_t dbits;       // digit width of every pass (8; at most 6 for partitions)
  // 32-bit payload of the first pass taken as pay64[i] - *pay_min (when
  // pay64 is set and no row-id column is given): int64 values whose range
  // fits 32 bits travel through the sort in place of row ids
  const long long *pay64;
  const long long *pay_min;
  uint64_t n;           // element count (upper bound when n_dev is set)
  const uint64_t *n_dev;  // device-resident element count, or NULL
  uint32_t flip;        // 0x80000000 for signed keys
  int key_mode;         // digits of: 0 the key, 1 hash0(key), 2 multiplicative hash
  uint32_t begin_bit, end_bit, npasses;
  int pairs;            // in/out are key_ptr32 arrays
  int has_vals;
  uint32_t *hist;       // [RS_MAX_PASSES][RS_RADIX]
  uint32_t *offsets;    // [RS_MAX_PASSES][RS_RADIX]
  SortPlan *plan;
  uint32_t *status;     // [RS_MAX_PASSES][tiles][RS_RADIX]
  uint32_t *counters;   // [RS_MAX_PASSES]
  uint64_t tiles;
  uint32_t *d_error;
};

__device__ __forceinline__ uint64_t sort_n(const SortParams &p) { return p.n_dev ? *p.n_dev : p.n; }

__device__ __forceinline__ uint32_t load_key_in(const SortParams &p, uint64_t i) {
  return p.pairs ? reinterpret_cast<const uint2 *>(p.in)[i].x
                 : reinterpret_cast<const uint32_t *>(p.in)[i];
}

// ---------------------------------------------------------------- histogram
template <int KEY_MODE>
__device__ __forceinline__ uint32_t hist_xform(uint32_t k, uint32_t flip) {
  if (KEY_MODE == PD_KEY_HASH0) return pd_hash0(k);
  if (KEY_MODE == PD_KEY_MULHASH) return pd_mulhash32(k);
  return k ^ flip;
}

template <int KEY_MODE>
__global__ void __launch_bounds__(RS_THREADS) k_sort_hist(SortParams p) {
  __shared__ uint32_t sh[RS_WARPS][RS_MAX_PASSES][RS_RADIX];
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < RS_WARPS * RS_MAX_PASSES * RS_RADIX; i += RS_THREADS)
    (&sh[0][0][0])[i] = 0;
  uint32_t shift[RS_MAX_PASSES], mask[RS_MAX_PASSES];
#pragma unroll
  for (int q = 0; q < RS_MAX_PASSES; ++q) {
    shift[q] = min(31u, p.begin_bit + q * p.dbits);
    uint32_t bits = q < (int)p.npasses ? min(p.dbits, p.end_bit - shift[q]) : 0u;
    mask[q] = (1u << bits) - 1u;
  }
  __syncthreads();
  uint32_t (*h)[RS_RADIX] = sh[warp];
  const uint32_t np = p.npasses, flip = p.flip;
  auto add = [&](uint32_t k) {
    const uint32_t t = hist_xform<KEY_MODE>(k, flip);
#pragma unroll
    for (int q = 0; q < RS_MAX_PASSES; ++q)
      if (q < (int)np) atomicAdd(&h[q][(t >> shift[q]) & mask[q]], 1u);
  };
  const uint64_t stride = (uint64_t)gridDim.x * RS_THREADS;
  const bool vec = !p.pairs && ((uintptr_t)p.in & 15u) == 0;
  const uint64_t n = sort_n(p);
  uint64_t done = 0;
  // U loads of a thread are in flight together (one 16-byte load
  // at a time left the read latency-bound at about 2.4 TB/s)
  constexpr int U = 4;
  if (vec) {
    const uint4 *in4 = reinterpret_cast<const uint4 *>(p.in);
    const uint64_t n4 = n / 4;
    uint64_t i = (uint64_t)blockIdx.x * RS_THREADS + tid;
    for (; i + (U - 1) * stride < n4; i += U * stride) {
      uint4 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) v[u] = __ldcs(in4 + i + u * stride);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        add(v[u].x);
        add(v[u].y);
        add(v[u].z);
        add(v[u].w);
      }
    }
    for (; i < n4; i += stride) {
      const uint4 v = __ldcs(in4 + i);
      add(v.x);
      add(v.y);
      add(v.z);
      add(v.w);
    }
    done = n4 * 4;
  }
  uint64_t i = done + (uint64_t)blockIdx.x * RS_THREADS + tid;
  for (; i + (U - 1) * stride < n; i += U * stride) {
    uint32_t k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) k[u] = load_key_in(p, i + u * stride);
#pragma unroll
    for (int u = 0; u < U; ++u) add(k[u]);
  }
  for (; i < n; i += stride) add(load_key_in(p, i));
  __syncthreads();
  for (uint32_t q = 0; q < p.npasses; ++q) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) s += sh[w][q][tid];
    if (s) atomicAdd(&p.hist[q * RS_RADIX + tid], s);
  }
}

// Block-wide exclusive scan of one value per thread (RS_THREADS threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *s_warp,
                                                         uint32_t *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  uint32_t wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < RS_WARPS; ++w) {
    uint32_t x = s_warp[w];
    if (w < warp) wpre += x;
    tot += x;
  }
  __syncthreads();
  if (total) *total = tot;
  return wpre + inc - v;
}

// -------------------------------------------------------------------- plan
__global__ void __launch_bounds__(RS_THREADS) k_sort_plan(SortParams p) {
  __shared__ uint32_t s_warp[RS_WARPS];
  __shared__ uint32_t s_trivial[RS_MAX_PASSES];
  const int d = threadIdx.x;
  const uint64_t n = sort_n(p);
  if (d < RS_MAX_PASSES) s_trivial[d] = 0;
  __syncthreads();
  for (uint32_t q = 0; q < p.npasses; ++q) {
    uint32_t c = p.hist[q * RS_RADIX + d];
    if ((uint64_t)c == n) s_trivial[q] = 1;
    p.offsets[q * RS_RADIX + d] = block_exclusive_scan(c, s_warp, nullptr);
  }
  __syncthreads();
  if (d == 0) {
    SortPlan pl{};
    uint32_t m = 0;
    for (uint32_t q = 0; q < p.npasses; ++q) {
      pl.active[q] = !s_trivial[q];
      m += pl.active[q];
    }
    pl.n_active = m;
    uint32_t j = 0, prev = BUF_IN;
    for (uint32_t q = 0; q < p.npasses; ++q) {
      if (!pl.active[q]) continue;
      ++j;
      pl.src[q] = prev;
      pl.dst[q] = ((m - j) % 2 == 0) ? BUF_OUT : BUF_ALT;
      pl.first[q] = (j == 1);
      prev = pl.dst[q];
    }
    *p.plan = pl;
  }
}

// No active pass (all keys share every digit, or n small): copy in -> out.
__global__ void __launch_bounds__(RS_THREADS) k_sort_copy(SortParams p) {
  if (p.plan->n_active != 0) return;
  const uint64_t stride = (uint64_t)gridDim.x * RS_THREADS;
  const uint64_t n = sort_n(p);
  for (uint64_t i = (uint64_t)blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += stride) {
    uint32_t k, v;
    if (p.pairs) {
      uint2 e = reinterpret_cast<const uint2 *>(p.in)[i];
      k = e.x;
      v = e.y;
    } else {
      k = reinterpret_cast<const uint32_t *>(p.in)[i];
      v = p.in_ptr ? p.in_ptr[i]
          : p.pay64 ? (uint32_t)(p.pay64[i] - *p.pay_min) : (uint32_t)(p.ptr_base + i);
    }
    if (p.pairs) reinterpret_cast<uint2 *>(p.out)[i] = make_uint2(k, v);
    else {
      reinterpret_cast<uint32_t *>(p.out)[i] = k;
      if (p.has_vals) p.out_ptr[i] = v;
      if (p.out_v64) p.out_v64[i] = p.in_v64[i];
    }
  }
}

// ------------------------------------------------------------ onesweep pass
template <int KEY_MODE>
__device__ __forceinline__ uint32_t sort_xform(uint32_t k, uint32_t flip) {
  if (KEY_MODE == PD_KEY_HASH0) return pd_hash0(k);
  if (KEY_MODE == PD_KEY_MULHASH) return pd_mulhash32(k);
  return k ^ flip;
}

// Decoupled look-back of one digit: the sum of the digit's counts in tiles
// before `tile`, read RS_LOOKBACK predecessor words per round (independent
// relaxed loads -- every word carries its own count, nothing else is read),
// then this tile's inclusive count published.  `st` is the digit's status
// word of tile 0; `count` is the tile's own count.  A wait that gives up
// sets the timeout bit and publishes what it has (the pass is then reported
// as failed).
#ifndef PD_RS_LOOKBACK
#define PD_RS_LOOKBACK 4  // predecessor words per look-back round of the digit pass
#endif
template <int RS_LOOKBACK>
__device__ __forceinline__ uint32_t rs_lookback(uint32_t *st, uint64_t tile, uint32_t count,
                                                uint32_t *d_error) {
  uint32_t excl = 0;
  int64_t t = (int64_t)tile - 1;
  uint32_t spins = 0;
  const uint64_t t0 = pd_globaltimer_ns();
  while (t >= 0) {
    uint32_t w[RS_LOOKBACK];
#pragma unroll
    for (int i = 0; i < RS_LOOKBACK; ++i)
      w[i] = (t - i >= 0) ? pd_load_relaxed_u32(st + (uint64_t)(t - i) * RS_RADIX) : RS_FLAG_INC;
    int used = 0;
    bool done = false, stalled = false;
#pragma unroll
    for (int i = 0; i < RS_LOOKBACK; ++i) {
      if (done || stalled) continue;
      const uint32_t flag = w[i] & ~RS_COUNT_MASK;
      if (flag == 0) {
        stalled = true;
        continue;
      }
      excl += w[i] & RS_COUNT_MASK;
      ++used;
      if (flag == RS_FLAG_INC) done = true;
    }
    if (done) break;
    t -= used;
    if (stalled) {
      if (pd_wait_expired(d_error, t0, ++spins)) break;
      __nanosleep(spins < 8 ? 64 : 256);
    }
  }
  pd_store_relaxed_u32(st + tile * RS_RADIX, RS_FLAG_INC | ((excl + count) & RS_COUNT_MASK));
  return excl;
}

// Lanes of `members` whose digit equals this lane's: one ballot per digit
// bit.  For 8-bit labels this is cheaper than the match.any instruction.
__device__ __forceinline__ unsigned match_digit(uint32_t d, unsigned members) {
  unsigned m = members;
#pragma unroll
  for (int b = 0; b < RS_RADIX_BITS; ++b) {
    const bool bit = (d >> b) & 1u;
    const unsigned v = __ballot_sync(members, bit);
    m &= bit ? v : ~v;
  }
  return m;
}

// One digit pass.  FULL tiles take a path without bounds checks; indices
// inside a tile are 32-bit; the digit is (xform(key) >> shift) & mask.
template <bool HAS_VALS, int KEY_MODE>
__global__ void __launch_bounds__(RS_THREADS, RS_MIN_CTAS)
k_sort_pass(SortParams p, uint32_t pass, uint32_t shift, uint32_t mask) {
  // the tile staged in digit order: (key, value) words, or keys alone
  extern __shared__ __align__(16) uint2 rs_stage[];  // RS_TILE (key, value) words or keys
  uint2 *s_kv = rs_stage;
  uint32_t *s_k = reinterpret_cast<uint32_t *>(rs_stage);
  __shared__ uint32_t s_whist[RS_WARPS][RS_RADIX];  // warp digit counts -> warp offsets in the digit
  __shared__ uint16_t s_wcnt[RS_WARPS][RS_RADIX];   // running staged positions of the ranking (< RS_TILE)
  __shared__ int32_t s_gdelta[RS_RADIX];
  __shared__ uint32_t s_warp[RS_WARPS];
  __shared__ uint32_t s_tile;

  const SortPlan *plan = p.plan;
  if (!plan->active[pass]) return;
  const uint32_t src = plan->src[pass], dst = plan->dst[pass];
  const bool first = plan->first[pass] != 0;
  const uint32_t flip = p.flip;
  auto dig = [&](uint32_t k) { return (sort_xform<KEY_MODE>(k, flip) >> shift) & mask; };

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // persistent: tiles are claimed in order until the input is exhausted
  for (;;) {
  __syncthreads();  // the previous tile's readers of shared memory are done
  if (tid == 0) s_tile = atomicAdd(&p.counters[pass], 1u);
#pragma unroll
  for (int w = 0; w < RS_WARPS; ++w) {
    s_whist[w][tid] = 0;
  }
#if PD_RS_MATCH == 1
#pragma unroll
  for (int j = 0; j < RS_MATCH_WORDS / (4 * RS_THREADS); ++j)
    reinterpret_cast<uint4 *>(rs_stage)[tid + j * RS_THREADS] = make_uint4(0, 0, 0, 0);
#endif
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t base = tile * (uint64_t)RS_TILE;
  const uint64_t n = sort_n(p);
  if (base >= n) break;  // past the (possibly device-resident) count: done
  const uint32_t tile_n = (uint32_t)min((uint64_t)RS_TILE, n - base);
  const bool full = tile_n == RS_TILE;
  const uint32_t wl = (uint32_t)warp * RS_WARP_TILE + lane;  // tile-local index of item 0

  // Source / destination views.  ALT is always structure-of-arrays.
  const bool src_pairs = (src != BUF_ALT) && p.pairs;
  const bool dst_pairs = (dst != BUF_ALT) && p.pairs;
  const void *skey = src == BUF_IN ? p.in : (src == BUF_OUT ? p.out : (const void *)p.alt_key);
  const uint32_t *sval = src == BUF_IN ? p.in_ptr : (src == BUF_OUT ? p.out_ptr : p.alt_ptr);
  void *dkey = dst == BUF_OUT ? p.out : (void *)p.alt_key;
  uint32_t *dval = dst == BUF_OUT ? p.out_ptr : p.alt_ptr;
  const uint32_t *skey32 = reinterpret_cast<const uint32_t *>(skey) + base;
  const uint2 *skey64 = reinterpret_cast<const uint2 *>(skey) + base;
  const uint32_t *sval32 = sval ? sval + base : nullptr;
  const bool gen_vals = first && src == BUF_IN && sval == nullptr && !src_pairs;
  const uint32_t vbase = (uint32_t)(p.ptr_base + base);
  const bool pay = gen_vals && p.pay64 != nullptr;
  const long long pmin = pay ? *p.pay_min : 0;
  const long long *spay = pay ? p.pay64 + base : nullptr;

  // Load keys and values up front (all loads in flight together):
  // warp-striped, item k of lane l is tile element wl + 32k.
  uint32_t key[RS_ITEMS];
  uint32_t val[HAS_VALS ? RS_ITEMS : 1];
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k) {
    const uint32_t li = wl + 32u * k;
    key[k] = 0;
    if (HAS_VALS) val[k] = 0;
    if (full || li < tile_n) {
      if (src_pairs) {
        uint2 e = __ldcs(skey64 + li);
        key[k] = e.x;
        if (HAS_VALS) val[k] = e.y;
      } else {
        key[k] = __ldcs(skey32 + li);
        if (HAS_VALS)
          val[k] = pay ? (uint32_t)(__ldcs(spay + li) - pmin) : gen_vals ? vbase + li : __ldcs(sval32 + li);
      }
    }
  }

  // Early counts: per-warp digit histograms (one shared atomic per key), so
  // the tile's counts are published before the ranking, and successors'
  // look-backs find them without waiting.
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k)
    if (full || wl + 32u * k < tile_n) atomicAdd(&s_whist[warp][dig(key[k])], 1u);
  __syncthreads();

  // Per digit (thread tid = digit): warp offsets, tile count, publish.
  const int d = tid;
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < RS_WARPS; ++w) {
    uint32_t t = s_whist[w][d];
    s_whist[w][d] = run;
    run += t;
  }
  const uint32_t count = run;
  uint32_t *st = p.status + ((uint64_t)pass * p.tiles) * RS_RADIX + d;
  if (tile == 0) pd_store_relaxed_u32(st, RS_FLAG_INC | count);
  else pd_store_relaxed_u32(st + tile * RS_RADIX, RS_FLAG_AGG | count);
  const uint32_t dstart = block_exclusive_scan(count, s_warp, nullptr);
  // each warp's first position of digit d in the staged tile seeds its
  // running counter, so the ranking below yields staged positions
#pragma unroll
  for (int w = 0; w < RS_WARPS; ++w) s_wcnt[w][d] = (uint16_t)(s_whist[w][d] + dstart);
  __syncthreads();

  // Warp-level stable ranking: the lanes of one digit are grouped, and the
  // lowest-numbered item and lane come first.
  uint32_t rank2[RS_ITEMS / 2];  // two 16-bit staged positions per register (< RS_TILE)
#pragma unroll
  for (int k = 0; k < RS_ITEMS / 2; ++k) rank2[k] = 0;
  const uint32_t lt = (1u << lane) - 1u;
  uint16_t *whist = s_wcnt[warp];
  if (full) {
#if PD_RS_MATCH == 1
    // Each lane sets its bit in the mask of its digit; after the warp
    // barrier the mask holds the lanes sharing the digit.  Two mask sets
    // alternate by item: the leader clears item k's mask after the shuffle
    // (every lane has read it by then), and item k+2 reuses that set only
    // after item k+1's barrier.  The barrier also orders the leaders'
    // counter updates from one item to the next.
    uint32_t *mbase = reinterpret_cast<uint32_t *>(rs_stage) + warp * 2 * RS_RADIX;
    const uint32_t lanebit = 1u << lane;
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
      const uint32_t d = dig(key[k]);
      uint32_t *mb = mbase + (k & 1) * RS_RADIX;
      atomicOr(&mb[d], lanebit);
      __syncwarp();
      const unsigned peers = mb[d];
      const int leader = 31 - __clz(peers);
      uint32_t old = 0;
      if (lane == leader) old = whist[d];
      old = __shfl_sync(0xffffffffu, old, leader);
      if (lane == leader) {
        whist[d] = (uint16_t)(old + __popc(peers));
        mb[d] = 0;
      }
      rank2[k >> 1] |= (old + __popc(peers & lt)) << (16 * (k & 1));
    }
    __syncwarp();
#else
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
      const uint32_t d = dig(key[k]);
      const unsigned peers = match_digit(d, 0xffffffffu);
      const int leader = __ffs(peers) - 1;
      uint32_t old = 0;
      if (lane == leader) {
        old = whist[d];
        whist[d] = (uint16_t)(old + __popc(peers));
      }
      old = __shfl_sync(0xffffffffu, old, leader);
      rank2[k >> 1] |= (old + __popc(peers & lt)) << (16 * (k & 1));
      __syncwarp();
    }
#endif
  } else {
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
      const bool valid = wl + 32u * k < tile_n;
      const unsigned vmask = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const uint32_t d = dig(key[k]);
        const unsigned peers = match_digit(d, vmask);
        const int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (lane == leader) {
          old = whist[d];
          whist[d] = old + __popc(peers);
        }
        old = __shfl_sync(vmask, old, leader);
        rank2[k >> 1] |= (old + __popc(peers & lt)) << (16 * (k & 1));
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // The digit's global offset.  (Looking back before the ranking instead,
  // to publish the inclusive counts earlier, was measured no faster.)
  const uint32_t excl = tile > 0 ? rs_lookback<PD_RS_LOOKBACK>(st, tile, count, p.d_error) : 0u;
  s_gdelta[d] = (int32_t)(p.offsets[pass * RS_RADIX + d] + excl) - (int32_t)dstart;
  __syncthreads();

  // Stage the tile in digit order.
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k) {
    if (full || wl + 32u * k < tile_n) {
      const uint32_t pos = (rank2[k >> 1] >> (16 * (k & 1))) & 0xFFFFu;
      if (HAS_VALS) s_kv[pos] = make_uint2(key[k], val[k]);
      else s_k[pos] = key[k];
    }
  }
  __syncthreads();

  // Write each digit run contiguously (global index < 2^30).
  uint32_t *dkey32 = reinterpret_cast<uint32_t *>(dkey);
  uint2 *dkey64 = reinterpret_cast<uint2 *>(dkey);
  auto put = [&](uint32_t i) {
    const uint2 e = HAS_VALS ? s_kv[i] : make_uint2(s_k[i], 0u);
    const uint32_t g = (uint32_t)(s_gdelta[dig(e.x)] + (int32_t)i);
    if (dst_pairs) {
      dkey64[g] = e;
    } else {
      dkey32[g] = e.x;
      if (HAS_VALS) dval[g] = e.y;
    }
  };
#if PD_RS_WFULL
  if (full) {
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) put(tid + j * RS_THREADS);
    continue;
  }
#endif
#pragma unroll 4
  for (uint32_t i = tid; i < tile_n; i += RS_THREADS) put(i);
  }
}

// ------------------------------------------------- small-radix partition pass
// A single stable pass on a digit of at most 6 bits (the hash join's radix
// partition): no per-item warp matching.  Each thread owns PP_ITEMS
// consecutive elements of the tile and counts them per digit in its own
// 16-bit shared-memory counters (no atomics; stable because a thread's items
// are consecutive and counted in order).  A raking scan over the packed
// counters, in (digit, thread) order, turns the counts into tile ranks and
// digit starts; the digits' global offsets come from the same decoupled
// look-back as the digit pass; the tile is staged in digit order and every
// digit run is written contiguously.
//
// Counter layout: word (lane, thread), lane = digit % LANES, holds the
// counters of digits lane and lane + LANES in its low and high halves, so a
// digit's rank order is (half, lane, thread) = (digit, thread).  Each
// thread's raking segment of LANES words is padded by one word, so the
// segment walks hit distinct banks.
constexpr int PP_ITEMS = RS_ITEMS;            // same tile as the digit pass
static_assert(PP_ITEMS % 4 == 0, "16-byte loads of a thread's items");

template <int BITS>
struct PartShape {
  static constexpr int B = 1 << BITS;          // digits
  static constexpr int LANES = B / 2;          // packed counter words per thread
  static constexpr int SEG = LANES;            // raking segment (words per thread)
  static constexpr int WORDS = LANES * RS_THREADS + RS_THREADS;  // + one pad word per segment
  static __device__ __forceinline__ int pad(int e) { return e + e / SEG; }
};

enum : int { PV_NONE = 0, PV_U32 = 1, PV_U64 = 2 };  // values carried by the pass

// Dynamic shared memory of a partition pass: the staging buffer; with 64-bit
// values the packed counters share it (they are dead once the positions are
// computed), so that three CTAs fit on an SM.
constexpr size_t pp_smem_bytes(int bits, int val) {
  const int b = bits < 2 ? 2 : bits;
  const size_t stage = (size_t)(val == PV_U64 ? 12 : val == PV_U32 ? 8 : 4) * RS_TILE;
  const size_t cnt = val == PV_U64 ? 4 * ((size_t)(1 << (b - 1)) * RS_THREADS + RS_THREADS) : 0;
  return stage > cnt ? stage : cnt;
}

__device__ __forceinline__ void prefetch_l2(const void *ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

template <int BITS, int VAL, int KEY_MODE>
__global__ void __launch_bounds__(RS_THREADS, 3)
k_part_pass(SortParams p, uint32_t pass, uint32_t shift) {
  using S = PartShape<BITS>;
  constexpr bool HAS_VALS = VAL == PV_U32;
  constexpr bool V64 = VAL == PV_U64;
  // staging: RS_TILE (key, value) words, keys alone, or keys then 64-bit
  // values (and, before the staging, their packed counters)
  extern __shared__ __align__(16) uint2 pp_stage[];
  __shared__ uint32_t s_cnt_own[V64 ? 1 : S::WORDS];
  uint32_t *s_cnt = V64 ? reinterpret_cast<uint32_t *>(pp_stage) : s_cnt_own;
  __shared__ uint32_t s_warp[RS_WARPS];
  __shared__ uint32_t s_dstart[S::B + 1];
  __shared__ int32_t s_gdelta[S::B];
  __shared__ uint32_t s_tile;
  uint2 *s_kv = pp_stage;
  uint32_t *s_k = reinterpret_cast<uint32_t *>(pp_stage);
  unsigned long long *s_v64 = reinterpret_cast<unsigned long long *>(s_k + RS_TILE);

  const SortPlan *plan = p.plan;
  if (!plan->active[pass]) return;
  const uint32_t src = plan->src[pass], dst = plan->dst[pass];
  const bool first = plan->first[pass] != 0;
  const uint32_t flip = p.flip;
  const uint32_t mask = S::B - 1;
  auto dig = [&](uint32_t k) { return (sort_xform<KEY_MODE>(k, flip) >> shift) & mask; };

  const int tid = threadIdx.x;
  // persistent: tiles are claimed in order until the input is exhausted
  for (;;) {
  __syncthreads();  // the previous tile's readers of shared memory are done
  if (tid == 0) s_tile = atomicAdd(&p.counters[pass], 1u);
  for (int i = tid; i < S::WORDS; i += RS_THREADS) s_cnt[i] = 0;
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t base = tile * (uint64_t)RS_TILE;
  const uint64_t n = sort_n(p);
  if (base >= n) break;
  const uint32_t tile_n = (uint32_t)min((uint64_t)RS_TILE, n - base);
  const uint32_t t0 = (uint32_t)tid * PP_ITEMS;  // tile-local index of this thread's first item

  // columns only (the caller routes pair layouts to the digit pass)
  const uint32_t *skey = (src == BUF_IN ? reinterpret_cast<const uint32_t *>(p.in)
                          : src == BUF_OUT ? reinterpret_cast<const uint32_t *>(p.out) : p.alt_key) + base;
  const uint32_t *sval = src == BUF_IN ? p.in_ptr : (src == BUF_OUT ? p.out_ptr : p.alt_ptr);
  if (sval) sval += base;
  uint32_t *dkey = dst == BUF_OUT ? reinterpret_cast<uint32_t *>(p.out) : p.alt_key;
  uint32_t *dval = dst == BUF_OUT ? p.out_ptr : p.alt_ptr;
  const bool gen_vals = first && src == BUF_IN && p.in_ptr == nullptr;
  const uint32_t vbase = (uint32_t)(p.ptr_base + base);
  const unsigned long long *sv64 =
      (src == BUF_IN ? p.in_v64 : src == BUF_OUT ? p.out_v64 : p.alt_v64) + (V64 ? base : 0);
  unsigned long long *dv64 = dst == BUF_OUT ? p.out_v64 : p.alt_v64;
  const bool vec = ((reinterpret_cast<uintptr_t>(skey) | reinterpret_cast<uintptr_t>(sval) |
                     (V64 ? reinterpret_cast<uintptr_t>(sv64) : 0)) & 15u) == 0;

  // 1. load this thread's consecutive items
  uint32_t key[PP_ITEMS];
  uint32_t val[HAS_VALS ? PP_ITEMS : 1];
  if (V64) {
    // 64-bit values are loaded only when they are staged (step 5), which
    // keeps them out of the registers meanwhile; their lines go to L2 now
    const char *vb = reinterpret_cast<const char *>(sv64);
    const uint32_t lines = (tile_n * 8u + 127u) / 128u;
    for (uint32_t l = tid; l < lines; l += RS_THREADS) prefetch_l2(vb + 128ull * l);
  }
  if (vec && t0 + PP_ITEMS <= tile_n) {
#pragma unroll
    for (int j = 0; j < PP_ITEMS / 4; ++j) {
      const uint4 a = __ldcs(reinterpret_cast<const uint4 *>(skey + t0) + j);
      key[4 * j] = a.x; key[4 * j + 1] = a.y; key[4 * j + 2] = a.z; key[4 * j + 3] = a.w;
      if (HAS_VALS && !gen_vals) {
        const uint4 b = __ldcs(reinterpret_cast<const uint4 *>(sval + t0) + j);
        val[4 * j] = b.x; val[4 * j + 1] = b.y; val[4 * j + 2] = b.z; val[4 * j + 3] = b.w;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < PP_ITEMS; ++i) {
      const bool in = t0 + i < tile_n;
      key[i] = in ? __ldcs(skey + t0 + i) : 0u;
      if (HAS_VALS && !gen_vals) val[i] = in ? __ldcs(sval + t0 + i) : 0u;
    }
  }
  if (HAS_VALS && gen_vals) {
    if (p.pay64) {
      const long long pmin = *p.pay_min;
#pragma unroll
      for (int i = 0; i < PP_ITEMS; ++i)
        val[i] = t0 + i < tile_n ? (uint32_t)(__ldcs(p.pay64 + base + t0 + i) - pmin) : 0u;
    } else {
#pragma unroll
      for (int i = 0; i < PP_ITEMS; ++i) val[i] = vbase + t0 + i;
    }
  }

  // 2. thread-private counting: local rank of each item within its digit
  uint32_t lrank[PP_ITEMS / 2];  // two 16-bit local ranks per register
#pragma unroll
  for (int i = 0; i < PP_ITEMS / 2; ++i) lrank[i] = 0;
#pragma unroll
  for (int i = 0; i < PP_ITEMS; ++i) {
    if (t0 + i < tile_n) {
      const uint32_t d = dig(key[i]);
      const int w = S::pad((int)(d % S::LANES) * RS_THREADS + tid);
      const uint32_t sh = (d / S::LANES) * 16;
      const uint32_t old = s_cnt[w];
      s_cnt[w] = old + (1u << sh);
      lrank[i >> 1] |= ((old >> sh) & 0xFFFFu) << (16 * (i & 1));
    }
  }
  __syncthreads();

  // 3. raking scan of the packed counters in (lane, thread) word order; the
  //    halves add without carries (a tile has fewer than 2^16 items)
  uint32_t seg = 0;
  uint32_t *mine = s_cnt + tid * (S::SEG + 1);
#pragma unroll
  for (int j = 0; j < S::SEG; ++j) seg += mine[j];
  uint32_t total = 0;
  const uint32_t excl = block_exclusive_scan(seg, s_warp, &total);
  // the high halves' digits come after all low halves' digits
  uint32_t run = excl + ((total & 0xFFFFu) << 16);
#pragma unroll
  for (int j = 0; j < S::SEG; ++j) {
    const uint32_t c = mine[j];
    mine[j] = run;
    run += c;
  }
  __syncthreads();
  // digit starts in the tile: the exclusive prefix of word (lane, thread 0)
  if (tid < S::B) {
    const uint32_t w = s_cnt[S::pad((tid % S::LANES) * RS_THREADS)];
    s_dstart[tid] = (w >> ((tid / S::LANES) * 16)) & 0xFFFFu;
  }
  if (tid == 0) s_dstart[S::B] = tile_n;
  __syncthreads();

  // 4. publish the tile's digit counts; look back for the digits' global
  //    offsets (one thread per digit, 8 predecessor words per round; a warp
  //    that spreads its digits sequentially over its lanes was measured
  //    slower); the other threads go on to the positions, which need none
  if (tid < S::B) {
    const int d = tid;
    const uint32_t count = s_dstart[d + 1] - s_dstart[d];
    uint32_t *st = p.status + ((uint64_t)pass * p.tiles) * RS_RADIX + d;
    uint32_t ex = 0;
    if (tile == 0) {
      pd_store_relaxed_u32(st, RS_FLAG_INC | count);
    } else {
      pd_store_relaxed_u32(st + tile * RS_RADIX, RS_FLAG_AGG | count);
      ex = rs_lookback<8>(st, tile, count, p.d_error);
    }
    s_gdelta[d] = (int32_t)(p.offsets[pass * RS_RADIX + d] + ex) - (int32_t)s_dstart[d];
  }

  // 5. stage the tile in digit order
  if (!V64) {
#pragma unroll
    for (int i = 0; i < PP_ITEMS; ++i) {
      if (t0 + i < tile_n) {
        const uint32_t d = dig(key[i]);
        const uint32_t w = s_cnt[S::pad((int)(d % S::LANES) * RS_THREADS + tid)];
        const uint32_t pos = ((w >> ((d / S::LANES) * 16)) & 0xFFFFu) +
                             ((lrank[i >> 1] >> (16 * (i & 1))) & 0xFFFFu);
        if (HAS_VALS) s_kv[pos] = make_uint2(key[i], val[i]);
        else s_k[pos] = key[i];
      }
    }
    __syncthreads();
  } else {
    // 64-bit values: each item's position in the digit-ordered tile (kept
    // in lrank); once every thread has read its counters, keys and values
    // are staged over them
#pragma unroll
    for (int i = 0; i < PP_ITEMS; ++i) {
      if (t0 + i < tile_n) {
        const uint32_t d = dig(key[i]);
        const uint32_t w = s_cnt[S::pad((int)(d % S::LANES) * RS_THREADS + tid)];
        const uint32_t sh = 16 * (i & 1);
        const uint32_t pos = ((w >> ((d / S::LANES) * 16)) & 0xFFFFu) + ((lrank[i >> 1] >> sh) & 0xFFFFu);
        lrank[i >> 1] = (lrank[i >> 1] & ~(0xFFFFu << sh)) | (pos << sh);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PP_ITEMS; ++i)
      if (t0 + i < tile_n) s_k[(lrank[i >> 1] >> (16 * (i & 1))) & 0xFFFFu] = key[i];
    if (vec && t0 + PP_ITEMS <= tile_n) {
#pragma unroll
      for (int j = 0; j < PP_ITEMS / 2; ++j) {
        const ulonglong2 b = __ldcs(reinterpret_cast<const ulonglong2 *>(sv64 + t0) + j);
        s_v64[lrank[j] & 0xFFFFu] = b.x;
        s_v64[lrank[j] >> 16] = b.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < PP_ITEMS; ++i)
        if (t0 + i < tile_n) s_v64[(lrank[i >> 1] >> (16 * (i & 1))) & 0xFFFFu] = __ldcs(sv64 + t0 + i);
    }
    __syncthreads();
  }

  // 6. each digit run written contiguously
#pragma unroll 4
  for (uint32_t i = tid; i < tile_n; i += RS_THREADS) {
    const uint2 e = HAS_VALS ? s_kv[i] : make_uint2(s_k[i], 0u);
    const uint32_t g = (uint32_t)(s_gdelta[dig(e.x)] + (int32_t)i);
    dkey[g] = e.x;
    if (HAS_VALS) dval[g] = e.y;
    if (V64) dv64[g] = s_v64[i];
  }
  }
}

using PartKernel = void (*)(SortParams, uint32_t, uint32_t);
template <int BITS, int VAL>
PartKernel pick_part_mode(int key_mode) {
  if (key_mode == PD_KEY_HASH0) return k_part_pass<BITS, VAL, PD_KEY_HASH0>;
  if (key_mode == PD_KEY_MULHASH) return k_part_pass<BITS, VAL, PD_KEY_MULHASH>;
  return k_part_pass<BITS, VAL, PD_KEY_PLAIN>;
}
template <int BITS>
PartKernel pick_part_bits(int val, int key_mode) {
  if (val == PV_U64) return pick_part_mode<BITS, PV_U64>(key_mode);
  if (val == PV_U32) return pick_part_mode<BITS, PV_U32>(key_mode);
  return pick_part_mode<BITS, PV_NONE>(key_mode);
}
// Digits of 1..6 bits (a 1-bit digit uses the 2-bit kernel: its upper
// digits stay empty).
PartKernel pick_part(uint32_t bits, int val, int key_mode) {
  switch (bits) {
    case 1: case 2: return pick_part_bits<2>(val, key_mode);
    case 3: return pick_part_bits<3>(val, key_mode);
    case 4: return pick_part_bits<4>(val, key_mode);
    case 5: return pick_part_bits<5>(val, key_mode);
    case 6: return pick_part_bits<6>(val, key_mode);
    default: return nullptr;
  }
}

using PassKernel = void (*)(SortParams, uint32_t, uint32_t, uint32_t);
PassKernel pick_pass(bool vals, int key_mode) {
  if (key_mode == PD_KEY_HASH0) return vals ? k_sort_pass<true, PD_KEY_HASH0> : k_sort_pass<false, PD_KEY_HASH0>;
  if (key_mode == PD_KEY_MULHASH)
    return vals ? k_sort_pass<true, PD_KEY_MULHASH> : k_sort_pass<false, PD_KEY_MULHASH>;
  return vals ? k_sort_pass<true, PD_KEY_PLAIN> : k_sort_pass<false, PD_KEY_PLAIN>;
}

struct SortLayout {
  size_t off_counters, off_hist, off_offsets, off_plan, off_status, off_alt_key, off_alt_ptr,
      off_alt_v64, total, memset_bytes;
  uint64_t tiles;
  uint32_t npasses;
};

// dbits: digit width of each pass (8 for a sort; at most 6 for a partition,
// which may also carry 64-bit values, v64).
bool sort_layout(const pimdal_sort_arguments_t *a, SortLayout *l, uint32_t dbits = RS_RADIX_BITS,
                 bool v64 = false) {
  uint32_t b = a->begin_bit, e = a->end_bit ? a->end_bit : 32;
  if (b >= e || e > 32 || dbits == 0 || dbits > RS_RADIX_BITS) return false;
  l->npasses = (e - b + dbits - 1) / dbits;
  if (l->npasses > RS_MAX_PASSES) return false;
  l->tiles = pd_ceil_div(a->nr_elements ? a->nr_elements : 1, RS_TILE);
  size_t o = 0;
  l->off_counters = o; o += 256;
  l->off_hist = o; o += sizeof(uint32_t) * RS_MAX_PASSES * RS_RADIX;
  l->off_status = o; o += pd_align_up(sizeof(uint32_t) * RS_MAX_PASSES * l->tiles * RS_RADIX, 256);
  l->memset_bytes = o;
  l->off_offsets = o; o += sizeof(uint32_t) * RS_MAX_PASSES * RS_RADIX;
  l->off_plan = o; o += 256;
  l->off_alt_key = o; o += pd_align_up(sizeof(uint32_t) * a->nr_elements, 256);
  l->off_alt_ptr = o; o += pd_align_up(sizeof(uint32_t) * a->nr_elements, 256);
  l->off_alt_v64 = o; o += v64 ? pd_align_up(8 * a->nr_elements, 256) : 0;
  l->total = o;
  return true;
}

}  // namespace

extern "C" int pimdal_sort_workspace_size(const pimdal_sort_arguments_t *a, size_t *bytes) {
  if (!a || !bytes) return PIMDAL_ERR_ARG;
  SortLayout l;
  if (!sort_layout(a, &l)) return PIMDAL_ERR_ARG;
  *bytes = l.total;
  return PIMDAL_OK;
}

// Stream-ordered sort with a given workspace (used by the operators that
// sort internally, e.g. the sort-merge join and the sort group-by).
int pd_sort_with_workspace(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, void *ws,
                           cudaStream_t s) {
  return pd_sort_ex(ctx, a, PD_KEY_PLAIN, ws, s, nullptr);
}

// Same, ordering by the digits of a transform of the key (a stable radix
// partition when the bit range is one digit wide).  *offsets_out, when given,
// receives the device address of the exclusive digit offsets of pass 0.
int pd_sort_ex(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
               cudaStream_t s, uint32_t **offsets_out) {
  return pd_sort_ex2(ctx, a, key_mode, ws, s, offsets_out, nullptr);
}

namespace {
int pd_sort_core(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
                 cudaStream_t s, uint32_t **offsets_out, const uint64_t *n_dev, uint32_t dbits,
                 const uint64_t *in_v64, uint64_t *out_v64, const int64_t *pay64 = nullptr,
                 const int64_t *pay_min = nullptr);
}

// Same, with the element count read on the device from *n_dev (a->nr_elements
// is then an upper bound that sizes the workspace and the grids).
int pd_sort_ex2(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
                cudaStream_t s, uint32_t **offsets_out, const uint64_t *n_dev) {
  return pd_sort_core(ctx, a, key_mode, ws, s, offsets_out, n_dev, RS_RADIX_BITS, nullptr, nullptr);
}

// A stable radix partition of key columns by bits [begin_bit, end_bit) of a
// key transform, in passes of at most PD_PART_DIGIT_BITS bits, carrying a
// 32-bit value column (in_ptr/out_ptr) and/or a 64-bit one (in_v64/out_v64).
size_t pd_partition_workspace(const pimdal_sort_arguments_t *a, bool v64) {
  SortLayout l;
  return sort_layout(a, &l, PD_PART_DIGIT_BITS, v64) ? l.total : 0;
}
int pd_sort_pay64(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, void *ws, cudaStream_t s,
                  const uint64_t *n_dev, const int64_t *pay64, const int64_t *pay_min) {
  return pd_sort_core(ctx, a, PD_KEY_PLAIN, ws, s, nullptr, n_dev, RS_RADIX_BITS, nullptr, nullptr,
                      pay64, pay_min);
}

int pd_partition(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
                 cudaStream_t s, const uint64_t *in_v64, uint64_t *out_v64) {
  if (a->layout != PIMDAL_LAYOUT_COLUMNS || (in_v64 == nullptr) != (out_v64 == nullptr))
    return PIMDAL_ERR_ARG;
  return pd_sort_core(ctx, a, key_mode, ws, s, nullptr, nullptr, PD_PART_DIGIT_BITS, in_v64, out_v64);
}

namespace {
// Grid of a persistent pass: the CTAs that fit on the GPU at once (each
// claims tiles until the input is exhausted), at most one per tile.
unsigned resident_grid(const pimdal_ctx *ctx, const void *kernel, int smem, uint64_t tiles) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, RS_THREADS, smem) !=
          cudaSuccess || per_sm <= 0) {
    cudaGetLastError();
    per_sm = 1;
  }
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)per_sm * ctx->sm_count));
}

int pd_sort_core(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
                 cudaStream_t s, uint32_t **offsets_out, const uint64_t *n_dev, uint32_t dbits,
                 const uint64_t *in_v64, uint64_t *out_v64, const int64_t *pay64,
                 const int64_t *pay_min) {
  SortLayout l;
  const bool v64 = out_v64 != nullptr;
  if (!sort_layout(a, &l, dbits, v64)) return PIMDAL_ERR_ARG;
  if (v64 && dbits > 6) return PIMDAL_ERR_ARG;  // only the small-radix pass carries them
  if (offsets_out) *offsets_out = (uint32_t *)((char *)ws + l.off_offsets);
  if (a->nr_elements > RS_COUNT_MASK) return PIMDAL_ERR_ARG;  // < 2^30 elements
  char *w = (char *)ws;
  SortParams p{};
  p.in = a->in;
  p.in_ptr = a->layout == PIMDAL_LAYOUT_COLUMNS ? a->in_ptr : nullptr;
  p.ptr_base = a->ptr_base;
  p.out = a->out;
  p.out_ptr = a->layout == PIMDAL_LAYOUT_COLUMNS ? a->out_ptr : nullptr;
  p.pairs = a->layout == PIMDAL_LAYOUT_PAIRS;
  p.has_vals = p.pairs || p.out_ptr != nullptr;
  p.alt_key = (uint32_t *)(w + l.off_alt_key);
  p.alt_ptr = (uint32_t *)(w + l.off_alt_ptr);
  p.in_v64 = (const unsigned long long *)in_v64;
  p.out_v64 = (unsigned long long *)out_v64;
  p.alt_v64 = v64 ? (unsigned long long *)(w + l.off_alt_v64) : nullptr;
  p.dbits = dbits;
  p.pay64 = (const long long *)pay64;
  p.pay_min = (const long long *)pay_min;
  if (pay64 && (a->in_ptr || !pay_min)) return PIMDAL_ERR_ARG;
  p.n = a->nr_elements;
  p.n_dev = n_dev;
  p.flip = a->key_dtype == PIMDAL_I32 ? 0x80000000u : 0u;
  p.key_mode = key_mode;
  p.begin_bit = a->begin_bit;
  p.end_bit = a->end_bit ? a->end_bit : 32;
  p.npasses = l.npasses;
  p.hist = (uint32_t *)(w + l.off_hist);
  p.offsets = (uint32_t *)(w + l.off_offsets);
  p.plan = (SortPlan *)(w + l.off_plan);
  p.status = (uint32_t *)(w + l.off_status);
  p.counters = (uint32_t *)(w + l.off_counters);
  p.tiles = l.tiles;
  p.d_error = ctx->d_error;

  PD_CHECK_CUDA(cudaMemsetAsync(w, 0, l.memset_bytes, s));
  const unsigned hist_blocks =
      (unsigned)std::min<uint64_t>(pd_ceil_div(p.n, (uint64_t)RS_THREADS * 16), (uint64_t)ctx->sm_count * 4);
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_SORT_HIST, s);
    auto hk = key_mode == PD_KEY_HASH0 ? k_sort_hist<PD_KEY_HASH0>
              : key_mode == PD_KEY_MULHASH ? k_sort_hist<PD_KEY_MULHASH> : k_sort_hist<PD_KEY_PLAIN>;
    hk<<<hist_blocks ? hist_blocks : 1, RS_THREADS, 0, s>>>(p);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_sort_plan<<<1, RS_THREADS, 0, s>>>(p);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    unsigned cb = (unsigned)std::min<uint64_t>(pd_ceil_div(p.n, RS_THREADS), (uint64_t)ctx->sm_count * 8);
    k_sort_copy<<<cb ? cb : 1, RS_THREADS, 0, s>>>(p);
  }
  // Digits of at most 6 bits over key columns (a radix partition, or a sort
  // on a single small digit): the small-radix pass.
  if ((dbits <= 6 || (l.npasses == 1 && p.end_bit - p.begin_bit <= 6)) && !p.pairs) {
    const int val = v64 ? PV_U64 : p.has_vals ? PV_U32 : PV_NONE;
    for (uint32_t q = 0; q < l.npasses; ++q) {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_PARTITION, s);
      const uint32_t shift = p.begin_bit + q * dbits;
      const uint32_t qbits = std::min(dbits, p.end_bit - shift);
      PartKernel k = pick_part(qbits, val, key_mode);
      const int smem = (int)pp_smem_bytes((int)qbits, val);
      PD_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      k<<<resident_grid(ctx, (const void *)k, smem, l.tiles), RS_THREADS, smem, s>>>(p, q, shift);
    }
    return pd_launch_status(ctx);
  }
  for (uint32_t q = 0; q < l.npasses; ++q) {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_SORT_PASS, s);
    const uint32_t shift = p.begin_bit + q * RS_RADIX_BITS;
    const uint32_t bits = std::min<uint32_t>(RS_RADIX_BITS, p.end_bit - shift);
    const uint32_t mask = (1u << bits) - 1u;
    auto k = pick_pass(p.has_vals != 0, key_mode);
    const int smem = (p.has_vals ? 8 : 4) * RS_TILE;
    PD_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k<<<resident_grid(ctx, (const void *)k, smem, l.tiles), RS_THREADS, smem, s>>>(p, q, shift, mask);
  }
  return pd_launch_status(ctx);
}
}  // namespace

extern "C" int pimdal_sort_kernel(pimdal_ctx_t *ctx, const pimdal_sort_arguments_t *a,
                                  pimdal_stream_t stream) {
  if (!ctx || !a) return PIMDAL_ERR_ARG;
  if (a->layout != PIMDAL_LAYOUT_COLUMNS && a->layout != PIMDAL_LAYOUT_PAIRS) return PIMDAL_ERR_ARG;
  if (a->key_dtype != PIMDAL_I32 && a->key_dtype != PIMDAL_U32) return PIMDAL_ERR_ARG;
  if (a->nr_elements == 0) return PIMDAL_OK;
  if (!a->in || !a->out || a->in == a->out) return PIMDAL_ERR_ARG;
  if (a->layout == PIMDAL_LAYOUT_PAIRS && (((uintptr_t)a->in | (uintptr_t)a->out) & 7u))
    return PIMDAL_ERR_ARG;  // key_ptr32 pairs are accessed as 8-byte words
  if (a->layout == PIMDAL_LAYOUT_COLUMNS && a->out_ptr && a->in_ptr == a->out_ptr)
    return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  size_t need;
  int st = pimdal_sort_workspace_size(a, &need);
  if (st) return st;
  void *ws = pd_workspace(ctx, need, s, &st);
  if (!ws) return st;
  return pd_sort_with_workspace(ctx, a, ws, s);
}
