// K-FILTER / K-MATCH: the Bloom-filter semi-join prefilter
// (pimdal_filter_kernel, pimdal_match_kernel).
//
// Reference behaviour: filter_kernel (pimdal/join/hash_join.c:116-149)
// builds, for every partition of already-partitioned key_ptr pairs, a filter
// of FILTER_SIZE = 16384 bits (pimdal/hash/hash_steps.c:15-16) by setting bit
// hashK(key) % 16384 for K = 1..4 (insert_bloom_filter, hash_steps.c:143-152;
// hash1..hash4 of pimdal/hash/hash_func.h:16-60).  match_kernel
// (hash_join.c:236-341) keeps, in input order, the rows whose key finds all
// four bits set in its partition's filter (probe_bloom_filter,
// hash_steps.c:163-185) and counts the kept rows of every partition.
//
// B200 design (HBM-bound streaming; the filters, 2 KB each, live in L2):
//  * k_filter_parts: one CTA per partition of at most 16384 rows (the
//    usual size) builds its filter in shared memory and stores it whole,
//    no global atomics.
//  * k_filter_build, for the rows of larger partitions only (skipped
//    entirely when there are none): CTAs stride over 2048-row tiles.  A tile spanning at
//    most 8 partitions builds their filters in shared memory (shared
//    atomics) and ORs the non-zero words into the global filters, at most
//    512 global atomics per partition; a tile spanning more partitions ORs
//    each row's bits into the global filters directly.  The partitions of a
//    tile's first and last row are found by two warps, 32 offsets per round.
//  * k_match: persistent CTAs claim 2048-row tiles in order (8 warp-striped
//    keys per thread, loads issued together).  A pre-pass finds every
//    tile's first and last partition in parallel; a tile reads its pair when
//    it is claimed.  A tile spanning at most 8 partitions stages their filters and
//    first rows in shared memory and counts its kept rows per partition
//    there; otherwise each row finds its partition by binary search and
//    reads its filter through L1.  Kept rows are ranked with ballots and a
//    block scan, and the tile's output offset comes from a decoupled
//    look-back over epoch-tagged status words (one warp polls, the rest of
//    the CTA waits at a barrier), so the output is in input order without a
//    second pass.  Row ids (or pairs) are read for the kept
//    rows only, after the look-back.
#include <algorithm>

#include "common.cuh"

namespace {

constexpr int BF_THREADS = 256;
constexpr int BF_WARPS = BF_THREADS / 32;
#ifndef PD_BF_ITEMS
#define PD_BF_ITEMS 8  // rows per thread of a match / filter tile (measured best; 4 was slower)
#endif
#ifndef PD_BF_RANGES
#define PD_BF_RANGES 1  // 1: tile partition ranges from a pre-pass (0: searched by each tile)
#endif
#ifndef PD_BF_MATCH_CTAS
// match CTAs per SM the kernel is compiled for: 8 (32 registers, a 44-byte
// spill) hide the per-tile barriers better than 6 (40 registers): 2.31 ->
// 1.99 ms for 2^28 probe rows at 5% match
#define PD_BF_MATCH_CTAS 8
#endif
constexpr int BF_ITEMS = PD_BF_ITEMS;
static_assert(BF_ITEMS <= 32, "one hit bit per row of a thread");
constexpr int BF_TILE = BF_THREADS * BF_ITEMS;          // 2048 rows by default
constexpr uint32_t BF_WORDS = PIMDAL_FILTER_BITS / 32;  // 512 words per filter
constexpr uint32_t BF_MASK = PIMDAL_FILTER_BITS - 1;
static_assert((PIMDAL_FILTER_BITS & BF_MASK) == 0, "the filter size is a power of two");
constexpr int BF_SMEM_PARTS = 8;  // filters a tile holds in shared memory
constexpr int BF_MATCH_CTAS = PD_BF_MATCH_CTAS;

// The largest p in [lo, hi] with ps[p] <= r, or lo - 1 when there is none
// (ps non-decreasing).  Over [0, part_n] this is r's partition, -1 before the
// first partition and part_n after the last.
__device__ __forceinline__ int64_t part_of(const uint64_t *ps, int64_t lo, int64_t hi, uint64_t r) {
  int64_t a = lo, b = hi;
  while (a <= b) {
    const int64_t m = (a + b) >> 1;
    if (ps[m] <= r) a = m + 1;
    else b = m - 1;
  }
  return b;
}

// The same answer found by one warp in rounds of 32 parallel loads (three
// rounds for 16384 partitions instead of 14 dependent loads).  Every round
// keeps the result inside [lo - 1, hi], whatever ps holds.
__device__ __forceinline__ int64_t warp_part_of(const uint64_t *ps, int64_t lo, int64_t hi,
                                                uint64_t r) {
  const int lane = threadIdx.x & 31;
  while (hi - lo + 1 > 32) {
    const int64_t step = (hi - lo + 32) / 32;  // ceil(range / 32)
    const int64_t idx = lo + lane * step;
    const bool le = idx <= hi && ps[idx] <= r;
    const int c = __popc(__ballot_sync(0xffffffffu, le));  // samples <= r: a prefix of the lanes
    if (c == 0) return lo - 1;
    lo += (int64_t)(c - 1) * step;
    hi = min(hi, lo + step - 1);
  }
  const int64_t idx = lo + lane;
  const bool le = idx <= hi && ps[idx] <= r;
  return lo + __popc(__ballot_sync(0xffffffffu, le)) - 1;
}

// Warps 0 and 1 locate a tile's first and last row (all threads call).
__device__ __forceinline__ void tile_parts(const uint64_t *ps, uint32_t part_n, uint64_t first,
                                           uint64_t last, int64_t *s_pa, int64_t *s_pb) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < 2) {
    const int64_t q = warp_part_of(ps, 0, part_n, warp == 0 ? first : last);
    if (lane == 0) *(warp == 0 ? s_pa : s_pb) = q;
  }
}

__device__ __forceinline__ uint32_t bit0(uint32_t k) { return pd_bloom_hash<0>(k) & BF_MASK; }
__device__ __forceinline__ uint32_t bit1(uint32_t k) { return pd_bloom_hash<1>(k) & BF_MASK; }
__device__ __forceinline__ uint32_t bit2(uint32_t k) { return pd_bloom_hash<2>(k) & BF_MASK; }
__device__ __forceinline__ uint32_t bit3(uint32_t k) { return pd_bloom_hash<3>(k) & BF_MASK; }

// Bit b of a filter is bit b % 8 of byte b / 8; in little-endian 32-bit
// words that is bit b % 32 of word b / 32.
__device__ __forceinline__ void set_bits(uint32_t *f, uint32_t k) {
  const uint32_t b[4] = {bit0(k), bit1(k), bit2(k), bit3(k)};
#pragma unroll
  for (int i = 0; i < 4; ++i) atomicOr(&f[b[i] >> 5], 1u << (b[i] & 31));
}

__device__ __forceinline__ bool test_bits(const uint32_t *f, uint32_t k) {
  const uint32_t b[4] = {bit0(k), bit1(k), bit2(k), bit3(k)};
  uint32_t all = 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) all &= f[b[i] >> 5] >> (b[i] & 31);
  return all & 1u;
}

__device__ __forceinline__ bool test_bits_global(const uint32_t *f, uint32_t k) {
  const uint32_t b[4] = {bit0(k), bit1(k), bit2(k), bit3(k)};
  uint32_t all = 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) all &= __ldg(f + (b[i] >> 5)) >> (b[i] & 31);
  return all & 1u;
}

struct FilterParams {
  const void *in;
  uint32_t *filter;
  const uint64_t *ps;
  uint32_t part_n;
  int pairs;
};

__device__ __forceinline__ uint32_t key_at(const void *in, int pairs, uint64_t r) {
  return pairs ? reinterpret_cast<const uint2 *>(in)[r].x : reinterpret_cast<const uint32_t *>(in)[r];
}

// Partitions of at most BF_PART_ROWS rows: one CTA per partition in turn
// assembles its filter in shared memory (eight key loads of a thread in
// flight together) and stores it whole -- no other CTA writes that filter, so
// no atomics reach global memory.  A larger partition (or a decreasing
// part_sizes entry) sets *large and is left to k_filter_build.
constexpr uint64_t BF_PART_ROWS = 16384;

__device__ __forceinline__ bool small_part(const uint64_t *ps, int64_t q) {
  const uint64_t a = ps[q], b = ps[q + 1];
  return b > a && b - a <= BF_PART_ROWS;
}

__global__ void __launch_bounds__(BF_THREADS) k_filter_parts(FilterParams p, uint32_t *large) {
  __shared__ __align__(16) uint32_t s_f[BF_WORDS];
  const int tid = threadIdx.x;
  for (uint32_t q = blockIdx.x; q < p.part_n; q += gridDim.x) {
    const uint64_t a = p.ps[q], b = p.ps[q + 1];
    if (b <= a) {
      if (b < a && tid == 0) *large = 1;
      continue;
    }
    if (b - a > BF_PART_ROWS) {
      if (tid == 0) *large = 1;
      continue;
    }
    for (uint32_t i = tid; i < BF_WORDS; i += BF_THREADS) s_f[i] = 0;
    __syncthreads();
    for (uint64_t r0 = a; r0 < b; r0 += 8 * BF_THREADS) {
      uint32_t k[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint64_t r = r0 + (uint64_t)j * BF_THREADS + tid;
        k[j] = r < b ? key_at(p.in, p.pairs, r) : 0u;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (r0 + (uint64_t)j * BF_THREADS + tid < b) set_bits(s_f, k[j]);
    }
    __syncthreads();
    uint4 *g = reinterpret_cast<uint4 *>(p.filter + (uint64_t)q * BF_WORDS);
    for (uint32_t i = tid; i < BF_WORDS / 4; i += BF_THREADS) g[i] = reinterpret_cast<const uint4 *>(s_f)[i];
    __syncthreads();  // s_f is cleared again for the next partition
  }
}

// The rows of the partitions k_filter_parts left (when *large is set).
__global__ void __launch_bounds__(BF_THREADS) k_filter_build(FilterParams p, const uint32_t *large) {
  __shared__ __align__(16) uint32_t s_f[BF_SMEM_PARTS * BF_WORDS];
  __shared__ int64_t s_pa, s_pb;
  const int tid = threadIdx.x;
  const uint64_t begin = p.ps[0], end = p.ps[p.part_n];
  if (*large == 0 || end <= begin) return;
  const uint64_t tiles = pd_ceil_div(end - begin, BF_TILE);
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint64_t a = begin + t * BF_TILE, b = min(a + (uint64_t)BF_TILE, end);
    tile_parts(p.ps, p.part_n, a, b - 1, &s_pa, &s_pb);
    __syncthreads();
    const int64_t pa = s_pa, pb = s_pb, np = pb - pa + 1;
    if (pa >= 0 && pb < (int64_t)p.part_n && np >= 1 && np <= BF_SMEM_PARTS) {
      // The tile's partitions pa..pb: their filters are assembled in shared
      // memory, then every non-zero word is ORed into the (contiguous)
      // global filters once.
      for (uint32_t i = tid; i < np * BF_WORDS; i += BF_THREADS) s_f[i] = 0;
      __syncthreads();
      for (uint64_t r = a + tid; r < b; r += BF_THREADS) {
        const int64_t q = np == 1 ? pa : part_of(p.ps, pa, pb, r);
        if (q < pa) continue;  // only with a decreasing part_sizes
        if (small_part(p.ps, q)) continue;  // stored whole by k_filter_parts
        set_bits(s_f + (q - pa) * BF_WORDS, key_at(p.in, p.pairs, r));
      }
      __syncthreads();
      uint32_t *g = p.filter + (uint64_t)pa * BF_WORDS;
      for (uint32_t i = tid; i < np * BF_WORDS; i += BF_THREADS)
        if (s_f[i]) atomicOr(&g[i], s_f[i]);
    } else {
      // many small partitions in one tile: bits go straight to global memory
      for (uint64_t r = a + tid; r < b; r += BF_THREADS) {
        const int64_t q = part_of(p.ps, pa < 0 ? 0 : pa, pb < 0 ? -1 : pb, r);
        if (q < 0 || q >= (int64_t)p.part_n) continue;  // only with a decreasing part_sizes
        if (small_part(p.ps, q)) continue;  // stored whole by k_filter_parts
        set_bits(p.filter + (uint64_t)q * BF_WORDS, key_at(p.in, p.pairs, r));
      }
    }
    __syncthreads();  // s_f and s_pa/s_pb are reused by the next tile
  }
}

struct MatchParams {
  const uint32_t *filter;
  const void *key;
  const uint32_t *row;  // columns layout: row ids, NULL = index
  int pairs;
  void *out_key;
  uint32_t *out_row;
  uint64_t cap;
  uint64_t *match_sizes;
  const uint64_t *ps;
  uint32_t part_n;
  uint64_t n;
  uint32_t tiles;
  uint64_t *status;
  uint32_t epoch;
  uint32_t *claim;
  uint32_t *d_error;
  uint64_t *d_count;
  const int2 *ranges;  // per tile: partitions of its first and last row
};

// Pre-pass of k_match: the partitions of every tile's first and last row,
// one thread per tile, all tiles in parallel.
__global__ void __launch_bounds__(256) k_match_ranges(MatchParams p, int2 *ranges) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.tiles) return;
  const uint64_t a = t * BF_TILE, b = min(a + (uint64_t)BF_TILE, p.n) - 1;
  ranges[t] = make_int2((int)part_of(p.ps, 0, p.part_n, a), (int)part_of(p.ps, 0, p.part_n, b));
}

__global__ void __launch_bounds__(BF_THREADS, BF_MATCH_CTAS) k_match(MatchParams p) {
  __shared__ __align__(16) uint32_t s_f[BF_SMEM_PARTS * BF_WORDS];  // the tile's filters
  __shared__ uint32_t s_bound[BF_SMEM_PARTS];  // first row of each of the tile's partitions
  __shared__ uint32_t s_cnt[BF_SMEM_PARTS];    // kept rows per partition of the tile
  __shared__ int64_t s_pa, s_pb;
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ uint32_t s_warp[BF_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t n = (uint32_t)p.n;
  while (true) {
    if (tid == 0) {
      const uint32_t t = atomicAdd(p.claim, 1u);
      if (t >= p.tiles && atomicAdd(p.claim + 1, 1u) == gridDim.x - 1) {
        p.claim[0] = 0;  // the last claimer of the launch resets the counters
        p.claim[1] = 0;
      }
      s_tile = t;
#if PD_BF_RANGES
      if (t < p.tiles) {
        const int2 rg = p.ranges[t];
        s_pa = rg.x;
        s_pb = rg.y;
      }
#endif
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= p.tiles) break;

    // Warp-striped rows: row k of this lane is wbase + 32k + lane (< 2^32).
    // Only the keys are read here (issued before the partition search, whose
    // latency they hide); row ids are read later for the kept rows alone.
    const uint32_t wbase = tile * BF_TILE + warp * (32 * BF_ITEMS);
    uint32_t key[BF_ITEMS];
#pragma unroll
    for (int k = 0; k < BF_ITEMS; ++k) {
      const uint32_t r = wbase + 32u * k + lane;
      key[k] = 0;
      if (r < n)
        key[k] = p.pairs ? reinterpret_cast<const uint2 *>(p.key)[r].x
                         : reinterpret_cast<const uint32_t *>(p.key)[r];
    }
#if !PD_BF_RANGES
    const uint32_t last = (uint32_t)(min((uint64_t)tile * BF_TILE + BF_TILE, p.n) - 1);
    tile_parts(p.ps, p.part_n, tile * BF_TILE, last, &s_pa, &s_pb);
    __syncthreads();
#endif
    const int64_t pa = s_pa, pb = s_pb, np = pb - pa + 1;
    const bool local = pa >= 0 && pb < (int64_t)p.part_n && np <= BF_SMEM_PARTS;
    if (local) {
      // the filters of partitions pa..pb (contiguous) and their first rows
      const uint4 *g = reinterpret_cast<const uint4 *>(p.filter + (uint64_t)pa * BF_WORDS);
      for (uint32_t i = tid; i < np * (BF_WORDS / 4); i += BF_THREADS)
        reinterpret_cast<uint4 *>(s_f)[i] = g[i];
      if (tid < np) {
        s_bound[tid] = (uint32_t)p.ps[pa + tid];
        s_cnt[tid] = 0;
      }
    }
    __syncthreads();

    uint32_t hits = 0;  // bit k: row k is kept
    if (local) {
#pragma unroll
      for (int k = 0; k < BF_ITEMS; ++k) {
        const uint32_t r = wbase + 32u * k + lane;
        uint32_t j = 0;
        for (int i = 1; i < np; ++i) j += r >= s_bound[i];
        if (r < n && test_bits(s_f + j * BF_WORDS, key[k])) {
          hits |= 1u << k;
          if (np > 1) atomicAdd(&s_cnt[j], 1u);
        }
      }
    } else {
      // rows outside every partition, or many partitions in one tile
      const int64_t lo = pa < 0 ? 0 : pa, hi = pb < 0 ? -1 : pb;
#pragma unroll
      for (int k = 0; k < BF_ITEMS; ++k) {
        const uint32_t r = wbase + 32u * k + lane;
        int64_t q = -1;
        bool hit = false;
        if (r < n) {
          q = part_of(p.ps, lo, hi, r);
          hit = q >= 0 && q < (int64_t)p.part_n &&
                test_bits_global(p.filter + (uint64_t)q * BF_WORDS, key[k]);
        }
        if (hit) hits |= 1u << k;
        const unsigned km = __ballot_sync(0xffffffffu, hit);
        if (hit) {
          const unsigned peers = __match_any_sync(km, (long long)q);
          if (lane == __ffs(peers) - 1)
            atomicAdd(reinterpret_cast<unsigned long long *>(p.match_sizes + q + 1),
                      (unsigned long long)__popc(peers));
        }
      }
    }

    // Block scan of the kept counts; tile look-back.
    const uint32_t wtot = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(hits));
    if (lane == 0) s_warp[warp] = wtot;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
#pragma unroll
    for (int w = 0; w < BF_WARPS; ++w) {
      const uint32_t x = s_warp[w];
      if (w < warp) wpre += x;
      total += x;
    }
    if (tile == 0) {
      if (tid == 0) {
        pd_store_relaxed_u64(p.status, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, total));
        s_prefix = 0;
      }
    } else {
      // One warp waits for the predecessors; the others wait at the barrier
      // below without taking issue slots from the SM's other CTAs.
      if (warp == 0) {
        if (lane == 0)
          pd_store_relaxed_u64(p.status + tile, pd_pack_status(p.epoch, PD_FLAG_AGGREGATE, total));
        const uint64_t pre = pd_lookback_warp(p.status, (int64_t)tile, p.epoch, p.d_error);
        if (lane == 0) {
          pd_store_relaxed_u64(p.status + tile, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, pre + total));
          s_prefix = (uint32_t)pre;
        }
      }
    }
    __syncthreads();
    if (local) {
      if (np == 1) {
        if (tid == 0 && total)
          atomicAdd(reinterpret_cast<unsigned long long *>(p.match_sizes + pa + 1),
                    (unsigned long long)total);
      } else if (tid < np && s_cnt[tid]) {
        atomicAdd(reinterpret_cast<unsigned long long *>(p.match_sizes + pa + tid + 1),
                  (unsigned long long)s_cnt[tid]);
      }
    }
    if (tid == 0 && tile == p.tiles - 1) *p.d_count = (uint64_t)s_prefix + total;

    // Kept rows in input order (k-major, then lane, within the warp).
    uint32_t w = s_prefix + wpre;
    bool overflow = false;
#pragma unroll
    for (int k = 0; k < BF_ITEMS; ++k) {
      const bool hit = (hits >> k) & 1u;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const uint32_t pos = w + __popc(m & lt);
        const uint32_t r = wbase + 32u * k + lane;
        if (pos < p.cap) {
          if (p.pairs) {
            reinterpret_cast<uint2 *>(p.out_key)[pos] = reinterpret_cast<const uint2 *>(p.key)[r];
          } else {
            reinterpret_cast<uint32_t *>(p.out_key)[pos] = key[k];
            if (p.out_row) p.out_row[pos] = p.row ? p.row[r] : r;
          }
        } else {
          overflow = true;
        }
      }
      w += __popc(m);
    }
    if (overflow) atomicOr(p.d_error, PD_DEVERR_CAPACITY);
    __syncthreads();  // shared state is reused by the next tile
  }
}

int match_grid(pimdal_ctx *ctx) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_match, BF_THREADS, 0);
    if (per_sm <= 0) per_sm = 1;
  }
  return per_sm * ctx->sm_count;
}

bool layout_ok(int32_t layout) { return layout == PIMDAL_LAYOUT_COLUMNS || layout == PIMDAL_LAYOUT_PAIRS; }

}  // namespace

extern "C" int pimdal_filter_kernel(pimdal_ctx_t *ctx, const pimdal_filter_arguments_t *a,
                                    pimdal_stream_t stream) {
  if (!ctx || !a || !a->in || !a->filter_ptr || !a->part_sizes || a->part_n == 0) return PIMDAL_ERR_ARG;
  if (((uintptr_t)a->filter_ptr & 15u) || !layout_ok(a->layout)) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  PD_CHECK_CUDA(cudaMemsetAsync(a->filter_ptr, 0, (size_t)a->part_n * PIMDAL_FILTER_BYTES, s));
  FilterParams p{};
  p.in = a->in;
  p.filter = (uint32_t *)a->filter_ptr;
  p.ps = a->part_sizes;
  p.part_n = a->part_n;
  p.pairs = a->layout == PIMDAL_LAYOUT_PAIRS;
  uint32_t *large = ctx->d_counters + PD_COUNTER_FILTER;
  PD_CHECK_CUDA(cudaMemsetAsync(large, 0, sizeof(uint32_t), s));
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_FILTER, s);
    k_filter_parts<<<ctx->sm_count * 8, BF_THREADS, 0, s>>>(p, large);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_FILTER, s);
    k_filter_build<<<ctx->sm_count * 8, BF_THREADS, 0, s>>>(p, large);
  }
  return pd_launch_status(ctx);
}

extern "C" int pimdal_match_workspace_size(const pimdal_match_arguments_t *a, size_t *bytes) {
  if (!a || !bytes) return PIMDAL_ERR_ARG;
  *bytes = PD_BF_RANGES ? sizeof(int2) * pd_ceil_div(a->size, BF_TILE) : 0;
  return PIMDAL_OK;
}

extern "C" int pimdal_match_kernel(pimdal_ctx_t *ctx, const pimdal_match_arguments_t *a,
                                   pimdal_merge_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result || !a->filter_ptr || !a->match_sizes || !a->part_sizes || a->part_n == 0)
    return PIMDAL_ERR_ARG;
  if (((uintptr_t)a->filter_ptr & 15u) || !layout_ok(a->layout) || a->size >= (1ull << 32))
    return PIMDAL_ERR_ARG;
  if ((a->size && !a->part_ptr) || (a->out_capacity && !a->out_ptr)) return PIMDAL_ERR_ARG;
  if (a->part_n >= (1u << 31)) return PIMDAL_ERR_ARG;  // partition indices are int32 here
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  PD_CHECK_CUDA(cudaMemsetAsync(a->match_sizes, 0, sizeof(uint64_t) * ((size_t)a->part_n + 1), s));
  if (a->size == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d_result, 0, sizeof(uint64_t), s));
    return PIMDAL_OK;
  }
  const uint64_t tiles = pd_ceil_div(a->size, BF_TILE);
  if (tiles > PD_STATUS_WORDS) return PIMDAL_ERR_ARG;
  int st;
  MatchParams p{};
  p.filter = (const uint32_t *)a->filter_ptr;
  p.key = a->part_ptr;
  p.row = a->layout == PIMDAL_LAYOUT_PAIRS ? nullptr : a->part_row;
  p.pairs = a->layout == PIMDAL_LAYOUT_PAIRS;
  p.out_key = a->out_ptr;
  p.out_row = a->layout == PIMDAL_LAYOUT_PAIRS ? nullptr : a->out_row;
  p.cap = a->out_capacity;
  p.match_sizes = a->match_sizes;
  p.ps = a->part_sizes;
  p.part_n = a->part_n;
  p.n = a->size;
  p.tiles = (uint32_t)tiles;
  p.status = ctx->d_status;
  p.claim = ctx->d_counters + PD_COUNTER_MATCH;
  p.d_error = ctx->d_error;
  p.d_count = &d_result->t_count;
#if PD_BF_RANGES
  int2 *ranges = (int2 *)pd_workspace(ctx, sizeof(int2) * tiles, s, &st);
  if (!ranges) return st;
  p.ranges = ranges;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_MATCH, s);
    k_match_ranges<<<(unsigned)pd_ceil_div(tiles, 256), 256, 0, s>>>(p, ranges);
  }
#endif
  p.epoch = pd_next_epoch(ctx, s, &st);
  if (st) return st;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_MATCH, s);
    const unsigned g = (unsigned)std::min<uint64_t>(tiles, (uint64_t)match_grid(ctx));
    k_match<<<g, BF_THREADS, 0, s>>>(p);
  }
  return pd_launch_status(ctx);
}
