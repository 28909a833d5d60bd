// K-PART / K-BUILD / K-PROBE: radix partitioning and the hash join
// (pimdal_part_kernel, pimdal_hash_kernel, pimdal_hj_probe, pimdal_hash_join).
//
// Reference behaviour: part_kernel (pimdal/join/hash_join.c:154-235,
// hash_steps.c:198-294) radix-partitions key_ptr pairs by bits of hash0(key);
// hash_kernel (hash_join.c:40-115, linear_hash.c:13-23) builds linear-probing
// tables; merge_kernel (hash_join.c:343-430, linear_hash.c:34-53) probes them
// and emits (probe ptr, build ptr).  The CPU operator
// reference/db_operators/hash_join.cpp:57-219 partitions both relations
// 16384 ways, builds a hash set per partition and probes it.
//
// B200 design:
//  * Partitioning is one onesweep pass of K-SORT on the digits of a hash of
//    the key (stable, coalesced runs); part_kernel uses hash0's bits so the
//    partition index a caller sees is the reference's.
//  * Tables are arrays of 64-bit slots (payload << 32 | key) filled with
//    atomicCAS linear probing.  The one row whose slot word would equal the
//    empty word (key and payload all ones) is counted on the side.
//  * A table that fits the L2 budget is built and probed directly.  A larger
//    one is split by the top bits of a multiplicative hash: both relations
//    are partitioned, and partition by partition one table buffer (reused, so
//    it stays L2-resident and is never written back) is cleared, built and
//    probed.  All partition bounds live on the device; no host sync.
//  * Bucketized linear probing: a key hashes to a bucket of 4 slots (one
//    32-byte sector) and takes the first free slot of the first bucket, from
//    there on, that has one; a lookup reads one sector and is done when the
//    key is found (no duplicate build key) or the bucket has a free slot.
//  * Probing: persistent CTAs claim 3072-row tiles of warp-striped rows; a
//    thread walks 2 rows at a time in lockstep (their bucket loads in flight
//    together); match counts are scanned and the tile's output
//    offset resolved by a decoupled look-back (one warp polls while the rest
//    of the CTA waits at a barrier) that chains across the per-partition
//    launches, so the output is in probe order within each
//    partition, partitions in order.
#include <algorithm>

#include "batch.cuh"

namespace {

constexpr uint64_t HJ_EMPTY = ~0ull;
constexpr int HJ_THREADS = 256;
#ifndef PD_HJ_ITEMS
// probe rows per thread of a tile (at most 16: 4 count bits each in 64); 12
// rows at 4 CTAs per SM (64 registers, a 20-byte spill) measured 3.5% faster
// than 16 rows at 3 CTAs (the probe of 2^28 rows: 3.08 -> 2.97 ms); 8 rows
// at 4 or 5 CTAs were slower
#define PD_HJ_ITEMS 12
#endif
constexpr int HJ_ITEMS = PD_HJ_ITEMS;
constexpr int HJ_TILE = HJ_THREADS * HJ_ITEMS;  // probe rows per tile (3072)
#ifndef PD_HJ_BATCH
#define PD_HJ_BATCH 2  // probe rows of a thread whose bucket loads are in flight together
#endif
#ifndef PD_HJ_KEYS_FIRST
#define PD_HJ_KEYS_FIRST 1  // a thread loads all its probe keys and row ids before any bucket
#endif
#ifndef PD_HJ_MIN_CTAS
#define PD_HJ_MIN_CTAS 4  // probe CTAs per SM (register budget)
#endif
constexpr int HJ_BATCH = PD_HJ_BATCH;
static_assert(HJ_ITEMS <= 16 && HJ_ITEMS % HJ_BATCH == 0, "probe tile shape");
constexpr uint32_t HJ_MIN_BITS = 10;

}  // namespace

// log2 of the slots of a table for nb build rows at load_pct percent.
uint32_t pd_hj_table_bits(uint64_t nb, uint32_t load_pct) {
  uint64_t cap = 1ull << HJ_MIN_BITS;
  while (cap * load_pct < nb * 100) cap <<= 1;
  uint32_t bits = 0;
  while ((1ull << bits) < cap) ++bits;
  return bits;
}

namespace {

// Home bucket of a key: buckets are aligned groups of 4 slots (one 32-byte
// sector); a table of 2^bits slots has 2^(bits-2) buckets.  The bucket is
// bits [64 - part_bits - (bits-2), 64 - part_bits) of key * PD_GOLDEN64,
// just below the bits that chose the partition.  part_bits + bits - 2 <= 30
// (the table layout caps all partitions together at 2^32 slots), so they all
// lie in the product's high word, computed here in 32-bit arithmetic.
__device__ __forceinline__ uint32_t bucket_of(uint32_t key, uint32_t part_bits, uint32_t bits) {
  const uint32_t hi = __umulhi(key, (uint32_t)PD_GOLDEN64) + key * (uint32_t)(PD_GOLDEN64 >> 32);
  return (hi << part_bits) >> (34 - bits);
}

struct JoinParams {
  // table
  unsigned long long *table;
  uint32_t bits, part_bits;
  uint32_t *side_count;
  uint32_t *dup_flag;           // set by the build when a key occurs twice
  // build side (partition p = rows [boff[p], boff[p+1]))
  const uint32_t *bkey, *bpay;  // bpay NULL: payload = row id
  const uint32_t *boff;         // device partition offsets (NULL: whole input)
  uint64_t nb;
  // probe side
  const uint32_t *pkey, *prow;  // prow NULL: row id = index
  const uint32_t *poff;
  const uint32_t *tilebase;     // first global tile of each partition
  uint64_t np;
  uint32_t part;
  // output
  uint32_t *out_pay, *out_row;
  uint64_t cap;
  uint64_t *status;
  uint32_t epoch;
  uint32_t *claim;
  uint32_t *d_error;
  uint64_t *d_count;
  uint64_t total_tiles;         // for d_count (direct path)
};

__device__ __forceinline__ void part_range(const uint32_t *off, uint32_t p, uint64_t n,
                                           uint64_t *lo, uint64_t *hi) {
  if (off) {
    *lo = off[p];
    *hi = off[p + 1];
  } else {
    *lo = 0;
    *hi = n;
  }
}

// Fills the table region with the empty word and zeroes the side count.
__global__ void __launch_bounds__(256) k_hj_clear(JoinParams p) {
  const uint64_t n = 1ull << p.bits;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  ulonglong2 e = make_ulonglong2(HJ_EMPTY, HJ_EMPTY);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 2; i += stride)
    reinterpret_cast<ulonglong2 *>(p.table)[i] = e;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *p.side_count = 0;
    *p.dup_flag = 0;
  }
}

// Inserts one build row (bucketized linear probing: the first free slot of the
// first bucket, from the home bucket on, that has one; every copy of a key
// therefore lies between its home bucket and the first bucket with a free
// slot).  The one row whose slot word would equal the empty word is counted
// on the side.
__device__ __forceinline__ void hj_insert(const JoinParams &p, uint32_t k, uint32_t v) {
  const unsigned long long e = ((unsigned long long)v << 32) | k;
  if (e == HJ_EMPTY) {
    atomicAdd(p.side_count, 1u);
    return;
  }
  const uint32_t gmask = (uint32_t)(((1ull << p.bits) - 1) >> 2);
  uint32_t g = bucket_of(k, p.part_bits, p.bits);
  bool done = false;
  bool dup = false;
  for (uint64_t t = 0; t <= gmask && !done; ++t) {
    unsigned long long *b = p.table + 4 * (uint64_t)g;
    // the whole bucket (one 32-byte sector) in two loads from L2; a slot a
    // concurrent insert has filled may still read empty, and its CAS then
    // returns the filled word, so duplicates are still seen
    const ulonglong2 lo = __ldcg(reinterpret_cast<const ulonglong2 *>(b));
    const ulonglong2 hi = __ldcg(reinterpret_cast<const ulonglong2 *>(b) + 1);
    const unsigned long long cur[4] = {lo.x, lo.y, hi.x, hi.y};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (done) break;
      if (cur[j] != HJ_EMPTY) {
        dup |= (uint32_t)cur[j] == k;
        continue;
      }
      const unsigned long long old = atomicCAS(b + j, HJ_EMPTY, e);
      if (old == HJ_EMPTY) done = true;
      else dup |= (uint32_t)old == k;
    }
    g = (g + 1) & gmask;
  }
  if (dup) *p.dup_flag = 1;
  if (!done) atomicOr(p.d_error, PD_DEVERR_TABLE_FULL);
}

__global__ void __launch_bounds__(256) k_hj_build(JoinParams p) {
  uint64_t lo, hi;
  part_range(p.boff, p.part, p.nb, &lo, &hi);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = lo + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += stride)
    hj_insert(p, p.bkey[i], p.bpay ? p.bpay[i] : (uint32_t)i);
}

// Resolves one bucket of a probe row: adds its matches to *c (first payload
// in *first) and returns true when the walk ends here -- the bucket has a free
// slot, or (no duplicate build key) a match was found.
__device__ __forceinline__ bool resolve_bucket(ulonglong2 lo, ulonglong2 hi, uint32_t key,
                                               bool stop_first, uint32_t *c, uint32_t *first) {
  const unsigned long long e[4] = {lo.x, lo.y, hi.x, hi.y};
  bool has_empty = false;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (e[j] == HJ_EMPTY) {
      has_empty = true;
    } else if ((uint32_t)e[j] == key) {
      if (*c == 0) *first = (uint32_t)(e[j] >> 32);
      ++*c;
    }
  }
  return has_empty || (stop_first && *c);
}

// Writes every match of key (bucket walk from its home bucket) from output
// position w on; returns the number of matches.
// (The table and output fields are passed by value: a reference to the
// parameter struct would make every caller copy it to local memory.)
__device__ __noinline__ uint32_t emit_all(const unsigned long long *table, uint32_t bits,
                                          uint32_t part_bits, uint32_t *out_pay, uint32_t *out_row,
                                          uint64_t cap, uint32_t key, uint64_t w, uint32_t row,
                                          bool *overflow, bool emit) {
  const uint32_t gmask = (uint32_t)(((1ull << bits) - 1) >> 2);
  uint32_t g = bucket_of(key, part_bits, bits);
  uint32_t c = 0;
  for (uint64_t t = 0; t <= gmask; ++t) {
    bool has_empty = false;
    for (int j = 0; j < 4; ++j) {
      const unsigned long long e = table[4 * (uint64_t)g + j];
      if (e == HJ_EMPTY) {
        has_empty = true;
      } else if ((uint32_t)e == key) {
        if (emit) {
          if (w < cap) { out_pay[w] = (uint32_t)(e >> 32); out_row[w] = row; } else *overflow = true;
        }
        ++w;
        ++c;
      }
    }
    if (has_empty) break;
    g = (g + 1) & gmask;
  }
  return c;
}

// One probe tile: rows [row0, min(row0 + HJ_TILE, hi)) of p, tile index gtile
// in p.status (the tile with index 0 starts the chain).  When count_last,
// the tile also stores the inclusive match count in *p.d_count.
__device__ __forceinline__ void hj_probe_tile(const JoinParams &p, uint64_t row0, uint64_t hi,
                                              uint64_t gtile, uint32_t side, bool stop_first,
                                              bool count_last) {
  __shared__ uint32_t s_warp[HJ_THREADS / 32];
  __shared__ uint64_t s_prefix;
  __shared__ uint32_t s_first[HJ_ITEMS][HJ_THREADS];  // first payload of each row
  __shared__ uint32_t s_row[HJ_ITEMS][HJ_THREADS];    // probe row id of each row (p.prow)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t mask = (1ull << p.bits) - 1;
  const uint32_t lt = (1u << lane) - 1u;
  // Warp-striped rows: row k of this lane is wbase + 32k + lane.
  const uint64_t wbase = row0 + (uint64_t)warp * (32 * HJ_ITEMS);

  // Phase 1: match counts (4 bits per row, 15 = "count again") and first payloads.
  uint64_t cnt4 = 0;
  uint32_t mine = 0;
#if PD_HJ_KEYS_FIRST
  // All keys and row ids of the thread are loaded together (one memory
  // latency per tile); row ids go straight to shared memory, where the
  // output phase reads them.
  uint32_t keys[HJ_ITEMS];
#pragma unroll
  for (int k = 0; k < HJ_ITEMS; ++k) {
    const uint64_t r = wbase + (uint64_t)k * 32 + lane;
    keys[k] = r < hi ? __ldcs(p.pkey + r) : 0u;
    s_row[k][tid] = (p.prow && r < hi) ? __ldcs(p.prow + r) : (uint32_t)r;
  }
#endif
#pragma unroll
  for (int b = 0; b < HJ_ITEMS; b += HJ_BATCH) {
    uint32_t key[HJ_BATCH], c[HJ_BATCH], fk[HJ_BATCH];
#if !PD_HJ_KEYS_FIRST
    uint32_t rowv[HJ_BATCH];
#endif
    uint32_t g[HJ_BATCH];
    bool active[HJ_BATCH];
#pragma unroll
    for (int i = 0; i < HJ_BATCH; ++i) {
      const uint64_t r = wbase + (uint64_t)(b + i) * 32 + lane;
      active[i] = r < hi;
#if PD_HJ_KEYS_FIRST
      key[i] = keys[b + i];
#else
      key[i] = active[i] ? __ldcs(p.pkey + r) : 0u;
      // row ids are loaded here, with the keys, so the output phase reads them
      // from shared memory instead of waiting on a load per row
      rowv[i] = (p.prow && active[i]) ? __ldcs(p.prow + r) : (uint32_t)r;
#endif
      g[i] = bucket_of(key[i], p.part_bits, p.bits);
      c[i] = 0;
      fk[i] = 0;
    }
    // Lockstep bucket walks: all loads of a round are in flight together;
    // almost every row resolves in its home bucket.
    const uint32_t gmask = (uint32_t)(mask >> 2);
    for (uint64_t round = 0; round <= gmask; ++round) {
      ulonglong2 glo[HJ_BATCH], ghi[HJ_BATCH];
      bool any = false;
#pragma unroll
      for (int i = 0; i < HJ_BATCH; ++i) {
        if (active[i]) {
          const ulonglong2 *q = reinterpret_cast<const ulonglong2 *>(p.table + 4 * (uint64_t)g[i]);
          glo[i] = q[0];
          ghi[i] = q[1];
          any = true;
        }
      }
      if (!any) break;
#pragma unroll
      for (int i = 0; i < HJ_BATCH; ++i) {
        if (!active[i]) continue;
        if (resolve_bucket(glo[i], ghi[i], key[i], stop_first && key[i] != 0xFFFFFFFFu, &c[i],
                           &fk[i]))
          active[i] = false;
        g[i] = (g[i] + 1) & gmask;
      }
    }
#pragma unroll
    for (int i = 0; i < HJ_BATCH; ++i) {
      const int k = b + i;
      const uint64_t r = wbase + (uint64_t)k * 32 + lane;
      uint32_t ci = c[i];
      if (r < hi && key[i] == 0xFFFFFFFFu) {
        // the side rows follow the table's matches; with none in the table
        // the first payload is the side row's (all ones)
        if (ci == 0 && side) fk[i] = 0xFFFFFFFFu;
        ci += side;
      }
      s_first[k][tid] = fk[i];
#if !PD_HJ_KEYS_FIRST
      s_row[k][tid] = rowv[i];
#endif
      mine += ci;
      cnt4 |= (uint64_t)(ci < 15 ? ci : 15u) << (4 * k);
    }
  }
  // Block scan of per-thread totals; tile look-back.
  uint32_t inc = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  const uint32_t wtot = __shfl_sync(0xffffffffu, inc, 31);
  if (lane == 0) s_warp[warp] = wtot;
  __syncthreads();
  uint32_t wpre = 0, total = 0;
#pragma unroll
  for (int w = 0; w < HJ_THREADS / 32; ++w) {
    uint32_t x = s_warp[w];
    if (w < warp) wpre += x;
    total += x;
  }
  if (gtile == 0) {
    if (tid == 0) {
      pd_store_relaxed_u64(p.status, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, total));
      s_prefix = 0;
    }
  } else {
    // One warp waits for the predecessors; the others wait at the barrier
    // below without taking issue slots from the SM's other CTAs.
    if (warp == 0) {
      if (lane == 0)
        pd_store_relaxed_u64(p.status + gtile, pd_pack_status(p.epoch, PD_FLAG_AGGREGATE, total));
      const uint64_t pre = pd_lookback_warp(p.status, (int64_t)gtile, p.epoch, p.d_error);
      if (lane == 0) {
        pd_store_relaxed_u64(p.status + gtile, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, pre + total));
        s_prefix = pre;
      }
    }
  }
  __syncthreads();
  // Phase 2: rows in order (k-major, then lane) -> consecutive output slots.
  uint64_t w = s_prefix + wpre;
  bool overflow = false;
#pragma unroll
  for (int k = 0; k < HJ_ITEMS; ++k) {
    const uint32_t c4 = (uint32_t)(cnt4 >> (4 * k)) & 15u;
    const uint64_t r = wbase + (uint64_t)k * 32 + lane;
    const bool simple = c4 <= 1;
    if (__all_sync(0xffffffffu, simple)) {
      const unsigned m = __ballot_sync(0xffffffffu, c4 == 1);
      if (c4 == 1) {
        const uint64_t pos = w + __popc(m & lt);
        const uint32_t row = s_row[k][tid];
        if (pos < p.cap) { p.out_pay[pos] = s_first[k][tid]; p.out_row[pos] = row; } else overflow = true;
      }
      w += __popc(m);
    } else {
      // some lane has several matches: exact counts by a second walk
      uint32_t c = 0;
      const uint32_t key = (r < hi && c4) ? p.pkey[r] : 0u;
      if (c4 == 1) c = 1;
      else if (c4 > 1) {
        bool dummy = false;
        c = emit_all(p.table, p.bits, p.part_bits, p.out_pay, p.out_row, p.cap, key, 0, 0, &dummy,
                     false);  // count only
        if (key == 0xFFFFFFFFu) c += side;
      }
      uint32_t ci = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, ci, o);
        if (lane >= o) ci += t;
      }
      const uint64_t pos = w + ci - c;
      const uint32_t row = c ? s_row[k][tid] : 0u;
      if (c4 == 1) {
        if (pos < p.cap) { p.out_pay[pos] = s_first[k][tid]; p.out_row[pos] = row; } else overflow = true;
      } else if (c) {
        uint64_t q = pos + emit_all(p.table, p.bits, p.part_bits, p.out_pay, p.out_row, p.cap, key,
                                    pos, row, &overflow, true);
        if (key == 0xFFFFFFFFu) {
          for (uint32_t m2 = 0; m2 < side; ++m2, ++q) {
            if (q < p.cap) { p.out_pay[q] = 0xFFFFFFFFu; p.out_row[q] = row; } else overflow = true;
          }
        }
      }
      w += __shfl_sync(0xffffffffu, ci, 31);
    }
  }
  if (overflow) atomicOr(p.d_error, PD_DEVERR_CAPACITY);
  if (count_last && tid == 0) *p.d_count = s_prefix + total;
  __syncthreads();
}

__global__ void __launch_bounds__(HJ_THREADS, PD_HJ_MIN_CTAS) k_hj_probe(JoinParams p) {
  __shared__ uint64_t s_tile;
  const int tid = threadIdx.x;
  uint64_t lo, hi;
  part_range(p.poff, p.part, p.np, &lo, &hi);
  const uint64_t tiles = pd_ceil_div(hi - lo, HJ_TILE);
  const uint64_t gbase = p.tilebase ? p.tilebase[p.part] : 0;
  const uint32_t side = *p.side_count;
  const bool stop_first = *p.dup_flag == 0;
  while (true) {
    if (tid == 0) {
      uint64_t t = atomicAdd(p.claim, 1u);
      if (t >= tiles && atomicAdd(p.claim + 1, 1u) == gridDim.x - 1) {
        p.claim[0] = 0;  // last claimer of the launch resets the counters
        p.claim[1] = 0;
      }
      s_tile = t;
    }
    __syncthreads();
    const uint64_t tl = s_tile;
    if (tl >= tiles) break;
    hj_probe_tile(p, lo + tl * HJ_TILE, hi, gbase + tl, side, stop_first, false);
  }
}

// Total match count: the inclusive prefix of the last global probe tile.
__global__ void k_hj_count(const uint64_t *status, const uint32_t *tilebase, uint32_t parts,
                           uint64_t total_tiles, uint32_t epoch, uint64_t *d_count) {
  uint64_t tiles = tilebase ? tilebase[parts] : total_tiles;
  uint64_t v = 0;
  if (tiles) {
    uint64_t w = pd_load_relaxed_u64(status + tiles - 1);
    v = w & PD_STATUS_VALUE_MASK;
  }
  *d_count = v;
}

// Exclusive offsets (uint32, P+1 entries) of two partitioned relations and the
// first global probe tile of each partition.
__global__ void k_hj_offsets(const uint32_t *boffs, const uint32_t *poffs, uint32_t parts,
                             uint64_t nb, uint64_t np, uint32_t *boff, uint32_t *poff,
                             uint32_t *tilebase) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint64_t t = 0;
  for (uint32_t q = 0; q < parts; ++q) {
    boff[q] = boffs[q];
    poff[q] = poffs[q];
    tilebase[q] = (uint32_t)t;
    uint64_t end = (q + 1 < parts) ? poffs[q + 1] : np;
    t += pd_ceil_div(end - poffs[q], HJ_TILE);
  }
  boff[parts] = (uint32_t)nb;
  poff[parts] = (uint32_t)np;
  tilebase[parts] = (uint32_t)t;
}

// ---------------------------------------------------------------------------
// Batched hash join (pd_hj_batch): every instance has its own table (never
// partitioned).  Build: CTAs take (instance, row block) items.  Probe:
// persistent CTAs claim probe tiles in instance-major order; each instance's
// tiles form their own look-back chain (status words from the instance's
// first tile), so every instance's output is in probe order, exactly as its
// plain unpartitioned join.  The look-back epoch lives on the device and is
// advanced by the run itself, so a captured run can be replayed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ JoinParams hjb_params(const pd_hj_batch &b, const pd_hj_inst &in) {
  JoinParams p{};
  p.table = in.table;
  p.bits = in.bits;
  p.part_bits = 0;
  p.side_count = in.header;
  p.dup_flag = in.header + 2;
  p.bkey = in.bkey;
  p.bpay = in.bpay;
  p.nb = in.nb;
  p.pkey = in.pkey;
  p.prow = in.prow;
  p.np = in.np;
  p.out_pay = in.out_pay;
  p.out_row = in.out_row;
  p.cap = in.cap;
  p.status = b.status + in.tile0;
  p.d_error = b.d_error;
  p.d_count = in.d_count;
  return p;
}

// Advances the device epoch (1..65535); instances without probe rows get a
// zero count (no tile of theirs will write it).
__global__ void k_hjb_begin(pd_hj_batch b) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *b.epoch = *b.epoch % 65535u + 1u;
  if (i < b.count && b.tile0[i + 1] == b.tile0[i]) *b.inst[i].d_count = 0;
}

// After a wrap of the epoch, stale words could carry the new epoch: clear them.
__global__ void __launch_bounds__(256) k_hjb_status_clear(pd_hj_batch b) {
  if (*b.epoch != 1u) return;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.total_tiles; i += stride)
    b.status[i] = 0;
}

__global__ void __launch_bounds__(256) k_hjb_build(pd_hj_batch b) {
  for (uint32_t it = blockIdx.x; it < b.nbitems; it += gridDim.x) {
    const uint2 item = b.bitems[it];
    const pd_hj_inst &in = b.inst[item.x];
    const JoinParams p = hjb_params(b, in);
    const uint64_t r1 = min((uint64_t)item.y + b.build_rows_per_item, in.nb);
    for (uint64_t i = item.y + threadIdx.x; i < r1; i += blockDim.x)
      hj_insert(p, p.bkey[i], p.bpay ? p.bpay[i] : (uint32_t)i);
  }
}

__global__ void __launch_bounds__(HJ_THREADS, PD_HJ_MIN_CTAS) k_hjb_probe(pd_hj_batch b) {
  __shared__ uint64_t s_tile;
  const int tid = threadIdx.x;
  const uint32_t epoch = *b.epoch;
  while (true) {
    if (tid == 0) {
      const uint64_t t = atomicAdd(b.counters, 1u);
      if (t >= b.total_tiles && atomicAdd(b.counters + 1, 1u) == gridDim.x - 1) {
        b.counters[0] = 0;  // the last claimer of the launch resets the queue
        b.counters[1] = 0;
      }
      s_tile = t;
    }
    __syncthreads();
    const uint64_t t = s_tile;
    if (t >= b.total_tiles) break;
    uint32_t lo = 0, hi = b.count;  // the instance whose tiles contain t
    while (hi - lo > 1) {
      const uint32_t m = (lo + hi) >> 1;
      if (b.tile0[m] <= t) lo = m; else hi = m;
    }
    const pd_hj_inst &in = b.inst[lo];
    JoinParams p = hjb_params(b, in);
    p.epoch = epoch;
    const uint64_t tl = t - in.tile0;
    const uint64_t tiles = pd_ceil_div(in.np, HJ_TILE);
    hj_probe_tile(p, tl * HJ_TILE, in.np, tl, *p.side_count, *p.dup_flag == 0, tl == tiles - 1);
  }
}

int probe_grid(pimdal_ctx *ctx) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hj_probe, HJ_THREADS, 0);
    if (per_sm <= 0) per_sm = 1;
  }
  return per_sm * ctx->sm_count;
}

// ---------------------------------------------------------------------------
// Shared-memory partitions (partition_bits HJS_MIN_BITS..HJS_MAX_BITS): both
// relations are radix-partitioned (stable passes of at most 6 bits) by the
// top partition_bits of the multiplicative hash, so that one partition's
// build rows fit a linear-probing table in one CTA's shared memory -- the
// cache-sized partitions of the reference's CPU join
// (reference/db_operators/hash_join.cpp:57-157, 16384 ways) and the
// bucket-sized ones of its DPU join (pimdal/join/hash_join.c:40-115).  A
// persistent CTA per SM claims partitions in order; for each it fills the
// table, counts the matches of the partition's probe rows, resolves the
// partition's output offset by a decoupled look-back over the partitions,
// then probes the rows again (now from L2) and writes the pairs in probe
// order.  A partition with more than HJS_CHUNK build rows is joined one
// chunk of build rows at a time (its output is then chunk-major).
// ---------------------------------------------------------------------------
constexpr int HJS_THREADS = 1024;
constexpr int HJS_WARPS = HJS_THREADS / 32;
constexpr uint32_t HJS_SLOT_BITS = 14;
constexpr uint32_t HJS_SLOTS = 1u << HJS_SLOT_BITS;  // 128 KB of 8-byte slots
constexpr uint32_t HJS_CHUNK = HJS_SLOTS / 4 * 3;    // build rows per table fill
#ifndef PD_HJS_ITEMS
#define PD_HJS_ITEMS 8    // probe rows per thread and tile of the writing pass
#endif
#ifndef PD_HJS_CITEMS
#define PD_HJS_CITEMS 8   // probe rows per thread and tile of the counting pass
#endif
constexpr int HJS_ITEMS = PD_HJS_ITEMS;
constexpr int HJS_CITEMS = PD_HJS_CITEMS;
constexpr uint32_t HJS_MIN_BITS = 9, HJS_MAX_BITS = 16;
constexpr size_t HJS_SMEM = 8ull * HJS_SLOTS;

struct JoinSmemParams {
  const uint32_t *bkey, *bpay;  // partitioned build rows
  const uint32_t *pkey, *prow;  // partitioned probe rows
  const uint32_t *boff, *poff;  // parts + 1 partition offsets each
  uint32_t part_bits, parts;
  uint32_t *out_pay, *out_row;
  uint64_t cap;
  uint64_t *status;
  uint32_t epoch;
  uint32_t *claim;
  uint32_t *d_error;
  uint64_t *d_count;
};

// off[q] = the first row whose partition (top `bits` of the multiplicative
// hash) is >= q, for q = 0..parts.
__global__ void __launch_bounds__(256) k_hjs_bounds(const uint32_t *key, uint64_t n, uint32_t bits,
                                                    uint32_t parts, uint32_t *off) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > parts) return;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((pd_mulhash32(key[mid]) >> (32 - bits)) < q) lo = mid + 1;
    else hi = mid;
  }
  off[q] = (uint32_t)lo;
}

// A key's home slot: the hash bits just below the ones that chose its
// partition.
__device__ __forceinline__ uint32_t hjs_slot(uint32_t key, uint32_t part_bits) {
  return (pd_mulhash32(key) << part_bits) >> (32 - HJS_SLOT_BITS);
}

// Clears the table and inserts build rows [r0, r1), r1 - r0 <= HJS_CHUNK (so
// every walk finds a free slot), after every thread is done with the table's
// previous contents.  The one row whose slot word would equal the empty word
// is counted in *s_side; *s_dup is set when a key occurs twice.
__device__ void hjs_fill(unsigned long long *tab, const JoinSmemParams &p, uint64_t r0, uint64_t r1,
                         uint32_t *s_side, uint32_t *s_dup) {
  __syncthreads();
  const ulonglong2 e2 = make_ulonglong2(HJ_EMPTY, HJ_EMPTY);
  for (uint32_t i = threadIdx.x; i < HJS_SLOTS / 2; i += HJS_THREADS)
    reinterpret_cast<ulonglong2 *>(tab)[i] = e2;
  if (threadIdx.x == 0) {
    *s_side = 0;
    *s_dup = 0;
  }
  __syncthreads();
  for (uint64_t i = r0 + threadIdx.x; i < r1; i += HJS_THREADS) {
    const uint32_t k = __ldcs(p.bkey + i), v = __ldcs(p.bpay + i);
    const unsigned long long e = ((unsigned long long)v << 32) | k;
    if (e == HJ_EMPTY) {
      atomicAdd(s_side, 1u);
      continue;
    }
    uint32_t s = hjs_slot(k, p.part_bits);
    for (uint32_t t = 0; t < HJS_SLOTS; ++t) {
      const unsigned long long old = atomicCAS(tab + s, HJ_EMPTY, e);
      if (old == HJ_EMPTY) break;
      if ((uint32_t)old == k) *s_dup = 1;
      s = (s + 1) & (HJS_SLOTS - 1);
    }
  }
  __syncthreads();
}

// Matches of key in the table (the walk ends at a free slot, or at the first
// match when no key occurs twice); *first gets the first match's payload.
__device__ __forceinline__ uint32_t hjs_find(const unsigned long long *tab, uint32_t key,
                                             uint32_t part_bits, bool stop_first, uint32_t *first) {
  uint32_t s = hjs_slot(key, part_bits), c = 0;
  for (uint32_t t = 0; t < HJS_SLOTS; ++t) {
    const unsigned long long e = tab[s];
    if (e == HJ_EMPTY) break;
    if ((uint32_t)e == key) {
      if (c == 0) *first = (uint32_t)(e >> 32);
      ++c;
      if (stop_first) break;
    }
    s = (s + 1) & (HJS_SLOTS - 1);
  }
  return c;
}

// Writes every match of key (then `side` all-ones payloads for the all-ones
// key) from output position w on; returns the next position.
__device__ uint64_t hjs_emit(const unsigned long long *tab, const JoinSmemParams &p, uint32_t key,
                             uint32_t row, uint32_t side, uint64_t w, bool *overflow) {
  uint32_t s = hjs_slot(key, p.part_bits);
  for (uint32_t t = 0; t < HJS_SLOTS; ++t) {
    const unsigned long long e = tab[s];
    if (e == HJ_EMPTY) break;
    if ((uint32_t)e == key) {
      if (w < p.cap) { p.out_pay[w] = (uint32_t)(e >> 32); p.out_row[w] = row; } else *overflow = true;
      ++w;
    }
    s = (s + 1) & (HJS_SLOTS - 1);
  }
  if (key == 0xFFFFFFFFu) {
    for (uint32_t m = 0; m < side; ++m, ++w) {
      if (w < p.cap) { p.out_pay[w] = 0xFFFFFFFFu; p.out_row[w] = row; } else *overflow = true;
    }
  }
  return w;
}

// One tile of a partition's probe rows [t0, min(t0 + HJS_THREADS * ITEMS,
// r1)): warp w takes rows t0 + w * 32 * ITEMS + 32k + lane.  COUNT: returns
// the thread's match total.  Otherwise writes the tile's pairs in probe order
// from output position *base on (the same in every thread) and advances
// *base past them.
template <bool COUNT, int ITEMS>
__device__ __forceinline__ uint32_t hjs_tile(const unsigned long long *tab, const JoinSmemParams &p,
                                             uint64_t t0, uint64_t r1, uint32_t side, bool stop_first,
                                             uint64_t *base, uint32_t *s_warp, bool *overflow) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t wb = t0 + (uint64_t)warp * (32 * ITEMS);
  uint32_t key[ITEMS], row[COUNT ? 1 : ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint64_t r = wb + 32 * k + lane;
    // the counting pass leaves the keys in L2 for the writing pass
    key[k] = r < r1 ? (COUNT ? __ldcg(p.pkey + r) : __ldcs(p.pkey + r)) : 0u;
    if (!COUNT) row[k] = r < r1 ? __ldcs(p.prow + r) : 0u;
  }
  uint32_t c[ITEMS], f[ITEMS], mine = 0;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    c[k] = 0;
    f[k] = 0;
    if (wb + 32 * k + lane < r1) {
      const bool ones = key[k] == 0xFFFFFFFFu;
      c[k] = hjs_find(tab, key[k], p.part_bits, stop_first && !ones, &f[k]) + (ones ? side : 0u);
    }
    mine += c[k];
  }
  if (COUNT) return mine;

  uint32_t wtot = mine;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wtot += __shfl_xor_sync(0xffffffffu, wtot, o);
  if (lane == 0) s_warp[warp] = wtot;
  __syncthreads();
  uint64_t w = *base;
  uint32_t total = 0;
#pragma unroll
  for (int i = 0; i < HJS_WARPS; ++i) {
    const uint32_t x = s_warp[i];
    if (i < warp) w += x;
    total += x;
  }
  __syncthreads();  // s_warp is written again by the next tile
  *base += total;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    // one table match (not the all-ones key, whose side rows need the walk)
    const bool one = c[k] == 1 && key[k] != 0xFFFFFFFFu;
    if (__all_sync(0xffffffffu, c[k] == 0 || one)) {
      const unsigned m = __ballot_sync(0xffffffffu, one);
      if (one) {
        const uint64_t pos = w + __popc(m & lt);
        if (pos < p.cap) { p.out_pay[pos] = f[k]; p.out_row[pos] = row[k]; } else *overflow = true;
      }
      w += __popc(m);
    } else {
      uint32_t ci = c[k];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, ci, o);
        if (lane >= o) ci += t;
      }
      const uint64_t pos = w + ci - c[k];
      if (one) {
        if (pos < p.cap) { p.out_pay[pos] = f[k]; p.out_row[pos] = row[k]; } else *overflow = true;
      } else if (c[k]) {
        hjs_emit(tab, p, key[k], row[k], side, pos, overflow);
      }
      w += __shfl_sync(0xffffffffu, ci, 31);
    }
  }
  return mine;
}

__device__ __forceinline__ uint64_t hjs_block_sum(uint64_t v, unsigned long long *s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) *s_red = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicAdd(s_red, (unsigned long long)v);
  __syncthreads();
  return *s_red;
}

// Persistent: one CTA per SM claims partitions in order.
__global__ void __launch_bounds__(HJS_THREADS, 1) k_hjs_join(JoinSmemParams p) {
  extern __shared__ __align__(16) unsigned long long hjs_tab[];
  __shared__ uint32_t s_warp[HJS_WARPS];
  __shared__ uint32_t s_side, s_dup, s_part;
  __shared__ unsigned long long s_red;
  __shared__ uint64_t s_prefix;
  const int tid = threadIdx.x;
  bool overflow = false;
  while (true) {
    __syncthreads();  // s_part and s_red of the previous partition have been read
    if (tid == 0) {
      const uint32_t q = atomicAdd(p.claim, 1u);
      if (q >= p.parts && atomicAdd(p.claim + 1, 1u) == gridDim.x - 1) {
        p.claim[0] = 0;  // last claimer of the launch resets the counters
        p.claim[1] = 0;
      }
      s_part = q;
    }
    __syncthreads();
    const uint32_t q = s_part;
    if (q >= p.parts) break;
    const uint64_t b0 = p.boff[q], b1 = p.boff[q + 1], r0 = p.poff[q], r1 = p.poff[q + 1];
    const uint32_t chunks = b1 > b0 ? (uint32_t)pd_ceil_div(b1 - b0, HJS_CHUNK) : 0u;
    // 1. count the partition's matches (over every chunk of its build rows)
    uint64_t mine = 0;
    for (uint32_t ch = 0; ch < chunks; ++ch) {
      hjs_fill(hjs_tab, p, b0 + (uint64_t)ch * HJS_CHUNK, min(b1, b0 + (uint64_t)(ch + 1) * HJS_CHUNK),
               &s_side, &s_dup);
      const uint32_t side = s_side;
      const bool stop_first = s_dup == 0;
      for (uint64_t t0 = r0; t0 < r1; t0 += HJS_THREADS * HJS_CITEMS)
        mine += hjs_tile<true, HJS_CITEMS>(hjs_tab, p, t0, r1, side, stop_first, nullptr, s_warp,
                                           &overflow);
    }
    const uint64_t total = hjs_block_sum(mine, &s_red);
    // 2. the partition's output offset
    if (tid < 32) {
      uint64_t pre = 0;
      if (q == 0) {
        if (tid == 0) pd_store_relaxed_u64(p.status, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, total));
      } else {
        if (tid == 0)
          pd_store_relaxed_u64(p.status + q, pd_pack_status(p.epoch, PD_FLAG_AGGREGATE, total));
        pre = pd_lookback_warp(p.status, (int64_t)q, p.epoch, p.d_error);
        if (tid == 0)
          pd_store_relaxed_u64(p.status + q, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, pre + total));
      }
      if (tid == 0) {
        s_prefix = pre;
        if (q == p.parts - 1) *p.d_count = pre + total;
      }
    }
    __syncthreads();
    // 3. write the pairs (a single chunk is still in the table)
    uint64_t base = s_prefix;
    for (uint32_t ch = 0; ch < chunks; ++ch) {
      if (chunks > 1)
        hjs_fill(hjs_tab, p, b0 + (uint64_t)ch * HJS_CHUNK, min(b1, b0 + (uint64_t)(ch + 1) * HJS_CHUNK),
                 &s_side, &s_dup);
      const uint32_t side = s_side;
      const bool stop_first = s_dup == 0;
      for (uint64_t t0 = r0; t0 < r1; t0 += HJS_THREADS * HJS_ITEMS)
        hjs_tile<false, HJS_ITEMS>(hjs_tab, p, t0, r1, side, stop_first, &base, s_warp, &overflow);
    }
  }
  if (overflow) atomicOr(p.d_error, PD_DEVERR_CAPACITY);
}

#ifndef PD_HJ_ONE_TABLE
#define PD_HJ_ONE_TABLE 1
#endif

struct HjLayout {
  uint32_t bits, part_bits;
  bool smem;  // shared-memory partitions (k_hjs_join)
  size_t table, side, boff, poff, tilebase, bk, bp, pk, pr, sort_ws, total;
};

// Shared-memory partitions: partitioned copies of both relations, their
// partition offsets and the partition passes' workspace.
bool hjs_layout(const pimdal_hash_join_arguments_t *a, HjLayout *l) {
  const uint32_t pb = a->partition_bits;
  l->smem = true;
  l->part_bits = pb;
  l->bits = 0;
  const size_t offs = pd_align_up(4 * ((1ull << pb) + 1), 256);
  size_t o = 0;
  l->table = l->side = l->tilebase = 0;
  l->boff = o; o += offs;
  l->poff = o; o += offs;
  l->bk = o; o += pd_align_up(4 * a->size_build, 256);
  l->bp = o; o += pd_align_up(4 * a->size_build, 256);
  l->pk = o; o += pd_align_up(4 * a->size_probe, 256);
  l->pr = o; o += pd_align_up(4 * a->size_probe, 256);
  pimdal_sort_arguments_t sa{};
  sa.key_dtype = PIMDAL_U32;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;
  sa.nr_elements = std::max(a->size_build, a->size_probe);
  sa.begin_bit = 32 - pb;
  sa.end_bit = 32;
  const size_t w = pd_partition_workspace(&sa, false);
  if (!w) return false;
  l->sort_ws = o; o += w;
  l->total = o;
  return true;
}

bool hj_layout(const pimdal_hash_join_arguments_t *a, HjLayout *l) {
  if (a->partition_bits >= HJS_MIN_BITS && a->partition_bits <= HJS_MAX_BITS) return hjs_layout(a, l);
  l->smem = false;
  const uint32_t load_pct = a->load_factor_pct ? a->load_factor_pct : 50;
  if (load_pct > 90) return false;
  const uint32_t bits = pd_hj_table_bits(a->size_build, load_pct);
  if (bits > 32) return false;  // bucket_of's 32-bit arithmetic
  uint64_t budget = a->l2_budget_bytes ? a->l2_budget_bytes : (48ull << 20);
  uint32_t pb = a->partition_bits;
  if (pb == 0xFFFFFFFFu) pb = 0;  // explicit "no partitioning"
  else if (pb == 0) {
    while ((8ull << bits) > (budget << pb) && pb < 8) ++pb;
  }
  if (pb > 8 || pb >= bits) return false;
  l->part_bits = pb;
#if PD_HJ_ONE_TABLE
  l->bits = bits;  // one table; partition q's rows touch only its slice q
#else
  l->bits = bits - pb;  // slots of one partition's table
#endif
  size_t o = 0;
  l->table = o; o += pd_align_up(8ull << l->bits, 256);
  l->side = o; o += 256;
  l->boff = o; o += pd_align_up(4 * 257, 256);
  l->poff = o; o += pd_align_up(4 * 257, 256);
  l->tilebase = o; o += pd_align_up(4 * 257, 256);
  l->bk = l->bp = l->pk = l->pr = l->sort_ws = 0;
  if (pb) {
    l->bk = o; o += pd_align_up(4 * a->size_build, 256);
    l->bp = o; o += pd_align_up(4 * a->size_build, 256);
    l->pk = o; o += pd_align_up(4 * a->size_probe, 256);
    l->pr = o; o += pd_align_up(4 * a->size_probe, 256);
    pimdal_sort_arguments_t sa{};
    sa.nr_elements = std::max(a->size_build, a->size_probe);
    sa.begin_bit = 32 - pb;
    sa.end_bit = 32;
    size_t w = 0;
    if (pimdal_sort_workspace_size(&sa, &w)) return false;
    l->sort_ws = o; o += w;
  }
  l->total = o;
  return true;
}

}  // namespace

uint32_t pd_hj_tile_rows() { return HJ_TILE; }

int pd_hj_batch_run(pimdal_ctx *ctx, const pd_hj_batch &b, cudaStream_t s) {
  if (b.table_words) PD_CHECK_CUDA(cudaMemsetAsync(b.tables, 0xFF, 8 * b.table_words, s));
  PD_CHECK_CUDA(cudaMemsetAsync(b.headers, 0, 32ull * b.count, s));
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_hjb_begin<<<(b.count + 255) / 256, 256, 0, s>>>(b);
  }
  if (b.total_tiles) {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    const unsigned g = (unsigned)std::min<uint64_t>(pd_ceil_div(b.total_tiles, 256), ctx->sm_count * 4ull);
    k_hjb_status_clear<<<g, 256, 0, s>>>(b);
  }
  if (b.nbitems) {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_BUILD, s);
    k_hjb_build<<<std::min<unsigned>(b.nbitems, ctx->sm_count * 8), 256, 0, s>>>(b);
  }
  if (b.total_tiles) {
    static int per_sm = 0;
    if (!per_sm) {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hjb_probe, HJ_THREADS, 0);
      if (per_sm <= 0) per_sm = 1;
    }
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_PROBE, s);
    const unsigned g = (unsigned)std::min<uint64_t>(b.total_tiles, (uint64_t)per_sm * ctx->sm_count);
    k_hjb_probe<<<g, HJ_THREADS, 0, s>>>(b);
  }
  return pd_launch_status(ctx);
}

// ---------------------------------------------------------------------------
// pimdal_hash_join
// ---------------------------------------------------------------------------
namespace {
// The autotuner's candidates: the partition fan-out the L2 budget suggests
// (at load factor 1/2) and two neighbours either side, times load factors
// 35/50/70 %.
std::vector<pimdal_hash_join_arguments_t> hj_candidates(const pimdal_hash_join_arguments_t *a) {
  std::vector<pimdal_hash_join_arguments_t> c;
  pimdal_hash_join_arguments_t t = *a;
  t.partition_bits = 0;
  t.load_factor_pct = 50;
  HjLayout l;
  if (!hj_layout(&t, &l)) return c;
  for (int d = -2; d <= 2; ++d) {
    const int pb = (int)l.part_bits + d;
    if (pb < 0 || pb > 8) continue;
    for (uint32_t lf : {35u, 50u, 70u}) {
      t.partition_bits = pb == 0 ? 0xFFFFFFFFu : (uint32_t)pb;
      t.load_factor_pct = lf;
      HjLayout m;
      if (hj_layout(&t, &m)) c.push_back(t);
    }
  }
  // shared-memory partitions of about a half and a quarter of a table's slots
  uint32_t sb = HJS_MIN_BITS;
  while (sb < HJS_MAX_BITS && (a->size_build >> sb) > HJS_SLOTS / 2) ++sb;
  for (uint32_t pb = sb; pb <= std::min(sb + 1, HJS_MAX_BITS); ++pb) {
    t.partition_bits = pb;
    t.load_factor_pct = 0;
    HjLayout m;
    if (hj_layout(&t, &m)) c.push_back(t);
  }
  return c;
}

std::vector<uint64_t> hj_shape(const pimdal_hash_join_arguments_t *a) {
  return {1, pd_log2_ceil(a->size_build), pd_log2_ceil(a->size_probe), a->l2_budget_bytes};
}

bool hj_auto(const pimdal_hash_join_arguments_t *a) {
  return a->partition_bits == 0 && a->load_factor_pct == 0;
}

// The join over shared-memory partitions: both relations partitioned by the
// top part_bits of the multiplicative hash (stable passes of at most 6 bits,
// row ids made in the first pass when a relation has no payload column),
// their partition offsets found by binary search, then k_hjs_join.
int hjs_run(pimdal_ctx *ctx, const pimdal_hash_join_arguments_t *a, const HjLayout &l, char *ws,
            pimdal_merge_results_t *d_result, cudaStream_t s) {
  const uint32_t pb = l.part_bits, parts = 1u << pb;
  int st;
  JoinSmemParams p{};
  p.part_bits = pb;
  p.parts = parts;
  p.out_pay = a->out_build_payload;
  p.out_row = a->out_probe_ptr;
  p.cap = a->out_capacity;
  p.status = ctx->d_status;
  p.claim = ctx->d_counters + PD_COUNTER_PROBE;
  p.d_error = ctx->d_error;
  p.d_count = &d_result->t_count;
  p.epoch = pd_next_epoch(ctx, s, &st);
  if (st) return st;
  pimdal_sort_arguments_t sa{};
  sa.key_dtype = PIMDAL_U32;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;
  sa.begin_bit = 32 - pb;
  sa.end_bit = 32;
  sa.nr_elements = a->size_build;
  sa.in = a->build_key;
  sa.in_ptr = a->build_payload;
  sa.out = ws + l.bk;
  sa.out_ptr = (uint32_t *)(ws + l.bp);
  if ((st = pd_partition(ctx, &sa, PD_KEY_MULHASH, ws + l.sort_ws, s, nullptr, nullptr))) return st;
  sa.nr_elements = a->size_probe;
  sa.in = a->probe_key;
  sa.in_ptr = a->probe_ptr;
  sa.out = ws + l.pk;
  sa.out_ptr = (uint32_t *)(ws + l.pr);
  if ((st = pd_partition(ctx, &sa, PD_KEY_MULHASH, ws + l.sort_ws, s, nullptr, nullptr))) return st;
  p.bkey = (const uint32_t *)(ws + l.bk);
  p.bpay = (const uint32_t *)(ws + l.bp);
  p.pkey = (const uint32_t *)(ws + l.pk);
  p.prow = (const uint32_t *)(ws + l.pr);
  p.boff = (const uint32_t *)(ws + l.boff);
  p.poff = (const uint32_t *)(ws + l.poff);
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    const unsigned g = (unsigned)pd_ceil_div(parts + 1, 256);
    k_hjs_bounds<<<g, 256, 0, s>>>(p.bkey, a->size_build, pb, parts, (uint32_t *)(ws + l.boff));
    k_hjs_bounds<<<g, 256, 0, s>>>(p.pkey, a->size_probe, pb, parts, (uint32_t *)(ws + l.poff));
  }
  PD_CHECK_CUDA(cudaFuncSetAttribute(k_hjs_join, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HJS_SMEM));
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_PROBE, s);
    k_hjs_join<<<ctx->sm_count, HJS_THREADS, HJS_SMEM, s>>>(p);
  }
  return pd_launch_status(ctx);
}
}  // namespace

extern "C" int pimdal_hash_join_workspace_size(const pimdal_hash_join_arguments_t *a, size_t *bytes) {
  if (!a || !bytes) return PIMDAL_ERR_ARG;
  HjLayout l;
  if (!hj_layout(a, &l)) return PIMDAL_ERR_ARG;
  *bytes = l.total;
  if (hj_auto(a)) {  // a tuned choice may be used instead: cover every candidate
    for (const auto &c : hj_candidates(a)) {
      HjLayout m;
      if (hj_layout(&c, &m)) *bytes = std::max(*bytes, m.total);
    }
  }
  return PIMDAL_OK;
}

extern "C" int pimdal_hash_join(pimdal_ctx_t *ctx, const pimdal_hash_join_arguments_t *a_in,
                                pimdal_merge_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a_in || !d_result) return PIMDAL_ERR_ARG;
  pimdal_hash_join_arguments_t eff = *a_in;
  if (hj_auto(a_in)) {  // the autotuner's choice for this shape, if any
    const auto it = ctx->op_tune.find(hj_shape(a_in));
    if (it != ctx->op_tune.end()) {
      eff.partition_bits = it->second.partition_bits;
      eff.load_factor_pct = it->second.load_factor_pct;
    }
  }
  const pimdal_hash_join_arguments_t *a = &eff;
  if ((a->size_build && !a->build_key) || (a->size_probe && !a->probe_key)) return PIMDAL_ERR_ARG;
  if (a->out_capacity && (!a->out_build_payload || !a->out_probe_ptr)) return PIMDAL_ERR_ARG;
  if (a->size_build >= (1ull << 32) || a->size_probe >= (1ull << 30)) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  if (a->size_build == 0 || a->size_probe == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d_result, 0, sizeof(uint64_t), s));
    return PIMDAL_OK;
  }
  HjLayout l;
  if (!hj_layout(a, &l)) return PIMDAL_ERR_ARG;
  int st;
  char *ws = (char *)pd_workspace(ctx, l.total, s, &st);
  if (!ws) return st;
  if (l.smem) return hjs_run(ctx, a, l, ws, d_result, s);
  const uint32_t parts = 1u << l.part_bits;
  const uint64_t total_tiles_direct = pd_ceil_div(a->size_probe, HJ_TILE);
  if (total_tiles_direct + parts > PD_STATUS_WORDS) return PIMDAL_ERR_ARG;

  JoinParams p{};
  p.table = (unsigned long long *)(ws + l.table);
  p.bits = l.bits;
  p.part_bits = l.part_bits;
  p.side_count = (uint32_t *)(ws + l.side);
  p.dup_flag = (uint32_t *)(ws + l.side) + 2;
  p.nb = a->size_build;
  p.np = a->size_probe;
  p.out_pay = a->out_build_payload;
  p.out_row = a->out_probe_ptr;
  p.cap = a->out_capacity;
  p.status = ctx->d_status;
  p.claim = ctx->d_counters + PD_COUNTER_PROBE;
  p.d_error = ctx->d_error;
  p.d_count = &d_result->t_count;
  p.epoch = pd_next_epoch(ctx, s, &st);
  if (st) return st;

  if (l.part_bits) {
    // Partition both relations by the top part_bits of the multiplicative hash.
    pimdal_sort_arguments_t sa{};
    sa.key_dtype = PIMDAL_U32;
    sa.layout = PIMDAL_LAYOUT_COLUMNS;
    sa.begin_bit = 32 - l.part_bits;
    sa.end_bit = 32;
    uint32_t *boffs, *poffs;
    sa.nr_elements = a->size_build;
    sa.in = a->build_key;
    sa.in_ptr = a->build_payload;
    sa.out = ws + l.bk;
    sa.out_ptr = (uint32_t *)(ws + l.bp);
    if ((st = pd_sort_ex(ctx, &sa, PD_KEY_MULHASH, ws + l.sort_ws, s, &boffs))) return st;
    // the build offsets live in the sort workspace: save them before reuse
    uint32_t *boff = (uint32_t *)(ws + l.boff), *poff = (uint32_t *)(ws + l.poff);
    PD_CHECK_CUDA(cudaMemcpyAsync(boff, boffs, 4 * parts, cudaMemcpyDeviceToDevice, s));
    sa.nr_elements = a->size_probe;
    sa.in = a->probe_key;
    sa.in_ptr = a->probe_ptr;
    sa.out = ws + l.pk;
    sa.out_ptr = (uint32_t *)(ws + l.pr);
    if ((st = pd_sort_ex(ctx, &sa, PD_KEY_MULHASH, ws + l.sort_ws, s, &poffs))) return st;
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_hj_offsets<<<1, 32, 0, s>>>(boff, poffs, parts, a->size_build, a->size_probe, boff, poff,
                                    (uint32_t *)(ws + l.tilebase));
    }
    p.bkey = (const uint32_t *)(ws + l.bk);
    p.bpay = (const uint32_t *)(ws + l.bp);
    p.pkey = (const uint32_t *)(ws + l.pk);
    p.prow = (const uint32_t *)(ws + l.pr);
    p.boff = boff;
    p.poff = poff;
    p.tilebase = (const uint32_t *)(ws + l.tilebase);
  } else {
    p.bkey = (const uint32_t *)a->build_key;
    p.bpay = a->build_payload;
    p.pkey = (const uint32_t *)a->probe_key;
    p.prow = a->probe_ptr;
  }
  const unsigned clear_grid = (unsigned)std::min<uint64_t>(pd_ceil_div(1ull << l.bits, 512), ctx->sm_count * 8ull);
  const unsigned build_grid = ctx->sm_count * 8;
  const int pgrid = probe_grid(ctx);
#if PD_HJ_ONE_TABLE
  if (l.part_bits) {
    // One table of 2^bits slots for all partitions, one build and one probe
    // launch over the partitioned rows.  A key's home bucket is the top bits
    // of the same hash whose top part_bits chose its partition, so the rows of
    // partition q touch only slice q of the table: the slice being built or
    // probed stays L2-resident, and no launch waits for a partition's tail.
    p.boff = p.poff = nullptr;
    p.tilebase = nullptr;
    p.part_bits = 0;
    p.part = 0;
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_hj_clear<<<clear_grid, 256, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_BUILD, s);
      k_hj_build<<<build_grid, 256, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_PROBE, s);
      k_hj_probe<<<pgrid, HJ_THREADS, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_hj_count<<<1, 1, 0, s>>>(p.status, nullptr, 1, total_tiles_direct, p.epoch, p.d_count);
    }
    return pd_launch_status(ctx);
  }
#endif
  for (uint32_t q = 0; q < parts; ++q) {
    p.part = q;
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
      k_hj_clear<<<clear_grid, 256, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_BUILD, s);
      k_hj_build<<<build_grid, 256, 0, s>>>(p);
    }
    {
      pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_PROBE, s);
      k_hj_probe<<<pgrid, HJ_THREADS, 0, s>>>(p);
    }
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_hj_count<<<1, 1, 0, s>>>(p.status, p.tilebase, parts, total_tiles_direct, p.epoch, p.d_count);
  }
  return pd_launch_status(ctx);
}

// ---------------------------------------------------------------------------
// Reference-shaped building blocks: pimdal_hash_kernel / pimdal_hj_probe use
// a caller-owned table of table_size slots preceded by one header word.
// ---------------------------------------------------------------------------
extern "C" size_t pimdal_hash_table_bytes(uint64_t table_size) { return 8 * (table_size + 4); }

extern "C" int pimdal_hash_kernel(pimdal_ctx_t *ctx, const pimdal_hash_arguments_t *a,
                                  pimdal_stream_t stream) {
  if (!ctx || !a || !a->table_ptr || ((uintptr_t)a->table_ptr & 31u)) return PIMDAL_ERR_ARG;
  if (a->size && !a->in_key) return PIMDAL_ERR_ARG;
  if (a->table_size < 16 || (a->table_size & (a->table_size - 1)) || a->size > a->table_size ||
      a->table_size > (1ull << 32))  // bucket_of's 32-bit arithmetic
    return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  JoinParams p{};
  p.table = (unsigned long long *)a->table_ptr + 4;
  p.side_count = (uint32_t *)a->table_ptr;
  p.dup_flag = (uint32_t *)a->table_ptr + 2;
  uint32_t bits = 0;
  while ((1ull << bits) < a->table_size) ++bits;
  p.bits = bits;
  p.bkey = (const uint32_t *)a->in_key;
  p.bpay = a->in_ptr;
  p.nb = a->size;
  p.d_error = ctx->d_error;
  PD_CHECK_CUDA(cudaMemsetAsync(a->table_ptr, 0, 32, s));
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_hj_clear<<<(unsigned)std::min<uint64_t>(pd_ceil_div(a->table_size, 512), ctx->sm_count * 8ull), 256, 0, s>>>(p);
  }
  if (a->size) {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_BUILD, s);
    k_hj_build<<<ctx->sm_count * 8, 256, 0, s>>>(p);
  }
  return pd_launch_status(ctx);
}

extern "C" int pimdal_hj_probe(pimdal_ctx_t *ctx, const pimdal_probe_arguments_t *a,
                               pimdal_merge_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result || !a->table_ptr || ((uintptr_t)a->table_ptr & 31u)) return PIMDAL_ERR_ARG;
  if (a->size && !a->in_key) return PIMDAL_ERR_ARG;
  if (a->out_capacity && (!a->out_inner || !a->out_outer)) return PIMDAL_ERR_ARG;
  if (a->table_size < 16 || (a->table_size & (a->table_size - 1)) || a->size >= (1ull << 32) ||
      a->table_size > (1ull << 32))
    return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  if (a->size == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d_result, 0, sizeof(uint64_t), s));
    return PIMDAL_OK;
  }
  const uint64_t tiles = pd_ceil_div(a->size, HJ_TILE);
  if (tiles > PD_STATUS_WORDS) return PIMDAL_ERR_ARG;
  int st;
  JoinParams p{};
  p.table = (unsigned long long *)a->table_ptr + 4;
  p.side_count = (uint32_t *)a->table_ptr;
  p.dup_flag = (uint32_t *)a->table_ptr + 2;
  uint32_t bits = 0;
  while ((1ull << bits) < a->table_size) ++bits;
  p.bits = bits;
  p.pkey = (const uint32_t *)a->in_key;
  p.prow = a->in_ptr;
  p.np = a->size;
  p.out_pay = a->out_inner;
  p.out_row = a->out_outer;
  p.cap = a->out_capacity;
  p.status = ctx->d_status;
  p.claim = ctx->d_counters + PD_COUNTER_PROBE;
  p.d_error = ctx->d_error;
  p.d_count = &d_result->t_count;
  p.epoch = pd_next_epoch(ctx, s, &st);
  if (st) return st;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_HJ_PROBE, s);
    k_hj_probe<<<probe_grid(ctx), HJ_THREADS, 0, s>>>(p);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_hj_count<<<1, 1, 0, s>>>(p.status, nullptr, 1, tiles, p.epoch, p.d_count);
  }
  return pd_launch_status(ctx);
}

// ---------------------------------------------------------------------------
// pimdal_part_kernel: stable radix partition by bits of hash0(key).
// ---------------------------------------------------------------------------
namespace {
__global__ void __launch_bounds__(256) k_part_hist(const uint32_t *key, uint64_t n, uint32_t sh,
                                                   uint32_t part_n, uint64_t *sizes) {
  extern __shared__ uint32_t s_h[];
  const bool smem = part_n <= 8192;
  if (smem)
    for (uint32_t i = threadIdx.x; i < part_n; i += blockDim.x) s_h[i] = 0;
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t b = (pd_hash0(key[i]) >> sh) & (part_n - 1);
    if (smem) atomicAdd(&s_h[b], 1u);
    else atomicAdd((unsigned long long *)&sizes[b + 1], 1ull);
  }
  __syncthreads();
  if (smem)
    for (uint32_t i = threadIdx.x; i < part_n; i += blockDim.x)
      if (s_h[i]) atomicAdd((unsigned long long *)&sizes[i + 1], (unsigned long long)s_h[i]);
}

// out[i] = i (row ids of a one-partition "partition").
__global__ void __launch_bounds__(256) k_iota(uint32_t *out, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = (uint32_t)i;
}

// In-place inclusive scan of sizes[1..part_n] (sizes[0] = 0) by one block.
__global__ void __launch_bounds__(1024) k_part_scan(uint64_t *sizes, uint32_t part_n) {
  __shared__ uint64_t s_carry;
  __shared__ uint64_t s_w[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < part_n; base += 1024) {
    uint32_t i = base + tid;
    uint64_t v = i < part_n ? sizes[i + 1] : 0, inc = v;
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
    if (i < part_n) sizes[i + 1] = s_carry + pre + inc;
    __syncthreads();
    if (tid == 0) s_carry += tot;
    __syncthreads();
  }
  if (tid == 0) sizes[0] = 0;
}
}  // namespace

extern "C" int pimdal_part_workspace_size(const pimdal_part_arguments_t *a, size_t *bytes) {
  if (!a || !bytes) return PIMDAL_ERR_ARG;
  uint32_t bits = 0;
  while ((1u << bits) < a->part_n) ++bits;
  pimdal_sort_arguments_t sa{};
  sa.nr_elements = a->size;
  sa.begin_bit = a->shift >= bits ? a->shift - bits : 0;
  sa.end_bit = a->shift ? a->shift : 32;
  if (bits == 0) sa.begin_bit = 0, sa.end_bit = 1;
  return pimdal_sort_workspace_size(&sa, bytes);
}

extern "C" int pimdal_part_kernel(pimdal_ctx_t *ctx, const pimdal_part_arguments_t *a,
                                  pimdal_stream_t stream) {
  if (!ctx || !a || !a->part_sizes) return PIMDAL_ERR_ARG;
  if (a->part_n == 0 || (a->part_n & (a->part_n - 1)) || a->part_n > 65536) return PIMDAL_ERR_ARG;
  if (a->layout != PIMDAL_LAYOUT_COLUMNS && a->layout != PIMDAL_LAYOUT_PAIRS) return PIMDAL_ERR_ARG;
  uint32_t bits = 0;
  while ((1u << bits) < a->part_n) ++bits;
  if (a->shift > 32 || a->shift < bits) return PIMDAL_ERR_ARG;
  if (a->size && (!a->in || !a->part_out)) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  PD_CHECK_CUDA(cudaMemsetAsync(a->part_sizes, 0, 8ull * (a->part_n + 1), s));
  if (a->size == 0) return PIMDAL_OK;
  if (a->layout == PIMDAL_LAYOUT_PAIRS) {
    // histogram of the pairs' keys: strided view of the key field
    return PIMDAL_ERR_NOT_SUPPORTED;
  }
  const uint32_t sh = a->shift - bits;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    size_t smem = a->part_n <= 8192 ? 4ull * a->part_n : 0;
    k_part_hist<<<ctx->sm_count * 4, 256, smem, s>>>((const uint32_t *)a->in, a->size, sh, a->part_n,
                                                    a->part_sizes);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_part_scan<<<1, 1024, 0, s>>>(a->part_sizes, a->part_n);
  }
  if (bits == 0) {
    PD_CHECK_CUDA(cudaMemcpyAsync(a->part_out, a->in, 4 * a->size, cudaMemcpyDeviceToDevice, s));
    if (a->part_out_ptr) {
      if (a->in_ptr) {
        PD_CHECK_CUDA(cudaMemcpyAsync(a->part_out_ptr, a->in_ptr, 4 * a->size,
                                      cudaMemcpyDeviceToDevice, s));
      } else {
        pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
        k_iota<<<ctx->sm_count * 4, 256, 0, s>>>(a->part_out_ptr, a->size);
      }
    }
    return pd_launch_status(ctx);
  }
  size_t need;
  int st = pimdal_part_workspace_size(a, &need);
  if (st) return st;
  void *ws = pd_workspace(ctx, need, s, &st);
  if (!ws) return st;
  pimdal_sort_arguments_t sa{};
  sa.nr_elements = a->size;
  sa.in = a->in;
  sa.in_ptr = a->in_ptr;
  sa.out = a->part_out;
  sa.out_ptr = a->part_out_ptr;
  sa.key_dtype = PIMDAL_U32;
  sa.layout = PIMDAL_LAYOUT_COLUMNS;
  sa.begin_bit = sh;
  sa.end_bit = a->shift;
  return pd_sort_ex(ctx, &sa, PD_KEY_HASH0, ws, s, nullptr);
}

// ---------------------------------------------------------------------------
// pimdal_select_join_aggregate: one query's filter -> join -> group-by in one
// pass over its fact range (the reference chains sel_kernel, merge_kernel,
// arithmetic_kernel and group_kernel with host steps between them, e.g.
// pimdal/main/tpc_h/query6/dpu/kernel_q6.c:112-156).  Each selected row
// probes the resident table exactly as pimdal_hj_probe does and adds its
// revenue to a shared-memory table indexed by the (small, dense) group key:
// one table per warp for key spaces up to 256 keys, one per CTA above.  The
// CTAs' tables are folded into a global table with one atomic per key, and a
// single CTA emits the non-empty groups in key order.  Integer sums do not
// depend on the order of the additions, so the result is bit-identical to
// the staged pipeline's.
// ---------------------------------------------------------------------------
namespace {

constexpr int SJA_THREADS = 256;
constexpr int SJA_WARPS = SJA_THREADS / 32;
constexpr uint32_t SJA_WARP_KEYS = 256;  // key spaces up to this get one table per warp
static_assert(PIMDAL_FUSED_MAX_KEYS * 12 <= 48 * 1024, "a CTA-wide table fits 48 KB");
static_assert(SJA_WARP_KEYS * SJA_WARPS <= PIMDAL_FUSED_MAX_KEYS, "per-warp tables fit too");

struct SjaParams {
  uint64_t n;
  const int32_t *date;
  int32_t lo, hi;
  const uint32_t *jkey;
  const unsigned long long *table;  // the slots, after the table's 32-byte header
  uint32_t bits;
  const uint32_t *side_count, *dup_flag;
  const uint8_t *flag;
  const int64_t *price;
  const int32_t *discount;
  uint32_t attr_mult, key_space;
  unsigned long long *g_sum, *g_cnt;  // key_space words each (workspace)
  uint32_t *d_error;
};

uint32_t sja_tables(uint32_t key_space) { return key_space <= SJA_WARP_KEYS ? SJA_WARPS : 1; }

// 8 CTAs per SM (32 registers): each row's loads and bucket walk form one
// dependent chain, and twice the warps of the former 4 CTAs per SM hide it
// (a 6e7-row request 1.03 -> 0.61 ms).
__global__ void __launch_bounds__(SJA_THREADS, 8) k_sja_aggregate(SjaParams p) {
  extern __shared__ __align__(16) unsigned long long sja_smem[];
  const uint32_t ks = p.key_space;
  const uint32_t tables = ks <= SJA_WARP_KEYS ? SJA_WARPS : 1;
  unsigned long long *s_sum = sja_smem;                                           // [tables][ks]
  unsigned int *s_cnt = reinterpret_cast<unsigned int *>(sja_smem + tables * ks);  // [tables][ks]
  const int tid = threadIdx.x, warp = tid >> 5;
  for (uint32_t i = tid; i < tables * ks; i += SJA_THREADS) {
    s_sum[i] = 0;
    s_cnt[i] = 0;
  }
  __syncthreads();
  unsigned long long *my_sum = s_sum + (warp % tables) * ks;
  unsigned int *my_cnt = s_cnt + (warp % tables) * ks;
  const uint32_t gmask = (uint32_t)(((1ull << p.bits) - 1) >> 2);
  const uint32_t side = *p.side_count;
  const bool no_dup = *p.dup_flag == 0;
  bool bad = false;
  const uint64_t stride = (uint64_t)gridDim.x * SJA_THREADS;
  for (uint64_t r = (uint64_t)blockIdx.x * SJA_THREADS + tid; r < p.n; r += stride) {
    const int32_t d = __ldcs(p.date + r);
    if (d < p.lo || d > p.hi) continue;
    const uint32_t key = __ldg(p.jkey + r);
    const uint32_t f = p.flag ? __ldg(p.flag + r) : 0u;
    const int64_t v = __ldg(p.price + r) * (int64_t)(100 - __ldg(p.discount + r));
    auto add = [&](uint32_t attr) {
      // the staged glue's key (k_revenue_keys): 32-bit, wrapping
      const uint32_t g = attr * p.attr_mult + f;
      if (g >= ks) {
        bad = true;
        return;
      }
      atomicAdd(&my_sum[g], (unsigned long long)v);
      atomicAdd(&my_cnt[g], 1u);
    };
    // the bucket walk of the probe: stop at a bucket with a free slot, or at
    // the first match when the build had no duplicate key
    const bool stop_first = no_dup && key != 0xFFFFFFFFu;
    uint32_t b = bucket_of(key, 0, p.bits);
    for (uint64_t step = 0; step <= gmask; ++step) {
      const ulonglong2 *q = reinterpret_cast<const ulonglong2 *>(p.table + 4 * (uint64_t)b);
      const ulonglong2 lo = q[0], hi = q[1];
      const unsigned long long e[4] = {lo.x, lo.y, hi.x, hi.y};
      bool empty = false, found = false;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (e[j] == HJ_EMPTY) {
          empty = true;
        } else if ((uint32_t)e[j] == key) {
          add((uint32_t)(e[j] >> 32));
          found = true;
        }
      }
      if (empty || (stop_first && found)) break;
      b = (b + 1) & gmask;
    }
    if (key == 0xFFFFFFFFu)  // build rows equal to the empty word, counted on the side
      for (uint32_t m = 0; m < side; ++m) add(0xFFFFFFFFu);
  }
  if (bad) atomicOr(p.d_error, PD_DEVERR_ARG);
  __syncthreads();
  for (uint32_t k = tid; k < ks; k += SJA_THREADS) {
    unsigned long long sum = 0, cnt = 0;
    for (uint32_t t = 0; t < tables; ++t) {
      sum += s_sum[t * ks + k];
      cnt += s_cnt[t * ks + k];
    }
    if (cnt) {
      atomicAdd(&p.g_sum[k], sum);
      atomicAdd(&p.g_cnt[k], cnt);
    }
  }
}

// One CTA: the non-empty groups in key order.
__global__ void __launch_bounds__(1024) k_sja_emit(const unsigned long long *g_sum,
                                                   const unsigned long long *g_cnt, uint32_t ks,
                                                   uint32_t *out_key, int64_t *out_sum,
                                                   int64_t *out_count, uint64_t cap,
                                                   uint64_t *t_count, uint32_t *d_error) {
  __shared__ uint32_t s_warp[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t base = 0;
  bool overflow = false;
  for (uint32_t k0 = 0; k0 < ks; k0 += 1024) {
    const uint32_t k = k0 + tid;
    const bool has = k < ks && g_cnt[k] != 0;
    const unsigned m = __ballot_sync(0xffffffffu, has);
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    uint32_t pre = 0, total = 0;
    for (int w = 0; w < 32; ++w) {
      const uint32_t x = s_warp[w];
      if (w < warp) pre += x;
      total += x;
    }
    if (has) {
      const uint64_t pos = base + pre + __popc(m & ((1u << lane) - 1u));
      if (pos < cap) {
        out_key[pos] = k;
        out_sum[pos] = (int64_t)g_sum[k];
        out_count[pos] = (int64_t)g_cnt[k];
      } else {
        overflow = true;
      }
    }
    base += total;
    __syncthreads();  // s_warp is rewritten by the next round
  }
  if (overflow) atomicOr(d_error, PD_DEVERR_CAPACITY);
  if (tid == 0) *t_count = base;
}

}  // namespace

extern "C" int pimdal_select_join_aggregate_workspace_size(
    const pimdal_select_join_aggregate_arguments_t *a, size_t *bytes) {
  if (!a || !bytes || a->key_space == 0 || a->key_space > PIMDAL_FUSED_MAX_KEYS) return PIMDAL_ERR_ARG;
  *bytes = 16ull * a->key_space;
  return PIMDAL_OK;
}

extern "C" int pimdal_select_join_aggregate(pimdal_ctx_t *ctx,
                                            const pimdal_select_join_aggregate_arguments_t *a,
                                            pimdal_aggr_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result || !a->table_ptr || ((uintptr_t)a->table_ptr & 31u)) return PIMDAL_ERR_ARG;
  if (a->table_size < 16 || (a->table_size & (a->table_size - 1)) || a->table_size > (1ull << 32))
    return PIMDAL_ERR_ARG;
  if (a->key_space == 0 || a->key_space > PIMDAL_FUSED_MAX_KEYS || a->size >= (1ull << 32))
    return PIMDAL_ERR_ARG;
  if (a->size && (!a->date || !a->jkey || !a->price || !a->discount)) return PIMDAL_ERR_ARG;
  if (a->out_capacity && (!a->out_key || !a->out_sum || !a->out_count)) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  const size_t ws_bytes = 16ull * a->key_space;
  int st;
  char *ws = (char *)pd_workspace(ctx, ws_bytes, s, &st);
  if (!ws) return st;
  PD_CHECK_CUDA(cudaMemsetAsync(ws, 0, ws_bytes, s));
  SjaParams p{};
  p.n = a->size;
  p.date = a->date;
  p.lo = a->date_lo;
  p.hi = a->date_hi;
  p.jkey = a->jkey;
  p.table = (const unsigned long long *)a->table_ptr + 4;
  p.side_count = (const uint32_t *)a->table_ptr;
  p.dup_flag = (const uint32_t *)a->table_ptr + 2;
  uint32_t bits = 0;
  while ((1ull << bits) < a->table_size) ++bits;
  p.bits = bits;
  p.flag = a->flag;
  p.price = a->price;
  p.discount = a->discount;
  p.attr_mult = a->attr_mult;
  p.key_space = a->key_space;
  p.g_sum = (unsigned long long *)ws;
  p.g_cnt = (unsigned long long *)ws + a->key_space;
  p.d_error = ctx->d_error;
  if (a->size) {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_FUSED, s);
    const size_t smem = 12ull * sja_tables(a->key_space) * a->key_space;
    const unsigned g = (unsigned)std::min<uint64_t>(pd_ceil_div(a->size, SJA_THREADS), ctx->sm_count * 8ull);
    k_sja_aggregate<<<g, SJA_THREADS, smem, s>>>(p);
  }
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_sja_emit<<<1, 1024, 0, s>>>(p.g_sum, p.g_cnt, a->key_space, a->out_key, a->out_sum,
                                  a->out_count, a->out_capacity, &d_result->t_count, ctx->d_error);
  }
  return pd_launch_status(ctx);
}

extern "C" int pimdal_hash_join_autotune(pimdal_ctx_t *ctx, const pimdal_hash_join_arguments_t *a,
                                         pimdal_merge_results_t *d_result, pimdal_tuning_t *best,
                                         int *cached, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result || !best) return PIMDAL_ERR_ARG;
  if (cached) *cached = 0;
  const auto key = hj_shape(a);
  const auto it = ctx->op_tune.find(key);
  if (it != ctx->op_tune.end()) {
    *best = it->second;
    best->candidates = 0;
    if (cached) *cached = 1;
    return PIMDAL_OK;
  }
  const auto cands = hj_candidates(a);
  if (cands.empty()) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  float best_ms = -1.f;
  size_t best_i = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    auto run = [&] { return pimdal_hash_join(ctx, &cands[i], d_result, stream); };
    if (pd_time_call(ctx, s, run) < 0.f) continue;  // warm-up (workspace, caches)
    const float ms = pd_time_call(ctx, s, run);
    if (ms >= 0.f && (best_ms < 0.f || ms < best_ms)) {
      best_ms = ms;
      best_i = i;
    }
  }
  if (best_ms < 0.f) return PIMDAL_ERR_CUDA;
  pimdal_tuning_t t{};
  t.partition_bits = cands[best_i].partition_bits;
  t.load_factor_pct = cands[best_i].load_factor_pct;
  t.ms = best_ms;
  t.candidates = (uint32_t)cands.size();
  ctx->op_tune[key] = t;
  *best = t;
  // the outputs are the chosen candidate's
  return pimdal_hash_join(ctx, &cands[best_i], d_result, stream);
}
