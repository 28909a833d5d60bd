// K-SEL: single-pass stable selection (pimdal_sel_kernel).
//
// Reference behaviour: sel_kernel (pimdal/select/sel.c:81-150) keeps, in input
// order, the key_ptr pairs for which pred() holds and reports t_count; its
// caller kernel_select.c:31-42 first turns the int32 column into (value,
// row id) pairs (create_ptr) and afterwards strips the row ids (out_val).
// The CPU operator reference/db_operators/select.cpp:39-75 counts per block,
// prefix-sums the counts and scatters.
//
// B200 design: one pass over HBM.  A CTA owns a 4096-element tile; each thread
// loads four 128-bit vectors (warp-striped, fully coalesced), evaluates the
// predicate, and the tile's rank of every selected element comes from a
// byte-packed warp scan plus a 32-entry (chunk, warp) scan.  The tile's global
// output offset comes from a decoupled look-back over epoch-tagged status
// words (no second pass over the input, no separate memset).  Selected
// elements are compacted in shared memory and written out with coalesced
// stores.  The create_ptr / out_val glue is fused: row ids are generated
// (ptr_base + index) unless a row-id column is given.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace {

constexpr int SEL_THREADS = 256;
constexpr int SEL_WARPS = SEL_THREADS / 32;
constexpr int SEL_VEC = 4;                          // elements per 128-bit column load
constexpr int SEL_CHUNKS = 4;                       // vector loads per thread
constexpr int SEL_ITEMS = SEL_VEC * SEL_CHUNKS;     // 16 elements per thread
constexpr int SEL_CHUNK_ELEMS = SEL_THREADS * SEL_VEC;  // 1024
constexpr int SEL_TILE = SEL_THREADS * SEL_ITEMS;   // 4096

struct SelParams {
  const void *in;
  const uint32_t *in_ptr;
  uint64_t ptr_base;
  void *out;
  uint32_t *out_ptr;
  uint64_t n;
  uint32_t lo32, range32;  // selected: (key - lo32) mod 2^32 <= range32, xor invert
  uint32_t invert;
  uint32_t vec_ok;  // input pointers 16-byte aligned
  uint64_t *status;
  uint32_t epoch;
  uint32_t *d_error;
  uint64_t *d_count;
};

// One subtract and one unsigned compare: for lo <= hi in the key's own order,
// lo <= v <= hi  <=>  (v - lo) mod 2^32 <= (hi - lo), for signed and unsigned
// 32-bit keys alike (the host clamps the interval to the key type's range).
template <bool SIGNED>
__device__ __forceinline__ bool sel_pred(uint32_t key, const SelParams &p) {
  return ((key - p.lo32) <= p.range32) != (p.invert != 0);
}

// LAYOUT: PIMDAL_LAYOUT_COLUMNS or PIMDAL_LAYOUT_PAIRS; HAS_PTR: a row-id
// column is given (COLUMNS only; PAIRS always carry their row id).
template <int LAYOUT, bool SIGNED, bool HAS_PTR>
__global__ void __launch_bounds__(SEL_THREADS) k_select(SelParams p) {
  __shared__ uint32_t s_key[SEL_TILE];
  __shared__ uint32_t s_ptr[SEL_TILE];
  __shared__ uint32_t s_off[SEL_CHUNKS * SEL_WARPS];
  __shared__ uint64_t s_prefix;
  __shared__ uint32_t s_total;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t tile = blockIdx.x;
  const uint64_t tile_base = tile * (uint64_t)SEL_TILE;
  const bool full = tile_base + SEL_TILE <= p.n;

  uint32_t key[SEL_ITEMS], ptr[SEL_ITEMS];
  uint32_t sel = 0;  // bit c*4+j

#pragma unroll
  for (int c = 0; c < SEL_CHUNKS; ++c) {
    const uint64_t e0 = tile_base + (uint64_t)c * SEL_CHUNK_ELEMS + (uint64_t)tid * SEL_VEC;
    if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
      const uint4 *src = reinterpret_cast<const uint4 *>(
          reinterpret_cast<const pimdal_key_ptr32_t *>(p.in) + e0);
      if (full && p.vec_ok) {
        uint4 a = __ldcs(src), b = __ldcs(src + 1);
        key[c * 4 + 0] = a.x; ptr[c * 4 + 0] = a.y;
        key[c * 4 + 1] = a.z; ptr[c * 4 + 1] = a.w;
        key[c * 4 + 2] = b.x; ptr[c * 4 + 2] = b.y;
        key[c * 4 + 3] = b.z; ptr[c * 4 + 3] = b.w;
      } else {
        const pimdal_key_ptr32_t *pp = reinterpret_cast<const pimdal_key_ptr32_t *>(p.in);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (e0 + j < p.n) { key[c * 4 + j] = pp[e0 + j].key; ptr[c * 4 + j] = pp[e0 + j].ptr; }
          else { key[c * 4 + j] = 0; ptr[c * 4 + j] = 0; }
        }
      }
    } else {
      const uint32_t *kin = reinterpret_cast<const uint32_t *>(p.in);
      if (full && p.vec_ok) {
        uint4 a = __ldcs(reinterpret_cast<const uint4 *>(kin + e0));
        key[c * 4 + 0] = a.x; key[c * 4 + 1] = a.y; key[c * 4 + 2] = a.z; key[c * 4 + 3] = a.w;
        if (HAS_PTR) {
          uint4 b = __ldcs(reinterpret_cast<const uint4 *>(p.in_ptr + e0));
          ptr[c * 4 + 0] = b.x; ptr[c * 4 + 1] = b.y; ptr[c * 4 + 2] = b.z; ptr[c * 4 + 3] = b.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          bool ok = e0 + j < p.n;
          key[c * 4 + j] = ok ? kin[e0 + j] : 0u;
          if (HAS_PTR) ptr[c * 4 + j] = ok ? p.in_ptr[e0 + j] : 0u;
        }
      }
      if (!HAS_PTR) {
#pragma unroll
        for (int j = 0; j < 4; ++j) ptr[c * 4 + j] = (uint32_t)(p.ptr_base + e0 + j);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      bool s = (e0 + j < p.n) && sel_pred<SIGNED>(key[c * 4 + j], p);
      sel |= (uint32_t)s << (c * 4 + j);
    }
  }

  // Byte-packed per-chunk counts (each <= 4, warp sums <= 128).
  uint32_t packed = 0;
#pragma unroll
  for (int c = 0; c < SEL_CHUNKS; ++c) packed |= (uint32_t)__popc((sel >> (c * 4)) & 0xFu) << (8 * c);
  uint32_t inc = packed;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  const uint32_t excl = inc - packed;
  if (lane == 31) {
#pragma unroll
    for (int c = 0; c < SEL_CHUNKS; ++c) s_off[c * SEL_WARPS + warp] = (inc >> (8 * c)) & 0xFFu;
  }
  __syncthreads();

  if (warp == 0) {
    // (chunk, warp) counts in tile order: chunk-major, then warp.
    uint32_t x = s_off[lane];
    uint32_t xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += t;
    }
    s_off[lane] = xi - x;
    const uint32_t total = __shfl_sync(0xffffffffu, xi, 31);
    uint64_t prefix = 0;
    if (tile == 0) {
      if (lane == 0) pd_store_release_u64(p.status, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, total));
    } else {
      if (lane == 0)
        pd_store_release_u64(p.status + tile, pd_pack_status(p.epoch, PD_FLAG_AGGREGATE, total));
      prefix = pd_lookback_warp(p.status, (int64_t)tile, p.epoch, p.d_error);
      if (lane == 0)
        pd_store_release_u64(p.status + tile,
                             pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, prefix + total));
    }
    if (lane == 0) {
      s_prefix = prefix;
      s_total = total;
      if (tile == gridDim.x - 1) *p.d_count = prefix + total;
    }
  }
  __syncthreads();

  // Compact the tile's selected elements into shared memory (stable order).
#pragma unroll
  for (int c = 0; c < SEL_CHUNKS; ++c) {
    uint32_t r = s_off[c * SEL_WARPS + warp] + ((excl >> (8 * c)) & 0xFFu);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if ((sel >> (c * 4 + j)) & 1u) {
        s_key[r] = key[c * 4 + j];
        s_ptr[r] = ptr[c * 4 + j];
        ++r;
      }
    }
  }
  __syncthreads();

  const uint32_t total = s_total;
  const uint64_t prefix = s_prefix;
  if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
    uint2 *out = reinterpret_cast<uint2 *>(p.out) + prefix;
    for (uint32_t i = tid; i < total; i += SEL_THREADS) out[i] = make_uint2(s_key[i], s_ptr[i]);
  } else {
    uint32_t *out = reinterpret_cast<uint32_t *>(p.out) + prefix;
    for (uint32_t i = tid; i < total; i += SEL_THREADS) out[i] = s_key[i];
    if (p.out_ptr) {
      uint32_t *op = p.out_ptr + prefix;
      for (uint32_t i = tid; i < total; i += SEL_THREADS) op[i] = s_ptr[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Large inputs: persistent CTAs, one per SM, each claiming ~450 KB chunks.
//   A. stream the chunk through a TMA bulk-copy ring (evict_last) and count;
//   B. publish the chunk count and resolve its output offset with one
//      block-wide decoupled look-back (1024 predecessors per round);
//   C. re-read the chunk (L2 hits) tile by tile, rank and write the rows.
// DRAM sees one read of the input and one write of the output; the look-back
// happens once per chunk instead of once per 16 KB tile.
// ---------------------------------------------------------------------------
constexpr int SL_THREADS = 1024;
constexpr int SL_WARPS = SL_THREADS / 32;
constexpr int SL_STAGE_BYTES = 32768;
constexpr int SL_STAGES = 4;
constexpr int SL_TILE = SL_THREADS * 8;  // phase-C tile: 8 elements per thread
constexpr uint64_t SL_CHUNK_MAX = 1u << 17;

struct SlParams {
  SelParams s;
  uint64_t chunk_elems, nchunks;
  uint32_t *claim;  // [0] next chunk, [1] CTAs done claiming (self-resetting)
};

__device__ __forceinline__ uint32_t block_reduce_sum_1024(uint32_t v, uint32_t *s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  uint32_t t = s_red[lane];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  __syncthreads();
  return t;
}

__device__ __forceinline__ bool sl_timed_out(const uint32_t *d_error) {
  return (*(const volatile uint32_t *)d_error & PD_DEVERR_TIMEOUT) != 0;
}

template <int LAYOUT, bool SIGNED, bool HAS_PTR>
__global__ void __launch_bounds__(SL_THREADS, 1) k_select_chunked(SlParams q) {
  extern __shared__ __align__(128) unsigned char s_ring[];
  __shared__ uint64_t s_bar[SL_STAGES];
  __shared__ uint32_t s_red[32];
  __shared__ uint32_t s_flags[2 * SL_WARPS];
  __shared__ uint64_t s_sum[SL_WARPS + 1];
  __shared__ uint32_t s_off[2 * SL_WARPS];
  __shared__ int s_state;
  __shared__ uint64_t s_chunk, s_prefix;

  const SelParams &p = q.s;
  constexpr int EB = (LAYOUT == PIMDAL_LAYOUT_PAIRS) ? 8 : 4;  // bytes per element
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int i = 0; i < SL_STAGES; ++i) pd_mbar_init(&s_bar[i], 1);
    pd_fence_mbar_init();
  }
  __syncthreads();
  const uint64_t pol = pd_policy_evict_last();
  uint32_t consumed = 0, issued = 0;  // ring stages (thread 0 issues)

  while (true) {
    if (tid == 0) {
      uint64_t c = atomicAdd(q.claim, 1u);
      if (c >= q.nchunks) {
        // Last claimer of the launch resets the counters for the next launch.
        if (atomicAdd(q.claim + 1, 1u) == gridDim.x - 1) {
          q.claim[0] = 0;
          q.claim[1] = 0;
        }
      }
      s_chunk = c;
    }
    __syncthreads();
    const uint64_t chunk = s_chunk;
    if (chunk >= q.nchunks) break;
    const uint64_t c0 = chunk * q.chunk_elems;
    const uint64_t c1 = min(p.n, c0 + q.chunk_elems);
    const char *src = reinterpret_cast<const char *>(p.in) + c0 * EB;
    const uint64_t bytes = (c1 - c0) * EB;
    const uint64_t bulk_bytes = bytes & ~(uint64_t)15;
    const uint32_t nst = (uint32_t)pd_ceil_div(bulk_bytes, SL_STAGE_BYTES);

    // ---- A: count through the bulk-copy ring ------------------------------
    // After a wait anywhere in the launch gave up, no further copy is issued.
    if (tid == 0 && !sl_timed_out(p.d_error)) {
      for (uint32_t j = 0; j < nst && j < (uint32_t)SL_STAGES; ++j) {
        uint32_t slot = issued % SL_STAGES;
        uint32_t b = (uint32_t)min((uint64_t)SL_STAGE_BYTES, bulk_bytes - (uint64_t)j * SL_STAGE_BYTES);
        pd_mbar_expect_tx(&s_bar[slot], b);
        pd_bulk_g2s(s_ring + slot * SL_STAGE_BYTES, src + (uint64_t)j * SL_STAGE_BYTES, b,
                    &s_bar[slot], pol);
        ++issued;
      }
    }
    uint32_t cnt = 0;
    for (uint32_t j = 0; j < nst; ++j) {
      const uint32_t slot = consumed % SL_STAGES, parity = (consumed / SL_STAGES) & 1u;
      const uint32_t b = (uint32_t)min((uint64_t)SL_STAGE_BYTES, bulk_bytes - (uint64_t)j * SL_STAGE_BYTES);
      uint32_t spins = 0;
      const uint64_t t0 = pd_globaltimer_ns();
      while (!pd_mbar_try_wait(&s_bar[slot], parity)) {
        if (pd_wait_expired(p.d_error, t0, ++spins)) break;
      }
      const uint4 *v = reinterpret_cast<const uint4 *>(s_ring + slot * SL_STAGE_BYTES);
      for (uint32_t i = tid; i < b / 16; i += SL_THREADS) {
        uint4 x = v[i];
        if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
          cnt += sel_pred<SIGNED>(x.x, p) + sel_pred<SIGNED>(x.z, p);
        } else {
          cnt += sel_pred<SIGNED>(x.x, p) + sel_pred<SIGNED>(x.y, p) + sel_pred<SIGNED>(x.z, p) +
                 sel_pred<SIGNED>(x.w, p);
        }
      }
      __syncthreads();
      if (tid == 0 && j + SL_STAGES < nst && !sl_timed_out(p.d_error)) {
        const uint32_t jn = j + SL_STAGES;
        const uint32_t bn = (uint32_t)min((uint64_t)SL_STAGE_BYTES, bulk_bytes - (uint64_t)jn * SL_STAGE_BYTES);
        pd_fence_proxy_async_smem();
        pd_mbar_expect_tx(&s_bar[slot], bn);
        pd_bulk_g2s(s_ring + slot * SL_STAGE_BYTES, src + (uint64_t)jn * SL_STAGE_BYTES, bn,
                    &s_bar[slot], pol);
        ++issued;
      }
      ++consumed;
    }
    // tail elements not covered by 16-byte bulk copies
    for (uint64_t e = c0 + bulk_bytes / EB + tid; e < c1; e += SL_THREADS) {
      uint32_t k = (LAYOUT == PIMDAL_LAYOUT_PAIRS)
                       ? reinterpret_cast<const pimdal_key_ptr32_t *>(p.in)[e].key
                       : reinterpret_cast<const uint32_t *>(p.in)[e];
      cnt += sel_pred<SIGNED>(k, p);
    }
    const uint32_t total = block_reduce_sum_1024(cnt, s_red);

    // ---- B: chunk offset ---------------------------------------------------
    if (chunk == 0) {
      if (tid == 0) {
        pd_store_relaxed_u64(p.status, pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, total));
        s_prefix = 0;
      }
    } else {
      if (tid == 0)
        pd_store_relaxed_u64(p.status + chunk, pd_pack_status(p.epoch, PD_FLAG_AGGREGATE, total));
      uint64_t pre = pd_block_lookback<SL_THREADS>(p.status, (int64_t)chunk, p.epoch, p.d_error, s_flags, s_sum,
                                    &s_state);
      if (tid == 0) {
        pd_store_relaxed_u64(p.status + chunk,
                             pd_pack_status(p.epoch, PD_FLAG_INCLUSIVE, pre + total));
        s_prefix = pre;
      }
    }
    __syncthreads();
    uint64_t out_base = s_prefix;
    if (chunk == q.nchunks - 1 && tid == 0) *p.d_count = out_base + total;

    // ---- C: rank and write, tile by tile (input re-read from L2) -----------
    for (uint64_t t0e = c0; t0e < c1; t0e += SL_TILE) {
      uint32_t key[8], ptr[8];
      uint32_t sel = 0;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const uint64_t e0 = t0e + (uint64_t)c * (SL_THREADS * 4) + (uint64_t)tid * 4;
        if (e0 + 4 <= c1) {
          if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
            const uint4 *s4 = reinterpret_cast<const uint4 *>(
                reinterpret_cast<const pimdal_key_ptr32_t *>(p.in) + e0);
            uint4 a = __ldcs(s4), b2 = __ldcs(s4 + 1);
            key[c * 4 + 0] = a.x; ptr[c * 4 + 0] = a.y; key[c * 4 + 1] = a.z; ptr[c * 4 + 1] = a.w;
            key[c * 4 + 2] = b2.x; ptr[c * 4 + 2] = b2.y; key[c * 4 + 3] = b2.z; ptr[c * 4 + 3] = b2.w;
          } else {
            uint4 a = __ldcs(reinterpret_cast<const uint4 *>(reinterpret_cast<const uint32_t *>(p.in) + e0));
            key[c * 4 + 0] = a.x; key[c * 4 + 1] = a.y; key[c * 4 + 2] = a.z; key[c * 4 + 3] = a.w;
            if (HAS_PTR) {
              uint4 b2 = __ldcs(reinterpret_cast<const uint4 *>(p.in_ptr + e0));
              ptr[c * 4 + 0] = b2.x; ptr[c * 4 + 1] = b2.y; ptr[c * 4 + 2] = b2.z; ptr[c * 4 + 3] = b2.w;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const bool ok = e0 + j < c1;
            if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
              const pimdal_key_ptr32_t *pp = reinterpret_cast<const pimdal_key_ptr32_t *>(p.in);
              key[c * 4 + j] = ok ? pp[e0 + j].key : 0u;
              ptr[c * 4 + j] = ok ? pp[e0 + j].ptr : 0u;
            } else {
              key[c * 4 + j] = ok ? reinterpret_cast<const uint32_t *>(p.in)[e0 + j] : 0u;
              if (HAS_PTR) ptr[c * 4 + j] = ok ? p.in_ptr[e0 + j] : 0u;
            }
          }
        }
        if (LAYOUT != PIMDAL_LAYOUT_PAIRS && !HAS_PTR) {
#pragma unroll
          for (int j = 0; j < 4; ++j) ptr[c * 4 + j] = (uint32_t)(p.ptr_base + e0 + j);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          bool s = (e0 + j < c1) && sel_pred<SIGNED>(key[c * 4 + j], p);
          sel |= (uint32_t)s << (c * 4 + j);
        }
      }
      // byte-packed counts of the 2 sub-chunks; warp scan; (sub-chunk, warp) scan
      uint32_t packed = (uint32_t)__popc(sel & 0xFu) | ((uint32_t)__popc((sel >> 4) & 0xFu) << 8);
      uint32_t inc = packed;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      const uint32_t excl = inc - packed;
      if (lane == 31) {
        s_off[warp] = inc & 0xFFu;
        s_off[SL_WARPS + warp] = (inc >> 8) & 0xFFu;
      }
      __syncthreads();
      if (warp == 0) {
        // entries in tile order: sub-chunk 0 warps 0..31, then sub-chunk 1
        uint32_t a = s_off[2 * lane], b2 = s_off[2 * lane + 1];
        uint32_t x = a + b2, xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, xi, o);
          if (lane >= o) xi += t;
        }
        uint32_t ex = xi - x;
        s_off[2 * lane] = ex;
        s_off[2 * lane + 1] = ex + a;
        if (lane == 31) s_red[0] = xi;
      }
      __syncthreads();
      const uint32_t tile_total = s_red[0];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint64_t r = out_base + s_off[c * SL_WARPS + warp] + ((excl >> (8 * c)) & 0xFFu);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if ((sel >> (c * 4 + j)) & 1u) {
            if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
              reinterpret_cast<uint2 *>(p.out)[r] = make_uint2(key[c * 4 + j], ptr[c * 4 + j]);
            } else {
              reinterpret_cast<uint32_t *>(p.out)[r] = key[c * 4 + j];
              if (p.out_ptr) p.out_ptr[r] = ptr[c * 4 + j];
            }
            ++r;
          }
        }
      }
      out_base += tile_total;
      __syncthreads();
    }
  }
  // Before the CTA exits, every bulk copy it issued must have landed: when a
  // wait above gave up, a copy may still be writing into this CTA's shared
  // memory.  Thread 0 (the only issuer) waits, bounded, for the last phase
  // issued on each ring slot; on the normal path these phases are complete
  // and each wait returns at once.
  if (tid == 0) {
    for (uint32_t slot = 0; slot < (uint32_t)SL_STAGES && slot < issued; ++slot) {
      const uint32_t uses = (issued - slot + SL_STAGES - 1) / SL_STAGES;  // issues on this slot
      const uint32_t parity = (uses - 1) & 1u;
      uint32_t spins = 0;
      const uint64_t t0 = pd_globaltimer_ns();
      while (!pd_mbar_try_wait(&s_bar[slot], parity)) {
        if (pd_wait_expired(p.d_error, t0, ++spins)) break;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Shapes and loads of the cooperative selection kernel below.
// ---------------------------------------------------------------------------
constexpr int SC_THREADS = 512;
constexpr int SC_WARPS = SC_THREADS / 32;
constexpr int SC_TILE_BYTES = 64 * 1024;

template <int LAYOUT, int SUB_ = SC_TILE_BYTES / 16 / SC_THREADS>
struct ScShape {
  static constexpr int EB = LAYOUT == PIMDAL_LAYOUT_PAIRS ? 8 : 4;  // bytes per element
  static constexpr int EPV = 16 / EB;                                // elements per 16-byte load
  static constexpr int SUB = SUB_;                                   // loads per thread
  static constexpr int EPT = SUB * EPV;                              // elements per thread
  static constexpr int TE = SC_THREADS * EPT;                        // elements per tile
};

// Striped (coalesced) loads: load k of thread t covers tile elements
// (k * SC_THREADS + t) * EPV + j.  key[k * EPV + j]; *valid has a bit per
// element inside the input.
template <int LAYOUT, int SUB_ = SC_TILE_BYTES / 16 / SC_THREADS>
__device__ __forceinline__ void sc_load_keys(const SelParams &p, uint64_t tile, uint32_t *key,
                                             uint32_t *valid) {
  using S = ScShape<LAYOUT, SUB_>;
  const uint64_t t0 = tile * S::TE;
  const uint4 *src = reinterpret_cast<const uint4 *>(reinterpret_cast<const char *>(p.in) + t0 * S::EB);
  *valid = 0;
#pragma unroll
  for (int k = 0; k < S::SUB; ++k) {
    const uint64_t e = t0 + ((uint64_t)k * SC_THREADS + threadIdx.x) * S::EPV;
    if (e + S::EPV <= p.n) {
      const uint4 v = src[k * SC_THREADS + threadIdx.x];
      if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
        key[2 * k] = v.x;
        key[2 * k + 1] = v.z;
      } else {
        key[4 * k] = v.x; key[4 * k + 1] = v.y; key[4 * k + 2] = v.z; key[4 * k + 3] = v.w;
      }
      *valid |= ((1u << S::EPV) - 1u) << (k * S::EPV);
    } else {
#pragma unroll
      for (int j = 0; j < S::EPV; ++j) {
        const bool ok = e + j < p.n;
        *valid |= (uint32_t)ok << (k * S::EPV + j);
        key[k * S::EPV + j] = !ok ? 0u
                              : LAYOUT == PIMDAL_LAYOUT_PAIRS
                                  ? reinterpret_cast<const pimdal_key_ptr32_t *>(p.in)[e + j].key
                                  : reinterpret_cast<const uint32_t *>(p.in)[e + j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Large aligned inputs (pimdal_sel_kernel): one cooperative launch (all CTAs
// co-resident, no look-back): each CTA counts a contiguous run of 64 KB tiles, a grid barrier (bounded wait) publishes the
// per-CTA counts, each CTA adds up the counts before it, then re-reads its
// tiles (L2 hits while the input fits in L2) and writes the selected
// elements in order with a running offset.
// ---------------------------------------------------------------------------
constexpr int CO_SUB = 8;  // 16-byte loads per thread per tile (tile = 64 KB)

// Grid-wide barrier for a cooperative launch: bar[0] arrivals (reset by the
// last arrival), bar[1] generation.  A wait that exceeds the bounded-wait
// limit sets PD_DEVERR_TIMEOUT; returns false (in every thread) when the
// device error word has that bit, so the caller writes nothing.
__device__ __forceinline__ bool co_grid_barrier(uint32_t *bar, uint32_t *d_error) {
  __shared__ bool s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t gen = pd_load_acquire_u32(bar + 1);
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      bar[0] = 0;
      __threadfence();
      pd_store_release_u32(bar + 1, gen + 1);
    } else {
      uint32_t spins = 0;
      const uint64_t t0 = pd_globaltimer_ns();
      while (pd_load_acquire_u32(bar + 1) == gen) {
        if (pd_wait_expired(d_error, t0, ++spins)) break;
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = !(*(volatile uint32_t *)d_error & PD_DEVERR_TIMEOUT);
  }
  __syncthreads();
  return s_ok;
}

template <int LAYOUT, bool SIGNED, bool HAS_PTR>
__global__ void __launch_bounds__(SC_THREADS) k_select_coop(SelParams p, uint64_t *counts,
                                                            uint32_t *bar, uint64_t tiles_per_cta) {
  using S = ScShape<LAYOUT, CO_SUB>;
  constexpr int E = S::SUB * SC_WARPS;  // (load, warp) entries of a tile, load major
  __shared__ uint32_t s_off[E];
  __shared__ uint32_t s_red[SC_WARPS];
  __shared__ uint64_t s_base;
  __shared__ uint32_t s_total;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t ntiles = pd_ceil_div(p.n, (uint64_t)S::TE);
  const uint64_t t0 = min(ntiles, (uint64_t)blockIdx.x * tiles_per_cta);
  const uint64_t t1 = min(ntiles, t0 + tiles_per_cta);

  // 1. count this CTA's tiles
  uint32_t c = 0;
  for (uint64_t t = t0; t < t1; ++t) {
    uint32_t key[S::EPT], valid, m = 0;
    sc_load_keys<LAYOUT, CO_SUB>(p, t, key, &valid);
#pragma unroll
    for (int j = 0; j < S::EPT; ++j) m |= (uint32_t)sel_pred<SIGNED>(key[j], p) << j;
    c += __popc(m & valid);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) s_red[warp] = c;
  __syncthreads();
  if (tid == 0) {
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < SC_WARPS; ++w) t += s_red[w];
    counts[blockIdx.x] = t;
  }
  // 2. every CTA's count is published
  if (!co_grid_barrier(bar, p.d_error)) return;
  // 3. this CTA's first output row: the counts of the CTAs before it
  {
    uint64_t pre = 0, all = 0;
    for (uint32_t i = tid; i < gridDim.x; i += SC_THREADS) {
      const uint64_t v = __ldcg(counts + i);
      all += v;
      if (i < blockIdx.x) pre += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      pre += __shfl_xor_sync(0xffffffffu, pre, o);
      all += __shfl_xor_sync(0xffffffffu, all, o);
    }
    __shared__ uint64_t s_pre[SC_WARPS], s_all[SC_WARPS];
    if (lane == 0) {
      s_pre[warp] = pre;
      s_all[warp] = all;
    }
    __syncthreads();
    if (tid == 0) {
      uint64_t a = 0, b = 0;
      for (int w = 0; w < SC_WARPS; ++w) {
        a += s_pre[w];
        b += s_all[w];
      }
      s_base = a;
      if (blockIdx.x == 0) *p.d_count = b;
    }
    __syncthreads();
  }
  // 4. re-read the tiles, rank and write
  uint64_t base = s_base;
  for (uint64_t t = t0; t < t1; ++t) {
    uint32_t key[S::EPT], valid, m = 0;
    sc_load_keys<LAYOUT, CO_SUB>(p, t, key, &valid);
#pragma unroll
    for (int j = 0; j < S::EPT; ++j) m |= (uint32_t)sel_pred<SIGNED>(key[j], p) << j;
    m &= valid;
    static_assert(S::SUB <= 8, "one byte per load in 64 bits");
    uint64_t packed = 0;  // per load: count (<= 4) in one byte; per warp < 256
#pragma unroll
    for (int k = 0; k < S::SUB; ++k)
      packed |= (uint64_t)__popc((m >> (k * S::EPV)) & ((1u << S::EPV) - 1u)) << (8 * k);
    uint64_t inc = packed;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t x = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += x;
    }
    const uint64_t excl = inc - packed;
    if (lane == 31) {
#pragma unroll
      for (int k = 0; k < S::SUB; ++k) s_off[k * SC_WARPS + warp] = (uint32_t)(inc >> (8 * k)) & 0xFFu;
    }
    __syncthreads();
    if (warp == 0) {
      uint32_t carry = 0;
#pragma unroll
      for (int i0 = 0; i0 < E; i0 += 32) {
        const int i = i0 + lane;
        const uint32_t v = i < E ? s_off[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (i < E) s_off[i] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
      }
      if (lane == 0) s_total = carry;
    }
    __syncthreads();
    if (m) {
      const uint64_t te = t * S::TE;
#pragma unroll
      for (int k = 0; k < S::SUB; ++k) {
        uint64_t o = base + s_off[k * SC_WARPS + warp] + ((excl >> (8 * k)) & 0xFFu);
        const uint64_t e = te + ((uint64_t)k * SC_THREADS + tid) * S::EPV;
#pragma unroll
        for (int j = 0; j < S::EPV; ++j) {
          if ((m >> (k * S::EPV + j)) & 1u) {
            if (LAYOUT == PIMDAL_LAYOUT_PAIRS) {
              const uint32_t ptr = reinterpret_cast<const pimdal_key_ptr32_t *>(p.in)[e + j].ptr;
              reinterpret_cast<uint2 *>(p.out)[o] = make_uint2(key[k * S::EPV + j], ptr);
            } else {
              reinterpret_cast<uint32_t *>(p.out)[o] = key[k * S::EPV + j];
              if (p.out_ptr) p.out_ptr[o] = HAS_PTR ? p.in_ptr[e + j] : (uint32_t)(p.ptr_base + e + j);
            }
            ++o;
          }
        }
      }
    }
    base += s_total;
    __syncthreads();  // s_off / s_total are rewritten by the next tile
  }
}

using CoKernel = void (*)(SelParams, uint64_t *, uint32_t *, uint64_t);
CoKernel pick_coop(int layout, bool is_signed, bool has_ptr) {
  if (layout == PIMDAL_LAYOUT_PAIRS)
    return is_signed ? k_select_coop<PIMDAL_LAYOUT_PAIRS, true, true>
                     : k_select_coop<PIMDAL_LAYOUT_PAIRS, false, true>;
  if (is_signed)
    return has_ptr ? k_select_coop<PIMDAL_LAYOUT_COLUMNS, true, true>
                   : k_select_coop<PIMDAL_LAYOUT_COLUMNS, true, false>;
  return has_ptr ? k_select_coop<PIMDAL_LAYOUT_COLUMNS, false, true>
                 : k_select_coop<PIMDAL_LAYOUT_COLUMNS, false, false>;
}

using SelKernel = void (*)(SelParams);
using SlKernel = void (*)(SlParams);

SlKernel pick_chunked(int layout, bool is_signed, bool has_ptr) {
  if (layout == PIMDAL_LAYOUT_PAIRS)
    return is_signed ? k_select_chunked<PIMDAL_LAYOUT_PAIRS, true, true>
                     : k_select_chunked<PIMDAL_LAYOUT_PAIRS, false, true>;
  if (is_signed)
    return has_ptr ? k_select_chunked<PIMDAL_LAYOUT_COLUMNS, true, true>
                   : k_select_chunked<PIMDAL_LAYOUT_COLUMNS, true, false>;
  return has_ptr ? k_select_chunked<PIMDAL_LAYOUT_COLUMNS, false, true>
                 : k_select_chunked<PIMDAL_LAYOUT_COLUMNS, false, false>;
}

SelKernel pick_kernel(int layout, bool is_signed, bool has_ptr) {
  if (layout == PIMDAL_LAYOUT_PAIRS)
    return is_signed ? k_select<PIMDAL_LAYOUT_PAIRS, true, true>
                     : k_select<PIMDAL_LAYOUT_PAIRS, false, true>;
  if (is_signed)
    return has_ptr ? k_select<PIMDAL_LAYOUT_COLUMNS, true, true>
                   : k_select<PIMDAL_LAYOUT_COLUMNS, true, false>;
  return has_ptr ? k_select<PIMDAL_LAYOUT_COLUMNS, false, true>
                 : k_select<PIMDAL_LAYOUT_COLUMNS, false, false>;
}

}  // namespace

// Turns a predicate descriptor into a closed interval [lo, hi] (+ inversion).
// Returns false for an invalid descriptor.
bool pd_pred_interval(const pimdal_pred_t &pr, int64_t *lo, int64_t *hi, uint32_t *invert) {
  const int64_t MIN = INT64_MIN, MAX = INT64_MAX;
  *invert = 0;
  switch (pr.op) {
    case PIMDAL_PRED_LT:
      if (pr.lo == MIN) { *lo = 1; *hi = 0; } else { *lo = MIN; *hi = pr.lo - 1; }
      return true;
    case PIMDAL_PRED_LE: *lo = MIN; *hi = pr.lo; return true;
    case PIMDAL_PRED_GT:
      if (pr.lo == MAX) { *lo = 1; *hi = 0; } else { *lo = pr.lo + 1; *hi = MAX; }
      return true;
    case PIMDAL_PRED_GE: *lo = pr.lo; *hi = MAX; return true;
    case PIMDAL_PRED_EQ: *lo = pr.lo; *hi = pr.lo; return true;
    case PIMDAL_PRED_NE: *lo = pr.lo; *hi = pr.lo; *invert = 1; return true;
    case PIMDAL_PRED_BETWEEN: *lo = pr.lo; *hi = pr.hi; return true;
    case PIMDAL_PRED_RANGE:
      if (pr.hi == MIN) { *lo = 1; *hi = 0; } else { *lo = pr.lo; *hi = pr.hi - 1; }
      return true;
  }
  return false;
}

extern "C" int pimdal_sel_workspace_size(const pimdal_sel_arguments_t *args, size_t *bytes) {
  if (!args || !bytes) return PIMDAL_ERR_ARG;
  *bytes = 0;  // only the context's lookback status words are used
  return PIMDAL_OK;
}

extern "C" int pimdal_sel_kernel(pimdal_ctx_t *ctx, const pimdal_sel_arguments_t *a,
                                 pimdal_sel_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result) return PIMDAL_ERR_ARG;
  if (a->layout != PIMDAL_LAYOUT_COLUMNS && a->layout != PIMDAL_LAYOUT_PAIRS) return PIMDAL_ERR_ARG;
  if (a->key_dtype != PIMDAL_I32 && a->key_dtype != PIMDAL_U32) return PIMDAL_ERR_ARG;
  if (a->size && (!a->in || !a->out)) return PIMDAL_ERR_ARG;
  if (a->layout == PIMDAL_LAYOUT_PAIRS && (((uintptr_t)a->in | (uintptr_t)a->out) & 7u))
    return PIMDAL_ERR_ARG;
  SelParams p{};
  int64_t lo, hi;
  if (!pd_pred_interval(a->pred, &lo, &hi, &p.invert)) return PIMDAL_ERR_ARG;
  {
    // clamp to the key type's range; an empty interval selects nothing
    const int64_t tmin = a->key_dtype == PIMDAL_I32 ? INT32_MIN : 0;
    const int64_t tmax = a->key_dtype == PIMDAL_I32 ? INT32_MAX : (int64_t)UINT32_MAX;
    lo = std::max(lo, tmin);
    hi = std::min(hi, tmax);
    if (lo > hi) {  // empty: "all in range, inverted" (or all, when inverted)
      p.lo32 = 0;
      p.range32 = 0xFFFFFFFFu;
      p.invert ^= 1u;
    } else {
      p.lo32 = (uint32_t)lo;
      p.range32 = (uint32_t)(hi - lo);
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  if (a->size == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d_result, 0, sizeof(uint64_t), s));
    return PIMDAL_OK;
  }
  const uint64_t tiles = pd_ceil_div(a->size, SEL_TILE);
  if (tiles > PD_STATUS_WORDS) return PIMDAL_ERR_ARG;
  int st;
  p.epoch = pd_next_epoch(ctx, s, &st);
  if (st) return st;
  p.in = a->in;
  p.in_ptr = a->layout == PIMDAL_LAYOUT_COLUMNS ? a->in_ptr : nullptr;
  p.ptr_base = a->ptr_base;
  p.out = a->out;
  p.out_ptr = a->layout == PIMDAL_LAYOUT_COLUMNS ? a->out_ptr : nullptr;
  p.n = a->size;
  p.vec_ok = ((((uintptr_t)a->in) | (uintptr_t)(p.in_ptr)) & 15u) == 0;
  p.status = ctx->d_status;
  p.d_error = ctx->d_error;
  p.d_count = &d_result->t_count;
  const bool is_signed = a->key_dtype == PIMDAL_I32;
  if (p.vec_ok && a->size >= (1u << 20)) {
    CoKernel k = pick_coop(a->layout, is_signed, p.in_ptr != nullptr);
    static int per_sm[2] = {0, 0};
    int &occ = per_sm[a->layout == PIMDAL_LAYOUT_PAIRS];
    if (!occ) {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, SC_THREADS, 0);
      if (occ <= 0) occ = 1;
    }
    const uint64_t te = (uint64_t)SC_THREADS * CO_SUB * (a->layout == PIMDAL_LAYOUT_PAIRS ? 2 : 4);
    const uint64_t ntiles = pd_ceil_div(a->size, te);
    const uint64_t want = std::min<uint64_t>(ntiles, (uint64_t)occ * ctx->sm_count);
    uint64_t tpc = pd_ceil_div(ntiles, want);
    unsigned grid = (unsigned)pd_ceil_div(ntiles, tpc);
    uint64_t *counts = ctx->d_status;  // per-CTA counts (epoch 0 words: never a live status)
    uint32_t *bar = ctx->d_counters + PD_COUNTER_SELECT;
    SelParams pp = p;
    void *args[] = {&pp, &counts, &bar, &tpc};
    pd_launch_scope scope(ctx, PIMDAL_KERNEL_SELECT, s);
    PD_CHECK_CUDA(cudaLaunchCooperativeKernel((const void *)k, dim3(grid), dim3(SC_THREADS), args, 0, s));
  } else {
    SelKernel k = pick_kernel(a->layout, is_signed, p.in_ptr != nullptr);
    pd_launch_scope scope(ctx, PIMDAL_KERNEL_SELECT, s);
    k<<<(unsigned)tiles, SEL_THREADS, 0, s>>>(p);
  }
  return pd_launch_status(ctx);
}

// ---------------------------------------------------------------------------
// pimdal_sel_kernel_noalloc: selection for callers that cannot allocate
// device memory.
//
// Some hosts of this operator may not call cudaMalloc at all: code running
// under a memory manager that owns every device allocation (a database
// buffer pool or a framework's caching allocator, which would see a foreign
// allocation as lost memory), or a real-time path where an allocation could
// block on a device-wide synchronisation.  pimdal_sel_kernel needs a
// pimdal_ctx, and creating one allocates.
// This entry point needs nothing but the caller's input, output and result
// buffers: its scratch (look-back status words, the chunk claim counters and
// an error word) is the file-scope device array below, which every GPU that
// loads this library holds until the process exits.
//
// Limits and rules:
//  * The scratch holds SEL_NA_STATUS_WORDS = 4096 look-back words, so a call
//    handles at most 4096 tiles or chunks: up to 2^29 rows when the input
//    (and row-id column) is 16-byte aligned, up to 2^24 rows otherwise.
//    Larger inputs are rejected with PIMDAL_ERR_WORKSPACE before anything is
//    launched.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) and clears it; make that first call before any
//    stream capture.
//  * All calls on one device share the array and it keeps the last call's
//    contents: the status words carry a per-call epoch, the counters reset
//    themselves, and the error word is cleared after every call.  Calls that
//    overlap on the GPU (different streams, no ordering between them) race on
//    the array and must not be issued; calls ordered on one stream are fine.
//  * A device-side failure (a bounded wait that gave up) is reported by
//    writing UINT64_MAX into d_result->t_count.
// ---------------------------------------------------------------------------
namespace {
constexpr uint32_t SEL_NA_STATUS_WORDS = 4096;
constexpr uint32_t SEL_NA_WORDS = SEL_NA_STATUS_WORDS + 8;  // + error word, claim counters
static __device__ __align__(256) uint64_t g_sel_noalloc_scratch[SEL_NA_WORDS];

struct SelNaDevice {
  bool ready = false;
  uint64_t *scratch = nullptr;  // device address of g_sel_noalloc_scratch
  uint32_t epoch = 0;
  int sm_count = 0;
};
constexpr int SEL_NA_MAX_DEVICES = 64;
SelNaDevice g_sel_na[SEL_NA_MAX_DEVICES];
std::mutex g_sel_na_mutex;

// Turns a recorded device error into the UINT64_MAX count, then clears the
// error word and the claim counters for the next call.
__global__ void k_sel_na_finish(uint64_t *scratch, uint64_t *d_count) {
  uint32_t *words = reinterpret_cast<uint32_t *>(scratch + SEL_NA_STATUS_WORDS);
  if (words[0]) *d_count = ~0ull;
  words[0] = 0;
  words[2] = 0;
  words[3] = 0;
}
}  // namespace

extern "C" int pimdal_sel_kernel_noalloc(const pimdal_sel_arguments_t *a,
                                         pimdal_sel_results_t *d_result, pimdal_stream_t stream) {
  if (!a || !d_result) return PIMDAL_ERR_ARG;
  if (a->layout != PIMDAL_LAYOUT_COLUMNS && a->layout != PIMDAL_LAYOUT_PAIRS) return PIMDAL_ERR_ARG;
  if (a->key_dtype != PIMDAL_I32 && a->key_dtype != PIMDAL_U32) return PIMDAL_ERR_ARG;
  if (a->size && (!a->in || !a->out)) return PIMDAL_ERR_ARG;
  if (a->layout == PIMDAL_LAYOUT_PAIRS && (((uintptr_t)a->in | (uintptr_t)a->out) & 7u))
    return PIMDAL_ERR_ARG;
  SelParams p{};
  int64_t lo, hi;
  if (!pd_pred_interval(a->pred, &lo, &hi, &p.invert)) return PIMDAL_ERR_ARG;
  const int64_t tmin = a->key_dtype == PIMDAL_I32 ? INT32_MIN : 0;
  const int64_t tmax = a->key_dtype == PIMDAL_I32 ? INT32_MAX : (int64_t)UINT32_MAX;
  lo = std::max(lo, tmin);
  hi = std::min(hi, tmax);
  if (lo > hi) {
    p.lo32 = 0;
    p.range32 = 0xFFFFFFFFu;
    p.invert ^= 1u;
  } else {
    p.lo32 = (uint32_t)lo;
    p.range32 = (uint32_t)(hi - lo);
  }
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SEL_NA_MAX_DEVICES)
    return PIMDAL_ERR_CUDA;

  std::lock_guard<std::mutex> lock(g_sel_na_mutex);
  SelNaDevice &d = g_sel_na[dev];
  if (!d.ready) {
    // One-time set-up on this device: the array's device address, and the
    // array cleared on the caller's stream (make this first call before any
    // stream capture).
    void *addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_sel_noalloc_scratch) != cudaSuccess || !addr) {
      cudaGetLastError();
      return PIMDAL_ERR_CUDA;
    }
    if (cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return PIMDAL_ERR_CUDA;
    PD_CHECK_CUDA(cudaMemsetAsync(addr, 0, sizeof(uint64_t) * SEL_NA_WORDS, s));
    d.scratch = (uint64_t *)addr;
    d.ready = true;
  }
  if (a->size == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d_result, 0, sizeof(uint64_t), s));
    return PIMDAL_OK;
  }
  p.in = a->in;
  p.in_ptr = a->layout == PIMDAL_LAYOUT_COLUMNS ? a->in_ptr : nullptr;
  p.ptr_base = a->ptr_base;
  p.out = a->out;
  p.out_ptr = a->layout == PIMDAL_LAYOUT_COLUMNS ? a->out_ptr : nullptr;
  p.n = a->size;
  p.vec_ok = ((((uintptr_t)a->in) | (uintptr_t)(p.in_ptr)) & 15u) == 0;
  p.status = d.scratch;
  p.d_error = reinterpret_cast<uint32_t *>(d.scratch + SEL_NA_STATUS_WORDS);
  p.d_count = &d_result->t_count;
  const bool is_signed = a->key_dtype == PIMDAL_I32;
  const bool chunked = p.vec_ok && a->size >= (1u << 20);
  SlParams q{};
  uint64_t words;
  if (chunked) {
    const uint64_t per_sm = pd_ceil_div(a->size, (uint64_t)d.sm_count);
    q.chunk_elems = std::min<uint64_t>(SL_CHUNK_MAX, pd_align_up(per_sm, SL_TILE));
    q.nchunks = pd_ceil_div(a->size, q.chunk_elems);
    words = q.nchunks;
  } else {
    words = pd_ceil_div(a->size, SEL_TILE);
  }
  if (words > SEL_NA_STATUS_WORDS) return PIMDAL_ERR_WORKSPACE;  // beyond the fixed scratch

  // Per-call epoch; stale status words are cleared when the 16-bit epoch wraps.
  d.epoch = (d.epoch + 1) & 0xFFFFu;
  if (d.epoch == 0) {
    PD_CHECK_CUDA(cudaMemsetAsync(d.scratch, 0, sizeof(uint64_t) * SEL_NA_STATUS_WORDS, s));
    d.epoch = 1;
  }
  p.epoch = d.epoch;
  if (chunked) {
    q.s = p;
    q.claim = reinterpret_cast<uint32_t *>(d.scratch + SEL_NA_STATUS_WORDS) + 2;
    const unsigned grid = (unsigned)std::min<uint64_t>(q.nchunks, (uint64_t)d.sm_count);
    SlKernel k = pick_chunked(a->layout, is_signed, p.in_ptr != nullptr);
    const int smem = SL_STAGES * SL_STAGE_BYTES;
    PD_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k<<<grid, SL_THREADS, smem, s>>>(q);
  } else {
    SelKernel k = pick_kernel(a->layout, is_signed, p.in_ptr != nullptr);
    k<<<(unsigned)words, SEL_THREADS, 0, s>>>(p);
  }
  k_sel_na_finish<<<1, 1, 0, s>>>(d.scratch, p.d_count);
  return cudaGetLastError() == cudaSuccess ? PIMDAL_OK : PIMDAL_ERR_CUDA;
}
