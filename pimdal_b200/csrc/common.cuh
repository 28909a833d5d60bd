// Shared internals of the pimdal_b200 CUDA library (sm_100a).
//
//  * pimdal_ctx: workspace, device error word, lookback status words.
//  * Decoupled look-back (single-pass prefix over tiles) with epoch-tagged
//    64-bit status words and bounded waits that report a timeout instead of
//    trapping.
//  * The seeded counter-based generator (host + device), shared bit-for-bit
//    with the numpy mirror in pimdal_b200/gen.py.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <map>
#include <vector>

#include "../../include/pimdal_gpu.h"

#define PD_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------------------
// Device error word bits (OR-ed by kernels, read by pimdal_ctx_sync_status).
// ---------------------------------------------------------------------------
enum : uint32_t {
  PD_DEVERR_TIMEOUT = 1u,     // a bounded spin gave up
  PD_DEVERR_TABLE_FULL = 2u,  // hash table had no free slot
  PD_DEVERR_CAPACITY = 4u,    // output buffer too small for the result
  PD_DEVERR_ARG = 8u          // a device-side argument check failed
};

// Slots of pimdal_ctx::d_counters (two words each: claim counter, CTAs done).
enum : uint32_t { PD_COUNTER_SELECT = 0, PD_COUNTER_PARTITION = 2, PD_COUNTER_GROUP = 4,
                  PD_COUNTER_PROBE = 6, PD_COUNTER_MERGE = 8, PD_COUNTER_MATCH = 10,
                  PD_COUNTER_FILTER = 12 };

// Lookback status word: [epoch:16][flag:2][value:46].
enum : uint32_t { PD_FLAG_INVALID = 0, PD_FLAG_AGGREGATE = 1, PD_FLAG_INCLUSIVE = 2 };
constexpr uint64_t PD_STATUS_VALUE_MASK = (1ull << 46) - 1;
constexpr uint32_t PD_STATUS_WORDS = 1u << 20;  // max tiles of one lookback launch
constexpr uint32_t PD_SPIN_LIMIT = 1u << 22;    // bounded wait (~seconds with backoff)

struct pd_prof_rec {
  int kernel;
  cudaEvent_t start, stop;
};

constexpr int PD_INGEST_MAX_THREADS = 16;  // host copy threads of pimdal_ingest

struct pimdal_ctx {
  int device = 0;
  int sm_count = 148;
  // workspace
  void *ws = nullptr;
  size_t ws_bytes = 0;
  bool ws_owned = false;
  // device words
  uint32_t *d_error = nullptr;   // error bits (word 0 of a zeroed 256-byte block)
  uint32_t *d_counters = nullptr;  // self-resetting work counters (words 16..63)
  uint64_t *d_status = nullptr;  // PD_STATUS_WORDS lookback status words
  uint32_t epoch = 0;            // 16-bit epoch of the last lookback launch
  uint64_t launches = 0;         // kernels launched through this context
  // per-kernel timing (pimdal_ctx_set_profiling)
  bool profiling = false;
  std::vector<pd_prof_rec> prof_pending;
  std::vector<cudaEvent_t> prof_free;
  uint64_t prof_launches[PIMDAL_KERNEL_COUNT] = {};
  double prof_ms[PIMDAL_KERNEL_COUNT] = {};
  // batch autotuner: best tuning per batch shape
  std::map<std::vector<uint64_t>, pimdal_batch_tuning_t> tune_cache;
  // plain-operator autotuner: best tuning per call shape
  std::map<std::vector<uint64_t>, pimdal_tuning_t> op_tune;
  // pimdal_ingest: pinned staging buffers (one per host copy thread) and the
  // events of their last transfers
  void *stage[PD_INGEST_MAX_THREADS] = {};
  cudaEvent_t stage_ev[PD_INGEST_MAX_THREADS] = {};
};

// Brackets one launch with timing events when profiling is on.
struct pd_launch_scope {
  pimdal_ctx *ctx;
  int kernel;
  cudaStream_t stream;
  cudaEvent_t start = nullptr;
  pd_launch_scope(pimdal_ctx *c, int k, cudaStream_t s);
  ~pd_launch_scope();
};

// Returns a workspace of at least `bytes` (256-byte aligned) or nullptr with
// *status set.  Grows an owned workspace; a caller-provided one is never grown.
void *pd_workspace(pimdal_ctx *ctx, size_t bytes, cudaStream_t stream, int *status);

// ceil(log2(x)) for x >= 1 (0 for x <= 1): the size class of a tuning shape.
inline uint64_t pd_log2_ceil(uint64_t x) {
  uint64_t b = 0;
  while ((1ull << b) < x && b < 63) ++b;
  return b;
}

// Device milliseconds of run() on stream s (events around it, waited for);
// a negative value when run() or the device reported an error, which is then
// read and cleared from the context.
template <typename F>
float pd_time_call(pimdal_ctx *ctx, cudaStream_t s, F run) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1.f;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return -1.f; }
  cudaEventRecord(e0, s);
  const int st = run();
  cudaEventRecord(e1, s);
  float ms = -1.f;
  if (st == PIMDAL_OK && pimdal_ctx_sync_status(ctx, s) == PIMDAL_OK &&
      cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
    ms = -1.f;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st == PIMDAL_OK ? ms : -1.f;
}

// Next lookback epoch (1..65535); clears the status words when it wraps.
uint32_t pd_next_epoch(pimdal_ctx *ctx, cudaStream_t stream, int *status);

// Maps the outcome of a launch to a status code.
int pd_launch_status(pimdal_ctx *ctx);

PD_HD uint64_t pd_align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }
PD_HD uint64_t pd_ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

#define PD_CHECK_CUDA(expr)                      \
  do {                                           \
    cudaError_t e__ = (expr);                    \
    if (e__ != cudaSuccess) return PIMDAL_ERR_CUDA; \
  } while (0)

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pd_store_release_u64(uint64_t *p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t pd_load_acquire_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void pd_store_release_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t pd_load_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void pd_store_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t pd_load_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void pd_store_relaxed_u64(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t pd_load_relaxed_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// ---- TMA bulk copies (non-multicast, this CTA's own shared memory) --------
__device__ __forceinline__ uint32_t pd_smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void pd_mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(pd_smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void pd_fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void pd_mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(pd_smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool pd_mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(pd_smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Orders this CTA's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same buffer.
__device__ __forceinline__ void pd_fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ uint64_t pd_policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// Global -> shared bulk copy completing on `bar`; src, dst 16-byte aligned,
// bytes a multiple of 16.  `pol` is an L2 cache policy.
__device__ __forceinline__ void pd_bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                            uint64_t *bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(pd_smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(pd_smem_u32(bar)), "l"(pol)
      : "memory");
}

__device__ __forceinline__ uint64_t pd_pack_status(uint32_t epoch, uint32_t flag, uint64_t v) {
  return ((uint64_t)epoch << 48) | ((uint64_t)flag << 46) | (v & PD_STATUS_VALUE_MASK);
}

__device__ __forceinline__ uint64_t pd_globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait shared by every spin in the library: returns true when the
// caller must give up -- either this wait exceeded PD_WAIT_NS (then the
// timeout bit is set) or another wait in the same launch already gave up
// (the error word is non-zero), so a broken dependency chain costs one
// timeout, not one per waiter.
constexpr uint64_t PD_WAIT_NS = 200ull * 1000 * 1000;
__device__ __forceinline__ bool pd_wait_expired(uint32_t *d_error, uint64_t t0, uint32_t spins) {
  if ((spins & 63u) == 0) {
    if (*(volatile uint32_t *)d_error & PD_DEVERR_TIMEOUT) return true;
    if (pd_globaltimer_ns() - t0 > PD_WAIT_NS) {
      atomicOr(d_error, PD_DEVERR_TIMEOUT);
      return true;
    }
  }
  return spins > PD_SPIN_LIMIT;
}

// Warp-cooperative decoupled look-back: returns the exclusive prefix of tile
// `tile` (sum of the values of tiles < tile).  Must be called by all 32 lanes
// of one warp.  On a bounded-wait expiry it sets PD_DEVERR_TIMEOUT and returns
// the partial sum (the result is then invalid but the kernel ends).
__device__ __forceinline__ uint64_t pd_lookback_warp(const uint64_t *status, int64_t tile,
                                                     uint32_t epoch, uint32_t *d_error) {
  const int lane = threadIdx.x & 31;
  uint64_t exclusive = 0;
  int64_t base = tile - 1;
  uint32_t spins = 0;
  const uint64_t t0 = pd_globaltimer_ns();
  while (true) {
    int64_t pred = base - lane;
    uint32_t flag = PD_FLAG_INCLUSIVE;
    uint64_t val = 0;
    if (pred >= 0) {
      uint64_t w = pd_load_acquire_u64(status + pred);
      flag = ((uint32_t)(w >> 48) == epoch) ? (uint32_t)((w >> 46) & 3u) : PD_FLAG_INVALID;
      val = w & PD_STATUS_VALUE_MASK;
    }
    unsigned incl = __ballot_sync(0xffffffffu, flag == PD_FLAG_INCLUSIVE);
    unsigned invalid = __ballot_sync(0xffffffffu, flag == PD_FLAG_INVALID);
    int first = incl ? (__ffs(incl) - 1) : 31;
    unsigned need = (first >= 31) ? 0xffffffffu : ((2u << first) - 1u);
    if (invalid & need) {
      bool give_up = false;
      ++spins;
      if (lane == 0) give_up = pd_wait_expired(d_error, t0, spins);
      if (__shfl_sync(0xffffffffu, give_up, 0)) {
        if (lane == 0) atomicOr(d_error, PD_DEVERR_TIMEOUT);
        return exclusive;
      }
      __nanosleep(spins < 64 ? 20 : 200);
      continue;
    }
    uint64_t contrib = (lane <= first) ? val : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
    exclusive += contrib;
    if (incl) break;
    base -= 32;
  }
  return exclusive;
}

// Block-wide decoupled look-back over epoch-tagged 64-bit status words: thread
// i inspects predecessor (chunk - 1 - i) in each round, so one round covers
// THREADS predecessors.  Called by all threads of the block; s_flags holds
// 2 * THREADS/32 words, s_sum THREADS/32 + 1.
template <int THREADS>
__device__ uint64_t pd_block_lookback(const uint64_t *status, int64_t chunk, uint32_t epoch,
                                   uint32_t *d_error, uint32_t *s_flags, uint64_t *s_sum,
                                   int *s_state) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t exclusive = 0;
  int64_t base = chunk - 1;
  uint32_t spins = 0;
  const uint64_t t0 = pd_globaltimer_ns();
  while (true) {
    int64_t pred = base - tid;
    uint32_t flag = PD_FLAG_INCLUSIVE;
    uint64_t val = 0;
    if (pred >= 0) {
      uint64_t w = pd_load_relaxed_u64(status + pred);
      flag = ((uint32_t)(w >> 48) == epoch) ? (uint32_t)((w >> 46) & 3u) : PD_FLAG_INVALID;
      val = w & PD_STATUS_VALUE_MASK;
    }
    unsigned incl = __ballot_sync(0xffffffffu, flag == PD_FLAG_INCLUSIVE);
    unsigned inval = __ballot_sync(0xffffffffu, flag == PD_FLAG_INVALID);
    int first = incl ? (__ffs(incl) - 1) : 32;
    uint64_t c = (lane <= first) ? val : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) {
      s_flags[2 * warp] = incl;
      s_flags[2 * warp + 1] = inval;
      s_sum[warp] = c;
    }
    __syncthreads();
    if (tid == 0) {
      // 0 = retry, 1 = done, 2 = continue further back
      int state = 2;
      uint64_t add = 0;
      for (int w = 0; w < (THREADS / 32); ++w) {
        unsigned in = s_flags[2 * w], iv = s_flags[2 * w + 1];
        int f = in ? (__ffs(in) - 1) : 32;
        unsigned need = (f >= 31) ? 0xffffffffu : ((2u << f) - 1u);
        if (iv & need) { state = 0; break; }
        add += s_sum[w];
        if (in) { state = 1; break; }
      }
      if (state == 0) {
        if (pd_wait_expired(d_error, t0, ++spins)) state = 3;
      } else {
        s_sum[(THREADS / 32)] = add;
      }
      *s_state = state;
    }
    __syncthreads();
    int state = *s_state;
    if (state == 3) return exclusive;
    if (state == 0) {
      __nanosleep(100);
      continue;
    }
    exclusive += s_sum[(THREADS / 32)];
    __syncthreads();
    if (state == 1) return exclusive;
    base -= THREADS;
  }
}

// ---------------------------------------------------------------------------
// Seeded counter-based generator (host + device).
//
// The 64-bit finaliser is SplitMix64's output function (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014).
// ---------------------------------------------------------------------------
constexpr uint64_t PD_GOLDEN64 = 0x9E3779B97F4A7C15ull;

PD_HD uint64_t pd_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Key of an independent sub-stream.
PD_HD uint64_t pd_stream_key(uint64_t seed, uint64_t stream) {
  return pd_mix64((seed * PD_GOLDEN64) ^ pd_mix64(stream + 0x632BE59BD9B4E019ull));
}
// i-th 64-bit draw of a sub-stream.
PD_HD uint64_t pd_rand(uint64_t key, uint64_t i) { return pd_mix64(key + (i + 1) * PD_GOLDEN64); }
// Second, independent draw for the same row.
PD_HD uint64_t pd_rand2(uint64_t r) { return pd_mix64(r ^ 0xD1B54A32D192ED03ull); }

// lo + floor(r_hi32 * span / 2^32), span = hi - lo + 1 <= 2^32.
PD_HD int64_t pd_uniform(uint64_t r, int64_t lo, uint64_t span) {
  return lo + (int64_t)(((r >> 32) * span) >> 32);
}
PD_HD double pd_unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// Bijective permutation of [0, n) (n = 0 means 2^32): four rounds of
// multiply-by-odd / add / xorshift modulo 2^b, then cycle-walking into [0, n).
struct pd_perm {
  uint32_t bits;
  uint64_t n, mask;
  uint64_t mul[4], add[4];
  uint32_t shift;
};
PD_HD pd_perm pd_make_perm(uint64_t seed, uint64_t n) {
  pd_perm p;
  p.n = n ? n : (1ull << 32);
  uint32_t b = 0;
  while ((1ull << b) < p.n) ++b;
  p.bits = b;
  p.mask = (b >= 64) ? ~0ull : ((1ull << b) - 1);
  p.shift = (b + 1) / 2;
  if (p.shift == 0) p.shift = 1;
  uint64_t k = pd_stream_key(seed, 0xFFFF0000ull);
  for (int r = 0; r < 4; ++r) {
    uint64_t c = pd_rand(k, (uint64_t)r);
    p.mul[r] = (c | 1ull) & p.mask;
    p.add[r] = (c >> 32) & p.mask;
  }
  return p;
}
PD_HD uint64_t pd_perm_pow2(const pd_perm &p, uint64_t x) {
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    x = (x * p.mul[r] + p.add[r]) & p.mask;
    x ^= x >> p.shift;
  }
  return x;
}
PD_HD uint64_t pd_perm_apply(const pd_perm &p, uint64_t x) {
  if (p.bits == 0) return 0;
  uint64_t y = pd_perm_pow2(p, x);
  // Cycle-walking needs < 2 steps on average (n > 2^(b-1)); the bound only
  // guarantees termination and is never reached in practice.
  for (int walk = 0; y >= p.n && walk < 4096; ++walk) y = pd_perm_pow2(p, y);
  return y < p.n ? y : y % p.n;
}

// ---------------------------------------------------------------------------
// Hash functions.
// ---------------------------------------------------------------------------
// hash0 of the reference's partitioning step (pimdal/hash/hash_func.h:5-14):
// the partition index of part_kernel is an interface-visible value (callers
// route partition p to consumer p), so it is kept identical.
PD_HD uint32_t pd_hash0(uint32_t key) {
  key += 272333u;
  key += ~(key << 5);
  key ^= (key >> 18);
  key += (key << 11);
  key ^= (key >> 17);
  return key;
}
// The four Bloom-filter hashes of the reference's filter_kernel /
// match_kernel (hash1..hash4, pimdal/hash/hash_func.h:16-60): a constant is
// added, then four shift-add / shift-xor mixing steps.  The filter bits are
// visible to callers (filters are caller memory), so the constants and shifts
// are kept identical.  F is 0..3 for hash1..hash4.
template <int F>
PD_HD uint32_t pd_bloom_hash(uint32_t k) {
  constexpr uint32_t add = F == 0 ? 593627u : F == 1 ? 274277u : F == 2 ? 855467u : 176521u;
  constexpr int s0 = F == 0 ? 22 : F == 1 ? 13 : F == 2 ? 4 : 10;
  constexpr int s1 = F == 0 ? 26 : F == 1 ? 20 : F == 2 ? 21 : 25;
  constexpr int s2 = F == 0 ? 10 : F == 1 ? 3 : F == 2 ? 5 : 5;
  constexpr int s3 = F == 0 ? 28 : F == 1 ? 9 : F == 2 ? 16 : 24;
  k += add;
  k += ~(k << s0);
  k ^= (k >> s1);
  k += (k << s2);
  k ^= (k >> s3);
  return k;
}

// Table-slot hash of this library (multiplicative / Fibonacci hashing):
// the top `bits` bits of key * 2^64/phi.
PD_HD uint64_t pd_hash_slot(uint32_t key, uint32_t bits) {
  return bits ? (((uint64_t)key * PD_GOLDEN64) >> (64 - bits)) : 0;
}
// Top 32 bits of the same product: partition digits are taken from its top
// bits, table slots from the bits below them.
PD_HD uint32_t pd_mulhash32(uint32_t key) { return (uint32_t)(((uint64_t)key * PD_GOLDEN64) >> 32); }

// ---------------------------------------------------------------------------
// Internal entry points shared between translation units.
// ---------------------------------------------------------------------------
enum : int { PD_KEY_PLAIN = 0, PD_KEY_HASH0 = 1, PD_KEY_MULHASH = 2 };
// A predicate as an inclusive interval [lo, hi] of int64 (and an inversion
// flag for NE); false for an unknown operator.
bool pd_pred_interval(const pimdal_pred_t &pr, int64_t *lo, int64_t *hi, uint32_t *invert);
int pd_sort_with_workspace(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, void *ws,
                           cudaStream_t s);
int pd_sort_ex(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
               cudaStream_t s, uint32_t **offsets_out);
int pd_sort_ex2(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
                cudaStream_t s, uint32_t **offsets_out, const uint64_t *n_dev);
// Stable radix partition of key columns by bits [a->begin_bit, a->end_bit) of
// a key transform, in passes of at most PD_PART_DIGIT_BITS bits, carrying the
// 32-bit column a->in_ptr -> a->out_ptr (row ids when a->in_ptr is NULL and
// a->out_ptr is set) and/or the 64-bit column in_v64 -> out_v64.
constexpr uint32_t PD_PART_DIGIT_BITS = 6;
// Sort of (key, payload) where the payload of row i is pay64[i] - *pay_min
// (int64 values whose range fits 32 bits; a->out_ptr receives the payloads,
// a->in_ptr must be NULL); the element count is read from *n_dev when given.
int pd_sort_pay64(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, void *ws, cudaStream_t s,
                  const uint64_t *n_dev, const int64_t *pay64, const int64_t *pay_min);
size_t pd_partition_workspace(const pimdal_sort_arguments_t *a, bool v64);
int pd_partition(pimdal_ctx *ctx, const pimdal_sort_arguments_t *a, int key_mode, void *ws,
                 cudaStream_t s, const uint64_t *in_v64, uint64_t *out_v64);
