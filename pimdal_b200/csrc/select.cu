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
  int64_t lo, hi;
  uint32_t invert;
  uint32_t vec_ok;  // input pointers 16-byte aligned
  uint64_t *status;
  uint32_t epoch;
  uint32_t *d_error;
  uint64_t *d_count;
};

template <bool SIGNED>
__device__ __forceinline__ bool sel_pred(uint32_t key, const SelParams &p) {
  int64_t v = SIGNED ? (int64_t)(int32_t)key : (int64_t)key;
  return ((v >= p.lo) & (v <= p.hi)) != (p.invert != 0);
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

using SelKernel = void (*)(SelParams);

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
  if (!pd_pred_interval(a->pred, &p.lo, &p.hi, &p.invert)) return PIMDAL_ERR_ARG;
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
  SelKernel k = pick_kernel(a->layout, a->key_dtype == PIMDAL_I32, p.in_ptr != nullptr);
  {
    pd_launch_scope scope(ctx, PIMDAL_KERNEL_SELECT, s);
    k<<<(unsigned)tiles, SEL_THREADS, 0, s>>>(p);
  }
  return pd_launch_status(ctx);
}
