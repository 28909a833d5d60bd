// Seeded column generator (pimdal_gen_column).  Replaces the per-OpenMP-thread
// std::default_random_engine generators of reference/db_operators/shared.cpp:10-60
// (whose output depends on the thread count) by a counter-based generator:
// row i's value is a pure function of (seed, stream_id, i).
#include "common.cuh"

namespace {

struct GenParams {
  int kind;
  int out_bytes;
  uint64_t draw_key;
  int64_t lo;
  uint64_t span;      // hi - lo + 1 (uniform draws)
  pd_perm perm;
  const double *cdf;
  uint64_t cdf_n;
  uint32_t match_permille;
  uint64_t probe_build;  // PROBE: number of build keys (spec.lo)
  uint64_t probe_span;   // PROBE: domain - build (non-matching draws)
};

// Index of the first CDF entry greater than u (numpy searchsorted 'right'),
// clamped to cdf_n - 1.
__device__ __forceinline__ uint64_t zipf_index(const double *cdf, uint64_t n, double u) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (cdf[mid] <= u) lo = mid + 1; else hi = mid;
  }
  return lo < n ? lo : n - 1;
}

__device__ __forceinline__ int64_t gen_value(const GenParams &p, uint64_t row) {
  uint64_t r = pd_rand(p.draw_key, row);
  switch (p.kind) {
    case PIMDAL_GEN_UNIFORM:
      return pd_uniform(r, p.lo, p.span);
    case PIMDAL_GEN_PERM:
      return (int64_t)pd_perm_apply(p.perm, row);
    case PIMDAL_GEN_PERM_UNIFORM:
      return (int64_t)pd_perm_apply(p.perm, (uint64_t)pd_uniform(r, p.lo, p.span));
    case PIMDAL_GEN_PERM_ZIPF:
      return (int64_t)pd_perm_apply(p.perm, zipf_index(p.cdf, p.cdf_n, pd_unit(r)));
    case PIMDAL_GEN_PROBE: {
      uint64_t r2 = pd_rand2(r);
      bool match = (uint32_t)pd_uniform(r2, 0, 1000) < p.match_permille;
      uint64_t idx;
      if (match) {
        idx = p.cdf ? zipf_index(p.cdf, p.cdf_n, pd_unit(r))
                    : (uint64_t)pd_uniform(r, 0, p.probe_build);
      } else {
        idx = p.probe_build + (uint64_t)pd_uniform(r, 0, p.probe_span);
      }
      return (int64_t)pd_perm_apply(p.perm, idx);
    }
  }
  return 0;
}

__global__ void __launch_bounds__(256) k_gen(GenParams p, void *dst, uint64_t n, uint64_t off) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    int64_t v = gen_value(p, off + i);
    if (p.out_bytes == 8) ((int64_t *)dst)[i] = v;
    else ((uint32_t *)dst)[i] = (uint32_t)v;
  }
}

}  // namespace

extern "C" int pimdal_gen_column(pimdal_ctx_t *ctx, const pimdal_gen_spec_t *s, void *dst,
                                 uint64_t n, uint64_t row_offset, pimdal_stream_t stream) {
  if (!ctx || !s || (!dst && n)) return PIMDAL_ERR_ARG;
  if (n == 0) return PIMDAL_OK;
  GenParams p{};
  p.kind = s->kind;
  p.out_bytes = (s->out_dtype == PIMDAL_I64) ? 8 : 4;
  p.draw_key = pd_stream_key(s->seed, s->stream_id);
  p.lo = s->lo;
  p.span = 0;  // only the uniform kinds use [lo, hi]
  if (s->hi >= s->lo) {
    p.span = (uint64_t)(s->hi - s->lo) + 1;
    if (p.span > (1ull << 32)) p.span = 0;
  }
  if (s->perm_domain > (1ull << 32)) return PIMDAL_ERR_ARG;
  p.perm = pd_make_perm(s->seed, s->perm_domain);
  p.cdf = s->cdf;
  p.cdf_n = s->cdf_n;
  p.match_permille = s->match_permille;
  switch (s->kind) {
    case PIMDAL_GEN_UNIFORM:
    case PIMDAL_GEN_PERM_UNIFORM:
      if (p.span == 0) return PIMDAL_ERR_ARG;  // span must be in [1, 2^32]
      break;
    case PIMDAL_GEN_PERM:
      break;
    case PIMDAL_GEN_PERM_ZIPF:
      if (!s->cdf || !s->cdf_n) return PIMDAL_ERR_ARG;
      break;
    case PIMDAL_GEN_PROBE: {
      uint64_t dom = s->perm_domain ? s->perm_domain : (1ull << 32);
      if (s->lo <= 0 || (uint64_t)s->lo >= dom || s->match_permille > 1000) return PIMDAL_ERR_ARG;
      if (s->cdf && !s->cdf_n) return PIMDAL_ERR_ARG;
      p.probe_build = (uint64_t)s->lo;
      p.probe_span = dom - (uint64_t)s->lo;
      break;
    }
    default:
      return PIMDAL_ERR_ARG;
  }
  cudaSetDevice(ctx->device);
  uint64_t blocks = pd_ceil_div(n, 256);
  uint64_t cap = (uint64_t)ctx->sm_count * 16;
  if (blocks > cap) blocks = cap;
  {
    pd_launch_scope scope(ctx, PIMDAL_KERNEL_GEN, (cudaStream_t)stream);
    k_gen<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(p, dst, n, row_offset);
  }
  return pd_launch_status(ctx);
}
