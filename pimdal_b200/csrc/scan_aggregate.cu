// K-SA: fused select -> arithmetic -> group-by scan (pimdal_select_aggregate).
//
// Reference behaviour: the query pipelines of pimdal/main/tpc_h run one DPU
// kernel per step with host or tasklet barriers between them -- sel_kernel
// for each predicate with a load_next gather of the next column in between,
// arithmetic_kernel (pimdal/general/arithmetic.c:35-67) for the products and
// reduce_kernel (pimdal/general/reduce.c:42-77) or a group_kernel for the
// sums (pimdal/main/tpc_h/query6/dpu/kernel_q6.c:112-156,
// pimdal/main/tpc_h/query1/dpu/kernel_q1_1.c:84-170 and kernel_q1_2.c).
//
// B200 design (HBM-bound, no tensor cores): one pass over the rows.
//  * Each thread takes SA_UNROLL rows per step (coalesced column loads, all
//    of a column's loads of the step in flight together).  The predicates
//    are tested in their order; a later column is read only for rows that
//    passed the earlier ones (a masked lane issues no load, so a sector whose
//    rows all failed is never fetched) -- the reference's late
//    materialisation, at sector granularity.
//  * Sums accumulate in shared memory in nsets copies of the table ([slot]
//    [set] layout): thread t adds into set t mod nsets, with plain adds when
//    every thread has its own set (nsets = 256) and shared-memory atomics
//    otherwise.  The host picks the most sets whose tables fit in
//    PD_SA_SMEM_TARGET bytes, so a small key space gets private slots and a
//    mid-sized one (TPC-H Q1: 6 keys x 6 sums) keeps the CTA small enough for
//    8 CTAs per SM; a large key space gets one shared table.  Each CTA
//    then adds its non-zero slots to a global table with one atomic each, and
//    one CTA emits the groups with rows, in key order.  Integer sums wrap mod
//    2^64 and do not depend on the order of the additions.
#include <algorithm>

#include "common.cuh"

namespace {

constexpr int SA_THREADS = 256;
#ifndef PD_SA_UNROLL
#define PD_SA_UNROLL 4  // rows per thread per step
#endif
#ifndef PD_SA_EAGER
#define PD_SA_EAGER 0   // 1: predicate columns read for every row, not only the selected ones
#endif
constexpr int SA_UNROLL = PD_SA_UNROLL;
#ifndef PD_SA_SMEM_TARGET
#define PD_SA_SMEM_TARGET (24 * 1024)  // shared-memory bytes of the table copies
#endif

struct SaCol {
  const void *p;
  int32_t dtype;
};

struct SaParams {
  uint64_t n;
  const uint32_t *rows;
  SaCol pc[PIMDAL_SA_MAX_PREDS];
  int64_t plo[PIMDAL_SA_MAX_PREDS];
  uint64_t prange[PIMDAL_SA_MAX_PREDS];  // selected: (v - lo) mod 2^64 <= range, xor pinv
  uint32_t pinv[PIMDAL_SA_MAX_PREDS];
  uint32_t npreds;
  SaCol gc[PIMDAL_SA_MAX_GROUP_COLS];
  uint32_t gmult[PIMDAL_SA_MAX_GROUP_COLS];
  uint32_t ngroup, ks;
  SaCol tc[PIMDAL_SA_MAX_EXPRS][PIMDAL_SA_MAX_TERMS];
  int64_t tadd[PIMDAL_SA_MAX_EXPRS][PIMDAL_SA_MAX_TERMS];
  uint32_t tneg[PIMDAL_SA_MAX_EXPRS][PIMDAL_SA_MAX_TERMS];
  uint32_t nterms[PIMDAL_SA_MAX_EXPRS];
  uint32_t nexprs;
  uint32_t nsets;                   // table copies (a power of two, 1 .. SA_THREADS)
  unsigned long long *g_acc;        // [ks][nexprs + 1] (slot 0: COUNT)
  uint32_t *d_error;
};

struct SaOut {
  uint32_t *key;
  int64_t *count;
  int64_t *sum[PIMDAL_SA_MAX_EXPRS];
  uint64_t cap;
};

// A column's values at this step's rows (0 where take[u] is false); the
// element type is resolved once per step, not once per row.
template <typename T>
__device__ __forceinline__ void sa_load_as(const void *col, const uint32_t (&row)[SA_UNROLL],
                                           const bool (&take)[SA_UNROLL], int64_t (&v)[SA_UNROLL]) {
  const T *q = reinterpret_cast<const T *>(col);
#pragma unroll
  for (int u = 0; u < SA_UNROLL; ++u) v[u] = take[u] ? (int64_t)__ldg(q + row[u]) : 0;
}

__device__ __forceinline__ void sa_load_rows(const SaCol &c, const uint32_t (&row)[SA_UNROLL],
                                             const bool (&take)[SA_UNROLL], int64_t (&v)[SA_UNROLL]) {
  switch (c.dtype) {
    case PIMDAL_I32: sa_load_as<int32_t>(c.p, row, take, v); break;
    case PIMDAL_U32: sa_load_as<uint32_t>(c.p, row, take, v); break;
    case PIMDAL_I64: sa_load_as<long long>(c.p, row, take, v); break;
    default: sa_load_as<unsigned char>(c.p, row, take, v); break;
  }
}

// 5 CTAs per SM (48 registers, a 40-byte spill): the scan is bound by the
// latency of its dependent column loads, and 5 CTAs hide more of it than 4
// at 64 registers (Q6 0.50 -> 0.43 ms, Q1 1.12 -> 0.98 ms on 6e7 rows).
__global__ void __launch_bounds__(SA_THREADS, 5) k_sa_scan(SaParams p) {
  extern __shared__ __align__(16) unsigned long long sa_acc[];
  const int tid = threadIdx.x;
  const uint32_t nv = p.nexprs + 1;
  const uint32_t slots = p.ks * nv;
  const uint32_t nsets = p.nsets;
  const uint32_t words = slots * nsets;
  const uint32_t set = tid & (nsets - 1);  // this thread's copy of the table
  for (uint32_t i = tid; i < words; i += SA_THREADS) sa_acc[i] = 0;
  __syncthreads();
  auto acc_add = [=](uint32_t key, uint32_t slot, unsigned long long v) {
    const uint32_t i = (key * nv + slot) * nsets + set;
    if (nsets == SA_THREADS) sa_acc[i] += v;
    else atomicAdd(&sa_acc[i], v);
  };
  // one key (no group columns): the sums stay in registers until the end
  const bool scalar = p.ks == 1;
  unsigned long long racc[PIMDAL_SA_MAX_EXPRS + 1];
#pragma unroll
  for (int e = 0; e <= PIMDAL_SA_MAX_EXPRS; ++e) racc[e] = 0;
  bool bad = false;
  const uint64_t step = (uint64_t)gridDim.x * SA_THREADS * SA_UNROLL;
  for (uint64_t base = (uint64_t)blockIdx.x * SA_THREADS * SA_UNROLL; base < p.n; base += step) {
    uint32_t row[SA_UNROLL];
    bool ok[SA_UNROLL], valid[SA_UNROLL];
#pragma unroll
    for (int u = 0; u < SA_UNROLL; ++u) {
      const uint64_t i = base + (uint64_t)u * SA_THREADS + tid;
      valid[u] = i < p.n;
      ok[u] = valid[u];
      row[u] = ok[u] ? (p.rows ? __ldg(p.rows + i) : (uint32_t)i) : 0u;
    }
    // predicates in order; a column is read only for rows still selected
#pragma unroll
    for (int q = 0; q < PIMDAL_SA_MAX_PREDS; ++q) {
      if (q < (int)p.npreds) {
        int64_t v[SA_UNROLL];
        sa_load_rows(p.pc[q], row, PD_SA_EAGER ? valid : ok, v);
        const int64_t lo = p.plo[q];
        const uint64_t range = p.prange[q];
        const bool inv = p.pinv[q] != 0;
#pragma unroll
        for (int u = 0; u < SA_UNROLL; ++u)
          ok[u] = ok[u] && (((uint64_t)(v[u] - lo) <= range) != inv);
      }
    }
    uint32_t key[SA_UNROLL];
#pragma unroll
    for (int u = 0; u < SA_UNROLL; ++u) key[u] = 0;
#pragma unroll
    for (int g = 0; g < PIMDAL_SA_MAX_GROUP_COLS; ++g) {
      if (g < (int)p.ngroup) {
        int64_t v[SA_UNROLL];
        sa_load_rows(p.gc[g], row, ok, v);
#pragma unroll
        for (int u = 0; u < SA_UNROLL; ++u) key[u] += (uint32_t)v[u] * p.gmult[g];
      }
    }
#pragma unroll
    for (int u = 0; u < SA_UNROLL; ++u) {
      if (ok[u] && key[u] >= p.ks) {
        bad = true;
        ok[u] = false;
      }
      if (scalar) racc[0] += ok[u] ? 1ull : 0ull;
      else if (ok[u]) acc_add(key[u], 0, 1ull);
    }
#pragma unroll
    for (int e = 0; e < PIMDAL_SA_MAX_EXPRS; ++e) {
      if (e >= (int)p.nexprs) continue;
      unsigned long long val[SA_UNROLL];
#pragma unroll
      for (int u = 0; u < SA_UNROLL; ++u) val[u] = 1ull;
#pragma unroll
      for (int t = 0; t < PIMDAL_SA_MAX_TERMS; ++t) {
        if (t < (int)p.nterms[e]) {
          const SaCol c = p.tc[e][t];
          const uint32_t neg = p.tneg[e][t];
          const int64_t add = p.tadd[e][t];
          int64_t x[SA_UNROLL];
          if (c.p) {
            sa_load_rows(c, row, ok, x);
          } else {
#pragma unroll
            for (int u = 0; u < SA_UNROLL; ++u) x[u] = 0;
          }
#pragma unroll
          for (int u = 0; u < SA_UNROLL; ++u) val[u] *= (unsigned long long)((neg ? -x[u] : x[u]) + add);
        }
      }
#pragma unroll
      for (int u = 0; u < SA_UNROLL; ++u) {
        if (scalar) racc[1 + e] += ok[u] ? val[u] : 0ull;
        else if (ok[u]) acc_add(key[u], 1 + e, val[u]);
      }
    }
  }
  if (scalar) {
#pragma unroll
    for (int e = 0; e <= PIMDAL_SA_MAX_EXPRS; ++e)
      if (e < (int)nv && racc[e]) acc_add(0, e, racc[e]);
  }
  if (bad) atomicOr(p.d_error, PD_DEVERR_ARG);
  __syncthreads();
  for (uint32_t s = tid; s < slots; s += SA_THREADS) {
    unsigned long long v = 0;
    for (uint32_t t = 0; t < nsets; ++t) v += sa_acc[s * nsets + t];
    if (v) atomicAdd(&p.g_acc[s], v);
  }
}

// One CTA: the groups with rows, in key order.
__global__ void __launch_bounds__(1024) k_sa_emit(const unsigned long long *g_acc, uint32_t ks,
                                                  uint32_t nexprs, SaOut o, uint64_t *t_count,
                                                  uint32_t *d_error) {
  __shared__ uint32_t s_warp[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t nv = nexprs + 1;
  const uint32_t k = tid;
  const bool has = k < ks && g_acc[(uint64_t)k * nv] != 0;
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
    const uint64_t pos = pre + __popc(m & ((1u << lane) - 1u));
    if (pos < o.cap) {
      o.key[pos] = k;
      o.count[pos] = (int64_t)g_acc[(uint64_t)k * nv];
#pragma unroll
      for (int e = 0; e < PIMDAL_SA_MAX_EXPRS; ++e)
        if (e < (int)nexprs && o.sum[e]) o.sum[e][pos] = (int64_t)g_acc[(uint64_t)k * nv + 1 + e];
    } else {
      atomicOr(d_error, PD_DEVERR_CAPACITY);
    }
  }
  if (tid == 0) *t_count = total;
}

static_assert(PIMDAL_SA_MAX_KEYS <= 1024, "one emit thread per key");

// pimdal_project: the expression at every row, grid-stride, the same term
// evaluation as the scan above; the output is written coalesced.
struct PjExpr {
  SaCol tc[PIMDAL_SA_MAX_TERMS];
  int64_t tadd[PIMDAL_SA_MAX_TERMS];
  uint32_t tneg[PIMDAL_SA_MAX_TERMS];
  uint32_t nterms;  // 0: the expression is absent (0)
};

struct PjParams {
  uint64_t n;
  const uint32_t *rows;
  PjExpr x[2];  // out = x[0] - x[1]
  uint32_t out64;
  uint32_t shift;
  void *out;
};

__device__ __forceinline__ void pj_eval(const PjExpr &e, const uint32_t (&row)[SA_UNROLL],
                                        const bool (&ok)[SA_UNROLL],
                                        unsigned long long (&val)[SA_UNROLL]) {
#pragma unroll
  for (int u = 0; u < SA_UNROLL; ++u) val[u] = e.nterms ? 1ull : 0ull;
#pragma unroll
  for (int t = 0; t < PIMDAL_SA_MAX_TERMS; ++t) {
    if (t < (int)e.nterms) {
      int64_t x[SA_UNROLL];
      if (e.tc[t].p) {
        sa_load_rows(e.tc[t], row, ok, x);
      } else {
#pragma unroll
        for (int u = 0; u < SA_UNROLL; ++u) x[u] = 0;
      }
#pragma unroll
      for (int u = 0; u < SA_UNROLL; ++u)
        val[u] *= (unsigned long long)((e.tneg[t] ? -x[u] : x[u]) + e.tadd[t]);
    }
  }
}

__global__ void __launch_bounds__(SA_THREADS) k_sa_project(PjParams p) {
  const int tid = threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * SA_THREADS * SA_UNROLL;
  for (uint64_t base = (uint64_t)blockIdx.x * SA_THREADS * SA_UNROLL; base < p.n; base += step) {
    uint32_t row[SA_UNROLL];
    bool ok[SA_UNROLL];
#pragma unroll
    for (int u = 0; u < SA_UNROLL; ++u) {
      const uint64_t i = base + (uint64_t)u * SA_THREADS + tid;
      ok[u] = i < p.n;
      row[u] = ok[u] ? (p.rows ? __ldg(p.rows + i) : (uint32_t)i) : 0u;
    }
    unsigned long long val[SA_UNROLL], sub[SA_UNROLL];
    pj_eval(p.x[0], row, ok, val);
    pj_eval(p.x[1], row, ok, sub);
#pragma unroll
    for (int u = 0; u < SA_UNROLL; ++u) val[u] -= sub[u];
#pragma unroll
    for (int u = 0; u < SA_UNROLL; ++u) {
      if (!ok[u]) continue;
      const uint64_t i = base + (uint64_t)u * SA_THREADS + tid;
      const long long v = (long long)val[u] >> p.shift;
      if (p.out64) reinterpret_cast<long long *>(p.out)[i] = v;
      else reinterpret_cast<uint32_t *>(p.out)[i] = (uint32_t)v;
    }
  }
}

bool sa_dtype_ok(int32_t d) {
  return d == PIMDAL_I32 || d == PIMDAL_U32 || d == PIMDAL_I64 || d == PIMDAL_U8;
}

}  // namespace

extern "C" int pimdal_select_aggregate_workspace_size(const pimdal_select_aggregate_arguments_t *a,
                                                      size_t *bytes) {
  if (!a || !bytes || a->key_space == 0 || a->key_space > PIMDAL_SA_MAX_KEYS ||
      a->n_exprs > PIMDAL_SA_MAX_EXPRS)
    return PIMDAL_ERR_ARG;
  *bytes = 8ull * a->key_space * (a->n_exprs + 1);
  return PIMDAL_OK;
}

extern "C" int pimdal_select_aggregate(pimdal_ctx_t *ctx,
                                       const pimdal_select_aggregate_arguments_t *a,
                                       pimdal_aggr_results_t *d_result, pimdal_stream_t stream) {
  if (!ctx || !a || !d_result) return PIMDAL_ERR_ARG;
  if (a->size >= (1ull << 32) || a->n_preds > PIMDAL_SA_MAX_PREDS ||
      a->n_group > PIMDAL_SA_MAX_GROUP_COLS || a->n_exprs > PIMDAL_SA_MAX_EXPRS ||
      a->key_space == 0 || a->key_space > PIMDAL_SA_MAX_KEYS)
    return PIMDAL_ERR_ARG;
  if (a->out_capacity && (!a->out_key || !a->out_count)) return PIMDAL_ERR_ARG;
  SaParams p{};
  p.n = a->size;
  p.rows = a->rows;
  p.npreds = a->n_preds;
  for (uint32_t q = 0; q < a->n_preds; ++q) {
    const pimdal_column_pred_t &c = a->pred[q];
    if (!sa_dtype_ok(c.dtype) || (a->size && !c.col)) return PIMDAL_ERR_ARG;
    int64_t lo, hi;
    if (!pd_pred_interval(c.pred, &lo, &hi, &p.pinv[q])) return PIMDAL_ERR_ARG;
    if (lo > hi) {  // an empty interval: "everything, inverted"
      p.plo[q] = 0;
      p.prange[q] = UINT64_MAX;
      p.pinv[q] ^= 1u;
    } else {
      p.plo[q] = lo;
      p.prange[q] = (uint64_t)hi - (uint64_t)lo;
    }
    p.pc[q] = {c.col, c.dtype};
  }
  p.ngroup = a->n_group;
  for (uint32_t g = 0; g < a->n_group; ++g) {
    const pimdal_group_col_t &c = a->group[g];
    if (!sa_dtype_ok(c.dtype) || (a->size && !c.col)) return PIMDAL_ERR_ARG;
    p.gc[g] = {c.col, c.dtype};
    p.gmult[g] = c.mult;
  }
  p.ks = a->key_space;
  p.nexprs = a->n_exprs;
  for (uint32_t e = 0; e < a->n_exprs; ++e) {
    const pimdal_expr_t &x = a->expr[e];
    if (x.n_terms == 0 || x.n_terms > PIMDAL_SA_MAX_TERMS) return PIMDAL_ERR_ARG;
    p.nterms[e] = x.n_terms;
    for (uint32_t t = 0; t < x.n_terms; ++t) {
      const pimdal_term_t &term = x.term[t];
      if (term.col && !sa_dtype_ok(term.dtype)) return PIMDAL_ERR_ARG;
      p.tc[e][t] = {term.col, term.dtype};
      p.tadd[e][t] = term.add;
      p.tneg[e][t] = term.negate != 0;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  const uint32_t nv = a->n_exprs + 1;
  const size_t ws_bytes = 8ull * a->key_space * nv;
  int st;
  char *ws = (char *)pd_workspace(ctx, ws_bytes, s, &st);
  if (!ws) return st;
  PD_CHECK_CUDA(cudaMemsetAsync(ws, 0, ws_bytes, s));
  p.g_acc = (unsigned long long *)ws;
  p.d_error = ctx->d_error;
  const uint64_t slots = (uint64_t)a->key_space * nv;
  p.nsets = SA_THREADS;
  while (p.nsets > 1 && slots * p.nsets * 8 > PD_SA_SMEM_TARGET) p.nsets >>= 1;
  const size_t smem = slots * p.nsets * 8;
  if (a->size) {
    PD_CHECK_CUDA(cudaFuncSetAttribute(k_sa_scan, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    int per_sm = 0;  // CTAs per SM at this shared-memory size
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sa_scan, SA_THREADS, smem) !=
            cudaSuccess || per_sm <= 0)
      per_sm = 1;
    const uint64_t want = pd_ceil_div(a->size, (uint64_t)SA_THREADS * SA_UNROLL);
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(want, (uint64_t)per_sm * ctx->sm_count));
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_SCAN_AGG, s);
    k_sa_scan<<<grid, SA_THREADS, smem, s>>>(p);
  }
  SaOut o{};
  o.key = a->out_key;
  o.count = a->out_count;
  for (uint32_t e = 0; e < a->n_exprs; ++e) o.sum[e] = a->out_sum[e];
  o.cap = a->out_capacity;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_sa_emit<<<1, 1024, 0, s>>>(p.g_acc, a->key_space, a->n_exprs, o, &d_result->t_count,
                                 ctx->d_error);
  }
  return pd_launch_status(ctx);
}

extern "C" int pimdal_project(pimdal_ctx_t *ctx, const pimdal_project_arguments_t *a,
                              pimdal_stream_t stream) {
  if (!ctx || !a) return PIMDAL_ERR_ARG;
  if (a->size >= (1ull << 32) || (a->size && !a->out)) return PIMDAL_ERR_ARG;
  if (a->out_dtype != PIMDAL_I64 && a->out_dtype != PIMDAL_I32) return PIMDAL_ERR_ARG;
  if (a->shift > 63) return PIMDAL_ERR_ARG;
  if (a->expr.n_terms == 0) return PIMDAL_ERR_ARG;
  PjParams p{};
  p.n = a->size;
  p.rows = a->rows;
  for (int k = 0; k < 2; ++k) {
    const pimdal_expr_t &x = k ? a->minus : a->expr;
    if (x.n_terms > PIMDAL_SA_MAX_TERMS) return PIMDAL_ERR_ARG;
    p.x[k].nterms = x.n_terms;
    for (uint32_t t = 0; t < x.n_terms; ++t) {
      const pimdal_term_t &term = x.term[t];
      if (term.col && !sa_dtype_ok(term.dtype)) return PIMDAL_ERR_ARG;
      p.x[k].tc[t] = {term.col, term.dtype};
      p.x[k].tadd[t] = term.add;
      p.x[k].tneg[t] = term.negate != 0;
    }
  }
  p.out64 = a->out_dtype == PIMDAL_I64;
  p.shift = a->shift;
  p.out = a->out;
  if (a->size == 0) return PIMDAL_OK;
  cudaStream_t s = (cudaStream_t)stream;
  cudaSetDevice(ctx->device);
  const uint64_t want = pd_ceil_div(a->size, (uint64_t)SA_THREADS * SA_UNROLL);
  const unsigned grid = (unsigned)std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 8);
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_sa_project<<<grid, SA_THREADS, 0, s>>>(p);
  }
  return pd_launch_status(ctx);
}
