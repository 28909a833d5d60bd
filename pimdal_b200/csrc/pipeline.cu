// Pipeline glue kernels of the served queries (pimdal_gather_u32,
// pimdal_revenue_keys): the column <-> pair conversions and arithmetic that
// the reference runs as separate DPU kernels between operators --
// arithmetic_kernel (pimdal/general/arithmetic.c:35-67, element-wise product
// of two key columns), the reduce chains of pimdal/general/reduce.c:42-77 and
// the glue of the query pipelines (e.g. pimdal/main/tpc_h/query6/dpu/
// kernel_q6.c:112-156).  Here they are fused into one pass each: a gather by
// row id, and a gather that builds a group key and an int64 revenue value
// price * (100 - discount) for every joined row.  Both are HBM-bound
// grid-stride loops; all arithmetic is integer.
#include <algorithm>

#include "common.cuh"

namespace {

__global__ void __launch_bounds__(256) k_gather_u32(const uint32_t *col, const uint32_t *idx,
                                                     uint64_t n, uint32_t *out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = __ldg(col + __ldcs(idx + i));
}

__global__ void __launch_bounds__(256) k_revenue_keys(pimdal_revenue_arguments_t a) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.size; i += stride) {
    const uint32_t sel = __ldcs(a.match_row + i);       // index into the selected rows
    const uint32_t row = a.sel_rows ? __ldg(a.sel_rows + sel) : sel;  // fact row
    uint32_t key = __ldcs(a.match_attr + i) * a.attr_mult;
    if (a.flag) key += __ldg(a.flag + row);
    a.out_key[i] = key;
    a.out_val[i] = __ldg(a.price + row) * (int64_t)(100 - __ldg(a.discount + row));
  }
}

unsigned grid_for(pimdal_ctx *ctx, uint64_t n) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(pd_ceil_div(n, 256), ctx->sm_count * 8ull));
}

}  // namespace

extern "C" int pimdal_gather_u32(pimdal_ctx_t *ctx, const uint32_t *col, const uint32_t *idx,
                                 uint64_t n, uint32_t *out, pimdal_stream_t stream) {
  if (!ctx || (n && (!col || !idx || !out))) return PIMDAL_ERR_ARG;
  if (!n) return PIMDAL_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = (cudaStream_t)stream;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_gather_u32<<<grid_for(ctx, n), 256, 0, s>>>(col, idx, n, out);
  }
  return pd_launch_status(ctx);
}

extern "C" int pimdal_revenue_keys(pimdal_ctx_t *ctx, const pimdal_revenue_arguments_t *a,
                                   pimdal_stream_t stream) {
  if (!ctx || !a) return PIMDAL_ERR_ARG;
  if (a->size && (!a->match_row || !a->match_attr || !a->price || !a->discount || !a->out_key ||
                  !a->out_val))
    return PIMDAL_ERR_ARG;
  if (!a->size) return PIMDAL_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = (cudaStream_t)stream;
  {
    pd_launch_scope sc(ctx, PIMDAL_KERNEL_OTHER, s);
    k_revenue_keys<<<grid_for(ctx, a->size), 256, 0, s>>>(*a);
  }
  return pd_launch_status(ctx);
}
