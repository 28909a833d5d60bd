// pimdal_ingest: a host column into device memory through the context's
// pinned staging buffers (host side only; no kernels).
//
// Reference behaviour: the TPC-H pipelines read parquet columns into Arrow
// buffers (pimdal/main/tpc_h/reader/read_table.cpp:18-34) and scatter them
// over the DPUs' MRAM (populate_mram / dist_table,
// pimdal/support/transfer_helper.h).  Here a column goes to one GPU's HBM.
// A DMA from pageable memory cannot overlap the host: the driver stages it
// through its own buffers and the call blocks.  So a pageable source is
// copied chunk by chunk into two pinned buffers in turn; each chunk's
// transfer is queued on the stream and overlaps the host copy of the next,
// and a buffer is refilled only after the event of its last transfer.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace {

bool host_pinned(const void *p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // pageable memory can report an error on older drivers
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" int pimdal_ingest(pimdal_ctx_t *ctx, const void *host_src, size_t bytes, void *dst,
                             pimdal_stream_t stream) {
  if (!ctx || (bytes && (!host_src || !dst))) return PIMDAL_ERR_ARG;
  if (!bytes) return PIMDAL_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = (cudaStream_t)stream;
  if (host_pinned(host_src)) {
    PD_CHECK_CUDA(cudaMemcpyAsync(dst, host_src, bytes, cudaMemcpyHostToDevice, s));
    return PIMDAL_OK;
  }
  for (int i = 0; i < 2; ++i) {
    if (!ctx->stage[i] && cudaHostAlloc(&ctx->stage[i], PIMDAL_INGEST_CHUNK, cudaHostAllocDefault) != cudaSuccess) {
      ctx->stage[i] = nullptr;
      return PIMDAL_ERR_OOM;
    }
    if (!ctx->stage_ev[i]) PD_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->stage_ev[i], cudaEventDisableTiming));
  }
  const char *src = (const char *)host_src;
  char *d = (char *)dst;
  int b = 0;
  for (size_t off = 0; off < bytes; off += PIMDAL_INGEST_CHUNK, b ^= 1) {
    const size_t n = std::min<size_t>(PIMDAL_INGEST_CHUNK, bytes - off);
    PD_CHECK_CUDA(cudaEventSynchronize(ctx->stage_ev[b]));  // its previous transfer is done
    std::memcpy(ctx->stage[b], src + off, n);
    PD_CHECK_CUDA(cudaMemcpyAsync(d + off, ctx->stage[b], n, cudaMemcpyHostToDevice, s));
    PD_CHECK_CUDA(cudaEventRecord(ctx->stage_ev[b], s));
  }
  return PIMDAL_OK;
}
