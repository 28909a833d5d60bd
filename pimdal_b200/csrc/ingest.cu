// pimdal_ingest: a host column into device memory through the context's
// pinned staging buffers (host side only; no kernels).
//
// Reference behaviour: the TPC-H pipelines read parquet columns into Arrow
// buffers (pimdal/main/tpc_h/reader/read_table.cpp:18-34) and scatter them
// over the DPUs' MRAM (populate_mram / dist_table,
// pimdal/support/transfer_helper.h).  Here a column goes to one GPU's HBM.
// A DMA from pageable memory cannot overlap the host: the driver stages it
// through its own buffers, one host thread at a time.  So a pageable source
// is split into chunks that PIMDAL_INGEST_THREADS host threads copy into
// their own pinned buffers; each chunk's transfer is queued on the stream
// and overlaps the host copies of the next chunks, and a buffer is refilled
// only after the event of its previous transfer.  The chunks land in
// disjoint parts of the destination, so their order on the stream does not
// matter, and all of them are queued before the call returns.  A pinned
// source needs no staging: its transfer reads it directly, later, in stream
// order.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

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

int ingest_threads() {
  static int t = 0;
  if (!t) {
    const char *e = std::getenv("PIMDAL_INGEST_THREADS");
    t = e ? std::atoi(e) : 8;
    t = std::max(1, std::min(t, PD_INGEST_MAX_THREADS));
  }
  return t;
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
  const size_t chunks = (bytes + PIMDAL_INGEST_CHUNK - 1) / PIMDAL_INGEST_CHUNK;
  const int nt = (int)std::min<size_t>(ingest_threads(), chunks);
  for (int i = 0; i < nt; ++i) {
    if (!ctx->stage[i] && cudaHostAlloc(&ctx->stage[i], PIMDAL_INGEST_CHUNK, cudaHostAllocDefault) != cudaSuccess) {
      ctx->stage[i] = nullptr;
      return PIMDAL_ERR_OOM;
    }
    if (!ctx->stage_ev[i]) PD_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->stage_ev[i], cudaEventDisableTiming));
  }
  const char *src = (const char *)host_src;
  char *d = (char *)dst;
  std::atomic<int> status{PIMDAL_OK};
  // Worker w copies chunks w, w + nt, ... through staging buffer w.
  auto work = [&](int w) {
    cudaSetDevice(ctx->device);
    for (size_t c = w; c < chunks && status.load() == PIMDAL_OK; c += nt) {
      const size_t off = c * PIMDAL_INGEST_CHUNK;
      const size_t n = std::min<size_t>(PIMDAL_INGEST_CHUNK, bytes - off);
      if (cudaEventSynchronize(ctx->stage_ev[w]) != cudaSuccess) {  // its previous transfer is done
        status = PIMDAL_ERR_CUDA;
        return;
      }
      std::memcpy(ctx->stage[w], src + off, n);
      if (cudaMemcpyAsync(d + off, ctx->stage[w], n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
          cudaEventRecord(ctx->stage_ev[w], s) != cudaSuccess) {
        status = PIMDAL_ERR_CUDA;
        return;
      }
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (int w = 0; w < nt; ++w) pool.emplace_back(work, w);
    for (auto &t : pool) t.join();
  }
  return status.load();
}
