// Context, workspace and status handling of the C ABI.
#include <new>

#include "common.cuh"

extern "C" int pimdal_abi_version(void) { return PIMDAL_ABI_VERSION; }

extern "C" const char *pimdal_status_string(int s) {
  switch (s) {
    case PIMDAL_OK: return "ok";
    case PIMDAL_ERR_ARG: return "bad argument";
    case PIMDAL_ERR_OOM: return "device allocation failed";
    case PIMDAL_ERR_WORKSPACE: return "workspace too small";
    case PIMDAL_ERR_TABLE_FULL: return "hash table full";
    case PIMDAL_ERR_DEVICE_TIMEOUT: return "bounded device wait timed out";
    case PIMDAL_ERR_CUDA: return "CUDA error";
    case PIMDAL_ERR_CAPACITY: return "output capacity exceeded";
    case PIMDAL_ERR_BUDGET: return "HBM budget exceeded";
    case PIMDAL_ERR_NOT_SUPPORTED: return "not supported";
    default: return "unknown status";
  }
}

extern "C" int pimdal_ctx_create(pimdal_ctx_t **out, int device) {
  if (!out) return PIMDAL_ERR_ARG;
  *out = nullptr;
  PD_CHECK_CUDA(cudaSetDevice(device));
  pimdal_ctx *ctx = new (std::nothrow) pimdal_ctx();
  if (!ctx) return PIMDAL_ERR_OOM;
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc(&ctx->d_error, 256) != cudaSuccess ||
      cudaMalloc(&ctx->d_status, sizeof(uint64_t) * PD_STATUS_WORDS) != cudaSuccess) {
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_status);
    delete ctx;
    return PIMDAL_ERR_OOM;
  }
  if (cudaMemset(ctx->d_error, 0, 256) != cudaSuccess ||
      cudaMemset(ctx->d_status, 0, sizeof(uint64_t) * PD_STATUS_WORDS) != cudaSuccess ||
      cudaDeviceSynchronize() != cudaSuccess) {
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_status);
    delete ctx;
    return PIMDAL_ERR_CUDA;
  }
  ctx->d_counters = ctx->d_error + 16;
  *out = ctx;
  return PIMDAL_OK;
}

static cudaEvent_t prof_event(pimdal_ctx *ctx) {
  if (!ctx->prof_free.empty()) {
    cudaEvent_t e = ctx->prof_free.back();
    ctx->prof_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

pd_launch_scope::pd_launch_scope(pimdal_ctx *c, int k, cudaStream_t s) : ctx(c), kernel(k), stream(s) {
  ctx->launches++;
  if (ctx->profiling) {
    start = prof_event(ctx);
    if (start) cudaEventRecord(start, stream);
  }
}

pd_launch_scope::~pd_launch_scope() {
  if (!start) return;
  cudaEvent_t stop = prof_event(ctx);
  if (!stop) return;
  cudaEventRecord(stop, stream);
  ctx->prof_pending.push_back({kernel, start, stop});
}

static void prof_drain(pimdal_ctx *ctx) {
  for (auto &r : ctx->prof_pending) {
    float ms = 0.f;
    cudaEventSynchronize(r.stop);
    if (cudaEventElapsedTime(&ms, r.start, r.stop) == cudaSuccess) {
      ctx->prof_launches[r.kernel]++;
      ctx->prof_ms[r.kernel] += ms;
    }
    ctx->prof_free.push_back(r.start);
    ctx->prof_free.push_back(r.stop);
  }
  ctx->prof_pending.clear();
}

extern "C" int pimdal_ctx_set_profiling(pimdal_ctx_t *ctx, int enable) {
  if (!ctx) return PIMDAL_ERR_ARG;
  prof_drain(ctx);
  ctx->profiling = enable != 0;
  return PIMDAL_OK;
}

extern "C" int pimdal_ctx_kernel_time(pimdal_ctx_t *ctx, int kernel_id, uint64_t *launches,
                                      double *total_ms) {
  if (!ctx || kernel_id < 0 || kernel_id >= PIMDAL_KERNEL_COUNT || !launches || !total_ms)
    return PIMDAL_ERR_ARG;
  prof_drain(ctx);
  *launches = ctx->prof_launches[kernel_id];
  *total_ms = ctx->prof_ms[kernel_id];
  ctx->prof_launches[kernel_id] = 0;
  ctx->prof_ms[kernel_id] = 0.0;
  return PIMDAL_OK;
}

extern "C" int pimdal_ctx_destroy(pimdal_ctx_t *ctx) {
  if (!ctx) return PIMDAL_ERR_ARG;
  cudaSetDevice(ctx->device);
  prof_drain(ctx);
  for (cudaEvent_t e : ctx->prof_free) cudaEventDestroy(e);
  for (int i = 0; i < PD_INGEST_MAX_THREADS; ++i) {
    if (ctx->stage_ev[i]) {
      cudaEventSynchronize(ctx->stage_ev[i]);
      cudaEventDestroy(ctx->stage_ev[i]);
    }
    if (ctx->stage[i]) cudaFreeHost(ctx->stage[i]);
  }
  if (ctx->ws_owned) cudaFree(ctx->ws);
  cudaFree(ctx->d_error);
  cudaFree(ctx->d_status);
  delete ctx;
  return PIMDAL_OK;
}

extern "C" int pimdal_ctx_set_workspace(pimdal_ctx_t *ctx, void *ptr, size_t bytes) {
  if (!ctx) return PIMDAL_ERR_ARG;
  if (ptr && ((uintptr_t)ptr & 255u)) return PIMDAL_ERR_ARG;
  if (ctx->ws_owned) cudaFree(ctx->ws);
  ctx->ws = ptr;
  ctx->ws_bytes = ptr ? bytes : 0;
  ctx->ws_owned = false;
  return PIMDAL_OK;
}

extern "C" int pimdal_ctx_sync_status(pimdal_ctx_t *ctx, pimdal_stream_t stream) {
  if (!ctx) return PIMDAL_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t word = 0;
  PD_CHECK_CUDA(cudaMemcpyAsync(&word, ctx->d_error, sizeof(word), cudaMemcpyDeviceToHost, s));
  PD_CHECK_CUDA(cudaStreamSynchronize(s));
  if (word) {
    PD_CHECK_CUDA(cudaMemsetAsync(ctx->d_error, 0, 256, s));
    PD_CHECK_CUDA(cudaStreamSynchronize(s));
  }
  if (word & PD_DEVERR_TIMEOUT) return PIMDAL_ERR_DEVICE_TIMEOUT;
  if (word & PD_DEVERR_TABLE_FULL) return PIMDAL_ERR_TABLE_FULL;
  if (word & PD_DEVERR_CAPACITY) return PIMDAL_ERR_CAPACITY;
  if (word & PD_DEVERR_ARG) return PIMDAL_ERR_ARG;
  return PIMDAL_OK;
}

extern "C" uint64_t pimdal_ctx_launch_count(const pimdal_ctx_t *ctx) {
  return ctx ? ctx->launches : 0;
}

void *pd_workspace(pimdal_ctx *ctx, size_t bytes, cudaStream_t stream, int *status) {
  *status = PIMDAL_OK;
  if (bytes == 0) return ctx->ws;
  if (ctx->ws && ctx->ws_bytes >= bytes) return ctx->ws;
  if (ctx->ws && !ctx->ws_owned) {
    *status = PIMDAL_ERR_WORKSPACE;
    return nullptr;
  }
  // Growing an owned workspace must not happen inside stream capture.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) == cudaSuccess &&
      cap != cudaStreamCaptureStatusNone) {
    *status = PIMDAL_ERR_WORKSPACE;
    return nullptr;
  }
  if (ctx->ws_owned) {
    cudaDeviceSynchronize();
    cudaFree(ctx->ws);
  }
  ctx->ws = nullptr;
  ctx->ws_bytes = 0;
  size_t grow = pd_align_up(bytes + bytes / 4, 1 << 20);
  if (cudaMalloc(&ctx->ws, grow) != cudaSuccess) {
    cudaGetLastError();
    ctx->ws = nullptr;
    ctx->ws_owned = false;
    *status = PIMDAL_ERR_OOM;
    return nullptr;
  }
  ctx->ws_bytes = grow;
  ctx->ws_owned = true;
  return ctx->ws;
}

uint32_t pd_next_epoch(pimdal_ctx *ctx, cudaStream_t stream, int *status) {
  *status = PIMDAL_OK;
  ctx->epoch = (ctx->epoch + 1) & 0xFFFFu;
  if (ctx->epoch == 0) {
    // Wrapped: stale words from 65535 launches ago could carry this epoch.
    if (cudaMemsetAsync(ctx->d_status, 0, sizeof(uint64_t) * PD_STATUS_WORDS, stream) !=
        cudaSuccess)
      *status = PIMDAL_ERR_CUDA;
    ctx->epoch = 1;
  }
  return ctx->epoch;
}

int pd_launch_status(pimdal_ctx *ctx) {
  (void)ctx;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PIMDAL_OK : PIMDAL_ERR_CUDA;
}
