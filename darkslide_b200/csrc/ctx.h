// The library context (dsgpu_ctx) and the helpers its entry points share:
// device guard, CUDA error mapping, grow-only scratch slots.
#pragma once
#include <cstdio>
#include <vector>

#include "internal.cuh"

enum Slot { S_IN = 0, S_IN2, S_OUT, S_OUT2, S_CFA, S_RGB, S_TMP, S_WORK, S_BATCH, S_COUNT };

struct ds_mark {
  int stage;
  cudaEvent_t a, b;
};

struct DsBatch;
void ds_batch_free(DsBatch* b);

struct dsgpu_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  void* slot[S_COUNT] = {};
  size_t slot_bytes[S_COUNT] = {};
  char last_error[256] = {};
  unsigned long long launches = 0;  // kernels this context has launched
  bool profiling = false;
  std::vector<ds_mark> marks;       // stage events recorded while profiling
  std::vector<cudaEvent_t> pool;    // idle events
  DsBatch* batch = nullptr;         // batched develop: descriptors, graph, autotune table
  cudaStream_t copy = nullptr;      // host-buffer calls: device-to-host copies overlapping compute
  std::vector<cudaEvent_t> band_ev; // one per band of a pipelined call
  // per-site black levels for the u16 entry points (dsgpu_set_black_pattern); bw == 0: none
  int black_bw = 0, black_bh = 0, black_x0 = 0, black_y0 = 0;
  float black_pat[DS_BLACK_MAX * DS_BLACK_MAX] = {};
};

// The u16 source of a call: the scalar black level, or the context's pattern.
inline ds_src_u16 u16_source(const dsgpu_ctx* ctx, const void* data, size_t pitch, float black,
                             const float white[3]) {
  ds_src_u16 s{static_cast<const uint16_t*>(data), pitch, black, {white[0], white[1], white[2]}};
  if (ctx->black_bw > 0) {
    s.bw = ctx->black_bw;
    s.bh = ctx->black_bh;
    s.bx0 = ctx->black_x0;
    s.by0 = ctx->black_y0;
    for (int i = 0; i < DS_BLACK_MAX * DS_BLACK_MAX; i++) s.bpat[i] = ctx->black_pat[i];
  }
  return s;
}

// Makes ctx->device current for the duration of a call and restores the
// caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

inline int map_cuda(dsgpu_ctx* ctx, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return DSGPU_OK;
  if (ctx) snprintf(ctx->last_error, sizeof(ctx->last_error), "%s: %s", where, cudaGetErrorString(e));
  cudaGetLastError();  // clear a non-sticky error
  return e == cudaErrorMemoryAllocation ? DSGPU_ERR_NOMEM : DSGPU_ERR_CUDA;
}

#define DS_TRY(expr)                                 \
  do {                                               \
    cudaError_t _e = (expr);                         \
    if (_e != cudaSuccess) return map_cuda(ctx, _e, #expr); \
  } while (0)

#define DS_CHECK(expr)          \
  do {                          \
    int _s = (expr);            \
    if (_s != DSGPU_OK) return _s; \
  } while (0)

// grow-only device scratch
inline int scratch(dsgpu_ctx* ctx, Slot s, size_t bytes, void** out) {
  if (bytes == 0) bytes = 16;
  if (ctx->slot_bytes[s] < bytes) {
    if (ctx->slot[s]) cudaFreeAsync(ctx->slot[s], ctx->stream);
    ctx->slot[s] = nullptr;
    ctx->slot_bytes[s] = 0;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, ctx->stream);
    if (e != cudaSuccess) return map_cuda(ctx, e, "cudaMallocAsync");
    ctx->slot[s] = p;
    ctx->slot_bytes[s] = bytes;
  }
  *out = ctx->slot[s];
  return DSGPU_OK;
}
