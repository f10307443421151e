// C ABI of libdsgpu: argument checks, context, scratch and host staging,
// and dispatch to the kernels. See include/dsgpu.h for the contract.
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "ctx.h"
#include "internal.cuh"
#include "scene.h"
#include "../../include/dsgpu_scene.h"

ds_scene ds_scene_make(const dsgpu_scene_desc* d);
cudaError_t ds_launch_scene(cudaStream_t st, const ds_scene& s, uint16_t* out);
cudaError_t ds_launch_scene_window(cudaStream_t st, const ds_scene& s, int x0, int y0, int cw, int ch,
                                   uint16_t* out);
void ds_scene_host(const ds_scene& s, int x0, int y0, int cw, int ch, uint16_t* out);
void ds_scene_truth(const ds_scene& s, int x0, int y0, int cw, int ch, float* out);
cudaError_t ds_measure_peaks(cudaStream_t st, int device, double* ffma_flops, double* ex2_per_s,
                             double* ffma2_flops);

cudaError_t ds_measure_mma_sync(cudaStream_t st, int device, double* flops);
struct DsCnn;
size_t ds_cnn_param_count();
cudaError_t ds_cnn_create(int max_batch, int crop, DsCnn** out);
void ds_cnn_destroy(DsCnn* net);
float* ds_cnn_param_ptr(DsCnn* net);
float* ds_cnn_grad_ptr(DsCnn* net);
float* ds_cnn_moment_ptr(DsCnn* net, int which);
long long* ds_cnn_step_ptr(DsCnn* net);
cudaError_t ds_cnn_gradients(DsCnn* net, cudaStream_t st, const float* rgb, const float* strength_map,
                             float strength, const float* tgt, int B, float* loss_sum_host);
cudaError_t ds_cnn_adam(DsCnn* net, cudaStream_t st, float lr);
void ds_cnn_set_clip(DsCnn* net, float clip);
void ds_cnn_set_loss(DsCnn* net, int relative);
void ds_cnn_set_marks(DsCnn* net, cudaEvent_t a, cudaEvent_t b);
cudaError_t ds_cnn_infer(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, float strength, float* out);
void ds_cnn_set_engine(DsCnn* net, int use_tc);
int ds_cnn_take_status(DsCnn* net, cudaStream_t st);
cudaError_t ds_cnn_denoise(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, float h_param, int search,
                           int patch, float tau, float strength_scale, float* out, unsigned char* flags_scratch,
                           unsigned* count_dev);
cudaError_t ds_cnn_reserve(DsCnn* net, int w, int h);
void ds_cnn_set_judge(DsCnn* net, float fraction, float limit, unsigned seed);
bool ds_cnn_judge_on(const DsCnn* net);
int ds_cnn_judge_tile(unsigned seed, float fraction, int t);
cudaError_t ds_cnn_reserve_judge(DsCnn* net, int w, int h, int patch);
cudaError_t ds_cnn_judge_reset(DsCnn* net, cudaStream_t st);
cudaError_t ds_cnn_judge_stats(DsCnn* net, cudaStream_t st, int* judged, int* failed, float* max_rms,
                               float* mean_rms);
int ds_cnn_halo_rows();
cudaError_t ds_cnn_denoise_band(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, int r0, int r1, int halo,
                                float h_param, int search, int patch, float tau, float strength_scale, float* out,
                                float* band_out, unsigned char* flags_scratch, unsigned* count_dev);


namespace {


// Stage timing (the analogue of the reference's Lap stage timer,
// pipeline/mod.rs:106-137): with profiling on, each stage of a call is
// bracketed by CUDA events on the context stream.
cudaEvent_t take_event(dsgpu_ctx* ctx) {
  cudaEvent_t e = nullptr;
  if (!ctx->pool.empty()) {
    e = ctx->pool.back();
    ctx->pool.pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

struct StageMark {
  dsgpu_ctx* ctx;
  int stage;
  cudaEvent_t a = nullptr;
  StageMark(dsgpu_ctx* c, int st) : ctx(c), stage(st) {
    if (ctx->profiling && (a = take_event(ctx))) cudaEventRecord(a, ctx->stream);
  }
  ~StageMark() {
    if (!a) return;
    cudaEvent_t b = take_event(ctx);
    if (!b) {
      ctx->pool.push_back(a);
      return;
    }
    cudaEventRecord(b, ctx->stream);
    ctx->marks.push_back({stage, a, b});
  }
};

// Profiling mark around the hidden conv layers of one CNN call (events
// recorded by the network's own driver).
struct HiddenMark {
  dsgpu_ctx* ctx;
  DsCnn* net;
  cudaEvent_t a = nullptr, b = nullptr;
  bool done = false;  // set once the call has been queued (both events recorded)
  HiddenMark(dsgpu_ctx* c, DsCnn* n) : ctx(c), net(n) {
    if (!ctx->profiling || !(a = take_event(ctx))) return;
    if (!(b = take_event(ctx))) {
      ctx->pool.push_back(a);
      a = nullptr;
      return;
    }
    ds_cnn_set_marks(net, a, b);
  }
  ~HiddenMark() {
    if (!a) return;
    ds_cnn_set_marks(net, nullptr, nullptr);
    if (done) {
      ctx->marks.push_back({DSGPU_STAGE_CNN_HIDDEN, a, b});
    } else {
      ctx->pool.push_back(a);
      ctx->pool.push_back(b);
    }
  }
};

int check_dims(int w, int h) {
  if (w < 0 || h < 0) return DSGPU_ERR_ARG;
  if (w > DSGPU_MAX_DIM || h > DSGPU_MAX_DIM) return DSGPU_ERR_SIZE;
  return DSGPU_OK;
}

int check_pat(const uint8_t* cfa, ds_pat* pat) {
  if (!cfa) return DSGPU_ERR_ARG;
  pat->packed = 0;
  for (int i = 0; i < 4; i++) {
    if (cfa[i] > 2) return DSGPU_ERR_CFA;
    pat->packed |= (uint32_t)cfa[i] << (8 * i);
  }
  return DSGPU_OK;
}

// Input staging: with DSGPU_HOST, copy host data into a scratch slot and
// return the device pointer; otherwise the pointer is used as is.
int stage_in(dsgpu_ctx* ctx, unsigned flags, Slot s, const void* p, size_t bytes, const void** dev) {
  if (!(flags & DSGPU_HOST)) {
    *dev = p;
    return DSGPU_OK;
  }
  void* d = nullptr;
  DS_CHECK(scratch(ctx, s, bytes, &d));
  StageMark mark(ctx, DSGPU_STAGE_COPY);
  if (bytes) DS_TRY(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
  *dev = d;
  return DSGPU_OK;
}

int stage_out_ptr(dsgpu_ctx* ctx, unsigned flags, Slot s, void* p, size_t bytes, void** dev) {
  if (!(flags & DSGPU_HOST)) {
    *dev = p;
    return DSGPU_OK;
  }
  return scratch(ctx, s, bytes, dev);
}

int finish(dsgpu_ctx* ctx, unsigned flags, void* host_dst, const void* dev_src, size_t bytes, void* host_dst2 = nullptr,
           const void* dev_src2 = nullptr, size_t bytes2 = 0) {
  if (flags & DSGPU_HOST) {
    StageMark mark(ctx, DSGPU_STAGE_COPY);
    if (host_dst && bytes) DS_TRY(cudaMemcpyAsync(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    if (host_dst2 && bytes2) DS_TRY(cudaMemcpyAsync(host_dst2, dev_src2, bytes2, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (flags & DSGPU_HOST) {
    DS_TRY(cudaStreamSynchronize(ctx->stream));
  } else if (!(flags & DSGPU_ASYNC)) {
    DS_TRY(cudaStreamSynchronize(ctx->stream));
  }
  return DSGPU_OK;
}

int nlm_args_ok(int channels, int search, int patch) {
  if (channels < 1 || channels > 4) return DSGPU_ERR_ARG;
  if (patch < 0 || patch > DSGPU_NLM_MAX_PATCH) return DSGPU_ERR_ARG;
  if (search > DSGPU_NLM_MAX_SEARCH) return DSGPU_ERR_ARG;
  return DSGPU_OK;
}

// NLM on device buffers; a negative search radius yields an empty offset set
// and therefore 0 / max(0, 1e-12) = 0 (enhance.rs:41, :71).
int run_nlm(dsgpu_ctx* ctx, const float* in, int w, int h, int channels, float h_param, int search, int patch,
            float* out, unsigned flags = 0) {
  const size_t n = (size_t)w * h * channels;
  if (n == 0) return DSGPU_OK;
  StageMark mark(ctx, DSGPU_STAGE_NLM);
  if (search < 0) {
    DS_TRY(cudaMemsetAsync(out, 0, n * sizeof(float), ctx->stream));
    return DSGPU_OK;
  }
  DS_TRY(ds_launch_nlm(ctx->stream, in, w, h, channels, h_param, search, patch, out,
                       (flags & DSGPU_FP16_STAGING) != 0));
  ctx->launches += 1;
  return DSGPU_OK;
}

// A pipelined host-buffer call queues copies into the caller's host buffers on
// the copy stream while kernels are still being launched. If a launch fails
// midway, the call must not return while those copies can still run: the
// caller may free or reuse its buffers as soon as the error comes back. This
// guard waits for both streams on every early return (and clears the sticky
// error state of a failed launch); the success path disarms it after its own
// synchronisation.
struct PipelineDrain {
  dsgpu_ctx* ctx;
  bool armed = true;
  explicit PipelineDrain(dsgpu_ctx* c) : ctx(c) {}
  ~PipelineDrain() {
    if (!armed) return;
    if (ctx->copy) cudaStreamSynchronize(ctx->copy);
    cudaStreamSynchronize(ctx->stream);
    cudaGetLastError();
  }
};

// Host-buffer develop, second half: NLM in bands of tile rows on the context
// stream, each band's rows copied to the host on the copy stream as soon as
// the band is done (so the 12 B/px result copy overlaps the next band's NLM);
// the clip plane is copied first. Returns when everything is in host memory.
int nlm_bands_to_host(dsgpu_ctx* ctx, const float* mid, int w, int h, float h_param, int search, int patch,
                      unsigned flags, const float* drgb, float* out_rgb, const float* dclip, float* out_clip) {
  constexpr int BANDS = 8;
  if (!ctx->copy) DS_TRY(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
  PipelineDrain drain_guard(ctx);
  while (ctx->band_ev.size() < BANDS + 1) {
    cudaEvent_t e;
    DS_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->band_ev.push_back(e);
  }
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const int bands = ty < BANDS ? ty : BANDS;
  cudaEvent_t ca = ctx->profiling ? take_event(ctx) : nullptr, cb = ca ? take_event(ctx) : nullptr;
  if (ca && !cb) {
    ctx->pool.push_back(ca);
    ca = nullptr;
  }
  DS_TRY(cudaEventRecord(ctx->band_ev[BANDS], ctx->stream));  // demosaic (and clip plane) done
  DS_TRY(cudaStreamWaitEvent(ctx->copy, ctx->band_ev[BANDS], 0));
  if (ca) DS_TRY(cudaEventRecord(ca, ctx->copy));
  if (out_clip)
    DS_TRY(cudaMemcpyAsync(out_clip, dclip, (size_t)w * h * sizeof(float), cudaMemcpyDeviceToHost, ctx->copy));
  {
    StageMark mark(ctx, DSGPU_STAGE_NLM);
    for (int b = 0; b < bands; b++) {
      const int t0 = (int)((long long)ty * b / bands), t1 = (int)((long long)ty * (b + 1) / bands);
      DS_TRY(ds_launch_nlm_rows(ctx->stream, mid, w, h, 3, h_param, search, patch, t0, t1, (float*)drgb,
                                (flags & DSGPU_FP16_STAGING) != 0));
      ctx->launches += 1;
      DS_TRY(cudaEventRecord(ctx->band_ev[b], ctx->stream));
      DS_TRY(cudaStreamWaitEvent(ctx->copy, ctx->band_ev[b], 0));
      const size_t r0 = (size_t)t0 * th, r1 = (size_t)t1 * th < (size_t)h ? (size_t)t1 * th : (size_t)h;
      const size_t row = (size_t)w * 3;
      DS_TRY(cudaMemcpyAsync(out_rgb + r0 * row, drgb + r0 * row, (r1 - r0) * row * sizeof(float),
                             cudaMemcpyDeviceToHost, ctx->copy));
    }
  }
  if (cb) {
    DS_TRY(cudaEventRecord(cb, ctx->copy));
    ctx->marks.push_back({DSGPU_STAGE_COPY, ca, cb});
  }
  DS_TRY(cudaStreamSynchronize(ctx->copy));
  drain_guard.armed = false;
  return DSGPU_OK;
}

// Host-buffer develop as a three-stage pipeline over row bands: the raw goes
// up in 8 row chunks on the copy stream; RCD runs in bands of 32-row tile
// rows on the context stream, each band waiting only for the chunks that
// hold its rows and its 10-row halo; NLM runs in 8 bands of tile rows, each
// after the RCD rows of its band and its S+P+1 halo; each finished NLM band
// goes back to the host on the copy stream while the next one computes.
// Every kernel is the one-frame kernel on a subset of its tile rows, so the
// output equals the device-buffer call's bit for bit.
int develop_pipelined(dsgpu_ctx* ctx, const uint16_t* raw, int w, int h, size_t pitch, ds_pat pat, float black,
                      const float white[3], const float mul[3], float h_param, int search, int patch, float* out_rgb,
                      float* out_clip, unsigned flags) {
  constexpr int CHUNKS = 8, BANDS = 8;
  const size_t n = (size_t)w * h;
  void *draw, *drgb, *mid, *dclip = nullptr;
  DS_CHECK(scratch(ctx, S_IN, ((size_t)(h - 1) * pitch + w) * sizeof(uint16_t), &draw));
  DS_CHECK(scratch(ctx, S_OUT, n * 3 * sizeof(float), &drgb));
  DS_CHECK(scratch(ctx, S_RGB, n * 3 * sizeof(float), &mid));
  if (out_clip) DS_CHECK(scratch(ctx, S_OUT2, n * sizeof(float), &dclip));
  if (!ctx->copy) DS_TRY(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
  PipelineDrain drain_guard(ctx);
  while (ctx->band_ev.size() < CHUNKS + BANDS + 1) {
    cudaEvent_t e;
    DS_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->band_ev.push_back(e);
  }
  cudaEvent_t* up_ev = ctx->band_ev.data();
  cudaEvent_t* band_ev = ctx->band_ev.data() + CHUNKS;
  cudaEvent_t start_ev = ctx->band_ev[CHUNKS + BANDS];
  cudaEvent_t ca = ctx->profiling ? take_event(ctx) : nullptr, cb = ca ? take_event(ctx) : nullptr;
  if (ca && !cb) {
    ctx->pool.push_back(ca);
    ca = nullptr;
  }
  // the copy stream starts after whatever the context stream already holds
  DS_TRY(cudaEventRecord(start_ev, ctx->stream));
  DS_TRY(cudaStreamWaitEvent(ctx->copy, start_ev, 0));
  if (ca) DS_TRY(cudaEventRecord(ca, ctx->copy));
  int chunk_end[CHUNKS];  // first raw row after chunk c
  for (int c = 0; c < CHUNKS; c++) {
    const int r0 = (int)((long long)h * c / CHUNKS), r1 = (int)((long long)h * (c + 1) / CHUNKS);
    chunk_end[c] = r1;
    if (r1 > r0)
      DS_TRY(cudaMemcpyAsync(static_cast<uint16_t*>(draw) + (size_t)r0 * pitch, raw + (size_t)r0 * pitch,
                             ((size_t)(r1 - 1 - r0) * pitch + w) * sizeof(uint16_t), cudaMemcpyHostToDevice,
                             ctx->copy));
    DS_TRY(cudaEventRecord(up_ev[c], ctx->copy));
  }
  const ds_src_u16 src = u16_source(ctx, draw, pitch, black, white);
  const int rcd_rows = (h + DS_RCD_TILE - 1) / DS_RCD_TILE;
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const int bands = ty < BANDS ? ty : BANDS;
  // band sizes shrink toward the end (weights 8,8,8,8,6,4,2,1), so that the
  // copy of the last band, which nothing overlaps, is small
  static const int wts[BANDS] = {8, 8, 8, 8, 6, 4, 2, 1};
  int cum[BANDS + 1] = {0};
  for (int b = 0; b < bands; b++) cum[b + 1] = cum[b] + (bands == BANDS ? wts[b] : 1);
  const int nlm_halo = search + patch + 1;
  int rcd_next = 0, chunks_waited = 0, tprev = 0;
  for (int b = 0; b < bands; b++) {
    const int t0 = tprev;
    int t1 = (int)((long long)ty * cum[b + 1] / cum[bands]);
    if (t1 <= t0) t1 = t0 + 1;  // every band holds at least one tile row
    if (b == bands - 1 || t1 > ty) t1 = ty;
    tprev = t1;
    if (t0 >= t1) continue;
    const int r1 = t1 * th < h ? t1 * th : h;  // output rows end of this band
    int need = (r1 + nlm_halo + DS_RCD_TILE - 1) / DS_RCD_TILE;  // RCD tile rows this band reads
    if (b == bands - 1 || need > rcd_rows) need = rcd_rows;
    if (need > rcd_next) {
      const int raw_end = need * DS_RCD_TILE + DS_RCD_HALO;  // raw rows that RCD band reads
      while (chunks_waited < CHUNKS && (chunks_waited == 0 || chunk_end[chunks_waited - 1] < raw_end)) {
        DS_TRY(cudaStreamWaitEvent(ctx->stream, up_ev[chunks_waited], 0));
        chunks_waited++;
      }
      DS_TRY(ds_launch_rcd_u16_rows(ctx->stream, src, w, h, pat, mul, (float*)mid, (float*)dclip, rcd_next, need));
      ctx->launches += 1;
      rcd_next = need;
    }
    DS_TRY(ds_launch_nlm_rows(ctx->stream, (const float*)mid, w, h, 3, h_param, search, patch, t0, t1,
                              (float*)drgb, (flags & DSGPU_FP16_STAGING) != 0));
    ctx->launches += 1;
    DS_TRY(cudaEventRecord(band_ev[b], ctx->stream));
    DS_TRY(cudaStreamWaitEvent(ctx->copy, band_ev[b], 0));
    const size_t r0 = (size_t)t0 * th, row = (size_t)w * 3;
    DS_TRY(cudaMemcpyAsync(out_rgb + r0 * row, static_cast<float*>(drgb) + r0 * row,
                           ((size_t)r1 - r0) * row * sizeof(float), cudaMemcpyDeviceToHost, ctx->copy));
  }
  if (out_clip)  // every RCD band is done before the last NLM band's event
    DS_TRY(cudaMemcpyAsync(out_clip, dclip, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->copy));
  if (cb) {
    DS_TRY(cudaEventRecord(cb, ctx->copy));
    ctx->marks.push_back({DSGPU_STAGE_COPY, ca, cb});
  }
  DS_TRY(cudaStreamSynchronize(ctx->copy));
  drain_guard.armed = false;
  return DSGPU_OK;
}

}  // namespace

extern "C" {

const char* dsgpu_strerror(int status) {
  switch (status) {
    case DSGPU_OK: return "ok";
    case DSGPU_ERR_ARG: return "invalid argument";
    case DSGPU_ERR_CFA: return "invalid CFA pattern";
    case DSGPU_ERR_SIZE: return "image too large";
    case DSGPU_ERR_NOMEM: return "out of memory";
    case DSGPU_ERR_CUDA: return "CUDA error";
    case DSGPU_ERR_NODEV: return "no usable sm_100 device";
    case DSGPU_ERR_TIMEOUT: return "device wait timed out";
    case DSGPU_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

int dsgpu_abi_version(void) { return DSGPU_ABI_VERSION; }

int dsgpu_create(int device, dsgpu_ctx** out) {
  if (!out) return DSGPU_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return DSGPU_ERR_NODEV;
  }
  if (device < 0 || device >= n) return DSGPU_ERR_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return DSGPU_ERR_NODEV;
  DeviceGuard g(device);
  if (!g.ok) return DSGPU_ERR_NODEV;
  dsgpu_ctx* ctx = new (std::nothrow) dsgpu_ctx();
  if (!ctx) return DSGPU_ERR_NOMEM;
  ctx->device = device;
  if (cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return DSGPU_ERR_CUDA;
  }
  ctx->stream = ctx->own;
  *out = ctx;
  return DSGPU_OK;
}

int dsgpu_destroy(dsgpu_ctx* ctx) {
  if (!ctx) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (int i = 0; i < S_COUNT; i++)
    if (ctx->slot[i]) cudaFreeAsync(ctx->slot[i], ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  for (auto& m : ctx->marks) {
    cudaEventDestroy(m.a);
    cudaEventDestroy(m.b);
  }
  for (auto e : ctx->pool) cudaEventDestroy(e);
  ds_batch_free(ctx->batch);
  for (auto e : ctx->band_ev) cudaEventDestroy(e);
  if (ctx->copy) cudaStreamDestroy(ctx->copy);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
  return DSGPU_OK;
}

int dsgpu_set_stream(dsgpu_ctx* ctx, void* stream) {
  if (!ctx) return DSGPU_ERR_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  return DSGPU_OK;
}

void* dsgpu_get_stream(dsgpu_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int dsgpu_synchronize(dsgpu_ctx* ctx) {
  if (!ctx) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  return DSGPU_OK;
}

int dsgpu_trim(dsgpu_ctx* ctx) {
  if (!ctx) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  for (int i = 0; i < S_COUNT; i++) {
    if (ctx->slot[i]) cudaFreeAsync(ctx->slot[i], ctx->stream);
    ctx->slot[i] = nullptr;
    ctx->slot_bytes[i] = 0;
  }
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  return DSGPU_OK;
}

const char* dsgpu_last_error(dsgpu_ctx* ctx) { return ctx ? ctx->last_error : "no context"; }

unsigned long long dsgpu_launch_count(dsgpu_ctx* ctx) { return ctx ? ctx->launches : 0ull; }

int dsgpu_profile(dsgpu_ctx* ctx, int enable) {
  if (!ctx) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  for (auto& m : ctx->marks) {
    ctx->pool.push_back(m.a);
    ctx->pool.push_back(m.b);
  }
  ctx->marks.clear();
  ctx->profiling = enable != 0;
  return DSGPU_OK;
}

int dsgpu_stage_ms(dsgpu_ctx* ctx, int stage, double* total_ms, int* count) {
  if (!ctx || !total_ms) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  double t = 0.0;
  int n = 0;
  for (auto& m : ctx->marks) {
    if (m.stage != stage) continue;
    float ms = 0.f;
    DS_TRY(cudaEventElapsedTime(&ms, m.a, m.b));
    t += ms;
    n++;
  }
  *total_ms = t;
  if (count) *count = n;
  return DSGPU_OK;
}

int dsgpu_measure_peaks(dsgpu_ctx* ctx, double* ffma_flops, double* ex2_per_s, double* ffma2_flops) {
  if (!ctx || !ffma_flops || !ex2_per_s) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  double f2 = 0.0;
  DS_TRY(ds_measure_peaks(ctx->stream, ctx->device, ffma_flops, ex2_per_s, &f2));
  if (ffma2_flops) *ffma2_flops = f2;
  ctx->launches += 6;
  return DSGPU_OK;
}

int dsgpu_measure_mma_sync(dsgpu_ctx* ctx, double* bf16_flops_per_s) {
  if (!ctx || !bf16_flops_per_s) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DS_TRY(ds_measure_mma_sync(ctx->stream, ctx->device, bf16_flops_per_s));
  ctx->launches += 2;
  return DSGPU_OK;
}

int dsgpu_set_black_pattern(dsgpu_ctx* ctx, const float* levels, int bw, int bh, int origin_x, int origin_y) {
  if (!ctx) return DSGPU_ERR_ARG;
  if (bw == 0 && bh == 0) {
    ctx->black_bw = ctx->black_bh = 0;
    return DSGPU_OK;
  }
  if (!levels || bw < 1 || bh < 1 || bw > DS_BLACK_MAX || bh > DS_BLACK_MAX || origin_x < 0 || origin_y < 0)
    return DSGPU_ERR_ARG;
  for (int i = 0; i < bw * bh; i++)
    if (!(levels[i] == levels[i])) return DSGPU_ERR_ARG;  // NaN
  ctx->black_bw = bw;
  ctx->black_bh = bh;
  ctx->black_x0 = origin_x % bw;
  ctx->black_y0 = origin_y % bh;
  for (int i = 0; i < DS_BLACK_MAX * DS_BLACK_MAX; i++) ctx->black_pat[i] = i < bw * bh ? levels[i] : 0.f;
  return DSGPU_OK;
}

int dsgpu_normalize_u16(dsgpu_ctx* ctx, const uint16_t* raw, int w, int h, size_t pitch, const uint8_t cfa[4],
                        float black, const float white[3], float* out, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(cfa, &pat));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!raw || !out || !white || pitch < (size_t)w) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, raw, ((size_t)(h - 1) * pitch + w) * sizeof(uint16_t), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, n * sizeof(float), &dout));
  DS_TRY(ds_launch_normalize_src(ctx->stream, u16_source(ctx, din, pitch, black, white), w, h, pat, (float*)dout));
  ctx->launches += 1;
  return finish(ctx, flags, out, dout, n * sizeof(float));
}

int dsgpu_clip_plane(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, float* out, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!cfa_data || !out) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, cfa_data, n * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, n * sizeof(float), &dout));
  DS_TRY(ds_launch_clip_plane(ctx->stream, (const float*)din, w, h, (float*)dout));
  ctx->launches += 1;
  return finish(ctx, flags, out, dout, n * sizeof(float));
}

int dsgpu_mhc(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, const uint8_t cfa[4], const float mul[3],
              float* out_rgb, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(cfa, &pat));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!cfa_data || !out_rgb || !mul) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, cfa_data, n * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &dout));
  DS_TRY(ds_launch_mhc(ctx->stream, (const float*)din, w, h, pat, mul, (float*)dout));
  ctx->launches += 1;
  return finish(ctx, flags, out_rgb, dout, n * 3 * sizeof(float));
}

// rcd_bayer (demosaic.rs:147-151): MHC below 16 pixels in either direction.
static int rcd_dev(dsgpu_ctx* ctx, const float* din, int w, int h, ds_pat pat, const float mul[3], float* drgb,
                   float* dclip) {
  StageMark mark(ctx, DSGPU_STAGE_DEMOSAIC);
  if (w < 16 || h < 16) {
    DS_TRY(ds_launch_mhc(ctx->stream, din, w, h, pat, mul, drgb));
    ctx->launches += 1;
    if (dclip) DS_TRY(ds_launch_clip_plane(ctx->stream, din, w, h, dclip));
    if (dclip) ctx->launches += 1;
    return DSGPU_OK;
  }
  DS_TRY(ds_launch_rcd_f32(ctx->stream, ds_src_f32{din, w}, w, h, pat, mul, drgb, dclip));
  ctx->launches += 1;
  return DSGPU_OK;
}

int dsgpu_rcd(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, const uint8_t cfa[4], const float mul[3],
              float* out_rgb, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(cfa, &pat));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!cfa_data || !out_rgb || !mul) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, cfa_data, n * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &dout));
  DS_CHECK(rcd_dev(ctx, (const float*)din, w, h, pat, mul, (float*)dout, nullptr));
  return finish(ctx, flags, out_rgb, dout, n * 3 * sizeof(float));
}

int dsgpu_demosaic(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, const uint8_t cfa[4], const float mul[3],
                   int quality, float* out_rgb, float* out_clip, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(cfa, &pat));
  if (quality != DSGPU_QUALITY_FULL && quality != DSGPU_QUALITY_DRAFT) return DSGPU_ERR_ARG;
  const size_t n = (size_t)w * h;
  const size_t on = quality == DSGPU_QUALITY_FULL ? n : (size_t)(w / 2) * (h / 2);
  if (n == 0) return DSGPU_OK;
  if (!cfa_data || !out_rgb || !mul) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void *drgb, *dclip = nullptr;
  DS_CHECK(stage_in(ctx, flags, S_IN, cfa_data, n * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, on * 3 * sizeof(float), &drgb));
  if (out_clip) DS_CHECK(stage_out_ptr(ctx, flags, S_OUT2, out_clip, on * sizeof(float), &dclip));
  if (quality == DSGPU_QUALITY_FULL) {
    DS_CHECK(rcd_dev(ctx, (const float*)din, w, h, pat, mul, (float*)drgb, (float*)dclip));
  } else {
    DS_TRY(ds_launch_superpixel(ctx->stream, (const float*)din, w, h, pat, mul, (float*)drgb, (float*)dclip));
    ctx->launches += 1;
  }
  return finish(ctx, flags, out_rgb, drgb, on * 3 * sizeof(float), out_clip, dclip, on * sizeof(float));
}

int dsgpu_box_blur(dsgpu_ctx* ctx, const float* in, int w, int h, int r, float* out, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  if (r < 0) return DSGPU_ERR_ARG;
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!in || !out) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  void* tmp;
  DS_CHECK(stage_in(ctx, flags, S_IN, in, n * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, n * sizeof(float), &dout));
  if (r == 0) {  // image.rs:270-272: a copy
    DS_TRY(cudaMemcpyAsync(dout, din, n * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    DS_CHECK(scratch(ctx, S_TMP, n * sizeof(float), &tmp));
    DS_TRY(ds_launch_box_blur(ctx->stream, (const float*)din, w, h, r, (float*)tmp, (float*)dout));
    ctx->launches += 2;
  }
  return finish(ctx, flags, out, dout, n * sizeof(float));
}

int dsgpu_nlm(dsgpu_ctx* ctx, const float* in, int w, int h, int channels, float h_param, int search, int patch,
              float* out, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  DS_CHECK(nlm_args_ok(channels, search, patch));
  const size_t n = (size_t)w * h * channels;
  if (n == 0) return DSGPU_OK;
  if (!in || !out) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, in, n * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, n * sizeof(float), &dout));
  DS_CHECK(run_nlm(ctx, (const float*)din, w, h, channels, h_param, search, patch, (float*)dout, flags));
  return finish(ctx, flags, out, dout, n * sizeof(float));
}

int dsgpu_develop_u16(dsgpu_ctx* ctx, const uint16_t* raw, int w, int h, size_t pitch, const uint8_t cfa[4],
                      float black, const float white[3], const float mul[3], float h_param, int search, int patch,
                      float* out_rgb, float* out_clip, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(cfa, &pat));
  DS_CHECK(nlm_args_ok(3, search, patch));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!raw || !out_rgb || !white || !mul || pitch < (size_t)w) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  if ((flags & DSGPU_HOST) && !(flags & DSGPU_HIGHLIGHTS) && w >= 16 && h >= 16 && search > 0)
    return develop_pipelined(ctx, raw, w, h, pitch, pat, black, white, mul, h_param, search, patch, out_rgb,
                             out_clip, flags);
  const void* din;
  void *drgb, *dclip = nullptr, *mid;
  DS_CHECK(stage_in(ctx, flags, S_IN, raw, ((size_t)(h - 1) * pitch + w) * sizeof(uint16_t), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &drgb));
  if (out_clip) DS_CHECK(stage_out_ptr(ctx, flags, S_OUT2, out_clip, n * sizeof(float), &dclip));
  DS_CHECK(scratch(ctx, S_RGB, n * 3 * sizeof(float), &mid));
  const bool hl = (flags & DSGPU_HIGHLIGHTS) != 0;
  void* hl_work = nullptr;
  float* hl_clip = (float*)dclip;  // highlights need the clip plane even when the caller does not
  if (hl) {
    const size_t hb = ds_highlights_scratch_bytes(w, h);
    DS_CHECK(scratch(ctx, S_WORK, hb + 64 + (dclip ? 0 : n * sizeof(float)), &hl_work));
    if (!hl_clip) hl_clip = reinterpret_cast<float*>(static_cast<char*>(hl_work) + hb + 64);
  }
  unsigned* hl_bits = hl ? reinterpret_cast<unsigned*>(static_cast<char*>(hl_work) + ds_highlights_scratch_bytes(w, h))
                         : nullptr;
  float* hl_rc = hl ? reinterpret_cast<float*>(hl_bits + 8) : nullptr;
  const ds_src_u16 src = u16_source(ctx, din, pitch, black, white);
  if (w < 16 || h < 16) {
    void* cfa_f;
    DS_CHECK(scratch(ctx, S_CFA, n * sizeof(float), &cfa_f));
    DS_TRY(ds_launch_normalize_src(ctx->stream, src, w, h, pat, (float*)cfa_f));
    ctx->launches += 1;
    DS_CHECK(rcd_dev(ctx, (const float*)cfa_f, w, h, pat, mul, (float*)mid, hl_clip));
  } else {
    StageMark mark(ctx, DSGPU_STAGE_DEMOSAIC);
    DS_TRY(ds_launch_rcd_u16(ctx->stream, src, w, h, pat, mul, (float*)mid, hl_clip));
    ctx->launches += 1;
  }
  if (hl) {  // Engine::base: reconstruct_highlights(img, clip, mul, cfa_clip_levels(cfa)) (pipeline/mod.rs:186-187)
    unsigned launches = 0;
    DS_TRY(ds_launch_clip_levels_u16(ctx->stream, src, w, h, pat, hl_bits, hl_rc));
    DS_TRY(ds_launch_highlights(ctx->stream, (float*)mid, hl_clip, w, h, mul, hl_rc, hl_work, &launches));
    ctx->launches += 2 + launches;
  }
  if ((flags & DSGPU_HOST) && search > 0)  // overlap the result's copy to the host with NLM
    return nlm_bands_to_host(ctx, (const float*)mid, w, h, h_param, search, patch, flags, (const float*)drgb,
                             out_rgb, (const float*)dclip, out_clip);
  DS_CHECK(run_nlm(ctx, (const float*)mid, w, h, 3, h_param, search, patch, (float*)drgb, flags));
  return finish(ctx, flags, out_rgb, drgb, n * 3 * sizeof(float), out_clip, dclip, n * sizeof(float));
}

// -------------------------------------------------------------- highlights

int dsgpu_cfa_clip_levels(dsgpu_ctx* ctx, const float* cfa, int w, int h, const uint8_t pat_codes[4], float* out3,
                          unsigned flags) {
  if (!ctx || !out3) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(pat_codes, &pat));
  const size_t n = (size_t)w * h;
  if (n == 0) {  // no samples: every maximum stays 0, below the 0.95 trust level
    out3[0] = out3[1] = out3[2] = FLT_MAX;
    return DSGPU_OK;
  }
  if (!cfa) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* work;
  DS_CHECK(stage_in(ctx, flags, S_IN, cfa, n * sizeof(float), &din));
  DS_CHECK(scratch(ctx, S_TMP, 64, &work));
  float* raw_clip = reinterpret_cast<float*>(static_cast<char*>(work) + 32);
  DS_TRY(ds_launch_clip_levels_f32(ctx->stream, (const float*)din, w, h, pat, (unsigned*)work, raw_clip));
  ctx->launches += 2;
  DS_TRY(cudaMemcpyAsync(out3, raw_clip, 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  return DSGPU_OK;
}

int dsgpu_reconstruct_highlights(dsgpu_ctx* ctx, float* rgb, const float* clip, int w, int h, const float mul[3],
                                 const float raw_clip[3], unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!rgb || !clip || !mul || !raw_clip) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void *dimg, *dclip;
  void* work;
  DS_CHECK(stage_in(ctx, flags, S_OUT, rgb, n * 3 * sizeof(float), &dimg));
  DS_CHECK(stage_in(ctx, flags, S_IN, clip, n * sizeof(float), &dclip));
  const size_t hb = ds_highlights_scratch_bytes(w, h);
  DS_CHECK(scratch(ctx, S_WORK, hb + 64, &work));
  float* rc = reinterpret_cast<float*>(static_cast<char*>(work) + hb);
  DS_TRY(cudaMemcpyAsync(rc, raw_clip, 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  unsigned launches = 0;
  DS_TRY(ds_launch_highlights(ctx->stream, (float*)dimg, (const float*)dclip, w, h, mul, rc, work, &launches));
  ctx->launches += launches;
  return finish(ctx, flags, rgb, dimg, n * 3 * sizeof(float));
}

// ------------------------------------------------------------- orientation

int dsgpu_apply_orientation(dsgpu_ctx* ctx, const float* in, int w, int h, int orientation, float* out,
                            unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  const size_t bytes = (size_t)w * h * 3 * sizeof(float);
  if (bytes == 0) return DSGPU_OK;
  if (!in || !out || in == out) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, in, bytes, &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, bytes, &dout));
  DS_TRY(ds_launch_orientation(ctx->stream, (const float*)din, w, h, orientation, (float*)dout));
  ctx->launches += 1;
  return finish(ctx, flags, out, dout, bytes);
}

// ----------------------------------------------------------------- denoise

int dsgpu_oklab_matrices(float* out27) {
  if (!out27) return DSGPU_ERR_ARG;
  ds_oklab_matrices(out27);
  return DSGPU_OK;
}

int dsgpu_estimate_noise(dsgpu_ctx* ctx, const float* plane, int w, int h, float* sigma, unsigned flags) {
  if (!ctx || !sigma) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  const size_t n = (size_t)w * h;
  if (n == 0) {  // enhance.rs:25-27
    *sigma = 0.0f;
    return DSGPU_OK;
  }
  if (!plane) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* work;
  DS_CHECK(stage_in(ctx, flags, S_IN, plane, n * sizeof(float), &din));
  DS_CHECK(scratch(ctx, S_WORK, ds_noise_scratch_bytes(w, h) + 8 * sizeof(float), &work));
  float* out3 = static_cast<float*>(work) + ds_noise_scratch_bytes(w, h) / sizeof(float);
  DS_TRY(ds_launch_estimate_noise(ctx->stream, (const float*)din, w, h, 0.0f, work, out3));
  ctx->launches += 2;
  float host4[4];
  DS_TRY(cudaMemcpyAsync(host4, out3, 4 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  *sigma = host4[3];  // without denoise's 1e-4 floor (enhance.rs:82)
  return DSGPU_OK;
}

int dsgpu_guided_filter(dsgpu_ctx* ctx, const float* I, const float* p, int w, int h, int r, float eps, float* out,
                        unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  if (r < 0) return DSGPU_ERR_ARG;
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!I || !p || !out) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void *dI, *dp;
  void *dout, *work;
  DS_CHECK(stage_in(ctx, flags, S_IN, I, n * sizeof(float), &dI));
  DS_CHECK(stage_in(ctx, flags, S_IN2, p, n * sizeof(float), &dp));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, n * sizeof(float), &dout));
  DS_CHECK(scratch(ctx, S_WORK, 9 * n * sizeof(float), &work));
  float* ws = static_cast<float*>(work);
  DS_TRY(ds_launch_guide_means(ctx->stream, (const float*)dI, w, h, r, ws, ws + n, ws + 8 * n, ws + 2 * n));
  DS_TRY(ds_launch_guided_filter(ctx->stream, (const float*)dI, (const float*)dp, w, h, r, nullptr, eps,
                                 (float*)dout, ws + 2 * n, ws, ws + n));
  ctx->launches += 5 + 11;
  return finish(ctx, flags, out, dout, n * sizeof(float));
}

int dsgpu_denoise(dsgpu_ctx* ctx, const float* in_rgb, int w, int h, float amount, float* out_rgb, unsigned flags) {
  if (!ctx) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!in_rgb || !out_rgb) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void *dout, *work;
  DS_CHECK(stage_in(ctx, flags, S_IN, in_rgb, n * 3 * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &dout));
  DS_CHECK(scratch(ctx, S_WORK, ds_denoise_scratch_bytes(w, h), &work));
  unsigned nl = 0;
  {
    StageMark mark(ctx, DSGPU_STAGE_NLM);
    DS_TRY(ds_launch_denoise(ctx->stream, (const float*)din, w, h, amount, work, (float*)dout, nullptr, &nl));
  }
  ctx->launches += nl;
  return finish(ctx, flags, out_rgb, dout, n * 3 * sizeof(float));
}

// --------------------------------------------------------------------- CNN

struct dsgpu_cnn {
  DsCnn* net = nullptr;
  int max_batch = 0, crop = 0;
};

int dsgpu_cnn_param_count(void) { return (int)ds_cnn_param_count(); }

int dsgpu_cnn_create(dsgpu_ctx* ctx, int max_batch, int crop, dsgpu_cnn** out) {
  if (!ctx || !out || max_batch < 0 || crop < 0 || crop > 4096 || (max_batch > 0 && crop < 1)) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  dsgpu_cnn* c = new (std::nothrow) dsgpu_cnn();
  if (!c) return DSGPU_ERR_NOMEM;
  cudaError_t e = ds_cnn_create(max_batch, crop, &c->net);
  if (e != cudaSuccess) {
    delete c;
    return map_cuda(ctx, e, "ds_cnn_create");
  }
  c->max_batch = max_batch;
  c->crop = crop;
  *out = c;
  return DSGPU_OK;
}

int dsgpu_cnn_destroy(dsgpu_ctx* ctx, dsgpu_cnn* c) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ds_cnn_destroy(c->net);
  delete c;
  return DSGPU_OK;
}

// which: 0 parameters, 1 Adam first moment, 2 Adam second moment
int dsgpu_cnn_state(dsgpu_ctx* ctx, dsgpu_cnn* c, int which, float* buf, int set, long long* step, unsigned flags) {
  if (!ctx || !c || which < 0 || which > 2) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  float* dev = which == 0 ? ds_cnn_param_ptr(c->net) : ds_cnn_moment_ptr(c->net, which - 1);
  const size_t bytes = ds_cnn_param_count() * sizeof(float);
  if (buf) {
    const cudaMemcpyKind k = (flags & DSGPU_HOST) ? (set ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost)
                                                  : cudaMemcpyDeviceToDevice;
    DS_TRY(cudaMemcpyAsync(set ? (void*)dev : (void*)buf, set ? (const void*)buf : (const void*)dev, bytes, k,
                           ctx->stream));
  }
  if (step) {
    if (set) *ds_cnn_step_ptr(c->net) = *step;
    else *step = *ds_cnn_step_ptr(c->net);
  }
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  return DSGPU_OK;
}

static int cnn_batch_args(dsgpu_cnn* c, const float* rgb, const float* tgt, int batch) {
  if (!rgb || !tgt || batch < 1 || batch > c->max_batch) return DSGPU_ERR_ARG;
  return DSGPU_OK;
}

int dsgpu_cnn_gradients(dsgpu_ctx* ctx, dsgpu_cnn* c, const float* rgb, const float* strength_map, float strength,
                        const float* target, int batch, float* grads, float* loss_sum, unsigned flags) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  DS_CHECK(cnn_batch_args(c, rgb, target, batch));
  if (flags & DSGPU_HOST) return DSGPU_ERR_ARG;  // device batches only
  DeviceGuard g(ctx->device);
  float loss = 0.f;
  DS_TRY(ds_cnn_gradients(c->net, ctx->stream, rgb, strength_map, strength, target, batch, &loss));
  if (loss_sum) *loss_sum = loss;
  if (grads)
    DS_TRY(cudaMemcpyAsync(grads, ds_cnn_grad_ptr(c->net), ds_cnn_param_count() * sizeof(float),
                           cudaMemcpyDeviceToDevice, ctx->stream));
  DS_TRY(cudaStreamSynchronize(ctx->stream));
  return ds_cnn_take_status(c->net, ctx->stream);  // a tensor-core kernel's bounded wait may have given up
}

int dsgpu_cnn_train_step(dsgpu_ctx* ctx, dsgpu_cnn* c, const float* rgb, const float* strength_map, float strength,
                         const float* target, int batch, float lr, float* loss_sum) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  DS_CHECK(cnn_batch_args(c, rgb, target, batch));
  DeviceGuard g(ctx->device);
  float loss = 0.f;
  DS_TRY(ds_cnn_gradients(c->net, ctx->stream, rgb, strength_map, strength, target, batch, loss_sum ? &loss : nullptr));
  DS_TRY(ds_cnn_adam(c->net, ctx->stream, lr));
  if (loss_sum) *loss_sum = loss;
  // a tensor-core kernel's bounded wait may have given up (checked when the
  // loss is read back, which synchronises anyway)
  return loss_sum ? ds_cnn_take_status(c->net, ctx->stream) : DSGPU_OK;
}

int dsgpu_cnn_set_clip(dsgpu_ctx* ctx, dsgpu_cnn* c, float max_norm) {
  if (!ctx || !c || !(max_norm >= 0.f)) return DSGPU_ERR_ARG;
  ds_cnn_set_clip(c->net, max_norm);
  return DSGPU_OK;
}

int dsgpu_cnn_set_loss(dsgpu_ctx* ctx, dsgpu_cnn* c, int relative) {
  if (!ctx || !c || relative < 0 || relative > 1) return DSGPU_ERR_ARG;
  ds_cnn_set_loss(c->net, relative);
  return DSGPU_OK;
}

int dsgpu_cnn_infer(dsgpu_ctx* ctx, dsgpu_cnn* c, const float* in_rgb, int w, int h, float strength, float* out_rgb,
                    unsigned flags) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!in_rgb || !out_rgb) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  DS_CHECK(stage_in(ctx, flags, S_IN, in_rgb, n * 3 * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &dout));
  {
    StageMark mark(ctx, DSGPU_STAGE_CNN);
    HiddenMark hidden(ctx, c->net);
    DS_TRY(ds_cnn_infer(c->net, ctx->stream, (const float*)din, w, h, strength, (float*)dout));
    hidden.done = true;
  }
  ctx->launches += 1 + 8;  // input packing + 8 conv layers
  DS_CHECK(finish(ctx, flags, out_rgb, dout, n * 3 * sizeof(float)));
  return (flags & DSGPU_ASYNC) ? DSGPU_OK : ds_cnn_take_status(c->net, ctx->stream);
}

int dsgpu_cnn_set_engine(dsgpu_ctx* ctx, dsgpu_cnn* c, int tensor_core_gen5) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  ds_cnn_set_engine(c->net, tensor_core_gen5);
  return DSGPU_OK;
}

int dsgpu_cnn_set_judge(dsgpu_ctx* ctx, dsgpu_cnn* c, float fraction, float limit, unsigned seed) {
  if (!ctx || !c || !(fraction >= 0.f && fraction <= 1.f) || !(limit >= 0.f)) return DSGPU_ERR_ARG;
  ds_cnn_set_judge(c->net, fraction, limit, seed);
  return DSGPU_OK;
}

int dsgpu_cnn_judge_stats(dsgpu_ctx* ctx, dsgpu_cnn* c, int* judged, int* failed, float* max_rms_over_sigma,
                          float* rms_over_sigma) {
  if (!ctx || !c || !judged || !failed || !max_rms_over_sigma || !rms_over_sigma) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DS_TRY(ds_cnn_judge_stats(c->net, ctx->stream, judged, failed, max_rms_over_sigma, rms_over_sigma));
  return DSGPU_OK;
}

int dsgpu_cnn_judge_tile(unsigned seed, float fraction, int tile_index) {
  if (tile_index < 0 || !(fraction >= 0.f && fraction <= 1.f)) return DSGPU_ERR_ARG;
  return ds_cnn_judge_tile(seed, fraction, tile_index);
}

// Scratch for the fallback: the tile flags (one byte per NLM tile) + u32 count
static int fallback_scratch(dsgpu_ctx* ctx, int w, int h, int patch, unsigned char** flags, unsigned** count) {
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const size_t nflags = ((size_t)tx * ty + 15) & ~(size_t)15;
  void* p;
  DS_CHECK(scratch(ctx, S_TMP, nflags + 16, &p));
  *flags = static_cast<unsigned char*>(p);
  *count = reinterpret_cast<unsigned*>(*flags + nflags);
  return DSGPU_OK;
}

int dsgpu_cnn_denoise(dsgpu_ctx* ctx, dsgpu_cnn* c, const float* in_rgb, int w, int h, float h_param, int search,
                      int patch, float tau, float* out_rgb, int* fallback_tiles, unsigned flags) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  DS_CHECK(nlm_args_ok(3, search, patch));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!in_rgb || !out_rgb || search < 1) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  const void* din;
  void* dout;
  unsigned char* fl;
  unsigned* cnt;
  DS_CHECK(stage_in(ctx, flags, S_IN, in_rgb, n * 3 * sizeof(float), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &dout));
  DS_CHECK(fallback_scratch(ctx, w, h, patch, &fl, &cnt));
  {
    StageMark mark(ctx, DSGPU_STAGE_CNN);
    HiddenMark hidden(ctx, c->net);
    DS_TRY(ds_cnn_denoise(c->net, ctx->stream, (const float*)din, w, h, h_param, search, patch, tau,
                          DSGPU_CNN_STRENGTH_SCALE, (float*)dout, fl, cnt));
    hidden.done = true;
  }
  ctx->launches += 1 + 8 + (tau > 0.f ? 2 : 0) + (ds_cnn_judge_on(c->net) ? 3 : 0);
  if (!(flags & DSGPU_ASYNC)) DS_CHECK(ds_cnn_take_status(c->net, ctx->stream));
  if (fallback_tiles) {
    unsigned hc = 0;
    if (tau > 0.f) {
      DS_TRY(cudaMemcpyAsync(&hc, cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
      DS_TRY(cudaStreamSynchronize(ctx->stream));
    }
    *fallback_tiles = (int)hc;
  }
  return finish(ctx, flags, out_rgb, dout, n * 3 * sizeof(float));
}

// Host-buffer learned develop as a three-stage pipeline over row bands, like
// develop_pipelined: the raw goes up in 8 row chunks on the copy stream; RCD
// runs in bands of its tile rows on the context stream, each waiting only for
// the chunks it reads; the network runs in 5 bands of NLM tile rows, each on
// its rows plus an 18-row halo above and below (the 8 dilated 3x3 layers reach
// 1+2+3+4+3+2+1+1 = 17 rows, the input's 3x3 local mean one more), so that
// the band's own rows come out as the whole-frame network computes them;
// the residual check and the NLM fallback follow on the band's tiles; each
// finished band goes back to the host on the copy stream while the next one
// computes. Fewer bands than the NLM pipeline: every band boundary costs 36
// rows of network work, and the copies (53 GB/s) keep up with larger bands.
static int develop_cnn_pipelined(dsgpu_ctx* ctx, DsCnn* net, const uint16_t* raw, int w, int h, size_t pitch,
                                 ds_pat pat, float black, const float white[3], const float mul[3], float h_param,
                                 int search, int patch, float tau, float* out_rgb, float* out_clip) {
  constexpr int CHUNKS = 8, BANDS = 5;
  const int halo = ds_cnn_halo_rows();  // 18 for dilations 1,2,3,4,3,2,1,1
  const size_t n = (size_t)w * h, row = (size_t)w * 3;
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const int bands = ty < BANDS ? ty : BANDS;
  // band sizes shrink toward the end (weights 8,8,8,4,1), so that the copy of
  // the last band, which nothing overlaps, is small
  static const int wts[BANDS] = {8, 8, 8, 4, 1};
  int cum[BANDS + 1] = {0};
  for (int b = 0; b < bands; b++) cum[b + 1] = cum[b] + (bands == BANDS ? wts[b] : 1);
  int bt[BANDS + 1] = {0};  // tile row where band b starts
  int max_rows = 0;
  for (int b = 0; b < bands; b++) {
    int t1 = (int)((long long)ty * cum[b + 1] / cum[bands]);
    if (t1 <= bt[b]) t1 = bt[b] + 1;  // every band holds at least one tile row
    if (b == bands - 1 || t1 > ty) t1 = ty;
    bt[b + 1] = t1 > bt[b] ? t1 : bt[b];
    const int r0 = bt[b] * th, r1 = bt[b + 1] * th < h ? bt[b + 1] * th : h;
    const int a0 = r0 - halo > 0 ? r0 - halo : 0, a1 = r1 + halo < h ? r1 + halo : h;
    if (a1 - a0 > max_rows) max_rows = a1 - a0;
  }
  void *draw, *drgb, *mid, *band, *dclip = nullptr;
  unsigned char* fl;
  unsigned* cnt;
  DS_CHECK(scratch(ctx, S_IN, ((size_t)(h - 1) * pitch + w) * sizeof(uint16_t), &draw));
  DS_CHECK(scratch(ctx, S_OUT, n * 3 * sizeof(float), &drgb));
  DS_CHECK(scratch(ctx, S_RGB, n * 3 * sizeof(float), &mid));
  DS_CHECK(scratch(ctx, S_WORK, (size_t)max_rows * row * sizeof(float), &band));
  if (out_clip) DS_CHECK(scratch(ctx, S_OUT2, n * sizeof(float), &dclip));
  DS_CHECK(fallback_scratch(ctx, w, h, patch, &fl, &cnt));
  DS_TRY(ds_cnn_reserve(net, w, max_rows));
  DS_TRY(ds_cnn_reserve_judge(net, w, h, patch));
  if (!ctx->copy) DS_TRY(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
  PipelineDrain drain_guard(ctx);
  while (ctx->band_ev.size() < CHUNKS + BANDS + 1) {
    cudaEvent_t e;
    DS_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->band_ev.push_back(e);
  }
  cudaEvent_t* up_ev = ctx->band_ev.data();
  cudaEvent_t* band_ev = ctx->band_ev.data() + CHUNKS;
  cudaEvent_t start_ev = ctx->band_ev[CHUNKS + BANDS];
  cudaEvent_t ca = ctx->profiling ? take_event(ctx) : nullptr, cb = ca ? take_event(ctx) : nullptr;
  if (ca && !cb) {
    ctx->pool.push_back(ca);
    ca = nullptr;
  }
  DS_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned), ctx->stream));
  if (ds_cnn_judge_on(net)) DS_TRY(ds_cnn_judge_reset(net, ctx->stream));
  // the copy stream starts after whatever the context stream already holds
  DS_TRY(cudaEventRecord(start_ev, ctx->stream));
  DS_TRY(cudaStreamWaitEvent(ctx->copy, start_ev, 0));
  if (ca) DS_TRY(cudaEventRecord(ca, ctx->copy));
  int chunk_end[CHUNKS];  // first raw row after chunk c
  for (int c = 0; c < CHUNKS; c++) {
    const int r0 = (int)((long long)h * c / CHUNKS), r1 = (int)((long long)h * (c + 1) / CHUNKS);
    chunk_end[c] = r1;
    if (r1 > r0)
      DS_TRY(cudaMemcpyAsync(static_cast<uint16_t*>(draw) + (size_t)r0 * pitch, raw + (size_t)r0 * pitch,
                             ((size_t)(r1 - 1 - r0) * pitch + w) * sizeof(uint16_t), cudaMemcpyHostToDevice,
                             ctx->copy));
    DS_TRY(cudaEventRecord(up_ev[c], ctx->copy));
  }
  const ds_src_u16 src = u16_source(ctx, draw, pitch, black, white);
  const int rcd_rows = (h + DS_RCD_TILE - 1) / DS_RCD_TILE;
  const int reach = halo > search + patch + 1 ? halo : search + patch + 1;  // RCD rows a band reads past its end
  int rcd_next = 0, chunks_waited = 0;
  for (int b = 0; b < bands; b++) {
    if (bt[b] >= bt[b + 1]) continue;
    const int r0 = bt[b] * th, r1 = bt[b + 1] * th < h ? bt[b + 1] * th : h;
    int need = (r1 + reach + DS_RCD_TILE - 1) / DS_RCD_TILE;  // RCD tile rows this band reads
    if (b == bands - 1 || need > rcd_rows) need = rcd_rows;
    if (need > rcd_next) {
      const int raw_end = need * DS_RCD_TILE + DS_RCD_HALO;  // raw rows that RCD band reads
      while (chunks_waited < CHUNKS && (chunks_waited == 0 || chunk_end[chunks_waited - 1] < raw_end)) {
        DS_TRY(cudaStreamWaitEvent(ctx->stream, up_ev[chunks_waited], 0));
        chunks_waited++;
      }
      DS_TRY(ds_launch_rcd_u16_rows(ctx->stream, src, w, h, pat, mul, (float*)mid, (float*)dclip, rcd_next, need));
      ctx->launches += 1;
      rcd_next = need;
    }
    DS_TRY(ds_cnn_denoise_band(net, ctx->stream, (const float*)mid, w, h, r0, r1, halo, h_param, search, patch, tau,
                               DSGPU_CNN_STRENGTH_SCALE, (float*)drgb, (float*)band, fl, cnt));
    ctx->launches += 1 + 8 + (tau > 0.f ? 2 : 0) + (ds_cnn_judge_on(net) ? 3 : 0);
    DS_TRY(cudaEventRecord(band_ev[b], ctx->stream));
    DS_TRY(cudaStreamWaitEvent(ctx->copy, band_ev[b], 0));
    DS_TRY(cudaMemcpyAsync(out_rgb + (size_t)r0 * row, static_cast<float*>(drgb) + (size_t)r0 * row,
                           (size_t)(r1 - r0) * row * sizeof(float), cudaMemcpyDeviceToHost, ctx->copy));
  }
  if (out_clip)  // every RCD band is done before the last band's event
    DS_TRY(cudaMemcpyAsync(out_clip, dclip, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->copy));
  if (cb) {
    DS_TRY(cudaEventRecord(cb, ctx->copy));
    ctx->marks.push_back({DSGPU_STAGE_COPY, ca, cb});
  }
  DS_TRY(cudaStreamSynchronize(ctx->copy));
  drain_guard.armed = false;
  return ds_cnn_take_status(net, ctx->stream);
}

int dsgpu_develop_u16_cnn(dsgpu_ctx* ctx, dsgpu_cnn* c, const uint16_t* raw, int w, int h, size_t pitch,
                          const uint8_t cfa[4], float black, const float white[3], const float mul[3], float h_param,
                          int search, int patch, float tau, float* out_rgb, float* out_clip, unsigned flags) {
  if (!ctx || !c) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(w, h));
  ds_pat pat;
  DS_CHECK(check_pat(cfa, &pat));
  DS_CHECK(nlm_args_ok(3, search, patch));
  const size_t n = (size_t)w * h;
  if (n == 0) return DSGPU_OK;
  if (!raw || !out_rgb || !white || !mul || pitch < (size_t)w || search < 1) return DSGPU_ERR_ARG;
  if (w < 16 || h < 16) return DSGPU_ERR_UNSUPPORTED;
  DeviceGuard g(ctx->device);
  if (flags & DSGPU_HOST)
    return develop_cnn_pipelined(ctx, c->net, raw, w, h, pitch, pat, black, white, mul, h_param, search, patch, tau,
                                 out_rgb, out_clip);
  const void* din;
  void *drgb, *dclip = nullptr, *mid;
  unsigned char* fl;
  unsigned* cnt;
  DS_CHECK(stage_in(ctx, flags, S_IN, raw, ((size_t)(h - 1) * pitch + w) * sizeof(uint16_t), &din));
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out_rgb, n * 3 * sizeof(float), &drgb));
  if (out_clip) DS_CHECK(stage_out_ptr(ctx, flags, S_OUT2, out_clip, n * sizeof(float), &dclip));
  DS_CHECK(scratch(ctx, S_RGB, n * 3 * sizeof(float), &mid));
  DS_CHECK(fallback_scratch(ctx, w, h, patch, &fl, &cnt));
  {
    StageMark mark(ctx, DSGPU_STAGE_DEMOSAIC);
    const ds_src_u16 src = u16_source(ctx, din, pitch, black, white);
    DS_TRY(ds_launch_rcd_u16(ctx->stream, src, w, h, pat, mul, (float*)mid, (float*)dclip));
    ctx->launches += 1;
  }
  {
    StageMark mark(ctx, DSGPU_STAGE_CNN);
    HiddenMark hidden(ctx, c->net);
    DS_TRY(ds_cnn_denoise(c->net, ctx->stream, (const float*)mid, w, h, h_param, search, patch, tau,
                          DSGPU_CNN_STRENGTH_SCALE, (float*)drgb, fl, cnt));
    hidden.done = true;
    ctx->launches += 1 + 8 + (tau > 0.f ? 2 : 0) + (ds_cnn_judge_on(c->net) ? 3 : 0);
  }
  DS_CHECK(finish(ctx, flags, out_rgb, drgb, n * 3 * sizeof(float), out_clip, dclip, n * sizeof(float)));
  return (flags & DSGPU_ASYNC) ? DSGPU_OK : ds_cnn_take_status(c->net, ctx->stream);
}

// ------------------------------------------------------------------ scenes

int dsgpu_scene_render_host(const dsgpu_scene_desc* d, int x0, int y0, int cw, int ch, uint16_t* out) {
  if (!d || !out || cw < 0 || ch < 0 || d->w <= 0 || d->h <= 0) return DSGPU_ERR_ARG;
  if (x0 < 0 || y0 < 0 || x0 + cw > d->w || y0 + ch > d->h) return DSGPU_ERR_ARG;
  ds_pat pat;
  DS_CHECK(check_pat(d->cfa, &pat));
  ds_scene s = ds_scene_make(d);
  ds_scene_host(s, x0, y0, cw, ch, out);
  return DSGPU_OK;
}

int dsgpu_scene_truth_host(const dsgpu_scene_desc* d, int x0, int y0, int cw, int ch, float* out) {
  if (!d || !out || cw < 0 || ch < 0 || d->w <= 0 || d->h <= 0) return DSGPU_ERR_ARG;
  if (x0 < 0 || y0 < 0 || x0 + cw > d->w || y0 + ch > d->h) return DSGPU_ERR_ARG;
  ds_scene s = ds_scene_make(d);
  ds_scene_truth(s, x0, y0, cw, ch, out);
  return DSGPU_OK;
}

int dsgpu_scene_render(dsgpu_ctx* ctx, const dsgpu_scene_desc* d, uint16_t* out, unsigned flags) {
  if (!ctx || !d || !out || d->w <= 0 || d->h <= 0) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(d->w, d->h));
  ds_pat pat;
  DS_CHECK(check_pat(d->cfa, &pat));
  DeviceGuard g(ctx->device);
  const size_t bytes = (size_t)d->w * d->h * sizeof(uint16_t);
  void* dout;
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, bytes, &dout));
  ds_scene s = ds_scene_make(d);
  DS_TRY(ds_launch_scene(ctx->stream, s, (uint16_t*)dout));
  ctx->launches += 1;
  return finish(ctx, flags, out, dout, bytes);
}

int dsgpu_scene_render_window(dsgpu_ctx* ctx, const dsgpu_scene_desc* d, int x0, int y0, int cw, int ch,
                              uint16_t* out, unsigned flags) {
  if (!ctx || !d || !out || d->w <= 0 || d->h <= 0 || cw < 0 || ch < 0) return DSGPU_ERR_ARG;
  if (x0 < 0 || y0 < 0 || x0 + cw > d->w || y0 + ch > d->h) return DSGPU_ERR_ARG;
  DS_CHECK(check_dims(d->w, d->h));
  ds_pat pat;
  DS_CHECK(check_pat(d->cfa, &pat));
  DeviceGuard g(ctx->device);
  const size_t bytes = (size_t)cw * ch * sizeof(uint16_t);
  if (bytes == 0) return DSGPU_OK;
  void* dout;
  DS_CHECK(stage_out_ptr(ctx, flags, S_OUT, out, bytes, &dout));
  ds_scene s = ds_scene_make(d);
  DS_TRY(ds_launch_scene_window(ctx->stream, s, x0, y0, cw, ch, (uint16_t*)dout));
  ctx->launches += 1;
  return finish(ctx, flags, out, dout, bytes);
}

}  // extern "C"
