// Batched develop (dsgpu_rcd_nlm_batch) and the tile-shape autotuner.
//
// A batch is n frames of any sizes, CFA layouts, levels and strengths. One
// CUDA graph runs
//   descriptor and work-queue upload (pinned host -> device) -> zero the
//   counters -> start stamp -> ONE persistent kernel that takes the RCD and
//   NLM tiles of every frame from a work queue ordered RCD(0), RCD(1),
//   NLM(0), RCD(2), NLM(1), ... (batch_fused_kernel, k_demosaic.cu)
// on the context stream (captured on a private stream, since capture is not
// allowed on the legacy default stream). The NLM kernel stamps the device clock when a
// frame's last tile finishes, which gives the per-frame completion times.
// The graph is captured once per batch layout (sizes, tile shapes, search,
// patch) and replayed; everything that may change between calls with the
// same layout (pointers, levels, strengths) goes through the descriptors.
//
// RCD tile shape per frame: from the context's autotune table, filled by
// dsgpu_autotune (timings of the separate batched RCD and NLM kernels on
// synthetic frames of each size class). Every shape produces the same output bit for bit, so the
// table changes speed only.
#include <cstring>
#include <vector>

#include "ctx.h"
#include "scene.h"
#include "../../include/dsgpu_scene.h"

ds_scene ds_scene_make(const dsgpu_scene_desc* d);
cudaError_t ds_launch_scene(cudaStream_t st, const ds_scene& s, uint16_t* out);
void ds_nlm_batch_tile_grid(int w, int h, int patch, int* tiles_x, int* tiles_y);

namespace {

struct TuneEntry {
  int w, h;
  int shape;       // RCD tile shape index
  int nlm_per_sm;  // persistent NLM CTAs per SM
  double rcd_ms[DS_RCD_SHAPES];
  double nlm_ms[2];
};

constexpr int DEFAULT_SHAPE = 0;       // 32 x 32
constexpr int DEFAULT_NLM_PER_SM = 2;  // the NLM kernel's occupancy limit

}  // namespace

struct DsBatch {
  ds_batch_frame* d_frames = nullptr;
  ds_batch_frame* h_frames = nullptr;      // pinned: the graph's upload source
  unsigned* d_done = nullptr;              // NLM tiles finished per frame (the tuner's NLM runs)
  ds_batch_seg* d_segs = nullptr;          // work queue of the fused kernel
  ds_batch_seg* h_segs = nullptr;          // pinned
  int* d_ctr = nullptr;                    // fused-kernel counters (see ds_batch_ctr_nlm)
  int* h_status = nullptr;                 // pinned copy of the status word
  unsigned long long* d_stamps = nullptr;  // [0] batch start, [1 + f] frame f done (device ns)
  unsigned long long* h_stamps = nullptr;  // pinned
  cudaEvent_t done_ev = nullptr;           // after the last launched batch
  cudaStream_t cap = nullptr;              // private capture stream (the caller's may be the legacy one)
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> sig;              // layout of the captured graph
  bool in_flight = false;
  int last_n = 0;
  std::vector<TuneEntry> table;
};

void ds_batch_free(DsBatch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->done_ev) cudaEventDestroy(b->done_ev);
  if (b->cap) cudaStreamDestroy(b->cap);
  cudaFree(b->d_frames);
  cudaFree(b->d_done);
  cudaFree(b->d_segs);
  cudaFree(b->d_ctr);
  cudaFreeHost(b->h_segs);
  cudaFreeHost(b->h_status);
  cudaFree(b->d_stamps);
  cudaFreeHost(b->h_frames);
  cudaFreeHost(b->h_stamps);
  delete b;
}

namespace {

int batch_state(dsgpu_ctx* ctx, DsBatch** out) {
  if (!ctx->batch) {
    DsBatch* b = new (std::nothrow) DsBatch();
    if (!b) return DSGPU_ERR_NOMEM;
    cudaError_t e = cudaMalloc(&b->d_frames, DSGPU_BATCH_MAX * sizeof(ds_batch_frame));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_done, DSGPU_BATCH_MAX * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_stamps, (DSGPU_BATCH_MAX + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_segs, 2 * DSGPU_BATCH_MAX * sizeof(ds_batch_seg));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ctr, ds_batch_ctr_nlm(DSGPU_BATCH_MAX) * sizeof(int) +
                                                        DSGPU_BATCH_MAX * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_segs, 2 * DSGPU_BATCH_MAX * sizeof(ds_batch_seg));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_frames, DSGPU_BATCH_MAX * sizeof(ds_batch_frame));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_stamps, (DSGPU_BATCH_MAX + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      ds_batch_free(b);
      return map_cuda(ctx, e, "batch state");
    }
    ctx->batch = b;
  }
  *out = ctx->batch;
  return DSGPU_OK;
}

// the table entry for a w x h frame: the exact class, else the nearest in pixel count
const TuneEntry* lookup(const DsBatch* b, int w, int h) {
  const TuneEntry* best = nullptr;
  long long bd = 0;
  for (const TuneEntry& t : b->table) {
    if (t.w == w && t.h == h) return &t;
    const long long d = (long long)t.w * t.h - (long long)w * h;
    const long long ad = d < 0 ? -d : d;
    if (!best || ad < bd) {
      best = &t;
      bd = ad;
    }
  }
  return best;
}

int sm_count(int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return sms;
}

// Fill descriptor d for frame fr with RCD tile shape `shape`; tile numbering
// continues from *rcd_total / *nlm_total.
void describe(ds_batch_frame& d, const dsgpu_frame& fr, ds_pat pat, int shape, int patch, float* rgb,
              int* rcd_total, int* nlm_total) {
  int tw, th;
  ds_rcd_batch_shape(shape, &tw, &th);
  d.src.data = fr.raw;
  d.src.pitch = fr.pitch_elems;
  d.src.black = fr.black;
  d.src.bw = d.src.bh = d.src.bx0 = d.src.by0 = 0;  // the scalar black level, unless the frame has a pattern
  for (int i = 0; i < DS_BLACK_MAX * DS_BLACK_MAX; i++) d.src.bpat[i] = 0.f;
  if (fr.black_pattern) {
    d.src.bw = fr.black_w;
    d.src.bh = fr.black_h;
    d.src.bx0 = fr.black_x0 % fr.black_w;
    d.src.by0 = fr.black_y0 % fr.black_h;
    for (int i = 0; i < fr.black_w * fr.black_h; i++) d.src.bpat[i] = fr.black_pattern[i];
  }
  for (int c = 0; c < 3; c++) {
    d.src.white[c] = fr.white[c];
    d.mul[c] = fr.mul[c];
  }
  d.w = fr.w;
  d.h = fr.h;
  d.pat = pat;
  d.sigma = ds_nlm_sigma(fr.h_param, patch);
  d.rgb = rgb;
  d.clip = fr.out_clip;
  d.out = fr.out_rgb;
  d.rcd_shape = shape;
  d.rcd_tiles_x = (fr.w + tw - 1) / tw;
  d.rcd_tiles = d.rcd_tiles_x * ((fr.h + th - 1) / th);
  d.rcd_tile0 = *rcd_total;
  *rcd_total += d.rcd_tiles;
  int tx, ty;
  ds_nlm_batch_tile_grid(fr.w, fr.h, patch, &tx, &ty);
  d.nlm_tiles_x = tx;
  d.nlm_tiles_y = ty;
  d.nlm_tile0 = *nlm_total;
  *nlm_total += tx * ty * 3;
}

int check_frame(const dsgpu_frame& f, ds_pat* pat) {
  if (!f.raw || !f.out_rgb) return DSGPU_ERR_ARG;
  if (f.w < 16 || f.h < 16) return DSGPU_ERR_UNSUPPORTED;  // the reference's MHC case: one-frame calls
  if (f.w > DSGPU_MAX_DIM || f.h > DSGPU_MAX_DIM) return DSGPU_ERR_SIZE;
  if (f.pitch_elems < (size_t)f.w) return DSGPU_ERR_ARG;
  if (f.black_pattern) {
    if (f.black_w < 1 || f.black_h < 1 || f.black_w > DS_BLACK_MAX || f.black_h > DS_BLACK_MAX || f.black_x0 < 0 ||
        f.black_y0 < 0)
      return DSGPU_ERR_ARG;
    for (int i = 0; i < f.black_w * f.black_h; i++)
      if (!(f.black_pattern[i] == f.black_pattern[i])) return DSGPU_ERR_ARG;  // NaN
  }
  pat->packed = 0;
  for (int i = 0; i < 4; i++) {
    if (f.cfa[i] > 2) return DSGPU_ERR_CFA;
    pat->packed |= (uint32_t)f.cfa[i] << (8 * i);
  }
  return DSGPU_OK;
}

}  // namespace

extern "C" {

int dsgpu_rcd_nlm_batch(dsgpu_ctx* ctx, const dsgpu_frame* frames, int n, int search, int patch, unsigned flags) {
  if (!ctx || !frames || n < 1 || n > DSGPU_BATCH_MAX) return DSGPU_ERR_ARG;
  if (flags & DSGPU_HOST) return DSGPU_ERR_UNSUPPORTED;
  if (search < 1) return DSGPU_ERR_UNSUPPORTED;
  if (search > DSGPU_NLM_MAX_SEARCH || patch < 0 || patch > DSGPU_NLM_MAX_PATCH) return DSGPU_ERR_ARG;
  std::vector<ds_pat> pats(n);
  for (int i = 0; i < n; i++) DS_CHECK(check_frame(frames[i], &pats[i]));
  DeviceGuard g(ctx->device);
  DsBatch* b;
  DS_CHECK(batch_state(ctx, &b));
  if (b->in_flight) {  // the previous batch's upload may still read the pinned descriptors
    DS_TRY(cudaEventSynchronize(b->done_ev));
    b->in_flight = false;
  }
  // scratch: every frame's demosaiced RGB, 256-byte aligned
  std::vector<size_t> off(n);
  size_t total = 0;
  for (int i = 0; i < n; i++) {
    off[i] = total;
    total += ((size_t)frames[i].w * frames[i].h * 3 * sizeof(float) + 255) / 256 * 256;
  }
  void* base;
  DS_CHECK(scratch(ctx, S_BATCH, total, &base));
  // the NLM launch width: the tuned value of the largest frame's class
  int big = 0;
  for (int i = 1; i < n; i++)
    if ((long long)frames[i].w * frames[i].h > (long long)frames[big].w * frames[big].h) big = i;
  const TuneEntry* tb = lookup(b, frames[big].w, frames[big].h);
  const int nlm_per_sm = tb ? tb->nlm_per_sm : DEFAULT_NLM_PER_SM;
  std::vector<long long> sig = {n, search, patch, nlm_per_sm};
  int rcd_total = 0, nlm_total = 0;
  for (int i = 0; i < n; i++) {
    const TuneEntry* t = lookup(b, frames[i].w, frames[i].h);
    const int shape = t ? t->shape : DEFAULT_SHAPE;
    describe(b->h_frames[i], frames[i], pats[i], shape, patch,
             reinterpret_cast<float*>(static_cast<char*>(base) + off[i]), &rcd_total, &nlm_total);
    sig.push_back(frames[i].w);
    sig.push_back(frames[i].h);
    sig.push_back(shape);
  }
  // the fused kernel's work queue: RCD(0), RCD(1), NLM(0), RCD(2), NLM(1), ..., NLM(n-1)
  int nseg = 0, item = 0;
  auto push = [&](int kind, int f) {
    const ds_batch_frame& d = b->h_frames[f];
    b->h_segs[nseg++] = ds_batch_seg{kind, f, item};
    item += kind == 0 ? d.rcd_tiles : d.nlm_tiles_x * d.nlm_tiles_y * 3;
  };
  for (int f = 0; f < n; f++) {
    push(0, f);
    if (f > 0) push(1, f - 1);
  }
  push(1, n - 1);
  if (!b->exec || sig != b->sig) {
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    const int sms = sm_count(ctx->device);
    cudaStream_t st = b->cap;  // captured here, launched on the context stream
    DS_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemcpyAsync(b->d_frames, b->h_frames, n * sizeof(ds_batch_frame), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->d_segs, b->h_segs, nseg * sizeof(ds_batch_seg), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(b->d_ctr, 0, ds_batch_ctr_nlm(DSGPU_BATCH_MAX) * sizeof(int) + n * sizeof(int), st);
    if (e == cudaSuccess) e = ds_launch_stamp(st, b->d_stamps);
    if (e == cudaSuccess)
      e = ds_launch_batch_fused(st, b->d_frames, n, b->d_segs, nseg, rcd_total + nlm_total, search, patch,
                                nlm_per_sm * sms, b->d_ctr, DSGPU_BATCH_MAX, b->d_stamps + 1);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      b->exec = nullptr;
      return map_cuda(ctx, e, "batch graph capture");
    }
    b->sig = sig;
  }
  DS_TRY(cudaGraphLaunch(b->exec, ctx->stream));
  DS_TRY(cudaEventRecord(b->done_ev, ctx->stream));
  b->in_flight = true;
  b->last_n = n;
  ctx->launches += 2;
  if (!(flags & DSGPU_ASYNC)) {
    DS_TRY(cudaMemcpyAsync(b->h_status, b->d_ctr + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    DS_TRY(cudaStreamSynchronize(ctx->stream));
    b->in_flight = false;
    if (*b->h_status != 0) return *b->h_status;  // a tile waited in vain for its frame's demosaic
  }
  return DSGPU_OK;
}

// Failure detection on the device, without a fault: one NLM work item whose
// frame's demosaic (one RCD tile) is never queued, so the item's bounded wait
// on the frame's RCD counter can only run out; the kernel then records
// DSGPU_ERR_TIMEOUT in its status word and returns, and the stream and the
// context stay usable. The NLM tile body is never reached (its buffers are
// allocated all the same).
int dsgpu_selftest_batch_timeout(dsgpu_ctx* ctx) {
  if (!ctx) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  constexpr int FW = 64, FH = 58;
  ds_batch_frame f{};
  f.w = FW;
  f.h = FH;
  f.pat.packed = 0u | (1u << 8) | (1u << 16) | (2u << 24);
  f.mul[0] = f.mul[1] = f.mul[2] = 1.f;
  f.sigma = 1.f;
  f.rcd_tiles = 1;  // waited for, never produced
  f.nlm_tiles_x = 1;
  f.nlm_tiles_y = 1;
  const ds_batch_seg seg{1, 0, 0};  // one NLM item of frame 0
  ds_batch_frame* df = nullptr;
  ds_batch_seg* ds = nullptr;
  int* dc = nullptr;
  unsigned long long* dst = nullptr;
  float* buf = nullptr;
  int status = DSGPU_OK, h = 0;
  cudaError_t e = cudaMalloc(&buf, (size_t)2 * FW * FH * 3 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&df, sizeof(ds_batch_frame));
  if (e == cudaSuccess) e = cudaMalloc(&ds, sizeof(ds_batch_seg));
  if (e == cudaSuccess) e = cudaMalloc(&dc, (size_t)ds_batch_ctr_nlm(1) * sizeof(int) + sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&dst, sizeof(unsigned long long));
  if (e == cudaSuccess) {
    f.rgb = buf;
    f.out = buf + (size_t)FW * FH * 3;
    e = cudaMemcpyAsync(df, &f, sizeof f, cudaMemcpyHostToDevice, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(ds, &seg, sizeof seg, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(dc, 0, (size_t)ds_batch_ctr_nlm(1) * sizeof(int) + sizeof(int), ctx->stream);
  if (e == cudaSuccess) e = ds_launch_batch_fused(ctx->stream, df, 1, ds, 1, 1, 3, 3, 1, dc, 1, dst);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, dc + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) status = map_cuda(ctx, e, "dsgpu_selftest_batch_timeout");
  else status = h;
  cudaFree(dst);
  cudaFree(dc);
  cudaFree(ds);
  cudaFree(df);
  cudaFree(buf);
  return status;  // DSGPU_ERR_TIMEOUT when the wait gave up as designed
}

int dsgpu_batch_frame_ms(dsgpu_ctx* ctx, double* frame_ms, int n) {
  if (!ctx || !frame_ms || n < 0) return DSGPU_ERR_ARG;
  DsBatch* b = ctx->batch;
  if (!b || b->last_n == 0) return DSGPU_ERR_ARG;  // no batch has run
  if (n > b->last_n) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DS_TRY(cudaEventSynchronize(b->done_ev));
  b->in_flight = false;
  DS_TRY(cudaMemcpy(b->h_stamps, b->d_stamps, (b->last_n + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  DS_TRY(cudaMemcpy(b->h_status, b->d_ctr + 1, sizeof(int), cudaMemcpyDeviceToHost));
  if (*b->h_status != 0) return *b->h_status;  // the batch stopped early: no valid times
  for (int i = 0; i < n; i++) frame_ms[i] = (double)(long long)(b->h_stamps[1 + i] - b->h_stamps[0]) * 1e-6;
  return DSGPU_OK;
}

int dsgpu_autotune(dsgpu_ctx* ctx, const int* sizes, int n_sizes, int search, int patch) {
  if (!ctx || !sizes || n_sizes < 1) return DSGPU_ERR_ARG;
  if (search < 1 || search > DSGPU_NLM_MAX_SEARCH || patch < 0 || patch > DSGPU_NLM_MAX_PATCH) return DSGPU_ERR_ARG;
  for (int i = 0; i < n_sizes; i++)
    if (sizes[2 * i] < 16 || sizes[2 * i + 1] < 16 || sizes[2 * i] > DSGPU_MAX_DIM || sizes[2 * i + 1] > DSGPU_MAX_DIM)
      return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DsBatch* b;
  DS_CHECK(batch_state(ctx, &b));
  if (b->in_flight) {
    DS_TRY(cudaEventSynchronize(b->done_ev));
    b->in_flight = false;
  }
  cudaStream_t st = ctx->stream;
  const int sms = sm_count(ctx->device);
  cudaEvent_t e0, e1;
  DS_TRY(cudaEventCreate(&e0));
  DS_TRY(cudaEventCreate(&e1));
  int status = DSGPU_OK;
  for (int c = 0; c < n_sizes && status == DSGPU_OK; c++) {
    const int w = sizes[2 * c], h = sizes[2 * c + 1];
    const size_t px = (size_t)w * h;
    uint16_t* raw = nullptr;
    float *rgb = nullptr, *out = nullptr;
    cudaError_t e = cudaMalloc(&raw, px * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc(&rgb, px * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&out, px * 3 * sizeof(float));
    dsgpu_scene_desc sd = {0x5EEDull + (unsigned)c, w, h, {0, 1, 1, 2}, 512, 16383, 0.5f, 6.0f};
    if (e == cudaSuccess) e = ds_launch_scene(st, ds_scene_make(&sd), raw);
    dsgpu_frame fr = {raw, (size_t)w, w, h, {0, 1, 1, 2}, 512.f, {16383.f, 16383.f, 16383.f}, {2.f, 1.f, 1.4285714f},
                      0.012f, out, nullptr};
    ds_pat pat;
    pat.packed = 0x02010100u;
    TuneEntry te = {w, h, DEFAULT_SHAPE, DEFAULT_NLM_PER_SM, {}, {}};
    // time a launch: one warm-up, then the best of `reps`
    auto best_of = [&](int reps, auto launch) -> double {
      double best = 1e30;
      cudaError_t le = launch();
      for (int r = 0; r < reps && le == cudaSuccess; r++) {
        cudaEventRecord(e0, st);
        le = launch();
        cudaEventRecord(e1, st);
        if (le == cudaSuccess) le = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (le == cudaSuccess) le = cudaEventElapsedTime(&ms, e0, e1);
        if (le == cudaSuccess && ms < best) best = ms;
      }
      if (le != cudaSuccess) e = le;
      return best;
    };
    for (int s = 0; s < DS_RCD_SHAPES && e == cudaSuccess; s++) {
      int rt = 0, nt = 0;
      describe(b->h_frames[0], fr, pat, s, patch, rgb, &rt, &nt);
      e = cudaMemcpyAsync(b->d_frames, b->h_frames, sizeof(ds_batch_frame), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess)
        te.rcd_ms[s] = best_of(3, [&] { return ds_launch_rcd_batch(st, b->d_frames, 1, rt, 2 * sms); });
      if (e == cudaSuccess && te.rcd_ms[s] < te.rcd_ms[te.shape]) te.shape = s;
    }
    for (int k = 1; k <= 2 && e == cudaSuccess; k++) {
      int rt = 0, nt = 0;
      describe(b->h_frames[0], fr, pat, te.shape, patch, rgb, &rt, &nt);
      e = cudaMemcpyAsync(b->d_frames, b->h_frames, sizeof(ds_batch_frame), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemsetAsync(b->d_done, 0, sizeof(unsigned), st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess)
        te.nlm_ms[k - 1] = best_of(2, [&] {
          return ds_launch_nlm_batch(st, b->d_frames, 1, nt, search, patch, k * sms, b->d_done, b->d_stamps + 1);
        });
    }
    if (e == cudaSuccess) te.nlm_per_sm = te.nlm_ms[0] < te.nlm_ms[1] ? 1 : 2;
    cudaStreamSynchronize(st);
    cudaFree(raw);
    cudaFree(rgb);
    cudaFree(out);
    if (e != cudaSuccess) {
      status = map_cuda(ctx, e, "dsgpu_autotune");
      break;
    }
    bool replaced = false;
    for (TuneEntry& t : b->table)
      if (t.w == w && t.h == h) {
        t = te;
        replaced = true;
      }
    if (!replaced) b->table.push_back(te);
    ctx->launches += DS_RCD_SHAPES * 4 + 2 * 3 + 1;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return status;
}

int dsgpu_autotune_get(dsgpu_ctx* ctx, int w, int h, int* rcd_tile_w, int* rcd_tile_h, int* nlm_ctas_per_sm,
                       double* rcd_ms) {
  if (!ctx || !rcd_tile_w || !rcd_tile_h || !nlm_ctas_per_sm) return DSGPU_ERR_ARG;
  const TuneEntry* t = ctx->batch ? lookup(ctx->batch, w, h) : nullptr;
  ds_rcd_batch_shape(t ? t->shape : DEFAULT_SHAPE, rcd_tile_w, rcd_tile_h);
  *nlm_ctas_per_sm = t ? t->nlm_per_sm : DEFAULT_NLM_PER_SM;
  if (rcd_ms)
    for (int s = 0; s < DS_RCD_SHAPES; s++) rcd_ms[s] = (t && t->w == w && t->h == h) ? t->rcd_ms[s] : -1.0;
  return DSGPU_OK;
}

int dsgpu_autotune_set(dsgpu_ctx* ctx, int w, int h, int rcd_tile_w, int rcd_tile_h, int nlm_ctas_per_sm) {
  if (!ctx || w < 16 || h < 16 || nlm_ctas_per_sm < 1 || nlm_ctas_per_sm > 2) return DSGPU_ERR_ARG;
  int shape = -1;
  for (int s = 0; s < DS_RCD_SHAPES; s++) {
    int tw, th;
    ds_rcd_batch_shape(s, &tw, &th);
    if (tw == rcd_tile_w && th == rcd_tile_h) shape = s;
  }
  if (shape < 0) return DSGPU_ERR_ARG;
  DeviceGuard g(ctx->device);
  DsBatch* b;
  DS_CHECK(batch_state(ctx, &b));
  TuneEntry te = {w, h, shape, nlm_ctas_per_sm, {}, {}};
  for (int s = 0; s < DS_RCD_SHAPES; s++) te.rcd_ms[s] = -1.0;
  te.nlm_ms[0] = te.nlm_ms[1] = -1.0;
  for (TuneEntry& t : b->table)
    if (t.w == w && t.h == h) {
      t = te;
      return DSGPU_OK;
    }
  b->table.push_back(te);
  return DSGPU_OK;
}

}  // extern "C"
