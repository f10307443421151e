/* dsgpu.h — C ABI of the B200 (sm_100a) RCD demosaic + NLM denoise library.
 *
 * This is the drop-in boundary for darkslide-core's raw-develop detail path.
 * Each entry point replaces one function of the reference (Rust, crates/core);
 * the reference citation is given beside each declaration. Argument meaning
 * follows the reference: a Bayer pattern is four colour codes (0=R, 1=G, 2=B)
 * indexed by (y%2)*2 + x%2 (decode.rs:26-28), images are row-major, RGB
 * images are interleaved float[3] per pixel (image.rs:7-13), planes are float
 * (image.rs:15-21), CFA data is normalised so 1.0 is white (decode.rs:49-56).
 *
 * Conventions
 *  - Every call returns DSGPU_OK (0) or a negative DSGPU_ERR_* code; the
 *    library never aborts. dsgpu_strerror() names a code.
 *  - Buffers are caller-allocated. Without DSGPU_HOST every pointer is device
 *    memory of the context's device and the work is enqueued on the context
 *    stream (dsgpu_set_stream); the call synchronises that stream before
 *    returning unless DSGPU_ASYNC is given. With DSGPU_HOST every pointer is
 *    host memory (pinned memory is fastest): the call copies inputs to device
 *    scratch, runs, copies results back and synchronises.
 *  - A context is used by one thread at a time (one context per caller
 *    thread), like the reference's Engine calls on the render worker.
 *  - Degenerate inputs are absorbed the way the reference absorbs them: RCD
 *    on w or h < 16 is MHC (demosaic.rs:149-151); NLM floors h^2 and the
 *    weight sum at 1e-12 (enhance.rs:40,71); a negative search radius gives
 *    an empty offset set and a zero image (enhance.rs:41,71).
 */
#ifndef DSGPU_H
#define DSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSGPU_ABI_VERSION 2

/* status codes */
#define DSGPU_OK 0
#define DSGPU_ERR_ARG (-1)      /* null pointer, negative size or radius out of range */
#define DSGPU_ERR_CFA (-2)      /* colour code outside {0,1,2} */
#define DSGPU_ERR_SIZE (-3)     /* image larger than the library limits */
#define DSGPU_ERR_NOMEM (-4)    /* device or pinned allocation failed */
#define DSGPU_ERR_CUDA (-5)     /* a CUDA runtime call failed */
#define DSGPU_ERR_NODEV (-6)    /* no usable sm_100 device */
#define DSGPU_ERR_TIMEOUT (-7)  /* a bounded device-side wait gave up */
#define DSGPU_ERR_UNSUPPORTED (-8)

/* flags */
#define DSGPU_HOST 1u  /* buffers are host memory */
#define DSGPU_ASYNC 2u /* device buffers: do not synchronise before returning */
/* dsgpu_nlm / dsgpu_develop_u16: the precision variant of NLM. The
 * horizontal patch-distance sums that the kernel hands between its two
 * phases through shared memory are staged in FP16 (rounded to nearest,
 * saturated to the largest finite half); differences, weights and sums stay
 * in FP32. Not bit-equal to the FP32 path; its error against the FP64 oracle
 * is measured by the tests and the profiles. */
#define DSGPU_FP16_STAGING 4u
/* dsgpu_develop_u16: reconstruct highlights between RCD and NLM, as
 * Engine::base does (pipeline/mod.rs:186-187): cfa_clip_levels of the
 * normalised mosaic, then reconstruct_highlights with the clip plane. */
#define DSGPU_HIGHLIGHTS 8u

/* demosaic quality (demosaic.rs:9-15) */
#define DSGPU_QUALITY_DRAFT 0
#define DSGPU_QUALITY_FULL 1

/* limits */
#define DSGPU_MAX_DIM 65535      /* w, h */
#define DSGPU_NLM_MAX_SEARCH 16  /* search radius S */
#define DSGPU_NLM_MAX_PATCH 7    /* patch radius P */

typedef struct dsgpu_ctx dsgpu_ctx;

const char* dsgpu_strerror(int status);
int dsgpu_abi_version(void);

/* Context: owns a CUDA stream (or borrows the caller's), device scratch and
 * pinned staging buffers. `device` is a CUDA ordinal. */
int dsgpu_create(int device, dsgpu_ctx** out);
int dsgpu_destroy(dsgpu_ctx* ctx);
/* Use the caller's cudaStream_t (NULL: back to the context's own stream). */
int dsgpu_set_stream(dsgpu_ctx* ctx, void* cuda_stream);
void* dsgpu_get_stream(dsgpu_ctx* ctx);
int dsgpu_synchronize(dsgpu_ctx* ctx);
/* Release cached scratch (it is regrown on demand). */
int dsgpu_trim(dsgpu_ctx* ctx);
/* Text of the last CUDA failure seen by this context ("" if none). */
const char* dsgpu_last_error(dsgpu_ctx* ctx);

/* Instrumentation; the analogue of the reference's Lap stage timer
 * (pipeline/mod.rs:106-137), which logs per-stage wall time.
 * dsgpu_profile(ctx, 1) starts recording CUDA events around each stage of
 * every later call on the context stream (and discards earlier records);
 * dsgpu_stage_ms() sums the recorded device time of one stage.
 * dsgpu_launch_count() is the number of kernels the context has launched.
 * dsgpu_measure_peaks() times FP32 FMA, ex2 and packed (f32x2) FMA
 * throughput microbenchmarks, the roofline denominators of the NLM kernel
 * (ffma2_flops_per_s may be NULL). */
#define DSGPU_STAGE_DEMOSAIC 0
#define DSGPU_STAGE_NLM 1
#define DSGPU_STAGE_COPY 2
#define DSGPU_STAGE_CNN 3
/* the six hidden 48 -> 48 conv layers of the learned path, one mark per call */
#define DSGPU_STAGE_CNN_HIDDEN 4
int dsgpu_profile(dsgpu_ctx* ctx, int enable);
int dsgpu_stage_ms(dsgpu_ctx* ctx, int stage, double* total_ms, int* count);
unsigned long long dsgpu_launch_count(dsgpu_ctx* ctx);
int dsgpu_measure_peaks(dsgpu_ctx* ctx, double* ffma_flops_per_s, double* ex2_per_s, double* ffma2_flops_per_s);
/* BF16 mma.sync (m16n8k16, FP32 accumulate) throughput microbenchmark. */
int dsgpu_measure_mma_sync(dsgpu_ctx* ctx, double* bf16_flops_per_s);

/* Per-site black levels, as load_raw's black_at takes them from the raw's
 * black-level record (decode.rs:266-270): a bw x bh pattern (1..4 each, row
 * major, one value per site) indexed at UNCROPPED sensor coordinates, so
 * that site (x, y) of a frame cropped at (origin_x, origin_y) subtracts
 * levels[((y + origin_y) % bh) * bw + (x + origin_x) % bw]. While a pattern
 * is set, every u16 entry point of this context (dsgpu_normalize_u16,
 * dsgpu_develop_u16, dsgpu_develop_u16_cnn) uses it in place of its scalar
 * black argument, in the numerator and in the white - black denominator
 * alike (decode.rs:303). bw = bh = 0 clears it. A batch takes its patterns
 * per frame (dsgpu_frame.black_pattern); the no-alloc entry point takes the
 * scalar black only. */
int dsgpu_set_black_pattern(dsgpu_ctx* ctx, const float* levels, int bw, int bh, int origin_x, int origin_y);
/* CFA normalisation of an integer raw: out = (raw - black) / max(white[c] - black, 1),
 * c the colour of the site; values are not clamped.
 * Replaces the integer branch of load_raw, decode.rs:292-306 (formula :303). */
int dsgpu_normalize_u16(dsgpu_ctx* ctx, const uint16_t* raw, int w, int h, size_t pitch_elems,
                        const uint8_t cfa[4], float black, const float white[3], float* out_cfa,
                        unsigned flags);

/* 3x3 clamped-edge max of [v >= 0.995]. Replaces clip_plane, demosaic.rs:31-42. */
int dsgpu_clip_plane(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, float* out_clip, unsigned flags);

/* Malvar-He-Cutler Bayer demosaic. Replaces mhc_bayer, demosaic.rs:90-124. */
int dsgpu_mhc(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, const uint8_t cfa[4], const float mul[3],
              float* out_rgb, unsigned flags);

/* RCD Bayer demosaic (MHC when w or h < 16). Replaces rcd_bayer, demosaic.rs:147-344. */
int dsgpu_rcd(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, const uint8_t cfa[4], const float mul[3],
              float* out_rgb, unsigned flags);

/* demosaic(cfa, mul, quality) for a Bayer pattern, demosaic.rs:20-27.
 * FULL: out_rgb is w*h*3 (RCD), out_clip w*h (clip_plane).
 * DRAFT: superpixel (demosaic.rs:45-87): out_rgb is (w/2)*(h/2)*3 and
 * out_clip (w/2)*(h/2). out_clip may be NULL. */
int dsgpu_demosaic(dsgpu_ctx* ctx, const float* cfa_data, int w, int h, const uint8_t cfa[4],
                   const float mul[3], int quality, float* out_rgb, float* out_clip, unsigned flags);

/* Separable clamped-edge box blur of radius r. Replaces box_blur, image.rs:269-313. */
int dsgpu_box_blur(dsgpu_ctx* ctx, const float* in, int w, int h, int r, float* out, unsigned flags);

/* Non-local means with patch radius `patch` and search radius `search`
 * on each of `channels` interleaved channels (1: a Plane; 3: an Image3
 * denoised per channel as channel()/nlm()/merge3() would).
 * Replaces nlm, enhance.rs:36-72. */
int dsgpu_nlm(dsgpu_ctx* ctx, const float* in, int w, int h, int channels, float h_param, int search,
              int patch, float* out, unsigned flags);

/* Robust noise sigma of a plane: median |Laplacian| of up to ~200k sampled
 * sites / 0.6745 / sqrt(20), 0 for planes without interior sites.
 * Replaces estimate_noise, enhance.rs:10-32. `sigma` is host memory. */
int dsgpu_estimate_noise(dsgpu_ctx* ctx, const float* plane, int w, int h, float* sigma, unsigned flags);

/* He et al. guided filter of p guided by I, box radius r, regulariser eps.
 * Replaces guided_filter, image.rs:385-405. */
int dsgpu_guided_filter(dsgpu_ctx* ctx, const float* I, const float* p, int w, int h, int r, float eps, float* out,
                        unsigned flags);

/* Oklab matrices of Oklab::new() (color.rs:394-399): to_lms, from_lms and
 * inverse M2, row-major, 27 floats. Host only. */
int dsgpu_oklab_matrices(float* out27);

/* Per-colour clip level actually reached in a normalised mosaic: the maximum
 * over every third row, kept when >= 0.95, else FLT_MAX. out3 is host
 * memory (the call waits). Replaces cfa_clip_levels, demosaic.rs:419-430. */
int dsgpu_cfa_clip_levels(dsgpu_ctx* ctx, const float* cfa, int w, int h, const uint8_t pattern[4], float* out3,
                          unsigned flags);
/* Highlight reconstruction in place on interleaved RGB (w*h*3): channels at
 * their clip level are rebuilt from colour ratios of nearby bright unclipped
 * pixels, fully clipped pixels become neutral. clip: the clip plane of
 * dsgpu_demosaic; raw_clip: host array of 3 (dsgpu_cfa_clip_levels). A no-op
 * when no clip-plane pixel is set. Replaces reconstruct_highlights,
 * demosaic.rs:435-502 (bit-exact). */
int dsgpu_reconstruct_highlights(dsgpu_ctx* ctx, float* rgb, const float* clip, int w, int h, const float mul[3],
                                 const float raw_clip[3], unsigned flags);

/* EXIF orientation (1-8) of an interleaved RGB image: out is h x w (width
 * h) for 5-8, else w x h; other codes copy. out must not alias in. Replaces
 * apply_orientation, decode.rs:414-426 (exact: a permutation). */
int dsgpu_apply_orientation(dsgpu_ctx* ctx, const float* in_rgb, int w, int h, int orientation, float* out_rgb,
                            unsigned flags);

/* Strong denoise of an interleaved linear RGB image, amount 0..100: Oklab L
 * through NLM (search 3, patch 1, h = sigma (0.6 + 1.6 amount/100)), chroma
 * through guided filters. Replaces denoise, enhance.rs:75-92. */
int dsgpu_denoise(dsgpu_ctx* ctx, const float* in_rgb, int w, int h, float amount, float* out_rgb, unsigned flags);

/* The detail path in one call: u16 raw -> normalise -> RCD -> per-channel NLM.
 * Equivalent to load_raw's normalisation (decode.rs:292-306), demosaic(Full)
 * (demosaic.rs:20-27) and nlm() on each channel (enhance.rs:36-72).
 * out_clip (w*h) may be NULL. The demosaiced intermediate lives in context
 * scratch. */
int dsgpu_develop_u16(dsgpu_ctx* ctx, const uint16_t* raw, int w, int h, size_t pitch_elems,
                      const uint8_t cfa[4], float black, const float white[3], const float mul[3],
                      float h_param, int search, int patch, float* out_rgb, float* out_clip, unsigned flags);

/* The same detail path for callers that cannot allocate device memory.
 * No counterpart in the reference. It is for callers that manage every byte
 * of device memory themselves (a pool or a framework's caching allocator
 * that must not be bypassed) or that run where cudaMalloc is not allowed or
 * would stall the device. dsgpu_develop_u16 allocates its demosaiced
 * intermediate in context scratch; this call instead uses one fixed array
 * of DSGPU_NOALLOC_SCRATCH_BYTES inside the library's device image, which
 * every GPU that loads the library holds until the process exits. It calls
 * no cudaMalloc, cudaFree or other allocating routine.
 *  - All pointers are device memory of the current device; DSGPU_HOST is
 *    rejected (DSGPU_ERR_ARG). Work goes on `cuda_stream` (NULL: the legacy
 *    default stream); the call synchronises it unless DSGPU_ASYNC is given.
 *  - Flags: DSGPU_ASYNC and DSGPU_FP16_STAGING act as in dsgpu_develop_u16
 *    (the output is bit-identical to it with the same flags);
 *    DSGPU_HIGHLIGHTS needs scratch this call does not have
 *    (DSGPU_ERR_UNSUPPORTED); any other bit is DSGPU_ERR_ARG.
 *  - There is no context, so no per-site black pattern
 *    (dsgpu_set_black_pattern) applies: every site uses the scalar `black`.
 *  - Frames above DSGPU_NOALLOC_MAX_PIXELS (w*h) are rejected with
 *    DSGPU_ERR_SIZE.
 *  - The first call on a device looks up the array's device address (once per
 *    device and CUDA context, with that device current); make that first
 *    call before any stream capture.
 *  - Every call shares the array and it keeps the last call's contents (each
 *    call overwrites what it reads). Calls that overlap on the GPU race on it:
 *    serialise them. */
#define DSGPU_NOALLOC_SCRATCH_BYTES (16u << 20)
#define DSGPU_NOALLOC_MAX_PIXELS (1 << 20) /* 16 B per pixel: RGB intermediate + normalised CFA */
int dsgpu_develop_u16_noalloc(void* cuda_stream, const uint16_t* raw, int w, int h, size_t pitch_elems,
                              const uint8_t cfa[4], float black, const float white[3], const float mul[3],
                              float h_param, int search, int patch, float* out_rgb, float* out_clip,
                              unsigned flags);

/* ------------------------------------------------------------ batched develop
 * The survey's dsgpu_rcd_nlm_batch: many frames of different sizes, CFA
 * layouts, levels and strengths through dsgpu_develop_u16's path in one
 * CUDA graph launch holding ONE persistent kernel that takes the RCD and NLM
 * tiles of every frame from a work queue (a frame's NLM starts right after
 * its demosaic; the reference develops one frame per call,
 * pipeline/mod.rs:172-252). Each frame's output equals dsgpu_develop_u16's
 * on the same frame bit for bit. */
typedef struct dsgpu_frame {
  const uint16_t* raw;  /* device, h rows of pitch_elems */
  size_t pitch_elems;
  int w, h;             /* 16 <= w, h <= DSGPU_MAX_DIM */
  uint8_t cfa[4];
  float black;
  float white[3];
  float mul[3];
  float h_param;        /* NLM strength of this frame */
  float* out_rgb;       /* device, w*h*3 */
  float* out_clip;      /* device, w*h, or NULL */
  /* Per-site black levels of this frame (as dsgpu_set_black_pattern, at
   * uncropped coordinates; the context's own pattern does not apply to a
   * batch): host pointer to black_w * black_h levels (1..4 each), or NULL
   * for the scalar black. */
  const float* black_pattern;
  int black_w, black_h;
  int black_x0, black_y0; /* the frame's crop origin */
} dsgpu_frame;
#define DSGPU_BATCH_MAX 256
/* Device pointers only (DSGPU_HOST -> DSGPU_ERR_UNSUPPORTED); search >= 1.
 * The demosaiced intermediates of all frames live in context scratch. The
 * graph is captured on the first call for a batch layout (frame sizes, tile
 * shapes, search, patch) and replayed by later calls with the same layout;
 * frame pointers and levels may change between calls. RCD tile shapes come
 * from the context's autotune table (dsgpu_autotune), else 32 x 32. */
int dsgpu_rcd_nlm_batch(dsgpu_ctx* ctx, const dsgpu_frame* frames, int n, int search, int patch, unsigned flags);
/* Failure-detection self-test (no counterpart in the reference): runs the
 * batched kernel on one NLM work item whose frame's demosaic is never queued,
 * so the item's bounded wait (2 s of device clock) must give up. Returns
 * DSGPU_ERR_TIMEOUT when it does, the context staying usable; DSGPU_OK would
 * mean the wait did not end as designed. Allocates its own small buffers. */
int dsgpu_selftest_batch_timeout(dsgpu_ctx* ctx);
/* Completion time of each frame of the last batch, ms after the batch started
 * on the device (measured with the device clock; waits for the batch).
 * Returns the batch's own status when it stopped early (DSGPU_ERR_TIMEOUT). */
int dsgpu_batch_frame_ms(dsgpu_ctx* ctx, double* frame_ms, int n);
/* Autotuner: for each size class (w, h) = (sizes[2i], sizes[2i+1]), time the
 * batched RCD kernel with every tile shape and the batched NLM kernel with 1
 * and 2 CTAs per SM on a synthetic frame of that size, and keep the fastest
 * in the context's table. */
int dsgpu_autotune(dsgpu_ctx* ctx, const int* sizes, int n_sizes, int search, int patch);
/* The table entry used for a w x h frame (the exact class, else the class
 * nearest in pixel count, else the defaults 32 x 32 and 2 CTAs per SM);
 * rcd_ms (may be NULL) receives the tuned RCD time per shape index (5) for
 * an exact class, else -1. */
int dsgpu_autotune_get(dsgpu_ctx* ctx, int w, int h, int* rcd_tile_w, int* rcd_tile_h, int* nlm_ctas_per_sm,
                       double* rcd_ms);
/* Set a table entry by hand (a table saved by a caller, or a test). */
int dsgpu_autotune_set(dsgpu_ctx* ctx, int w, int h, int rcd_tile_w, int rcd_tile_h, int nlm_ctas_per_sm);

/* ------------------------------------------------------------ learned path
 * A residual CNN standing in for nlm(): 8 conv3x3 layers (4 -> 48 -> ... ->
 * 48 -> 3, ReLU), input = RGB plus a constant map of the NLM strength h,
 * output = input + network. BF16 tensor-core kernels, FP32 accumulation,
 * FP32 master weights and Adam state. Parameters are a flat float array:
 * for each layer, weights [9 taps][cout][cin] then biases [cout].
 * No counterpart in the reference (it has no learned denoiser); it is trained
 * to reproduce enhance.rs:36-72 and falls back to it per tile. */
typedef struct dsgpu_cnn dsgpu_cnn;
int dsgpu_cnn_param_count(void);
/* max_batch crops of crop x crop pixels for training (0, 0: inference only) */
int dsgpu_cnn_create(dsgpu_ctx* ctx, int max_batch, int crop, dsgpu_cnn** out);
int dsgpu_cnn_destroy(dsgpu_ctx* ctx, dsgpu_cnn* net);
/* get (set = 0) or set (set = 1) parameters (which 0) or Adam moments
 * (which 1, 2); buf may be NULL to move only the step counter. */
int dsgpu_cnn_state(dsgpu_ctx* ctx, dsgpu_cnn* net, int which, float* buf, int set, long long* step,
                    unsigned flags);
/* Gradient of sum-of-squares / (3 n) between the network's output on
 * (rgb[batch][crop][crop][3], strength map or constant) and target, into
 * grads (device, param_count floats; may be NULL); loss_sum = sum of squared
 * errors. Device buffers. */
int dsgpu_cnn_gradients(dsgpu_ctx* ctx, dsgpu_cnn* net, const float* rgb, const float* strength_map,
                        float strength, const float* target, int batch, float* grads, float* loss_sum,
                        unsigned flags);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on the same loss. Device buffers. */
int dsgpu_cnn_train_step(dsgpu_ctx* ctx, dsgpu_cnn* net, const float* rgb, const float* strength_map,
                         float strength, const float* target, int batch, float lr, float* loss_sum);
/* Clip the global L2 norm of the gradient to max_norm before each Adam step
 * of dsgpu_cnn_train_step (0, the default: no clipping). */
int dsgpu_cnn_set_clip(dsgpu_ctx* ctx, dsgpu_cnn* net, float max_norm);
/* Loss of dsgpu_cnn_gradients / dsgpu_cnn_train_step: relative = 0 (default)
 * sum((out - target)^2) / (3 n); relative = 1 weights every pixel's squared
 * error by 1 / strength^2 (its strength input), so that low-noise frames
 * weigh as much as noisy ones. */
int dsgpu_cnn_set_loss(dsgpu_ctx* ctx, dsgpu_cnn* net, int relative);
/* out = in + network(in, strength) on a whole interleaved RGB image
 * (strength = DSGPU_CNN_STRENGTH_SCALE * h). */
#define DSGPU_CNN_STRENGTH_SCALE 50.0f
int dsgpu_cnn_infer(dsgpu_ctx* ctx, dsgpu_cnn* net, const float* in_rgb, int w, int h, float strength,
                    float* out_rgb, unsigned flags);
/* Engine: 1 (default) the tcgen05 tensor cores with TMEM accumulators for
 * inference and for all of training's convolutions: forward pass, data
 * gradients, weight and bias gradients (the batch laid out as one frame of
 * crops with zero rows between them); 0 the warp-level mma.sync kernels
 * throughout. A bounded device wait that gives up makes the call return
 * DSGPU_ERR_TIMEOUT. */
int dsgpu_cnn_set_engine(dsgpu_ctx* ctx, dsgpu_cnn* net, int tensor_core_gen5);
/* The learned stand-in for nlm(in, h_param, search, patch) with its per-tile
 * fallback: the network runs on the whole image, then every NLM tile (16 x
 * (64 - 2 patch) pixels) whose removed component out - in has an RMS above
 * tau * h / 1.5 (or is not finite) is recomputed by plain NLM. tau <= 0
 * disables the fallback.
 * *fallback_tiles (may be NULL) receives the number of tiles recomputed. */
int dsgpu_cnn_denoise(dsgpu_ctx* ctx, dsgpu_cnn* net, const float* in_rgb, int w, int h, float h_param,
                      int search, int patch, float tau, float* out_rgb, int* fallback_tiles, unsigned flags);
/* Judge mode of the learned path (plain GPU NLM as the judge of the
 * network's error; no counterpart in the reference): plain NLM recomputes a
 * seeded sample of the NLM tiles, and on each sampled tile the network's
 * output is compared with it. A sampled tile keeps the NLM result when the
 * RMS of (network - NLM) over the tile exceeds limit * sigma (sigma = h / 1.5,
 * the noise level the strength implies), when the network's output is not
 * finite, or when the residual check failed it; otherwise it keeps the
 * network's output. Tile t (row-major in the NLM tile grid) is sampled when
 * dsgpu_cnn_judge_tile(seed, fraction, t) is 1, so the sample is the same
 * for device-buffer and band-pipelined (DSGPU_HOST) calls. fraction in
 * [0, 1]; 0 (the default) turns the judge off. Applies to dsgpu_cnn_denoise
 * and dsgpu_develop_u16_cnn; its cost is NLM on `fraction` of the tiles. */
int dsgpu_cnn_set_judge(dsgpu_ctx* ctx, dsgpu_cnn* net, float fraction, float limit, unsigned seed);
/* The judge's record of the last call: tiles sampled, tiles that kept NLM,
 * and the largest and the root-mean-square (over the sampled tiles) of the
 * network's per-tile RMS error against NLM, in units of sigma. */
int dsgpu_cnn_judge_stats(dsgpu_ctx* ctx, dsgpu_cnn* net, int* judged, int* failed, float* max_rms_over_sigma,
                          float* rms_over_sigma);
/* 1 when tile `tile_index` is in the judge's sample for (seed, fraction), else 0. */
int dsgpu_cnn_judge_tile(unsigned seed, float fraction, int tile_index);
/* u16 raw -> normalise -> RCD -> learned denoise with NLM fallback (the
 * learned counterpart of dsgpu_develop_u16; w or h < 16 gives
 * DSGPU_ERR_UNSUPPORTED, search < 1 DSGPU_ERR_ARG). With DSGPU_HOST the call
 * runs as a band pipeline: chunked upload, RCD and the network in row bands
 * (each band with the network's 18-row halo), copies back overlapped with
 * the next band; the result is bit-identical to the device-buffer call. */
int dsgpu_develop_u16_cnn(dsgpu_ctx* ctx, dsgpu_cnn* net, const uint16_t* raw, int w, int h, size_t pitch_elems,
                          const uint8_t cfa[4], float black, const float white[3], const float mul[3],
                          float h_param, int search, int patch, float tau, float* out_rgb, float* out_clip,
                          unsigned flags);

#ifdef __cplusplus
}
#endif
#endif /* DSGPU_H */
