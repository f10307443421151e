// Non-local means (enhance.rs:36-72) as one tiled kernel.
//
// The reference loops over the (2S+1)^2 search offsets; for each it builds
// the squared-difference plane against the clamped shifted plane (:49-53),
// box-filters it with a clamped separable box of radius P (:54,
// image.rs:269-313), turns the mean distance into a weight exp(-d/h^2)
// (:58) and accumulates weight*sample and weight (:59-60); the result is
// a/max(s,1e-12) (:71).
//
// B200 design. Per (pixel, channel, offset) update the kernel needs one ex2
// and ~8 FP32 operations; what binds is the shared-memory traffic of the
// separable box sums (one 128-byte wavefront per clock per SM), so the
// layout minimises shared bytes per update:
//  - one CTA (128 threads, four per SM, so that the CTAs' row phases, heavy
//    on shared stores, overlap the others' column phases, heavy on ex2) owns
//    a 16-wide tile of one channel, TY = 64 - 2P rows tall, so that the
//    horizontal box sums it needs cover exactly 64 rows; the three channels
//    of a tile are adjacent in launch order, so the interleaved RGB lines
//    they all read come from L2 (the batch kernels run the same body on
//    32-wide tiles and 256 threads, two CTAs per SM);
//  - the staged plane's pitch is sized for search radius 10 or for the
//    maximum, whichever the call needs, so that four CTAs fit at S <= 10;
//  - the tile plus its S+P+1 halo is staged once in shared memory, PRE-SCALED
//    by sigma = sqrt(log2(e) / (h^2 (2P+1)^2)): the squared differences of
//    scaled samples sum directly to the ex2 exponent, so a weight costs one
//    ex2 and no multiply;
//  - offsets are processed in blocks of 4 dx x 2 dy (8 planes of H):
//    phase A: thread t owns H row t%64, a 16-wide segment and one dy of the
//      block (its 22 centre samples kept in registers for the whole kernel)
//      and forms the horizontal running sums of all four dx from ONE
//      25-sample load of the shifted row;
//    phase B: thread t owns one column, a quarter of the tile's rows and two
//      of the four dx, sums 2P+1 H rows as a running vertical sum, and
//      accumulates; the shifted sample of row r at dy0+1 is the one of row
//      r+1 at dy0, so one column load serves both dy. The two dx halves of a
//      pixel's sums meet once, at the end;
//  - all shared pitches are odd, so a warp's 32 rows (phase A) hit 32
//    distinct banks; in phase B a 16-wide tile's warp is two half-warps on
//    neighbouring H planes, whose stride is 16 (mod 32) words.
// Clamped edges: the staged copy is loaded at clamped coordinates, so the
// shifted sample p_clamped(x+o) is a plain shared read; the reference's box
// filter clamps the DIFFERENCE plane, so H rows are clamped per row and, in
// tiles whose patch window leaves the image, columns per element.
#include <cuda_fp16.h>

#include <type_traits>

#include "internal.cuh"
#include "nlm_tile.cuh"

namespace {

using namespace nlmk;

// grid: (tiles_x * C, tile rows); block x = tile_x * C + channel, so the C
// channels of a tile run side by side
template <int P, bool F16, int SM>
__global__ void __launch_bounds__(NLM_THREADS, 4) nlm_tile_kernel(const float* __restrict__ in, int W, int H, int C,
                                                                  int S, float sigma, const float* __restrict__ h_dev,
                                                                  float norm2_log2e,
                                                                  const unsigned char* __restrict__ tile_flags,
                                                                  float* __restrict__ out, int ty0) {
  const int ty = blockIdx.y + ty0;  // tile row (a launch may cover a band of tile rows)
  const int tx = blockIdx.x / C, ch = blockIdx.x - tx * C;
  const int tiles_x = gridDim.x / C;
  // tile-list mode (the learned path's fallback): only flagged tiles run
  if (tile_flags && !tile_flags[ty * tiles_x + tx]) return;
  if (h_dev) {  // strength computed on the device (enhance.rs:40 floor included)
    const float hh = *h_dev;
    sigma = sqrtf(norm2_log2e / fmaxf(hh * hh, 1e-12f));
  }
  extern __shared__ float4 smem4[];
  nlm_tile<P, F16, SM>(in, W, H, C, S, sigma, out, tx, ty, ch, reinterpret_cast<float*>(smem4));
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void stamp_kernel(unsigned long long* t) { *t = globaltimer_ns(); }

// Persistent NLM over the tiles of all frames (3 channels each). When the
// last tile of frame f is done, stamps[f] = the device clock (ns), so the
// host can report per-frame completion times.
template <int P>
__global__ void __launch_bounds__(NLM_BATCH_THREADS, 2) nlm_batch_kernel(const ds_batch_frame* __restrict__ frames, int n,
                                                                   int total, int S, unsigned* __restrict__ done,
                                                                   unsigned long long* __restrict__ stamps) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    int lo = 0, hi = n - 1;  // the last frame whose first tile is <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (frames[mid].nlm_tile0 <= t) lo = mid;
      else hi = mid - 1;
    }
    const ds_batch_frame& F = frames[lo];
    const int per = F.nlm_tiles_x * F.nlm_tiles_y;
    const int local = t - F.nlm_tile0;
    const int ch = local / per, r = local - ch * per;
    const int ty = r / F.nlm_tiles_x, tx = r - ty * F.nlm_tiles_x;
    __syncthreads();  // the previous tile is done with shared memory
    nlm_tile<P, false, DSGPU_NLM_MAX_SEARCH, NLM_BATCH_TX>(F.rgb, F.w, F.h, 3, S, F.sigma, F.out, tx, ty, ch, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(&done[lo], 1u) + 1u == (unsigned)(3 * per)) stamps[lo] = globaltimer_ns();
    }
  }
}

template <int P>
cudaError_t launch_nlm_batch_p(cudaStream_t st, const ds_batch_frame* frames, int n, int total, int S, int grid,
                               unsigned* done, unsigned long long* stamps) {
  const size_t smem = nlm_smem_bytes(S, P, false, DSGPU_NLM_MAX_SEARCH, NLM_BATCH_TX);
  cudaError_t e = cudaFuncSetAttribute(nlm_batch_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  nlm_batch_kernel<P><<<grid, NLM_BATCH_THREADS, smem, st>>>(frames, n, total, S, done, stamps);
  return cudaGetLastError();
}

// tile rows [ty0, ty1) (ty1 < 0: to the last)
template <int P, bool F16>
cudaError_t launch_nlm_p(cudaStream_t st, const float* in, int w, int h, int C, int S, float sigma,
                         const float* h_dev, float norm2_log2e, const unsigned char* flags, float* out, int ty0,
                         int ty1) {
  constexpr int TY = HRW - 2 * P;
  const int tiles_y = (h + TY - 1) / TY;
  if (ty1 < 0 || ty1 > tiles_y) ty1 = tiles_y;
  if (ty0 >= ty1) return cudaSuccess;
  dim3 grid((w + NLM_TX - 1) / NLM_TX * C, ty1 - ty0);
  if (S <= 10) {
    const size_t smem = nlm_smem_bytes(S, P, F16, 10);
    cudaError_t e =
        cudaFuncSetAttribute(nlm_tile_kernel<P, F16, 10>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    nlm_tile_kernel<P, F16, 10><<<grid, NLM_THREADS, smem, st>>>(in, w, h, C, S, sigma, h_dev, norm2_log2e, flags,
                                                                out, ty0);
  } else {
    const size_t smem = nlm_smem_bytes(S, P, F16);
    cudaError_t e = cudaFuncSetAttribute(nlm_tile_kernel<P, F16, DSGPU_NLM_MAX_SEARCH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    nlm_tile_kernel<P, F16, DSGPU_NLM_MAX_SEARCH><<<grid, NLM_THREADS, smem, st>>>(in, w, h, C, S, sigma, h_dev,
                                                                                  norm2_log2e, flags, out, ty0);
  }
  return cudaGetLastError();
}

}  // namespace

namespace {

template <bool F16>
cudaError_t dispatch_nlm_t(cudaStream_t st, const float* in, int w, int h, int C, int S, int P, float sigma,
                           const float* h_dev, float* out, const unsigned char* flags, int ty0, int ty1) {
  const float norm = P == 0 ? 1.0f : 1.0f / (float)(2 * P + 1);
  const float n2l = norm * norm * 1.4426950408889634f;
  switch (P) {
    case 0: return launch_nlm_p<0, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 1: return launch_nlm_p<1, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 2: return launch_nlm_p<2, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 3: return launch_nlm_p<3, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 4: return launch_nlm_p<4, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 5: return launch_nlm_p<5, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 6: return launch_nlm_p<6, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    case 7: return launch_nlm_p<7, F16>(st, in, w, h, C, S, sigma, h_dev, n2l, flags, out, ty0, ty1);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t dispatch_nlm(cudaStream_t st, const float* in, int w, int h, int C, int S, int P, float sigma,
                         const float* h_dev, float* out, const unsigned char* flags = nullptr, bool f16 = false,
                         int ty0 = 0, int ty1 = -1) {
  return f16 ? dispatch_nlm_t<true>(st, in, w, h, C, S, P, sigma, h_dev, out, flags, ty0, ty1)
             : dispatch_nlm_t<false>(st, in, w, h, C, S, P, sigma, h_dev, out, flags, ty0, ty1);
}

}  // namespace

cudaError_t ds_launch_nlm(cudaStream_t st, const float* in, int w, int h, int channels, float h_param, int search,
                          int patch, float* out, bool fp16_staging) {
  if (search == 0) {  // only the centre offset: weight 1, out = p exactly (enhance.rs:41-71)
    return cudaMemcpyAsync(out, in, (size_t)w * h * channels * sizeof(float), cudaMemcpyDeviceToDevice, st);
  }
  // enhance.rs:40: h2 = max(h*h, 1e-12) in f32; box_blur's norm is 1/(2r+1)
  // in f32, applied once per pass (image.rs:274, 285, 307). The weight is
  // exp(-sum d^2 * norm^2 / h2) = 2^-(sum (sigma d)^2).
  const float h2 = fmaxf(h_param * h_param, 1e-12f);
  const float norm = patch == 0 ? 1.0f : 1.0f / (float)(2 * patch + 1);
  const double sig2 = (double)norm * (double)norm / (double)h2 * 1.4426950408889634;
  return dispatch_nlm(st, in, w, h, channels, search, patch, (float)sqrt(sig2), nullptr, out, nullptr, fp16_staging);
}

// NLM of the tile rows [ty0, ty1) only (the rows ty0*(64-2P) .. of the output)
cudaError_t ds_launch_nlm_rows(cudaStream_t st, const float* in, int w, int h, int channels, float h_param,
                               int search, int patch, int ty0, int ty1, float* out, bool fp16_staging) {
  if (search <= 0) return cudaErrorInvalidValue;
  return dispatch_nlm(st, in, w, h, channels, search, patch, ds_nlm_sigma(h_param, patch), nullptr, out, nullptr,
                      fp16_staging, ty0, ty1);
}

// NLM tile geometry (the fallback's flag grid): tiles_x x tiles_y of 64 x (64 - 2P)
void ds_nlm_tile_grid(int w, int h, int patch, int* tiles_x, int* tiles_y, int* tile_w, int* tile_h) {
  const int ty = HRW - 2 * patch;
  *tile_w = NLM_TX;
  *tile_h = ty;
  *tiles_x = (w + NLM_TX - 1) / NLM_TX;
  *tiles_y = (h + ty - 1) / ty;
}

// The batch kernels' NLM tile grid (their tiles are NLM_BATCH_TX wide).
void ds_nlm_batch_tile_grid(int w, int h, int patch, int* tiles_x, int* tiles_y) {
  const int ty = HRW - 2 * patch;
  *tiles_x = (w + NLM_BATCH_TX - 1) / NLM_BATCH_TX;
  *tiles_y = (h + ty - 1) / ty;
}

// NLM on the flagged tiles only (flags[tiles_y][tiles_x], 1 = recompute).
cudaError_t ds_launch_nlm_tiles(cudaStream_t st, const float* in, int w, int h, int channels, float h_param,
                                int search, int patch, const unsigned char* flags, float* out) {
  if (search <= 0) return cudaErrorInvalidValue;
  const float h2 = fmaxf(h_param * h_param, 1e-12f);
  const float norm = patch == 0 ? 1.0f : 1.0f / (float)(2 * patch + 1);
  const double sig2 = (double)norm * (double)norm / (double)h2 * 1.4426950408889634;
  return dispatch_nlm(st, in, w, h, channels, search, patch, (float)sqrt(sig2), nullptr, out, flags);
}

// NLM on the flagged tiles of tile rows [ty0, ty1) only.
cudaError_t ds_launch_nlm_tiles_rows(cudaStream_t st, const float* in, int w, int h, int channels, float h_param,
                                     int search, int patch, const unsigned char* flags, int ty0, int ty1,
                                     float* out) {
  if (search <= 0) return cudaErrorInvalidValue;
  return dispatch_nlm(st, in, w, h, channels, search, patch, ds_nlm_sigma(h_param, patch), nullptr, out, flags, false,
                      ty0, ty1);
}

// The same with the strength h read from device memory (search > 0).
cudaError_t ds_launch_nlm_dev_h(cudaStream_t st, const float* in, int w, int h, int channels, const float* h_dev,
                                int search, int patch, float* out) {
  if (search == 0)
    return cudaMemcpyAsync(out, in, (size_t)w * h * channels * sizeof(float), cudaMemcpyDeviceToDevice, st);
  return dispatch_nlm(st, in, w, h, channels, search, patch, 1.0f, h_dev, out);
}

// NLM pre-scale of strength h (the sigma ds_launch_nlm computes)
float ds_nlm_sigma(float h_param, int patch) {
  const float h2 = fmaxf(h_param * h_param, 1e-12f);
  const float norm = patch == 0 ? 1.0f : 1.0f / (float)(2 * patch + 1);
  const double sig2 = (double)norm * (double)norm / (double)h2 * 1.4426950408889634;
  return (float)sqrt(sig2);
}

cudaError_t ds_launch_stamp(cudaStream_t st, unsigned long long* t) {
  stamp_kernel<<<1, 1, 0, st>>>(t);
  return cudaGetLastError();
}

cudaError_t ds_launch_nlm_batch(cudaStream_t st, const ds_batch_frame* frames, int n, int total_tiles, int search,
                                int patch, int grid, unsigned* done, unsigned long long* stamps) {
  if (n <= 0 || total_tiles <= 0) return cudaSuccess;
  if (search <= 0 || search > DSGPU_NLM_MAX_SEARCH) return cudaErrorInvalidValue;
  switch (patch) {
    case 0: return launch_nlm_batch_p<0>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 1: return launch_nlm_batch_p<1>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 2: return launch_nlm_batch_p<2>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 3: return launch_nlm_batch_p<3>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 4: return launch_nlm_batch_p<4>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 5: return launch_nlm_batch_p<5>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 6: return launch_nlm_batch_p<6>(st, frames, n, total_tiles, search, grid, done, stamps);
    case 7: return launch_nlm_batch_p<7>(st, frames, n, total_tiles, search, grid, done, stamps);
    default: return cudaErrorInvalidValue;
  }
}
