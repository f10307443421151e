// Non-local means (enhance.rs:36-72) as one tiled kernel.
//
// The reference loops over the (2S+1)^2 search offsets; for each it builds
// the squared-difference plane against the clamped shifted plane (:49-53),
// box-filters it with a clamped separable box of radius P (:54,
// image.rs:269-313), turns the mean distance into a weight exp(-d/h^2)
// (:58) and accumulates weight*sample and weight (:59-60); the result is
// a/max(s,1e-12) (:71).
//
// B200 design. The kernel is bound by shared-memory bandwidth (one 128-byte
// wavefront per clock per SM) long before the ex2 unit (16/clock/SM), so the
// layout minimises shared bytes per (pixel, channel, offset) update:
//  - one CTA owns a 64-wide tile of one channel, TY = 64 - 2P rows tall, so
//    that the horizontal box sums it needs cover exactly 64 rows;
//  - the tile plus its S+P+1 halo is staged once in shared memory, PRE-SCALED
//    by sigma = sqrt(log2(e) / (h^2 (2P+1)^2)): the squared differences of
//    scaled samples sum directly to the ex2 exponent, so a weight costs one
//    ex2 and no multiply;
//  - offsets are processed in 2x2 blocks {dx0, dx0+1} x {dy0, dy0+1}:
//    phase A: thread t owns H row t%64 (a 16-wide segment, its 22 centre
//      samples kept in registers for the whole kernel) and forms the
//      horizontal running sums for the block's offsets from one 23-sample
//      load of each shifted row (so one load serves both dx);
//    phase B: thread t owns one column and a quarter of the tile's rows,
//      sums 2P+1 H rows as a running vertical sum, and accumulates; the
//      shifted sample of row r at dy0+1 is the one of row r+1 at dy0, so one
//      column load serves both dy;
//  - all shared pitches are odd, so a warp's 32 rows (phase A) or 32 columns
//    (phase B) hit 32 distinct banks.
// Clamped edges: the staged copy is loaded at clamped coordinates, so the
// shifted sample p_clamped(x+o) is a plain shared read; the reference's box
// filter clamps the DIFFERENCE plane, so H rows are clamped per row and, in
// tiles whose patch window leaves the image, columns per element.
#include <cuda_fp16.h>

#include <type_traits>

#include "internal.cuh"

namespace {

constexpr int NLM_THREADS = 256;
constexpr int TX = 64;   // tile width
constexpr int HRW = 64;  // H rows per offset (TY + 2P)
constexpr int SEG = 16;  // phase-A segment width
constexpr int HP = TX + 1;  // odd H pitch

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr int HBR = HRW + 4;  // H rows allocated: phase B of the last quarter reads past row 63

// Plane pitch: odd and fixed per P (sized for the largest search radius) so
// that every shared address offset is a compile-time constant.
__host__ __device__ constexpr int nlm_pitch(int P) { return (TX + 2 * (DSGPU_NLM_MAX_SEARCH + P + 1)) | 1; }

struct NlmGeom {
  int R, PW, PH, PHA;  // halo, region width, region height, allocated rows
};

__host__ __device__ inline NlmGeom nlm_geom(int S, int P) {
  NlmGeom g;
  const int TY = HRW - 2 * P;
  g.R = S + P + 1;
  g.PW = TX + 2 * g.R;
  g.PH = TY + 2 * g.R;
  g.PHA = g.PH + 4;  // phase B of the last quarter reads up to 3 rows past the region
  return g;
}

// plane bytes (f32, or f16 when staged in half precision), rounded to 16
size_t nlm_plane_bytes(int S, int P, bool f16) {
  const NlmGeom g = nlm_geom(S, P);
  return ((size_t)nlm_pitch(P) * g.PHA * (f16 ? 2 : 4) + 15) / 16 * 16;
}

size_t nlm_smem_bytes(int S, int P, bool f16 = false) {
  return nlm_plane_bytes(S, P, f16) + (size_t)4 * HBR * HP * sizeof(float);
}

__device__ __forceinline__ float ldp(const float* p) { return *p; }
__device__ __forceinline__ float ldp(const __half* p) { return __half2float(*p); }
__device__ __forceinline__ void stp(float* p, float v) { *p = v; }
__device__ __forceinline__ void stp(__half* p, float v) { *p = __float2half_rn(v); }

// One 64 x (64 - 2P) tile (tile_x, tile_y) of channel ch of a W x H x C
// image; smem holds nlm_smem_bytes(S, P, F16) bytes.
// F16 (the precision variant): the pre-scaled plane is staged in half
// precision, centred on the tile's centre sample (NLM weights depend only on
// differences, so the offset costs nothing there and keeps the half-precision
// error of the staged values small; it is added back to the result), while
// distances, weights and sums stay in FP32 and the weight sum (the
// normalisation) is accumulated with Kahan compensation.
template <int P, bool F16 = false>
__device__ __forceinline__ void nlm_tile(const float* __restrict__ in, int W, int H, int C, int S, float sigma,
                                         float* __restrict__ out, int tile_x, int tile_y, int ch, float* smem) {
  using T = typename std::conditional<F16, __half, float>::type;
  constexpr int TY = HRW - 2 * P;
  constexpr int DW = SEG + 2 * P;  // differences per phase-A segment
  constexpr int RB = (TY + 3) / 4; // phase-B rows per thread (a quarter of the tile)
  constexpr int PP = nlm_pitch(P);
  const NlmGeom g = nlm_geom(S, P);
  T* PL = reinterpret_cast<T*>(smem);  // scaled plane, pitch PP
  float* HB = reinterpret_cast<float*>(reinterpret_cast<char*>(smem) +
                                       ((size_t)PP * g.PHA * sizeof(T) + 15) / 16 * 16);  // 4 offsets x HBR rows x HP

  const int X0 = tile_x * TX, Y0 = tile_y * TY;
  const int tid = threadIdx.x;
  const int ox0 = X0 - g.R, oy0 = Y0 - g.R;  // global site of plane (0,0)

  float off = 0.f;  // F16: the tile's centre sample
  if (F16) off = in[((size_t)clampi(Y0 + TY / 2, 0, H - 1) * W + clampi(X0 + TX / 2, 0, W - 1)) * C + ch];
  for (int i = tid; i < g.PW * g.PH; i += NLM_THREADS) {
    const int ly = i / g.PW, lx = i - ly * g.PW;
    const int gx = clampi(ox0 + lx, 0, W - 1), gy = clampi(oy0 + ly, 0, H - 1);
    const float v = in[((size_t)gy * W + gx) * C + ch];
    stp(&PL[ly * PP + lx], F16 ? (v - off) * sigma : v * sigma);
  }
  for (int i = tid; i < (g.PHA - g.PH) * PP; i += NLM_THREADS) stp(&PL[g.PH * PP + i], 0.f);

  // ---- phase-A role: H row `arow` (tile row arow - P), segment at ax0
  const int arow = tid & (HRW - 1);
  const int ax0 = (tid >> 6) * SEG;
  const int aprow = clampi(Y0 + arow - P, 0, H - 1) - oy0;  // plane row of the clamped H row
  const bool xin = (X0 - P >= 0) && (X0 + TX + P <= W);
  const int acol0 = ax0 - P + g.R;  // plane column of difference 0 (interior tiles)
  // ---- phase-B role: column bcol, rows [brow0, brow0 + RB) (clipped to TY)
  const int bcol = tid & (TX - 1);
  const int brow0 = (tid >> 6) * RB;

  __syncthreads();
  float pv[DW];  // centre samples of this thread's phase-A segment
#pragma unroll
  for (int k = 0; k < DW; k++) {
    const int col = xin ? acol0 + k : clampi(X0 + ax0 - P + k, 0, W - 1) - ox0;
    pv[k] = ldp(&PL[aprow * PP + col]);
  }
  float a[RB], s[RB], cs[F16 ? RB : 1];  // cs: Kahan compensation of s (F16)
#pragma unroll
  for (int r = 0; r < RB; r++) {
    a[r] = 0.f;
    s[r] = 0.f;
    if (F16) cs[r] = 0.f;
  }

  // One 2x2 block of offsets {dx0, dx0+1} x {dy0, dy0+NJ-1}.
  auto block = [&](int dx0, int dy0, auto nj_tag) {
    constexpr int NJ = decltype(nj_tag)::value;
    // phase A: horizontal sums, stored NEGATED (-sum d^2) so that phase B's
    // vertical sum is the ex2 argument itself
#pragma unroll
    for (int j = 0; j < NJ; j++) {
      const T* qrow = PL + (aprow + dy0 + j) * PP + dx0;
      float d0[DW], d1[DW];
      if (xin) {
        float q[DW + 1];
#pragma unroll
        for (int k = 0; k <= DW; k++) q[k] = ldp(&qrow[acol0 + k]);
#pragma unroll
        for (int k = 0; k < DW; k++) {
          d0[k] = pv[k] - q[k];
          d1[k] = pv[k] - q[k + 1];
        }
      } else {
#pragma unroll
        for (int k = 0; k < DW; k++) {
          const int col = clampi(X0 + ax0 - P + k, 0, W - 1) - ox0;
          d0[k] = pv[k] - ldp(&qrow[col]);
          d1[k] = pv[k] - ldp(&qrow[col + 1]);
        }
      }
      float h0 = 0.f, h1 = 0.f;
#pragma unroll
      for (int k = 0; k <= 2 * P; k++) {
        h0 = fmaf(-d0[k], d0[k], h0);
        h1 = fmaf(-d1[k], d1[k], h1);
      }
      float* H0 = HB + (j * 2 + 0) * (HBR * HP) + arow * HP + ax0;
      float* H1 = HB + (j * 2 + 1) * (HBR * HP) + arow * HP + ax0;
      H0[0] = h0;
      H1[0] = h1;
#pragma unroll
      for (int k = 1; k < SEG; k++) {
        h0 = fmaf(-d0[k + 2 * P], d0[k + 2 * P], h0);
        h0 = fmaf(d0[k - 1], d0[k - 1], h0);
        h1 = fmaf(-d1[k + 2 * P], d1[k + 2 * P], h1);
        h1 = fmaf(d1[k - 1], d1[k - 1], h1);
        H0[k] = h0;
        H1[k] = h1;
      }
    }
    __syncthreads();
    // phase B: vertical sums, weights, accumulation for (dx0 + i, dy0 + j)
#pragma unroll
    for (int i = 0; i < 2; i++) {
      if (dx0 + i <= S) {  // false only for the dx tail of an odd search width
        const T* qc = PL + (brow0 + g.R + dy0) * PP + bcol + g.R + dx0 + i;
        float qv[RB + NJ - 1];
#pragma unroll
        for (int r = 0; r < RB + NJ - 1; r++) qv[r] = ldp(&qc[r * PP]);
#pragma unroll
        for (int j = 0; j < NJ; j++) {
          const float* hc = HB + (j * 2 + i) * (HBR * HP) + brow0 * HP + bcol;
          float hv[RB + 2 * P];
#pragma unroll
          for (int r = 0; r < RB + 2 * P; r++) hv[r] = hc[r * HP];
          float v = 0.f;
#pragma unroll
          for (int r = 0; r <= 2 * P; r++) v += hv[r];
#pragma unroll
          for (int r = 0; r < RB; r++) {
            if (r > 0) v = v + hv[r + 2 * P] - hv[r - 1];
            const float wgt = ex2(v);
            a[r] = fmaf(wgt, qv[r + j], a[r]);
            if (F16) {  // Kahan: s[r] + cs[r] carries the sum of weights
              const float y = wgt - cs[r];
              const float t = s[r] + y;
              cs[r] = (t - s[r]) - y;
              s[r] = t;
            } else {
              s[r] += wgt;
            }
          }
        }
      }
    }
    __syncthreads();
  };

  int dy0 = -S;
  for (; dy0 + 1 <= S; dy0 += 2)
    for (int dx0 = -S; dx0 <= S; dx0 += 2) block(dx0, dy0, std::integral_constant<int, 2>{});
  if (dy0 <= S)  // the dy tail of an odd search width
    for (int dx0 = -S; dx0 <= S; dx0 += 2) block(dx0, dy0, std::integral_constant<int, 1>{});

  const float inv_sigma = 1.0f / sigma;
#pragma unroll
  for (int r = 0; r < RB; r++) {
    const int y = brow0 + r;
    const int gx = X0 + bcol, gy = Y0 + y;
    if (y < TY && gx < W && gy < H) {
      const float o = __fdiv_rn(a[r] * inv_sigma, fmaxf(F16 ? s[r] - cs[r] : s[r], 1e-12f));
      out[((size_t)gy * W + gx) * C + ch] = F16 ? o + off : o;
    }
  }
}

template <int P, bool F16>
__global__ void __launch_bounds__(NLM_THREADS, 2) nlm_tile_kernel(const float* __restrict__ in, int W, int H, int C,
                                                                  int S, float sigma, const float* __restrict__ h_dev,
                                                                  float norm2_log2e,
                                                                  const unsigned char* __restrict__ tile_flags,
                                                                  float* __restrict__ out, int ty0) {
  const int ty = blockIdx.y + ty0;  // tile row (a launch may cover a band of tile rows)
  // tile-list mode (the learned path's fallback): only flagged tiles run
  if (tile_flags && !tile_flags[ty * gridDim.x + blockIdx.x]) return;
  if (h_dev) {  // strength computed on the device (enhance.rs:40 floor included)
    const float hh = *h_dev;
    sigma = sqrtf(norm2_log2e / fmaxf(hh * hh, 1e-12f));
  }
  extern __shared__ float4 smem4[];
  nlm_tile<P, F16>(in, W, H, C, S, sigma, out, blockIdx.x, ty, blockIdx.z, reinterpret_cast<float*>(smem4));
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
__global__ void __launch_bounds__(NLM_THREADS, 2) nlm_batch_kernel(const ds_batch_frame* __restrict__ frames, int n,
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
    nlm_tile<P>(F.rgb, F.w, F.h, 3, S, F.sigma, F.out, tx, ty, ch, smem);
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
  const size_t smem = nlm_smem_bytes(S, P);
  cudaError_t e = cudaFuncSetAttribute(nlm_batch_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  nlm_batch_kernel<P><<<grid, NLM_THREADS, smem, st>>>(frames, n, total, S, done, stamps);
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
  const size_t smem = nlm_smem_bytes(S, P, F16);
  cudaError_t e =
      cudaFuncSetAttribute(nlm_tile_kernel<P, F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((w + TX - 1) / TX, ty1 - ty0, C);
  nlm_tile_kernel<P, F16><<<grid, NLM_THREADS, smem, st>>>(in, w, h, C, S, sigma, h_dev, norm2_log2e, flags, out,
                                                            ty0);
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
  *tile_w = TX;
  *tile_h = ty;
  *tiles_x = (w + TX - 1) / TX;
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
