// The learned stand-in for NLM: a residual CNN of 8 conv3x3 layers
// (7 -> 48 -> ... -> 48 -> 3, ReLU between; dilations 1,2,3,4,3,2,1,1),
// input = demosaiced RGB split into its 3x3 local mean and the remainder
// (cnn_input_px) plus the NLM strength, output = input RGB + network output.
// It is trained on the GPU to reproduce plain NLM (enhance.rs:36-72) and
// runs with NLM as the per-tile fallback.
//
// Tensor-core kernels: BF16 operands, FP32 accumulation (mma.sync m16n8k16 fed
// by ldmatrix from shared memory). Activations are NHWC bf16 with the channel
// count padded to a multiple of 16 (input 16, hidden 48; the last layer's
// gradient 16). Every conv is an implicit GEMM: M = 16 output pixels of one
// tile row per warp, N = output channels, K = 9 taps x input channels.
//   forward       conv_fwd_kernel<CIN, COUT, EPI_RELU / EPI_RESID>
//   data gradient conv_fwd_kernel with the tap-flipped, transposed weights and
//                 EPI_MASK (the ReLU mask of the layer below)
//   weight grad   conv_wgrad_kernel<CIN, COUTW>: M = out channels, N = in
//                 channels, K = pixels; per-CTA partial sums reduced in a
//                 fixed order (deterministic)
// These form the mma.sync training engine, kept as the cross-check of the
// default tcgen05 engine, whose forward, data-gradient and weight-gradient
// kernels (conv_tc_kernel, wgrad_tc_kernel) are in k_cnn_tc.cu.
#include <cuda_bf16.h>

#include <cstring>
#include <vector>

#include "internal.cuh"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int CT_W = 16, CT_H = 8;             // output tile: 8 rows of 16 pixels
// staged input tile of a conv with dilation D: the output tile plus a D-pixel halo
__host__ __device__ constexpr int ct_xw(int D) { return CT_W + 2 * D; }
__host__ __device__ constexpr int ct_xh(int D) { return CT_H + 2 * D; }
constexpr int CNN_THREADS = 256;

enum { EPI_RELU = 0, EPI_MASK = 1, EPI_RESID = 2 };

// shared-memory row stride (bytes) for c bf16 channels: an odd number of
// 16-byte chunks, so the 8 rows of an ldmatrix phase hit 8 distinct chunks
__host__ __device__ constexpr int row_stride(int c) { return c * 2 + 16; }

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(unsigned a, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void ldsm_x2(unsigned a, unsigned& r0, unsigned& r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned a, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void mma16816(float* d, unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct TileIdx {
  int b, x0, y0;
};
__device__ __forceinline__ TileIdx tile_of(int t, int tiles_x, int tiles_y) {
  TileIdx r;
  const int per = tiles_x * tiles_y;
  r.b = t / per;
  const int q = t - r.b * per;
  const int ty = q / tiles_x;
  r.x0 = (q - ty * tiles_x) * CT_W;
  r.y0 = ty * CT_H;
  return r;
}

// stage an NHWC tile (zero outside the image)
template <int C, int PW, int PH>
__device__ __forceinline__ void stage_tile(unsigned char* dst, const bf16* __restrict__ src, int b, int H, int W,
                                           int x0, int y0) {
  constexpr int CH = C * 2 / 16, RS = row_stride(C);
  for (int i = threadIdx.x; i < PH * PW * CH; i += CNN_THREADS) {
    const int pix = i / CH, ch = i - pix * CH;
    const int py = pix / PW, px = pix - py * PW;
    const int gy = y0 + py, gx = x0 + px;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (gy >= 0 && gy < H && gx >= 0 && gx < W)
      v = reinterpret_cast<const uint4*>(src + (((size_t)b * H + gy) * W + gx) * C)[ch];
    *reinterpret_cast<uint4*>(dst + pix * RS + ch * 16) = v;
  }
}

template <int CIN, int COUT, int EPI, int D>
__global__ void __launch_bounds__(CNN_THREADS) conv_fwd_kernel(const bf16* __restrict__ x, int B, int H, int W,
                                                               const bf16* __restrict__ wt,
                                                               const float* __restrict__ bias, bf16* __restrict__ y,
                                                               const bf16* __restrict__ mask,
                                                               const float* __restrict__ resid,
                                                               float* __restrict__ yf) {
  static_assert(CIN % 16 == 0 && COUT % 8 == 0, "channel padding");
  constexpr int RSX = row_stride(CIN), RSW = row_stride(CIN), NT = COUT / 8;
  extern __shared__ __align__(16) unsigned char sm[];
  unsigned char* ws = sm;                    // [9][COUT] rows of CIN bf16
  unsigned char* xs = sm + 9 * COUT * RSW;   // [ct_xh(D)][ct_xw(D)] pixels of CIN bf16
  constexpr int XW = ct_xw(D), XH = ct_xh(D);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  {
    constexpr int CH = CIN * 2 / 16;
    for (int i = tid; i < 9 * COUT * CH; i += CNN_THREADS) {
      const int row = i / CH, ch = i - row * CH;
      *reinterpret_cast<uint4*>(ws + row * RSW + ch * 16) = reinterpret_cast<const uint4*>(wt)[i];
    }
  }
  const int tiles_x = (W + CT_W - 1) / CT_W, tiles_y = (H + CT_H - 1) / CT_H;
  const int ntiles = B * tiles_x * tiles_y;
  const int g = lane >> 2, c = lane & 3;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileIdx ti = tile_of(t, tiles_x, tiles_y);
    __syncthreads();  // weights staged / previous tile consumed
    stage_tile<CIN, XW, XH>(xs, x, ti.b, H, W, ti.x0 - D, ti.y0 - D);
    __syncthreads();
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
      const int ky = tap / 3, kx = tap % 3;
#pragma unroll
      for (int kc = 0; kc < CIN / 16; kc++) {
        unsigned a0, a1, a2, a3;
        ldsm_x4(smem_u32(xs + ((warp + ky * D) * XW + (lane & 15) + kx * D) * RSX + (kc * 16 + (lane >> 4) * 8) * 2),
                a0, a1, a2, a3);
#pragma unroll
        for (int j = 0; j + 1 < NT; j += 2) {
          const int co = (j + (lane >> 4)) * 8 + (lane & 7);
          unsigned b0, b1, b2, b3;
          ldsm_x4(smem_u32(ws + (tap * COUT + co) * RSW + (kc * 16 + ((lane >> 3) & 1) * 8) * 2), b0, b1, b2, b3);
          mma16816(acc[j], a0, a1, a2, a3, b0, b1);
          mma16816(acc[j + 1], a0, a1, a2, a3, b2, b3);
        }
        if (NT & 1) {
          const int co = (NT - 1) * 8 + (lane & 7);
          unsigned b0, b1;
          ldsm_x2(smem_u32(ws + (tap * COUT + co) * RSW + (kc * 16 + ((lane >> 3) & 1) * 8) * 2), b0, b1);
          mma16816(acc[NT - 1], a0, a1, a2, a3, b0, b1);
        }
      }
    }
    // epilogue: rows g and g+8 of the warp's 16 pixels, channels 2c, 2c+1 of each n8 tile
    const int gy = ti.y0 + warp;
    if (gy < H) {
#pragma unroll
      for (int half = 0; half < 2; half++) {
        const int gx = ti.x0 + g + half * 8;
        if (gx >= W) continue;
        const size_t pix = ((size_t)ti.b * H + gy) * W + gx;
#pragma unroll
        for (int j = 0; j < NT; j++) {
          const int co = j * 8 + 2 * c;
          float v0 = acc[j][half * 2], v1 = acc[j][half * 2 + 1];
          if (EPI == EPI_RELU) {
            v0 = fmaxf(v0 + bias[co], 0.f);
            v1 = fmaxf(v1 + bias[co + 1], 0.f);
            *reinterpret_cast<__nv_bfloat162*>(y + pix * COUT + co) = __floats2bfloat162_rn(v0, v1);
          } else if (EPI == EPI_MASK) {
            const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(mask + pix * COUT + co);
            v0 = __bfloat162float(m.x) > 0.f ? v0 : 0.f;
            v1 = __bfloat162float(m.y) > 0.f ? v1 : 0.f;
            *reinterpret_cast<__nv_bfloat162*>(y + pix * COUT + co) = __floats2bfloat162_rn(v0, v1);
          } else {  // EPI_RESID: out = input RGB + conv + bias, channels 0..2 in fp32
            if (co < 3) yf[pix * 3 + co] = resid[pix * 3 + co] + (v0 + bias[co]);
            if (co + 1 < 3) yf[pix * 3 + co + 1] = resid[pix * 3 + co + 1] + (v1 + bias[co + 1]);
          }
        }
      }
    }
  }
}

// Weight gradient: dW[tap][co][ci] = sum_p dY[p][co] X[p + tap][ci]. A warp
// owns up to 4 (tap, 16-channel block of co) units; K runs over the 16
// pixels of each tile row. Partial sums per CTA go to `part`.
template <int CIN, int COUTW, int D>
__global__ void __launch_bounds__(CNN_THREADS) conv_wgrad_kernel(const bf16* __restrict__ x,
                                                                 const bf16* __restrict__ dy, int B, int H, int W,
                                                                 float* __restrict__ part) {
  constexpr int RSX = row_stride(CIN), RSD = row_stride(COUTW);
  constexpr int MT = COUTW / 16, UNITS = 9 * MT, UPW = (UNITS + 7) / 8, NT = CIN / 8;
  extern __shared__ __align__(16) unsigned char sm[];
  constexpr int XW = ct_xw(D), XH = ct_xh(D);
  unsigned char* xs = sm;                          // [XH][XW] x CIN
  unsigned char* ds = sm + XH * XW * RSX;          // [CT_H][CT_W] x COUTW
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, c = lane & 3;
  float acc[UPW][NT][4];
#pragma unroll
  for (int u = 0; u < UPW; u++)
#pragma unroll
    for (int j = 0; j < NT; j++) acc[u][j][0] = acc[u][j][1] = acc[u][j][2] = acc[u][j][3] = 0.f;
  const int tiles_x = (W + CT_W - 1) / CT_W, tiles_y = (H + CT_H - 1) / CT_H;
  const int ntiles = B * tiles_x * tiles_y;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileIdx ti = tile_of(t, tiles_x, tiles_y);
    __syncthreads();
    stage_tile<CIN, XW, XH>(xs, x, ti.b, H, W, ti.x0 - D, ti.y0 - D);
    stage_tile<COUTW, CT_W, CT_H>(ds, dy, ti.b, H, W, ti.x0, ti.y0);  // zero outside the image
    __syncthreads();
#pragma unroll
    for (int u = 0; u < UPW; u++) {
      const int unit = warp + u * 8;
      if (unit >= UNITS) break;
      const int tap = unit / MT, mt = unit - tap * MT;
      const int ky = tap / 3, kx = tap % 3;
#pragma unroll 1
      for (int r = 0; r < CT_H; r++) {  // K: the 16 pixels of tile row r
        unsigned a0, a1, a2, a3;
        // A = dY^T: matrices (pixels 0-7, co 0-7), (pixels 0-7, co 8-15), (pixels 8-15, co 0-7), (8-15, 8-15)
        {
          const int pix = (lane & 7) + ((lane >> 4) & 1) * 8;
          const int cb = ((lane >> 3) & 1) * 8;
          ldsm_x4_t(smem_u32(ds + (r * CT_W + pix) * RSD + (mt * 16 + cb) * 2), a0, a1, a2, a3);
        }
#pragma unroll
        for (int j = 0; j < NT; j += 2) {
          // B = X shifted by the tap: matrices (pixels 0-7, ci j), (pixels 8-15, ci j), (0-7, j+1), (8-15, j+1)
          const int pix = (lane & 7) + ((lane >> 3) & 1) * 8;
          const int cj = (j + (lane >> 4)) * 8;
          unsigned b0, b1, b2, b3;
          ldsm_x4_t(smem_u32(xs + ((r + ky * D) * XW + pix + kx * D) * RSX + cj * 2), b0, b1, b2, b3);
          mma16816(acc[u][j], a0, a1, a2, a3, b0, b1);
          if (j + 1 < NT) mma16816(acc[u][j + 1], a0, a1, a2, a3, b2, b3);
        }
      }
    }
  }
  // write this CTA's partial sums: part[block][tap][co][ci]
  float* P = part + (size_t)blockIdx.x * 9 * COUTW * CIN;
#pragma unroll
  for (int u = 0; u < UPW; u++) {
    const int unit = warp + u * 8;
    if (unit >= UNITS) break;
    const int tap = unit / MT, mt = unit - tap * MT;
#pragma unroll
    for (int j = 0; j < NT; j++) {
      const int co = mt * 16 + g, ci = j * 8 + 2 * c;
      float* p0 = P + ((size_t)tap * COUTW + co) * CIN + ci;
      p0[0] = acc[u][j][0];
      p0[1] = acc[u][j][1];
      p0[8 * CIN] = acc[u][j][2];
      p0[8 * CIN + 1] = acc[u][j][3];
    }
  }
}

// Per-CTA channel sums of dY (bias gradient partials). Each thread reads one
// 16-byte group of 8 channels of a pixel per load, so a warp's loads cover
// whole pixel rows; the CTA's pixel lanes are summed in a fixed order.
template <int C>
__global__ void __launch_bounds__(CNN_THREADS) bias_grad_kernel(const bf16* __restrict__ dy, size_t n,
                                                                float* __restrict__ part) {
  constexpr int G = C / 8;             // 8-channel groups per pixel
  constexpr int PL = CNN_THREADS / G;  // pixel lanes per CTA
  __shared__ float s[PL * C];
  const int t = threadIdx.x;
  if (t < PL * G) {
    const int gi = t % G, pl = t / G;
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] = 0.f;
    const uint4* src = reinterpret_cast<const uint4*>(dy) + gi;
    const size_t stride = (size_t)gridDim.x * PL;
#pragma unroll 4
    for (size_t p = (size_t)blockIdx.x * PL + pl; p < n; p += stride) {
      const uint4 v = __ldg(src + p * G);
      const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float2 f = __bfloat1622float2(h2[q]);
        acc[2 * q] += f.x;
        acc[2 * q + 1] += f.y;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) s[pl * C + gi * 8 + j] = acc[j];
  }
  __syncthreads();
  if (t < C) {
    float sum = 0.f;
    for (int pl = 0; pl < PL; pl++) sum += s[pl * C + t];
    part[(size_t)blockIdx.x * C + t] = sum;
  }
}

// grads[layer] (real shape [9][cout][cin] then [cout]) from the per-CTA
// partials: a CTA takes RG_X consecutive parameters; thread row y sums the
// partials y, y + RG_Y, ... (its loads coalesced across the parameters), and
// the RG_Y row sums are added in a fixed order, so the result is
// deterministic.
constexpr int RG_X = 128, RG_Y = 8;
__global__ void __launch_bounds__(RG_X * RG_Y) reduce_grads_kernel(const float* __restrict__ wpart, int nw, int coutw,
                                                                    int cinp, const float* __restrict__ bpart, int nb,
                                                                    int cb, int cout, int cin, float* __restrict__ gw) {
  __shared__ float red[RG_Y][RG_X];
  const int i = blockIdx.x * RG_X + threadIdx.x;
  const int nwreal = 9 * cout * cin;
  float acc = 0.f;
  if (i < nwreal) {
    const int tap = i / (cout * cin), r = i - tap * cout * cin, co = r / cin, ci = r - co * cin;
    const size_t off = ((size_t)tap * coutw + co) * cinp + ci, stride = (size_t)9 * coutw * cinp;
    for (int k = threadIdx.y; k < nw; k += RG_Y) acc += wpart[off + (size_t)k * stride];
  } else if (i < nwreal + cout) {
    for (int k = threadIdx.y; k < nb; k += RG_Y) acc += bpart[(i - nwreal) + (size_t)k * cb];
  }
  red[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0 && i < nwreal + cout) {
    float sum = 0.f;
#pragma unroll
    for (int y = 0; y < RG_Y; y++) sum += red[y][threadIdx.x];
    gw[i] = sum;
  }
}

// The network's input at one pixel (8 bf16 values): channels 0-2 the RGB
// minus its 3x3 local mean (clamped at the image edges), 3-5 that mean, 6 the
// strength, 7 zero. The mean is taken in FP32 (row by row, then / 9) before
// anything is rounded to BF16, so the detail the network sees keeps BF16's
// relative precision at its own small magnitude instead of the pixel level's.
__device__ __forceinline__ void cnn_input_px(const float* __restrict__ rgb, int W, int H, int x, int y, float strength,
                                             bf16* v) {
  const float* c = rgb + ((size_t)y * W + x) * 3;
  float m[3] = {0.f, 0.f, 0.f};
  for (int dy = -1; dy <= 1; dy++) {
    const int yy = y + dy < 0 ? 0 : (y + dy >= H ? H - 1 : y + dy);
    for (int dx = -1; dx <= 1; dx++) {
      const int xx = x + dx < 0 ? 0 : (x + dx >= W ? W - 1 : x + dx);
      const float* q = rgb + ((size_t)yy * W + xx) * 3;
#pragma unroll
      for (int k = 0; k < 3; k++) m[k] = m[k] + q[k];
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    m[k] = __fdiv_rn(m[k], 9.0f);
    v[k] = __float2bfloat16_rn(c[k] - m[k]);
    v[3 + k] = __float2bfloat16_rn(m[k]);
  }
  v[6] = __float2bfloat16_rn(strength);
  v[7] = __float2bfloat16_rn(0.f);
}

// B crops of H x W RGB (fp32) and their strength (map or constant) -> NHWC16 bf16
__global__ void pack_input_kernel(const float* __restrict__ rgb, int B, int H, int W,
                                  const float* __restrict__ strength_map, float strength, bf16* __restrict__ x) {
  const size_t n = (size_t)B * H * W;
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int b = (int)(p / ((size_t)H * W));
  const int r = (int)(p - (size_t)b * H * W), py = r / W, px = r - py * W;
  __align__(16) bf16 v[16];
  cnn_input_px(rgb + (size_t)b * H * W * 3, W, H, px, py, strength_map ? strength_map[p] : strength, v);
#pragma unroll
  for (int k = 8; k < 16; k++) v[k] = __float2bfloat16_rn(0.f);
  reinterpret_cast<uint4*>(x + p * 16)[0] = reinterpret_cast<uint4*>(v)[0];
  reinterpret_cast<uint4*>(x + p * 16)[1] = reinterpret_cast<uint4*>(v)[1];
}

// The tensor-core engine's input: [2][hp][wp][8] bf16 (block 0 as above,
// block 1 zero; columns w..wp-1 and rows h..hp-1 zero).
__global__ void pack_input_tc_kernel(const float* __restrict__ rgb, int w, int h, int wp, int hp, float strength,
                                     bf16* __restrict__ x) {
  const size_t n = (size_t)wp * hp;
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int py = (int)(p / wp), px = (int)(p - (size_t)py * wp);
  __align__(16) bf16 v[8];
  if (px < w && py < h) {
    cnn_input_px(rgb, w, h, px, py, strength, v);
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = __float2bfloat16_rn(0.f);
  }
  reinterpret_cast<uint4*>(x)[p] = reinterpret_cast<uint4*>(v)[0];
  reinterpret_cast<uint4*>(x)[n + p] = make_uint4(0u, 0u, 0u, 0u);
}

// MSE over n pixels x 3 channels: dY = 2 (out - t) / (3n) into NHWC16 bf16
// (channels 3..15 zero); per-CTA partial sums of (out - t)^2.
// relative != 0: every pixel's squared error is weighted by 1 / s^2, s its
// strength input (smap[p], or s_const without a map), so frames of every
// noise level count by their error relative to the noise.
__global__ void mse_kernel(const float* __restrict__ out, const float* __restrict__ tgt, size_t n,
                           const float* __restrict__ smap, float s_const, int relative, bf16* __restrict__ dy,
                           float* __restrict__ part) {
  __shared__ float s[CNN_THREADS];
  const float scale = 2.0f / (3.0f * (float)n);
  float acc = 0.f;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    __align__(16) bf16 v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __float2bfloat16_rn(0.f);
    float w = 1.f;
    if (relative) {
      const float sp = smap ? smap[p] : s_const;
      if (sp > 0.f) w = 1.f / (sp * sp);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float d = out[p * 3 + k] - tgt[p * 3 + k];
      acc += w * d * d;
      v[k] = __float2bfloat16_rn(w * d * scale);
    }
    reinterpret_cast<uint4*>(dy + p * 16)[0] = reinterpret_cast<uint4*>(v)[0];
    reinterpret_cast<uint4*>(dy + p * 16)[1] = reinterpret_cast<uint4*>(v)[1];
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int k = CNN_THREADS / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// Sum of squares of the n gradients into *out (one CTA, fixed order: deterministic).
// Per-CTA partial sums of squared gradients (SQ_BLOCKS CTAs).
constexpr int SQ_BLOCKS = 64;
__global__ void __launch_bounds__(CNN_THREADS) grad_sqsum_kernel(const float* __restrict__ gr, int n,
                                                                 float* __restrict__ part) {
  __shared__ float s[CNN_THREADS];
  float acc = 0.f;
  for (int i = blockIdx.x * CNN_THREADS + threadIdx.x; i < n; i += gridDim.x * CNN_THREADS) acc += gr[i] * gr[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int k = CNN_THREADS / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// Adam; with clip > 0 the gradient is first scaled by min(1, clip / |g|)
// (global L2 norm: the SQ_BLOCKS partials of grad_sqsum_kernel, added in a
// fixed order by every thread).
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ gr, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2, const float* __restrict__ gsq, float clip) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = gr[i];
  if (clip > 0.f) {
    float sq = 0.f;
    for (int b = 0; b < SQ_BLOCKS; b++) sq += gsq[b];
    const float norm = sqrtf(sq);
    if (norm > clip) gi *= clip / norm;
  }
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// master fp32 [9][cout][cin] + [cout] -> forward weights bf16 [9][coutp][cinp],
// bias fp32 [coutp], and (when wd) data-gradient weights bf16
// [9][cinp_d][coutp_d] with the taps flipped: wd[8 - tap][ci][co] = w[tap][co][ci].
__global__ void pack_weights_kernel(const float* __restrict__ w, int cout, int cin, int coutp, int cinp,
                                    bf16* __restrict__ wf, float* __restrict__ bias, bf16* __restrict__ wd,
                                    int cinp_d, int coutp_d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = 9 * coutp * cinp;
  if (i < nf) {
    const int tap = i / (coutp * cinp), r = i - tap * coutp * cinp, co = r / cinp, ci = r - co * cinp;
    const float v = (co < cout && ci < cin) ? w[(tap * cout + co) * cin + ci] : 0.f;
    wf[i] = __float2bfloat16_rn(v);
  }
  if (i < coutp) bias[i] = i < cout ? w[9 * cout * cin + i] : 0.f;
  if (wd) {
    const int nd = 9 * cinp_d * coutp_d;
    if (i < nd) {
      const int tp = i / (cinp_d * coutp_d), r = i - tp * cinp_d * coutp_d, ci = r / coutp_d, co = r - ci * coutp_d;
      const int tap = 8 - tp;
      const float v = (co < cout && ci < cin) ? w[(tap * cout + co) * cin + ci] : 0.f;
      wd[i] = __float2bfloat16_rn(v);
    }
  }
}

// Residual check of the learned output: one CTA per NLM tile (tile_w x
// tile_h). The tile falls back to NLM when the RMS of what the network
// removed, out - in, exceeds tau * sigma (sigma = the noise level implied by
// the NLM strength, h / 1.5), or when the output is not finite.
__global__ void residual_check_kernel(const float* __restrict__ in, const float* __restrict__ out, int w, int h,
                                      int tile_w, int tile_h, float limit2, unsigned char* __restrict__ flags,
                                      unsigned* __restrict__ count, int ty0) {
  __shared__ float s[CNN_THREADS];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const int ty = blockIdx.y + ty0;  // tile row (a launch may cover a band of tile rows)
  const int x0 = blockIdx.x * tile_w, y0 = ty * tile_h;
  float acc = 0.f;
  int n = 0;
  for (int i = threadIdx.x; i < tile_w * tile_h; i += CNN_THREADS) {
    const int y = y0 + i / tile_w, x = x0 + i % tile_w;
    if (x >= w || y >= h) continue;
    const size_t p = ((size_t)y * w + x) * 3;
    for (int k = 0; k < 3; k++) {
      const float o = out[p + k];
      if (!isfinite(o)) bad = 1;
      const float d = o - in[p + k];
      acc += d * d;
    }
    n += 3;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int k = CNN_THREADS / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int tw = min(tile_w, w - x0), th = min(tile_h, h - y0);
    const float mean = s[0] / (float)(3 * tw * th);
    const unsigned char f = (bad || !(mean <= limit2)) ? 1 : 0;
    flags[ty * gridDim.x + blockIdx.x] = f;
    if (f) atomicAdd(count, 1u);
  }
  (void)n;
}

// Judge mode (plain NLM as the judge of the network's error). Tile t of the
// NLM tile grid is judged when a 32-bit mix of (seed, t) is below
// fraction * 2^32, so the sample depends only on the seed and the tile grid
// (the same tiles whether the frame runs whole or in bands).
__host__ __device__ __forceinline__ unsigned judge_mix(unsigned seed, unsigned t) {
  unsigned x = seed * 0x9E3779B9u ^ (t + 0x7F4A7C15u);
  x ^= x >> 16;
  x *= 0x85EBCA6Bu;
  x ^= x >> 13;
  x *= 0xC2B2AE35u;
  x ^= x >> 16;
  return x;
}

// One CTA per tile of tile rows [ty0, ty0 + gridDim.y): marks the judged
// tiles and saves the network's output there (NLM overwrites it next).
__global__ void judge_save_kernel(const float* __restrict__ out, int w, int h, int tile_w, int tile_h,
                                  unsigned seed, unsigned long long thr, float* __restrict__ save,
                                  unsigned char* __restrict__ jflags, unsigned* __restrict__ stats, int ty0) {
  const int ty = blockIdx.y + ty0;
  const int t = ty * gridDim.x + blockIdx.x;
  const bool sel = (unsigned long long)judge_mix(seed, (unsigned)t) < thr;
  if (threadIdx.x == 0) {
    jflags[t] = sel ? 1 : 0;
    if (sel) atomicAdd(&stats[0], 1u);
  }
  if (!sel) return;
  const int x0 = blockIdx.x * tile_w, y0 = ty * tile_h;
  const int tw = min(tile_w, w - x0), th = min(tile_h, h - y0);
  for (int i = threadIdx.x; i < tw * th * 3; i += blockDim.x) {
    const int y = y0 + i / (tw * 3), r = i - (y - y0) * tw * 3;
    const size_t p = ((size_t)y * w + x0) * 3 + r;
    save[p] = out[p];
  }
}

// After NLM has rewritten the judged tiles: per judged tile, the RMS of the
// network's output against NLM's, over sigma. The tile keeps NLM's result
// when that exceeds the limit, when the network's output is not finite, or
// when the residual check already failed it; otherwise the network's output
// goes back. Judged tiles are settled here, so their residual flag is
// cleared (the fallback pass skips them).
__global__ void judge_decide_kernel(const float* __restrict__ save, float* __restrict__ out, int w, int h,
                                    int tile_w, int tile_h, const unsigned char* __restrict__ jflags,
                                    unsigned char* __restrict__ rflags, float inv_sigma2, float limit2,
                                    unsigned* __restrict__ stats, int ty0) {
  __shared__ float red[CNN_THREADS];
  __shared__ int bad, keep_nlm;
  const int ty = blockIdx.y + ty0;
  const int t = ty * gridDim.x + blockIdx.x;
  if (!jflags[t]) return;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const int x0 = blockIdx.x * tile_w, y0 = ty * tile_h;
  const int tw = min(tile_w, w - x0), th = min(tile_h, h - y0);
  float acc = 0.f;
  for (int i = threadIdx.x; i < tw * th * 3; i += CNN_THREADS) {
    const int y = y0 + i / (tw * 3), r = i - (y - y0) * tw * 3;
    const size_t p = ((size_t)y * w + x0) * 3 + r;
    const float a = save[p];
    if (!isfinite(a)) bad = 1;
    const float d = a - out[p];
    acc += d * d;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int k = CNN_THREADS / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float e2 = red[0] / (float)(3 * tw * th) * inv_sigma2;  // (rms / sigma)^2
    const int fail = bad || rflags[t] || !(e2 <= limit2);
    keep_nlm = fail;
    rflags[t] = 0;
    if (fail) atomicAdd(&stats[1], 1u);
    if (isfinite(e2)) {
      atomicMax(&stats[2], __float_as_uint(e2));  // non-negative floats order as their bits
      atomicAdd(reinterpret_cast<float*>(&stats[3]), e2);
    }
  }
  __syncthreads();
  if (keep_nlm) return;
  for (int i = threadIdx.x; i < tw * th * 3; i += CNN_THREADS) {
    const int y = y0 + i / (tw * 3), r = i - (y - y0) * tw * 3;
    const size_t p = ((size_t)y * w + x0) * 3 + r;
    out[p] = save[p];
  }
}

// Layout conversion of the tensor-core training engine. A batch of B crops
// of H x W pixels lives in the tensor-core layout as one frame [C/8][Hp][Wp][8]
// whose crop b occupies rows b * period .. b * period + H - 1 (period = H +
// the largest dilation; the rows between crops and the padding are zero).
// NHWC -> tensor-core layout (only the crops' pixels are written): the packed
// input and the loss gradient, which the NHWC kernels produce.
template <int C>
__global__ void nhwc_to_tc_kernel(const bf16* __restrict__ x, int B, int H, int W, int period, int wp, size_t plane,
                                  bf16* __restrict__ y) {
  const size_t n = (size_t)B * H * W * (C / 8);
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int cb = (int)(i % (C / 8));
  const size_t p = i / (C / 8);
  const int b = (int)(p / ((size_t)H * W));
  const int r = (int)(p - (size_t)b * H * W), py = r / W, px = r - py * W;
  const uint4 v = reinterpret_cast<const uint4*>(x)[i];
  reinterpret_cast<uint4*>(y)[(size_t)cb * plane + (size_t)(b * period + py) * wp + px] = v;
}

// ------------------------------------------------------------------ host side

template <int CIN, int COUT, int EPI, int D>
cudaError_t launch_fwd_d(cudaStream_t st, int grid, const bf16* x, int B, int H, int W, const bf16* wt,
                         const float* bias, bf16* y, const bf16* mask, const float* resid, float* yf) {
  const size_t smem = (size_t)9 * COUT * row_stride(CIN) + (size_t)ct_xh(D) * ct_xw(D) * row_stride(CIN);
  cudaError_t e = cudaFuncSetAttribute(conv_fwd_kernel<CIN, COUT, EPI, D>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  conv_fwd_kernel<CIN, COUT, EPI, D><<<grid, CNN_THREADS, smem, st>>>(x, B, H, W, wt, bias, y, mask, resid, yf);
  return cudaGetLastError();
}

// conv with dilation d (1..4) over the per-dilation instantiations
template <int CIN, int COUT, int EPI>
cudaError_t launch_fwd(cudaStream_t st, int grid, int d, const bf16* x, int B, int H, int W, const bf16* wt,
                       const float* bias, bf16* y, const bf16* mask, const float* resid, float* yf) {
  switch (d) {
    case 1: return launch_fwd_d<CIN, COUT, EPI, 1>(st, grid, x, B, H, W, wt, bias, y, mask, resid, yf);
    case 2: return launch_fwd_d<CIN, COUT, EPI, 2>(st, grid, x, B, H, W, wt, bias, y, mask, resid, yf);
    case 3: return launch_fwd_d<CIN, COUT, EPI, 3>(st, grid, x, B, H, W, wt, bias, y, mask, resid, yf);
    case 4: return launch_fwd_d<CIN, COUT, EPI, 4>(st, grid, x, B, H, W, wt, bias, y, mask, resid, yf);
    default: return cudaErrorInvalidValue;
  }
}

template <int CIN, int COUTW, int D>
cudaError_t launch_wgrad_d(cudaStream_t st, int grid, const bf16* x, const bf16* dy, int B, int H, int W,
                           float* part) {
  const size_t smem = (size_t)ct_xh(D) * ct_xw(D) * row_stride(CIN) + (size_t)CT_H * CT_W * row_stride(COUTW);
  cudaError_t e = cudaFuncSetAttribute(conv_wgrad_kernel<CIN, COUTW, D>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  conv_wgrad_kernel<CIN, COUTW, D><<<grid, CNN_THREADS, smem, st>>>(x, dy, B, H, W, part);
  return cudaGetLastError();
}

template <int CIN, int COUTW>
cudaError_t launch_wgrad(cudaStream_t st, int grid, int d, const bf16* x, const bf16* dy, int B, int H, int W,
                         float* part) {
  switch (d) {
    case 1: return launch_wgrad_d<CIN, COUTW, 1>(st, grid, x, dy, B, H, W, part);
    case 2: return launch_wgrad_d<CIN, COUTW, 2>(st, grid, x, dy, B, H, W, part);
    case 3: return launch_wgrad_d<CIN, COUTW, 3>(st, grid, x, dy, B, H, W, part);
    case 4: return launch_wgrad_d<CIN, COUTW, 4>(st, grid, x, dy, B, H, W, part);
    default: return cudaErrorInvalidValue;
  }
}

// layer table: real and padded channel counts
struct LayerSpec {
  int cin, cout;     // real
  int cinp, coutp;   // forward padding
  int dil;           // dilation of the 3x3 taps (offsets (ky-1)*dil, (kx-1)*dil)
};
constexpr int NL = 8;
// Dilations 1, 2, 3, 4, 3, 2, 1, 1: a 35 x 35 receptive field (8 undilated
// layers see 17 x 17), covering NLM's 27 x 27 support at 7x7 / 21x21.
constexpr LayerSpec LAYERS[NL] = {{7, 48, 16, 48, 1},  {48, 48, 48, 48, 2}, {48, 48, 48, 48, 3},
                                  {48, 48, 48, 48, 4}, {48, 48, 48, 48, 3}, {48, 48, 48, 48, 2},
                                  {48, 48, 48, 48, 1}, {48, 3, 48, 8, 1}};

// Rows (and columns) of input beyond an output region that the network reads:
// each layer reaches its dilation, and the input packing's 3x3 local mean one more.
constexpr int cnn_reach() {
  int r = 1;
  for (int l = 0; l < NL; l++) r += LAYERS[l].dil;
  return r;
}

// the largest dilation: zero rows between the crops of a tensor-core training batch
constexpr int cnn_max_dil() {
  int d = 1;
  for (int l = 0; l < NL; l++) d = LAYERS[l].dil > d ? LAYERS[l].dil : d;
  return d;
}

}  // namespace

int ds_cnn_halo_rows() { return cnn_reach(); }

// ----------------------------------------------------------------- network

cudaError_t ds_tc_layer(cudaStream_t st, int kind, int dil, const void* x, int H, int W, const void* wt,
                        const float* bias, void* y, const float* resid, float* yf, const void* mask, int period,
                        int valid, int* err);
cudaError_t ds_tc_wgrad(cudaStream_t st, int kind, int dil, const void* x, const void* dy, int H, int W,
                        float* wpart, float* bpart, int max_grid, int* grid, int* err);
cudaError_t ds_cnn_forward_tc(cudaStream_t st, const void* x16, void* a, void* b, int H, int W,
                              const void* const* wf, const float* const* bias, const int* dil, const float* rgb,
                              float* out, int* err, cudaEvent_t hidden_begin, cudaEvent_t hidden_end);

struct DsCnn {
  int device = 0;
  bool use_tc = true;    // inference on tcgen05 (false: the mma.sync kernels)
  int* err = nullptr;    // device status word of the tcgen05 kernels
  int max_batch = 0, crop = 0;
  int n_params = 0;
  int off[NL + 1] = {};  // offsets of each layer in the flat parameter array
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  bf16* wf[NL] = {};
  bf16* wd[NL] = {};
  float* bias[NL] = {};
  long long step = 0;
  bool packed = false;   // wf/wd/bias match params (cleared whenever params may change)
  float clip = 0.f;      // global gradient-norm clip of the Adam step (0: off)
  int relative_loss = 0; // 1: squared errors weighted by 1 / strength^2
  cudaEvent_t mark_a = nullptr, mark_b = nullptr;  // profiling: around the hidden layers of inference
  float* gsq = nullptr;  // device: SQ_BLOCKS partial sums of squared gradients
  // training buffers (max_batch crops of crop x crop)
  bf16* act[NL] = {};   // act[0] = packed input (16 ch), act[l] = output of layer l (48 ch), l = 1..7
  bf16* gA = nullptr;   // gradient ping
  bf16* gB = nullptr;   // gradient pong
  bf16* dy8 = nullptr;  // 16 ch
  float* out = nullptr;
  float *wpart = nullptr, *bpart = nullptr, *lpart = nullptr;
  int wgrid = 0, bgrid = 0;
  // training on the tensor cores: the batch as one frame of crops (see
  // nhwc_to_tc_kernel); activations, the output gradient and the ping-pong
  // data gradients in the tensor-core layout
  bf16* tact[NL] = {};
  bf16 *tg[2] = {}, *tdy8 = nullptr;
  int t_period = 0, t_wp = 0, t_hp = 0;
  // inference buffers (grown on demand)
  bf16 *ia = nullptr, *ib = nullptr;
  size_t infer_px = 0;
  // judge mode: plain NLM recomputes a seeded sample of the NLM tiles and
  // judges the network's output there (fraction 0: off)
  float judge_frac = 0.f, judge_limit = 0.f;
  unsigned judge_seed = 0;
  float* judge_save = nullptr;            // the network's output on the judged tiles (frame layout)
  size_t judge_px = 0;
  unsigned char* judge_flags = nullptr;   // one byte per NLM tile: judged
  size_t judge_tiles = 0;
  unsigned* judge_stats = nullptr;        // judged, failed, max (rms/sigma)^2 bits, sum (rms/sigma)^2 bits
  std::vector<void*> allocs;

  void* alloc(size_t bytes, cudaError_t& e) {
    void* p = nullptr;
    e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e == cudaSuccess) allocs.push_back(p);
    return p;
  }
  ~DsCnn() {
    for (void* p : allocs) cudaFree(p);
    if (judge_save) cudaFree(judge_save);
    if (judge_flags) cudaFree(judge_flags);
  }
};

size_t ds_cnn_param_count() {
  size_t n = 0;
  for (int l = 0; l < NL; l++) n += (size_t)9 * LAYERS[l].cout * LAYERS[l].cin + LAYERS[l].cout;
  return n;
}

cudaError_t ds_cnn_create(int max_batch, int crop, DsCnn** out) {
  DsCnn* net = new DsCnn();
  cudaError_t e = cudaGetDevice(&net->device);
  if (e != cudaSuccess) {
    delete net;
    return e;
  }
  net->max_batch = max_batch;
  net->crop = crop;
  int o = 0;
  for (int l = 0; l < NL; l++) {
    net->off[l] = o;
    o += 9 * LAYERS[l].cout * LAYERS[l].cin + LAYERS[l].cout;
  }
  net->off[NL] = o;
  net->n_params = o;
  const size_t pb = (size_t)o * sizeof(float);
  net->params = (float*)net->alloc(pb, e);
  if (e == cudaSuccess) net->grads = (float*)net->alloc(pb, e);
  if (e == cudaSuccess) net->m = (float*)net->alloc(pb, e);
  if (e == cudaSuccess) net->v = (float*)net->alloc(pb, e);
  for (int l = 0; l < NL && e == cudaSuccess; l++) {
    const LayerSpec L = LAYERS[l];
    net->wf[l] = (bf16*)net->alloc((size_t)9 * L.coutp * L.cinp * sizeof(bf16), e);
    if (e == cudaSuccess) net->bias[l] = (float*)net->alloc((size_t)L.coutp * sizeof(float), e);
    if (e == cudaSuccess && l > 0) {
      const int cd = l == NL - 1 ? 16 : L.coutp;  // the last layer's gradient is stored with 16 channels
      net->wd[l] = (bf16*)net->alloc((size_t)9 * L.cinp * cd * sizeof(bf16), e);
    }
  }
  if (e == cudaSuccess && max_batch > 0) {
    const size_t px = (size_t)max_batch * crop * crop;
    net->act[0] = (bf16*)net->alloc(px * 16 * sizeof(bf16), e);
    for (int l = 1; l < NL && e == cudaSuccess; l++) net->act[l] = (bf16*)net->alloc(px * 48 * sizeof(bf16), e);
    if (e == cudaSuccess) net->gA = (bf16*)net->alloc(px * 48 * sizeof(bf16), e);
    if (e == cudaSuccess) net->gB = (bf16*)net->alloc(px * 48 * sizeof(bf16), e);
    if (e == cudaSuccess) net->dy8 = (bf16*)net->alloc(px * 16 * sizeof(bf16), e);
    if (e == cudaSuccess) net->out = (float*)net->alloc(px * 3 * sizeof(float), e);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
    net->wgrid = sms * 2;
    net->bgrid = sms * 4;
    if (e == cudaSuccess) net->wpart = (float*)net->alloc((size_t)net->wgrid * 9 * 48 * 48 * sizeof(float), e);
    if (e == cudaSuccess) net->bpart = (float*)net->alloc((size_t)net->bgrid * 48 * sizeof(float), e);
    if (e == cudaSuccess) net->lpart = (float*)net->alloc((size_t)1024 * sizeof(float), e);
    // the tensor-core engine's batch frame: crops cnn_max_dil() rows apart, zero between them
    net->t_period = crop + cnn_max_dil();
    net->t_wp = (crop + 3) / 4 * 4;
    net->t_hp = (max_batch * net->t_period + 11) / 12 * 12;
    const size_t tplane = (size_t)net->t_wp * net->t_hp * 16;  // bytes of an 8-channel block
    for (int l = 0; l < NL && e == cudaSuccess; l++) net->tact[l] = (bf16*)net->alloc(tplane * (l == 0 ? 2 : 6), e);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) net->tg[k] = (bf16*)net->alloc(tplane * 6, e);
    if (e == cudaSuccess) net->tdy8 = (bf16*)net->alloc(tplane * 2, e);
    // zero once: the epilogues write every row of the frame, so the padding rows stay zero
    for (int l = 0; l < NL && e == cudaSuccess; l++) e = cudaMemset(net->tact[l], 0, tplane * (l == 0 ? 2 : 6));
    for (int k = 0; k < 2 && e == cudaSuccess; k++) e = cudaMemset(net->tg[k], 0, tplane * 6);
    if (e == cudaSuccess) e = cudaMemset(net->tdy8, 0, tplane * 2);
  }
  if (e == cudaSuccess) net->err = (int*)net->alloc(sizeof(int), e);
  if (e == cudaSuccess) net->gsq = (float*)net->alloc(SQ_BLOCKS * sizeof(float), e);
  if (e == cudaSuccess) net->judge_stats = (unsigned*)net->alloc(4 * sizeof(unsigned), e);
  if (e == cudaSuccess) e = cudaMemset(net->judge_stats, 0, 4 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(net->err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(net->m, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(net->v, 0, pb);
  if (e != cudaSuccess) {
    delete net;
    return e;
  }
  *out = net;
  return cudaSuccess;
}

void ds_cnn_destroy(DsCnn* net) { delete net; }

int ds_cnn_params(const DsCnn* net) { return net->n_params; }
float* ds_cnn_param_ptr(DsCnn* net) {
  net->packed = false;  // the caller may write through it
  return net->params;
}
float* ds_cnn_grad_ptr(DsCnn* net) { return net->grads; }
float* ds_cnn_moment_ptr(DsCnn* net, int which) { return which == 0 ? net->m : net->v; }
long long* ds_cnn_step_ptr(DsCnn* net) { return &net->step; }

cudaError_t ds_cnn_pack(DsCnn* net, cudaStream_t st) {
  if (net->packed) return cudaSuccess;
  for (int l = 0; l < NL; l++) {
    const LayerSpec L = LAYERS[l];
    const int cd = l == NL - 1 ? 16 : L.coutp;
    const int n = 9 * L.coutp * L.cinp > 9 * L.cinp * cd ? 9 * L.coutp * L.cinp : 9 * L.cinp * cd;
    pack_weights_kernel<<<(n + 255) / 256, 256, 0, st>>>(net->params + net->off[l], L.cout, L.cin, L.coutp, L.cinp,
                                                         net->wf[l], net->bias[l], net->wd[l], L.cinp, cd);
  }
  const cudaError_t e = cudaGetLastError();
  net->packed = e == cudaSuccess;
  return e;
}

// Forward through all layers. x16: packed input; rgb: fp32 input RGB (the
// residual); out: fp32 RGB. acts: per-layer outputs (act[l] for l=1..7).
static cudaError_t forward(DsCnn* net, cudaStream_t st, const bf16* x16, const float* rgb, int B, int H, int W,
                           bf16* const* acts, float* out, cudaEvent_t hidden_begin = nullptr,
                           cudaEvent_t hidden_end = nullptr) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
  const int grid = sms * 3;
  cudaError_t e = launch_fwd<16, 48, EPI_RELU>(st, grid, LAYERS[0].dil, x16, B, H, W, net->wf[0], net->bias[0],
                                               acts[1], nullptr, nullptr, nullptr);
  if (e == cudaSuccess && hidden_begin) e = cudaEventRecord(hidden_begin, st);
  for (int l = 1; l < NL - 1 && e == cudaSuccess; l++)
    e = launch_fwd<48, 48, EPI_RELU>(st, grid, LAYERS[l].dil, acts[l], B, H, W, net->wf[l], net->bias[l],
                                     acts[l + 1], nullptr, nullptr, nullptr);
  if (e == cudaSuccess && hidden_end) e = cudaEventRecord(hidden_end, st);
  if (e == cudaSuccess)
    e = launch_fwd<48, 8, EPI_RESID>(st, grid, LAYERS[NL - 1].dil, acts[NL - 1], B, H, W, net->wf[NL - 1],
                                     net->bias[NL - 1], nullptr, nullptr, rgb, out);
  return e;
}

// Gradients of the MSE between the network's output on (rgb, strength) and
// tgt into net->grads (real parameter layout); *loss_sum = sum of squared
// errors. Inputs are device arrays of B crops of crop x crop pixels.
cudaError_t ds_cnn_gradients(DsCnn* net, cudaStream_t st, const float* rgb, const float* strength_map,
                             float strength, const float* tgt, int B, float* loss_sum_host) {
  const int H = net->crop, W = net->crop;
  const size_t n = (size_t)B * H * W;
  cudaError_t e = ds_cnn_pack(net, st);
  if (e != cudaSuccess) return e;
  pack_input_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(rgb, B, H, W, strength_map, strength,
                                                                  net->act[0]);
  // the tensor-core engine: forward, data and weight gradients on tcgen05 over the batch laid out
  // as one frame of crops
  const bool tc = net->use_tc;
  const int period = net->t_period, HF = B * period, wp = net->t_wp;
  const size_t tplane = (size_t)wp * ((HF + 11) / 12 * 12);  // pixels of an 8-channel block of the frame
  auto to_tc = [&](const bf16* x, int C, bf16* y) {
    const size_t m = n * (C / 8);
    if (C == 16) nhwc_to_tc_kernel<16><<<(unsigned)((m + 255) / 256), 256, 0, st>>>(x, B, H, W, period, wp, tplane, y);
    else nhwc_to_tc_kernel<48><<<(unsigned)((m + 255) / 256), 256, 0, st>>>(x, B, H, W, period, wp, tplane, y);
    return cudaGetLastError();
  };
  if (tc) {
    if (B > net->max_batch) return cudaErrorInvalidValue;
    // the two 16-channel frames are written at the crops' pixels only: zero the rest first
    if ((e = cudaMemsetAsync(net->tact[0], 0, tplane * 2 * 16, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(net->tdy8, 0, tplane * 2 * 16, st)) != cudaSuccess) return e;
    if ((e = to_tc(net->act[0], 16, net->tact[0])) != cudaSuccess) return e;
    for (int l = 0; l < NL && e == cudaSuccess; l++) {
      const int kind = l == 0 ? 0 : (l == NL - 1 ? 2 : 1);
      e = ds_tc_layer(st, kind, LAYERS[l].dil, net->tact[l], HF, W, net->wf[l], net->bias[l],
                      l == NL - 1 ? nullptr : net->tact[l + 1], rgb, net->out, nullptr, period, H, net->err);
    }
    if (e != cudaSuccess) return e;
  } else if ((e = forward(net, st, net->act[0], rgb, B, H, W, net->act, net->out)) != cudaSuccess) {
    return e;
  }
  const int lgrid = 512;
  mse_kernel<<<lgrid, CNN_THREADS, 0, st>>>(net->out, tgt, n, strength_map, strength, net->relative_loss, net->dy8,
                                            net->lpart);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
  const int grid = sms * 3;
  // a layer's weight and bias gradients from nw / nb partial sums
  auto reduce = [&](int l, int coutw, int cinp, int cb, int nw, int nb) {
    const LayerSpec L = LAYERS[l];
    const int nreal = 9 * L.cout * L.cin + L.cout;
    reduce_grads_kernel<<<(nreal + RG_X - 1) / RG_X, dim3(RG_X, RG_Y), 0, st>>>(
        net->wpart, nw, coutw, cinp, net->bpart, nb, cb, L.cout, L.cin, net->grads + net->off[l]);
  };
  if (tc) {
    // per layer, top down: weight and bias gradients of layer l from (tact[l], its output
    // gradient), then the data gradient below it; every tensor stays in the frame layout
    int wg = 0;
    if ((e = to_tc(net->dy8, 16, net->tdy8)) != cudaSuccess) return e;
    if ((e = ds_tc_wgrad(st, 2, LAYERS[7].dil, net->tact[7], net->tdy8, HF, W, net->wpart, net->bpart, net->wgrid,
                         &wg, net->err)) != cudaSuccess)
      return e;
    reduce(7, 16, 48, 16, wg, wg);
    if ((e = ds_tc_layer(st, 3, LAYERS[7].dil, net->tdy8, HF, W, net->wd[7], nullptr, net->tg[0], nullptr, nullptr,
                         net->tact[7], period, H, net->err)) != cudaSuccess)
      return e;
    int tgi = 0;  // the data gradient is in net->tg[tgi]
    for (int l = 6; l >= 1; l--) {
      if ((e = ds_tc_wgrad(st, 1, LAYERS[l].dil, net->tact[l], net->tg[tgi], HF, W, net->wpart, net->bpart,
                           net->wgrid, &wg, net->err)) != cudaSuccess)
        return e;
      reduce(l, 48, 48, 48, wg, wg);
      if ((e = ds_tc_layer(st, 4, LAYERS[l].dil, net->tg[tgi], HF, W, net->wd[l], nullptr, net->tg[tgi ^ 1], nullptr,
                           nullptr, net->tact[l], period, H, net->err)) != cudaSuccess)
        return e;
      tgi ^= 1;
    }
    if ((e = ds_tc_wgrad(st, 0, LAYERS[0].dil, net->tact[0], net->tg[tgi], HF, W, net->wpart, net->bpart, net->wgrid,
                         &wg, net->err)) != cudaSuccess)
      return e;
    reduce(0, 48, 16, 48, wg, wg);
  } else {
    // mma.sync: layer 8: dW from (act7, dy8); dA7 = dgrad(dy8) * [act7 > 0]
    if ((e = launch_wgrad<48, 16>(st, net->wgrid, LAYERS[7].dil, net->act[7], net->dy8, B, H, W, net->wpart)) !=
        cudaSuccess)
      return e;
    bias_grad_kernel<16><<<net->bgrid, CNN_THREADS, 0, st>>>(net->dy8, n, net->bpart);
    reduce(7, 16, 48, 16, net->wgrid, net->bgrid);
    bf16* g = net->gA;
    bf16* gnext = net->gB;
    if ((e = launch_fwd<16, 48, EPI_MASK>(st, grid, LAYERS[7].dil, net->dy8, B, H, W, net->wd[7], nullptr, g,
                                          net->act[7], nullptr, nullptr)) != cudaSuccess)
      return e;
    for (int l = 6; l >= 1; l--) {  // layers 7..2 (index l): dW from (act[l], g); g_next = dgrad(g) * [act[l] > 0]
      if ((e = launch_wgrad<48, 48>(st, net->wgrid, LAYERS[l].dil, net->act[l], g, B, H, W, net->wpart)) !=
          cudaSuccess)
        return e;
      bias_grad_kernel<48><<<net->bgrid, CNN_THREADS, 0, st>>>(g, n, net->bpart);
      reduce(l, 48, 48, 48, net->wgrid, net->bgrid);
      if ((e = launch_fwd<48, 48, EPI_MASK>(st, grid, LAYERS[l].dil, g, B, H, W, net->wd[l], nullptr, gnext,
                                            net->act[l], nullptr, nullptr)) != cudaSuccess)
        return e;
      bf16* tmp = g;
      g = gnext;
      gnext = tmp;
    }
    // layer 1: dW from (packed input, g)
    if ((e = launch_wgrad<16, 48>(st, net->wgrid, LAYERS[0].dil, net->act[0], g, B, H, W, net->wpart)) !=
        cudaSuccess)
      return e;
    bias_grad_kernel<48><<<net->bgrid, CNN_THREADS, 0, st>>>(g, n, net->bpart);
    reduce(0, 48, 16, 48, net->wgrid, net->bgrid);
  }
  if (loss_sum_host) {
    float part[512];
    if ((e = cudaMemcpyAsync(part, net->lpart, lgrid * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    double s = 0;
    for (int i = 0; i < lgrid; i++) s += part[i];
    *loss_sum_host = (float)s;
  }
  return cudaGetLastError();
}

cudaError_t ds_cnn_adam(DsCnn* net, cudaStream_t st, float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  net->step++;
  net->packed = false;
  const float c1 = 1.0f - (float)pow(b1, (double)net->step), c2 = 1.0f - (float)pow(b2, (double)net->step);
  if (net->clip > 0.f) grad_sqsum_kernel<<<SQ_BLOCKS, CNN_THREADS, 0, st>>>(net->grads, net->n_params, net->gsq);
  adam_kernel<<<(net->n_params + 255) / 256, 256, 0, st>>>(net->params, net->grads, net->m, net->v, net->n_params, lr,
                                                           b1, b2, eps, c1, c2, net->gsq, net->clip);
  return cudaGetLastError();
}

// Inference on a whole (w x h) RGB image; out = input + network(input).
// Grows the inference activations to hold a w x h frame (the tensor-core
// engine pads rows to 4 pixels and planes to 12 rows, a multiple of every
// dilation). cudaFree synchronises the device, so a caller that runs the
// network on bands of different heights reserves the largest one first.
cudaError_t ds_cnn_reserve(DsCnn* net, int w, int h) {
  const size_t na = (size_t)((w + 3) / 4 * 4) * ((h + 11) / 12 * 12);
  cudaError_t e = cudaSuccess;
  if (net->infer_px < na) {
    if (net->ia) cudaFree(net->ia);
    if (net->ib) cudaFree(net->ib);
    net->ia = net->ib = nullptr;
    net->infer_px = 0;
    if ((e = cudaMalloc(&net->ia, na * 48 * sizeof(bf16))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&net->ib, na * 48 * sizeof(bf16))) != cudaSuccess) return e;
    net->infer_px = na;
  }
  return e;
}

cudaError_t ds_cnn_infer(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, float strength, float* out) {
  const size_t n = (size_t)w * h;
  const int wp = (w + 3) / 4 * 4, hp = (h + 11) / 12 * 12;
  const size_t na = (size_t)wp * hp;
  cudaError_t e = ds_cnn_reserve(net, w, h);
  if (e != cudaSuccess) return e;
  if ((e = ds_cnn_pack(net, st)) != cudaSuccess) return e;
  // ping-pong: input packed into ib (16 ch), layers alternate ia/ib
  if (net->use_tc) {
    if (hp > h) {  // padding rows of all 6 planes of both activation buffers read as zero
      const size_t plane = na * 8 * sizeof(bf16), pad = (size_t)(hp - h) * wp * 8 * sizeof(bf16);
      const size_t off = (size_t)h * wp * 8;
      if ((e = cudaMemset2DAsync(net->ia + off, plane, 0, pad, 6, st)) != cudaSuccess) return e;
      if ((e = cudaMemset2DAsync(net->ib + off, plane, 0, pad, 6, st)) != cudaSuccess) return e;
    }
    pack_input_tc_kernel<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(rgb, w, h, wp, hp, strength, net->ib);
    const void* wf[NL];
    const float* bs[NL];
    for (int l = 0; l < NL; l++) {
      wf[l] = net->wf[l];
      bs[l] = net->bias[l];
    }
    int dil[NL];
    for (int l = 0; l < NL; l++) dil[l] = LAYERS[l].dil;
    return ds_cnn_forward_tc(st, net->ib, net->ia, net->ib, h, w, wf, bs, dil, rgb, out, net->err, net->mark_a,
                             net->mark_b);
  }
  pack_input_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(rgb, 1, h, w, nullptr, strength, net->ib);
  bf16* acts[NL] = {net->ib, net->ia, net->ib, net->ia, net->ib, net->ia, net->ib, net->ia};
  return forward(net, st, net->ib, rgb, 1, h, w, acts, out, net->mark_a, net->mark_b);
}

void ds_cnn_set_engine(DsCnn* net, int use_tc) { net->use_tc = use_tc != 0; }

void ds_cnn_set_clip(DsCnn* net, float clip) { net->clip = clip > 0.f ? clip : 0.f; }

void ds_cnn_set_loss(DsCnn* net, int relative) { net->relative_loss = relative != 0; }

void ds_cnn_set_marks(DsCnn* net, cudaEvent_t a, cudaEvent_t b) {
  net->mark_a = a;
  net->mark_b = b;
}

// DSGPU_OK, or the status the tensor-core kernels left (the word is reset).
int ds_cnn_take_status(DsCnn* net, cudaStream_t st) {
  int h = 0;
  if (cudaMemcpyAsync(&h, net->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DSGPU_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DSGPU_ERR_CUDA;
  if (h != 0) cudaMemsetAsync(net->err, 0, sizeof(int), st);
  return h;
}

// ---- judge mode, host side
void ds_cnn_set_judge(DsCnn* net, float fraction, float limit, unsigned seed) {
  net->judge_frac = fraction > 0.f ? (fraction < 1.f ? fraction : 1.f) : 0.f;
  net->judge_limit = limit;
  net->judge_seed = seed;
}

bool ds_cnn_judge_on(const DsCnn* net) { return net->judge_frac > 0.f; }

// whether tile t is judged under (seed, fraction)
int ds_cnn_judge_tile(unsigned seed, float fraction, int t) {
  const unsigned long long thr = (unsigned long long)((double)fraction * 4294967296.0);
  return (unsigned long long)judge_mix(seed, (unsigned)t) < thr ? 1 : 0;
}

// Grows the judge buffers to a w x h frame (cudaFree synchronises the
// device, so a band pipeline reserves before its first launch).
cudaError_t ds_cnn_reserve_judge(DsCnn* net, int w, int h, int patch) {
  if (!ds_cnn_judge_on(net)) return cudaSuccess;
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const size_t px = (size_t)w * h, tiles = (size_t)tx * ty;
  cudaError_t e = cudaSuccess;
  if (net->judge_px < px) {
    if (net->judge_save) cudaFree(net->judge_save);
    net->judge_save = nullptr;
    net->judge_px = 0;
    if ((e = cudaMalloc(&net->judge_save, px * 3 * sizeof(float))) != cudaSuccess) return e;
    net->judge_px = px;
  }
  if (net->judge_tiles < tiles) {
    if (net->judge_flags) cudaFree(net->judge_flags);
    net->judge_flags = nullptr;
    net->judge_tiles = 0;
    if ((e = cudaMalloc(&net->judge_flags, tiles)) != cudaSuccess) return e;
    net->judge_tiles = tiles;
  }
  return e;
}

cudaError_t ds_cnn_judge_reset(DsCnn* net, cudaStream_t st) {
  return cudaMemsetAsync(net->judge_stats, 0, 4 * sizeof(unsigned), st);
}

// judged tiles, failed tiles, max and RMS over the judged tiles of (rms / sigma), of the last call
cudaError_t ds_cnn_judge_stats(DsCnn* net, cudaStream_t st, int* judged, int* failed, float* max_rms,
                               float* mean_rms) {
  unsigned hs[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(hs, net->judge_stats, sizeof(hs), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  float mx, sum;
  memcpy(&mx, &hs[2], 4);
  memcpy(&sum, &hs[3], 4);
  *judged = (int)hs[0];
  *failed = (int)hs[1];
  *max_rms = sqrtf(mx);
  *mean_rms = hs[0] ? sqrtf(sum / (float)hs[0]) : 0.f;
  return cudaSuccess;
}

namespace {
// Residual check, judge and fallback on the NLM tile rows [t0, t1), the
// network's output already in `out`.
cudaError_t check_judge_fallback(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, float h_param,
                                 int search, int patch, float tau, float* out, unsigned char* rflags,
                                 unsigned* count_dev, int t0, int t1) {
  const bool judge = ds_cnn_judge_on(net);
  if (tau <= 0.f && !judge) return cudaSuccess;  // no fallback
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const float sigma = h_param / 1.5f;
  cudaError_t e;
  if (tau > 0.f) {
    residual_check_kernel<<<dim3(tx, t1 - t0), CNN_THREADS, 0, st>>>(rgb, out, w, h, tw, th,
                                                                     tau * tau * sigma * sigma, rflags, count_dev, t0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  } else if ((e = cudaMemsetAsync(rflags + (size_t)t0 * tx, 0, (size_t)(t1 - t0) * tx, st)) != cudaSuccess) {
    return e;
  }
  if (judge) {
    if (net->judge_px < (size_t)w * h || net->judge_tiles < (size_t)tx * ty) return cudaErrorInvalidValue;
    const unsigned long long thr = (unsigned long long)((double)net->judge_frac * 4294967296.0);
    judge_save_kernel<<<dim3(tx, t1 - t0), CNN_THREADS, 0, st>>>(out, w, h, tw, th, net->judge_seed, thr,
                                                                 net->judge_save, net->judge_flags, net->judge_stats,
                                                                 t0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = ds_launch_nlm_tiles_rows(st, rgb, w, h, 3, h_param, search, patch, net->judge_flags, t0, t1, out)) !=
        cudaSuccess)
      return e;
    const float s2 = sigma * sigma > 1e-30f ? sigma * sigma : 1e-30f;
    judge_decide_kernel<<<dim3(tx, t1 - t0), CNN_THREADS, 0, st>>>(net->judge_save, out, w, h, tw, th,
                                                                   net->judge_flags, rflags, 1.0f / s2,
                                                                   net->judge_limit * net->judge_limit,
                                                                   net->judge_stats, t0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (tau <= 0.f) return cudaSuccess;
  return ds_launch_nlm_tiles_rows(st, rgb, w, h, 3, h_param, search, patch, rflags, t0, t1, out);
}
}  // namespace

// The learned stand-in with its fallback: CNN, residual check per NLM tile,
// (judge mode) NLM on a seeded sample of tiles judging the network there,
// NLM on the flagged tiles (written over the CNN output). flags_scratch holds
// the tile flags followed by a u32 count; *count_dev receives it.
cudaError_t ds_cnn_denoise(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, float h_param, int search,
                           int patch, float tau, float strength_scale, float* out, unsigned char* flags_scratch,
                           unsigned* count_dev) {
  cudaError_t e = ds_cnn_reserve_judge(net, w, h, patch);
  if (e != cudaSuccess) return e;
  if ((e = ds_cnn_infer(net, st, rgb, w, h, h_param * strength_scale, out)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(count_dev, 0, sizeof(unsigned), st)) != cudaSuccess) return e;
  if (ds_cnn_judge_on(net) && (e = ds_cnn_judge_reset(net, st)) != cudaSuccess) return e;
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  return check_judge_fallback(net, st, rgb, w, h, h_param, search, patch, tau, out, flags_scratch, count_dev, 0, ty);
}

// The same for output rows [r0, r1) only, r0 a multiple of the NLM tile
// height: the network runs on rows [r0 - halo, r1 + halo) (clipped to the
// frame) into band_out, whose rows [r0, r1) are exact when halo covers the
// receptive field (35 rows, plus 1 for the input's local mean); they are
// copied into out, then the residual check, the judge and the NLM fallback
// run on the NLM tile rows of the band. count_dev (and, in judge mode, the
// judge statistics: ds_cnn_judge_reset) must be zeroed before the first band,
// and the judge buffers reserved for the whole frame (ds_cnn_reserve_judge).
cudaError_t ds_cnn_denoise_band(DsCnn* net, cudaStream_t st, const float* rgb, int w, int h, int r0, int r1, int halo,
                                float h_param, int search, int patch, float tau, float strength_scale, float* out,
                                float* band_out, unsigned char* flags_scratch, unsigned* count_dev) {
  const int a0 = r0 - halo > 0 ? r0 - halo : 0, a1 = r1 + halo < h ? r1 + halo : h;
  const size_t row = (size_t)w * 3;
  cudaError_t e = ds_cnn_infer(net, st, rgb + (size_t)a0 * row, w, a1 - a0, h_param * strength_scale, band_out);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(out + (size_t)r0 * row, band_out + (size_t)(r0 - a0) * row,
                           (size_t)(r1 - r0) * row * sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return e;
  int tx, ty, tw, th;
  ds_nlm_tile_grid(w, h, patch, &tx, &ty, &tw, &th);
  const int t0 = r0 / th, t1 = (r1 + th - 1) / th;
  return check_judge_fallback(net, st, rgb, w, h, h_param, search, patch, tau, out, flags_scratch, count_dev, t0, t1);
}
