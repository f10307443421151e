// Non-local means (enhance.rs:36-72) as one tiled kernel.
//
// The reference loops over the (2S+1)^2 search offsets; for each it builds
// the squared-difference plane against the clamped shifted plane (:49-53),
// box-filters it with a clamped separable box of radius P (:54,
// image.rs:269-313), turns the mean distance into a weight exp(-d/h^2)
// (:58) and accumulates weight*sample and weight (:59-60); the result is
// a/max(s,1e-12) (:71).
//
// Here one CTA owns a TX x TY tile of one channel and keeps its a/s
// accumulators in registers across all offsets. Per offset:
//   phase A: each thread takes a 16-wide row segment of the tile (plus P rows
//            above/below), forms the differences against the shifted
//            samples from the shared-memory copy of the tile + (S+P) halo,
//            and writes the horizontal (2P+1)-sums as a running sum into a
//            shared H buffer (double-buffered, so one barrier per offset);
//   phase B: each thread reads a 4x4 block of H columns (float4), forms the
//            vertical (2P+1)-sums as a running sum, and accumulates
//            w = 2^(sum * kexp) (kexp = -log2(e) / (2P+1)^2 / h^2) times the
//            shifted sample.
// Clamped edges: the shared copy is loaded at clamped coordinates, so the
// shifted sample p_clamped(x+o) is a plain shared read; the box filter of the
// reference clamps the DIFFERENCE plane, so rows are clamped per segment and,
// in tiles whose patch window leaves the image, columns per element.
#include "internal.cuh"

namespace {

constexpr int NLM_THREADS = 256;
constexpr int TX = 64, TY = 64;
constexpr int SEG = 16;
constexpr int SEGS_PER_ROW = TX / SEG;

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__host__ __device__ constexpr int nlm_h_rows(int P) { return TY + 2 * P; }

__host__ size_t nlm_smem_bytes(int S, int P) {
  const int R = S + P;
  const size_t pr = (size_t)(TX + 2 * R) * (TY + 2 * R);
  const size_t pr_al = (pr + 3) & ~(size_t)3;
  return (pr_al + 2 * (size_t)nlm_h_rows(P) * TX) * sizeof(float);
}

template <int P>
__global__ void __launch_bounds__(NLM_THREADS) nlm_tile_kernel(const float* __restrict__ in, int W, int H, int C,
                                                               int S, float kexp, float* __restrict__ out) {
  constexpr int HR = nlm_h_rows(P);
  constexpr int NSEG = HR * SEGS_PER_ROW;
  constexpr int DW = SEG + 2 * P;
  const int R = S + P;
  const int PW = TX + 2 * R, PH = TY + 2 * R;
  extern __shared__ float4 smem4[];
  float* PR = reinterpret_cast<float*>(smem4);
  float* HB = PR + ((PW * PH + 3) & ~3);

  const int ch = blockIdx.z;
  const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
  const int tid = threadIdx.x;

  for (int i = tid; i < PW * PH; i += NLM_THREADS) {
    const int ly = i / PW, lx = i - ly * PW;
    const int gx = clampi(X0 - R + lx, 0, W - 1), gy = clampi(Y0 - R + ly, 0, H - 1);
    PR[i] = in[((size_t)gy * W + gx) * C + ch];
  }
  __syncthreads();

  const bool xin = (X0 - P >= 0) && (X0 + TX + P <= W);
  const int bx = (tid & 15) * 4, by = (tid >> 4) * 4;
  float a[16], s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    a[i] = 0.f;
    s[i] = 0.f;
  }

  int par = 0;
  for (int dy = -S; dy <= S; dy++) {
    for (int dx = -S; dx <= S; dx++) {
      float* Hb = HB + par * (HR * TX);
      // phase A: horizontal sums of the squared differences
      for (int seg = tid; seg < NSEG; seg += NLM_THREADS) {
        const int row = seg / SEGS_PER_ROW;
        const int x0 = (seg - row * SEGS_PER_ROW) * SEG;
        const int gy = clampi(Y0 + row - P, 0, H - 1);
        const float* rp = PR + (gy - (Y0 - R)) * PW;
        const float* rq = rp + dy * PW + dx;
        float d[DW];
        if (xin) {
          const int lx0 = x0 - P + R;
#pragma unroll
          for (int k = 0; k < DW; k++) d[k] = rp[lx0 + k] - rq[lx0 + k];
        } else {
#pragma unroll
          for (int k = 0; k < DW; k++) {
            const int lx = clampi(X0 + x0 - P + k, 0, W - 1) - (X0 - R);
            d[k] = rp[lx] - rq[lx];
          }
        }
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k <= 2 * P; k++) acc = fmaf(d[k], d[k], acc);
        float* hrow = Hb + row * TX + x0;
        hrow[0] = acc;
#pragma unroll
        for (int j = 1; j < SEG; j++) {
          acc = fmaf(d[j + 2 * P], d[j + 2 * P], acc);
          acc = fmaf(-d[j - 1], d[j - 1], acc);
          hrow[j] = acc;
        }
      }
      __syncthreads();
      // phase B: vertical sums, weights, accumulation
      float4 hv[4 + 2 * P];
#pragma unroll
      for (int r = 0; r < 4 + 2 * P; r++) hv[r] = *reinterpret_cast<const float4*>(Hb + (by + r) * TX + bx);
      const float* qrow = PR + (by + R + dy) * PW + bx + R + dx;
#pragma unroll
      for (int col = 0; col < 4; col++) {
        auto hc = [&](int r) -> float {
          return col == 0 ? hv[r].x : col == 1 ? hv[r].y : col == 2 ? hv[r].z : hv[r].w;
        };
        float v = 0.f;
#pragma unroll
        for (int r = 0; r <= 2 * P; r++) v += hc(r);
#pragma unroll
        for (int t = 0; t < 4; t++) {
          if (t > 0) v = v + hc(t + 2 * P) - hc(t - 1);
          const float wgt = ex2_approx(v * kexp);
          const float q = qrow[t * PW + col];
          a[t * 4 + col] = fmaf(wgt, q, a[t * 4 + col]);
          s[t * 4 + col] += wgt;
        }
      }
      par ^= 1;
    }
  }

#pragma unroll
  for (int t = 0; t < 4; t++)
#pragma unroll
    for (int col = 0; col < 4; col++) {
      const int gx = X0 + bx + col, gy = Y0 + by + t;
      if (gx < W && gy < H)
        out[((size_t)gy * W + gx) * C + ch] = __fdiv_rn(a[t * 4 + col], fmaxf(s[t * 4 + col], 1e-12f));
    }
}

template <int P>
cudaError_t launch_nlm_p(cudaStream_t st, const float* in, int w, int h, int C, int S, float kexp, float* out) {
  const size_t smem = nlm_smem_bytes(S, P);
  cudaError_t e = cudaFuncSetAttribute(nlm_tile_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((w + TX - 1) / TX, (h + TY - 1) / TY, C);
  nlm_tile_kernel<P><<<grid, NLM_THREADS, smem, st>>>(in, w, h, C, S, kexp, out);
  return cudaGetLastError();
}

}  // namespace

cudaError_t ds_launch_nlm(cudaStream_t st, const float* in, int w, int h, int channels, float h_param, int search,
                          int patch, float* out) {
  // enhance.rs:40: h2 = max(h*h, 1e-12) in f32; box_blur's norm is 1/(2r+1)
  // in f32 and is applied once per pass (image.rs:274, 285, 307).
  const float h2 = fmaxf(h_param * h_param, 1e-12f);
  const float norm = patch == 0 ? 1.0f : 1.0f / (float)(2 * patch + 1);
  const double kexp = -((double)norm * (double)norm) / (double)h2 * 1.4426950408889634;
  const float k = (float)kexp;
  switch (patch) {
    case 0: return launch_nlm_p<0>(st, in, w, h, channels, search, k, out);
    case 1: return launch_nlm_p<1>(st, in, w, h, channels, search, k, out);
    case 2: return launch_nlm_p<2>(st, in, w, h, channels, search, k, out);
    case 3: return launch_nlm_p<3>(st, in, w, h, channels, search, k, out);
    case 4: return launch_nlm_p<4>(st, in, w, h, channels, search, k, out);
    case 5: return launch_nlm_p<5>(st, in, w, h, channels, search, k, out);
    case 6: return launch_nlm_p<6>(st, in, w, h, channels, search, k, out);
    case 7: return launch_nlm_p<7>(st, in, w, h, channels, search, k, out);
    default: return cudaErrorInvalidValue;
  }
}
