// Separable clamped-edge box blur, image.rs:269-313.
//
// The reference runs a running sum along each row (acc starts at the clamped
// sum of the first window; out = acc * norm; acc += at(x+r+1) - at(x-r)),
// then the same down each column. Floating-point results depend on that
// order, so each GPU thread owns one row (horizontal pass) or one column
// (vertical pass) and repeats the sequence exactly; compiled with
// -fmad=false, the result is bit-identical to the reference.
#include "internal.cuh"

namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__global__ void box_h_kernel(const float* __restrict__ in, int w, int h, int r, float norm, float* __restrict__ out) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= h) return;
  const float* row = in + (size_t)y * w;
  float* o = out + (size_t)y * w;
  float acc = 0.0f;
  for (int i = -r; i <= r; i++) acc += row[clampi(i, 0, w - 1)];
  for (int x = 0; x < w; x++) {
    o[x] = acc * norm;
    acc += row[clampi(x + r + 1, 0, w - 1)] - row[clampi(x - r, 0, w - 1)];
  }
}

__global__ void box_v_kernel(const float* __restrict__ in, int w, int h, int r, float norm, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  float acc = 0.0f;
  for (int i = -r; i <= r; i++) acc += in[(size_t)clampi(i, 0, h - 1) * w + x];
  for (int y = 0; y < h; y++) {
    out[(size_t)y * w + x] = acc * norm;
    acc += in[(size_t)clampi(y + r + 1, 0, h - 1) * w + x] - in[(size_t)clampi(y - r, 0, h - 1) * w + x];
  }
}

// Horizontal pass with coalesced loads: a CTA stages 32 rows x (BOX_CHUNK +
// 2r + 1) columns in shared memory (one chunk at a time) and thread t runs
// row t's running sum through it, carrying the sum across chunks, so the
// arithmetic is exactly the one-thread-per-row sequence above.
constexpr int BOX_ROWS = 32;
constexpr int BOX_CHUNK = 256;
constexpr int BOX_MAX_TILED_R = 64;

__global__ void __launch_bounds__(256) box_h_tiled_kernel(const float* __restrict__ in, int w, int h, int r, float norm,
                                                          float* __restrict__ out) {
  extern __shared__ float tile[];  // BOX_ROWS x pitch
  const int pitch = BOX_CHUNK + 2 * r + 1;  // odd: the 32 rows hit 32 banks
  const int y0 = blockIdx.x * BOX_ROWS;
  const int t = threadIdx.x;
  const int row = t;  // threads 0..31 run the sums
  float acc = 0.0f;
  for (int x0 = 0; x0 < w; x0 += BOX_CHUNK) {
    // stage columns [x0 - r, x0 + BOX_CHUNK + r] (clamped) of the 32 rows
    const int span = pitch;
    for (int i = t; i < BOX_ROWS * span; i += blockDim.x) {
      const int ry = i / span, cx = i - ry * span;
      const int gy = min(y0 + ry, h - 1);
      tile[ry * pitch + cx] = in[(size_t)gy * w + clampi(x0 - r + cx, 0, w - 1)];
    }
    __syncthreads();
    if (row < BOX_ROWS && y0 + row < h) {
      const float* tr = tile + row * pitch + r;  // tr[j] = column x0 + j (clamped)
      float* o = out + (size_t)(y0 + row) * w;
      if (x0 == 0)
        for (int i = -r; i <= r; i++) acc += tr[i];
      const int n = min(BOX_CHUNK, w - x0);
      for (int j = 0; j < n; j++) {
        o[x0 + j] = acc * norm;
        acc += tr[j + r + 1] - tr[j - r];
      }
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t ds_launch_box_blur(cudaStream_t st, const float* in, int w, int h, int r, float* tmp, float* out) {
  const float norm = 1.0f / (float)(2 * r + 1);
  if (r <= BOX_MAX_TILED_R) {
    const size_t smem = (size_t)BOX_ROWS * (BOX_CHUNK + 2 * r + 1) * sizeof(float);
    cudaError_t e0 = cudaFuncSetAttribute(box_h_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e0 != cudaSuccess) return e0;
    box_h_tiled_kernel<<<(h + BOX_ROWS - 1) / BOX_ROWS, 256, smem, st>>>(in, w, h, r, norm, tmp);
  } else {
    box_h_kernel<<<(h + 127) / 128, 128, 0, st>>>(in, w, h, r, norm, tmp);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  box_v_kernel<<<(w + 127) / 128, 128, 0, st>>>(tmp, w, h, r, norm, out);
  return cudaGetLastError();
}
