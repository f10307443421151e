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

}  // namespace

cudaError_t ds_launch_box_blur(cudaStream_t st, const float* in, int w, int h, int r, float* tmp, float* out) {
  const float norm = 1.0f / (float)(2 * r + 1);
  box_h_kernel<<<(h + 127) / 128, 128, 0, st>>>(in, w, h, r, norm, tmp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  box_v_kernel<<<(w + 127) / 128, 128, 0, st>>>(tmp, w, h, r, norm, out);
  return cudaGetLastError();
}
