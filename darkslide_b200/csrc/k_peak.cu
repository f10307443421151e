// Throughput microbenchmarks for the roofline of the NLM kernel, which is
// bound by the SFU (ex2) and FP32 pipes rather than by HBM or tensor cores:
//   ffma_kernel: 8 independent FFMA chains per thread -> FP32 FLOP/s
//   ex2_kernel : 8 independent ex2.approx chains per thread -> ex2/s
//   ffma2_kernel: 8 independent fma.rn.f32x2 chains per thread -> packed FP32 FLOP/s
// Each runs on every SM (grid = 8 x SM count) for a fixed iteration count.
#include "internal.cuh"

namespace {

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__global__ void __launch_bounds__(256) ffma_kernel(int iters, float seed, float* sink) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = seed + threadIdx.x * 1e-7f + i;
  const float m = 0.999999f, c = 1e-7f;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 16; k++)
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = fmaf(a[i], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; i++) s += a[i];
  if (s == 12345.678f) sink[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) ex2_kernel(int iters, float seed, float* sink) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = seed + threadIdx.x * 1e-7f + i * 0.01f;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 16; k++)
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = ex2_approx(-a[i]);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; i++) s += a[i];
  if (s == 12345.678f) sink[0] = s;
}

// packed FP32: 8 independent fma.rn.f32x2 chains (two lanes each) per thread
__global__ void __launch_bounds__(256) ffma2_kernel(int iters, float seed, float* sink) {
  unsigned long long a[8];
  const float m = 0.999999f, c = 1e-7f;
  unsigned long long mm, cc;
  asm("mov.b64 %0, {%1, %2};" : "=l"(mm) : "f"(m), "f"(m));
  asm("mov.b64 %0, {%1, %2};" : "=l"(cc) : "f"(c), "f"(c));
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const float lo = seed + threadIdx.x * 1e-7f + i, hi = lo + 0.5f;
    asm("mov.b64 %0, {%1, %2};" : "=l"(a[i]) : "f"(lo), "f"(hi));
  }
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 16; k++)
#pragma unroll
      for (int i = 0; i < 8; i++) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[i]) : "l"(mm), "l"(cc));
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a[i]));
    s += lo + hi;
  }
  if (s == 12345.678f) sink[0] = s;
}

// legacy warp-level tensor core: 8 independent mma.sync m16n8k16 bf16 chains
__global__ void __launch_bounds__(256) mma_sync_kernel(int iters, unsigned seed, float* sink) {
  float d[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++) d[i][0] = d[i][1] = d[i][2] = d[i][3] = 0.f;
  const unsigned a0 = seed ^ threadIdx.x, a1 = a0 * 3u, a2 = a0 * 5u, a3 = a0 * 7u, b0 = a0 * 11u, b1 = a0 * 13u;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++)
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
          "{%0,%1,%2,%3};"
          : "+f"(d[i][0]), "+f"(d[i][1]), "+f"(d[i][2]), "+f"(d[i][3])
          : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; i++) s += d[i][0] + d[i][1] + d[i][2] + d[i][3];
  if (s == 12345.678f) sink[0] = s;
}

}  // namespace

// BF16 mma.sync throughput (FLOP/s), for the CNN kernels' roofline.
cudaError_t ds_measure_mma_sync(cudaStream_t st, int device, double* flops) {
  int sms = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  float* sink = nullptr;
  if ((e = cudaMallocAsync(&sink, 16, st)) != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = sms * 4, threads = 256, iters = 2048;
  float ms = 0.f;
  for (int rep = 0; rep < 2; rep++) {
    cudaEventRecord(a, st);
    mma_sync_kernel<<<blocks, threads, 0, st>>>(iters, 12345u, sink);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
  }
  *flops = 2.0 * 16 * 8 * 16 * 8.0 * iters * blocks * (threads / 32) / (ms * 1e-3);
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(sink, st);
  cudaStreamSynchronize(st);
  return e;
}

// Times both kernels with CUDA events on `st`; returns FLOP/s and ex2/s.
cudaError_t ds_measure_peaks(cudaStream_t st, int device, double* ffma_flops, double* ex2_per_s,
                             double* ffma2_flops) {
  int sms = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  float* sink = nullptr;
  if ((e = cudaMallocAsync(&sink, 16, st)) != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = sms * 8, threads = 256;
  const int it_f = 256, it_e = 1024;
  float ms = 0.f;
  for (int rep = 0; rep < 2; rep++) {  // first rep warms up
    cudaEventRecord(a, st);
    ffma_kernel<<<blocks, threads, 0, st>>>(it_f, 1.0f, sink);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
  }
  *ffma_flops = 2.0 * 8 * 16 * (double)it_f * blocks * threads / (ms * 1e-3);
  for (int rep = 0; rep < 2; rep++) {
    cudaEventRecord(a, st);
    ex2_kernel<<<blocks, threads, 0, st>>>(it_e, 0.5f, sink);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
  }
  *ex2_per_s = 8.0 * 16 * (double)it_e * blocks * threads / (ms * 1e-3);
  for (int rep = 0; rep < 2; rep++) {
    cudaEventRecord(a, st);
    ffma2_kernel<<<blocks, threads, 0, st>>>(it_f, 1.0f, sink);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
  }
  *ffma2_flops = 2.0 * 2 * 8 * 16 * (double)it_f * blocks * threads / (ms * 1e-3);
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(sink, st);
  cudaStreamSynchronize(st);
  return e;
}
