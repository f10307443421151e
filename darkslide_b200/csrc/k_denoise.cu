// enhance::denoise (enhance.rs:75-92) on the GPU:
//   Oklab L/a/b planes (color.rs:401-406) -> noise sigma of L
//   (estimate_noise, enhance.rs:10-32) -> NLM of L with search 3, patch 1 and
//   h = sigma (0.6 + 1.6k) -> blend -> guided filters of a and b guided by the
//   blended L (image.rs:385-405) -> back to ProPhoto (color.rs:408-412), >= 0.
// Compiled with -fmad=false: the elementwise steps round every product as the
// reference does. sigma stays on the device: the NLM kernel and the guided
// filter's eps read it from there, so the whole composite runs without a
// host round trip.
#include "color.h"
#include "internal.cuh"

namespace {

struct OkM {
  float to_lms[9], from_lms[9], m2[9], m2_inv[9];
};

__device__ __forceinline__ void mv(const float* m, float a, float b, float c, float& o0, float& o1, float& o2) {
  o0 = m[0] * a + m[1] * b + m[2] * c;  // color.rs:11-13, left to right
  o1 = m[3] * a + m[4] * b + m[5] * c;
  o2 = m[6] * a + m[7] * b + m[8] * c;
}

__global__ void oklab_fwd_kernel(const float* __restrict__ rgb, size_t n, OkM m, float* __restrict__ L,
                                 float* __restrict__ A, float* __restrict__ B) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float l0, l1, l2;
  mv(m.to_lms, rgb[i * 3], rgb[i * 3 + 1], rgb[i * 3 + 2], l0, l1, l2);
  mv(m.m2, cbrtf(l0), cbrtf(l1), cbrtf(l2), L[i], A[i], B[i]);
}

__global__ void oklab_inv_kernel(const float* __restrict__ L, const float* __restrict__ A,
                                 const float* __restrict__ B, size_t n, OkM m, float* __restrict__ rgb) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float l0, l1, l2, r, g, b;
  mv(m.m2_inv, L[i], A[i], B[i], l0, l1, l2);
  mv(m.from_lms, l0 * l0 * l0, l1 * l1 * l1, l2 * l2 * l2, r, g, b);
  rgb[i * 3] = fmaxf(r, 0.0f);
  rgb[i * 3 + 1] = fmaxf(g, 0.0f);
  rgb[i * 3 + 2] = fmaxf(b, 0.0f);
}

// estimate_noise samples: |4c - l - r - u - d| at i = 0, step, 2 step, ...
// (enhance.rs:12-24), border sites skipped; the keys are the float bits
// (non-negative floats order like their bit patterns). Order is irrelevant:
// only the median is used.
__global__ void noise_samples_kernel(const float* __restrict__ p, int w, int h, long long step, long long nsamp,
                                     unsigned* __restrict__ keys, unsigned* __restrict__ count) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nsamp) return;
  const long long i = j * step;
  const int x = (int)(i % w), y = (int)(i / w);
  if (x < 1 || y < 1 || x + 1 >= w || y + 1 >= h) return;
  const float c = p[i];
  const float lap = 4.0f * c - p[i - 1] - p[i + 1] - p[i - w] - p[i + w];
  keys[atomicAdd(count, 1u)] = __float_as_uint(fabsf(lap));
}

// One CTA: radix-select the median key (select_nth_unstable at len/2,
// enhance.rs:28-29) in four 8-bit passes, then sigma = v / 0.6745 / sqrt(20)
// floored at 1e-4 (enhance.rs:31, :82). Also writes the NLM strength
// sigma (0.6 + 1.6k) and the guided filter's eps = (2 sigma)^2 (:84, :88).
__global__ void __launch_bounds__(1024) noise_select_kernel(const unsigned* __restrict__ keys,
                                                            const unsigned* __restrict__ count, float k,
                                                            float* __restrict__ out3) {
  __shared__ unsigned hist[256];
  __shared__ unsigned s_prefix, s_k;
  const unsigned n = *count;
  if (threadIdx.x == 0) {
    s_prefix = 0;
    s_k = n / 2;
  }
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    const unsigned mask = shift == 24 ? 0u : (~0u << (shift + 8));
    const unsigned pre = s_prefix;
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
      const unsigned key = keys[i];
      if ((key & mask) == pre) atomicAdd(&hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned cum = 0, kk = s_k;
      for (int b = 0; b < 256; b++) {
        if (cum + hist[b] > kk) {
          s_prefix = pre | ((unsigned)b << shift);
          s_k = kk - cum;
          break;
        }
        cum += hist[b];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    float sigma = 0.0f;  // enhance.rs:25-27: no samples -> 0
    if (n > 0) sigma = __fdiv_rn(__fdiv_rn(__uint_as_float(s_prefix), 0.6745f), __fsqrt_rn(20.0f));
    out3[3] = sigma;  // estimate_noise itself (enhance.rs:31), before denoise's floor
    sigma = fmaxf(sigma, 1e-4f);
    out3[0] = sigma;
    out3[1] = sigma * (0.6f + 1.6f * k);
    const float s2 = sigma * 2.0f;
    out3[2] = s2 * s2;
  }
}

__global__ void blend_kernel(const float* __restrict__ l, const float* __restrict__ lf, size_t n, float t,
                             float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = l[i] + (lf[i] - l[i]) * t;  // enhance.rs:86
}

__global__ void mul_kernel(const float* __restrict__ a, const float* __restrict__ b, size_t n, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] * b[i];
}

// image.rs:395-400; eps from the device (host value when eps_dev is null)
__global__ void guided_coef_kernel(const float* __restrict__ mi, const float* __restrict__ mp,
                                   const float* __restrict__ mip, const float* __restrict__ mii, size_t n,
                                   const float* __restrict__ eps_dev, float eps_host, float* __restrict__ ca,
                                   float* __restrict__ cb) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float eps = eps_dev ? *eps_dev : eps_host;
  const float cov = mip[i] - mi[i] * mp[i];
  const float var = mii[i] - mi[i] * mi[i];
  const float a = __fdiv_rn(cov, var + eps);
  ca[i] = a;
  cb[i] = mp[i] - a * mi[i];
}

__global__ void guided_out_kernel(const float* __restrict__ ma, const float* __restrict__ mb,
                                  const float* __restrict__ I, size_t n, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = ma[i] * I[i] + mb[i];  // image.rs:404
}

inline unsigned nblk(size_t n) { return (unsigned)((n + 255) / 256); }

OkM ok_matrices() {
  const dscolor::OklabMatrices o = dscolor::oklab_matrices();
  OkM m;
  std::memcpy(m.to_lms, o.to_lms, sizeof(m.to_lms));
  std::memcpy(m.from_lms, o.from_lms, sizeof(m.from_lms));
  std::memcpy(m.m2, o.m2, sizeof(m.m2));
  std::memcpy(m.m2_inv, o.m2_inv, sizeof(m.m2_inv));
  return m;
}

}  // namespace

// Scratch layout for the composite (all in units of n = w*h floats):
// L A B LF L2 MI MII MP IP MIP CA CB MA MB TMP = 15 planes, then the noise
// keys (up to 2*200000 + 1 u32), the key count and 3 scalars.
size_t ds_denoise_scratch_bytes(int w, int h) {
  const size_t n = (size_t)w * h;
  return (15 * n + 400008 + 8) * sizeof(float);
}

size_t ds_noise_scratch_bytes(int w, int h) {
  (void)w;
  (void)h;
  return (400008 + 8) * sizeof(float);
}

// Into out3 (4 device floats): sigma floored at 1e-4 as denoise uses it, the
// NLM strength and guided-filter eps for amount k, and the unfloored sigma.
cudaError_t ds_launch_estimate_noise(cudaStream_t st, const float* p, int w, int h, float k, void* scratch,
                                     float* out3) {
  unsigned* keys = static_cast<unsigned*>(scratch);
  unsigned* count = keys + 400008;
  const long long n = (long long)w * h;
  const long long step = n / 200000 > 1 ? n / 200000 : 1;  // enhance.rs:12
  const long long nsamp = (n + step - 1) / step;
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  if (nsamp > 0) noise_samples_kernel<<<(unsigned)((nsamp + 255) / 256), 256, 0, st>>>(p, w, h, step, nsamp, keys, count);
  noise_select_kernel<<<1, 1024, 0, st>>>(keys, count, k, out3);
  return cudaGetLastError();
}

cudaError_t ds_launch_guided_filter(cudaStream_t st, const float* I, const float* p, int w, int h, int r,
                                    const float* eps_dev, float eps_host, float* out, float* scratch /*7 planes*/,
                                    const float* mean_i, const float* mean_ii) {
  const size_t n = (size_t)w * h;
  float* mp = scratch;
  float* ip = scratch + n;
  float* mip = scratch + 2 * n;
  float* ca = scratch + 3 * n;
  float* cb = scratch + 4 * n;
  float* ma = scratch + 5 * n;
  float* tmp = scratch + 6 * n;
  float* mb = ip;  // ip is dead once mip is formed
  cudaError_t e;
  if ((e = ds_launch_box_blur(st, p, w, h, r, tmp, mp)) != cudaSuccess) return e;
  mul_kernel<<<nblk(n), 256, 0, st>>>(I, p, n, ip);
  if ((e = ds_launch_box_blur(st, ip, w, h, r, tmp, mip)) != cudaSuccess) return e;
  guided_coef_kernel<<<nblk(n), 256, 0, st>>>(mean_i, mp, mip, mean_ii, n, eps_dev, eps_host, ca, cb);
  if ((e = ds_launch_box_blur(st, ca, w, h, r, tmp, ma)) != cudaSuccess) return e;
  if ((e = ds_launch_box_blur(st, cb, w, h, r, tmp, mb)) != cudaSuccess) return e;
  guided_out_kernel<<<nblk(n), 256, 0, st>>>(ma, mb, I, n, out);
  return cudaGetLastError();
}

// mean_i = box(I), mean_ii = box(I*I): shared by every guided filter with guide I
cudaError_t ds_launch_guide_means(cudaStream_t st, const float* I, int w, int h, int r, float* mean_i, float* mean_ii,
                                  float* tmp, float* tmp2) {
  const size_t n = (size_t)w * h;
  cudaError_t e;
  if ((e = ds_launch_box_blur(st, I, w, h, r, tmp, mean_i)) != cudaSuccess) return e;
  mul_kernel<<<nblk(n), 256, 0, st>>>(I, I, n, tmp2);
  return ds_launch_box_blur(st, tmp2, w, h, r, tmp, mean_ii);
}

cudaError_t ds_launch_denoise(cudaStream_t st, const float* rgb, int w, int h, float amount, void* scratch,
                              float* out, float* sigma_dev_out, unsigned* launches) {
  const size_t n = (size_t)w * h;
  float* base = static_cast<float*>(scratch);
  float *L = base, *A = base + n, *B = base + 2 * n, *LF = base + 3 * n, *L2 = base + 4 * n;
  float *MI = base + 5 * n, *MII = base + 6 * n, *GS = base + 7 * n;  // GS: 7 guided-filter planes + 1
  float* noise = base + 15 * n;
  float* scal = noise + 400012;  // after the keys and their count
  const OkM m = ok_matrices();
  const float k = amount / 100.0f;  // enhance.rs:83
  cudaError_t e;
  unsigned nl = 0;
  oklab_fwd_kernel<<<nblk(n), 256, 0, st>>>(rgb, n, m, L, A, B);
  nl++;
  if ((e = ds_launch_estimate_noise(st, L, w, h, k, noise, scal)) != cudaSuccess) return e;
  nl += 2;
  if ((e = ds_launch_nlm_dev_h(st, L, w, h, 1, scal + 1, 3, 1, LF)) != cudaSuccess) return e;
  nl++;
  blend_kernel<<<nblk(n), 256, 0, st>>>(L, LF, n, 0.5f + 0.5f * k, L2);
  nl++;
  const int mx = w > h ? w : h;
  float rf = ((float)mx / 600.0f) * (1.0f + 2.0f * k);  // enhance.rs:87
  rf = rf > 2.0f ? rf : 2.0f;
  const int r = (int)rf;
  if ((e = ds_launch_guide_means(st, L2, w, h, r, MI, MII, GS + 6 * n, GS)) != cudaSuccess) return e;
  nl += 5;
  // a2 into LF (dead), b2 into L (dead after the blend)
  if ((e = ds_launch_guided_filter(st, L2, A, w, h, r, scal + 2, 0.0f, LF, GS, MI, MII)) != cudaSuccess) return e;
  if ((e = ds_launch_guided_filter(st, L2, B, w, h, r, scal + 2, 0.0f, L, GS, MI, MII)) != cudaSuccess) return e;
  nl += 2 * 11;
  oklab_inv_kernel<<<nblk(n), 256, 0, st>>>(L2, LF, L, n, m, out);
  nl++;
  if (sigma_dev_out) {
    if ((e = cudaMemcpyAsync(sigma_dev_out, scal, sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
  }
  if (launches) *launches = nl;
  return cudaGetLastError();
}

void ds_oklab_matrices(float out[27]) {
  const dscolor::OklabMatrices o = dscolor::oklab_matrices();
  std::memcpy(out, o.to_lms, 9 * sizeof(float));
  std::memcpy(out + 9, o.from_lms, 9 * sizeof(float));
  std::memcpy(out + 18, o.m2_inv, 9 * sizeof(float));
}
