// Inference convolutions of the learned path on the 5th-generation tensor
// cores (tcgen05). Same network and tensors as k_cnn.cu (NHWC bf16
// activations, [9][cout][cin] bf16 weights); the difference is the engine:
//
//   - operands in shared memory, in the canonical no-swizzle K-major layout:
//     core matrices of 8 rows x 16 bytes; the staged input tile is stored
//     channel-block-major ([8-channel block][pixel][8 channels]), so the A
//     operand of every 3x3 tap is the same layout shifted by whole pixels
//     (one descriptor per tap, no im2col copy);
//   - one CTA = 128 threads; a tile is TR output rows x 128 pixels; per row
//     and per tap/16-channel step one elected thread issues
//     tcgen05.mma.cta_group::1.kind::f16 (M 128 = pixels, N = output channels,
//     K 16, BF16 in, FP32 accumulate) into that row's TMEM accumulator;
//   - tcgen05.commit arrives on an mbarrier; the four warps wait for it (with
//     a time-bounded wait that reports DSGPU_ERR_TIMEOUT through `err` instead of
//     hanging), read their 32 TMEM lanes with tcgen05.ld and run the
//     epilogue (bias, ReLU or residual) straight to global memory;
//   - CTAs are persistent (weights staged once), two per SM so one CTA's
//     loads overlap the other's MMAs.
// No TMA multicast and no cluster features are used.
#include <cuda_bf16.h>

#include "internal.cuh"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int TC_THREADS = 128;
constexpr int TC_M = 128;    // pixels per MMA (one output row segment)
constexpr int TC_TR = 2;     // output rows per tile
constexpr int TC_PW = TC_M + 2;  // staged pixels per row (1-pixel halo each side)
constexpr int TC_PR = TC_TR + 2; // staged rows
constexpr int TC_NPIX = TC_PW * TC_PR;
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;  // give up on an MMA batch after 2 s

enum { TC_RELU = 0, TC_RESID = 1 };

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// canonical no-swizzle K-major shared-memory matrix descriptor (version 1)
__device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 A/B, FP32 D, both K-major, M x N
__host__ __device__ constexpr unsigned umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                         unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tmem_ld16(unsigned addr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for mbarrier phase `parity`; false once TC_WAIT_NS have passed.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (globaltimer_ns() - t0 > TC_WAIT_NS) return false;
  }
}

template <int CIN, int COUT_G, int N, int EPI>
__global__ void __launch_bounds__(TC_THREADS) conv_tc_kernel(const bf16* __restrict__ x, int H, int W,
                                                             const bf16* __restrict__ wt /*[9][COUT_G][CIN]*/,
                                                             const float* __restrict__ bias, bf16* __restrict__ y,
                                                             const float* __restrict__ resid,
                                                             float* __restrict__ yf, int* __restrict__ err) {
  static_assert(CIN % 16 == 0 && N % 16 == 0 && N >= COUT_G, "shapes");
  constexpr int CB = CIN / 8;                  // 8-channel blocks of the input
  constexpr int A_BYTES = CB * TC_NPIX * 16;   // staged tile, [cb][pixel][8]
  constexpr int B_BYTES = 9 * CB * N * 16;     // weights, [tap][cb][co][8]
  constexpr int NCOLS = (TC_TR * N <= 32) ? 32 : (TC_TR * N <= 64) ? 64 : (TC_TR * N <= 128) ? 128 : 256;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* As = sm;
  unsigned char* Bs = sm + A_BYTES;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + A_BYTES + B_BYTES);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(sm + A_BYTES + B_BYTES + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // weights: [tap][co][cin] -> [tap][cb][co][8], output channels >= COUT_G zero
  for (int i = tid; i < 9 * CB * N; i += TC_THREADS) {
    const int tap = i / (CB * N), r = i - tap * CB * N, cb = r / N, co = r - cb * N;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (co < COUT_G) v = *reinterpret_cast<const uint4*>(wt + ((size_t)tap * COUT_G + co) * CIN + cb * 8);
    *reinterpret_cast<uint4*>(Bs + (size_t)i * 16) = v;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(NCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;
  const unsigned bar_a = smem_u32(bar);
  const unsigned a_base = smem_u32(As), b_base = smem_u32(Bs);
  constexpr unsigned IDESC = umma_idesc(TC_M, N);

  const int tiles_x = (W + TC_M - 1) / TC_M, tiles_y = (H + TC_TR - 1) / TC_TR;
  const int ntiles = tiles_x * tiles_y;
  unsigned phase = 0;
  bool ok = true;
  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int ty = t / tiles_x, x0 = (t - ty * tiles_x) * TC_M, y0 = ty * TC_TR;
    // stage rows y0-1 .. y0+TC_TR, pixels x0-1 .. x0+TC_M (zero outside the image)
    for (int i = tid; i < TC_NPIX * CB; i += TC_THREADS) {
      const int pix = i / CB, cb = i - pix * CB;
      const int pr = pix / TC_PW, pc = pix - pr * TC_PW;
      const int gy = y0 - 1 + pr, gx = x0 - 1 + pc;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gy >= 0 && gy < H && gx >= 0 && gx < W)
        v = *reinterpret_cast<const uint4*>(x + ((size_t)gy * W + gx) * CIN + cb * 8);
      *reinterpret_cast<uint4*>(As + ((size_t)cb * TC_NPIX + pix) * 16) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0 && lane == 0) {
#pragma unroll 1
      for (int r = 0; r < TC_TR; r++) {
        unsigned acc = 0;
#pragma unroll 1
        for (int tap = 0; tap < 9; tap++) {
          const int ky = tap / 3, kx = tap % 3;
#pragma unroll
          for (int kc = 0; kc < CIN / 16; kc++) {
            const unsigned a_addr = a_base + (unsigned)((2 * kc) * TC_NPIX + (r + ky) * TC_PW + kx) * 16u;
            const unsigned b_addr = b_base + (unsigned)((tap * CB + 2 * kc) * N) * 16u;
            mma_bf16(tmem + (unsigned)(r * N), umma_desc(a_addr, TC_NPIX * 16, 128), umma_desc(b_addr, N * 16, 128),
                     IDESC, acc);
            acc = 1;
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                   : "memory");
    }
    __syncwarp();
    // every thread waits (bounded); the CTA then agrees on the outcome so
    // that all threads take the same path to the same barriers
    const int timed_out = __syncthreads_or(!mbar_wait(bar_a, phase));
    if (timed_out) {
      if (tid == 0) atomicExch(err, DSGPU_ERR_TIMEOUT);
      ok = false;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      // epilogue: lane l of warp w holds pixel 32w + l of each row
      const int px = x0 + warp * 32 + lane;
#pragma unroll 1
      for (int r = 0; r < TC_TR; r++) {
        const int gy = y0 + r;
        float v[N];
#pragma unroll
        for (int j = 0; j < N / 16; j++)
          tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(r * N + j * 16), v + j * 16);
        if (gy >= H || px >= W) continue;
        const size_t pix = (size_t)gy * W + px;
        if (EPI == TC_RELU) {
#pragma unroll
          for (int c = 0; c < COUT_G; c += 8) {
            __align__(16) __nv_bfloat162 o[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
              o[k] = __floats2bfloat162_rn(fmaxf(v[c + 2 * k] + bias[c + 2 * k], 0.f),
                                           fmaxf(v[c + 2 * k + 1] + bias[c + 2 * k + 1], 0.f));
            *reinterpret_cast<uint4*>(y + pix * COUT_G + c) = *reinterpret_cast<uint4*>(o);
          }
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++) yf[pix * 3 + c] = resid[pix * 3 + c] + (v[c] + bias[c]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // every thread is done with this tile's TMEM and shared tile
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS));
}

template <int CIN, int COUT_G, int N, int EPI>
cudaError_t launch_tc(cudaStream_t st, const bf16* x, int H, int W, const bf16* wt, const float* bias, bf16* y,
                      const float* resid, float* yf, int* err) {
  constexpr size_t smem = (size_t)(CIN / 8) * TC_NPIX * 16 + (size_t)9 * (CIN / 8) * N * 16 + 16;
  cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT_G, N, EPI>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = ((W + TC_M - 1) / TC_M) * ((H + TC_TR - 1) / TC_TR);
  const int grid = tiles < 2 * sms ? tiles : 2 * sms;
  conv_tc_kernel<CIN, COUT_G, N, EPI><<<grid, TC_THREADS, smem, st>>>(x, H, W, wt, bias, y, resid, yf, err);
  return cudaGetLastError();
}

}  // namespace

// One image through the 8 layers on the tensor cores. x16: packed input
// (16 ch); a, b: ping-pong activations (48 ch); wf/bias: per-layer forward
// weights (layer 8's with 8 output channels); rgb/out: fp32 RGB.
cudaError_t ds_cnn_forward_tc(cudaStream_t st, const void* x16, void* a, void* b, int H, int W,
                              const void* const* wf, const float* const* bias, const float* rgb, float* out,
                              int* err) {
  const bf16* in = static_cast<const bf16*>(x16);
  bf16* pa = static_cast<bf16*>(a);
  bf16* pb = static_cast<bf16*>(b);
  cudaError_t e = launch_tc<16, 48, 48, TC_RELU>(st, in, H, W, static_cast<const bf16*>(wf[0]), bias[0], pa, nullptr,
                                                 nullptr, err);
  for (int l = 1; l < 7 && e == cudaSuccess; l++) {
    e = launch_tc<48, 48, 48, TC_RELU>(st, pa, H, W, static_cast<const bf16*>(wf[l]), bias[l], pb, nullptr, nullptr,
                                       err);
    bf16* t = pa;
    pa = pb;
    pb = t;
  }
  if (e == cudaSuccess)
    e = launch_tc<48, 8, 16, TC_RESID>(st, pa, H, W, static_cast<const bf16*>(wf[7]), bias[7], nullptr, rgb, out,
                                       err);
  return e;
}
