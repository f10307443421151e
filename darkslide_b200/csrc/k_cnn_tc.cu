// Inference convolutions of the learned path on the 5th-generation tensor
// cores (tcgen05). Same network and tensors as k_cnn.cu (NHWC bf16
// activations, [9][cout][cin] bf16 weights); the difference is the engine.
//
// Layout. Operands sit in shared memory in the canonical no-swizzle K-major
// layout (core matrices of 8 rows x 16 bytes). The input tile (TR+2 rows x
// 130 pixels, one pixel of halo each side) is stored channel-block-major,
// [8-channel block][row][pixel][8 channels], so the A operand (M = 128
// pixels, K = 16 channels) of any tap is the same layout shifted by whole
// pixels: one descriptor per (input row, kx), no im2col copy. One TMA box per
// 8-channel block loads it, zero-filled outside the image.
//
// Stacked taps. Input row j feeds output rows j, j-1, j-2 through weight
// rows ky = 0, 1, 2. The three ky weight blocks are stacked along N, and the
// output-row accumulators are laid out in TMEM in descending row order, so
// one MMA per (input row, kx, 16 channels) with N = 3 x 48 covers all three
// output rows (N = 48 or 96 at the tile's top and bottom edges). A 128 x 48 x
// 16 MMA is bound by reading its 4 KB A operand from shared memory, not by
// math, so stacking cuts the tensor time per output row by ~1.7x. The first
// MMA into an output row's accumulator is split off with accumulate = 0.
//
// Roles (one persistent CTA of 192 threads per SM, weights staged once):
//   warp 5  TMA producer: input tile k into shared-memory stage k % 2;
//   warp 4  MMA issuer: tcgen05.mma.cta_group::1.kind::f16 (BF16 in, FP32
//           accumulate) into TMEM accumulator set k % 2, then tcgen05.commit
//           to release the smem stage and to hand the set to the epilogue;
//   warps 0-3  epilogue: tcgen05.ld of their 32 TMEM lanes (pixels), bias,
//           ReLU or residual, straight to global memory; they release the
//           accumulator set after reading it.
// Every mbarrier wait is bounded in time (2 s); a wait that gives up sets a
// CTA-wide abort flag, which every other wait honours, reports
// DSGPU_ERR_TIMEOUT through `err`, and the CTA waits (bounded) for its copies
// and MMAs in flight before freeing its TMEM. No TMA multicast and no cluster
// features are used.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "internal.cuh"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int TC_EPI_WARPS = 4;
constexpr int TC_THREADS = 32 * (TC_EPI_WARPS + 2);  // + MMA warp + TMA warp
constexpr int TC_M = 128;                          // pixels per MMA (one output-row segment)
constexpr int TC_TR = 4;                           // output rows per tile
constexpr int TC_PW = TC_M + 2;                    // staged pixels per row (1-pixel halo each side)
constexpr int TC_PR = TC_TR + 2;                   // staged rows
constexpr int TC_SLAB = ((TC_PW * TC_PR * 16 + 127) / 128) * 128;  // bytes per 8-channel block, 128-B aligned
constexpr int TC_TMEM_COLS = 512;                  // accumulator sets at columns 0 and 256
constexpr size_t TC_MIN_SMEM = 120 * 1024;         // keeps one CTA per SM (the TMEM plan assumes it)
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

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

template <int ACC>
__device__ __forceinline__ void mma_bf16(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "n"(ACC));
}

__device__ __forceinline__ void tmem_ld16_async(unsigned addr, unsigned* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the completion of mbarrier phase `parity`. Gives up after
// TC_WAIT_NS (setting *abort) or as soon as another role has set *abort.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, volatile int* abort) {
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    if (mbar_test(bar, parity)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > TC_WAIT_NS) {
      *abort = 1;
      return false;
    }
  }
}

// The same wait for the drain after an abort: bounded, ignores the flag.
__device__ __forceinline__ void mbar_drain(unsigned bar, unsigned parity) {
  const unsigned long long t0 = globaltimer_ns();
  while (!mbar_test(bar, parity) && globaltimer_ns() - t0 < TC_WAIT_NS) {
  }
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// TMA load of one 3-D box (channels, x, y) into shared memory, completing on bar
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int c, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// x: [H][W][CIN] bf16 through `xmap` (box 8 x TC_PW x TC_PR); wt: [9][COUT_G][CIN]
// bf16; NK: output channels per ky block (COUT_G padded to a multiple of 16).
template <int CIN, int COUT_G, int NK, int EPI>
__global__ void __launch_bounds__(TC_THREADS, 1)
    conv_tc_kernel(const __grid_constant__ CUtensorMap xmap, int H, int W, const bf16* __restrict__ wt,
                   const float* __restrict__ bias, bf16* __restrict__ y, const float* __restrict__ resid,
                   float* __restrict__ yf, int* __restrict__ err) {
  static_assert(CIN % 16 == 0 && NK % 16 == 0 && NK >= COUT_G && TC_TR * NK <= 256 && 3 * NK <= 256, "shapes");
  constexpr int CB = CIN / 8;              // 8-channel blocks of the input
  constexpr int A_BYTES = CB * TC_SLAB;    // one staged tile
  constexpr int NS = 3 * NK;               // stacked B rows (ky, co)
  constexpr int B_BYTES = 3 * CB * NS * 16;  // weights, [kx][cb][ky*NK + co][8]
  constexpr unsigned TX_BYTES = CB * 8 * TC_PW * TC_PR * 2;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* As = sm;                  // two stages
  unsigned char* Bs = sm + 2 * A_BYTES;
  float* bias_s = reinterpret_cast<float*>(sm + 2 * A_BYTES + B_BYTES);  // NK floats
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(sm + 2 * A_BYTES + B_BYTES + NK * 4);
  // bars: full[2], empty[2], tfull[2], tempty[2]
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 8) + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned bar0 = smem_u32(bars);
  auto full = [&](int s) { return bar0 + 8u * s; };
  auto empty = [&](int s) { return bar0 + 16u + 8u * s; };
  auto tfull = [&](int s) { return bar0 + 32u + 8u * s; };
  auto tempty = [&](int s) { return bar0 + 48u + 8u * s; };

  for (int i = tid; i < 3 * CB * NS; i += TC_THREADS) {
    const int kx = i / (CB * NS), r = i - kx * CB * NS, cb = r / NS, n = r - cb * NS;
    const int ky = n / NK, co = n - ky * NK;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (co < COUT_G)
      v = *reinterpret_cast<const uint4*>(wt + ((size_t)(ky * 3 + kx) * COUT_G + co) * CIN + cb * 8);
    *reinterpret_cast<uint4*>(Bs + (size_t)i * 16) = v;
  }
  for (int i = tid; i < NK; i += TC_THREADS) bias_s[i] = i < COUT_G ? bias[i] : 0.f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < 2; s++) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
      mbar_init(tfull(s), 1);
      mbar_init(tempty(s), TC_EPI_WARPS);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // weights -> async proxy
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  const int tiles_x = (W + TC_M - 1) / TC_M, tiles_y = (H + TC_TR - 1) / TC_TR;
  const int ntiles = tiles_x * tiles_y;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto tile_xy = [&](int k, int& x0, int& y0) {
    const int t = blockIdx.x + k * gridDim.x;
    const int ty = t / tiles_x;
    x0 = (t - ty * tiles_x) * TC_M;
    y0 = ty * TC_TR;
  };

  if (warp == TC_EPI_WARPS + 1) {
    // ---------------- TMA producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&xmap)) : "memory");
      int k = 0;
      for (; k < my_tiles; k++) {
        const int s = k & 1;
        if (!mbar_wait(empty(s), ((k >> 1) & 1) ^ 1, abort_flag)) break;
        int x0, y0;
        tile_xy(k, x0, y0);
        mbar_expect_tx(full(s), TX_BYTES);
        const unsigned dst = smem_u32(As) + (unsigned)(s * A_BYTES);
#pragma unroll
        for (int cb = 0; cb < CB; cb++) tma_load_3d(dst + cb * TC_SLAB, &xmap, cb * 8, x0 - 1, y0 - 1, full(s));
      }
      // loads issued but never consumed (abort only): wait for them to land
      for (int q = k - 2 < 0 ? 0 : k - 2; q < k; q++) mbar_drain(full(q & 1), (q >> 1) & 1);
    }
  } else if (warp == TC_EPI_WARPS) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const unsigned long long adesc0 = umma_desc(smem_u32(As), TC_SLAB, 128);
      const unsigned long long bdesc0 = umma_desc(smem_u32(Bs), NS * 16, 128);
      int k = 0;
      for (; k < my_tiles; k++) {
        const int s = k & 1;
        if (!mbar_wait(full(s), (k >> 1) & 1, abort_flag)) break;
        if (!mbar_wait(tempty(s), ((k >> 1) & 1) ^ 1, abort_flag)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned long long adesc = adesc0 + (unsigned long long)(s * (A_BYTES >> 4));
        const unsigned dbase = tmem + (unsigned)(s * 256);
        // descriptor offsets are in 16-byte units on the 14-bit start-address
        // field; all of shared memory fits in it, so the sums never carry out
#pragma unroll
        for (int j = 0; j < TC_PR; j++) {
          const int ky_lo = j - (TC_TR - 1) > 0 ? j - (TC_TR - 1) : 0;
          const int ky_hi = j < 2 ? j : 2;
          const int nky = ky_hi - ky_lo + 1;
          const unsigned dcol = dbase + (unsigned)((TC_TR - 1 - j + ky_lo) * NK);  // accumulator of row j - ky_lo
#pragma unroll
          for (int kx = 0; kx < 3; kx++) {
#pragma unroll
            for (int kc = 0; kc < CIN / 16; kc++) {
              const unsigned aoff = (unsigned)((2 * kc) * (TC_SLAB / 16) + j * TC_PW + kx);
              const unsigned boff = (unsigned)((kx * CB + 2 * kc) * NS + ky_lo * NK);
              if (kx == 0 && kc == 0 && ky_lo == 0) {
                // first contribution to output row j: start its accumulator
                mma_bf16<0>(dcol, adesc + aoff, bdesc0 + boff, umma_idesc(TC_M, NK));
                if (nky == 2) mma_bf16<1>(dcol + NK, adesc + aoff, bdesc0 + boff + NK, umma_idesc(TC_M, NK));
                if (nky == 3) mma_bf16<1>(dcol + NK, adesc + aoff, bdesc0 + boff + NK, umma_idesc(TC_M, 2 * NK));
              } else if (nky == 1) {
                mma_bf16<1>(dcol, adesc + aoff, bdesc0 + boff, umma_idesc(TC_M, NK));
              } else if (nky == 2) {
                mma_bf16<1>(dcol, adesc + aoff, bdesc0 + boff, umma_idesc(TC_M, 2 * NK));
              } else {
                mma_bf16<1>(dcol, adesc + aoff, bdesc0 + boff, umma_idesc(TC_M, 3 * NK));
              }
            }
          }
        }
        mma_commit(empty(s));  // smem stage s free once these MMAs have read it
        mma_commit(tfull(s));  // accumulator set s complete
      }
      if (k > 0) mbar_drain(tfull((k - 1) & 1), ((k - 1) >> 1) & 1);  // MMAs in flight (abort only)
    }
  } else {
    // ---------------- epilogue: warp w owns TMEM lanes 32w..32w+31 (pixels)
    for (int k = 0; k < my_tiles; k++) {
      const int s = k & 1;
      bool ok = true;
      if (lane == 0) ok = mbar_wait(tfull(s), (k >> 1) & 1, abort_flag);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int x0, y0;
      tile_xy(k, x0, y0);
      const unsigned tbase = tmem + (unsigned)(s * 256) + ((unsigned)(warp * 32) << 16);
      const int px = x0 + warp * 32 + lane;
#pragma unroll 1
      for (int r = 0; r < TC_TR; r++) {
        unsigned u[NK];
        const unsigned col = tbase + (unsigned)((TC_TR - 1 - r) * NK);
#pragma unroll
        for (int c = 0; c < NK / 16; c++) tmem_ld16_async(col + c * 16, u + c * 16);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (r == TC_TR - 1) {  // every read of set s done: hand it back to the MMA warp
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(tempty(s));
        }
        const int gy = y0 + r;
        if (gy >= H || px >= W) continue;
        const size_t pix = (size_t)gy * W + px;
        if (EPI == TC_RELU) {
#pragma unroll
          for (int c = 0; c < COUT_G; c += 8) {
            __align__(16) __nv_bfloat162 o[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
              o[q] = __floats2bfloat162_rn(fmaxf(__uint_as_float(u[c + 2 * q]) + bias_s[c + 2 * q], 0.f),
                                           fmaxf(__uint_as_float(u[c + 2 * q + 1]) + bias_s[c + 2 * q + 1], 0.f));
            *reinterpret_cast<uint4*>(y + pix * COUT_G + c) = *reinterpret_cast<uint4*>(o);
          }
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++) yf[pix * 3 + c] = resid[pix * 3 + c] + (__uint_as_float(u[c]) + bias_s[c]);
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(err, DSGPU_ERR_TIMEOUT);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

template <int CIN, int COUT_G, int NK, int EPI>
cudaError_t launch_tc(cudaStream_t st, const bf16* x, int H, int W, const bf16* wt, const float* bias, bf16* y,
                      const float* resid, float* yf, int* err) {
  constexpr size_t need = (size_t)2 * (CIN / 8) * TC_SLAB + (size_t)3 * (CIN / 8) * 3 * NK * 16 + NK * 4 + 8 * 8 + 16;
  constexpr size_t smem = need > TC_MIN_SMEM ? need : TC_MIN_SMEM;
  static_assert(need <= 227 * 1024, "shared memory");
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(x) & 15) != 0) return cudaErrorInvalidValue;
  CUtensorMap map;
  const cuuint64_t dims[3] = {(cuuint64_t)CIN, (cuuint64_t)W, (cuuint64_t)H};
  const cuuint64_t strides[2] = {(cuuint64_t)CIN * 2, (cuuint64_t)W * CIN * 2};
  const cuuint32_t box[3] = {8, (cuuint32_t)TC_PW, (cuuint32_t)TC_PR};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(x), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT_G, NK, EPI>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = ((W + TC_M - 1) / TC_M) * ((H + TC_TR - 1) / TC_TR);
  const int grid = tiles < sms ? tiles : sms;
  conv_tc_kernel<CIN, COUT_G, NK, EPI><<<grid, TC_THREADS, smem, st>>>(map, H, W, wt, bias, y, resid, yf, err);
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
