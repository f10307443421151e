// The learned path's convolutions on the 5th-generation tensor cores
// (tcgen05): inference, and training's forward pass, data gradients
// (conv_tc_kernel) and weight and bias gradients (wgrad_tc_kernel, at the end
// of the file). Same network and weights as k_cnn.cu ([9][cout][cin] bf16);
// the difference is the engine and the activation layout.
//
// Layout. Activations live in HBM channel-block-major, [C/8][H][Wp][8] bf16
// (16 bytes per pixel and block; Wp = W rounded up to 4, padding columns
// zero), so one row of a block is contiguous. The operands sit in shared
// memory in the canonical no-swizzle K-major layout (core matrices of 8 rows
// x 16 bytes). The input tile (TR+2 rows x 136 pixels, x0-4 .. x0+131) is
// stored the same way, [block][row][pixel][8 channels], so the A operand
// (M = 128 pixels, K = 16 channels) of any tap is the layout shifted by whole
// pixels: one descriptor per (input row, kx), no im2col copy. The TMA tensor
// map sees a block as 64-byte groups of 4 pixels (a 16-byte innermost box
// row would move a 32-byte sector per 16 bytes); one box per block loads the
// tile, zero-filled outside the image. The epilogue's stores of a block are
// 512 contiguous bytes per warp.
//
// Pipeline. The staged input goes through a ring of shared-memory slots, one
// per (tile, 16-channel K step): 6 for tiles of up to 5 output rows (TMA runs
// up to two tiles of a 48-channel input ahead of the MMAs), 3 for taller ones.
// A slot is released by the tcgen05.commit of its K step's MMAs, or, where the
// ring holds exactly one tile per accumulator set, by the tile's completion
// commit (fewer commits: each one slows the MMA stream).
//
// Stacked taps. Input row j feeds output rows j, j-1, j-2 through weight
// rows ky = 0, 1, 2. The three ky weight blocks are stacked along N, and the
// output-row accumulators are laid out in TMEM in descending row order, so
// one MMA per (input row, kx, 16 channels) with N = 3 x 48 covers all three
// output rows (N = 48 or 96 at the tile's top and bottom edges). Measured on
// B200, a 128 x N x 16 BF16 MMA from shared memory costs the same for every N
// up to 144 (76 cycles back to back; ~97 cycles inside this pipeline, where
// commits are interleaved), so the time goes with the number of MMAs and
// stacking the taps divides it by ~1.7. Every MMA accumulates: the epilogue
// zeroes the accumulator rows it has read (tcgen05.st) before handing a set
// back, and zeroes both sets at start. (Starting each row with a split-off
// accumulate = 0 MMA instead cost 15-20 % of a 48-channel layer.)
//
// Roles (one persistent CTA of 320 threads per SM, weights staged once):
//   warp 9  TMA producer: the K steps of tile k into ring slots;
//   warp 8  MMA issuer: tcgen05.mma.cta_group::1.kind::f16 (BF16 in, FP32
//           accumulate) into TMEM accumulator set k % 2, then tcgen05.commit
//           to release the smem stage and to hand the set to the epilogue;
//   warps 0-7  epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (pixels)
//           of its half of the tile's rows with tcgen05.ld, adds bias, applies
//           ReLU (packing to BF16 in registers) or keeps the residual, zeroes
//           those rows, hands the accumulator set back, and only then stores
//           straight to global memory, so the next tile's MMAs never wait for
//           stores.
// Every mbarrier wait is bounded in time (2 s); a wait that gives up sets a
// CTA-wide abort flag, which every other wait honours, reports
// DSGPU_ERR_TIMEOUT through `err`, and the CTA waits (bounded) for its copies
// and MMAs in flight before freeing its TMEM. No TMA multicast and no cluster
// features are used.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <vector>

#include "internal.cuh"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int TC_EPI_WARPS = 8;                    // two per TMEM lane quarter
constexpr int TC_THREADS = 32 * (TC_EPI_WARPS + 2);  // + MMA warp + TMA warp
constexpr int TC_M = 128;                          // pixels per MMA (one output-row segment)
// Output rows per tile, per layer (measured at 24 MP; every choice gives the
// same output bit for bit): the staged rows carry 2 halo rows per tile, whose
// MMAs cost as much as full ones, so taller tiles issue fewer MMAs per output
// row, as long as two accumulator sets (TR x NK columns each) still fit in
// TMEM and the staging ring in shared memory. 48 -> 48 layers: 5 rows
// (1.155 -> 1.11 ms against 4; 10 rows, one accumulator set, 1.20-1.25 ms);
// the 16 -> 48 input layer: 4 (5: 1.6% slower); the 48 -> 3 output layer
// (16 columns a row): 10 (1.05 -> 0.80 ms against 4).
constexpr int TC_TR_HIDDEN = 5, TC_TR_INPUT = 4, TC_TR_OUTPUT = 10;
constexpr int TC_PG = 4;                           // pixels per TMA element group (64-byte box rows)
constexpr int TC_PW = TC_M + 2 * TC_PG;            // staged pixels per row: x0-4 .. x0+131
constexpr int TC_TMEM_COLS = 512;                  // accumulator sets at columns 0 and 256
constexpr size_t TC_MIN_SMEM = 120 * 1024;         // keeps one CTA per SM (the TMEM plan assumes it)
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

// epilogues: bias + ReLU to BF16 (forward); fp32 residual output (the last
// layer); ReLU mask of the layer below to BF16, no bias (data gradient)
enum { TC_RELU = 0, TC_RESID = 1, TC_MASK = 2 };

// Shape of a tile of TR output rows: PR staged rows; SLAB bytes per 8-channel
// block of the staged tile; a ring slot (SUB) holds the 16 channels of one K
// step; RING slots; NSETS TMEM accumulator sets of TR * NK columns (two when
// they fit in half of TMEM, so the epilogue of one tile overlaps the MMAs of
// the next; else one).
template <int TR, int NK>
struct TcShape {
  static constexpr int PR = TR + 2;
  static constexpr int SLAB = TC_PW * PR * 16;
  static constexpr int SUB = 2 * SLAB;
  static constexpr int RING = TR <= 5 ? 6 : 3;
  static constexpr int NSETS = TR * NK <= 256 ? 2 : 1;
  static_assert(SLAB % 128 == 0, "TMA destinations must stay 128-byte aligned");
  static_assert(TR * NK <= TC_TMEM_COLS, "accumulators fit TMEM");
};

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

// 16 columns of zeros into this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_zero16(unsigned addr) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(addr),
      "r"(0u)
      : "memory");
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

// TMA load of one 5-D box (channel within a 4-pixel group, group, row residue
// y mod D, row quotient y div D, block) into shared memory, completing on bar
__device__ __forceinline__ void tma_load_5d(unsigned dst, const CUtensorMap* map, int x, int yr, int yq, int cb,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(x), "r"(yr), "r"(yq), "r"(cb), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// x: [CIN/8][Hp][Wp][8] bf16 (Wp = W rounded up to 4, Hp = H rounded up to
// 12; padding columns and rows zero) through `xmap` (4-pixel groups, rows
// split into residue and quotient by DIL; box 32 x TC_PW/4 x 1 x TC_PR x 1);
// wt: [9][COUT_G][CIN] bf16; NK: output channels per ky block (COUT_G padded
// to a multiple of 16); y: [COUT_G/8][Hp][Wp][8] bf16 (ReLU; padding columns
// written as zero, padding rows left alone) or yf: [H][W][3] fp32 = resid +
// conv (residual). EPI TC_MASK: y = conv x [mask > 0], mask a BF16 tensor
// laid out like y (the ReLU mask of the layer below, for the data gradient).
// Batches (training): period > 0 means the frame is crops of `valid` rows
// stacked `period` rows apart; the rows between them (at least the largest
// dilation) are written as zero, so the next layer reads zero padding there,
// and the residual output yf / resid are the crops without those rows.
// DIL: dilation of the taps. A tile is TR output rows
// DIL apart (y0, y0 + DIL, ...) by 128 pixels; on that subsampled row grid a
// dilated conv is an undilated one, so the staging and the stacked-tap MMAs
// are the same for every DIL.
template <int CIN, int COUT_G, int NK, int EPI, int DIL, int TR>
__global__ void __launch_bounds__(TC_THREADS, 1)
    conv_tc_kernel(const __grid_constant__ CUtensorMap xmap, int H, int W, const bf16* __restrict__ wt,
                   const float* __restrict__ bias, bf16* __restrict__ y, const float* __restrict__ resid,
                   float* __restrict__ yf, const bf16* __restrict__ mask, int period, int valid,
                   int* __restrict__ err) {
  static_assert(CIN % 16 == 0 && NK % 16 == 0 && NK >= COUT_G && 3 * NK <= 256, "shapes");
  typedef TcShape<TR, NK> S;
  constexpr int TC_PR = S::PR, TC_SLAB = S::SLAB, TC_SUB = S::SUB, TC_RING = S::RING, NSETS = S::NSETS;
  constexpr int CB = CIN / 8;              // 8-channel blocks of the input
  constexpr int KS = CIN / 16;             // K steps (ring slots) per tile
  constexpr int A_BYTES = TC_RING * TC_SUB;
  constexpr int NS = 3 * NK;               // stacked B rows (ky, co)
  constexpr int B_BYTES = 3 * CB * NS * 16;  // weights, [kx][cb][ky*NK + co][8]
  constexpr unsigned TX_BYTES = 2 * 8 * TC_PW * TC_PR * 2;  // one slot
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* As = sm;                  // ring of TC_RING slots
  unsigned char* Bs = sm + A_BYTES;
  float* bias_s = reinterpret_cast<float*>(sm + A_BYTES + B_BYTES);  // NK floats
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(sm + A_BYTES + B_BYTES + NK * 4);
  // bars: full[TC_RING], empty[TC_RING], tfull[2], tempty[2], drain
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 2 * TC_RING + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot) + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned bar0 = smem_u32(bars);
  auto full = [&](int q) { return bar0 + 8u * q; };
  auto empty = [&](int q) { return bar0 + 8u * (TC_RING + q); };
  auto tfull = [&](int s) { return bar0 + 8u * (2 * TC_RING + s); };
  auto tempty = [&](int s) { return bar0 + 8u * (2 * TC_RING + 2 + s); };
  const unsigned drain = bar0 + 8u * (2 * TC_RING + 4);
  // Slot release. When the ring holds exactly NSETS tiles, tile k's slots are next filled for tile
  // k + NSETS, which uses the same accumulator set: the producer then waits for that set's
  // completion commit of tile k, and the MMA warp commits once per tile instead of once per K step
  // (every tcgen05.commit slows the MMA stream down). The set's next phase needs tile k + NSETS's
  // own loads, so this parity wait cannot be overtaken.
  constexpr bool TILE_RELEASE = TC_RING % KS == 0 && TC_RING / KS == NSETS;
  const int Wp = (W + TC_PG - 1) / TC_PG * TC_PG;

  for (int i = tid; i < 3 * CB * NS; i += TC_THREADS) {
    const int kx = i / (CB * NS), r = i - kx * CB * NS, cb = r / NS, n = r - cb * NS;
    const int ky = n / NK, co = n - ky * NK;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (co < COUT_G)
      v = *reinterpret_cast<const uint4*>(wt + ((size_t)(ky * 3 + kx) * COUT_G + co) * CIN + cb * 8);
    *reinterpret_cast<uint4*>(Bs + (size_t)i * 16) = v;
  }
  for (int i = tid; i < NK; i += TC_THREADS) bias_s[i] = (bias && i < COUT_G) ? bias[i] : 0.f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < TC_RING; q++) {
      mbar_init(full(q), 1);
      mbar_init(empty(q), 1);
    }
    for (int s = 0; s < 2; s++) {
      mbar_init(tfull(s), 1);
      mbar_init(tempty(s), TC_EPI_WARPS);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // weights -> async proxy
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  // row bands of DIL * TR rows, each split into DIL tiles by row residue
  const int tiles_x = (W + TC_M - 1) / TC_M, tiles_y = (H + DIL * TR - 1) / (DIL * TR) * DIL;
  const int ntiles = tiles_x * tiles_y;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  // tile k of this CTA: first pixel x0, first output row y0 (then y0 + DIL, ...)
  auto tile_xy = [&](int k, int& x0, int& y0) {
    const int t = blockIdx.x + k * gridDim.x;
    const int ty = t / tiles_x;
    x0 = (t - ty * tiles_x) * TC_M;
    const int band = ty / DIL;
    y0 = band * DIL * TR + (ty - band * DIL);
  };

  if (warp == TC_EPI_WARPS + 1) {
    // ---------------- TMA producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&xmap)) : "memory");
      int g = 0;  // ring slot uses so far
      for (int k = 0; k < my_tiles; k++) {
        int x0, y0;
        tile_xy(k, x0, y0);
        bool ok = true;
        for (int kc = 0; kc < KS; kc++, g++) {
          const int q = g % TC_RING;
          if (TILE_RELEASE) {
            if (kc == 0 && k >= NSETS && !(ok = mbar_wait(tfull(k % NSETS), ((k - NSETS) / NSETS) & 1, abort_flag)))
              break;
          } else if (!(ok = mbar_wait(empty(q), ((g / TC_RING) & 1) ^ 1, abort_flag))) {
            break;
          }
          mbar_expect_tx(full(q), TX_BYTES);
          const unsigned dst = smem_u32(As) + (unsigned)(q * TC_SUB);
          // staged rows y0 - DIL, y0, ..., y0 + TR * DIL: residue y0 % DIL, quotients from y0 / DIL - 1
          const int yr = y0 % DIL, yq = y0 / DIL - 1;
          tma_load_5d(dst, &xmap, x0 / TC_PG - 1, yr, yq, 2 * kc, full(q));
          tma_load_5d(dst + TC_SLAB, &xmap, x0 / TC_PG - 1, yr, yq, 2 * kc + 1, full(q));
        }
        if (!ok) break;
      }
      // loads issued but maybe never consumed (abort only): wait for them to land
      for (int h = g - TC_RING < 0 ? 0 : g - TC_RING; h < g; h++) mbar_drain(full(h % TC_RING), (h / TC_RING) & 1);
    }
  } else if (warp == TC_EPI_WARPS) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const unsigned long long adesc0 = umma_desc(smem_u32(As), TC_SLAB, 128);
      const unsigned long long bdesc0 = umma_desc(smem_u32(Bs), NS * 16, 128);
      int g = 0, k = 0;
      bool ok = true;
      for (; k < my_tiles && ok; k++) {
        const int s = k % NSETS, use = k / NSETS;  // accumulator set and how often it was used before
        // phase `use` of tempty(s): the set zeroed (at start, then after each epilogue read-out)
        if (!(ok = mbar_wait(tempty(s), use & 1, abort_flag))) break;
        const unsigned dbase = tmem + (unsigned)(s * 256);
#pragma unroll 1
        for (int kc = 0; kc < KS; kc++, g++) {
          const int q = g % TC_RING;
          if (!(ok = mbar_wait(full(q), (g / TC_RING) & 1, abort_flag))) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          // descriptor offsets are in 16-byte units on the 14-bit start-address
          // field; all of shared memory fits in it, so the sums never carry out
          const unsigned long long adesc = adesc0 + (unsigned long long)(q * (TC_SUB >> 4));
          const unsigned long long bdesc = bdesc0 + (unsigned long long)(2 * kc * NS);
#pragma unroll
          for (int j = 0; j < TC_PR; j++) {
            const int ky_lo = j - (TR - 1) > 0 ? j - (TR - 1) : 0;
            const int ky_hi = j < 2 ? j : 2;
            const int nky = ky_hi - ky_lo + 1;
            const unsigned dcol = dbase + (unsigned)((TR - 1 - j + ky_lo) * NK);  // accumulator of row j - ky_lo
#pragma unroll
            for (int kx = 0; kx < 3; kx++) {
              // staged pixel 0 is x0 - 4: output pixel x0 + m reads x0 + m + (kx - 1) DIL
              const unsigned aoff = (unsigned)(j * TC_PW + TC_PG - DIL + kx * DIL);
              const unsigned long long b = bdesc + (unsigned)(kx * CB * NS + ky_lo * NK);
              const unsigned long long a = adesc + aoff;
              // the epilogue hands every accumulator set back zeroed, so each MMA accumulates
              mma_bf16<1>(dcol, a, b, umma_idesc(TC_M, nky * NK));
            }
          }
          if (!TILE_RELEASE) mma_commit(empty(q));  // ring slot q free once these MMAs have read it
        }
        if (ok) mma_commit(tfull(s));  // accumulator set s complete
      }
      if (g > 0) {  // MMAs still in flight (after an abort): one commit covers them all
        mma_commit(drain);
        const unsigned long long t0 = globaltimer_ns();
        while (!mbar_test(drain, 0) && globaltimer_ns() - t0 < TC_WAIT_NS) {
        }
      }
    }
  } else {
    // ---------------- epilogue: warp w owns TMEM lanes 32 (w % 4)..+31 (pixels) and RPW output rows.
    // It reads all its rows out of TMEM first (bias and ReLU applied, packed to BF16 in registers),
    // hands the accumulator set back, then stores: the MMAs of the next tile need not wait for
    // the stores, which matters when a single set holds the tile.
    constexpr int RPW = (TR + 1) / 2;  // output rows per epilogue warp (the second four may hold one fewer)
    constexpr int PK = EPI != TC_RESID ? COUT_G / 2 : 3;  // per row: BF16 pairs, or the 3 residual floats
    static_assert(TC_EPI_WARPS == 8, "two epilogue warps per TMEM lane quarter");
    const int quarter = warp & 3, r0 = (warp >> 2) * RPW, rn = TR - r0 < RPW ? TR - r0 : RPW;
    const int Hp = (H + 11) / 12 * 12;
    const size_t plane = (size_t)Hp * Wp;
    // zero this warp's rows of accumulator set s (its lane quarter), then hand the set to the MMA warp
    auto zero_and_release = [&](int s) {
      const unsigned zbase = tmem + (unsigned)(s * 256) + ((unsigned)(quarter * 32) << 16);
#pragma unroll
      for (int i = 0; i < RPW; i++) {
        if (i >= rn) break;
#pragma unroll
        for (int c = 0; c < NK; c += 16) tmem_zero16(zbase + (unsigned)((TR - 1 - (r0 + i)) * NK + c));
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty(s));
    };
    for (int s = 0; s < NSETS; s++) zero_and_release(s);
    for (int k = 0; k < my_tiles; k++) {
      const int s = k % NSETS, use = k / NSETS;
      bool ok = true;
      if (lane == 0) ok = mbar_wait(tfull(s), use & 1, abort_flag);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int x0, y0;
      tile_xy(k, x0, y0);
      const unsigned tbase = tmem + (unsigned)(s * 256) + ((unsigned)(quarter * 32) << 16);
      const int px = x0 + quarter * 32 + lane;
      const bool in = px < W;  // padding columns are written as zero
      unsigned pk[RPW][PK];
#pragma unroll
      for (int i = 0; i < RPW; i++) {
        if (i >= rn) break;
        const unsigned col = tbase + (unsigned)((TR - 1 - (r0 + i)) * NK);
        if (EPI != TC_RESID) {
          const int gy = y0 + (r0 + i) * DIL;
          // written as zero: padding columns, rows past the frame, rows between batch crops
          const bool live = in && gy < H && (period == 0 || gy % period < valid);
#pragma unroll
          for (int c16 = 0; c16 < COUT_G; c16 += 16) {  // 16 columns at a time keeps the registers low
            unsigned u[16];
            tmem_ld16_async(col + c16, u);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            uint4 mk[2] = {make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u)};
            if (EPI == TC_MASK && live) {
#pragma unroll
              for (int h = 0; h < 2; h++)
                if (c16 + 8 * h < COUT_G)
                  mk[h] = *reinterpret_cast<const uint4*>(
                      mask + ((size_t)((c16 + 8 * h) / 8) * plane + (size_t)gy * Wp + px) * 8);
            }
#pragma unroll
            for (int c = c16; c < c16 + 16 && c < COUT_G; c += 2) {
              float v0 = __uint_as_float(u[c - c16]), v1 = __uint_as_float(u[c - c16 + 1]);
              if (EPI == TC_RELU) {
                v0 = fmaxf(v0 + bias_s[c], 0.f);
                v1 = fmaxf(v1 + bias_s[c + 1], 0.f);
              } else {
                const unsigned mw = reinterpret_cast<const unsigned*>(&mk[(c - c16) / 8])[((c - c16) % 8) / 2];
                const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(&mw);
                v0 = __bfloat162float(m.x) > 0.f ? v0 : 0.f;
                v1 = __bfloat162float(m.y) > 0.f ? v1 : 0.f;
              }
              __nv_bfloat162 o = __floats2bfloat162_rn(live ? v0 : 0.f, live ? v1 : 0.f);
              pk[i][c / 2] = *reinterpret_cast<unsigned*>(&o);
            }
          }
        } else {
          unsigned u[16];
          tmem_ld16_async(col, u);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int c = 0; c < PK; c++) pk[i][c] = __float_as_uint(__uint_as_float(u[c]) + bias_s[c]);
        }
      }
      // this warp's reads of set s done: zero its rows and hand the set back to the MMA warp
      zero_and_release(s);
#pragma unroll
      for (int i = 0; i < RPW; i++) {
        if (i >= rn) break;
        const int gy = y0 + (r0 + i) * DIL;
        if (gy >= H || px >= Wp) continue;
        if (EPI != TC_RESID) {
          const size_t pix = (size_t)gy * Wp + px;
#pragma unroll
          for (int c = 0; c < COUT_G; c += 8)
            *reinterpret_cast<uint4*>(y + ((size_t)(c / 8) * plane + pix) * 8) =
                make_uint4(pk[i][c / 2], pk[i][c / 2 + 1], pk[i][c / 2 + 2], pk[i][c / 2 + 3]);
        } else if (in && (period == 0 || gy % period < valid)) {
          // a batch's residual output holds the crops without the rows between them
          const size_t pix = ((size_t)(period ? gy / period * valid + gy % period : gy)) * W + px;
#pragma unroll
          for (int c = 0; c < 3; c++) yf[pix * 3 + c] = resid[pix * 3 + c] + __uint_as_float(pk[i][c]);
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

// ------------------------------------------------------------ weight gradients
// Weight and bias gradients of one layer of a training batch (the frame of
// crops of the forward and data-gradient kernels). For tap (ky, kx) at
// dilation D, substituting q = p + (ky - 1) D rows,
//   dW[ky][kx][co][ci] = sum_p dY[p][co] X[p + ((ky - 1) D, (kx - 1) D)][ci]
//                      = sum_q dY[q - (ky - 1) D rows][co] X[q + (kx - 1) D px][ci],
// so the row shift rides on dY and the column shift on X. A chunk of TK
// pixels of frame row q is staged as three row-shifted copies of dY (rows
// q + D, q, q - D: the A operand, M = (ky, co)) and three column-shifted
// copies of X (the B operand, N = (kx, ci)), each [8-channel block][pixel][8]
// as the TMA box lands, which is the canonical no-swizzle MN-major layout
// (core matrices of 8 pixels x 8 channels, 128 contiguous bytes; the next 8
// pixels 128 bytes on, the next channel block one block on). One MMA per
// (16-pixel K step, 128 rows of A) covers all nine taps at once. A 48 -> 48
// layer has 144 rows of A: a second M = 128 MMA starts 16 rows before their
// end, and of its rows only the last 16 are read out. Sixteen more columns of
// B, a block of ones and a block of zeros, give the bias gradient
// sum_q dY[q][co] in the ky = 1 rows. Rows outside the frame and pixels past
// a row's ends read as zero (TMA fill), and the frame's rows between crops and
// its padding columns are zero, so every chunk is summed whole, unmasked.
// A CTA accumulates its contiguous range of chunks in TMEM (FP32) and writes
// one partial sum per weight; the host adds the CTAs' partials in a fixed
// order, so the result is deterministic.
template <int CIN, int COUTW>
struct WgShape {
  static constexpr int TK = 64;                   // pixels per chunk
  static constexpr int STAGES = 4;
  static constexpr int GB = TK * 16;              // bytes of one 8-channel block of a chunk
  static constexpr int CBI = CIN / 8, CBO = COUTW / 8;
  static constexpr int NGA = 3 * CBO;             // A blocks (ky, co block)
  static constexpr int NM = (NGA + 15) / 16;      // M = 128 MMAs per K step
  static constexpr int AG = NGA < 16 ? 16 : NGA;  // A blocks an MMA may address
  static constexpr int NGB = 3 * CBI + 2;         // B blocks (kx, ci block), then ones and zeros
  static constexpr int N = NGB * 8;
  static constexpr int STAGE = (AG + NGB) * GB;
  static constexpr int TMEM_COLS = NM * N <= 256 ? 256 : 512;
  static constexpr unsigned TX = (unsigned)(3 * CBO + 3 * CBI) * GB;  // bytes the loads of a chunk bring
  static_assert(N % 16 == 0 && N <= 256 && NM * N <= 512, "MMA and TMEM shapes");
  static_assert(GB % 128 == 0, "TMA destinations stay 128-byte aligned");
  // first A block of MMA m: 16 m, the last one ending at the last real block
  static __host__ __device__ constexpr int a_first(int m) { return NGA <= 16 ? 0 : (16 * m < NGA - 16 ? 16 * m : NGA - 16); }
};
constexpr int WG_THREADS = 192;  // warps 0-3 read TMEM out, warp 4 issues the MMAs, warp 5 loads

// TMA load of one 4-D box (channel, pixel, row, 8-channel block) at pixel x,
// row y, channel 0, block 0
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(x), "r"(y), "r"(0), "r"(bar)
      : "memory");
}

// tcgen05.mma with the accumulate flag taken at run time
__device__ __forceinline__ void mma_bf16_pred(unsigned tmem_d, unsigned long long a, unsigned long long b,
                                              unsigned idesc, int acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// x: [CIN/8][Hp][Wp][8], dy: [COUTW/8][Hp][Wp][8]. The loads that start at a
// chunk's first pixel (every dY copy, the unshifted X copy) go through xmap4 /
// dmap4, which see a block row as 64-byte groups of 4 pixels (boxes of 4
// pixels x 8 channels x TK / 4 groups x 1 row x every block); the two
// column-shifted X copies, which start at any pixel, through xmap (16-byte box
// rows of one pixel; such a row moves a 32-byte sector, so these are the only
// loads that fetch twice their bytes). Both forms land in shared memory as
// [block][pixel][8]. H: frame rows; wpart: [grid][9][COUTW][CIN], bpart:
// [grid][COUTW] (one partial sum per CTA).
template <int CIN, int COUTW>
__global__ void __launch_bounds__(WG_THREADS, 1)
    wgrad_tc_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap xmap4,
                    const __grid_constant__ CUtensorMap dmap4, int H, int Wp, int dil, float* __restrict__ wpart,
                    float* __restrict__ bpart, int* __restrict__ err) {
  typedef WgShape<CIN, COUTW> S;
  extern __shared__ __align__(128) unsigned char sm[];
  // bars: full[STAGES], empty[STAGES], done, drain
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(sm + (size_t)S::STAGES * S::STAGE);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 2 * S::STAGES + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot) + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned bar0 = smem_u32(bars);
  auto full = [&](int s) { return bar0 + 8u * s; };
  auto empty = [&](int s) { return bar0 + 8u * (S::STAGES + s); };
  const unsigned done = bar0 + 8u * (2 * S::STAGES), drain = done + 8u;
  auto a_of = [&](int s) { return sm + (size_t)s * S::STAGE; };
  auto b_of = [&](int s) { return sm + (size_t)s * S::STAGE + (size_t)S::AG * S::GB; };

  // the blocks no load writes: A blocks past the real ones (zero), B's ones and zeros
  for (int s = 0; s < S::STAGES; s++) {
    uint4* az = reinterpret_cast<uint4*>(a_of(s) + (size_t)S::NGA * S::GB);
    for (int i = tid; i < (S::AG - S::NGA) * S::GB / 16; i += WG_THREADS) az[i] = make_uint4(0u, 0u, 0u, 0u);
    uint4* bo = reinterpret_cast<uint4*>(b_of(s) + (size_t)3 * S::CBI * S::GB);
    const unsigned one2 = 0x3F803F80u;  // two BF16 ones
    for (int i = tid; i < 2 * S::GB / 16; i += WG_THREADS)
      bo[i] = i < S::GB / 16 ? make_uint4(one2, one2, one2, one2) : make_uint4(0u, 0u, 0u, 0u);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(S::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < S::STAGES; s++) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    mbar_init(done, 1);
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // ones and zeros -> async proxy
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  // this CTA's chunks: a contiguous range of (row, TK-pixel run) in row-major order
  const int cpr = (Wp + S::TK - 1) / S::TK;
  const long long total = (long long)H * cpr;
  const int c0 = (int)(total * blockIdx.x / gridDim.x);
  const int nch = (int)(total * (blockIdx.x + 1) / gridDim.x) - c0;

  if (warp == 5) {
    // ---------------- TMA producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&xmap)) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&xmap4)) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&dmap4)) : "memory");
      int c = 0;
      for (; c < nch; c++) {
        const int s = c % S::STAGES;
        if (!mbar_wait(empty(s), ((c / S::STAGES) & 1) ^ 1, abort_flag)) break;
        mbar_expect_tx(full(s), S::TX);
        const int g = c0 + c, q = g / cpr, x0 = (g - q * cpr) * S::TK;
        const unsigned a = smem_u32(a_of(s)), b = smem_u32(b_of(s));
        // x0 is a multiple of TK, so the unshifted loads start on a 4-pixel group
#pragma unroll
        for (int k = 0; k < 3; k++) {
          tma_load_4d(a + (unsigned)(k * S::CBO * S::GB), &dmap4, x0 / TC_PG, q - (k - 1) * dil, full(s));  // ky = k
          if (k == 1)
            tma_load_4d(b + (unsigned)(S::CBI * S::GB), &xmap4, x0 / TC_PG, q, full(s));  // kx = 1
          else
            tma_load_4d(b + (unsigned)(k * S::CBI * S::GB), &xmap, x0 + (k - 1) * dil, q, full(s));  // kx = 0, 2
        }
      }
      // loads issued but maybe never consumed (abort only): wait for them to land
      for (int h = c - S::STAGES < 0 ? 0 : c - S::STAGES; h < c; h++)
        mbar_drain(full(h % S::STAGES), (h / S::STAGES) & 1);
    }
  } else if (warp == 4) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const unsigned idesc = umma_idesc(TC_M, S::N) | (1u << 15) | (1u << 16);  // A and B MN-major
      int c = 0;
      bool ok = true;
      for (; c < nch; c++) {
        const int s = c % S::STAGES;
        if (!(ok = mbar_wait(full(s), (c / S::STAGES) & 1, abort_flag))) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned a = smem_u32(a_of(s)), b = smem_u32(b_of(s));
#pragma unroll
        for (int k = 0; k < S::TK / 16; k++) {  // 16 pixels = 256 bytes of every block
          const unsigned long long bd = umma_desc(b + (unsigned)(k * 256), 128, S::GB);
#pragma unroll
          for (int m = 0; m < S::NM; m++) {
            const unsigned long long ad = umma_desc(a + (unsigned)(S::a_first(m) * S::GB + k * 256), 128, S::GB);
            mma_bf16_pred(tmem + (unsigned)(m * S::N), ad, bd, idesc, c > 0 || k > 0);
          }
        }
        mma_commit(empty(s));  // stage s free once these MMAs have read it
      }
      if (ok && nch > 0) mma_commit(done);
      if (c > 0) {  // MMAs still in flight (after an abort): one commit covers them all
        mma_commit(drain);
        const unsigned long long t0 = globaltimer_ns();
        while (!mbar_test(drain, 0) && globaltimer_ns() - t0 < TC_WAIT_NS) {
        }
      }
    }
  } else {
    // ---------------- read-out: warp w owns TMEM lanes 32 w .. 32 w + 31 (rows of A)
    bool ok = true;
    if (lane == 0 && nch > 0) ok = mbar_wait(done, 0, abort_flag);
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int L = warp * 32 + lane;
      float* wp = wpart + (size_t)blockIdx.x * 9 * COUTW * CIN;
#pragma unroll
      for (int m = 0; m < S::NM; m++) {
        const int R = 8 * S::a_first(m) + L;  // row of A: (ky, co)
        const bool live = R >= 128 * m && R < 8 * S::NGA;
        const int ky = R / COUTW, co = R - ky * COUTW;
#pragma unroll 1
        for (int c16 = 0; c16 < S::N; c16 += 16) {
          unsigned u[16];
          tmem_ld16_async(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(m * S::N + c16), u);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (!live) continue;
          float f[16];
#pragma unroll
          for (int j = 0; j < 16; j++) f[j] = nch > 0 ? __uint_as_float(u[j]) : 0.f;
          if (c16 < 3 * CIN) {
            const int kx = c16 / CIN, ci0 = c16 - kx * CIN;
            float4* dst = reinterpret_cast<float4*>(wp + ((size_t)(ky * 3 + kx) * COUTW + co) * CIN + ci0);
#pragma unroll
            for (int j = 0; j < 4; j++) dst[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
          } else if (c16 == 3 * CIN && ky == 1) {
            bpart[(size_t)blockIdx.x * COUTW + co] = f[0];
          }
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(err, DSGPU_ERR_TIMEOUT);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS));
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

template <int CIN, int COUT_G, int NK, int EPI, int DIL, int TR>
cudaError_t launch_tc_d(cudaStream_t st, const bf16* x, int H, int W, const bf16* wt, const float* bias, bf16* y,
                        const float* resid, float* yf, const bf16* mask, int period, int valid, int* err) {
  static_assert(DIL >= 1 && DIL <= TC_PG && 12 % DIL == 0, "the staged row holds a halo of up to 4 pixels");
  typedef TcShape<TR, NK> S;
  constexpr size_t need = (size_t)S::RING * S::SUB + (size_t)3 * (CIN / 8) * 3 * NK * 16 + NK * 4 +
                         (2 * S::RING + 5) * 8 + 16;
  constexpr size_t smem = need > TC_MIN_SMEM ? need : TC_MIN_SMEM;
  static_assert(need <= 227 * 1024, "shared memory");
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(x) & 15) != 0) return cudaErrorInvalidValue;
  CUtensorMap map;
  const int Wp = (W + TC_PG - 1) / TC_PG * TC_PG, Hp = (H + 11) / 12 * 12;
  // row y = q * DIL + r; Hp is a multiple of DIL, so every (r, q) is a row of the plane
  const cuuint64_t dims[5] = {8 * TC_PG, (cuuint64_t)(Wp / TC_PG), (cuuint64_t)DIL, (cuuint64_t)(Hp / DIL),
                              (cuuint64_t)(CIN / 8)};
  const cuuint64_t strides[4] = {16 * TC_PG, (cuuint64_t)Wp * 16, (cuuint64_t)Wp * 16 * DIL,
                                 (cuuint64_t)Wp * Hp * 16};
  const cuuint32_t box[5] = {8 * TC_PG, (cuuint32_t)(TC_PW / TC_PG), 1, (cuuint32_t)S::PR, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(x), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT_G, NK, EPI, DIL, TR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = ((W + TC_M - 1) / TC_M) * ((H + DIL * TR - 1) / (DIL * TR) * DIL);
  const int grid = tiles < sms ? tiles : sms;
  conv_tc_kernel<CIN, COUT_G, NK, EPI, DIL, TR><<<grid, TC_THREADS, smem, st>>>(map, H, W, wt, bias, y, resid, yf,
                                                                                mask, period, valid, err);
  return cudaGetLastError();
}

template <int CIN, int COUT_G, int NK, int EPI,
          int TR = (NK <= 16 ? TC_TR_OUTPUT : (CIN >= 48 ? TC_TR_HIDDEN : TC_TR_INPUT))>
cudaError_t launch_tc(cudaStream_t st, int dil, const bf16* x, int H, int W, const bf16* wt, const float* bias,
                      bf16* y, const float* resid, float* yf, int* err, const bf16* mask = nullptr, int period = 0,
                      int valid = 0) {
  switch (dil) {
    case 1: return launch_tc_d<CIN, COUT_G, NK, EPI, 1, TR>(st, x, H, W, wt, bias, y, resid, yf, mask, period, valid, err);
    case 2: return launch_tc_d<CIN, COUT_G, NK, EPI, 2, TR>(st, x, H, W, wt, bias, y, resid, yf, mask, period, valid, err);
    case 3: return launch_tc_d<CIN, COUT_G, NK, EPI, 3, TR>(st, x, H, W, wt, bias, y, resid, yf, mask, period, valid, err);
    case 4: return launch_tc_d<CIN, COUT_G, NK, EPI, 4, TR>(st, x, H, W, wt, bias, y, resid, yf, mask, period, valid, err);
    default: return cudaErrorInvalidValue;
  }
}

template <int CIN, int COUTW>
cudaError_t launch_wgrad_tc(cudaStream_t st, int dil, const bf16* x, const bf16* dy, int H, int W, float* wpart,
                            float* bpart, int max_grid, int* grid_out, int* err) {
  typedef WgShape<CIN, COUTW> S;
  constexpr size_t smem = (size_t)S::STAGES * S::STAGE + (2 * S::STAGES + 2) * 8 + 16;
  static_assert(smem <= 227 * 1024, "shared memory");
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dy)) & 15) != 0 || H < 1 || W < 1 || dil < 1 ||
      max_grid < 1)
    return cudaErrorInvalidValue;
  const int Wp = (W + TC_PG - 1) / TC_PG * TC_PG, Hp = (H + 11) / 12 * 12;
  static_assert(S::TK % TC_PG == 0, "chunks start on a 4-pixel group");
  // px: pixels per innermost element group (1: any start pixel; TC_PG: 64-byte rows)
  auto make = [&](CUtensorMap* m, const bf16* p, int blocks, int px) {
    const cuuint64_t dims[4] = {(cuuint64_t)(8 * px), (cuuint64_t)(Wp / px), (cuuint64_t)Hp, (cuuint64_t)blocks};
    const cuuint64_t strides[3] = {(cuuint64_t)(16 * px), (cuuint64_t)Wp * 16, (cuuint64_t)Wp * Hp * 16};
    const cuuint32_t box[4] = {(cuuint32_t)(8 * px), (cuuint32_t)(S::TK / px), 1, (cuuint32_t)blocks};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(p), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  CUtensorMap xmap, xmap4, dmap4;
  if (!make(&xmap, x, S::CBI, 1) || !make(&xmap4, x, S::CBI, TC_PG) || !make(&dmap4, dy, S::CBO, TC_PG))
    return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(wgrad_tc_kernel<CIN, COUTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long chunks = (long long)H * ((Wp + S::TK - 1) / S::TK);
  int grid = sms < max_grid ? sms : max_grid;
  if (chunks < grid) grid = (int)chunks;
  wgrad_tc_kernel<CIN, COUTW><<<grid, WG_THREADS, smem, st>>>(xmap, xmap4, dmap4, H, Wp, dil, wpart, bpart, err);
  *grid_out = grid;
  return cudaGetLastError();
}

}  // namespace

// Weight and bias gradients of one layer of a training batch on the tensor
// cores, as per-CTA partial sums (see wgrad_tc_kernel). kind: 0 the input
// layer (16 input, 48 output channels), 1 a hidden layer (48, 48), 2 the
// output layer (48 input channels, a 16-channel gradient). x: the layer's
// input, dy: the gradient at its output (ReLU mask applied), both in the
// tensor-core layout of an H-row frame W pixels wide; wpart[grid][9][cout][cin]
// and bpart[grid][cout] receive the partials of the *grid CTAs used (at most
// max_grid).
cudaError_t ds_tc_wgrad(cudaStream_t st, int kind, int dil, const void* x, const void* dy, int H, int W,
                        float* wpart, float* bpart, int max_grid, int* grid, int* err) {
  const bf16* xi = static_cast<const bf16*>(x);
  const bf16* di = static_cast<const bf16*>(dy);
  switch (kind) {
    case 0: return launch_wgrad_tc<16, 48>(st, dil, xi, di, H, W, wpart, bpart, max_grid, grid, err);
    case 1: return launch_wgrad_tc<48, 48>(st, dil, xi, di, H, W, wpart, bpart, max_grid, grid, err);
    case 2: return launch_wgrad_tc<48, 16>(st, dil, xi, di, H, W, wpart, bpart, max_grid, grid, err);
    default: return cudaErrorInvalidValue;
  }
}

// One conv layer of a training batch on the tensor cores (the batch is a frame
// of crops `valid` rows tall stacked `period` rows apart; see conv_tc_kernel).
// kind: 0 forward 16 -> 48 (input layer), 1 forward 48 -> 48, 2 forward
// 48 -> 3 with the residual (yf = resid + conv, both compact crops), 3 data
// gradient 16 -> 48 (the output layer's), 4 data gradient 48 -> 48; the data
// gradients apply the ReLU mask `mask` and no bias.
cudaError_t ds_tc_layer(cudaStream_t st, int kind, int dil, const void* x, int H, int W, const void* wt,
                        const float* bias, void* y, const float* resid, float* yf, const void* mask, int period,
                        int valid, int* err) {
  const bf16* xi = static_cast<const bf16*>(x);
  const bf16* w = static_cast<const bf16*>(wt);
  bf16* yo = static_cast<bf16*>(y);
  const bf16* m = static_cast<const bf16*>(mask);
  switch (kind) {
    case 0: return launch_tc<16, 48, 48, TC_RELU>(st, dil, xi, H, W, w, bias, yo, nullptr, nullptr, err, nullptr, period, valid);
    case 1: return launch_tc<48, 48, 48, TC_RELU>(st, dil, xi, H, W, w, bias, yo, nullptr, nullptr, err, nullptr, period, valid);
    case 2: return launch_tc<48, 8, 16, TC_RESID>(st, dil, xi, H, W, w, bias, nullptr, resid, yf, err, nullptr, period, valid);
    case 3: return launch_tc<16, 48, 48, TC_MASK>(st, dil, xi, H, W, w, nullptr, yo, nullptr, nullptr, err, m, period, valid);
    case 4: return launch_tc<48, 48, 48, TC_MASK>(st, dil, xi, H, W, w, nullptr, yo, nullptr, nullptr, err, m, period, valid);
    default: return cudaErrorInvalidValue;
  }
}

// One image through the 8 layers on the tensor cores. x16: packed input
// (16 ch, [2][Hp][Wp][8]); a, b: ping-pong activations (48 ch,
// [6][Hp][Wp][8]; the padding rows H..Hp-1 must be zero); wf/bias: per-layer
// forward weights (layer 8's with 8 output channels); dil: per-layer
// dilations; rgb/out: fp32 RGB; hidden_begin/end (may be null): events
// recorded around layers 2-7.
cudaError_t ds_cnn_forward_tc(cudaStream_t st, const void* x16, void* a, void* b, int H, int W,
                              const void* const* wf, const float* const* bias, const int* dil, const float* rgb,
                              float* out, int* err, cudaEvent_t hidden_begin, cudaEvent_t hidden_end) {
  const bf16* in = static_cast<const bf16*>(x16);
  bf16* pa = static_cast<bf16*>(a);
  bf16* pb = static_cast<bf16*>(b);
  cudaError_t e = launch_tc<16, 48, 48, TC_RELU>(st, dil[0], in, H, W, static_cast<const bf16*>(wf[0]), bias[0], pa,
                                                 nullptr, nullptr, err);
  if (e == cudaSuccess && hidden_begin) e = cudaEventRecord(hidden_begin, st);
  for (int l = 1; l < 7 && e == cudaSuccess; l++) {
    e = launch_tc<48, 48, 48, TC_RELU>(st, dil[l], pa, H, W, static_cast<const bf16*>(wf[l]), bias[l], pb, nullptr,
                                       nullptr, err);
    bf16* t = pa;
    pa = pb;
    pb = t;
  }
  if (e == cudaSuccess && hidden_end) e = cudaEventRecord(hidden_end, st);
  if (e == cudaSuccess)
    e = launch_tc<48, 8, 16, TC_RESID>(st, dil[7], pa, H, W, static_cast<const bf16*>(wf[7]), bias[7], nullptr, rgb,
                                       out, err);
  return e;
}

