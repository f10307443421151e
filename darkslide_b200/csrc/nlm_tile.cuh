// The NLM tile body (enhance.rs:36-72) shared by the one-frame kernels
// (k_nlm.cu) and the fused batch kernel (k_demosaic.cu); the design notes are
// at the top of k_nlm.cu. Everything here has internal linkage.
#pragma once
#include <cuda_fp16.h>

#include <type_traits>

#include "internal.cuh"

namespace {
namespace nlmk {

// Tile widths: the one-frame kernels run 16-wide tiles on 128-thread CTAs,
// four per SM (four independent barrier domains, so one CTA's row phase,
// heavy on shared stores, overlaps the column phases of the others); the
// batch kernels, whose CTAs also run 256-thread RCD tiles, run 32-wide tiles
// on 256 threads, two per SM. Threads = 8 x width either way.
constexpr int NLM_TX = 16;
constexpr int NLM_THREADS = 8 * NLM_TX;
constexpr int NLM_BATCH_TX = 32;
constexpr int NLM_BATCH_THREADS = 8 * NLM_BATCH_TX;
constexpr int HRW = 64;     // H rows per offset (TY + 2P)
constexpr int SEG = 16;     // phase-A segment width
constexpr int NI = 4;       // dx per block (one shifted-row load serves all four)
constexpr int NJ = 2;       // dy per block (one shifted-column load serves both)
constexpr int NPLANE = NI * NJ;
constexpr int HBR = HRW + 4;  // H rows allocated: phase B of the last quarter reads up to row 66
// H row pitch (odd: conflict-free row stores and column loads) and plane
// stride (= 16 mod 32 words, so that two half-warps reading neighbouring
// planes hit disjoint banks) of a tile width
__host__ __device__ constexpr int nlm_hp(int tx) { return tx + 1; }
__host__ __device__ constexpr int nlm_hps(int tx) {
  return HBR * nlm_hp(tx) + ((16 - (HBR * nlm_hp(tx)) % 32) + 32) % 32;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// two floats as a half2 word (lo in the low half), rounded to nearest and
// saturated to the largest finite half (a box sum past it gives a weight of 0
// either way, and a finite value keeps the running sums free of inf - inf)
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  float2 r;
  asm("{\n .reg .b64 ra, rb, rr;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " sub.rn.f32x2 rr, ra, rb;\n mov.b64 {%0, %1}, rr;\n}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ unsigned pack_h2(float lo, float hi) {
  unsigned r;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ float2 unpack_h2(unsigned w) {
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}

__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Plane pitch: odd and fixed per P (sized for the largest search radius) so
// that every shared address offset is a compile-time constant.
__host__ __device__ constexpr int nlm_pitch(int P, int SM = DSGPU_NLM_MAX_SEARCH, int tx = NLM_TX) {
  return (tx + 2 * (SM + P + 1)) | 1;
}
// the pitch class of a search radius: 10 (the common radii) or the maximum
__host__ __device__ constexpr int nlm_smax(int S) { return S <= 10 ? 10 : DSGPU_NLM_MAX_SEARCH; }

struct NlmGeom {
  int R, PW, PH, PHA;  // halo, region width, region height, allocated rows
};

__host__ __device__ inline NlmGeom nlm_geom(int S, int P, int tx = NLM_TX) {
  NlmGeom g;
  const int TY = HRW - 2 * P;
  g.R = S + P + 1;
  g.PW = tx + 2 * g.R;
  g.PH = TY + 2 * g.R;
  g.PHA = g.PH + 4;  // phase B of the last quarter reads up to 3 rows past the region
  return g;
}

// plane bytes (f32, or f16 when staged in half precision), rounded to 16
// FP32 plane bytes, rounded to 16
size_t nlm_plane_bytes(int S, int P, int sm = DSGPU_NLM_MAX_SEARCH, int tx = NLM_TX) {
  const NlmGeom g = nlm_geom(S, P, tx);
  return ((size_t)nlm_pitch(P, sm, tx) * g.PHA * 4 + 15) / 16 * 16;
}

// plane + H planes: NPLANE of FP32, or (f16) NPLANE / 2 of half2 pairs
size_t nlm_smem_bytes(int S, int P, bool f16 = false, int sm = DSGPU_NLM_MAX_SEARCH, int tx = NLM_TX) {
  return nlm_plane_bytes(S, P, sm, tx) + (size_t)(f16 ? NPLANE / 2 : NPLANE) * nlm_hps(tx) * sizeof(float);
}

__device__ __forceinline__ float ldp(const float* p) { return *p; }
__device__ __forceinline__ void stp(float* p, float v) { *p = v; }

// One TX x (64 - 2P) tile (tile_x, tile_y) of channel ch of a W x H x C
// image, by 8 TX threads; smem holds nlm_smem_bytes(S, P, F16, SM, TX) bytes.
//
// Offsets are taken in blocks of up to NI dx x NJ dy. Phase A (thread =
// H row, 16-wide segment and one dy of the block) forms the horizontal box
// sums of every dx of the block from ONE load of the shifted row; phase B
// (thread = column, quarter of the tile's rows and one half of the block's
// dx) sums them vertically, weights and accumulates. A pixel's sums are
// split between the two dx halves and added once at the end.
//
// F16 (the precision variant): the horizontal box sums handed from phase A
// to phase B, most of the shared-memory traffic, are staged in half
// precision: planes i and i + 2 of a block share one half2 word, which a
// phase-B thread (it owns exactly those two planes) reads with one load and
// sums as one packed pair. Differences, weights and sums stay in FP32.
//
// XIN: every patch window of the tile's columns lies inside the image (no
// column clamping in phase A). The two cases are separate code so that the
// border case's per-element clamping does not cost the interior registers.
template <int P, bool F16, bool XIN, int SM, int TX>
__device__ __forceinline__ void nlm_tile_body(const float* __restrict__ in, int W, int H, int C, int S, float sigma,
                                              float* __restrict__ out, int tile_x, int tile_y, int ch, float* smem) {
  using T = float;  // the staged plane is FP32 in both variants
  constexpr int NT = 8 * TX;  // threads
  constexpr int HP = nlm_hp(TX), HPS = nlm_hps(TX);
  constexpr int TY = HRW - 2 * P;
  constexpr int DW = SEG + 2 * P;   // differences per phase-A segment
  constexpr int RB = (TY + 3) / 4;  // phase-B rows per thread (a quarter of the tile)
  constexpr int PP = nlm_pitch(P, SM, TX);
  const NlmGeom g = nlm_geom(S, P, TX);
  T* PL = reinterpret_cast<T*>(smem);  // scaled plane, pitch PP
  float* HB = reinterpret_cast<float*>(reinterpret_cast<char*>(smem) +
                                       ((size_t)PP * g.PHA * sizeof(T) + 15) / 16 * 16);  // NPLANE x HBR rows x HP

  const int X0 = tile_x * TX, Y0 = tile_y * TY;
  const int tid = threadIdx.x;
  const int ox0 = X0 - g.R, oy0 = Y0 - g.R;  // global site of plane (0,0)

  for (int i = tid; i < g.PW * g.PH; i += NT) {
    const int ly = i / g.PW, lx = i - ly * g.PW;
    const int gx = clampi(ox0 + lx, 0, W - 1), gy = clampi(oy0 + ly, 0, H - 1);
    stp(&PL[ly * PP + lx], in[((size_t)gy * W + gx) * C + ch] * sigma);
  }
  for (int i = tid; i < (g.PHA - g.PH) * PP; i += NT) stp(&PL[g.PH * PP + i], 0.f);

  // ---- phase-A role: H row `arow` (tile row arow - P), segment at ax0, dy index aj
  const int arow = tid & (HRW - 1);
  const int ax0 = ((tid >> 6) & (TX / SEG - 1)) * SEG;
  const int aj = tid / (HRW * (TX / SEG));
  const int aprow = clampi(Y0 + arow - P, 0, H - 1) - oy0;  // plane row of the clamped H row
  const int acol0 = ax0 - P + g.R;  // plane column of difference 0 (interior tiles)
  // ---- phase-B role: column bcol, rows [brow0, brow0 + RB) (clipped to TY), dx half bk
  const int bcol = tid & (TX - 1);
  // consecutive groups of TX threads take the two dx halves (at TX = 16 the
  // two half-warps of a warp, which read neighbouring planes)
  const int bk = (tid / TX) & 1;
  const int brow0 = (tid / (2 * TX)) * RB;

  __syncthreads();
  float pv[DW];  // centre samples of this thread's phase-A segment
#pragma unroll
  for (int k = 0; k < DW; k++) {
    const int col = XIN ? acol0 + k : clampi(X0 + ax0 - P + k, 0, W - 1) - ox0;
    pv[k] = ldp(&PL[aprow * PP + col]);
  }
  // weighted sums, and weight sums as two halves added at the end (FP32:
  // packed pairs over the two dy planes of a block; FP16: the first half only)
  float a[RB];
  float2 s2[RB];
#pragma unroll
  for (int r = 0; r < RB; r++) {
    a[r] = 0.f;
    s2[r] = make_float2(0.f, 0.f);
  }

  // One block of offsets {dx0 .. dx0+BI-1} x {dy0 .. dy0+BJ-1}; plane (i, j)
  // of the block is HB + (j * NI + i) * HPS.
  auto block = [&](int dx0, int dy0, auto ni_tag, auto nj_tag) {
    constexpr int BI = decltype(ni_tag)::value;
    constexpr int BJ = decltype(nj_tag)::value;
    // phase A: horizontal sums, stored NEGATED (-sum d^2) so that phase B's
    // vertical sum is the ex2 argument itself
    if constexpr (F16) {
      // planes i0 and i0 + 2 of the block side by side in one half2 slot
      // (pair plane j * 2 + i0), saturated to the largest finite half
      if (aj < BJ) {
        const T* qrow = PL + (aprow + dy0 + aj) * PP + dx0;
        float q[DW + BI - 1];  // the shifted row in registers (interior tiles only)
        (void)q;
        if constexpr (XIN) {
#pragma unroll
          for (int m = 0; m < DW + BI - 1; m++) q[m] = ldp(&qrow[acol0 + m]);
        }
        unsigned* Hrow = reinterpret_cast<unsigned*>(HB) + (size_t)aj * 2 * HPS + arow * HP + ax0;
#pragma unroll
        for (int i0 = 0; i0 < 2 && i0 < BI; i0++) {
          const bool two = i0 + 2 < BI;
          auto dif = [&](int k, int i) {
            if constexpr (XIN) {
              return pv[k] - q[k + i];
            } else {
              const int col = clampi(X0 + ax0 - P + k, 0, W - 1) - ox0;
              return pv[k] - ldp(&qrow[col + i]);
            }
          };
          float h0 = 0.f, h1 = 0.f;
#pragma unroll
          for (int k = 0; k <= 2 * P; k++) {
            const float d0 = dif(k, i0);
            h0 = fmaf(-d0, d0, h0);
            if (two) {
              const float d1 = dif(k, i0 + 2);
              h1 = fmaf(-d1, d1, h1);
            }
          }
          unsigned* Hi = Hrow + i0 * HPS;
          Hi[0] = pack_h2(h0, h1);
#pragma unroll
          for (int k = 1; k < SEG; k++) {
            const float de0 = dif(k + 2 * P, i0), dl0 = dif(k - 1, i0);
            h0 = fmaf(-de0, de0, h0);
            h0 = fmaf(dl0, dl0, h0);
            if (two) {
              const float de1 = dif(k + 2 * P, i0 + 2), dl1 = dif(k - 1, i0 + 2);
              h1 = fmaf(-de1, de1, h1);
              h1 = fmaf(dl1, dl1, h1);
            }
            Hi[k] = pack_h2(h0, h1);
          }
        }
      }
    } else {
    if (aj < BJ) {
      const T* qrow = PL + (aprow + dy0 + aj) * PP + dx0;
      float q[DW + BI - 1];  // the shifted row in registers (interior tiles only)
      (void)q;
      if constexpr (XIN) {
#pragma unroll
        for (int m = 0; m < DW + BI - 1; m++) q[m] = ldp(&qrow[acol0 + m]);
      }
      float* Hrow = HB + (size_t)aj * NI * HPS + arow * HP + ax0;
#pragma unroll
      for (int i = 0; i < BI; i++) {
        // difference k of plane i; computed where it enters the window and
        // again where it leaves (cheaper than keeping 22 of them live)
        auto dif = [&](int k) {
          if constexpr (XIN) {
            return pv[k] - q[k + i];
          } else {
            const int col = clampi(X0 + ax0 - P + k, 0, W - 1) - ox0;
            return pv[k] - ldp(&qrow[col + i]);
          }
        };
        float h = 0.f;
#pragma unroll
        for (int k = 0; k <= 2 * P; k++) {
          const float d = dif(k);
          h = fmaf(-d, d, h);
        }
        float* Hi = Hrow + i * HPS;
        Hi[0] = h;
#pragma unroll
        for (int k = 1; k < SEG; k++) {
          const float de = dif(k + 2 * P), dl = dif(k - 1);
          h = fmaf(-de, de, h);
          h = fmaf(dl, dl, h);
          Hi[k] = h;
        }
      }
    }
    }
    __syncthreads();
    // phase B: vertical sums, weights, accumulation for dx0 + i (i = bk, bk + 2)
    if constexpr (F16) {
      // both of the thread's planes from one half2 slot; their running sums
      // side by side in one packed pair
      if (bk < BI) {
        const bool two = bk + 2 < BI;
        const T* qc = PL + (brow0 + g.R + dy0) * PP + bcol + g.R + dx0 + bk;
        float q0[RB + BJ - 1], q1[RB + BJ - 1];
#pragma unroll
        for (int r = 0; r < RB + BJ - 1; r++) {
          q0[r] = ldp(&qc[r * PP]);
          q1[r] = two ? ldp(&qc[r * PP + 2]) : 0.f;
        }
#pragma unroll
        for (int j = 0; j < BJ; j++) {
          const unsigned* hc = reinterpret_cast<const unsigned*>(HB) + (j * 2 + bk) * HPS + brow0 * HP + bcol;
          unsigned hv[RB + 2 * P];
#pragma unroll
          for (int r = 0; r < RB + 2 * P; r++) hv[r] = hc[r * HP];
          float2 hf[RB + 2 * P];  // each pair unpacked once, used where it enters and where it leaves
#pragma unroll
          for (int r = 0; r < RB + 2 * P; r++) hf[r] = unpack_h2(hv[r]);
          float2 v = make_float2(0.f, 0.f);
#pragma unroll
          for (int r = 0; r <= 2 * P; r++) v = f2add(v, hf[r]);
#pragma unroll
          for (int r = 0; r < RB; r++) {
            if (r > 0) v = f2sub(f2add(v, hf[r + 2 * P]), hf[r - 1]);
            const float w0 = ex2(v.x);
            a[r] = fmaf(w0, q0[r + j], a[r]);
            s2[r].x += w0;  // one scalar sum here: a second half costs registers this variant lacks
            if (two) {
              const float w1 = ex2(v.y);
              a[r] = fmaf(w1, q1[r + j], a[r]);
              s2[r].x += w1;
            }
          }
        }
      }
    } else {
    // phase B: vertical sums, weights, accumulation for dx0 + i (i = bk, bk + 2)
#pragma unroll
    for (int ii = 0; ii < 2; ii++) {
      const int i = bk + 2 * ii;
      if (i < BI) {
        const T* qc = PL + (brow0 + g.R + dy0) * PP + bcol + g.R + dx0 + i;
        float qv[RB + BJ - 1];
#pragma unroll
        for (int r = 0; r < RB + BJ - 1; r++) qv[r] = ldp(&qc[r * PP]);
        if constexpr (BJ == 2) {
          // both dy of the block at once: their vertical sums and weight sums
          // run as packed pairs (the same sums, half the instructions)
          const float* hc0 = HB + i * HPS + brow0 * HP + bcol;
          const float* hc1 = hc0 + NI * HPS;
          float2 hv[RB + 2 * P];
#pragma unroll
          for (int r = 0; r < RB + 2 * P; r++) hv[r] = make_float2(hc0[r * HP], hc1[r * HP]);
          float2 v = make_float2(0.f, 0.f);
#pragma unroll
          for (int r = 0; r <= 2 * P; r++) v = f2add(v, hv[r]);
#pragma unroll
          for (int r = 0; r < RB; r++) {
            if (r > 0) v = f2sub(f2add(v, hv[r + 2 * P]), hv[r - 1]);
            const float w0 = ex2(v.x), w1 = ex2(v.y);
            a[r] = fmaf(w0, qv[r], a[r]);
            a[r] = fmaf(w1, qv[r + 1], a[r]);
            s2[r] = f2add(s2[r], make_float2(w0, w1));
          }
        } else {
          const float* hc = HB + i * HPS + brow0 * HP + bcol;
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
            a[r] = fmaf(wgt, qv[r], a[r]);
            s2[r].x += wgt;
          }
        }
      }
    }
    }
    __syncthreads();
  };

  // blocks of NI dx x NJ dy, then the dx tail (fewer than NI columns of
  // offsets) and the dy tail (one row of offsets when 2S+1 is odd)
  const int n_off = 2 * S + 1;
  const int dx_main = n_off / NI * NI;  // dx in [-S, -S + dx_main) go in full blocks
  const int dx_tail = n_off - dx_main;
  auto row_of_blocks = [&](int dy0, auto nj_tag) {
    for (int dx0 = -S; dx0 < -S + dx_main; dx0 += NI) block(dx0, dy0, std::integral_constant<int, NI>{}, nj_tag);
    const int dxt = -S + dx_main;
    switch (dx_tail) {
      case 1: block(dxt, dy0, std::integral_constant<int, 1>{}, nj_tag); break;
      case 2: block(dxt, dy0, std::integral_constant<int, 2>{}, nj_tag); break;
      case 3: block(dxt, dy0, std::integral_constant<int, 3>{}, nj_tag); break;
      default: break;
    }
  };
  int dy0 = -S;
  for (; dy0 + NJ - 1 <= S; dy0 += NJ) row_of_blocks(dy0, std::integral_constant<int, NJ>{});
  if (dy0 <= S) row_of_blocks(dy0, std::integral_constant<int, 1>{});  // the dy tail of an odd search width

  // the two dx halves of each pixel's sums: half 1 hands its sums over
  // through shared memory (the H planes are free now), half 0 adds and writes
  float* XA = HB;
  float* XS = HB + TX * 4 * RB;
  const int slot = (tid / (2 * TX)) * RB * TX + bcol;  // (quarter, row r) x column
  if (bk == 1) {
#pragma unroll
    for (int r = 0; r < RB; r++) {
      XA[slot + r * TX] = a[r];
      XS[slot + r * TX] = s2[r].x + s2[r].y;
    }
  }
  __syncthreads();
  if (bk == 0) {
    const float inv_sigma = 1.0f / sigma;
#pragma unroll
    for (int r = 0; r < RB; r++) {
      const int y = brow0 + r;
      const int gx = X0 + bcol, gy = Y0 + y;
      if (y < TY && gx < W && gy < H) {
        const float at = a[r] + XA[slot + r * TX];
        const float st = (s2[r].x + s2[r].y) + XS[slot + r * TX];
        const float o = __fdiv_rn(at * inv_sigma, fmaxf(st, 1e-12f));
        out[((size_t)gy * W + gx) * C + ch] = o;
      }
    }
  }
}

template <int P, bool F16 = false, int SM = DSGPU_NLM_MAX_SEARCH, int TX = NLM_TX>
__device__ __forceinline__ void nlm_tile(const float* __restrict__ in, int W, int H, int C, int S, float sigma,
                                         float* __restrict__ out, int tile_x, int tile_y, int ch, float* smem) {
  const int X0 = tile_x * TX;
  if (X0 - P >= 0 && X0 + TX + P <= W)
    nlm_tile_body<P, F16, true, SM, TX>(in, W, H, C, S, sigma, out, tile_x, tile_y, ch, smem);
  else
    nlm_tile_body<P, F16, false, SM, TX>(in, W, H, C, S, sigma, out, tile_x, tile_y, ch, smem);
}

}  // namespace nlmk
}  // namespace
