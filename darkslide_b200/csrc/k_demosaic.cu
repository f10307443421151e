// Demosaic kernels: CFA normalisation, clip plane, MHC, superpixel and the
// fused RCD tile kernel.
//
// This file is compiled with -fmad=false: the reference (Rust) rounds every
// product before adding it, so the GPU must not contract a*b+c into FMAs for
// these kernels to reproduce it bit for bit. Divisions are IEEE (__fdiv_rn).
#include <cfloat>

#include "internal.cuh"
#include "nlm_tile.cuh"

namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ------------------------------------------------------------ normalisation
// decode.rs:292-306: v = (raw - black) / max(white[c] - black, 1)
__device__ __forceinline__ float norm_u16(uint16_t raw, float black, float white_c) {
  return __fdiv_rn((float)raw - black, fmaxf(white_c - black, 1.0f));
}

__global__ void normalize_u16_kernel(const ds_src_u16 src, int w, int h, ds_pat pat, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w) return;
  const int c = pat.at(x, y);
  const float wc = c == 0 ? src.white[0] : (c == 1 ? src.white[1] : src.white[2]);
  out[(size_t)y * w + x] = norm_u16(src.data[(size_t)y * src.pitch + x], ds_black_at(src, x, y), wc);
}

// ---------------------------------------------------------------- clip plane
// demosaic.rs:31-42 (CLIP = 0.995, demosaic.rs:17)
__global__ void clip_plane_kernel(const float* __restrict__ cfa, int w, int h, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w) return;
  float m = 0.0f;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      const float v = cfa[(size_t)clampi(y + dy, 0, h - 1) * w + clampi(x + dx, 0, w - 1)];
      m = fmaxf(m, v >= 0.995f ? 1.0f : 0.0f);
    }
  out[(size_t)y * w + x] = m;
}

// ------------------------------------------------------------------- MHC
// demosaic.rs:90-124. `at(dx,dy)` returns data*mul at the clamped site,
// without max(0). The formulas keep the reference's evaluation order.
template <class At>
__device__ __forceinline__ void mhc_formulas(At p, int c, int row_c, float& o0, float& o1, float& o2) {
  const float v = p(0, 0);
  const float g_at_rb = __fdiv_rn(4.0f * v + 2.0f * (p(0, -1) + p(-1, 0) + p(1, 0) + p(0, 1)) -
                                      (p(0, -2) + p(-2, 0) + p(2, 0) + p(0, 2)),
                                  8.0f);
  const float rb_g_row = __fdiv_rn(5.0f * v + 4.0f * (p(-1, 0) + p(1, 0)) -
                                       (p(-2, 0) + p(2, 0) + p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) +
                                       0.5f * (p(0, -2) + p(0, 2)),
                                   8.0f);
  const float rb_g_col = __fdiv_rn(5.0f * v + 4.0f * (p(0, -1) + p(0, 1)) -
                                       (p(0, -2) + p(0, 2) + p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) +
                                       0.5f * (p(-2, 0) + p(2, 0)),
                                   8.0f);
  const float rb_diag = __fdiv_rn(6.0f * v + 2.0f * (p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) -
                                      1.5f * (p(0, -2) + p(-2, 0) + p(2, 0) + p(0, 2)),
                                  8.0f);
  if (c == 1) {
    if (row_c == 0) { o0 = rb_g_row; o1 = v; o2 = rb_g_col; }
    else            { o0 = rb_g_col; o1 = v; o2 = rb_g_row; }
  } else if (c == 0) { o0 = v; o1 = g_at_rb; o2 = rb_diag; }
  else               { o0 = rb_diag; o1 = g_at_rb; o2 = v; }
  o0 = fmaxf(o0, 0.0f);
  o1 = fmaxf(o1, 0.0f);
  o2 = fmaxf(o2, 0.0f);
}

__global__ void mhc_kernel(const float* __restrict__ cfa, int w, int h, ds_pat pat, float m0, float m1, float m2,
                           float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w) return;
  auto p = [&](int dx, int dy) {
    const int sx = clampi(x + dx, 0, w - 1), sy = clampi(y + dy, 0, h - 1);
    const int c = pat.at(sx, sy);
    return cfa[(size_t)sy * w + sx] * (c == 0 ? m0 : (c == 1 ? m1 : m2));
  };
  float o0, o1, o2;
  mhc_formulas(p, pat.at(x, y), pat.at(x + 1, y), o0, o1, o2);
  float* o = out + ((size_t)y * w + x) * 3;
  o[0] = o0;
  o[1] = o1;
  o[2] = o2;
}

// --------------------------------------------------------------- superpixel
// demosaic.rs:45-87 for a Bayer (2x2) pattern: output (w/2, h/2).
__global__ void superpixel_kernel(const float* __restrict__ cfa, int w, int h, ds_pat pat, float m0, float m1,
                                  float m2, float* __restrict__ out, float* __restrict__ clip) {
  const int ow = w / 2;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= ow) return;
  const float CLIP = 0.995f;
  float acc[3] = {0.f, 0.f, 0.f}, mx[3] = {0.f, 0.f, 0.f};
  unsigned n[3] = {0, 0, 0}, clipped = 0;
  for (int dy = 0; dy < 2; dy++)
    for (int dx = 0; dx < 2; dx++) {
      const int sx = x * 2 + dx, sy = y * 2 + dy;
      const int c = pat.at(sx, sy);
      const float v = cfa[(size_t)sy * w + sx];
      if (v >= CLIP) clipped++;
      mx[c] = fmaxf(mx[c], v);
      acc[c] += v;
      n[c]++;
    }
  const float mul[3] = {m0, m1, m2};
  float* o = out + ((size_t)y * ow + x) * 3;
  for (int c = 0; c < 3; c++) {
    const float v = mx[c] >= CLIP ? mx[c] : (n[c] > 0 ? __fdiv_rn(acc[c], (float)n[c]) : 0.0f);
    o[c] = v * mul[c];
  }
  if (clip) clip[(size_t)y * ow + x] = fminf(__fdiv_rn((float)clipped, 4.0f) * 2.0f, 1.0f);
}

// ------------------------------------------------------------------ RCD tile
// One CTA produces a RTX x RTY tile of RGB (and clip) output. Every RCD pass of
// demosaic.rs:147-344 runs on the tile plus the halo it needs, in shared
// memory, in the reference's order and with its global border rules (each
// stage value at a site follows the site's GLOBAL coordinates: bv/bh/bp/bq on
// [3, W-3), vh/pq on [4, W-4) else 0.5, lpf on [2, W-2) at R/B sites, RCD
// writes on [4, W-4), MHC elsewhere).
//
// Receptive radius: 4.4 reads 4.3 output at +-3; 4.3 reads g at +-2 and pq at
// +-1; g reads c at +-4, lpf at +-2, vh at +-1; vh reads bv/bh at +-1, which
// read c at +-3. So the tile loads a 10-sample halo (local stage regions
// along x: m [0,52), b* and lpf [3,49), vh/pq [4,48), g [5,47), r43/b43
// [7,45), output [10,42)).
// Tile of the one-frame kernel: 64 x 40. The passes keep five planes live at
// once (stages 1 and 2 run in two halves, and two passes write in place from
// registers), so a 64 x 40 tile (84 x 60 sites with its halo, 2.0 computed
// sites per output pixel against 3.0 for 32 x 24) takes 103 KB and two CTAs
// share an SM. Every tiling gives the same output bit for bit.
constexpr int RTX = 64, RTY = DS_RCD_TILE;
constexpr int RH = 10;  // halo
constexpr int RCD_THREADS = 256;  // the batch kernels' block (shared with the NLM tile body)
// The one-frame kernel's block: 512 threads, two CTAs per SM.
constexpr int RCD_THREADS_1F = 512;
// shared bytes of a TX x TY tile: npl stage planes of (TX+20) x (TY+20) floats + the clip bytes
__host__ __device__ constexpr size_t rcd_smem(int tx, int ty, int npl = 5) {
  return (size_t)npl * (tx + 2 * RH) * (ty + 2 * RH) * sizeof(float) + (size_t)(tx + 2 * RH) * (ty + 2 * RH);
}
constexpr size_t RCD_SMEM = rcd_smem(RTX, RTY);

struct SrcF32 {
  ds_src_f32 s;
  __device__ __forceinline__ float load(int gx, int gy, int) const { return s.data[(size_t)gy * s.pitch + gx]; }
};
struct SrcU16 {
  ds_src_u16 s;
  __device__ __forceinline__ float load(int gx, int gy, int c) const {
    const float wc = c == 0 ? s.white[0] : (c == 1 ? s.white[1] : s.white[2]);
    return norm_u16(s.data[(size_t)gy * s.pitch + gx], ds_black_at(s, gx, gy), wc);
  }
};

__device__ __forceinline__ float sq(float v) { return v * v; }

// One TXT x TYT output tile (tile_x, tile_y) of a W x H frame; smem holds
// rcd_smem(TXT, TYT) bytes. The value at every site depends only on the
// frame and the site's global coordinates, so any tiling gives the same
// output bit for bit.
// RING: some site of the tile's stage regions lies in the frame's 4-site
// border ring, where RCD falls back to MHC, which reads data*mul WITHOUT
// max(0) (demosaic.rs:93-98). Other tiles never need the unclamped value, so
// their staged plane holds c = max(data*mul, 0) (demosaic.rs:154) directly
// and the passes skip a max per read.
// FULL (implies !RING): the whole staged region lies inside the frame, so no
// load is clamped and every stage's border rule holds at every site the tile
// computes; the tile skips those tests.
template <class Src, int TXT, int TYT, int NT, int NPL, bool RING, bool FULL = false>
__device__ __forceinline__ void rcd_tile_body(const Src& src, int W, int H, ds_pat pat, float m0, float m1, float m2,
                                         float* __restrict__ out_rgb, float* __restrict__ out_clip, int tile_x,
                                         int tile_y, float* smem) {
  static_assert(TXT % 2 == 0 && TYT % 2 == 0, "tile sides must be even");
  constexpr int RSX = TXT + 2 * RH, RSY = TYT + 2 * RH, RA = RSX * RSY;
  // NPL = 5 stage planes, reused as the passes retire them:
  //   M   data*mul (clamped-site load; max(0) outside RING tiles) ... later b after 4.3
  //   LP  lpf ................................................... later r after 4.3
  //   VH  vh
  //   X   bv, then bp, then pq
  //   Y   bh, then bq, then g
  // pq and b replace planes that their own pass still reads, so each thread
  // holds its sites' values in registers until every thread is done reading.
  // NPL = 7 (the batch kernels' 256-thread tiles, whose shared memory is
  // sized by the NLM tile anyway) gives pq and b planes of their own and
  // writes them directly.
  static_assert(NPL == 5 || NPL == 7, "five or seven planes");
  float* M = smem;
  float* LP = M + RA;
  float* VH = LP + RA;
  float* X = VH + RA;
  float* Y = X + RA;
  uint8_t* CL = reinterpret_cast<uint8_t*>(smem + NPL * RA);  // [v >= CLIP]
  float* BV = X;
  float* BH = Y;
  float* BP = X;
  float* BQ = Y;
  float* PQ = NPL == 5 ? X : Y + RA;
  float* G = Y;
  float* R43 = LP;
  float* B43 = NPL == 5 ? M : Y + 2 * RA;

  const int tid = threadIdx.x;
  const int gx0 = tile_x * TXT - RH, gy0 = tile_y * TYT - RH;  // global site of local (0,0)
  const float eps = 1e-5f;

  // stage 0: load with clamped coordinates
  for (int i = tid; i < RA; i += NT) {
    const int ly = i / RSX, lx = i - ly * RSX;
    const int gx = FULL ? gx0 + lx : clampi(gx0 + lx, 0, W - 1), gy = FULL ? gy0 + ly : clampi(gy0 + ly, 0, H - 1);
    const int col = pat.at(gx, gy);
    const float v = src.load(gx, gy, col);
    const float vm = v * (col == 0 ? m0 : (col == 1 ? m1 : m2));
    M[i] = RING ? vm : fmaxf(vm, 0.0f);
    CL[i] = v >= 0.995f ? 1 : 0;
  }
  __syncthreads();

  auto C = [&](int k) { return RING ? fmaxf(M[k], 0.0f) : M[k]; };  // demosaic.rs:154
  const int w1 = RSX, w2 = 2 * RSX, w3 = 3 * RSX, w4 = 4 * RSX;

  // The passes' regions (local sites): stage 1 [3, edge - 3), stage 2 [4, edge - 4).
  constexpr int S1X = RSX - 6, S1N = S1X * (RSY - 6);
  constexpr int S2X = RSX - 8, S2N = S2X * (RSY - 8);
  auto grad7 = [&](int k, int s1, int s2, int s3, float c6) {  // (:160-172, :251-260) along the step s1
    return sq((C(k - s3) - C(k - s1) - C(k + s1) + C(k + s3)) - 3.0f * (C(k - s2) + C(k + s2)) + c6);
  };
  // stage 1a: bv, bh (:160-172) and lpf (:188-201)
  for (int i = tid; i < S1N; i += NT) {
    const int ly = 3 + i / S1X, lx = 3 + i % S1X;
    const int gx = gx0 + lx, gy = gy0 + ly;
    const int k = ly * RSX + lx;
    float bv = 0.f, bh = 0.f, lp = 0.f;
    if (FULL || (gx >= 3 && gx < W - 3 && gy >= 3 && gy < H - 3)) {
      const float c6 = 6.0f * C(k);
      bv = grad7(k, w1, w2, w3, c6);
      bh = grad7(k, 1, 2, 3, c6);
    }
    if ((FULL || (gx >= 2 && gx < W - 2 && gy >= 2 && gy < H - 2)) && pat.at(gx, gy) != 1) {
      lp = C(k) + 0.5f * (C(k - w1) + C(k + w1) + C(k - 1) + C(k + 1)) +
           0.25f * (C(k - w1 - 1) + C(k - w1 + 1) + C(k + w1 - 1) + C(k + w1 + 1));
    }
    BV[k] = bv;
    BH[k] = bh;
    LP[k] = lp;
  }
  __syncthreads();

  // stage 2a: vh (:173-184) on [4, edge-4)
  for (int i = tid; i < S2N; i += NT) {
    const int ly = 4 + i / S2X, lx = 4 + i % S2X;
    const int gx = gx0 + lx, gy = gy0 + ly;
    const int k = ly * RSX + lx;
    float vh = 0.5f;
    if (FULL || (gx >= 4 && gx < W - 4 && gy >= 4 && gy < H - 4)) {
      const float vs = fmaxf(BV[k - w1] + BV[k] + BV[k + w1], eps);
      const float hs = fmaxf(BH[k - 1] + BH[k] + BH[k + 1], eps);
      vh = __fdiv_rn(vs, vs + hs);
    }
    VH[k] = vh;
  }
  __syncthreads();

  // stage 1b: bp, bq (:251-260) into the planes bv and bh held
  for (int i = tid; i < S1N; i += NT) {
    const int ly = 3 + i / S1X, lx = 3 + i % S1X;
    const int gx = gx0 + lx, gy = gy0 + ly;
    const int k = ly * RSX + lx;
    float bp = 0.f, bq = 0.f;
    if (FULL || (gx >= 3 && gx < W - 3 && gy >= 3 && gy < H - 3)) {
      const float c6 = 6.0f * C(k);
      bp = grad7(k, w1 + 1, w2 + 2, w3 + 3, c6);
      bq = grad7(k, w1 - 1, w2 - 2, w3 - 3, c6);
    }
    BP[k] = bp;
    BQ[k] = bq;
  }
  __syncthreads();

  // stage 2b: pq (:261-272) on [4, edge-4). With five planes it replaces bp
  // in place, so every thread first forms its sites' values in registers.
  auto pq_at = [&](int k) {
    const float ps = fmaxf(BP[k - w1 - 1] + BP[k] + BP[k + w1 + 1], eps);
    const float qs = fmaxf(BQ[k - w1 + 1] + BQ[k] + BQ[k + w1 - 1], eps);
    return __fdiv_rn(ps, ps + qs);
  };
  if constexpr (NPL == 7) {
    for (int i = tid; i < S2N; i += NT) {
      const int ly = 4 + i / S2X, lx = 4 + i % S2X;
      const int gx = gx0 + lx, gy = gy0 + ly;
      const int k = ly * RSX + lx;
      PQ[k] = FULL || (gx >= 4 && gx < W - 4 && gy >= 4 && gy < H - 4) ? pq_at(k) : 0.5f;
    }
  } else {
    constexpr int NPQ = (S2N + NT - 1) / NT;
    float pqv[NPQ];
#pragma unroll
    for (int n = 0; n < NPQ; n++) {
      const int i = tid + n * NT;
      pqv[n] = 0.5f;
      if (i < S2N) {
        const int ly = 4 + i / S2X, lx = 4 + i % S2X;
        const int gx = gx0 + lx, gy = gy0 + ly;
        const int k = ly * RSX + lx;
        if (FULL || (gx >= 4 && gx < W - 4 && gy >= 4 && gy < H - 4)) pqv[n] = pq_at(k);
      }
    }
    __syncthreads();
#pragma unroll
    for (int n = 0; n < NPQ; n++) {
      const int i = tid + n * NT;
      if (i < S2N) PQ[(4 + i / S2X) * RSX + 4 + i % S2X] = pqv[n];
    }
  }
  __syncthreads();

  auto disc = [&](const float* d, int k) {  // :216-220
    const float central = d[k];
    const float neigh = 0.25f * (d[k - w1 - 1] + d[k - w1 + 1] + d[k + w1 - 1] + d[k + w1 + 1]);
    return fabsf(0.5f - central) < fabsf(0.5f - neigh) ? neigh : central;
  };
  auto mhc_at = [&](int k, int gx, int gy, float& o0, float& o1, float& o2) {  // ring sites only
    auto p = [&](int dx, int dy) { return M[k + dy * RSX + dx]; };
    mhc_formulas(p, pat.at(gx, gy), pat.at(gx + 1, gy), o0, o1, o2);
  };

  // Sites of one colour class come every other column, so the heavy stages
  // below enumerate only the sites that need work (no divergence between
  // neighbouring lanes): col_start() is the first local column >= lx0 in row
  // ly whose global colour is (or, with want_g=false, is not) green.
  auto col_start = [&](int ly, int lx0, bool want_g) {
    const int gy = gy0 + ly, gx = gx0 + lx0;
    const bool g_here = pat.at(gx, gy) == 1;
    return lx0 + ((g_here == want_g) ? 0 : 1);
  };
  auto inner = [&](int gx, int gy) { return FULL || (gx >= 4 && gx < W - 4 && gy >= 4 && gy < H - 4); };

  // stage 3: green (:203-214 init, :222-245 step 3) on [5, edge-5): (RSY-10)
  // rows x (RSX-10)/2 sites of each class
  constexpr int S3Y = RSY - 10, S3H = (RSX - 10) / 2;
  for (int i = tid; i < S3Y * S3H; i += NT) {  // green sites: native sample
    const int ly = 5 + i / S3H, lx = col_start(ly, 5, true) + 2 * (i % S3H);
    if (lx >= RSX - 5) continue;
    G[ly * RSX + lx] = C(ly * RSX + lx);
  }
  for (int i = tid; i < S3Y * S3H; i += NT) {  // R/B sites
    const int ly = 5 + i / S3H, lx = col_start(ly, 5, false) + 2 * (i % S3H);
    if (lx >= RSX - 5) continue;
    const int gx = gx0 + lx, gy = gy0 + ly;
    const int k = ly * RSX + lx;
    float g;
    if (inner(gx, gy)) {
      const float vd = disc(VH, k);
      const float n_grad = eps + fabsf(C(k - w1) - C(k + w1)) + fabsf(C(k) - C(k - w2)) + fabsf(C(k - w1) - C(k - w3)) +
                           fabsf(C(k - w2) - C(k - w4));
      const float s_grad = eps + fabsf(C(k - w1) - C(k + w1)) + fabsf(C(k) - C(k + w2)) + fabsf(C(k + w1) - C(k + w3)) +
                           fabsf(C(k + w2) - C(k + w4));
      const float w_grad = eps + fabsf(C(k - 1) - C(k + 1)) + fabsf(C(k) - C(k - 2)) + fabsf(C(k - 1) - C(k - 3)) +
                           fabsf(C(k - 2) - C(k - 4));
      const float e_grad = eps + fabsf(C(k - 1) - C(k + 1)) + fabsf(C(k) - C(k + 2)) + fabsf(C(k + 1) - C(k + 3)) +
                           fabsf(C(k + 2) - C(k + 4));
      const float l0 = LP[k];
      const float n_est = __fdiv_rn(C(k - w1) * 2.0f * l0, eps + l0 + LP[k - w2]);
      const float s_est = __fdiv_rn(C(k + w1) * 2.0f * l0, eps + l0 + LP[k + w2]);
      const float w_est = __fdiv_rn(C(k - 1) * 2.0f * l0, eps + l0 + LP[k - 2]);
      const float e_est = __fdiv_rn(C(k + 1) * 2.0f * l0, eps + l0 + LP[k + 2]);
      const float v_est = __fdiv_rn(s_grad * n_est + n_grad * s_est, n_grad + s_grad);
      const float h_est = __fdiv_rn(w_grad * e_est + e_grad * w_est, e_grad + w_grad);
      g = fmaxf(vd * h_est + (1.0f - vd) * v_est, 0.0f);
    } else {
      float o0, o1, o2;
      mhc_at(k, gx, gy, o0, o1, o2);
      g = o1;
    }
    G[k] = g;
  }
  __syncthreads();

  // stage 4: R at B and B at R (:276-308) on [7, edge-7). The pre-pass clone
  // read at the diagonal +-1/+-3 sites of an R (B) site holds native B (R)
  // samples, i.e. c. Interior green sites are never read (4.4 reads R/B
  // sites only); ring green sites keep their MHC values.
  // R43 goes to the lpf plane (retired after stage 3) directly; with five
  // planes B43 replaces the data plane, which this pass still reads, so each
  // thread keeps its sites' values in registers until every thread is done
  // reading.
  constexpr int S4Y = RSY - 14, S4H = (RSX - 14) / 2, S4N = S4Y * S4H;
  constexpr int NB4 = (S4N + NT - 1) / NT, NBR = NPL == 5 ? NB4 : 1;
  float b4[NBR], bg4[RING ? NBR : 1];
  int k4[NBR], kg4[RING ? NBR : 1];
#pragma unroll
  for (int n = 0; n < NB4; n++) {  // R/B sites
    const int i = tid + n * NT;
    if constexpr (NPL == 5) k4[n] = -1;
    if (i >= S4N) continue;
    const int ly = 7 + i / S4H, lx = col_start(ly, 7, false) + 2 * (i % S4H);
    if (lx >= RSX - 7) continue;
    const int gx = gx0 + lx, gy = gy0 + ly;
    const int k = ly * RSX + lx;
    const int col = pat.at(gx, gy);
    float r, b;
    if (inner(gx, gy)) {
      const float pd = disc(PQ, k);
      const float g0 = G[k];
      const float nw_g = eps + fabsf(C(k - w1 - 1) - C(k + w1 + 1)) + fabsf(C(k - w1 - 1) - C(k - w3 - 3)) + fabsf(g0 - G[k - w2 - 2]);
      const float ne_g = eps + fabsf(C(k - w1 + 1) - C(k + w1 - 1)) + fabsf(C(k - w1 + 1) - C(k - w3 + 3)) + fabsf(g0 - G[k - w2 + 2]);
      const float sw_g = eps + fabsf(C(k + w1 - 1) - C(k - w1 + 1)) + fabsf(C(k + w1 - 1) - C(k + w3 - 3)) + fabsf(g0 - G[k + w2 - 2]);
      const float se_g = eps + fabsf(C(k + w1 + 1) - C(k - w1 - 1)) + fabsf(C(k + w1 + 1) - C(k + w3 + 3)) + fabsf(g0 - G[k + w2 + 2]);
      const float nw_e = C(k - w1 - 1) - G[k - w1 - 1];
      const float ne_e = C(k - w1 + 1) - G[k - w1 + 1];
      const float sw_e = C(k + w1 - 1) - G[k + w1 - 1];
      const float se_e = C(k + w1 + 1) - G[k + w1 + 1];
      const float p_est = __fdiv_rn(nw_g * se_e + se_g * nw_e, nw_g + se_g);
      const float q_est = __fdiv_rn(ne_g * sw_e + sw_g * ne_e, ne_g + sw_g);
      const float v = fmaxf(g0 + (1.0f - pd) * p_est + pd * q_est, 0.0f);
      if (col == 2) { r = v; b = C(k); }
      else          { r = C(k); b = v; }
    } else {
      float o0, o1, o2;
      mhc_at(k, gx, gy, o0, o1, o2);
      r = col == 0 ? C(k) : o0;
      b = col == 2 ? C(k) : o2;
    }
    R43[k] = r;
    if constexpr (NPL == 5) {
      b4[n] = b;
      k4[n] = k;
    } else {
      B43[k] = b;
    }
  }
  if constexpr (RING) {
#pragma unroll
    for (int n = 0; n < NB4; n++) {  // green sites of the ring
      const int i = tid + n * NT;
      if constexpr (NPL == 5) kg4[n] = -1;
      if (i >= S4N) continue;
      const int ly = 7 + i / S4H, lx = col_start(ly, 7, true) + 2 * (i % S4H);
      if (lx >= RSX - 7) continue;
      const int gx = gx0 + lx, gy = gy0 + ly;
      if (inner(gx, gy)) continue;
      const int k = ly * RSX + lx;
      float o0, o1, o2;
      mhc_at(k, gx, gy, o0, o1, o2);
      R43[k] = o0;
      if constexpr (NPL == 5) {
        bg4[n] = o2;
        kg4[n] = k;
      } else {
        B43[k] = o2;
      }
    }
  }
  if constexpr (NPL == 5) {
    __syncthreads();
#pragma unroll
    for (int n = 0; n < NB4; n++) {
      if (k4[n] >= 0) B43[k4[n]] = b4[n];
      if (RING && kg4[n] >= 0) B43[kg4[n]] = bg4[n];
    }
  }
  __syncthreads();

  // stage 5: the tile's output; R and B at green sites (:310-341)
  constexpr int TH = TXT / 2;
  auto clip_at = [&](int k) {
    unsigned m = 0;
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) m |= CL[k + dy * RSX + dx];
    return m ? 1.0f : 0.0f;
  };
  for (int i = tid; i < TYT * TH; i += NT) {  // green sites
    const int ly = RH + i / TH, lx = col_start(ly, RH, true) + 2 * (i % TH);
    if (lx >= RH + TXT) continue;
    const int gx = gx0 + lx, gy = gy0 + ly;
    if (!FULL && (gx >= W || gy >= H)) continue;
    const int k = ly * RSX + lx;
    float r = R43[k], b = B43[k];
    const float g = G[k];
    if (inner(gx, gy)) {
      const float vd = disc(VH, k);
      auto pass44 = [&](const float* cc) {
        const float n_g = eps + fabsf(g - G[k - w2]) + fabsf(cc[k - w1] - cc[k + w1]) + fabsf(cc[k - w1] - cc[k - w3]);
        const float s_g = eps + fabsf(g - G[k + w2]) + fabsf(cc[k + w1] - cc[k - w1]) + fabsf(cc[k + w1] - cc[k + w3]);
        const float w_g = eps + fabsf(g - G[k - 2]) + fabsf(cc[k - 1] - cc[k + 1]) + fabsf(cc[k - 1] - cc[k - 3]);
        const float e_g = eps + fabsf(g - G[k + 2]) + fabsf(cc[k + 1] - cc[k - 1]) + fabsf(cc[k + 1] - cc[k + 3]);
        const float n_e = cc[k - w1] - G[k - w1];
        const float s_e = cc[k + w1] - G[k + w1];
        const float w_e = cc[k - 1] - G[k - 1];
        const float e_e = cc[k + 1] - G[k + 1];
        const float v_est = __fdiv_rn(n_g * s_e + s_g * n_e, n_g + s_g);
        const float h_est = __fdiv_rn(e_g * w_e + w_g * e_e, e_g + w_g);
        return fmaxf(g + (1.0f - vd) * v_est + vd * h_est, 0.0f);
      };
      r = pass44(R43);
      b = pass44(B43);
    }
    float* o = out_rgb + ((size_t)gy * W + gx) * 3;
    o[0] = r;
    o[1] = g;
    o[2] = b;
    if (out_clip) out_clip[(size_t)gy * W + gx] = clip_at(k);
  }
  for (int i = tid; i < TYT * TH; i += NT) {  // R/B sites: values settled by stage 4
    const int ly = RH + i / TH, lx = col_start(ly, RH, false) + 2 * (i % TH);
    if (lx >= RH + TXT) continue;
    const int gx = gx0 + lx, gy = gy0 + ly;
    if (!FULL && (gx >= W || gy >= H)) continue;
    const int k = ly * RSX + lx;
    float* o = out_rgb + ((size_t)gy * W + gx) * 3;
    o[0] = R43[k];
    o[1] = G[k];
    o[2] = B43[k];
    if (out_clip) out_clip[(size_t)gy * W + gx] = clip_at(k);
  }
}

// One TXT x TYT output tile; see rcd_tile_body. A tile needs the ring code
// when its stage-3 region (the widest one that can fall back to MHC: local
// sites [5, edge - 5)) reaches the border ring [0, 4) or [W - 4, W).
template <class Src, int TXT, int TYT, int NT = RCD_THREADS, int NPL = 7>
__device__ __forceinline__ void rcd_tile(const Src& src, int W, int H, ds_pat pat, float m0, float m1, float m2,
                                         float* __restrict__ out_rgb, float* __restrict__ out_clip, int tile_x,
                                         int tile_y, float* smem) {
  constexpr int RSX = TXT + 2 * RH, RSY = TYT + 2 * RH;
  const int gx0 = tile_x * TXT - RH, gy0 = tile_y * TYT - RH;
  const bool ring = gx0 + 5 < 4 || gx0 + RSX - 5 > W - 4 || gy0 + 5 < 4 || gy0 + RSY - 5 > H - 4;
  const bool full = gx0 >= 0 && gx0 + RSX <= W && gy0 >= 0 && gy0 + RSY <= H;
  if (full)
    rcd_tile_body<Src, TXT, TYT, NT, NPL, false, true>(src, W, H, pat, m0, m1, m2, out_rgb, out_clip, tile_x, tile_y, smem);
  else if (ring)
    rcd_tile_body<Src, TXT, TYT, NT, NPL, true>(src, W, H, pat, m0, m1, m2, out_rgb, out_clip, tile_x, tile_y, smem);
  else
    rcd_tile_body<Src, TXT, TYT, NT, NPL, false>(src, W, H, pat, m0, m1, m2, out_rgb, out_clip, tile_x, tile_y, smem);
}

template <class Src>
__global__ void __launch_bounds__(RCD_THREADS_1F, 2) rcd_tile_kernel(Src src, int W, int H, ds_pat pat, float m0,
                                                                      float m1, float m2, float* __restrict__ out_rgb,
                                                                      float* __restrict__ out_clip, int ty0) {
  extern __shared__ float4 smem4[];
  rcd_tile<Src, RTX, RTY, RCD_THREADS_1F, 5>(src, W, H, pat, m0, m1, m2, out_rgb, out_clip, blockIdx.x,
                                          blockIdx.y + ty0, reinterpret_cast<float*>(smem4));
}
// Tile shapes of the batched kernels (w x h).
constexpr int RCD_SHAPE_W[DS_RCD_SHAPES] = {32, 64, 48, 24, 16};
constexpr int RCD_SHAPE_H[DS_RCD_SHAPES] = {32, 16, 24, 48, 64};
constexpr size_t smax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t RCD_BATCH_SMEM = smax(smax(smax(rcd_smem(32, 32, 7), rcd_smem(64, 16, 7)),
                                             smax(rcd_smem(48, 24, 7), rcd_smem(24, 48, 7))),
                                        rcd_smem(16, 64, 7));

// index of the frame owning global tile t: the last f with tile0(f) <= t
template <class Get>
__device__ __forceinline__ int find_frame(int n, int t, Get tile0) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile0(mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int NT>
__device__ __noinline__ void rcd_batch_tile(const ds_batch_frame& F, int local, float* smem);

// Persistent RCD over the tiles of all frames; each frame uses its own tile shape.
__global__ void __launch_bounds__(RCD_THREADS, 2) rcd_batch_kernel(const ds_batch_frame* __restrict__ frames, int n,
                                                                   int total) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    const int f = find_frame(n, t, [&](int i) { return frames[i].rcd_tile0; });
    const ds_batch_frame& F = frames[f];
    __syncthreads();  // the previous tile is done with shared memory
    rcd_batch_tile<RCD_THREADS>(F, t - F.rcd_tile0, smem);  // the fused kernel's RCD tile
  }
}

// ------------------------------------------------------------------ highlights
// cfa_clip_levels (demosaic.rs:419-430): per-colour maximum of every third
// row. Values are clamped at 0 (the reference starts its maxima at 0), so the
// float bit patterns order like the values and atomicMax on them is exact.
template <class Src>
__global__ void clip_levels_kernel(Src src, int w, int h, ds_pat pat, unsigned* __restrict__ mx_bits) {
  __shared__ unsigned smx[3];
  if (threadIdx.x < 3) smx[threadIdx.x] = 0u;
  __syncthreads();
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = 3 * blockIdx.y;
  if (x < w) {
    const int c = pat.at(x, y);
    const float v = src.load(x, y, c);
    if (v > 0.f) atomicMax(&smx[c], __float_as_uint(v));
  }
  __syncthreads();
  if (threadIdx.x < 3 && smx[threadIdx.x]) atomicMax(&mx_bits[threadIdx.x], smx[threadIdx.x]);
}

// levels >= 0.95 are trusted, others become FLT_MAX (demosaic.rs:429)
__global__ void clip_levels_final_kernel(const unsigned* __restrict__ mx_bits, float* __restrict__ raw_clip) {
  const int c = threadIdx.x;
  if (c < 3) {
    const float m = __uint_as_float(mx_bits[c]);
    raw_clip[c] = m >= 0.95f ? m : FLT_MAX;
  }
}

struct HlLevels {
  float lvl[3];
  __device__ __forceinline__ HlLevels(const float* raw_clip, float m0, float m1, float m2) {
    const float mul[3] = {m0, m1, m2};
#pragma unroll
    for (int c = 0; c < 3; c++) lvl[c] = raw_clip[c] == FLT_MAX ? FLT_MAX : raw_clip[c] * mul[c] * 0.97f;
  }
  __device__ __forceinline__ bool clipped(float v, int c, float clip) const {
    return v >= lvl[c] || (clip > 0.f && v >= lvl[c] * 0.8f);
  }
};

// demosaic.rs:445-462: the weight and colour-ratio planes of bright unclipped
// pixels away from clipped ones; also raises *any when the clip plane has a
// set pixel (the reference returns early otherwise, :436-438).
__global__ void hl_weights_kernel(const float* __restrict__ img, const float* __restrict__ clip,
                                  const float* __restrict__ near_clip, const float* __restrict__ raw_clip, float m0,
                                  float m1, float m2, size_t n, float* __restrict__ wgt, float* __restrict__ rr,
                                  float* __restrict__ br, int* __restrict__ any) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const HlLevels L(raw_clip, m0, m1, m2);
  const float cl = clip[i];
  if (cl > 0.f) *any = 1;
  const float p0 = img[3 * i], p1 = img[3 * i + 1], p2 = img[3 * i + 2];
  float k = 0.f, r = 0.f, b = 0.f;
  if (!(near_clip[i] > 0.f || L.clipped(p0, 0, cl) || L.clipped(p1, 1, cl) || L.clipped(p2, 2, cl) || p1 <= 1e-4f)) {
    const float lmin = fminf(fminf(fminf(L.lvl[0], L.lvl[1]), L.lvl[2]), 4.0f);
    const float y = __fdiv_rn(__fdiv_rn(p0 + p1 + p2, 3.0f), lmin);
    k = fminf(y * y, 1.0f);
    r = fminf(fmaxf(__fdiv_rn(p0, p1), 0.1f), 10.0f) * k;
    b = fminf(fmaxf(__fdiv_rn(p2, p1), 0.1f), 10.0f) * k;
  }
  wgt[i] = k;
  rr[i] = r;
  br[i] = b;
}

// demosaic.rs:466-500: rebuild clipped channels from the blurred ratios
__global__ void hl_apply_kernel(float* __restrict__ img, const float* __restrict__ clip,
                                const float* __restrict__ raw_clip, float m0, float m1, float m2, size_t n,
                                const float* __restrict__ wb, const float* __restrict__ rrb,
                                const float* __restrict__ brb, const int* __restrict__ any) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !*any) return;
  const HlLevels L(raw_clip, m0, m1, m2);
  float p[3] = {img[3 * i], img[3 * i + 1], img[3 * i + 2]};
  const float cv = clip[i];
  const bool cl[3] = {L.clipped(p[0], 0, cv), L.clipped(p[1], 1, cv), L.clipped(p[2], 2, cv)};
  const int nc = (int)cl[0] + (int)cl[1] + (int)cl[2];
  if (nc == 0) return;
  if (nc == 3) {
    const float m = fmaxf(fmaxf(p[0], p[1]), p[2]);
    img[3 * i] = img[3 * i + 1] = img[3 * i + 2] = m;
    return;
  }
  const float wv = wb[i];
  float r = 1.0f, b = 1.0f;
  if (wv > 1e-4f) {
    r = __fdiv_rn(rrb[i], wv);
    b = __fdiv_rn(brb[i], wv);
  }
  const float trust = fminf(wv * 3.0f, 1.0f);
  r = 1.0f + (r - 1.0f) * trust;
  b = 1.0f + (b - 1.0f) * trust;
  const float ratio[3] = {r, 1.0f, b};
  float g = p[1];
#pragma unroll
  for (int c = 0; c < 3; c++)
    if (!cl[c]) g = fmaxf(g, __fdiv_rn(p[c], ratio[c]));
#pragma unroll
  for (int c = 0; c < 3; c++)
    if (cl[c]) p[c] = fmaxf(p[c], g * ratio[c]);
  const float top = fmaxf(fmaxf(p[0], p[1]), p[2]);
  const float t3 = __fdiv_rn((float)nc, 3.0f);
  const float t = t3 * t3;
#pragma unroll
  for (int c = 0; c < 3; c++) img[3 * i + c] = p[c] + (top - p[c]) * t * 0.5f;
}

// One RCD tile of a batch frame (local tile index), with the frame's tile shape.
template <int NT>
__device__ __noinline__ void rcd_batch_tile(const ds_batch_frame& F, int local, float* smem) {
  const int ty = local / F.rcd_tiles_x, tx = local - ty * F.rcd_tiles_x;
  const SrcU16 src{F.src};
  switch (F.rcd_shape) {
    case 0: rcd_tile<SrcU16, 32, 32, NT>(src, F.w, F.h, F.pat, F.mul[0], F.mul[1], F.mul[2], F.rgb, F.clip, tx, ty, smem); break;
    case 1: rcd_tile<SrcU16, 64, 16, NT>(src, F.w, F.h, F.pat, F.mul[0], F.mul[1], F.mul[2], F.rgb, F.clip, tx, ty, smem); break;
    case 2: rcd_tile<SrcU16, 48, 24, NT>(src, F.w, F.h, F.pat, F.mul[0], F.mul[1], F.mul[2], F.rgb, F.clip, tx, ty, smem); break;
    case 3: rcd_tile<SrcU16, 24, 48, NT>(src, F.w, F.h, F.pat, F.mul[0], F.mul[1], F.mul[2], F.rgb, F.clip, tx, ty, smem); break;
    default: rcd_tile<SrcU16, 16, 64, NT>(src, F.w, F.h, F.pat, F.mul[0], F.mul[1], F.mul[2], F.rgb, F.clip, tx, ty, smem); break;
  }
}

__device__ __forceinline__ unsigned long long batch_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The whole batch in one persistent launch: CTAs take work items from a
// global counter in queue order RCD(0), RCD(1), NLM(0), RCD(2), NLM(1), ...,
// so a frame's NLM starts right after its demosaic (per-frame latency) while
// the next frame's demosaic is in flight. An NLM tile first waits, bounded by
// 2 s of device clock, until its frame's RCD tiles are all done; items are
// taken in queue order by resident CTAs and RCD items never wait, so the wait
// always ends unless a tile failed, in which case counters[1] gets
// DSGPU_ERR_TIMEOUT and the CTA stops. When a frame's last NLM tile is done,
// stamps[f] = the device clock. The tile bodies are those of the one-frame
// kernels, so every frame's output equals the one-frame path's bit for bit.
template <int P>
__global__ void __launch_bounds__(nlmk::NLM_BATCH_THREADS, 2) batch_fused_kernel(const ds_batch_frame* __restrict__ frames,
                                                                     int n, const ds_batch_seg* __restrict__ segs,
                                                                     int nseg, int total, int S, int* counters,
                                                                     int max_frames,
                                                                     unsigned long long* __restrict__ stamps) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  __shared__ int item, go;
  unsigned* rcd_done = reinterpret_cast<unsigned*>(counters + DS_BATCH_CTR_RCD);
  unsigned* nlm_done = reinterpret_cast<unsigned*>(counters + DS_BATCH_CTR_RCD + max_frames);
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int t = item;
    if (t >= total) break;
    int lo = 0, hi = nseg - 1;  // the segment holding item t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (segs[mid].start <= t) lo = mid;
      else hi = mid - 1;
    }
    const ds_batch_seg sg = segs[lo];
    const ds_batch_frame& F = frames[sg.frame];
    const int local = t - sg.start;
    if (sg.kind == 0) {
      rcd_batch_tile<nlmk::NLM_BATCH_THREADS>(F, local, smem);  // out of line: keeps the NLM body's registers to itself
      __syncthreads();
      if (tid == 0) {
        __threadfence();  // the tile's output before its count
        atomicAdd(&rcd_done[sg.frame], 1u);
      }
    } else {
      if (tid == 0) {
        const unsigned need = (unsigned)F.rcd_tiles;
        const unsigned long long t0 = batch_clock_ns();
        int ok = 1;
        while ((unsigned)atomicAdd(&rcd_done[sg.frame], 0u) < need) {
          if (batch_clock_ns() - t0 > 2000000000ull) {
            ok = 0;
            atomicExch(&counters[1], DSGPU_ERR_TIMEOUT);
            break;
          }
          __nanosleep(200);
        }
        __threadfence();  // the frame's demosaiced pixels before the tile reads them
        go = ok;
      }
      __syncthreads();
      if (!go) break;
      const int per = F.nlm_tiles_x * F.nlm_tiles_y;
      const int ch = local / per, r = local - ch * per;
      const int ty = r / F.nlm_tiles_x, tx = r - ty * F.nlm_tiles_x;
      nlmk::nlm_tile<P, false, DSGPU_NLM_MAX_SEARCH, nlmk::NLM_BATCH_TX>(F.rgb, F.w, F.h, 3, S, F.sigma, F.out, tx, ty, ch,
                                                                      smem);
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        if (atomicAdd(&nlm_done[sg.frame], 1u) + 1u == (unsigned)(3 * per)) stamps[sg.frame] = batch_clock_ns();
      }
    }
    __syncthreads();  // every thread has read `item` and is done with shared memory
  }
}

template <int P>
cudaError_t launch_batch_fused_p(cudaStream_t st, const ds_batch_frame* frames, int n, const ds_batch_seg* segs,
                                 int nseg, int total, int S, int grid, int* counters, int max_frames,
                                 unsigned long long* stamps) {
  const size_t nlm = nlmk::nlm_smem_bytes(S, P, false, DSGPU_NLM_MAX_SEARCH, nlmk::NLM_BATCH_TX);
  const size_t smem = nlm > RCD_BATCH_SMEM ? nlm : RCD_BATCH_SMEM;
  cudaError_t e = cudaFuncSetAttribute(batch_fused_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  batch_fused_kernel<P><<<grid, nlmk::NLM_BATCH_THREADS, smem, st>>>(frames, n, segs, nseg, total, S, counters, max_frames,
                                                         stamps);
  return cudaGetLastError();
}

template <class Src>
// tile rows [ty0, ty1) of RTY rows (ty1 < 0: to the last)
cudaError_t launch_rcd(cudaStream_t st, Src src, int w, int h, ds_pat pat, const float mul[3], float* out_rgb,
                       float* out_clip, int ty0 = 0, int ty1 = -1) {
  const int tiles_y = (h + RTY - 1) / RTY;
  if (ty1 < 0 || ty1 > tiles_y) ty1 = tiles_y;
  if (ty0 >= ty1) return cudaSuccess;
  // the attribute is per function and device: set it on every call (cheap)
  cudaError_t e = cudaFuncSetAttribute(rcd_tile_kernel<Src>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)RCD_SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid((w + RTX - 1) / RTX, ty1 - ty0);
  rcd_tile_kernel<Src><<<grid, RCD_THREADS_1F, RCD_SMEM, st>>>(src, w, h, pat, mul[0], mul[1], mul[2], out_rgb,
                                                            out_clip, ty0);
  return cudaGetLastError();
}

}  // namespace

cudaError_t ds_launch_normalize_src(cudaStream_t st, const ds_src_u16& src, int w, int h, ds_pat pat, float* out) {
  dim3 grid((w + 255) / 256, h);
  normalize_u16_kernel<<<grid, 256, 0, st>>>(src, w, h, pat, out);
  return cudaGetLastError();
}

cudaError_t ds_launch_normalize_u16(cudaStream_t st, const uint16_t* raw, int w, int h, size_t pitch, ds_pat pat,
                                    float black, const float white[3], float* out) {
  const ds_src_u16 src{raw, pitch, black, {white[0], white[1], white[2]}};
  return ds_launch_normalize_src(st, src, w, h, pat, out);
}

cudaError_t ds_launch_clip_plane(cudaStream_t st, const float* cfa, int w, int h, float* out) {
  dim3 grid((w + 255) / 256, h);
  clip_plane_kernel<<<grid, 256, 0, st>>>(cfa, w, h, out);
  return cudaGetLastError();
}

cudaError_t ds_launch_mhc(cudaStream_t st, const float* cfa, int w, int h, ds_pat pat, const float mul[3],
                          float* out_rgb) {
  dim3 grid((w + 255) / 256, h);
  mhc_kernel<<<grid, 256, 0, st>>>(cfa, w, h, pat, mul[0], mul[1], mul[2], out_rgb);
  return cudaGetLastError();
}

cudaError_t ds_launch_superpixel(cudaStream_t st, const float* cfa, int w, int h, ds_pat pat, const float mul[3],
                                 float* out_rgb, float* out_clip) {
  const int ow = w / 2, oh = h / 2;
  if (ow == 0 || oh == 0) return cudaSuccess;
  dim3 grid((ow + 255) / 256, oh);
  superpixel_kernel<<<grid, 256, 0, st>>>(cfa, w, h, pat, mul[0], mul[1], mul[2], out_rgb, out_clip);
  return cudaGetLastError();
}

cudaError_t ds_launch_rcd_f32(cudaStream_t st, ds_src_f32 src, int w, int h, ds_pat pat, const float mul[3],
                              float* out_rgb, float* out_clip) {
  return launch_rcd(st, SrcF32{src}, w, h, pat, mul, out_rgb, out_clip);
}

cudaError_t ds_launch_rcd_u16(cudaStream_t st, ds_src_u16 src, int w, int h, ds_pat pat, const float mul[3],
                              float* out_rgb, float* out_clip) {
  return launch_rcd(st, SrcU16{src}, w, h, pat, mul, out_rgb, out_clip);
}

// the 32-row tile rows [ty0, ty1) only; they read raw rows [32 ty0 - 10, 32 ty1 + 10)
cudaError_t ds_launch_rcd_u16_rows(cudaStream_t st, ds_src_u16 src, int w, int h, ds_pat pat, const float mul[3],
                                   float* out_rgb, float* out_clip, int ty0, int ty1) {
  return launch_rcd(st, SrcU16{src}, w, h, pat, mul, out_rgb, out_clip, ty0, ty1);
}

void ds_rcd_batch_shape(int s, int* tile_w, int* tile_h) {
  s = s < 0 || s >= DS_RCD_SHAPES ? 0 : s;
  *tile_w = RCD_SHAPE_W[s];
  *tile_h = RCD_SHAPE_H[s];
}

cudaError_t ds_launch_rcd_batch(cudaStream_t st, const ds_batch_frame* frames, int n, int total_tiles, int grid) {
  if (n <= 0 || total_tiles <= 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(rcd_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)RCD_BATCH_SMEM);
  if (e != cudaSuccess) return e;
  rcd_batch_kernel<<<grid, RCD_THREADS, RCD_BATCH_SMEM, st>>>(frames, n, total_tiles);
  return cudaGetLastError();
}

// ---- highlights (host side)

// image.rs:363-373 box_radii_for_gauss, in f32 as written there
void ds_box_radii_for_gauss(float sigma, int n, int* radii) {
  const float w_ideal = sqrtf(12.0f * sigma * sigma / (float)n + 1.0f);
  int wl = (int)floorf(w_ideal);
  if (wl % 2 == 0) wl -= 1;
  const int wu = wl + 2;
  const float m_ideal = (12.0f * sigma * sigma - (float)(n * wl * wl) - 4.0f * (float)n * (float)wl - 3.0f * (float)n) /
                        (-4.0f * (float)wl - 4.0f);
  const int m = (int)roundf(m_ideal);
  for (int i = 0; i < n; i++) {
    const int r = ((i < m ? wl : wu) - 1) / 2;
    radii[i] = r > 0 ? r : 0;
  }
}

template <class Src>
static cudaError_t launch_clip_levels(cudaStream_t st, Src src, int w, int h, ds_pat pat, unsigned* bits,
                                      float* raw_clip) {
  cudaError_t e = cudaMemsetAsync(bits, 0, 3 * sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  if (w > 0 && h > 0) {
    dim3 grid((w + 255) / 256, (h + 2) / 3);
    clip_levels_kernel<Src><<<grid, 256, 0, st>>>(src, w, h, pat, bits);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  clip_levels_final_kernel<<<1, 32, 0, st>>>(bits, raw_clip);
  return cudaGetLastError();
}

cudaError_t ds_launch_clip_levels_f32(cudaStream_t st, const float* cfa, int w, int h, ds_pat pat, unsigned* bits,
                                      float* raw_clip) {
  return launch_clip_levels(st, SrcF32{ds_src_f32{cfa, w}}, w, h, pat, bits, raw_clip);
}

cudaError_t ds_launch_clip_levels_u16(cudaStream_t st, ds_src_u16 src, int w, int h, ds_pat pat, unsigned* bits,
                                      float* raw_clip) {
  return launch_clip_levels(st, SrcU16{src}, w, h, pat, bits, raw_clip);
}

size_t ds_highlights_scratch_bytes(int w, int h) { return (size_t)w * h * sizeof(float) * 10 + 256; }

// reconstruct_highlights (demosaic.rs:435-502) in place on img; raw_clip is a
// device array of 3 (from ds_launch_clip_levels_*); scratch holds
// ds_highlights_scratch_bytes(w, h).
cudaError_t ds_launch_highlights(cudaStream_t st, float* img, const float* clip, int w, int h, const float mul[3],
                                 const float* raw_clip, void* scratch, unsigned* launches) {
  const size_t n = (size_t)w * h;
  if (n == 0) return cudaSuccess;
  float* f = static_cast<float*>(scratch);
  float *near_clip = f, *wgt = f + n, *rr = f + 2 * n, *br = f + 3 * n, *wb = f + 4 * n, *rrb = f + 5 * n,
        *brb = f + 6 * n, *ta = f + 7 * n, *tb = f + 8 * n, *tmp = f + 9 * n;
  int* any = reinterpret_cast<int*>(f + 10 * n);
  cudaError_t e = cudaMemsetAsync(any, 0, sizeof(int), st);
  if (e == cudaSuccess) e = ds_launch_box_blur(st, clip, w, h, 3, tmp, near_clip);
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (e == cudaSuccess) {
    hl_weights_kernel<<<blocks, 256, 0, st>>>(img, clip, near_clip, raw_clip, mul[0], mul[1], mul[2], n, wgt, rr, br,
                                              any);
    e = cudaGetLastError();
  }
  const float sigma = fmaxf((float)(w > h ? w : h) / 120.0f, 2.0f);  // demosaic.rs:442
  int r[3];
  ds_box_radii_for_gauss(sigma, 3, r);
  const float* src[3] = {wgt, rr, br};
  float* dst[3] = {wb, rrb, brb};
  for (int k = 0; k < 3 && e == cudaSuccess; k++) {  // gaussian_blur (image.rs:327-338), sigma >= 2
    e = ds_launch_box_blur(st, src[k], w, h, r[0], tmp, ta);
    if (e == cudaSuccess) e = ds_launch_box_blur(st, ta, w, h, r[1], tmp, tb);
    if (e == cudaSuccess) e = ds_launch_box_blur(st, tb, w, h, r[2], tmp, dst[k]);
  }
  if (e == cudaSuccess) {
    hl_apply_kernel<<<blocks, 256, 0, st>>>(img, clip, raw_clip, mul[0], mul[1], mul[2], n, wb, rrb, brb, any);
    e = cudaGetLastError();
  }
  if (launches) *launches += 3 + 2 * 10;
  return e;
}

// ---- orientation (decode.rs:414-426)

// Source pixel of output (x, y) for EXIF orientation o of a w x h image.
__device__ __forceinline__ void orient_src(int o, int w, int h, int x, int y, int& sx, int& sy) {
  switch (o) {
    case 2: sx = w - 1 - x; sy = y; break;
    case 3: sx = w - 1 - x; sy = h - 1 - y; break;
    case 4: sx = x; sy = h - 1 - y; break;
    case 5: sx = y; sy = x; break;
    case 6: sx = y; sy = h - 1 - x; break;
    case 7: sx = w - 1 - y; sy = h - 1 - x; break;
    case 8: sx = w - 1 - y; sy = x; break;
    default: sx = x; sy = y; break;
  }
}

// One 32 x 32 output tile: its source block is read row by row (coalesced)
// into shared memory, then written out row by row (coalesced); the mapping
// is affine with unit coefficients, so the block is 32 x 32 as well.
__global__ void orient_kernel(const float* __restrict__ in, int w, int h, int o, int ow, int oh,
                              float* __restrict__ out) {
  __shared__ float t[3][32][33];
  const int X0 = blockIdx.x * 32, Y0 = blockIdx.y * 32;
  int ax, ay, bx, by;
  orient_src(o, w, h, X0, Y0, ax, ay);
  orient_src(o, w, h, X0 + 31, Y0 + 31, bx, by);
  const int sx0 = ax < bx ? ax : bx, sy0 = ay < by ? ay : by;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int sx = sx0 + threadIdx.x, sy = sy0 + j;
    if (sx >= 0 && sx < w && sy >= 0 && sy < h) {
      const float* p = in + ((size_t)sy * w + sx) * 3;
      t[0][j][threadIdx.x] = p[0];
      t[1][j][threadIdx.x] = p[1];
      t[2][j][threadIdx.x] = p[2];
    }
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int x = X0 + threadIdx.x, y = Y0 + j;
    if (x >= ow || y >= oh) continue;
    int sx, sy;
    orient_src(o, w, h, x, y, sx, sy);
    float* q = out + ((size_t)y * ow + x) * 3;
    q[0] = t[0][sy - sy0][sx - sx0];
    q[1] = t[1][sy - sy0][sx - sx0];
    q[2] = t[2][sy - sy0][sx - sx0];
  }
}

// apply_orientation: out is (h x w) for orientations 5-8, else (w x h)
cudaError_t ds_launch_orientation(cudaStream_t st, const float* in, int w, int h, int o, float* out) {
  const bool swap = o >= 5 && o <= 8;
  const int ow = swap ? h : w, oh = swap ? w : h;
  if (ow == 0 || oh == 0) return cudaSuccess;
  if (o < 2 || o > 8)  // the identity (and unknown codes, which the reference leaves alone)
    return cudaMemcpyAsync(out, in, (size_t)w * h * 3 * sizeof(float), cudaMemcpyDeviceToDevice, st);
  dim3 grid((ow + 31) / 32, (oh + 31) / 32);
  orient_kernel<<<grid, dim3(32, 8), 0, st>>>(in, w, h, o, ow, oh, out);
  return cudaGetLastError();
}

cudaError_t ds_launch_batch_fused(cudaStream_t st, const ds_batch_frame* frames, int n, const ds_batch_seg* segs,
                                  int nseg, int total_items, int search, int patch, int grid, int* counters,
                                  int max_frames, unsigned long long* stamps) {
  if (n <= 0 || total_items <= 0) return cudaSuccess;
  if (search <= 0 || search > DSGPU_NLM_MAX_SEARCH) return cudaErrorInvalidValue;
  switch (patch) {
    case 0: return launch_batch_fused_p<0>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 1: return launch_batch_fused_p<1>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 2: return launch_batch_fused_p<2>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 3: return launch_batch_fused_p<3>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 4: return launch_batch_fused_p<4>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 5: return launch_batch_fused_p<5>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 6: return launch_batch_fused_p<6>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    case 7: return launch_batch_fused_p<7>(st, frames, n, segs, nseg, total_items, search, grid, counters, max_frames, stamps);
    default: return cudaErrorInvalidValue;
  }
}
