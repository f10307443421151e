// dsref — CPU oracle for the RCD demosaic + NLM denoise path.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker: the GPU library
// never links, loads or calls it. Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py may use it.
//
// It restates, in C++, the CPU code of darkslide-core (Rust) for this path,
// operation for operation and in the same evaluation order, so that an f32
// build reproduces the reference bit for bit wherever the reference itself is
// deterministic:
//   decode.rs:264-306   CFA normalisation (u16 -> (raw-black)/max(white-black,1))
//   demosaic.rs:17      CLIP = 0.995
//   demosaic.rs:20-27   demosaic(Full, Bayer) = rcd_bayer + clip_plane
//   demosaic.rs:31-42   clip_plane
//   demosaic.rs:45-87   superpixel (Draft quality, Bayer 2x2)
//   demosaic.rs:90-124  mhc_bayer
//   demosaic.rs:147-344 rcd_bayer
//   image.rs:269-313    box_blur (separable running sums, clamped edges)
//   enhance.rs:10-32    estimate_noise
//   enhance.rs:36-72    nlm (offset chunks reduced in chunk order)
//   enhance.rs:75-92    denoise (Oklab L NLM + guided chroma)
//   image.rs:385-405    guided_filter
//   demosaic.rs:419-502 cfa_clip_levels, reconstruct_highlights
//   image.rs:327-338, 363-373  gaussian_blur (sigma >= 2), box_radii_for_gauss
//   color.rs:6-98, 380-419  matrix helpers, Bradford, ProPhoto, Oklab
// Every kernel is a template on the arithmetic type; the double instantiation
// is the FP64 oracle.
//
// Parity pin: the reference is Rust and no Rust toolchain exists here, so the
// reference itself cannot be run. Its own tests (demosaic.rs:514-537,
// enhance.rs:137-151, image.rs:455-462) are property tests and hold no golden
// vectors; tests/test_oracle.py restates them against this oracle, and a
// second, independent numpy restatement (tests/np_restate.py) cross-checks it.
// Exact-value parity with the Rust binary is therefore UNPINNED.
//
// Build with -ffp-contract=off: Rust never fuses a*b+c, so neither may we.

#include <algorithm>
#include <cfloat>
#include <cmath>

// The seeded synthetic mosaic generator of the library (host half of a
// header shared with the device renderer), so that the CPU legs of the
// benchmark and the tests can make their inputs without loading the GPU
// library. It is input generation, not part of the restated path.
#include "../darkslide_b200/csrc/scene.h"
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename T> inline T tmax(T a, T b) { return std::fmax(a, b); }  // Rust f32::max (NaN-ignoring)
template <typename T> inline T tabs(T a) { return std::fabs(a); }
inline float texp(float v) { return expf(v); }
inline double texp(double v) { return std::exp(v); }

struct Pat {
  uint8_t c[4];
  // decode.rs:26-28 color_at(x,y) = colors[(y % 2) * 2 + x % 2] for a 2x2 pattern
  inline int at(size_t x, size_t y) const { return c[(y & 1) * 2 + (x & 1)]; }
};

inline long clampi(long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------- clip_plane
// demosaic.rs:31-42: 3x3 clamped-edge max of [v >= CLIP]
template <typename T>
void clip_plane(const float* cfa, size_t w, size_t h, T* out) {
  const float CLIP = 0.995f;  // demosaic.rs:17
  std::vector<T> raw(w * h);
  for (size_t i = 0; i < w * h; i++) raw[i] = cfa[i] >= CLIP ? T(1) : T(0);
#pragma omp parallel for schedule(static)
  for (long y = 0; y < (long)h; y++)
    for (long x = 0; x < (long)w; x++) {
      T m = 0;
      for (long dy = -1; dy <= 1; dy++)
        for (long dx = -1; dx <= 1; dx++) {
          long sx = clampi(x + dx, 0, (long)w - 1), sy = clampi(y + dy, 0, (long)h - 1);
          m = tmax(m, raw[sy * w + sx]);
        }
      out[y * w + x] = m;
    }
}

// ---------------------------------------------------------------- superpixel
// demosaic.rs:45-87 for a Bayer pattern (t = 2): output (w/2, h/2).
void superpixel(const float* cfa, size_t w, size_t h, Pat pat, const float mul[3], float* out, float* clip) {
  const float CLIP = 0.995f;
  const size_t ow = w / 2, oh = h / 2;
#pragma omp parallel for schedule(static)
  for (long y = 0; y < (long)oh; y++)
    for (size_t x = 0; x < ow; x++) {
      float acc[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
      unsigned n[3] = {0, 0, 0}, clipped = 0;
      for (size_t dy = 0; dy < 2; dy++)
        for (size_t dx = 0; dx < 2; dx++) {
          const size_t sx = x * 2 + dx, sy = y * 2 + dy;
          const int c = pat.at(sx, sy);
          const float v = cfa[sy * w + sx];
          if (v >= CLIP) clipped++;
          mx[c] = std::fmax(mx[c], v);
          acc[c] += v;
          n[c]++;
        }
      for (int c = 0; c < 3; c++) {
        const float v = mx[c] >= CLIP ? mx[c] : (n[c] > 0 ? acc[c] / (float)n[c] : 0.0f);
        out[(y * ow + x) * 3 + c] = v * mul[c];
      }
      clip[y * ow + x] = std::fmin((float)clipped / 4.0f * 2.0f, 1.0f);
    }
}

// ----------------------------------------------------------------- mhc_bayer
// demosaic.rs:90-124. Reads data*mul with clamp-to-edge, NOT clamped at 0.
template <typename T>
void mhc_bayer(const float* cfa, size_t w, size_t h, Pat pat, const T mul[3], T* out /*w*h*3*/) {
  auto at = [&](long x, long y) -> T {
    x = clampi(x, 0, (long)w - 1);
    y = clampi(y, 0, (long)h - 1);
    return T(cfa[y * w + x]) * mul[pat.at(x, y)];
  };
#pragma omp parallel for schedule(static)
  for (long y = 0; y < (long)h; y++)
    for (long x = 0; x < (long)w; x++) {
      const int c = pat.at(x, y);
      const T v = at(x, y);
      auto p = [&](long dx, long dy) { return at(x + dx, y + dy); };
      const T g_at_rb = (T(4) * v + T(2) * (p(0, -1) + p(-1, 0) + p(1, 0) + p(0, 1)) -
                         (p(0, -2) + p(-2, 0) + p(2, 0) + p(0, 2))) / T(8);
      const T rb_g_row = (T(5) * v + T(4) * (p(-1, 0) + p(1, 0)) -
                          (p(-2, 0) + p(2, 0) + p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) +
                          T(0.5) * (p(0, -2) + p(0, 2))) / T(8);
      const T rb_g_col = (T(5) * v + T(4) * (p(0, -1) + p(0, 1)) -
                          (p(0, -2) + p(0, 2) + p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) +
                          T(0.5) * (p(-2, 0) + p(2, 0))) / T(8);
      const T rb_diag = (T(6) * v + T(2) * (p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) -
                         T(1.5) * (p(0, -2) + p(-2, 0) + p(2, 0) + p(0, 2))) / T(8);
      T o0, o1, o2;
      if (c == 1) {
        const int row_c = pat.at(x + 1, y);  // demosaic.rs:116
        if (row_c == 0) { o0 = rb_g_row; o1 = v; o2 = rb_g_col; }
        else            { o0 = rb_g_col; o1 = v; o2 = rb_g_row; }
      } else if (c == 0) { o0 = v; o1 = g_at_rb; o2 = rb_diag; }
      else               { o0 = rb_diag; o1 = g_at_rb; o2 = v; }
      T* o = out + (y * w + x) * 3;
      o[0] = tmax(o0, T(0));
      o[1] = tmax(o1, T(0));
      o[2] = tmax(o2, T(0));
    }
}

// ----------------------------------------------------------------- rcd_bayer
// demosaic.rs:147-344, pass for pass.
template <typename T>
void rcd_bayer(const float* cfa, size_t w, size_t h, Pat pat, const T mul[3], T* out /*w*h*3*/) {
  if (w < 16 || h < 16) {  // demosaic.rs:149-151
    mhc_bayer<T>(cfa, w, h, pat, mul, out);
    return;
  }
  const size_t n = w * h;
  auto fc = [&](size_t x, size_t y) { return pat.at(x, y); };
  std::vector<T> c(n);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) c[i] = tmax(T(cfa[i]) * mul[fc(i % w, i / w)], T(0));  // :154
  const T eps = T(1e-5f);  // :155 (an f32 literal in the reference)
  auto sq = [](T v) { return v * v; };
  const long w1 = w, w2 = 2 * w, w3 = 3 * w, w4 = 4 * w;
  const size_t border = 4;

  // step 1 (:160-184)
  std::vector<T> bv(n, T(0)), bh(n, T(0));
#pragma omp parallel for schedule(static)
  for (long y = 3; y < (long)h - 3; y++)
    for (size_t x = 3; x < w - 3; x++) {
      const long i = y * w + x;
      bv[i] = sq((c[i - w3] - c[i - w1] - c[i + w1] + c[i + w3]) - T(3) * (c[i - w2] + c[i + w2]) + T(6) * c[i]);
      bh[i] = sq((c[i - 3] - c[i - 1] - c[i + 1] + c[i + 3]) - T(3) * (c[i - 2] + c[i + 2]) + T(6) * c[i]);
    }
  std::vector<T> vh(n, T(0.5));
#pragma omp parallel for schedule(static)
  for (long y = border; y < (long)(h - border); y++)
    for (size_t x = border; x < w - border; x++) {
      const long i = y * w + x;
      const T vs = tmax(bv[i - w1] + bv[i] + bv[i + w1], eps);
      const T hs = tmax(bh[i - 1] + bh[i] + bh[i + 1], eps);
      vh[i] = vs / (vs + hs);
    }
  std::vector<T>().swap(bv);
  std::vector<T>().swap(bh);

  // step 2 (:188-201)
  std::vector<T> lpf(n, T(0));
#pragma omp parallel for schedule(static)
  for (long y = 2; y < (long)h - 2; y++)
    for (size_t x = 2; x < w - 2; x++) {
      if (fc(x, y) == 1) continue;
      const long i = y * w + x;
      lpf[i] = c[i] + T(0.5) * (c[i - w1] + c[i + w1] + c[i - 1] + c[i + 1]) +
               T(0.25) * (c[i - w1 - 1] + c[i - w1 + 1] + c[i + w1 - 1] + c[i + w1 + 1]);
    }

  // r/g/b init (:203-214)
  std::vector<T> base(n * 3);
  mhc_bayer<T>(cfa, w, h, pat, mul, base.data());
  std::vector<T> r(n), g(n), b(n);
  for (size_t i = 0; i < n; i++) {
    const int col = fc(i % w, i / w);
    r[i] = col == 0 ? c[i] : base[i * 3 + 0];
    g[i] = col == 1 ? c[i] : base[i * 3 + 1];
    b[i] = col == 2 ? c[i] : base[i * 3 + 2];
  }
  std::vector<T>().swap(base);

  auto disc = [&](const std::vector<T>& d, long i) -> T {  // :216-220
    const T central = d[i];
    const T neigh = T(0.25) * (d[i - w1 - 1] + d[i - w1 + 1] + d[i + w1 - 1] + d[i + w1 + 1]);
    return tabs(T(0.5) - central) < tabs(T(0.5) - neigh) ? neigh : central;
  };

  // step 3: green at R/B (:222-245)
#pragma omp parallel for schedule(static)
  for (long y = border; y < (long)(h - border); y++)
    for (size_t x = border; x < w - border; x++) {
      if (fc(x, y) == 1) continue;
      const long i = y * w + x;
      const T vd = disc(vh, i);
      const T n_grad = eps + tabs(c[i - w1] - c[i + w1]) + tabs(c[i] - c[i - w2]) + tabs(c[i - w1] - c[i - w3]) + tabs(c[i - w2] - c[i - w4]);
      const T s_grad = eps + tabs(c[i - w1] - c[i + w1]) + tabs(c[i] - c[i + w2]) + tabs(c[i + w1] - c[i + w3]) + tabs(c[i + w2] - c[i + w4]);
      const T w_grad = eps + tabs(c[i - 1] - c[i + 1]) + tabs(c[i] - c[i - 2]) + tabs(c[i - 1] - c[i - 3]) + tabs(c[i - 2] - c[i - 4]);
      const T e_grad = eps + tabs(c[i - 1] - c[i + 1]) + tabs(c[i] - c[i + 2]) + tabs(c[i + 1] - c[i + 3]) + tabs(c[i + 2] - c[i + 4]);
      const T n_est = c[i - w1] * T(2) * lpf[i] / (eps + lpf[i] + lpf[i - w2]);
      const T s_est = c[i + w1] * T(2) * lpf[i] / (eps + lpf[i] + lpf[i + w2]);
      const T w_est = c[i - 1] * T(2) * lpf[i] / (eps + lpf[i] + lpf[i - 2]);
      const T e_est = c[i + 1] * T(2) * lpf[i] / (eps + lpf[i] + lpf[i + 2]);
      const T v_est = (s_grad * n_est + n_grad * s_est) / (n_grad + s_grad);
      const T h_est = (w_grad * e_est + e_grad * w_est) / (e_grad + w_grad);
      g[i] = tmax(vd * h_est + (T(1) - vd) * v_est, T(0));
    }
  std::vector<T>().swap(lpf);

  // step 4.1/4.2 (:248-272)
  std::vector<T> bp(n, T(0)), bq(n, T(0));
#pragma omp parallel for schedule(static)
  for (long y = 3; y < (long)h - 3; y++)
    for (size_t x = 3; x < w - 3; x++) {
      const long i = y * w + x;
      bp[i] = sq((c[i - w3 - 3] - c[i - w1 - 1] - c[i + w1 + 1] + c[i + w3 + 3]) - T(3) * (c[i - w2 - 2] + c[i + w2 + 2]) + T(6) * c[i]);
      bq[i] = sq((c[i - w3 + 3] - c[i - w1 + 1] - c[i + w1 - 1] + c[i + w3 - 3]) - T(3) * (c[i - w2 + 2] + c[i + w2 - 2]) + T(6) * c[i]);
    }
  std::vector<T> pq(n, T(0.5));
#pragma omp parallel for schedule(static)
  for (long y = border; y < (long)(h - border); y++)
    for (size_t x = border; x < w - border; x++) {
      const long i = y * w + x;
      const T ps = tmax(bp[i - w1 - 1] + bp[i] + bp[i + w1 + 1], eps);
      const T qs = tmax(bq[i - w1 + 1] + bq[i] + bq[i + w1 - 1], eps);
      pq[i] = ps / (ps + qs);
    }
  std::vector<T>().swap(bp);
  std::vector<T>().swap(bq);

  // step 4.3: R at B and B at R (:276-308); chan is the pre-pass clone
  auto pass43 = [&](std::vector<T>& target, int at_color) {
    const std::vector<T> cc = target;
#pragma omp parallel for schedule(static)
    for (long y = border; y < (long)(h - border); y++)
      for (size_t x = border; x < w - border; x++) {
        if (fc(x, y) != at_color) continue;
        const long i = y * w + x;
        const T pd = disc(pq, i);
        const T nw_g = eps + tabs(cc[i - w1 - 1] - cc[i + w1 + 1]) + tabs(cc[i - w1 - 1] - cc[i - w3 - 3]) + tabs(g[i] - g[i - w2 - 2]);
        const T ne_g = eps + tabs(cc[i - w1 + 1] - cc[i + w1 - 1]) + tabs(cc[i - w1 + 1] - cc[i - w3 + 3]) + tabs(g[i] - g[i - w2 + 2]);
        const T sw_g = eps + tabs(cc[i + w1 - 1] - cc[i - w1 + 1]) + tabs(cc[i + w1 - 1] - cc[i + w3 - 3]) + tabs(g[i] - g[i + w2 - 2]);
        const T se_g = eps + tabs(cc[i + w1 + 1] - cc[i - w1 - 1]) + tabs(cc[i + w1 + 1] - cc[i + w3 + 3]) + tabs(g[i] - g[i + w2 + 2]);
        const T nw_e = cc[i - w1 - 1] - g[i - w1 - 1];
        const T ne_e = cc[i - w1 + 1] - g[i - w1 + 1];
        const T sw_e = cc[i + w1 - 1] - g[i + w1 - 1];
        const T se_e = cc[i + w1 + 1] - g[i + w1 + 1];
        const T p_est = (nw_g * se_e + se_g * nw_e) / (nw_g + se_g);
        const T q_est = (ne_g * sw_e + sw_g * ne_e) / (ne_g + sw_g);
        target[i] = tmax(g[i] + (T(1) - pd) * p_est + pd * q_est, T(0));
      }
  };
  pass43(r, 2);
  pass43(b, 0);

  // step 4.4: R and B at G (:310-341); chan is the post-4.3 clone
  auto pass44 = [&](std::vector<T>& target) {
    const std::vector<T> cc = target;
#pragma omp parallel for schedule(static)
    for (long y = border; y < (long)(h - border); y++)
      for (size_t x = border; x < w - border; x++) {
        if (fc(x, y) != 1) continue;
        const long i = y * w + x;
        const T vd = disc(vh, i);
        const T n_g = eps + tabs(g[i] - g[i - w2]) + tabs(cc[i - w1] - cc[i + w1]) + tabs(cc[i - w1] - cc[i - w3]);
        const T s_g = eps + tabs(g[i] - g[i + w2]) + tabs(cc[i + w1] - cc[i - w1]) + tabs(cc[i + w1] - cc[i + w3]);
        const T w_g = eps + tabs(g[i] - g[i - 2]) + tabs(cc[i - 1] - cc[i + 1]) + tabs(cc[i - 1] - cc[i - 3]);
        const T e_g = eps + tabs(g[i] - g[i + 2]) + tabs(cc[i + 1] - cc[i - 1]) + tabs(cc[i + 1] - cc[i + 3]);
        const T n_e = cc[i - w1] - g[i - w1];
        const T s_e = cc[i + w1] - g[i + w1];
        const T w_e = cc[i - 1] - g[i - 1];
        const T e_e = cc[i + 1] - g[i + 1];
        const T v_est = (n_g * s_e + s_g * n_e) / (n_g + s_g);
        const T h_est = (e_g * w_e + w_g * e_e) / (e_g + w_g);
        target[i] = tmax(g[i] + (T(1) - vd) * v_est + vd * h_est, T(0));
      }
  };
  pass44(r);
  pass44(b);

#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) {
    out[i * 3 + 0] = r[i];
    out[i * 3 + 1] = g[i];
    out[i * 3 + 2] = b[i];
  }
}

// ------------------------------------------------------------------ box_blur
// image.rs:269-313: horizontal running sum per row, then vertical running sum
// per 64-column strip; each pass multiplies by 1/(2r+1).
template <typename T>
void box_blur(const T* p, size_t w, size_t h, size_t r, T* out) {
  if (r == 0 || w == 0 || h == 0) {
    std::memcpy(out, p, w * h * sizeof(T));
    return;
  }
  const T norm = T(1) / T(2 * r + 1);
  std::vector<T> tmp(w * h);
  const long R = (long)r;
#pragma omp parallel for schedule(static)
  for (long y = 0; y < (long)h; y++) {
    const T* row = p + y * w;
    auto at = [&](long i) { return row[clampi(i, 0, (long)w - 1)]; };
    T acc = 0;
    for (long i = -R; i <= R; i++) acc += at(i);
    T* o = tmp.data() + y * w;
    for (long x = 0; x < (long)w; x++) {
      o[x] = acc * norm;
      acc += at(x + R + 1) - at(x - R);
    }
  }
  const size_t STRIP = 64;
  const long nstrips = (long)((w + STRIP - 1) / STRIP);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < nstrips; s++) {
    const size_t x0 = s * STRIP, x1 = std::min(x0 + STRIP, w), sw = x1 - x0;
    std::vector<T> acc(sw, T(0));
    auto at = [&](long y, size_t x) { return tmp[clampi(y, 0, (long)h - 1) * w + x]; };
    for (long i = -R; i <= R; i++)
      for (size_t k = 0; k < sw; k++) acc[k] += at(i, x0 + k);
    for (long y = 0; y < (long)h; y++)
      for (size_t k = 0; k < sw; k++) {
        out[y * w + x0 + k] = acc[k] * norm;
        acc[k] += at(y + R + 1, x0 + k) - at(y - R, x0 + k);
      }
  }
}

// ----------------------------------------------------------------------- nlm
// enhance.rs:36-72. Offsets in (dy outer, dx inner) order are split into
// chunks of ceil(N / nthreads); each chunk accumulates its own a/s planes and
// the chunks are summed in order, exactly as the rayon code does for a pool
// of `nthreads` threads.
template <typename T>
void nlm(const T* p, size_t w, size_t hh, T h_param, long search, size_t patch, int nthreads, T* out) {
  const size_t n = w * hh;
  const T h2 = tmax(h_param * h_param, T(1e-12f));
  std::vector<std::pair<long, long>> offs;
  for (long dy = -search; dy <= search; dy++)
    for (long dx = -search; dx <= search; dx++) offs.push_back({dx, dy});
  const size_t nt = nthreads > 0 ? (size_t)nthreads : 1;
  const size_t csz = std::max<size_t>((offs.size() + nt - 1) / nt, 1);
  const size_t nchunks = (offs.size() + csz - 1) / csz;
  std::vector<std::vector<T>> pa(nchunks), ps(nchunks);
  auto get_clamped = [&](long x, long y) {
    return p[clampi(y, 0, (long)hh - 1) * w + clampi(x, 0, (long)w - 1)];
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (long ci = 0; ci < (long)nchunks; ci++) {
    std::vector<T> a(n, T(0)), s(n, T(0)), diff(n), dist(n);
    const size_t o0 = ci * csz, o1 = std::min(o0 + csz, offs.size());
    for (size_t oi = o0; oi < o1; oi++) {
      const long dx = offs[oi].first, dy = offs[oi].second;
      for (long y = 0; y < (long)hh; y++)
        for (long x = 0; x < (long)w; x++) {
          const T q = get_clamped(x + dx, y + dy);
          const T d = p[y * w + x] - q;
          diff[y * w + x] = d * d;
        }
      // box_blur is itself OpenMP-parallel; nested regions run serially here
      box_blur<T>(diff.data(), w, hh, patch, dist.data());
      for (long y = 0; y < (long)hh; y++)
        for (long x = 0; x < (long)w; x++) {
          const size_t i = y * w + x;
          const T wt = texp(-(dist[i] / h2));
          a[i] += wt * get_clamped(x + dx, y + dy);
          s[i] += wt;
        }
    }
    pa[ci].swap(a);
    ps[ci].swap(s);
  }
  std::vector<T> acc(n, T(0)), wsum(n, T(0));
  for (size_t ci = 0; ci < nchunks; ci++)
    for (size_t i = 0; i < n; i++) {
      acc[i] += pa[ci][i];
      wsum[i] += ps[ci][i];
    }
  for (size_t i = 0; i < n; i++) out[i] = acc[i] / tmax(wsum[i], T(1e-12f));
}

// ------------------------------------------------------------ estimate_noise
// enhance.rs:10-32
float estimate_noise(const float* p, size_t w, size_t h) {
  const size_t step = std::max<size_t>((w * h) / 200000, 1);
  std::vector<float> v;
  for (size_t i = 0; i < w * h; i += step) {
    const size_t x = i % w, y = i / w;
    if (x < 1 || y < 1 || x + 1 >= w || y + 1 >= h) continue;
    const float c = p[i];
    const float lap = 4.0f * c - p[i - 1] - p[i + 1] - p[i - w] - p[i + w];
    v.push_back(std::fabs(lap));
  }
  if (v.empty()) return 0.0f;
  const size_t mid = v.size() / 2;
  std::nth_element(v.begin(), v.begin() + mid, v.end());
  return v[mid] / 0.6745f / std::sqrt(20.0f);
}


// -------------------------------------------------------------- colour / Oklab
// color.rs:6-100 (matrix helpers, chromaticities, Bradford) and :380-419
// (Oklab from linear ProPhoto). Matrix products accumulate in f64 and round
// to f32 (color.rs:15-23); inversion runs in f64 (color.rs:25-42).
typedef float M3[3][3];

void mul_mv3(const M3 m, const float v[3], float o[3]) {  // color.rs:11-13
  o[0] = m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2];
  o[1] = m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2];
  o[2] = m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2];
}

void mul_mm3(const M3 a, const M3 b, M3 o) {  // color.rs:15-23
  M3 t;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double acc = 0.0;
      for (int k = 0; k < 3; k++) acc += (double)a[i][k] * (double)b[k][j];
      t[i][j] = (float)acc;
    }
  std::memcpy(o, t, sizeof(M3));
}

void invert3(const M3 mf, M3 o) {  // color.rs:25-42
  double m[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) m[i][j] = mf[i][j];
  const double det = m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                     m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if (std::fabs(det) < 1e-12) {
    const M3 id = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    std::memcpy(o, id, sizeof(M3));
    return;
  }
  const double inv = 1.0 / det;
  const double r[3][3] = {
      {(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * inv, (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv, (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv},
      {(m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv, (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv, (m[1][0] * m[0][2] - m[0][0] * m[1][2]) * inv},
      {(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * inv, (m[2][0] * m[0][1] - m[0][0] * m[2][1]) * inv, (m[0][0] * m[1][1] - m[1][0] * m[0][1]) * inv}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o[i][j] = (float)r[i][j];
}

void xy_to_xyz(const float xy[2], float o[3]) {  // color.rs:65-69
  const float x = xy[0], y = std::fmax(xy[1], 1e-6f);
  o[0] = x / y;
  o[1] = 1.0f;
  o[2] = (1.0f - x - y) / y;
}

const float D50_XY[2] = {0.34567f, 0.35850f};  // color.rs:62-63
const float D65_XY[2] = {0.31271f, 0.32902f};

void bradford(const float src[2], const float dst[2], M3 o) {  // color.rs:80-88
  const M3 B = {{0.8951f, 0.2664f, -0.1614f}, {-0.7502f, 1.7135f, 0.0367f}, {0.0389f, -0.0685f, 1.0296f}};
  float xs[3], xd[3], s[3], d[3];
  xy_to_xyz(src, xs);
  xy_to_xyz(dst, xd);
  mul_mv3(B, xs, s);
  mul_mv3(B, xd, d);
  const M3 scale = {{d[0] / s[0], 0, 0}, {0, d[1] / s[1], 0}, {0, 0, d[2] / s[2]}};
  M3 binv, t;
  invert3(B, binv);
  mul_mm3(scale, B, t);
  mul_mm3(binv, t, o);
}

void prophoto_to_xyz(M3 o) {  // color.rs:90-98 with the ProPhoto primaries of :129 (white D50)
  const float r[2] = {0.734699f, 0.265301f}, g[2] = {0.159597f, 0.840403f}, b[2] = {0.036598f, 0.000105f};
  float pr[3], pg[3], pb[3], wv[3], sv[3];
  xy_to_xyz(r, pr);
  xy_to_xyz(g, pg);
  xy_to_xyz(b, pb);
  const M3 m = {{pr[0], pg[0], pb[0]}, {pr[1], pg[1], pb[1]}, {pr[2], pg[2], pb[2]}};
  M3 minv;
  invert3(m, minv);
  xy_to_xyz(D50_XY, wv);
  mul_mv3(minv, wv, sv);
  const M3 dg = {{sv[0], 0, 0}, {0, sv[1], 0}, {0, 0, sv[2]}};
  mul_mm3(m, dg, o);  // white == D50: no further adaptation
}

struct Oklab {  // color.rs:380-419
  M3 to_lms, from_lms, m2, m2_inv;
  Oklab() {
    const M3 M1 = {{0.818933f, 0.36186674f, -0.12885971f}, {0.032984544f, 0.9293119f, 0.03614564f}, {0.0482003f, 0.26436627f, 0.6338517f}};
    const M3 M2 = {{0.21045426f, 0.7936178f, -0.004072047f}, {1.9779985f, -2.4285922f, 0.4505937f}, {0.025904037f, 0.78277177f, -0.80867577f}};
    M3 brad, pp, t;
    bradford(D50_XY, D65_XY, brad);
    prophoto_to_xyz(pp);
    mul_mm3(brad, pp, t);
    mul_mm3(M1, t, to_lms);
    invert3(to_lms, from_lms);
    std::memcpy(m2, M2, sizeof(M3));
    invert3(M2, m2_inv);
  }
  void from_prophoto(const float p[3], float o[3]) const {
    float lms[3];
    mul_mv3(to_lms, p, lms);
    for (int i = 0; i < 3; i++) lms[i] = std::cbrt(lms[i]);
    mul_mv3(m2, lms, o);
  }
  void to_prophoto(const float lab[3], float o[3]) const {
    float l[3];
    mul_mv3(m2_inv, lab, l);
    const float c[3] = {l[0] * l[0] * l[0], l[1] * l[1] * l[1], l[2] * l[2] * l[2]};
    mul_mv3(from_lms, c, o);
  }
};

// ------------------------------------------------------------- guided filter
// image.rs:385-405 (He et al.), every box via box_blur (image.rs:269-313).
void guided_filter(const float* I, const float* p, size_t w, size_t h, size_t r, float eps, float* out) {
  const size_t n = w * h;
  std::vector<float> mean_i(n), mean_p(n), ip(n), ii(n), mean_ip(n), mean_ii(n), a(n), b(n), ma(n), mb(n);
  box_blur<float>(I, w, h, r, mean_i.data());
  box_blur<float>(p, w, h, r, mean_p.data());
  for (size_t k = 0; k < n; k++) {
    ip[k] = I[k] * p[k];
    ii[k] = I[k] * I[k];
  }
  box_blur<float>(ip.data(), w, h, r, mean_ip.data());
  box_blur<float>(ii.data(), w, h, r, mean_ii.data());
  for (size_t k = 0; k < n; k++) {
    const float cov = mean_ip[k] - mean_i[k] * mean_p[k];
    const float var = mean_ii[k] - mean_i[k] * mean_i[k];
    a[k] = cov / (var + eps);
    b[k] = mean_p[k] - a[k] * mean_i[k];
  }
  box_blur<float>(a.data(), w, h, r, ma.data());
  box_blur<float>(b.data(), w, h, r, mb.data());
  for (size_t k = 0; k < n; k++) out[k] = ma[k] * I[k] + mb[k];
}

// ---------------------------------------------------------------- highlights
// demosaic.rs:419-430 cfa_clip_levels: per-colour maximum over every third
// row, trusted as a clip level only when >= 0.95.
void cfa_clip_levels(const float* cfa, long w, long h, const Pat& pat, float out[3]) {
  float mx[3] = {0.f, 0.f, 0.f};
  for (long y = 0; y < h; y += 3)
    for (long x = 0; x < w; x++) {
      const int c = pat.at(x, y);
      mx[c] = std::fmax(mx[c], cfa[y * w + x]);
    }
  for (int c = 0; c < 3; c++) out[c] = mx[c] >= 0.95f ? mx[c] : FLT_MAX;
}

// image.rs:363-373 box_radii_for_gauss, f32 as written there.
void box_radii_for_gauss(float sigma, int n, int* radii) {
  const float w_ideal = std::sqrt(12.0f * sigma * sigma / (float)n + 1.0f);
  int wl = (int)std::floor(w_ideal);
  if (wl % 2 == 0) wl -= 1;
  const int wu = wl + 2;
  const float m_ideal = (12.0f * sigma * sigma - (float)(n * wl * wl) - 4.0f * (float)n * (float)wl - 3.0f * (float)n) /
                        (-4.0f * (float)wl - 4.0f);
  const int m = (int)std::round(m_ideal);
  for (int i = 0; i < n; i++) radii[i] = std::max(((i < m ? wl : wu) - 1) / 2, 0);
}

// image.rs:327-338 gaussian_blur for sigma >= 2 (three box blurs); the
// highlight code only calls it with sigma >= 2.
void gaussian_blur_boxes(const float* p, long w, long h, float sigma, float* out) {
  int r[3];
  box_radii_for_gauss(sigma, 3, r);
  std::vector<float> a((size_t)w * h), b((size_t)w * h);
  box_blur<float>(p, w, h, r[0], a.data());
  box_blur<float>(a.data(), w, h, r[1], b.data());
  box_blur<float>(b.data(), w, h, r[2], out);
}

// demosaic.rs:435-502 reconstruct_highlights, in place on interleaved RGB.
void reconstruct_highlights(float* img, const float* clip, long w, long h, const float mul[3], const float raw_clip[3]) {
  const size_t n = (size_t)w * h;
  bool any = false;
  for (size_t i = 0; i < n && !any; i++) any = clip[i] > 0.0f;
  if (!any) return;
  float lvl[3];
  for (int c = 0; c < 3; c++) lvl[c] = raw_clip[c] == FLT_MAX ? FLT_MAX : raw_clip[c] * mul[c] * 0.97f;
  auto is_clipped = [&](const float* p, int c, size_t i) {
    return p[c] >= lvl[c] || (clip[i] > 0.0f && p[c] >= lvl[c] * 0.8f);
  };
  const float sigma = std::fmax((float)std::max(w, h) / 120.0f, 2.0f);
  const float lmin = std::fmin(std::fmin(std::fmin(lvl[0], lvl[1]), lvl[2]), 4.0f);
  std::vector<float> near_clip(n), wgt(n, 0.f), rr(n, 0.f), br(n, 0.f);
  box_blur<float>(clip, w, h, 3, near_clip.data());
  for (size_t i = 0; i < n; i++) {
    const float* p = img + 3 * i;
    if (near_clip[i] > 0.0f || is_clipped(p, 0, i) || is_clipped(p, 1, i) || is_clipped(p, 2, i) || p[1] <= 1e-4f)
      continue;
    const float y = (p[0] + p[1] + p[2]) / 3.0f / lmin;
    const float k = std::fmin(y * y, 1.0f);
    wgt[i] = k;
    rr[i] = std::clamp(p[0] / p[1], 0.1f, 10.0f) * k;
    br[i] = std::clamp(p[2] / p[1], 0.1f, 10.0f) * k;
  }
  std::vector<float> wb(n), rrb(n), brb(n);
  gaussian_blur_boxes(wgt.data(), w, h, sigma, wb.data());
  gaussian_blur_boxes(rr.data(), w, h, sigma, rrb.data());
  gaussian_blur_boxes(br.data(), w, h, sigma, brb.data());
  for (size_t i = 0; i < n; i++) {
    float* p = img + 3 * i;
    const bool cl[3] = {is_clipped(p, 0, i), is_clipped(p, 1, i), is_clipped(p, 2, i)};
    const int nc = (int)cl[0] + (int)cl[1] + (int)cl[2];
    if (nc == 0) continue;
    const float m = std::fmax(std::fmax(p[0], p[1]), p[2]);
    if (nc == 3) {
      p[0] = p[1] = p[2] = m;
      continue;
    }
    const float wv = wb[i];
    float r = 1.0f, b = 1.0f;
    if (wv > 1e-4f) {
      r = rrb[i] / wv;
      b = brb[i] / wv;
    }
    const float trust = std::fmin(wv * 3.0f, 1.0f);
    r = 1.0f + (r - 1.0f) * trust;
    b = 1.0f + (b - 1.0f) * trust;
    const float ratio[3] = {r, 1.0f, b};
    float g = p[1];
    for (int c = 0; c < 3; c++)
      if (!cl[c]) g = std::fmax(g, p[c] / ratio[c]);
    for (int c = 0; c < 3; c++)
      if (cl[c]) p[c] = std::fmax(p[c], g * ratio[c]);
    const float top = std::fmax(std::fmax(p[0], p[1]), p[2]);
    const float t = ((float)nc / 3.0f) * ((float)nc / 3.0f);  // powi(2)
    for (int c = 0; c < 3; c++) p[c] += (top - p[c]) * t * 0.5f;
  }
}

// ------------------------------------------------------------------ denoise
// enhance.rs:75-92
void denoise(const float* img, size_t w, size_t h, float amount, int nthreads, float* out, float* sigma_out) {
  const Oklab ok;
  const size_t n = w * h;
  std::vector<float> l(n), a(n), b(n), lf(n), l2(n), a2(n), b2(n);
  for (size_t i = 0; i < n; i++) {
    float lab[3];
    ok.from_prophoto(img + i * 3, lab);
    l[i] = lab[0];
    a[i] = lab[1];
    b[i] = lab[2];
  }
  const float sigma = std::fmax(estimate_noise(l.data(), w, h), 1e-4f);
  if (sigma_out) *sigma_out = sigma;
  const float k = amount / 100.0f;
  nlm<float>(l.data(), w, h, sigma * (0.6f + 1.6f * k), 3, 1, nthreads, lf.data());
  for (size_t i = 0; i < n; i++) l2[i] = l[i] + (lf[i] - l[i]) * (0.5f + 0.5f * k);
  const size_t r = (size_t)std::fmax(((float)std::max(w, h) / 600.0f) * (1.0f + 2.0f * k), 2.0f);
  const float eps = (sigma * 2.0f) * (sigma * 2.0f);
  guided_filter(l2.data(), a.data(), w, h, r, eps, a2.data());
  guided_filter(l2.data(), b.data(), w, h, r, eps, b2.data());
  for (size_t i = 0; i < n; i++) {
    const float lab[3] = {l2[i], a2[i], b2[i]};
    float o[3];
    ok.to_prophoto(lab, o);
    for (int c = 0; c < 3; c++) out[i * 3 + c] = std::fmax(o[c], 0.0f);
  }
}

}  // namespace

extern "C" {

int dsref_omp_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void dsref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// decode.rs:292-306 (integer raws): v = (raw - black) / max(white[c] - black, 1)
void dsref_normalize_u16(const uint16_t* raw, int w, int h, size_t pitch, const uint8_t cfa[4], float black,
                         const float white[3], float* out) {
  Pat pat;
  std::memcpy(pat.c, cfa, 4);
#pragma omp parallel for schedule(static)
  for (long y = 0; y < h; y++)
    for (long x = 0; x < w; x++) {
      const int c = pat.at(x, y);
      const float raw_v = (float)raw[y * pitch + x];
      out[y * w + x] = (raw_v - black) / std::fmax(white[c] - black, 1.0f);
    }
}

// The same with load_raw's per-site black level (decode.rs:266-270): black_at
// is the bw x bh pattern at UNCROPPED coordinates (x + ox, y + oy), used in
// the numerator and in the white - black denominator of :303.
void dsref_normalize_u16_bp(const uint16_t* raw, int w, int h, size_t pitch, const uint8_t cfa[4],
                            const float* levels, int bw, int bh, int ox, int oy, const float white[3], float* out) {
  Pat pat;
  std::memcpy(pat.c, cfa, 4);
#pragma omp parallel for schedule(static)
  for (long y = 0; y < h; y++)
    for (long x = 0; x < w; x++) {
      const int c = pat.at(x, y);
      const float raw_v = (float)raw[y * pitch + x];
      const float b = levels[((y + oy) % bh) * bw + (x + ox) % bw];
      out[y * w + x] = (raw_v - b) / std::fmax(white[c] - b, 1.0f);
    }
}

void dsref_clip_plane_f32(const float* cfa, int w, int h, float* out) { clip_plane<float>(cfa, w, h, out); }

void dsref_mhc_f32(const float* cfa, int w, int h, const uint8_t pat[4], const float mul[3], float* out) {
  Pat p;
  std::memcpy(p.c, pat, 4);
  mhc_bayer<float>(cfa, w, h, p, mul, out);
}

void dsref_superpixel_f32(const float* cfa, int w, int h, const uint8_t pat[4], const float mul[3], float* out,
                          float* clip) {
  Pat p;
  std::memcpy(p.c, pat, 4);
  superpixel(cfa, w, h, p, mul, out, clip);
}

void dsref_rcd_f32(const float* cfa, int w, int h, const uint8_t pat[4], const float mul[3], float* out) {
  Pat p;
  std::memcpy(p.c, pat, 4);
  rcd_bayer<float>(cfa, w, h, p, mul, out);
}

void dsref_rcd_f64(const float* cfa, int w, int h, const uint8_t pat[4], const float mul[3], double* out) {
  Pat p;
  std::memcpy(p.c, pat, 4);
  const double m[3] = {mul[0], mul[1], mul[2]};
  rcd_bayer<double>(cfa, w, h, p, m, out);
}

void dsref_box_blur_f32(const float* in, int w, int h, int r, float* out) { box_blur<float>(in, w, h, r, out); }
void dsref_box_blur_f64(const double* in, int w, int h, int r, double* out) { box_blur<double>(in, w, h, r, out); }

void dsref_nlm_f32(const float* in, int w, int h, float h_param, int search, int patch, int nthreads, float* out) {
  nlm<float>(in, w, h, h_param, search, patch, nthreads, out);
}

void dsref_nlm_f64(const double* in, int w, int h, double h_param, int search, int patch, int nthreads, double* out) {
  nlm<double>(in, w, h, h_param, search, patch, nthreads, out);
}

float dsref_estimate_noise_f32(const float* p, int w, int h) { return estimate_noise(p, w, h); }

// Oklab matrices (to_lms, from_lms, m2_inv), row-major, 27 floats.
void dsref_oklab_matrices(float* out) {
  const Oklab ok;
  std::memcpy(out, ok.to_lms, sizeof(M3));
  std::memcpy(out + 9, ok.from_lms, sizeof(M3));
  std::memcpy(out + 18, ok.m2_inv, sizeof(M3));
}

void dsref_oklab_from_prophoto(const float* rgb, int n, float* lab) {
  const Oklab ok;
  for (int i = 0; i < n; i++) ok.from_prophoto(rgb + 3 * i, lab + 3 * i);
}

void dsref_oklab_to_prophoto(const float* lab, int n, float* rgb) {
  const Oklab ok;
  for (int i = 0; i < n; i++) ok.to_prophoto(lab + 3 * i, rgb + 3 * i);
}

void dsref_guided_filter_f32(const float* I, const float* p, int w, int h, int r, float eps, float* out) {
  guided_filter(I, p, w, h, r, eps, out);
}

void dsref_cfa_clip_levels(const float* cfa, int w, int h, const uint8_t pat[4], float* out3) {
  Pat p;
  std::memcpy(p.c, pat, 4);
  cfa_clip_levels(cfa, w, h, p, out3);
}

void dsref_box_radii_for_gauss(float sigma, int n, int* radii) { box_radii_for_gauss(sigma, n, radii); }

void dsref_reconstruct_highlights(float* img, const float* clip, int w, int h, const float mul[3],
                                  const float raw_clip[3]) {
  reconstruct_highlights(img, clip, w, h, mul, raw_clip);
}

void dsref_denoise_f32(const float* img, int w, int h, float amount, int nthreads, float* out, float* sigma) {
  denoise(img, w, h, amount, nthreads, out, sigma);
}

// The seeded synthetic mosaic (the library's scene generator; no counterpart
// in the reference): the cw x ch window at (x0, y0) of the w x h frame.
void dsref_scene_render(uint64_t seed, int w, int h, const uint8_t cfa[4], int black, int white, float gain,
                        float read_sigma, int x0, int y0, int cw, int ch, uint16_t* out) {
  ds_scene s;
  ds_scene_init(&s, seed, w, h, cfa, black, white, gain, read_sigma);
#pragma omp parallel for schedule(static)
  for (long y = 0; y < ch; y++)
    for (long x = 0; x < cw; x++) out[y * cw + x] = ds_scene_pixel(&s, x0 + (int)x, y0 + (int)y);
}

// Noise-free scene values (RGB, before white balance) of the same window.
void dsref_scene_truth(uint64_t seed, int w, int h, const uint8_t cfa[4], int black, int white, float gain,
                       float read_sigma, int x0, int y0, int cw, int ch, float* out) {
  ds_scene s;
  ds_scene_init(&s, seed, w, h, cfa, black, white, gain, read_sigma);
#pragma omp parallel for schedule(static)
  for (long y = 0; y < ch; y++)
    for (long x = 0; x < cw; x++)
      for (int c = 0; c < 3; c++)
        out[(y * cw + x) * 3 + c] = ds_mul(ds_scene_value(&s, x0 + (int)x, y0 + (int)y, c), s.ch_gain[c]);
}

}  // extern "C"
