// Seeded synthetic Bayer mosaic generator, shared by the host (C++) and the
// device (CUDA) so that both produce the same u16 mosaic bit for bit.
//
// Scene: 8 smooth 2-D sinusoids (random orientation, 0.5-8 cycles per frame,
// random phase and amplitude) plus 40 step edges (20 axis-aligned, 20
// diagonal; random position and per-channel height), clamped to [0.05, 0.9]
// of the white-minus-black range, times per-channel gains (R 0.5, G 1.0,
// B 0.7) and sampled at the CFA sites.
// Noise: DN = (lambda + sqrt(lambda) N1) / g + sigma_read N2 + black, with
// lambda = signal_DN * g electrons (Gaussian approximation of Poisson; lambda
// is at least ~50 e for every configuration used), rounded and clamped to
// [0, white].
//
// Determinism: only IEEE basic operations (add, mul, div, sqrt, rint) are
// used per pixel, never contracted into FMAs (device code uses the _rn
// intrinsics; host code is compiled with -ffp-contract=off). The sine is a
// project-written Taylor polynomial after Cody-Waite reduction; random
// numbers come from SplitMix64 on (seed, pixel index). Scene parameters are
// drawn once on the host.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define DS_HD __host__ __device__ __forceinline__
#else
#define DS_HD inline
#endif

#define DS_SCENE_NSIN 8
#define DS_SCENE_NEDGE 40

typedef struct ds_scene {
  uint64_t seed;
  int32_t w, h;
  uint8_t cfa[4];       // 2x2 colour codes 0=R 1=G 2=B, index (y%2)*2 + x%2
  int32_t black, white; // DN
  float gain_e_per_dn;  // conversion gain g
  float read_sigma;     // DN
  float ch_gain[3];     // R, G, B scene gains
  float sin_kx[DS_SCENE_NSIN], sin_ky[DS_SCENE_NSIN], sin_ph[DS_SCENE_NSIN], sin_amp[DS_SCENE_NSIN];
  int32_t edge_type[DS_SCENE_NEDGE];  // 0: x>pos  1: y>pos  2: x+y>pos  3: x-y>pos
  int32_t edge_pos[DS_SCENE_NEDGE];
  float edge_h[DS_SCENE_NEDGE][3];
  float base;           // mid level before clamping
} ds_scene;

DS_HD uint64_t ds_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

#ifdef __CUDA_ARCH__
DS_HD float ds_add(float a, float b) { return __fadd_rn(a, b); }
DS_HD float ds_sub(float a, float b) { return __fsub_rn(a, b); }
DS_HD float ds_mul(float a, float b) { return __fmul_rn(a, b); }
DS_HD float ds_div(float a, float b) { return __fdiv_rn(a, b); }
DS_HD float ds_sqrt(float a) { return __fsqrt_rn(a); }
DS_HD float ds_rint(float a) { return rintf(a); }
DS_HD float ds_floor(float a) { return floorf(a); }
#else
#include <math.h>
DS_HD float ds_add(float a, float b) { return a + b; }
DS_HD float ds_sub(float a, float b) { return a - b; }
DS_HD float ds_mul(float a, float b) { return a * b; }
DS_HD float ds_div(float a, float b) { return a / b; }
DS_HD float ds_sqrt(float a) { return sqrtf(a); }
DS_HD float ds_rint(float a) { return rintf(a); }
DS_HD float ds_floor(float a) { return floorf(a); }
#endif

// sin(x) for |x| < ~1e3: reduce by 2*pi with a two-part constant, fold into
// [-pi/2, pi/2], then the Taylor series to x^11 (error < 1e-8 there).
DS_HD float ds_sin(float x) {
  const float INV_2PI = 0.15915494309189535f;
  const float TWO_PI_HI = 6.28125f;                 // exact in 8 bits
  const float TWO_PI_LO = 0.0019353071795864769f;   // 2*pi - TWO_PI_HI
  const float PI = 3.14159265358979f, HALF_PI = 1.57079632679490f;
  float k = ds_rint(ds_mul(x, INV_2PI));
  float r = ds_sub(ds_sub(x, ds_mul(k, TWO_PI_HI)), ds_mul(k, TWO_PI_LO));
  if (r > HALF_PI) r = ds_sub(PI, r);
  if (r < -HALF_PI) r = ds_sub(-PI, r);
  float r2 = ds_mul(r, r);
  // Horner on 1 - r2/6 (1 - r2/20 (1 - r2/42 (1 - r2/72 (1 - r2/110))))
  float t = ds_sub(1.0f, ds_mul(r2, 1.0f / 110.0f));
  t = ds_sub(1.0f, ds_mul(ds_mul(r2, 1.0f / 72.0f), t));
  t = ds_sub(1.0f, ds_mul(ds_mul(r2, 1.0f / 42.0f), t));
  t = ds_sub(1.0f, ds_mul(ds_mul(r2, 1.0f / 20.0f), t));
  t = ds_sub(1.0f, ds_mul(ds_mul(r2, 1.0f / 6.0f), t));
  return ds_mul(r, t);
}

// uniform in (0,1) from 16 bits
DS_HD float ds_u16f(uint32_t v) { return ds_mul(ds_add((float)(v & 0xFFFFu), 0.5f), 1.0f / 65536.0f); }

// approximately standard normal: 8 uniforms, (sum - 4) * sqrt(12/8)
DS_HD float ds_gauss8(uint64_t a, uint64_t b) {
  float s = 0.0f;
  for (int i = 0; i < 4; i++) s = ds_add(s, ds_u16f((uint32_t)(a >> (16 * i))));
  for (int i = 0; i < 4; i++) s = ds_add(s, ds_u16f((uint32_t)(b >> (16 * i))));
  return ds_mul(ds_sub(s, 4.0f), 1.2247448713915890f);
}

// Noise-free scene value for colour channel c at pixel (x, y), in [0.05, 0.9].
DS_HD float ds_scene_value(const ds_scene* s, int x, int y, int c) {
  float v = s->base;
  const float fx = (float)x, fy = (float)y;
  for (int i = 0; i < DS_SCENE_NSIN; i++) {
    float arg = ds_add(ds_add(ds_mul(s->sin_kx[i], fx), ds_mul(s->sin_ky[i], fy)), s->sin_ph[i]);
    v = ds_add(v, ds_mul(s->sin_amp[i], ds_sin(arg)));
  }
  for (int j = 0; j < DS_SCENE_NEDGE; j++) {
    const int t = s->edge_type[j], p = s->edge_pos[j];
    const int lhs = t == 0 ? x : t == 1 ? y : t == 2 ? x + y : x - y;
    if (lhs > p) v = ds_add(v, s->edge_h[j][c]);
  }
  v = v < 0.05f ? 0.05f : v;
  v = v > 0.9f ? 0.9f : v;
  return v;
}

// Noisy u16 DN for pixel (x, y).
DS_HD uint16_t ds_scene_pixel(const ds_scene* s, int x, int y) {
  const int c = s->cfa[(y & 1) * 2 + (x & 1)];
  const float range = (float)(s->white - s->black);
  const float sig_dn = ds_mul(ds_mul(ds_scene_value(s, x, y, c), s->ch_gain[c]), range);
  const float lam = ds_mul(sig_dn, s->gain_e_per_dn);
  const uint64_t idx = (uint64_t)y * (uint64_t)s->w + (uint64_t)x;
  const uint64_t k0 = ds_splitmix64(s->seed ^ (idx * 4 + 0x5851F42D4C957F2Dull));
  const uint64_t k1 = ds_splitmix64(k0 ^ 0x14057B7EF767814Full);
  const uint64_t k2 = ds_splitmix64(k1 ^ 0x2545F4914F6CDD1Dull);
  const uint64_t k3 = ds_splitmix64(k2 ^ 0x9E3779B97F4A7C15ull);
  const float n1 = ds_gauss8(k0, k1), n2 = ds_gauss8(k2, k3);
  const float e = ds_add(lam, ds_mul(ds_sqrt(lam), n1));
  float dn = ds_add(ds_add(ds_div(e, s->gain_e_per_dn), ds_mul(s->read_sigma, n2)), (float)s->black);
  dn = ds_floor(ds_add(dn, 0.5f));
  if (dn < 0.0f) dn = 0.0f;
  if (dn > (float)s->white) dn = (float)s->white;
  return (uint16_t)dn;
}

#include <math.h>
#include <string.h>
#ifdef __CUDACC__
#define DS_HOST_ONLY __host__
#else
#define DS_HOST_ONLY
#endif
// Draw the scene parameters for `seed` (host only; the struct is then passed
// by value to the device renderer).
DS_HOST_ONLY static inline void ds_scene_init(ds_scene* s, uint64_t seed, int w, int h, const uint8_t cfa[4], int black,
                                 int white, float gain_e_per_dn, float read_sigma) {
  memset(s, 0, sizeof(*s));
  s->seed = seed;
  s->w = w;
  s->h = h;
  memcpy(s->cfa, cfa, 4);
  s->black = black;
  s->white = white;
  s->gain_e_per_dn = gain_e_per_dn;
  s->read_sigma = read_sigma;
  s->ch_gain[0] = 0.5f;
  s->ch_gain[1] = 1.0f;
  s->ch_gain[2] = 0.7f;
  s->base = 0.475f;
  uint64_t st = seed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
  auto uni = [&]() {  // uniform [0,1) with 53 bits
    st = ds_splitmix64(st);
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  const double L = (double)(w > h ? w : h);
  const double TWO_PI = 6.283185307179586;
  for (int i = 0; i < DS_SCENE_NSIN; i++) {
    const double f = 0.5 + 7.5 * uni();
    const double th = TWO_PI * uni();
    s->sin_kx[i] = (float)(TWO_PI * f * cos(th) / L);
    s->sin_ky[i] = (float)(TWO_PI * f * sin(th) / L);
    s->sin_ph[i] = (float)(TWO_PI * uni());
    s->sin_amp[i] = (float)(0.01 + 0.05 * uni());
  }
  for (int j = 0; j < DS_SCENE_NEDGE; j++) {
    const int t = j / 10;
    s->edge_type[j] = t;
    const double u = uni();
    s->edge_pos[j] = t == 0 ? (int)(u * w) : t == 1 ? (int)(u * h) : t == 2 ? (int)(u * (w + h)) : (int)(u * (w + h)) - h;
    const double mag = 0.02 + 0.05 * uni();
    const double sgn = uni() < 0.5 ? -1.0 : 1.0;
    for (int c = 0; c < 3; c++) s->edge_h[j][c] = (float)(sgn * mag + 0.02 * (uni() - 0.5));
  }
}
