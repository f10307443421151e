// Host-side colour matrices for Oklab, restating darkslide-core's
// color.rs:6-98 and :380-399: 3x3 products accumulate in f64 and round to f32
// (color.rs:15-23), inversion runs in f64 (color.rs:25-42), Bradford
// adaptation (color.rs:80-88), ProPhoto RGB -> XYZ(D50) from its primaries
// (color.rs:90-98, :129), and Oklab's LMS matrices (color.rs:382-399).
// Computed once on the host and passed to the kernels by value.
#pragma once
#include <cmath>
#include <cstring>

namespace dscolor {

typedef float M3[3][3];

inline void mul_mv(const M3 m, const float v[3], float o[3]) {
  o[0] = m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2];
  o[1] = m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2];
  o[2] = m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2];
}

inline void mul_mm(const M3 a, const M3 b, M3 o) {
  M3 t;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double acc = 0.0;
      for (int k = 0; k < 3; k++) acc += (double)a[i][k] * (double)b[k][j];
      t[i][j] = (float)acc;
    }
  std::memcpy(o, t, sizeof(M3));
}

inline void invert(const M3 mf, M3 o) {
  double m[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) m[i][j] = mf[i][j];
  const double det = m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                     m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                     m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if (std::fabs(det) < 1e-12) {
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) o[i][j] = i == j ? 1.0f : 0.0f;
    return;
  }
  const double v = 1.0 / det;
  const double r[3][3] = {
      {(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * v, (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * v,
       (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * v},
      {(m[1][2] * m[2][0] - m[1][0] * m[2][2]) * v, (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * v,
       (m[1][0] * m[0][2] - m[0][0] * m[1][2]) * v},
      {(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * v, (m[2][0] * m[0][1] - m[0][0] * m[2][1]) * v,
       (m[0][0] * m[1][1] - m[1][0] * m[0][1]) * v}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o[i][j] = (float)r[i][j];
}

inline void xy_to_xyz(const float xy[2], float o[3]) {
  const float x = xy[0], y = std::fmax(xy[1], 1e-6f);
  o[0] = x / y;
  o[1] = 1.0f;
  o[2] = (1.0f - x - y) / y;
}

inline void bradford(const float src[2], const float dst[2], M3 o) {
  const M3 B = {{0.8951f, 0.2664f, -0.1614f}, {-0.7502f, 1.7135f, 0.0367f}, {0.0389f, -0.0685f, 1.0296f}};
  float xs[3], xd[3], s[3], d[3];
  xy_to_xyz(src, xs);
  xy_to_xyz(dst, xd);
  mul_mv(B, xs, s);
  mul_mv(B, xd, d);
  const M3 scale = {{d[0] / s[0], 0.f, 0.f}, {0.f, d[1] / s[1], 0.f}, {0.f, 0.f, d[2] / s[2]}};
  M3 binv, t;
  invert(B, binv);
  mul_mm(scale, B, t);
  mul_mm(binv, t, o);
}

// Oklab::new() of color.rs:394-399: to_lms, from_lms = inv(to_lms), M2, inv(M2)
struct OklabMatrices {
  M3 to_lms, from_lms, m2, m2_inv;
};

inline OklabMatrices oklab_matrices() {
  const float D50[2] = {0.34567f, 0.35850f}, D65[2] = {0.31271f, 0.32902f};
  // ProPhoto primaries, white D50 (no adaptation step)
  const float pr_xy[2] = {0.734699f, 0.265301f}, pg_xy[2] = {0.159597f, 0.840403f}, pb_xy[2] = {0.036598f, 0.000105f};
  float pr[3], pg[3], pb[3], wv[3], sv[3];
  xy_to_xyz(pr_xy, pr);
  xy_to_xyz(pg_xy, pg);
  xy_to_xyz(pb_xy, pb);
  const M3 m = {{pr[0], pg[0], pb[0]}, {pr[1], pg[1], pb[1]}, {pr[2], pg[2], pb[2]}};
  M3 minv, pp;
  invert(m, minv);
  xy_to_xyz(D50, wv);
  mul_mv(minv, wv, sv);
  const M3 dg = {{sv[0], 0.f, 0.f}, {0.f, sv[1], 0.f}, {0.f, 0.f, sv[2]}};
  mul_mm(m, dg, pp);
  const M3 M1 = {{0.818933f, 0.36186674f, -0.12885971f},
                 {0.032984544f, 0.9293119f, 0.03614564f},
                 {0.0482003f, 0.26436627f, 0.6338517f}};
  const M3 M2 = {{0.21045426f, 0.7936178f, -0.004072047f},
                 {1.9779985f, -2.4285922f, 0.4505937f},
                 {0.025904037f, 0.78277177f, -0.80867577f}};
  OklabMatrices o;
  M3 brad, t;
  bradford(D50, D65, brad);
  mul_mm(brad, pp, t);
  mul_mm(M1, t, o.to_lms);
  invert(o.to_lms, o.from_lms);
  std::memcpy(o.m2, M2, sizeof(M3));
  invert(M2, o.m2_inv);
  return o;
}

}  // namespace dscolor
