/* dsgpu_scene.h — seeded synthetic Bayer mosaics for tests and benchmarks.
 *
 * No counterpart in the reference: the reference's own inputs are camera
 * raws fetched from the network. This generator produces the workload the
 * benchmarks are quoted on: a sum of 8 smooth 2-D sinusoids and 40 step edges
 * (20 axis-aligned, 20 diagonal) with per-channel gains R 0.5, G 1.0, B 0.7,
 * sampled at the CFA sites, with Poisson-Gaussian noise (conversion gain
 * g e/DN, read noise sigma DN) on top of the black level, rounded and clamped
 * to [0, white]. The host and device renderers give identical mosaics.
 */
#ifndef DSGPU_SCENE_H
#define DSGPU_SCENE_H

#include <stdint.h>

#include "dsgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsgpu_scene_desc {
  uint64_t seed;
  int w, h;
  uint8_t cfa[4];
  int black, white;
  float gain_e_per_dn;
  float read_sigma_dn;
} dsgpu_scene_desc;

/* CPU render of the crop [x0, x0+cw) x [y0, y0+ch) of the frame into out (cw*ch u16). */
int dsgpu_scene_render_host(const dsgpu_scene_desc* d, int x0, int y0, int cw, int ch, uint16_t* out);

/* Noise-free normalised scene (value * channel gain, before white balance)
 * of the crop, interleaved RGB float (cw*ch*3). */
int dsgpu_scene_truth_host(const dsgpu_scene_desc* d, int x0, int y0, int cw, int ch, float* out_rgb);

/* GPU render of the whole frame (w*h u16) on the context stream. */
int dsgpu_scene_render(dsgpu_ctx* ctx, const dsgpu_scene_desc* d, uint16_t* out, unsigned flags);

/* GPU render of the crop [x0, x0+cw) x [y0, y0+ch) of the frame (cw*ch u16),
 * equal to the same window of the whole-frame render. */
int dsgpu_scene_render_window(dsgpu_ctx* ctx, const dsgpu_scene_desc* d, int x0, int y0, int cw, int ch,
                              uint16_t* out, unsigned flags);

#ifdef __cplusplus
}
#endif
#endif /* DSGPU_SCENE_H */
