// Internal declarations shared by the dsgpu translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/dsgpu.h"

// 2x2 Bayer pattern, colour code at (x, y) = c[(y & 1) * 2 + (x & 1)]
// (decode.rs:26-28 for a 2x2 pattern; the bit test also gives the right
// parity for the negative coordinates of out-of-image halo sites).
struct ds_pat {
  uint32_t packed;  // byte k = colour of pattern index k
  __host__ __device__ __forceinline__ int at(int x, int y) const {
    return (packed >> ((((y & 1) << 1) | (x & 1)) * 8)) & 0xFFu;
  }
};

// Where a demosaic kernel reads its CFA samples from.
struct ds_src_f32 {  // normalised float CFA (CfaImage::data)
  const float* data;
  int pitch;  // elements
};
constexpr int DS_BLACK_MAX = 4;  // black-level patterns of up to 4 x 4 sites
struct ds_src_u16 {  // integer raw + the normalisation of decode.rs:292-306
  const uint16_t* data;
  size_t pitch;  // elements
  float black;   // the black level of every site while bw == 0
  float white[3];
  // Per-site black levels (black_at, decode.rs:266-270): site (x, y) of the
  // frame takes bpat[((y + by0) % bh) * bw + (x + bx0) % bw], the pattern
  // being indexed at uncropped sensor coordinates (x + crop_x, y + crop_y).
  // bw == 0 (an aggregate initialisation that stops after `white`): `black`.
  int bw, bh, bx0, by0;
  float bpat[DS_BLACK_MAX * DS_BLACK_MAX];
};
__host__ __device__ __forceinline__ float ds_black_at(const ds_src_u16& s, int x, int y) {
  return s.bw ? s.bpat[((y + s.by0) % s.bh) * s.bw + (x + s.bx0) % s.bw] : s.black;
}

// One frame of a batched develop (u16 raw -> RCD -> NLM), as the batched
// kernels read it from device memory. Tiles of all frames are numbered
// consecutively: frame f owns RCD tiles [rcd_tile0, rcd_tile0 + rcd tiles)
// and NLM tiles [nlm_tile0, nlm_tile0 + nlm_tiles_x * nlm_tiles_y * 3).
struct ds_batch_frame {
  ds_src_u16 src;
  int w, h;
  ds_pat pat;
  float mul[3];
  float sigma;      // NLM pre-scale of the frame's strength h
  float* rgb;       // RCD output (scratch), w*h*3
  float* clip;      // clip plane or null
  float* out;       // NLM output, w*h*3
  int rcd_shape;    // index into the RCD tile shapes (ds_rcd_batch_shape)
  int rcd_tiles_x;
  int rcd_tiles;    // RCD tiles of this frame
  int rcd_tile0;
  int nlm_tiles_x, nlm_tiles_y;
  int nlm_tile0;
};

// A run of work items of the fused batch kernel: the RCD (kind 0) or NLM
// (kind 1) tiles of one frame, items [start, next segment's start).
struct ds_batch_seg {
  int kind, frame, start;
};
// Counters of the fused kernel: [0] next work item, [1] status, then the
// RCD and NLM tiles finished per frame.
constexpr int DS_BATCH_CTR_RCD = 2;
inline int ds_batch_ctr_nlm(int max_frames) { return DS_BATCH_CTR_RCD + max_frames; }
cudaError_t ds_launch_batch_fused(cudaStream_t st, const ds_batch_frame* frames, int n, const ds_batch_seg* segs,
                                  int nseg, int total_items, int search, int patch, int grid, int* counters,
                                  int max_frames, unsigned long long* stamps);

// batched kernels: one persistent launch each over all frames' tiles
constexpr int DS_RCD_SHAPES = 5;
void ds_rcd_batch_shape(int s, int* tile_w, int* tile_h);
cudaError_t ds_launch_rcd_batch(cudaStream_t st, const ds_batch_frame* frames, int n, int total_tiles, int grid);
cudaError_t ds_launch_nlm_batch(cudaStream_t st, const ds_batch_frame* frames, int n, int total_tiles, int search,
                                int patch, int grid, unsigned* done, unsigned long long* stamps);
cudaError_t ds_launch_stamp(cudaStream_t st, unsigned long long* t);
float ds_nlm_sigma(float h_param, int patch);

// kernel launchers (return cudaGetLastError() of the launch)
cudaError_t ds_launch_normalize_u16(cudaStream_t st, const uint16_t* raw, int w, int h, size_t pitch, ds_pat pat,
                                    float black, const float white[3], float* out);
cudaError_t ds_launch_normalize_src(cudaStream_t st, const ds_src_u16& src, int w, int h, ds_pat pat, float* out);
cudaError_t ds_launch_clip_plane(cudaStream_t st, const float* cfa, int w, int h, float* out);
cudaError_t ds_launch_mhc(cudaStream_t st, const float* cfa, int w, int h, ds_pat pat, const float mul[3],
                          float* out_rgb);
cudaError_t ds_launch_rcd_f32(cudaStream_t st, ds_src_f32 src, int w, int h, ds_pat pat, const float mul[3],
                              float* out_rgb, float* out_clip);
cudaError_t ds_launch_rcd_u16(cudaStream_t st, ds_src_u16 src, int w, int h, ds_pat pat, const float mul[3],
                              float* out_rgb, float* out_clip);
constexpr int DS_RCD_TILE = 40;  // rows of a tile row of the one-frame RCD kernel (tiles are 64 x 40)
constexpr int DS_RCD_HALO = 10;  // rows (and columns) of input beyond a tile that RCD reads
cudaError_t ds_launch_rcd_u16_rows(cudaStream_t st, ds_src_u16 src, int w, int h, ds_pat pat, const float mul[3],
                                   float* out_rgb, float* out_clip, int ty0, int ty1);
cudaError_t ds_launch_superpixel(cudaStream_t st, const float* cfa, int w, int h, ds_pat pat, const float mul[3],
                                 float* out_rgb, float* out_clip);
cudaError_t ds_launch_box_blur(cudaStream_t st, const float* in, int w, int h, int r, float* tmp, float* out);
// highlight reconstruction (demosaic.rs:419-502)
void ds_box_radii_for_gauss(float sigma, int n, int* radii);
cudaError_t ds_launch_clip_levels_f32(cudaStream_t st, const float* cfa, int w, int h, ds_pat pat, unsigned* bits,
                                      float* raw_clip);
cudaError_t ds_launch_clip_levels_u16(cudaStream_t st, ds_src_u16 src, int w, int h, ds_pat pat, unsigned* bits,
                                      float* raw_clip);
size_t ds_highlights_scratch_bytes(int w, int h);
cudaError_t ds_launch_orientation(cudaStream_t st, const float* in, int w, int h, int orientation, float* out);
cudaError_t ds_launch_highlights(cudaStream_t st, float* img, const float* clip, int w, int h, const float mul[3],
                                 const float* raw_clip, void* scratch, unsigned* launches);
// fp16_staging: the precision variant (plane staged in half precision,
// sums in FP32 with a compensated weight sum); see k_nlm.cu
cudaError_t ds_launch_nlm(cudaStream_t st, const float* in, int w, int h, int channels, float h_param, int search,
                          int patch, float* out, bool fp16_staging = false);
cudaError_t ds_launch_nlm_dev_h(cudaStream_t st, const float* in, int w, int h, int channels, const float* h_dev,
                                int search, int patch, float* out);
void ds_nlm_tile_grid(int w, int h, int patch, int* tiles_x, int* tiles_y, int* tile_w, int* tile_h);
cudaError_t ds_launch_nlm_rows(cudaStream_t st, const float* in, int w, int h, int channels, float h_param,
                               int search, int patch, int ty0, int ty1, float* out, bool fp16_staging);
cudaError_t ds_launch_nlm_tiles(cudaStream_t st, const float* in, int w, int h, int channels, float h_param,
                                int search, int patch, const unsigned char* flags, float* out);
cudaError_t ds_launch_nlm_tiles_rows(cudaStream_t st, const float* in, int w, int h, int channels, float h_param,
                                     int search, int patch, const unsigned char* flags, int ty0, int ty1,
                                     float* out);
// denoise composite (enhance.rs:75-92) and its parts
size_t ds_denoise_scratch_bytes(int w, int h);
size_t ds_noise_scratch_bytes(int w, int h);
cudaError_t ds_launch_estimate_noise(cudaStream_t st, const float* p, int w, int h, float k, void* scratch,
                                     float* out3);
cudaError_t ds_launch_guided_filter(cudaStream_t st, const float* I, const float* p, int w, int h, int r,
                                    const float* eps_dev, float eps_host, float* out, float* scratch,
                                    const float* mean_i, const float* mean_ii);
cudaError_t ds_launch_guide_means(cudaStream_t st, const float* I, int w, int h, int r, float* mean_i, float* mean_ii,
                                  float* tmp, float* tmp2);
cudaError_t ds_launch_denoise(cudaStream_t st, const float* rgb, int w, int h, float amount, void* scratch,
                              float* out, float* sigma_dev_out, unsigned* launches);
void ds_oklab_matrices(float out[27]);
