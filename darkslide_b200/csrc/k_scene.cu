// Synthetic mosaic renderers (device kernel and host loop) over scene.h.
// Compiled with -fmad=false and -Xcompiler -ffp-contract=off so that the
// device and host renders agree bit for bit.
#include <thread>
#include <vector>

#include "internal.cuh"
#include "scene.h"
#include "../../include/dsgpu_scene.h"

namespace {

// The window [x0, x0+cw) x [y0, y0+ch) of the frame into out (cw*ch).
__global__ void scene_kernel(ds_scene s, int x0, int y0, int cw, uint16_t* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= cw) return;
  out[(size_t)y * cw + x] = ds_scene_pixel(&s, x0 + x, y0 + y);
}

template <class F>
void parallel_rows(int n, F f) {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if ((unsigned)n < nt) nt = n > 0 ? (unsigned)n : 1u;
  std::vector<std::thread> ts;
  for (unsigned t = 0; t < nt; t++)
    ts.emplace_back([=] {
      for (int r = (int)t; r < n; r += (int)nt) f(r);
    });
  for (auto& t : ts) t.join();
}

}  // namespace

ds_scene ds_scene_make(const dsgpu_scene_desc* d) {
  ds_scene s;
  ds_scene_init(&s, d->seed, d->w, d->h, d->cfa, d->black, d->white, d->gain_e_per_dn, d->read_sigma_dn);
  return s;
}

cudaError_t ds_launch_scene_window(cudaStream_t st, const ds_scene& s, int x0, int y0, int cw, int ch,
                                   uint16_t* out) {
  if (cw <= 0 || ch <= 0) return cudaSuccess;
  dim3 grid((cw + 255) / 256, ch);
  scene_kernel<<<grid, 256, 0, st>>>(s, x0, y0, cw, out);
  return cudaGetLastError();
}

cudaError_t ds_launch_scene(cudaStream_t st, const ds_scene& s, uint16_t* out) {
  return ds_launch_scene_window(st, s, 0, 0, s.w, s.h, out);
}

void ds_scene_host(const ds_scene& s, int x0, int y0, int cw, int ch, uint16_t* out) {
  parallel_rows(ch, [&](int r) {
    for (int c = 0; c < cw; c++) out[(size_t)r * cw + c] = ds_scene_pixel(&s, x0 + c, y0 + r);
  });
}

void ds_scene_truth(const ds_scene& s, int x0, int y0, int cw, int ch, float* out) {
  parallel_rows(ch, [&](int r) {
    for (int c = 0; c < cw; c++)
      for (int k = 0; k < 3; k++)
        out[((size_t)r * cw + c) * 3 + k] = ds_mul(ds_scene_value(&s, x0 + c, y0 + r, k), s.ch_gain[k]);
  });
}
