// dsgpu_develop_u16_noalloc: the u16 -> RCD -> NLM path for callers that
// cannot allocate device memory.
//
// Some callers own every byte of device memory themselves (a pool or a
// framework's caching allocator that must not be bypassed), or call from a
// place where cudaMalloc is not allowed or would stall the device (a render
// worker with a latency budget). dsgpu_develop_u16 keeps its demosaiced
// intermediate in context scratch that it allocates on first use; this entry
// point instead uses one fixed array in the library's device image,
// g_develop_scratch below, so it allocates nothing.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds its DSGPU_NOALLOC_SCRATCH_BYTES until the process exits. In
// host code its name is only a host-side stand-in, not a device address, so
// the address is looked up with cudaGetSymbolAddress once per device (with
// that device current) on the first call made on that device, and cached.
//
// That first call should therefore come before any stream capture. The cache
// is keyed on the device's current CUDA context as well: if the process tears
// the primary context down (cudaDeviceReset) the module is loaded again at a
// new address, and the next call looks the address up again.
//
// All calls share the one array and it keeps the last call's contents. The
// path overwrites every byte it reads before reading it, so nothing needs
// clearing; but two calls whose work overlaps on the GPU (different streams,
// or different host threads) race on the array and must be serialised by the
// caller.
//
// Flags: DSGPU_ASYNC and DSGPU_FP16_STAGING are honoured exactly as
// dsgpu_develop_u16 honours them. DSGPU_HOST needs device staging buffers and
// DSGPU_HIGHLIGHTS needs highlight scratch (clip levels, blurred planes), so
// both are refused, and so is any unknown bit. Per-site black patterns
// (dsgpu_set_black_pattern) belong to a context, which this call does not
// have: the scalar `black` applies to every site.
#include <cuda.h>

#include <mutex>

#include "internal.cuh"

namespace {

constexpr int kMaxDevices = 64;
__device__ __align__(256) unsigned char g_develop_scratch[DSGPU_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};  // the context each cached address belongs to

// The calling thread's current context, through the runtime's driver entry
// point (the library does not link libcuda). Null if it cannot be read.
CUcontext current_context() {
  using GetCtx = CUresult (*)(CUcontext*);
  static GetCtx fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (GetCtx) nullptr;
    }
    return reinterpret_cast<GetCtx>(p);
  }();
  CUcontext c = nullptr;
  if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
  return c;
}

// Device address of g_develop_scratch on the current device, looked up once
// per device and context.
int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return DSGPU_ERR_NODEV;
  }
  // cudaGetDevice does not create the primary context; the symbol lookup
  // below does, so the context is read again after it.
  const CUcontext before = current_context();
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev] || !before || g_scratch_ctx[dev] != before) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_develop_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return DSGPU_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = current_context();
  }
  *out = g_scratch_addr[dev];
  return DSGPU_OK;
}

}  // namespace

extern "C" int dsgpu_develop_u16_noalloc(void* cuda_stream, const uint16_t* raw, int w, int h, size_t pitch,
                                         const uint8_t cfa[4], float black, const float white[3],
                                         const float mul[3], float h_param, int search, int patch, float* out_rgb,
                                         float* out_clip, unsigned flags) {
  if (flags & DSGPU_HOST) return DSGPU_ERR_ARG;  // host staging would need device buffers
  if (flags & DSGPU_HIGHLIGHTS) return DSGPU_ERR_UNSUPPORTED;  // highlight scratch is not in the array
  if (flags & ~(DSGPU_ASYNC | DSGPU_FP16_STAGING)) return DSGPU_ERR_ARG;
  if (w < 0 || h < 0) return DSGPU_ERR_ARG;
  if (w > DSGPU_MAX_DIM || h > DSGPU_MAX_DIM) return DSGPU_ERR_SIZE;
  if (!cfa) return DSGPU_ERR_ARG;
  ds_pat pat;
  pat.packed = 0;
  for (int i = 0; i < 4; i++) {
    if (cfa[i] > 2) return DSGPU_ERR_CFA;
    pat.packed |= (uint32_t)cfa[i] << (8 * i);
  }
  if (patch < 0 || patch > DSGPU_NLM_MAX_PATCH || search > DSGPU_NLM_MAX_SEARCH) return DSGPU_ERR_ARG;
  const size_t n = (size_t)w * h;
  if (n > (size_t)DSGPU_NOALLOC_MAX_PIXELS) return DSGPU_ERR_SIZE;
  if (n == 0) return DSGPU_OK;
  if (!raw || !out_rgb || !white || !mul || pitch < (size_t)w) return DSGPU_ERR_ARG;

  void* base = nullptr;
  int st = scratch_address(&base);
  if (st != DSGPU_OK) return st;
  // layout: [RGB intermediate: n*3 floats][normalised CFA: n floats]
  float* mid = static_cast<float*>(base);
  float* cfa_f = mid + n * 3;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

  cudaError_t e;
  if (w < 16 || h < 16) {  // rcd_bayer falls back to MHC (demosaic.rs:149-151)
    if ((e = ds_launch_normalize_u16(s, raw, w, h, pitch, pat, black, white, cfa_f)) != cudaSuccess) goto fail;
    if ((e = ds_launch_mhc(s, cfa_f, w, h, pat, mul, mid)) != cudaSuccess) goto fail;
    if (out_clip && (e = ds_launch_clip_plane(s, cfa_f, w, h, out_clip)) != cudaSuccess) goto fail;
  } else {
    ds_src_u16 src{raw, pitch, black, {white[0], white[1], white[2]}};
    if ((e = ds_launch_rcd_u16(s, src, w, h, pat, mul, mid, out_clip)) != cudaSuccess) goto fail;
  }
  if (search < 0) {  // empty offset set: 0 / max(0, 1e-12) = 0 (enhance.rs:41, :71)
    if ((e = cudaMemsetAsync(out_rgb, 0, n * 3 * sizeof(float), s)) != cudaSuccess) goto fail;
  } else if ((e = ds_launch_nlm(s, mid, w, h, 3, h_param, search, patch, out_rgb,
                                (flags & DSGPU_FP16_STAGING) != 0)) != cudaSuccess) {
    goto fail;
  }
  if (!(flags & DSGPU_ASYNC) && (e = cudaStreamSynchronize(s)) != cudaSuccess) goto fail;
  return DSGPU_OK;
fail:
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? DSGPU_ERR_NOMEM : DSGPU_ERR_CUDA;
}
