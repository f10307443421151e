"""darkslide_b200 — B200-native RCD demosaic + NLM denoise.

A drop-in for darkslide-core's raw-develop detail path. This module mirrors
the reference's stage API (crates/core, Rust) over the C ABI of libdsgpu.so:

  CfaPattern, CfaImage      decode.rs:16-56
  Plane, Image3             image.rs:7-21
  Quality                   demosaic.rs:9-15
  demosaic(cfa, mul, q)     demosaic.rs:20-27  -> (Image3, Plane)
  rcd_bayer / mhc_bayer     demosaic.rs:147 / :90
  clip_plane                demosaic.rs:31
  box_blur(p, r)            image.rs:269
  nlm(p, h, search, patch)  enhance.rs:36
  normalize_u16             decode.rs:292-306 (integer raws)
  develop_u16               the three steps above in one device pass
  estimate_noise            enhance.rs:10-32
  guided_filter             image.rs:385-405
  denoise(img, amount)      enhance.rs:75-92 (Oklab, NLM on L, guided chroma)
  Oklab                     color.rs:380-419 (matrices)

Buffers may be numpy arrays (host memory: the call stages them through the
device) or CUDA torch tensors (device memory: the call is ordered on torch's
current stream). All arithmetic runs in the CUDA kernels; there is no CPU
path.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import Context, DsgpuError, SceneDesc, default_context, lib

__all__ = [
    "CfaPattern", "CfaImage", "Plane", "Image3", "Quality", "demosaic", "rcd_bayer", "mhc_bayer", "clip_plane",
    "box_blur", "nlm", "normalize_u16", "develop_u16", "cfa_clip_levels", "reconstruct_highlights", "apply_orientation", "BatchFrame", "develop_batch", "batch_frame_ms",
    "autotune", "autotune_get", "autotune_set", "estimate_noise", "guided_filter", "denoise", "Oklab", "Context", "DsgpuError", "default_context", "Scene",
    "RGGB", "BGGR", "GRBG", "GBRG",
]


@dataclass
class CfaPattern:
    """Repeating colour filter pattern; colours 0=R 1=G 2=B (decode.rs:16-47)."""

    width: int = 2
    height: int = 2
    colors: list = field(default_factory=lambda: [0, 1, 1, 2])

    def color_at(self, x: int, y: int) -> int:
        return int(self.colors[(y % self.height) * self.width + (x % self.width)])

    def is_bayer(self) -> bool:
        return self.width == 2 and self.height == 2

    def is_xtrans(self) -> bool:
        return self.width == 6 and self.height == 6

    def shifted(self, dx: int, dy: int) -> "CfaPattern":
        cols = [self.color_at(x + dx, y + dy) for y in range(self.height) for x in range(self.width)]
        return CfaPattern(self.width, self.height, cols)

    def codes(self) -> np.ndarray:
        if not self.is_bayer():
            raise DsgpuError(_lib.DSGPU_ERR_UNSUPPORTED, "CfaPattern", "only 2x2 Bayer patterns are on this path")
        return np.asarray(self.colors, dtype=np.uint8)


RGGB = CfaPattern(2, 2, [0, 1, 1, 2])
BGGR = CfaPattern(2, 2, [2, 1, 1, 0])
GRBG = CfaPattern(2, 2, [1, 0, 2, 1])
GBRG = CfaPattern(2, 2, [1, 2, 0, 1])


@dataclass
class CfaImage:
    """Mosaiced sensor data, black-subtracted and scaled so 1.0 = clipping (decode.rs:49-56)."""

    w: int
    h: int
    data: object  # (h, w) float32: numpy array or CUDA tensor
    pattern: CfaPattern


@dataclass
class Plane:
    """Single channel f32 image (image.rs:15-21); data is (h, w)."""

    w: int
    h: int
    data: object


@dataclass
class Image3:
    """Interleaved RGB f32 image (image.rs:7-13); data is (h, w, 3)."""

    w: int
    h: int
    data: object

    def channel(self, c: int) -> Plane:
        return Plane(self.w, self.h, self.data[..., c].copy() if isinstance(self.data, np.ndarray)
                     else self.data[..., c].contiguous())


class Quality(enum.IntEnum):
    DRAFT = _lib.DSGPU_QUALITY_DRAFT
    FULL = _lib.DSGPU_QUALITY_FULL


# ------------------------------------------------------------------ buffers
def _is_torch(x) -> bool:
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


class _Call:
    """Resolves the buffers of one call: host numpy arrays (DSGPU_HOST) or
    CUDA tensors (device pointers ordered on torch's current stream)."""

    def __init__(self, ref, ctx: Context | None):
        self.torch = _is_torch(ref)
        if self.torch:
            import torch
            if not ref.is_cuda:
                raise DsgpuError(_lib.DSGPU_ERR_ARG, "darkslide_b200", "torch tensors must be on a CUDA device")
            dev = ref.device.index if ref.device.index is not None else torch.cuda.current_device()
            self.ctx = ctx or default_context(dev)
            self.ctx.set_stream(torch.cuda.current_stream(ref.device).cuda_stream)
            self.flags = _lib.DSGPU_ASYNC
            self.device = ref.device
        else:
            self.ctx = ctx or default_context(0)
            self.flags = _lib.DSGPU_HOST

    def inp(self, x, dtype):
        if self.torch:
            import torch
            tdt = {np.float32: torch.float32, np.uint16: torch.uint16}[dtype]
            if x.dtype != tdt:
                raise DsgpuError(_lib.DSGPU_ERR_ARG, "darkslide_b200", f"expected {tdt}, got {x.dtype}")
            x = x.contiguous()
            return x, ctypes.c_void_p(x.data_ptr())
        a = np.ascontiguousarray(x, dtype=dtype)
        return a, a.ctypes.data_as(ctypes.c_void_p)

    def out(self, shape, dtype=np.float32):
        if self.torch:
            import torch
            t = torch.empty(shape, dtype=torch.float32, device=self.device)
            return t, ctypes.c_void_p(t.data_ptr())
        a = np.empty(shape, dtype=dtype)
        return a, a.ctypes.data_as(ctypes.c_void_p)


def _f3(v) -> np.ndarray:
    a = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float32), (3,)))
    return a


def _vp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------- stage functions
def normalize_u16(raw, pattern: CfaPattern, black: float, white, ctx: Context | None = None) -> CfaImage:
    """decode.rs:292-306: (raw - black) / max(white[c] - black, 1) per site."""
    c = _Call(raw, ctx)
    h, w = raw.shape
    src, p = c.inp(raw, np.uint16)
    out, po = c.out((h, w))
    pat = pattern.codes()
    wh = _f3(white)
    c.ctx.check(lib().dsgpu_normalize_u16(c.ctx.handle, p, w, h, w, _vp(pat), float(black), _vp(wh), po, c.flags),
                "dsgpu_normalize_u16")
    return CfaImage(w, h, out, pattern)


def clip_plane(cfa: CfaImage, ctx: Context | None = None) -> Plane:
    """demosaic.rs:31-42."""
    c = _Call(cfa.data, ctx)
    src, p = c.inp(cfa.data, np.float32)
    out, po = c.out((cfa.h, cfa.w))
    c.ctx.check(lib().dsgpu_clip_plane(c.ctx.handle, p, cfa.w, cfa.h, po, c.flags), "dsgpu_clip_plane")
    return Plane(cfa.w, cfa.h, out)


def mhc_bayer(cfa: CfaImage, mul, ctx: Context | None = None) -> Image3:
    """demosaic.rs:90-124."""
    c = _Call(cfa.data, ctx)
    src, p = c.inp(cfa.data, np.float32)
    out, po = c.out((cfa.h, cfa.w, 3))
    pat, m = cfa.pattern.codes(), _f3(mul)
    c.ctx.check(lib().dsgpu_mhc(c.ctx.handle, p, cfa.w, cfa.h, _vp(pat), _vp(m), po, c.flags), "dsgpu_mhc")
    return Image3(cfa.w, cfa.h, out)


def rcd_bayer(cfa: CfaImage, mul, ctx: Context | None = None) -> Image3:
    """demosaic.rs:147-344 (MHC when w or h < 16)."""
    c = _Call(cfa.data, ctx)
    src, p = c.inp(cfa.data, np.float32)
    out, po = c.out((cfa.h, cfa.w, 3))
    pat, m = cfa.pattern.codes(), _f3(mul)
    c.ctx.check(lib().dsgpu_rcd(c.ctx.handle, p, cfa.w, cfa.h, _vp(pat), _vp(m), po, c.flags), "dsgpu_rcd")
    return Image3(cfa.w, cfa.h, out)


def demosaic(cfa: CfaImage, mul, quality: Quality = Quality.FULL, ctx: Context | None = None):
    """demosaic.rs:20-27 for a Bayer pattern: returns (Image3, clip Plane)."""
    if not cfa.pattern.is_bayer():
        raise DsgpuError(_lib.DSGPU_ERR_UNSUPPORTED, "demosaic", "X-Trans demosaic is not on this path")
    c = _Call(cfa.data, ctx)
    src, p = c.inp(cfa.data, np.float32)
    ow, oh = (cfa.w, cfa.h) if quality == Quality.FULL else (cfa.w // 2, cfa.h // 2)
    rgb, pr = c.out((oh, ow, 3))
    clip, pc = c.out((oh, ow))
    pat, m = cfa.pattern.codes(), _f3(mul)
    c.ctx.check(lib().dsgpu_demosaic(c.ctx.handle, p, cfa.w, cfa.h, _vp(pat), _vp(m), int(quality), pr, pc, c.flags),
                "dsgpu_demosaic")
    return Image3(ow, oh, rgb), Plane(ow, oh, clip)


def box_blur(p: Plane, r: int, ctx: Context | None = None) -> Plane:
    """image.rs:269-313."""
    c = _Call(p.data, ctx)
    src, pi = c.inp(p.data, np.float32)
    out, po = c.out((p.h, p.w))
    c.ctx.check(lib().dsgpu_box_blur(c.ctx.handle, pi, p.w, p.h, int(r), po, c.flags), "dsgpu_box_blur")
    return Plane(p.w, p.h, out)


def nlm(p, h_param: float, search: int, patch: int, ctx: Context | None = None, fp16_staging: bool = False):
    """enhance.rs:36-72. ``p`` is a Plane, or an Image3 denoised per channel.
    ``fp16_staging``: the precision variant (DSGPU_FP16_STAGING)."""
    chans = 3 if isinstance(p, Image3) else 1
    c = _Call(p.data, ctx)
    src, pi = c.inp(p.data, np.float32)
    shape = (p.h, p.w, 3) if chans == 3 else (p.h, p.w)
    out, po = c.out(shape)
    c.ctx.check(lib().dsgpu_nlm(c.ctx.handle, pi, p.w, p.h, chans, float(h_param), int(search), int(patch), po,
                                c.flags | (_lib.DSGPU_FP16_STAGING if fp16_staging else 0)), "dsgpu_nlm")
    return Image3(p.w, p.h, out) if chans == 3 else Plane(p.w, p.h, out)


def cfa_clip_levels(cfa: "CfaImage", ctx: Context | None = None) -> np.ndarray:
    """demosaic.rs:419-430: per-colour clip level of a normalised mosaic
    (float32 max where the maximum stays below 0.95)."""
    c = _Call(cfa.data, ctx)
    _, p = c.inp(cfa.data, np.float32)
    out = np.empty(3, np.float32)
    pat = cfa.pattern.codes()
    c.ctx.check(lib().dsgpu_cfa_clip_levels(c.ctx.handle, p, cfa.w, cfa.h, _vp(pat),
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), c.flags),
                "dsgpu_cfa_clip_levels")
    return out


def reconstruct_highlights(img: "Image3", clip: "Plane", mul, raw_clip, ctx: Context | None = None) -> "Image3":
    """demosaic.rs:435-502 on a copy of img (Image3); clip is the demosaic's
    clip Plane, raw_clip the levels of cfa_clip_levels."""
    c = _Call(img.data, ctx)
    if c.torch:
        data = img.data.contiguous().clone()
        pi = ctypes.c_void_p(data.data_ptr())
        _, pc = c.inp(clip.data, np.float32)
    else:
        data = np.array(img.data, dtype=np.float32, order="C", copy=True)
        pi = data.ctypes.data_as(ctypes.c_void_p)
        _, pc = c.inp(clip.data, np.float32)
    m, rc = _f3(mul), np.ascontiguousarray(raw_clip, np.float32)
    c.ctx.check(lib().dsgpu_reconstruct_highlights(c.ctx.handle, pi, pc, img.w, img.h, _vp(m), _vp(rc), c.flags),
                "dsgpu_reconstruct_highlights")
    return Image3(img.w, img.h, data)


def apply_orientation(img: "Image3", orientation: int, ctx: Context | None = None) -> "Image3":
    """decode.rs:414-426: the image in EXIF orientation 1-8 (5-8 swap w and h)."""
    c = _Call(img.data, ctx)
    _, pi = c.inp(img.data, np.float32)
    swap = 5 <= int(orientation) <= 8
    ow, oh = (img.h, img.w) if swap else (img.w, img.h)
    out, po = c.out((oh, ow, 3))
    c.ctx.check(lib().dsgpu_apply_orientation(c.ctx.handle, pi, img.w, img.h, int(orientation), po, c.flags),
                "dsgpu_apply_orientation")
    return Image3(ow, oh, out)


@dataclass
class BatchFrame:
    """One frame of develop_batch: a CUDA uint16 tensor (h, w), its CFA
    pattern, levels, white balance and NLM strength; `out` (h, w, 3) and
    optional `clip` (h, w) float32 CUDA tensors receive the result.
    `black_pattern` (optional, (bh, bw) up to 4 x 4) gives per-site black
    levels at uncropped coordinates, `black_origin` the frame's crop origin
    (load_raw's black_at); without it the scalar `black` applies."""
    raw: object
    pattern: "CfaPattern"
    black: float
    white: object
    mul: object
    h_param: float
    out: object
    clip: object = None
    black_pattern: object = None
    black_origin: tuple = (0, 0)


def develop_batch(frames, search: int, patch: int, ctx: Context | None = None, sync: bool = True) -> None:
    """u16 raw -> normalise -> RCD -> NLM for many frames (different sizes,
    CFA layouts, levels and strengths) in one CUDA graph launch
    (dsgpu_rcd_nlm_batch). Work goes on torch's current stream."""
    import torch

    frames = list(frames)
    dev = frames[0].raw.device
    cx = ctx or default_context(dev.index or 0)
    cx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    arr = (_lib.Frame * len(frames))()
    keep = []  # black patterns, alive for the call
    for d, f in zip(arr, frames):
        h, w = f.raw.shape
        d.raw = f.raw.data_ptr()
        d.pitch_elems = f.raw.stride(0)
        d.w, d.h = w, h
        d.cfa[:] = [int(v) for v in f.pattern.codes()]
        d.black = float(f.black)
        d.white[:] = [float(v) for v in _f3(f.white)]
        d.mul[:] = [float(v) for v in _f3(f.mul)]
        d.h_param = float(f.h_param)
        d.out_rgb = f.out.data_ptr()
        d.out_clip = f.clip.data_ptr() if f.clip is not None else None
        if f.black_pattern is not None:
            bp = np.ascontiguousarray(np.asarray(f.black_pattern, np.float32))
            if bp.ndim != 2:
                raise DsgpuError(_lib.DSGPU_ERR_ARG, "develop_batch", "black_pattern must be a (bh, bw) array")
            keep.append(bp)
            d.black_pattern = bp.ctypes.data
            d.black_h, d.black_w = bp.shape
            d.black_x0, d.black_y0 = int(f.black_origin[0]), int(f.black_origin[1])
    flags = 0 if sync else _lib.DSGPU_ASYNC
    cx.check(lib().dsgpu_rcd_nlm_batch(cx.handle, arr, len(frames), int(search), int(patch), flags),
             "dsgpu_rcd_nlm_batch")


def batch_frame_ms(n: int, ctx: Context | None = None) -> np.ndarray:
    """Completion time (ms after the batch started on the device) of each of
    the first n frames of the last develop_batch."""
    cx = ctx or default_context(0)
    out = np.zeros(n, np.float64)
    cx.check(lib().dsgpu_batch_frame_ms(cx.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n),
             "dsgpu_batch_frame_ms")
    return out


def autotune(sizes, search: int, patch: int, ctx: Context | None = None) -> None:
    """Tune the batched kernels for each (w, h) size class (dsgpu_autotune)."""
    cx = ctx or default_context(0)
    flat = np.ascontiguousarray(np.asarray(sizes, np.int32).reshape(-1))
    cx.check(lib().dsgpu_autotune(cx.handle, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), flat.size // 2,
                                  int(search), int(patch)), "dsgpu_autotune")


def autotune_get(w: int, h: int, ctx: Context | None = None) -> dict:
    """The table entry used for a w x h frame: RCD tile shape, NLM CTAs per
    SM and (exact classes) the tuned RCD time of every shape."""
    cx = ctx or default_context(0)
    tw, th, k = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    ms = (ctypes.c_double * 5)()
    cx.check(lib().dsgpu_autotune_get(cx.handle, int(w), int(h), ctypes.byref(tw), ctypes.byref(th),
                                      ctypes.byref(k), ms), "dsgpu_autotune_get")
    return {"rcd_tile": (tw.value, th.value), "nlm_ctas_per_sm": k.value, "rcd_ms": list(ms)}


def autotune_set(w: int, h: int, rcd_tile, nlm_ctas_per_sm: int, ctx: Context | None = None) -> None:
    cx = ctx or default_context(0)
    cx.check(lib().dsgpu_autotune_set(cx.handle, int(w), int(h), int(rcd_tile[0]), int(rcd_tile[1]),
                                      int(nlm_ctas_per_sm)), "dsgpu_autotune_set")


def develop_u16(raw, pattern: CfaPattern, black: float, white, mul, h_param: float, search: int, patch: int,
                with_clip: bool = False, ctx: Context | None = None, fp16_staging: bool = False,
                highlights: bool = False):
    """u16 raw -> normalise -> RCD -> per-channel NLM in one device pass.
    Returns the denoised Image3 (and the clip Plane when ``with_clip``).
    ``fp16_staging``: NLM's precision variant (DSGPU_FP16_STAGING);
    ``highlights``: reconstruct highlights between RCD and NLM (DSGPU_HIGHLIGHTS)."""
    c = _Call(raw, ctx)
    h, w = raw.shape
    src, p = c.inp(raw, np.uint16)
    rgb, pr = c.out((h, w, 3))
    clip, pc = c.out((h, w)) if with_clip else (None, ctypes.c_void_p(0))
    pat, wh, m = pattern.codes(), _f3(white), _f3(mul)
    c.ctx.check(lib().dsgpu_develop_u16(c.ctx.handle, p, w, h, w, _vp(pat), float(black), _vp(wh), _vp(m),
                                        float(h_param), int(search), int(patch), pr, pc,
                                        c.flags | (_lib.DSGPU_FP16_STAGING if fp16_staging else 0)
                                        | (_lib.DSGPU_HIGHLIGHTS if highlights else 0)),
                "dsgpu_develop_u16")
    img = Image3(w, h, rgb)
    return (img, Plane(w, h, clip)) if with_clip else img


def estimate_noise(p: Plane, ctx: Context | None = None) -> float:
    """enhance.rs:10-32: robust noise sigma (MAD of a Laplacian high pass)."""
    c = _Call(p.data, ctx)
    src, pi = c.inp(p.data, np.float32)
    sig = ctypes.c_float()
    c.ctx.check(lib().dsgpu_estimate_noise(c.ctx.handle, pi, p.w, p.h, ctypes.byref(sig), c.flags & _lib.DSGPU_HOST),
                "dsgpu_estimate_noise")
    return float(sig.value)


def guided_filter(i: Plane, p: Plane, r: int, eps: float, ctx: Context | None = None) -> Plane:
    """image.rs:385-405."""
    c = _Call(i.data, ctx)
    _, pI = c.inp(i.data, np.float32)
    _, pP = c.inp(p.data, np.float32)
    out, po = c.out((i.h, i.w))
    c.ctx.check(lib().dsgpu_guided_filter(c.ctx.handle, pI, pP, i.w, i.h, int(r), float(eps), po, c.flags),
                "dsgpu_guided_filter")
    return Plane(i.w, i.h, out)


def denoise(img: Image3, amount: float, ctx: Context | None = None) -> Image3:
    """enhance.rs:75-92: Oklab L through NLM (3, 1), chroma through guided filters."""
    c = _Call(img.data, ctx)
    _, pi = c.inp(img.data, np.float32)
    out, po = c.out((img.h, img.w, 3))
    c.ctx.check(lib().dsgpu_denoise(c.ctx.handle, pi, img.w, img.h, float(amount), po, c.flags), "dsgpu_denoise")
    return Image3(img.w, img.h, out)


class Oklab:
    """Oklab::new() of color.rs:394-399 (matrices computed by the library)."""

    def __init__(self):
        m = np.empty(27, np.float32)
        st = lib().dsgpu_oklab_matrices(_vp(m))
        if st != 0:
            raise DsgpuError(st, "dsgpu_oklab_matrices")
        self.to_lms, self.from_lms, self.m2_inv = m.reshape(3, 3, 3)


# ------------------------------------------------------------ synthetic input
@dataclass
class Scene:
    """Seeded synthetic Bayer mosaic (include/dsgpu_scene.h)."""

    seed: int
    w: int
    h: int
    pattern: CfaPattern = field(default_factory=lambda: RGGB)
    black: int = 512
    white: int = 16383
    gain: float = 0.5
    read_sigma: float = 6.0

    def desc(self) -> SceneDesc:
        d = SceneDesc()
        d.seed, d.w, d.h = int(self.seed), int(self.w), int(self.h)
        for i, v in enumerate(self.pattern.codes()):
            d.cfa[i] = int(v)
        d.black, d.white = int(self.black), int(self.white)
        d.gain_e_per_dn, d.read_sigma_dn = float(self.gain), float(self.read_sigma)
        return d

    def render_host(self, x0: int = 0, y0: int = 0, cw: int | None = None, ch: int | None = None) -> np.ndarray:
        cw = self.w - x0 if cw is None else cw
        ch = self.h - y0 if ch is None else ch
        out = np.empty((ch, cw), np.uint16)
        d = self.desc()
        st = lib().dsgpu_scene_render_host(ctypes.byref(d), x0, y0, cw, ch, _vp(out))
        if st != 0:
            raise DsgpuError(st, "dsgpu_scene_render_host")
        return out

    def truth_host(self, x0: int = 0, y0: int = 0, cw: int | None = None, ch: int | None = None) -> np.ndarray:
        cw = self.w - x0 if cw is None else cw
        ch = self.h - y0 if ch is None else ch
        out = np.empty((ch, cw, 3), np.float32)
        d = self.desc()
        st = lib().dsgpu_scene_truth_host(ctypes.byref(d), x0, y0, cw, ch, _vp(out))
        if st != 0:
            raise DsgpuError(st, "dsgpu_scene_truth_host")
        return out

    def render(self, device=None, ctx: Context | None = None, window=None):
        """GPU render into a CUDA uint16 tensor: the whole frame (h, w), or
        window = (x0, y0, cw, ch), that crop of it (ch, cw)."""
        import torch
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        cx = ctx or default_context(dev.index or 0)
        cx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        d = self.desc()
        if window is None:
            t = torch.empty((self.h, self.w), dtype=torch.uint16, device=dev)
            cx.check(lib().dsgpu_scene_render(cx.handle, ctypes.byref(d), ctypes.c_void_p(t.data_ptr()), 0),
                     "dsgpu_scene_render")
            return t
        x0, y0, cw, ch = (int(v) for v in window)
        t = torch.empty((ch, cw), dtype=torch.uint16, device=dev)
        cx.check(lib().dsgpu_scene_render_window(cx.handle, ctypes.byref(d), x0, y0, cw, ch,
                                                 ctypes.c_void_p(t.data_ptr()), 0), "dsgpu_scene_render_window")
        return t

    def sigma_norm(self, level: float = 0.5) -> float:
        """Noise sigma in normalised units at scene level `level` (green)."""
        rng = self.white - self.black
        dn = level * rng
        var = dn / self.gain + self.read_sigma ** 2
        return float(np.sqrt(var) / rng)
