"""ctypes wrapper of the CPU oracle (libdsref.so).

TEST INFRASTRUCTURE ONLY: the checker for the GPU library. Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference arm load
it. The GPU library never depends on it.

Each function restates darkslide-core's CPU code (see dsref.cpp for the
file:line of every routine). Parity with the Rust reference itself is
unpinned: the Rust toolchain is absent, and the reference's own tests are
property tests without golden vectors.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdsref.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile libdsref.so with the committed Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        i, f, d, sz = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
        L.dsref_omp_threads.restype = i
        L.dsref_set_threads.argtypes = [i]
        L.dsref_normalize_u16.argtypes = [_u16p, i, i, sz, _u8p, f, _f32p, _f32p]
        L.dsref_normalize_u16_bp.argtypes = [_u16p, i, i, sz, _u8p, _f32p, i, i, i, i, _f32p, _f32p]
        L.dsref_clip_plane_f32.argtypes = [_f32p, i, i, _f32p]
        L.dsref_mhc_f32.argtypes = [_f32p, i, i, _u8p, _f32p, _f32p]
        L.dsref_superpixel_f32.argtypes = [_f32p, i, i, _u8p, _f32p, _f32p, _f32p]
        L.dsref_rcd_f32.argtypes = [_f32p, i, i, _u8p, _f32p, _f32p]
        L.dsref_rcd_f64.argtypes = [_f32p, i, i, _u8p, _f32p, _f64p]
        L.dsref_box_blur_f32.argtypes = [_f32p, i, i, i, _f32p]
        L.dsref_box_blur_f64.argtypes = [_f64p, i, i, i, _f64p]
        L.dsref_nlm_f32.argtypes = [_f32p, i, i, f, i, i, i, _f32p]
        L.dsref_nlm_f64.argtypes = [_f64p, i, i, d, i, i, i, _f64p]
        L.dsref_cfa_clip_levels.argtypes = [_f32p, i, i, _u8p, _f32p]
        L.dsref_box_radii_for_gauss.argtypes = [f, i, np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")]
        L.dsref_reconstruct_highlights.argtypes = [_f32p, _f32p, i, i, _f32p, _f32p]
        L.dsref_estimate_noise_f32.argtypes = [_f32p, i, i]
        L.dsref_estimate_noise_f32.restype = f
        L.dsref_oklab_matrices.argtypes = [_f32p]
        L.dsref_oklab_from_prophoto.argtypes = [_f32p, i, _f32p]
        L.dsref_oklab_to_prophoto.argtypes = [_f32p, i, _f32p]
        L.dsref_guided_filter_f32.argtypes = [_f32p, _f32p, i, i, i, f, _f32p]
        L.dsref_denoise_f32.argtypes = [_f32p, i, i, f, i, _f32p, _f32p]
        u64 = ctypes.c_uint64
        L.dsref_scene_render.argtypes = [u64, i, i, _u8p, i, i, f, f, i, i, i, i, _u16p]
        L.dsref_scene_truth.argtypes = [u64, i, i, _u8p, i, i, f, f, i, i, i, i, _f32p]
        _lib = L
    return _lib


def threads() -> int:
    return lib().dsref_omp_threads()


def set_threads(n: int) -> None:
    lib().dsref_set_threads(int(n))


def _pat(cfa) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(cfa, dtype=np.uint8).reshape(4))


def normalize_u16(raw: np.ndarray, cfa, black: float, white) -> np.ndarray:
    """decode.rs:292-306. ``raw`` is (h, w) uint16; returns (h, w) float32."""
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    h, w = raw.shape
    out = np.empty((h, w), np.float32)
    wh = np.ascontiguousarray(np.broadcast_to(np.asarray(white, np.float32), (3,)))
    lib().dsref_normalize_u16(raw, w, h, w, _pat(cfa), float(black), wh, out)
    return out


def normalize_u16_bp(raw: np.ndarray, cfa, levels, origin, white) -> np.ndarray:
    """decode.rs:266-306 with a per-site black pattern ``levels`` (bh, bw),
    indexed at uncropped coordinates (x + origin[0], y + origin[1])."""
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    h, w = raw.shape
    lv = np.ascontiguousarray(np.asarray(levels, np.float32))
    bh, bw = lv.shape
    out = np.empty((h, w), np.float32)
    wh = np.ascontiguousarray(np.broadcast_to(np.asarray(white, np.float32), (3,)))
    lib().dsref_normalize_u16_bp(raw, w, h, w, _pat(cfa), lv.ravel(), bw, bh, int(origin[0]), int(origin[1]), wh, out)
    return out


def clip_plane(cfa_data: np.ndarray) -> np.ndarray:
    """demosaic.rs:31-42."""
    a = np.ascontiguousarray(cfa_data, dtype=np.float32)
    h, w = a.shape
    out = np.empty((h, w), np.float32)
    lib().dsref_clip_plane_f32(a, w, h, out)
    return out


def mhc(cfa_data: np.ndarray, cfa, mul) -> np.ndarray:
    """demosaic.rs:90-124; returns (h, w, 3) float32."""
    a = np.ascontiguousarray(cfa_data, dtype=np.float32)
    h, w = a.shape
    out = np.empty((h, w, 3), np.float32)
    lib().dsref_mhc_f32(a, w, h, _pat(cfa), np.ascontiguousarray(mul, np.float32), out)
    return out


def rcd(cfa_data: np.ndarray, cfa, mul, fp64: bool = False) -> np.ndarray:
    """demosaic.rs:147-344; returns (h, w, 3) float32 (float64 for the FP64 oracle)."""
    a = np.ascontiguousarray(cfa_data, dtype=np.float32)
    h, w = a.shape
    m = np.ascontiguousarray(mul, np.float32)
    if fp64:
        out = np.empty((h, w, 3), np.float64)
        lib().dsref_rcd_f64(a, w, h, _pat(cfa), m, out)
    else:
        out = np.empty((h, w, 3), np.float32)
        lib().dsref_rcd_f32(a, w, h, _pat(cfa), m, out)
    return out


def superpixel(cfa_data: np.ndarray, cfa, mul):
    """demosaic.rs:45-87 (Draft quality) for a Bayer pattern: (rgb, clip) at half size."""
    a = np.ascontiguousarray(cfa_data, dtype=np.float32)
    h, w = a.shape
    out = np.empty((h // 2, w // 2, 3), np.float32)
    clip = np.empty((h // 2, w // 2), np.float32)
    lib().dsref_superpixel_f32(a, w, h, _pat(cfa), np.ascontiguousarray(mul, np.float32), out, clip)
    return out, clip


def demosaic(cfa_data: np.ndarray, cfa, mul):
    """demosaic.rs:20-27 for Quality::Full on a Bayer pattern: (rgb, clip)."""
    return rcd(cfa_data, cfa, mul), clip_plane(cfa_data)


def box_blur(p: np.ndarray, r: int) -> np.ndarray:
    """image.rs:269-313."""
    if p.dtype == np.float64:
        a = np.ascontiguousarray(p)
        out = np.empty_like(a)
        lib().dsref_box_blur_f64(a, a.shape[1], a.shape[0], int(r), out)
        return out
    a = np.ascontiguousarray(p, dtype=np.float32)
    out = np.empty_like(a)
    lib().dsref_box_blur_f32(a, a.shape[1], a.shape[0], int(r), out)
    return out


def nlm(p: np.ndarray, h_param: float, search: int, patch: int, nthreads: int | None = None,
        fp64: bool = False) -> np.ndarray:
    """enhance.rs:36-72 on one plane. ``nthreads`` is the rayon pool size whose
    offset chunking is reproduced (defaults to this host's OpenMP thread count)."""
    nt = threads() if nthreads is None else int(nthreads)
    if fp64:
        a = np.ascontiguousarray(p, dtype=np.float64)
        out = np.empty_like(a)
        lib().dsref_nlm_f64(a, a.shape[1], a.shape[0], float(h_param), int(search), int(patch), nt, out)
        return out
    a = np.ascontiguousarray(p, dtype=np.float32)
    out = np.empty_like(a)
    lib().dsref_nlm_f32(a, a.shape[1], a.shape[0], float(h_param), int(search), int(patch), nt, out)
    return out


def nlm_rgb(img: np.ndarray, h_param: float, search: int, patch: int, nthreads: int | None = None,
            fp64: bool = False) -> np.ndarray:
    """Per-channel NLM of an interleaved (h, w, 3) image (image.rs:99-101 channel,
    enhance.rs:36 nlm, image.rs:380-382 merge3)."""
    return np.stack([nlm(img[..., c], h_param, search, patch, nthreads, fp64) for c in range(3)], axis=-1)


def estimate_noise(p: np.ndarray) -> float:
    """enhance.rs:10-32."""
    a = np.ascontiguousarray(p, dtype=np.float32)
    return float(lib().dsref_estimate_noise_f32(a, a.shape[1], a.shape[0]))


def oklab_matrices() -> np.ndarray:
    """(3, 3, 3): to_lms, from_lms, m2_inv of Oklab::new() (color.rs:395-398)."""
    out = np.empty(27, np.float32)
    lib().dsref_oklab_matrices(out)
    return out.reshape(3, 3, 3)


def oklab_from_prophoto(rgb: np.ndarray) -> np.ndarray:
    """color.rs:401-406 on an (..., 3) array."""
    a = np.ascontiguousarray(rgb, dtype=np.float32)
    out = np.empty_like(a)
    lib().dsref_oklab_from_prophoto(a, a.size // 3, out)
    return out


def oklab_to_prophoto(lab: np.ndarray) -> np.ndarray:
    """color.rs:408-412 on an (..., 3) array."""
    a = np.ascontiguousarray(lab, dtype=np.float32)
    out = np.empty_like(a)
    lib().dsref_oklab_to_prophoto(a, a.size // 3, out)
    return out


def guided_filter(I: np.ndarray, p: np.ndarray, r: int, eps: float) -> np.ndarray:
    """image.rs:385-405."""
    a = np.ascontiguousarray(I, dtype=np.float32)
    b = np.ascontiguousarray(p, dtype=np.float32)
    out = np.empty_like(a)
    lib().dsref_guided_filter_f32(a, b, a.shape[1], a.shape[0], int(r), float(eps), out)
    return out


def denoise(img: np.ndarray, amount: float, nthreads: int | None = None):
    """enhance.rs:75-92 on an (h, w, 3) image; returns (out, sigma)."""
    a = np.ascontiguousarray(img, dtype=np.float32)
    h, w, _ = a.shape
    out = np.empty_like(a)
    sig = np.zeros(1, np.float32)
    nt = threads() if nthreads is None else int(nthreads)
    lib().dsref_denoise_f32(a, w, h, float(amount), nt, out, sig)
    return out, float(sig[0])


def cfa_clip_levels(cfa_data: np.ndarray, cfa) -> np.ndarray:
    """demosaic.rs:419-430: per-colour clip level (FLT_MAX where untrusted)."""
    a = np.ascontiguousarray(cfa_data, dtype=np.float32)
    out = np.empty(3, np.float32)
    lib().dsref_cfa_clip_levels(a, a.shape[1], a.shape[0], _pat(cfa), out)
    return out


def box_radii_for_gauss(sigma: float, n: int = 3) -> list:
    """image.rs:363-373."""
    out = np.empty(n, np.int32)
    lib().dsref_box_radii_for_gauss(float(sigma), int(n), out)
    return [int(v) for v in out]


def reconstruct_highlights(img: np.ndarray, clip: np.ndarray, mul, raw_clip) -> np.ndarray:
    """demosaic.rs:435-502 on a copy of an interleaved (h, w, 3) image."""
    out = np.array(img, dtype=np.float32, order="C", copy=True)
    c = np.ascontiguousarray(clip, dtype=np.float32)
    lib().dsref_reconstruct_highlights(out, c, out.shape[1], out.shape[0], np.ascontiguousarray(mul, np.float32),
                                       np.ascontiguousarray(raw_clip, np.float32))
    return out


def apply_orientation(img: np.ndarray, o: int) -> np.ndarray:
    """decode.rs:414-426 on an (h, w, 3) array: output pixel (x, y) takes the
    source pixel the reference's match arm names."""
    h, w = img.shape[:2]
    if o in (5, 6, 7, 8):
        oh, ow = w, h
    else:
        oh, ow = h, w
    y, x = np.mgrid[0:oh, 0:ow]
    src = {2: (w - 1 - x, y), 3: (w - 1 - x, h - 1 - y), 4: (x, h - 1 - y), 5: (y, x), 6: (y, h - 1 - x),
           7: (w - 1 - y, h - 1 - x), 8: (w - 1 - y, x)}.get(o, (x, y))
    return img[src[1], src[0]]


def scene_render(seed: int, w: int, h: int, cfa, black: int, white: int, gain: float, read_sigma: float,
                 x0: int = 0, y0: int = 0, cw: int | None = None, ch: int | None = None) -> np.ndarray:
    """The seeded synthetic mosaic (the library's scene generator, compiled
    into this library from the same header): the cw x ch window at (x0, y0)
    of the w x h frame, u16. Equal to darkslide_b200.Scene(...).render_host."""
    cw = w - x0 if cw is None else cw
    ch = h - y0 if ch is None else ch
    out = np.empty((ch, cw), np.uint16)
    lib().dsref_scene_render(int(seed), w, h, _pat(cfa), int(black), int(white), float(gain), float(read_sigma),
                             x0, y0, cw, ch, out)
    return out


def scene_truth(seed: int, w: int, h: int, cfa, black: int, white: int, gain: float, read_sigma: float,
                x0: int = 0, y0: int = 0, cw: int | None = None, ch: int | None = None) -> np.ndarray:
    """Noise-free RGB of the same scene window (channel gains applied, no
    white balance); equal to darkslide_b200.Scene(...).truth_host."""
    cw = w - x0 if cw is None else cw
    ch = h - y0 if ch is None else ch
    out = np.empty((ch, cw, 3), np.float32)
    lib().dsref_scene_truth(int(seed), w, h, _pat(cfa), int(black), int(white), float(gain), float(read_sigma),
                            x0, y0, cw, ch, out)
    return out
