"""dsgpu_develop_u16_noalloc: the detail path for callers that cannot
allocate device memory (they manage all device memory themselves, or call
where cudaMalloc is not allowed or would stall the device). It keeps its
intermediate in a fixed array inside the library instead of context
scratch. It launches the same kernels as dsgpu_develop_u16 on the same
inputs, so its output must equal dsgpu_develop_u16's bit for bit, call after
call, even though every call reuses the same array.

This file is collected last so that a run stopping at the first failure has
run every other test first."""
import ctypes

import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

pytestmark = pytest.mark.gpu

WB = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch


def _call(torch, which, raw, sc, h_param, search, patch, with_clip=True, flags=0):
    """One develop through the C ABI; returns (rgb, clip or None)."""
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    vp = ctypes.c_void_p
    w, h = sc.w, sc.h
    pat = sc.pattern.codes()
    white = np.full(3, sc.white, np.float32)
    rgb = torch.full((h, w, 3), float("nan"), dtype=torch.float32, device=dev)
    clip = torch.full((h, w), float("nan"), dtype=torch.float32, device=dev) if with_clip else None
    args = (vp(raw.data_ptr()), w, h, w, vp(pat.ctypes.data), float(sc.black), vp(white.ctypes.data),
            vp(WB.ctypes.data), float(h_param), search, patch, vp(rgb.data_ptr()),
            vp(clip.data_ptr() if clip is not None else 0), flags)
    if which == "ctx":
        ctx = ds.default_context(0)
        ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        ctx.check(L.dsgpu_develop_u16(ctx.handle, *args), "dsgpu_develop_u16")
    else:
        st = L.dsgpu_develop_u16_noalloc(vp(torch.cuda.current_stream(dev).cuda_stream), *args)
        assert st == 0, _lib.strerror(st)
    torch.cuda.synchronize()
    return rgb.cpu().numpy(), (clip.cpu().numpy() if clip is not None else None)


def _check_equal(torch, sc, h_param, search, patch, with_clip=True, flags=0):
    torch.cuda.set_device(0)
    raw = sc.render(torch.device("cuda", 0))
    a_rgb, a_clip = _call(torch, "ctx", raw, sc, h_param, search, patch, with_clip, flags)
    b_rgb, b_clip = _call(torch, "noalloc", raw, sc, h_param, search, patch, with_clip, flags)
    assert np.isfinite(b_rgb).all()
    np.testing.assert_array_equal(a_rgb, b_rgb)
    if with_clip:
        np.testing.assert_array_equal(a_clip, b_clip)
    return b_rgb


def test_noalloc_matches_allocating_entry_point_twice(torch_cuda):
    # two calls in a row on different frames: the second reuses the array
    # the first one left behind
    cases = [
        (ds.Scene(seed=1, w=1024, h=768, pattern=ds.RGGB, black=256, white=4095, gain=0.5, read_sigma=3), 0.08, 10, 3),
        (ds.Scene(seed=2, w=600, h=400, pattern=ds.GBRG, black=512, white=16383, gain=0.25, read_sigma=12), 0.03, 3, 1),
    ]
    for sc, h_param, search, patch in cases:
        _check_equal(torch_cuda, sc, h_param, search, patch)


def test_noalloc_same_frame_twice_is_identical(torch_cuda):
    sc = ds.Scene(seed=3, w=320, h=256, pattern=ds.BGGR, black=512, white=16383, gain=0.5, read_sigma=6)
    first = _check_equal(torch_cuda, sc, 0.02, 10, 3)
    second = _check_equal(torch_cuda, sc, 0.02, 10, 3)
    np.testing.assert_array_equal(first, second)


def test_noalloc_at_the_pixel_limit(torch_cuda):
    # exactly DSGPU_NOALLOC_MAX_PIXELS (1024 x 1024) is accepted
    sc = ds.Scene(seed=4, w=1024, h=1024, pattern=ds.GRBG, black=256, white=4095, gain=0.5, read_sigma=3)
    assert sc.w * sc.h == _lib.DSGPU_NOALLOC_MAX_PIXELS
    _check_equal(torch_cuda, sc, 0.08, 10, 3)


def test_noalloc_branches(torch_cuda):
    # frames under 16 px are MHC (demosaic.rs:149-151) through the array's
    # normalised-CFA part
    small = ds.Scene(seed=5, w=12, h=20, pattern=ds.RGGB, black=256, white=4095, gain=0.5, read_sigma=3)
    _check_equal(torch_cuda, small, 0.08, 10, 3)
    sc = ds.Scene(seed=6, w=200, h=150, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    _check_equal(torch_cuda, sc, 0.02, 10, 3, with_clip=False)  # no clip plane asked for
    zeros = _check_equal(torch_cuda, sc, 0.02, -1, 3)  # empty offset set: zeros (enhance.rs:41, :71)
    assert not zeros.any()
    _check_equal(torch_cuda, sc, 0.02, 0, 3)  # centre offset only: the demosaic itself
    _check_equal(torch_cuda, sc, 0.02, 10, 3, flags=_lib.DSGPU_FP16_STAGING)  # the precision variant


def test_noalloc_rejects_what_it_cannot_do(torch_cuda):
    L = _lib.lib()
    vp = ctypes.c_void_p
    pat = ds.RGGB.codes()
    white = np.full(3, 4095, np.float32)
    one = ctypes.c_void_p(16)  # never dereferenced: the call must reject first

    def call(w, h, flags=0):
        return L.dsgpu_develop_u16_noalloc(vp(0), one, w, h, w, vp(pat.ctypes.data), 256.0, vp(white.ctypes.data),
                                           vp(WB.ctypes.data), 0.1, 3, 1, one, vp(0), flags)

    assert call(1025, 1024) == _lib.DSGPU_ERR_SIZE  # over DSGPU_NOALLOC_MAX_PIXELS
    assert call(64, 64, _lib.DSGPU_HOST) == _lib.DSGPU_ERR_ARG
    assert call(64, 64, _lib.DSGPU_HIGHLIGHTS) == _lib.DSGPU_ERR_UNSUPPORTED
    assert call(64, 64, 1 << 7) == _lib.DSGPU_ERR_ARG  # unknown flag bit
