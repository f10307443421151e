"""dsgpu_develop_u16_noalloc: the detail path for callers that cannot
allocate device memory (they manage all device memory themselves, or call
where cudaMalloc is not allowed or would stall the device). It keeps its
intermediate in a fixed array inside the library instead of context
scratch, so its output must equal dsgpu_develop_u16's on the same inputs,
call after call, even though every call reuses the same array.

This file is collected last so that a run stopping at the first failure has
run every other test first."""
import ctypes

import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

pytestmark = pytest.mark.gpu

WB = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
NLM_TOL = 2e-4  # the NLM tolerance of the parity tests


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch


def _run_both(torch, sc, h_param, search, patch):
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    L = _lib.lib()
    vp = ctypes.c_void_p
    raw = sc.render(dev)
    w, h = sc.w, sc.h
    pat = sc.pattern.codes()
    white = np.full(3, sc.white, np.float32)
    outs = {}
    for name in ("ctx", "noalloc"):
        rgb = torch.full((h, w, 3), float("nan"), dtype=torch.float32, device=dev)
        clip = torch.full((h, w), float("nan"), dtype=torch.float32, device=dev)
        args = (vp(raw.data_ptr()), w, h, w, vp(pat.ctypes.data), float(sc.black), vp(white.ctypes.data),
                vp(WB.ctypes.data), float(h_param), search, patch, vp(rgb.data_ptr()), vp(clip.data_ptr()), 0)
        if name == "ctx":
            ctx = ds.default_context(0)
            ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
            ctx.check(L.dsgpu_develop_u16(ctx.handle, *args), "dsgpu_develop_u16")
        else:
            st = L.dsgpu_develop_u16_noalloc(vp(torch.cuda.current_stream(dev).cuda_stream), *args)
            assert st == 0, _lib.strerror(st)
        torch.cuda.synchronize()
        outs[name] = (rgb.cpu().numpy(), clip.cpu().numpy())
    return outs


def test_noalloc_matches_allocating_entry_point_twice(torch_cuda):
    # two calls in a row on different frames: the second reuses the array
    # the first one left behind
    cases = [
        (ds.Scene(seed=1, w=1024, h=768, pattern=ds.RGGB, black=256, white=4095, gain=0.5, read_sigma=3), 0.08, 10, 3),
        (ds.Scene(seed=2, w=600, h=400, pattern=ds.GBRG, black=512, white=16383, gain=0.25, read_sigma=12), 0.03, 3, 1),
    ]
    for sc, h_param, search, patch in cases:
        outs = _run_both(torch_cuda, sc, h_param, search, patch)
        (a_rgb, a_clip), (b_rgb, b_clip) = outs["ctx"], outs["noalloc"]
        assert np.isfinite(b_rgb).all()
        assert np.abs(a_rgb - b_rgb).max() <= NLM_TOL
        np.testing.assert_array_equal(a_clip, b_clip)


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
