"""Crops as load_raw takes them (decode.rs:259-306): a frame inside a larger
raw, passed as a pointer offset with the full raw's row pitch and the CFA
pattern shifted by the crop origin. Every u16 entry point gives exactly what
it gives for a contiguous copy of the crop: plain develop on device and host
buffers, the learned develop, and normalise with a black pattern anchored at
the crop origin."""
import ctypes
import os

import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

pytestmark = pytest.mark.gpu

MUL = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
WHITE = np.full(3, 16383, np.float32)
FW, FH = 700, 500          # the full raw
CX, CY, W, H = 37, 22, 401, 333  # the crop (odd x origin: the pattern shifts)
vp = ctypes.c_void_p


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    dev = torch.device("cuda", 0)
    sc = ds.Scene(seed=3, w=FW, h=FH, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render(dev)
    torch.cuda.synchronize()
    return torch, dev, raw, 1.5 * sc.sigma_norm()


def _crop_pointer_dev(raw):
    return vp(raw.data_ptr() + (CY * FW + CX) * 2)


def test_plain_develop_pitched(env):
    torch, dev, raw, hp = env
    ctx = ds.Context(0)
    L = _lib.lib()
    pat = ds.RGGB.shifted(CX, CY)
    codes = pat.codes()
    exp = ds.develop_u16(raw[CY:CY + H, CX:CX + W].contiguous(), pat, 512, WHITE, MUL, hp, 10, 3,
                         ctx=ctx).data.cpu().numpy()
    out = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    ctx.check(L.dsgpu_develop_u16(ctx.handle, _crop_pointer_dev(raw), W, H, FW, vp(codes.ctypes.data), 512.0,
                                  vp(WHITE.ctypes.data), vp(MUL.ctypes.data), float(hp), 10, 3, vp(out.data_ptr()),
                                  vp(0), 0), "develop pitched")
    np.testing.assert_array_equal(out.cpu().numpy(), exp)
    raw_h = raw.cpu().numpy()
    out_h = np.empty((H, W, 3), np.float32)
    ctx.check(L.dsgpu_develop_u16(ctx.handle, vp(raw_h.ctypes.data + (CY * FW + CX) * 2), W, H, FW,
                                  vp(codes.ctypes.data), 512.0, vp(WHITE.ctypes.data), vp(MUL.ctypes.data), float(hp),
                                  10, 3, vp(out_h.ctypes.data), vp(0), _lib.DSGPU_HOST), "develop pitched host")
    np.testing.assert_array_equal(out_h, exp)


def test_learned_develop_pitched(env):
    from darkslide_b200 import cnn

    torch, dev, raw, hp = env
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    L = _lib.lib()
    pat = ds.RGGB.shifted(CX, CY)
    codes = pat.codes()
    exp = net.develop_u16(raw[CY:CY + H, CX:CX + W].contiguous(), pat, 512, WHITE, MUL, hp).data.cpu().numpy()
    out = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    ctx.check(L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, _crop_pointer_dev(raw), W, H, FW, vp(codes.ctypes.data),
                                      512.0, vp(WHITE.ctypes.data), vp(MUL.ctypes.data), float(hp), 10, 3, 3.0,
                                      vp(out.data_ptr()), vp(0), 0), "learned pitched")
    np.testing.assert_array_equal(out.cpu().numpy(), exp)
    raw_h = raw.cpu().numpy()
    out_h = np.empty((H, W, 3), np.float32)
    ctx.check(L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, vp(raw_h.ctypes.data + (CY * FW + CX) * 2), W, H, FW,
                                      vp(codes.ctypes.data), 512.0, vp(WHITE.ctypes.data), vp(MUL.ctypes.data),
                                      float(hp), 10, 3, 3.0, vp(out_h.ctypes.data), vp(0), _lib.DSGPU_HOST),
              "learned pitched host")
    np.testing.assert_array_equal(out_h, exp)


def test_normalize_pitched_with_black_pattern(env, oracle):
    torch, dev, raw, hp = env
    ctx = ds.Context(0)
    L = _lib.lib()
    levels = [[501.0, 509.0], [497.5, 515.0]]
    full = oracle.normalize_u16_bp(raw.cpu().numpy(), ds.RGGB.codes(), levels, (0, 0), WHITE)
    ctx.set_black_pattern(levels, (CX, CY))
    codes = ds.RGGB.shifted(CX, CY).codes()
    out = torch.empty((H, W), dtype=torch.float32, device=dev)
    ctx.check(L.dsgpu_normalize_u16(ctx.handle, _crop_pointer_dev(raw), W, H, FW, vp(codes.ctypes.data), 512.0,
                                    vp(WHITE.ctypes.data), vp(out.data_ptr()), 0), "normalize pitched")
    np.testing.assert_array_equal(out.cpu().numpy(), full[CY:CY + H, CX:CX + W])
