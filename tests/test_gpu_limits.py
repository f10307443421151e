"""The size limits: frames at DSGPU_MAX_DIM in one dimension and the minimum
(16) in the other, through the plain develop (RCD bit-exact, NLM against the
oracle), its host-buffer pipeline, the learned develop and a batch; one past
the limit is DSGPU_ERR_SIZE."""
import os

import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

pytestmark = pytest.mark.gpu

MAXD = 65535
MUL = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
WHITE = [16383.0] * 3


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch, torch.device("cuda", 0)


@pytest.mark.parametrize("w,h", [(MAXD, 16), (16, MAXD), (MAXD, 23)])
def test_extreme_frames(env, oracle, w, h):
    torch, dev = env
    ctx = ds.Context(0)
    sc = ds.Scene(seed=w % 97 + h, w=w, h=h, pattern=ds.GBRG, black=512, white=16383, gain=0.5, read_sigma=6)
    hp = 1.5 * sc.sigma_norm()
    raw = sc.render(dev)
    torch.cuda.synchronize()
    raw_h = raw.cpu().numpy()
    cfa = oracle.normalize_u16(raw_h, ds.GBRG.codes(), 512, WHITE)
    rgb = oracle.rcd(cfa, ds.GBRG.codes(), MUL)
    got_rcd = ds.develop_u16(raw, ds.GBRG, 512, WHITE, MUL, hp, 0, 2, ctx=ctx).data.cpu().numpy()
    np.testing.assert_array_equal(got_rcd, rgb)
    got = ds.develop_u16(raw, ds.GBRG, 512, WHITE, MUL, hp, 4, 2, ctx=ctx).data.cpu().numpy()
    assert np.abs(got - oracle.nlm_rgb(rgb, hp, 4, 2)).max() <= 2e-4
    host = ds.develop_u16(raw_h, ds.GBRG, 512, WHITE, MUL, hp, 4, 2, ctx=ctx).data  # band pipeline
    np.testing.assert_array_equal(np.asarray(host), got)


@pytest.mark.parametrize("w,h", [(MAXD, 16), (16, MAXD)])
def test_extreme_frames_learned(env, w, h):
    from darkslide_b200 import cnn

    torch, dev = env
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    sc = ds.Scene(seed=5, w=w, h=h, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    hp = 1.5 * sc.sigma_norm()
    raw = sc.render(dev)
    torch.cuda.synchronize()
    got = net.develop_u16(raw, ds.RGGB, 512, WHITE, MUL, hp, tau=0.5).data.cpu().numpy()
    exp, _ = net.denoise(ds.develop_u16(raw, ds.RGGB, 512, WHITE, MUL, hp, 0, 3, ctx=ctx), hp, 10, 3, 0.5)
    np.testing.assert_array_equal(got, exp.data.cpu().numpy())
    host = net.develop_u16(raw.cpu().numpy(), ds.RGGB, 512, WHITE, MUL, hp, tau=0.5).data
    np.testing.assert_array_equal(np.asarray(host), got)


def test_batch_extreme_frames(env):
    torch, dev = env
    ctx = ds.Context(0)
    frames = []
    for k, (w, h) in enumerate([(MAXD, 16), (16, MAXD)]):
        sc = ds.Scene(seed=70 + k, w=w, h=h, pattern=ds.BGGR, black=512, white=16383, gain=0.5, read_sigma=6)
        raw = sc.render(dev)
        frames.append(ds.BatchFrame(raw, ds.BGGR, 512, WHITE, MUL, 1.5 * sc.sigma_norm(),
                                    torch.empty((h, w, 3), dtype=torch.float32, device=dev)))
    torch.cuda.synchronize()
    ds.develop_batch(frames, 10, 3, ctx=ctx)
    for f in frames:
        one = ds.develop_u16(f.raw, ds.BGGR, 512, WHITE, MUL, f.h_param, 10, 3, ctx=ctx).data
        np.testing.assert_array_equal(f.out.cpu().numpy(), one.cpu().numpy())


def test_past_the_limit(env):
    torch, dev = env
    ctx = ds.Context(0)
    L = _lib.lib()
    vp = __import__("ctypes").c_void_p
    buf = torch.zeros(16 * (MAXD + 1), dtype=torch.int16, device=dev)
    out = torch.empty(16 * (MAXD + 1) * 3, dtype=torch.float32, device=dev)
    pat = ds.RGGB.codes()
    white = np.full(3, 16383, np.float32)
    for w, h in [(MAXD + 1, 16), (16, MAXD + 1)]:
        assert L.dsgpu_develop_u16(ctx.handle, vp(buf.data_ptr()), w, h, w, vp(pat.ctypes.data), 512.0,
                                   vp(white.ctypes.data), vp(MUL.ctypes.data), 0.01, 10, 3, vp(out.data_ptr()),
                                   vp(0), 0) == _lib.DSGPU_ERR_SIZE
        assert L.dsgpu_normalize_u16(ctx.handle, vp(buf.data_ptr()), w, h, w, vp(pat.ctypes.data), 512.0,
                                     vp(white.ctypes.data), vp(out.data_ptr()), 0) == _lib.DSGPU_ERR_SIZE
