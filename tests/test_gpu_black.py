"""Per-site black levels (load_raw's black_at, decode.rs:266-270) on the GPU:
dsgpu_set_black_pattern against the oracle, through every u16 entry point of
a context (normalise, develop on device and host buffers, with highlights,
the learned develop), and its argument errors."""
import os

import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

pytestmark = pytest.mark.gpu

MUL = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
WHITE = np.array([16383.0, 15800.0, 16100.0], np.float32)
PATTERNS = [([[503.0, 509.5], [498.0, 515.0]], (1, 2)), ([[480, 490, 500, 510], [520, 530, 540, 550]], (6, 3)),
            ([[505.0]], (0, 0)), ([[500, 501, 502], [503, 504, 505], [506, 507, 508]], (4, 5))]


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch, torch.device("cuda", 0)


def _raw(torch, dev, w, h, pat, seed):
    sc = ds.Scene(seed=seed, w=w, h=h, pattern=pat, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render(dev)
    torch.cuda.synchronize()
    return sc, raw


@pytest.mark.parametrize("k", range(len(PATTERNS)))
def test_normalize_and_rcd_bitexact(env, oracle, k):
    torch, dev = env
    levels, origin = PATTERNS[k]
    pat = [ds.RGGB, ds.BGGR, ds.GRBG, ds.GBRG][k]
    ctx = ds.Context(0)
    ctx.set_black_pattern(levels, origin)
    for w, h in [(301, 203), (13, 11)]:  # the second is below RCD's 16 x 16 (the MHC path)
        _, raw = _raw(torch, dev, w, h, pat, 40 + k)
        exp_cfa = oracle.normalize_u16_bp(raw.cpu().numpy(), pat.codes(), levels, origin, WHITE)
        got_cfa = ds.normalize_u16(raw, pat, 512, WHITE, ctx=ctx).data.cpu().numpy()
        np.testing.assert_array_equal(got_cfa, exp_cfa)
        host = ds.normalize_u16(raw.cpu().numpy(), pat, 512, WHITE, ctx=ctx).data  # host buffers
        np.testing.assert_array_equal(np.asarray(host), exp_cfa)
        if w >= 16:
            rgb = ds.develop_u16(raw, pat, 512, WHITE, MUL, 0.01, 0, 3, ctx=ctx).data.cpu().numpy()  # search 0: RCD
            np.testing.assert_array_equal(rgb, oracle.rcd(exp_cfa, pat.codes(), MUL))
    ctx.set_black_pattern(None)  # cleared: the scalar black again
    _, raw = _raw(torch, dev, 64, 48, pat, 99)
    np.testing.assert_array_equal(ds.normalize_u16(raw, pat, 512, WHITE, ctx=ctx).data.cpu().numpy(),
                                  oracle.normalize_u16(raw.cpu().numpy(), pat.codes(), 512, WHITE))


def test_develop_with_pattern(env, oracle):
    """NLM on top (2e-4 of the FP64-checked oracle), the host-buffer band
    pipeline bit-identical to the device call, and highlights."""
    torch, dev = env
    levels, origin = PATTERNS[1]
    ctx = ds.Context(0)
    ctx.set_black_pattern(levels, origin)
    w, h = 420, 300
    sc, raw = _raw(torch, dev, w, h, ds.BGGR, 7)
    hp = 1.5 * sc.sigma_norm()
    cfa = oracle.normalize_u16_bp(raw.cpu().numpy(), ds.BGGR.codes(), levels, origin, WHITE)
    exp = oracle.nlm_rgb(oracle.rcd(cfa, ds.BGGR.codes(), MUL), hp, 4, 2)
    dev_out = ds.develop_u16(raw, ds.BGGR, 512, WHITE, MUL, hp, 4, 2, ctx=ctx).data.cpu().numpy()
    assert np.abs(dev_out - exp).max() <= 2e-4
    host_out = ds.develop_u16(raw.cpu().numpy(), ds.BGGR, 512, WHITE, MUL, hp, 4, 2, ctx=ctx).data
    np.testing.assert_array_equal(np.asarray(host_out), dev_out)
    hl = ds.develop_u16(raw, ds.BGGR, 512, WHITE, MUL, hp, 4, 2, ctx=ctx, highlights=True).data.cpu().numpy()
    img = oracle.reconstruct_highlights(oracle.rcd(cfa, ds.BGGR.codes(), MUL), oracle.clip_plane(cfa), MUL,
                                        oracle.cfa_clip_levels(cfa, ds.BGGR.codes()))
    assert np.abs(hl - oracle.nlm_rgb(img, hp, 4, 2)).max() <= 2e-4


def test_learned_develop_with_pattern(env):
    """The learned develop reads the same normalised mosaic: it equals RCD
    (with the pattern) followed by the learned denoise, on device and host."""
    from darkslide_b200 import cnn

    torch, dev = env
    levels, origin = PATTERNS[0]
    ctx = ds.Context(0)
    ctx.set_black_pattern(levels, origin)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    w, h = 256, 200
    sc, raw = _raw(torch, dev, w, h, ds.RGGB, 12)
    hp = 1.5 * sc.sigma_norm()
    got = net.develop_u16(raw, ds.RGGB, 512, WHITE, MUL, hp).data.cpu().numpy()
    rgb = ds.develop_u16(raw, ds.RGGB, 512, WHITE, MUL, hp, 0, 3, ctx=ctx)
    exp, _ = net.denoise(rgb, hp, 10, 3, 3.0)
    np.testing.assert_array_equal(got, exp.data.cpu().numpy())
    host = net.develop_u16(raw.cpu().numpy(), ds.RGGB, 512, WHITE, MUL, hp).data
    np.testing.assert_array_equal(np.asarray(host), got)


def test_black_pattern_argument_errors(env):
    ctx = ds.Context(0)
    L = _lib.lib()
    vp = __import__("ctypes").c_void_p
    lv = np.full(25, 512.0, np.float32)
    assert L.dsgpu_set_black_pattern(ctx.handle, vp(lv.ctypes.data), 5, 1, 0, 0) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_set_black_pattern(ctx.handle, vp(lv.ctypes.data), 2, 0, 0, 0) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_set_black_pattern(ctx.handle, vp(0), 2, 2, 0, 0) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_set_black_pattern(ctx.handle, vp(lv.ctypes.data), 2, 2, -1, 0) == _lib.DSGPU_ERR_ARG
    lv[1] = np.nan
    assert L.dsgpu_set_black_pattern(ctx.handle, vp(lv.ctypes.data), 2, 2, 0, 0) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_set_black_pattern(ctx.handle, vp(0), 0, 0, 0, 0) == _lib.DSGPU_OK
    assert L.dsgpu_set_black_pattern(vp(0), vp(0), 0, 0, 0, 0) == _lib.DSGPU_ERR_ARG
