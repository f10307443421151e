"""Highlight reconstruction and orientation on the GPU (cfa_clip_levels, reconstruct_highlights,
demosaic.rs:419-502) against the oracle, bit for bit, and the develop path
with DSGPU_HIGHLIGHTS (Engine::base's order: RCD, highlights, then NLM)."""
import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu

PATTERNS = [ds.RGGB, ds.BGGR, ds.GRBG, ds.GBRG]
MUL = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)


def clipped_cfa(seed, h, w, pat):
    """A normalised mosaic with saturated regions (a bright pattern pushed past white)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    base = 0.55 + 0.7 * np.sin(xx / 9.0) * np.cos(yy / 13.0) + rng.normal(0, 0.01, (h, w))
    gains = np.array([0.8, 1.0, 0.6], np.float32)
    codes = np.asarray(pat.codes(), np.int64).reshape(2, 2)
    return np.minimum(base * gains[codes[yy % 2, xx % 2]], 1.0).astype(np.float32)


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return ds.Context(0)


@pytest.mark.parametrize("k", range(4))
@pytest.mark.parametrize("hw", [(48, 64), (301, 517), (64, 9504)])
def test_highlights_bitexact(ctx, oracle, k, hw):
    pat = PATTERNS[k]
    cfa = clipped_cfa(k * 7 + hw[1], *hw, pat)
    lv = oracle.cfa_clip_levels(cfa, pat.codes())
    got_lv = ds.cfa_clip_levels(ds.CfaImage(hw[1], hw[0], cfa, pat), ctx=ctx)
    np.testing.assert_array_equal(got_lv, lv)
    img, clip = ds.demosaic(ds.CfaImage(hw[1], hw[0], cfa, pat), MUL, ctx=ctx)
    exp = oracle.reconstruct_highlights(oracle.rcd(cfa, pat.codes(), MUL), oracle.clip_plane(cfa), MUL, lv)
    got = ds.reconstruct_highlights(img, clip, MUL, got_lv, ctx=ctx)
    assert not np.array_equal(exp, img.data)  # there was something to rebuild
    np.testing.assert_array_equal(got.data, exp)


def test_highlights_noop_without_clipping(ctx):
    img = np.random.default_rng(2).uniform(0, 0.8, (40, 50, 3)).astype(np.float32)
    got = ds.reconstruct_highlights(ds.Image3(50, 40, img), ds.Plane(50, 40, np.zeros((40, 50), np.float32)), MUL,
                                    [1.0, 1.0, 1.0], ctx=ctx)
    np.testing.assert_array_equal(got.data, img)


@pytest.mark.parametrize("pat", [ds.RGGB, ds.GBRG])
def test_develop_with_highlights(ctx, oracle, pat):
    h, w = 160, 224
    cfa = clipped_cfa(11, h, w, pat)
    raw = np.round(cfa * (16383 - 512) + 512).clip(0, 16383).astype(np.uint16)
    white = np.full(3, 16383, np.float32)
    hp = 0.03
    got = ds.develop_u16(raw, pat, 512, white, MUL, hp, 4, 2, ctx=ctx, highlights=True).data
    c = oracle.normalize_u16(raw, pat.codes(), 512, white)
    img = oracle.rcd(c, pat.codes(), MUL)
    img = oracle.reconstruct_highlights(img, oracle.clip_plane(c), MUL, oracle.cfa_clip_levels(c, pat.codes()))
    exp = oracle.nlm_rgb(img, hp, 4, 2)
    assert np.abs(got - exp).max() <= 2e-4
    plain = ds.develop_u16(raw, pat, 512, white, MUL, hp, 4, 2, ctx=ctx).data
    assert np.abs(plain - got).max() > 1e-3  # the flag changed the result


@pytest.mark.parametrize("o", range(0, 10))
@pytest.mark.parametrize("hw", [(37, 70), (64, 64), (5, 130)])
def test_apply_orientation(ctx, oracle, o, hw):
    img = np.random.default_rng(o).uniform(0, 1, hw + (3,)).astype(np.float32)
    got = ds.apply_orientation(ds.Image3(hw[1], hw[0], img), o, ctx=ctx)
    exp = oracle.apply_orientation(img, o)
    assert (got.h, got.w) == exp.shape[:2]
    np.testing.assert_array_equal(got.data, exp)
