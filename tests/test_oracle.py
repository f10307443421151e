"""The CPU oracle: the reference's own property tests, a cross-check
against an independent numpy restatement, and the committed golden fixtures."""
import glob
import os

import numpy as np
import pytest

import np_restate as R

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
PATTERNS = [[0, 1, 1, 2], [2, 1, 1, 0], [1, 0, 2, 1], [1, 2, 0, 1]]


def lcg_noise(n):
    """enhance.rs:139-143: seed = seed*1664525 + 1013904223; (seed>>8)/2^24 - 0.5"""
    seed = 1
    out = np.empty(n, np.float32)
    for i in range(n):
        seed = (seed * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = np.float32(seed >> 8) / np.float32(1 << 24) - np.float32(0.5)
    return out


def test_flat_field_is_preserved(oracle):
    """demosaic.rs:514-521: 32x32 RGGB flat [0.2,0.4,0.3], mul 1, Full quality."""
    pat = [0, 1, 1, 2]
    v = np.array([0.2, 0.4, 0.3], np.float32)
    yy, xx = np.mgrid[0:32, 0:32]
    col = np.asarray(pat).reshape(2, 2)[yy % 2, xx % 2]
    cfa = v[col].astype(np.float32)
    rgb = oracle.rcd(cfa, pat, [1, 1, 1])
    p = rgb[16, 16]
    assert np.all(np.abs(p - v) < 1e-4), p


def test_nlm_reduces_noise(oracle):
    """enhance.rs:137-151 with the reference's own LCG noise."""
    p = np.where(np.arange(64)[None, :] < 32, 0.3, 0.7).astype(np.float32) * np.ones((64, 1), np.float32)
    noisy = (p.ravel() + lcg_noise(64 * 64) * np.float32(0.1)).reshape(64, 64).astype(np.float32)
    s = oracle.estimate_noise(noisy)
    assert 0.01 < s < 0.06, s
    d = oracle.nlm(noisy, s * 1.5, 3, 1)
    err = lambda q: float(((q - p) ** 2).sum())
    assert err(d) < err(noisy) * 0.5


def test_box_blur_preserves_constant(oracle):
    """image.rs:455-459 (box part)."""
    p = np.full((23, 37), 0.5, np.float32)
    b = oracle.box_blur(p, 4)
    assert np.all(np.abs(b - 0.5) < 1e-5)


@pytest.mark.parametrize("pat", PATTERNS)
@pytest.mark.parametrize("hw", [(16, 16), (17, 33), (40, 37), (12, 20), (64, 48)])
def test_oracle_matches_numpy_restatement_rcd(oracle, pat, hw):
    rng = np.random.default_rng(hash((tuple(pat), hw)) & 0xFFFF)
    cfa = rng.uniform(-0.05, 1.05, hw).astype(np.float32)
    mul = [2.0, 1.0, 1.4285714]
    a = oracle.rcd(cfa, pat, mul)
    with np.errstate(all="ignore"):
        b = R.rcd(cfa, pat, mul)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(oracle.clip_plane(cfa), R.clip_plane(cfa))
    np.testing.assert_array_equal(oracle.mhc(cfa, pat, mul), R.mhc(cfa, pat, mul))


@pytest.mark.parametrize("r", [0, 1, 3, 5])
def test_oracle_matches_numpy_restatement_box(oracle, r):
    p = np.random.default_rng(r).uniform(0, 1, (29, 41)).astype(np.float32)
    np.testing.assert_array_equal(oracle.box_blur(p, r), R.box_blur(p, r))


@pytest.mark.parametrize("nthreads", [1, 3, 8])
@pytest.mark.parametrize("sp", [(3, 1), (2, 0), (0, 2), (4, 3), (-1, 1)])
def test_oracle_matches_numpy_restatement_nlm(oracle, nthreads, sp):
    s, p = sp
    img = np.random.default_rng(7).uniform(0, 1, (23, 31)).astype(np.float32)
    a = oracle.nlm(img, 0.1, s, p, nthreads=nthreads)
    b = R.nlm(img, 0.1, s, p, nthreads=nthreads)
    # identical up to the last ulp of exp (glibc expf vs exp rounded from f64)
    np.testing.assert_allclose(a, b, rtol=4e-7, atol=1e-7)


def test_nlm_edge_cases(oracle):
    img = np.random.default_rng(3).uniform(0, 1, (9, 11)).astype(np.float32)
    assert np.all(oracle.nlm(img, 0.1, -1, 1) == 0)  # empty offset set -> 0/1e-12
    np.testing.assert_array_equal(oracle.nlm(img, 0.1, 0, 3), img)  # centre weight only


def test_fp64_oracle_close_to_fp32(oracle):
    rng = np.random.default_rng(11)
    cfa = rng.uniform(0, 1, (40, 48)).astype(np.float32)
    a32 = oracle.rcd(cfa, [0, 1, 1, 2], [2, 1, 1.4])
    a64 = oracle.rcd(cfa, [0, 1, 1, 2], [2, 1, 1.4], fp64=True)
    assert np.abs(a32 - a64).max() < 1e-4
    p = a32[..., 1].copy()
    n32 = oracle.nlm(p, 0.05, 3, 1)
    n64 = oracle.nlm(p.astype(np.float64), 0.05, 3, 1, fp64=True)
    assert np.abs(n32 - n64).max() < 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))), ids=os.path.basename)
def test_golden_fixtures(oracle, path):
    z = np.load(path)
    name = os.path.basename(path)
    if name.startswith("nlm_"):
        out = oracle.nlm(z["inp"], float(z["h"]), int(z["search"]), int(z["patch"]), nthreads=1)
        np.testing.assert_array_equal(out, z["out"])
    elif name.startswith("box_"):
        np.testing.assert_array_equal(oracle.box_blur(z["inp"], int(z["r"])), z["out"])
    else:
        cfa = oracle.normalize_u16(z["raw"], z["pattern"], float(z["black"]), z["white"])
        np.testing.assert_array_equal(cfa, z["cfa"])
        np.testing.assert_array_equal(oracle.rcd(cfa, z["pattern"], z["mul"]), z["rgb"])
        np.testing.assert_array_equal(oracle.clip_plane(cfa), z["clip"])
        # the integer pre-stage against its closed form in float64 then rounded
        col = np.asarray(z["pattern"]).reshape(2, 2)
        yy, xx = np.mgrid[0:cfa.shape[0], 0:cfa.shape[1]]
        wc = z["white"][col[yy % 2, xx % 2]]
        ref = ((z["raw"].astype(np.float32) - z["black"]) / np.maximum(wc - z["black"], np.float32(1))).astype(np.float32)
        np.testing.assert_array_equal(cfa, ref)


def test_oklab_roundtrip_and_white(oracle):
    """color.rs:502-512."""
    w = oracle.oklab_from_prophoto(np.array([1.0, 1.0, 1.0], np.float32))
    assert abs(w[0] - 1.0) < 1e-3 and abs(w[1]) < 1e-3 and abs(w[2]) < 1e-3
    c = np.array([0.3, 0.1, 0.6], np.float32)
    back = oracle.oklab_to_prophoto(oracle.oklab_from_prophoto(c))
    assert np.all(np.abs(back - c) < 1e-4)


def test_guided_preserves_edge(oracle):
    """image.rs:464-471."""
    p = np.where(np.arange(40)[None, :] < 20, 0.1, 0.9).astype(np.float32) * np.ones((30, 1), np.float32)
    g = oracle.guided_filter(p, p, 4, 1e-4)
    assert abs(g[5, 5] - 0.1) < 0.02 and abs(g[5, 35] - 0.9) < 0.02


def test_denoise_reduces_noise(oracle):
    rng = np.random.default_rng(2)
    clean = np.stack([np.where(np.arange(80)[None, :] < 40, 0.2, 0.6) * np.ones((60, 1))] * 3, -1).astype(np.float32)
    noisy = (clean + rng.normal(0, 0.03, clean.shape)).astype(np.float32)
    out, sigma = oracle.denoise(noisy, 60)
    assert sigma > 0
    assert ((out - clean) ** 2).sum() < ((noisy - clean) ** 2).sum() * 0.5


def test_cnn_reference_gradients_match_finite_differences():
    """The FP64 CNN reference (oracle/cnn_ref.py) against central differences."""
    import cnn_ref as C

    rng = np.random.default_rng(0)
    n = sum(9 * co * ci + co for ci, co in C.LAYERS)
    p = rng.normal(0, 0.1, n)
    rgb = rng.uniform(0, 1, (1, 5, 6, 3))
    tgt = rgb + rng.normal(0, 0.05, rgb.shape)
    x = C.pack_input(rgb.astype(np.float32), 0.5)
    g, _ = C.gradients(p, x, rgb, tgt)
    loss = lambda q: C.gradients(q, x, rgb, tgt)[1] / (3 * 30)
    for idx in [0, 100, 2900, 25000, n - 5, n - 1]:
        e = np.zeros(n)
        e[idx] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(g[idx] - fd) <= 1e-6 + 1e-5 * abs(fd), (idx, g[idx], fd)


def _clipped_frame(seed, h, w, pat):
    """A mosaic with saturated regions: a bright gradient pushed past white."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    base = 0.5 + 0.7 * np.sin(xx / 7.0) * np.cos(yy / 11.0) + rng.normal(0, 0.01, (h, w))
    gains = np.array([0.8, 1.0, 0.6], np.float32)
    cm = R._color_map(pat, h, w)
    return np.minimum(base * gains[cm], 1.0).astype(np.float32)


@pytest.mark.parametrize("pat", PATTERNS)
@pytest.mark.parametrize("hw", [(40, 52), (97, 61)])
def test_oracle_matches_numpy_restatement_highlights(oracle, pat, hw):
    cfa = _clipped_frame(hash((tuple(pat), hw)) & 0xFFFF, *hw, pat)
    mul = np.array([2.0, 1.0, 1.4285714], np.float32)
    lv = oracle.cfa_clip_levels(cfa, pat)
    np.testing.assert_array_equal(lv, R.cfa_clip_levels(cfa, pat))
    img = oracle.rcd(cfa, pat, mul)
    clip = oracle.clip_plane(cfa)
    assert clip.any() and lv[1] < np.finfo(np.float32).max
    a = oracle.reconstruct_highlights(img, clip, mul, lv)
    np.testing.assert_array_equal(a, R.reconstruct_highlights(img, clip, mul, lv))
    assert not np.array_equal(a, img)  # something was rebuilt


@pytest.mark.parametrize("sigma", [2.0, 2.5, 8.3, 50.0, 79.2])
def test_box_radii_match(oracle, sigma):
    assert oracle.box_radii_for_gauss(sigma) == R.box_radii_for_gauss(sigma)


def test_highlights_untouched_without_clipping(oracle):
    img = np.random.default_rng(3).uniform(0, 0.8, (20, 30, 3)).astype(np.float32)
    out = oracle.reconstruct_highlights(img, np.zeros((20, 30), np.float32), [2, 1, 1.4], [1.0, 1.0, 1.0])
    np.testing.assert_array_equal(out, img)


def _norm_bp_numpy(raw, codes, levels, origin, white):
    """decode.rs:266-306, restated with numpy float32 arithmetic."""
    h, w = raw.shape
    lv = np.asarray(levels, np.float32)
    bh, bw = lv.shape
    yy, xx = np.mgrid[0:h, 0:w]
    b = lv[(yy + origin[1]) % bh, (xx + origin[0]) % bw]
    c = np.asarray(codes, np.int64).reshape(2, 2)[yy % 2, xx % 2]
    wc = np.asarray(white, np.float32)[c]
    return ((raw.astype(np.float32) - b) / np.maximum(wc - b, np.float32(1.0))).astype(np.float32)


@pytest.mark.parametrize("levels,origin", [([[512.0]], (0, 0)), ([[510.0, 514.0], [511.0, 517.5]], (0, 0)),
                                           ([[510.0, 514.0], [511.0, 517.5]], (1, 3)),
                                           ([[500, 501, 502, 503], [504, 505, 506, 507.25]], (5, 2))])
def test_oracle_black_pattern(oracle, levels, origin):
    """The per-site black level of load_raw (black_at, decode.rs:266-270) in
    the oracle against a numpy restatement, bit for bit; a 1x1 pattern is the
    scalar black; a frame cropped at `origin` equals the crop of the frame
    normalised from the sensor origin."""
    rng = np.random.default_rng(len(levels) * 7 + origin[0])
    raw = rng.integers(0, 16384, (37, 53), dtype=np.uint16)
    raw[0, :5] = [0, 1, 16383, 500, 517]  # below, at and above black; white
    white = [16383.0, 15000.0, 16000.0]
    codes = [1, 0, 2, 1]  # GRBG
    got = oracle.normalize_u16_bp(raw, codes, levels, origin, white)
    np.testing.assert_array_equal(got, _norm_bp_numpy(raw, codes, levels, origin, white))
    if np.asarray(levels).size == 1:
        np.testing.assert_array_equal(got, oracle.normalize_u16(raw, codes, float(levels[0][0]), white))
    full = oracle.normalize_u16_bp(raw, codes, levels, (0, 0), white)
    ox, oy = 2, 4  # crop: the pattern shifts with the crop origin (CfaPattern::shifted)
    shifted = [codes[((oy + r) % 2) * 2 + (ox + q) % 2] for r in range(2) for q in range(2)]
    crop = oracle.normalize_u16_bp(raw[oy:, ox:], shifted, levels, (ox, oy), white)
    np.testing.assert_array_equal(crop, full[oy:, ox:])
