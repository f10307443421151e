"""GPU parity: the CUDA path (called through the C ABI) against the CPU
oracle on the same inputs.

Tolerances
  - CFA normalisation, clip plane, MHC, superpixel, RCD, box blur: bit-exact
    (compared with ==), since those kernels round every operation as the
    reference does.
  - NLM: the GPU weights come from ex2.approx and sums run in a different
    order (running sums, FMA), so NLM is checked against the f32 oracle with
    max |gpu - oracle| <= NLM_TOL = 2e-4 (the target is 1e-3), and against the
    FP64 oracle with the same bound.
"""
import os

import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
PATTERNS = {"RGGB": ds.RGGB, "BGGR": ds.BGGR, "GRBG": ds.GRBG, "GBRG": ds.GBRG}
WB = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
NLM_TOL = 2e-4


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return ds.default_context(0)


def cfa_img(data, pat):
    h, w = data.shape
    return ds.CfaImage(w, h, np.ascontiguousarray(data, np.float32), pat)


# ------------------------------------------------------------ scene + pre-stage
@pytest.mark.parametrize("wh", [(257, 193), (2000, 1500)])
def test_scene_gpu_render_equals_host(ctx, wh):
    sc = ds.Scene(seed=42, w=wh[0], h=wh[1], pattern=ds.GRBG, black=512, white=16383, gain=0.25, read_sigma=12)
    gpu = sc.render().cpu().numpy()
    np.testing.assert_array_equal(gpu, sc.render_host())


def test_scene_gpu_window_equals_frame(ctx):
    sc = ds.Scene(seed=7, w=3001, h=2003, pattern=ds.RGGB, black=256, white=4095, gain=0.6, read_sigma=5)
    full = sc.render().cpu().numpy()
    for win in [(0, 0, 512, 512), (1234, 777, 300, 211), (2489, 1491, 512, 512)]:
        x0, y0, cw, ch = win
        got = sc.render(window=win).cpu().numpy()
        np.testing.assert_array_equal(got, full[y0:y0 + ch, x0:x0 + cw])
    np.testing.assert_array_equal(sc.render(window=(5, 9, 40, 30)).cpu().numpy(), sc.render_host(5, 9, 40, 30))


@pytest.mark.parametrize("name", list(PATTERNS))
def test_normalize_u16_bitexact(ctx, oracle, name):
    rng = np.random.default_rng(1)
    raw = rng.integers(0, 16384, (61, 77), dtype=np.uint16)  # below black and above white too
    white = np.array([16383, 15000, 16000], np.float32)
    got = ds.normalize_u16(raw, PATTERNS[name], 512, white, ctx=ctx).data
    exp = oracle.normalize_u16(raw, PATTERNS[name].codes(), 512, white)
    np.testing.assert_array_equal(got, exp)


# ----------------------------------------------------------------- demosaic
@pytest.mark.parametrize("path", sorted(f for f in os.listdir(GOLDEN) if f[:4] in ("rggb", "bggr", "grbg", "gbrg")))
def test_golden_demosaic(ctx, path):
    z = np.load(os.path.join(GOLDEN, path))
    pat = ds.CfaPattern(2, 2, list(z["pattern"]))
    cfa = ds.normalize_u16(z["raw"], pat, float(z["black"]), z["white"], ctx=ctx)
    np.testing.assert_array_equal(cfa.data, z["cfa"])
    rgb, clip = ds.demosaic(cfa, z["mul"], ds.Quality.FULL, ctx=ctx)
    np.testing.assert_array_equal(rgb.data, z["rgb"])
    np.testing.assert_array_equal(clip.data, z["clip"])


@pytest.mark.parametrize("name", list(PATTERNS))
@pytest.mark.parametrize("hw", [(16, 16), (17, 33), (48, 64), (77, 100), (33, 16), (768, 1024)])
@pytest.mark.parametrize("mul", ["wb", "one"])
def test_rcd_bitexact(ctx, oracle, name, hw, mul):
    rng = np.random.default_rng(hw[0] * 1000 + hw[1])
    data = rng.uniform(-0.05, 1.05, hw).astype(np.float32)
    m = WB if mul == "wb" else np.ones(3, np.float32)
    got = ds.rcd_bayer(cfa_img(data, PATTERNS[name]), m, ctx=ctx).data
    exp = oracle.rcd(data, PATTERNS[name].codes(), m)
    assert np.array_equal(got, exp), f"{int((got != exp).sum())} differing values, max {np.abs(got - exp).max()}"


@pytest.mark.parametrize("hw", [(1, 1), (2, 3), (5, 7), (15, 40), (12, 20)])
def test_tiny_images_are_mhc(ctx, oracle, hw):
    data = np.random.default_rng(5).uniform(0, 1, hw).astype(np.float32)
    img = cfa_img(data, ds.RGGB)
    got = ds.rcd_bayer(img, WB, ctx=ctx).data
    np.testing.assert_array_equal(got, oracle.mhc(data, ds.RGGB.codes(), WB))
    np.testing.assert_array_equal(ds.mhc_bayer(img, WB, ctx=ctx).data, oracle.mhc(data, ds.RGGB.codes(), WB))


@pytest.mark.parametrize("name", list(PATTERNS))
def test_clip_and_draft(ctx, oracle, name):
    rng = np.random.default_rng(9)
    data = rng.uniform(0.9, 1.01, (41, 58)).astype(np.float32)
    img = cfa_img(data, PATTERNS[name])
    np.testing.assert_array_equal(ds.clip_plane(img, ctx=ctx).data, oracle.clip_plane(data))
    rgb, clip = ds.demosaic(img, WB, ds.Quality.DRAFT, ctx=ctx)
    er, ec = oracle.superpixel(data, PATTERNS[name].codes(), WB)
    np.testing.assert_array_equal(rgb.data, er)
    np.testing.assert_array_equal(clip.data, ec)


def test_flat_field_is_preserved(ctx):
    """demosaic.rs:514-521 on the GPU path."""
    v = np.array([0.2, 0.4, 0.3], np.float32)
    yy, xx = np.mgrid[0:32, 0:32]
    col = np.array([0, 1, 1, 2]).reshape(2, 2)[yy % 2, xx % 2]
    rgb, _ = ds.demosaic(cfa_img(v[col], ds.RGGB), [1, 1, 1], ds.Quality.FULL, ctx=ctx)
    assert np.all(np.abs(rgb.data[16, 16] - v) < 1e-4)
    d, _ = ds.demosaic(cfa_img(v[col], ds.RGGB), [1, 1, 1], ds.Quality.DRAFT, ctx=ctx)
    assert np.all(np.abs(d.data[8, 8] - v) < 1e-4)


# ---------------------------------------------------------------- box blur
@pytest.mark.parametrize("r", [0, 1, 3, 4, 9])
@pytest.mark.parametrize("hw", [(23, 37), (130, 70)])
def test_box_blur_bitexact(ctx, oracle, r, hw):
    p = np.random.default_rng(r).uniform(0, 1, hw).astype(np.float32)
    got = ds.box_blur(ds.Plane(hw[1], hw[0], p), r, ctx=ctx).data
    np.testing.assert_array_equal(got, oracle.box_blur(p, r))


def test_box_blur_preserves_constant(ctx):
    p = np.full((23, 37), 0.5, np.float32)
    assert np.all(np.abs(ds.box_blur(ds.Plane(37, 23, p), 4, ctx=ctx).data - 0.5) < 1e-5)


# --------------------------------------------------------------------- NLM
@pytest.mark.parametrize("path", sorted(f for f in os.listdir(GOLDEN) if f.startswith("nlm_")))
def test_golden_nlm(ctx, path):
    z = np.load(os.path.join(GOLDEN, path))
    p = z["inp"]
    got = ds.nlm(ds.Plane(p.shape[1], p.shape[0], p), float(z["h"]), int(z["search"]), int(z["patch"]), ctx=ctx).data
    assert np.abs(got - z["out"]).max() <= NLM_TOL


@pytest.mark.parametrize("sp", [(3, 1), (10, 3), (0, 2), (2, 0), (5, 5), (16, 7), (1, 4)])
@pytest.mark.parametrize("hw", [(70, 90), (130, 67), (9, 13)])
def test_nlm_vs_oracle(ctx, oracle, sp, hw):
    s, p = sp
    rng = np.random.default_rng(s * 100 + p)
    base = np.where(np.arange(hw[1])[None, :] < hw[1] // 2, 0.3, 0.7).astype(np.float32)
    img = (base + rng.normal(0, 0.03, hw)).astype(np.float32)
    h = 0.05
    got = ds.nlm(ds.Plane(hw[1], hw[0], img), h, s, p, ctx=ctx).data
    exp = oracle.nlm(img, h, s, p)
    exp64 = oracle.nlm(img.astype(np.float64), h, s, p, fp64=True)
    assert np.abs(got - exp).max() <= NLM_TOL
    assert np.abs(got - exp64).max() <= NLM_TOL


def test_nlm_edge_cases(ctx):
    img = np.random.default_rng(3).uniform(0, 1, (40, 50)).astype(np.float32)
    pl = ds.Plane(50, 40, img)
    assert np.all(ds.nlm(pl, 0.1, -1, 1, ctx=ctx).data == 0)
    np.testing.assert_array_equal(ds.nlm(pl, 0.1, 0, 3, ctx=ctx).data, img)
    const = ds.Plane(50, 40, np.full((40, 50), 0.37, np.float32))
    np.testing.assert_allclose(ds.nlm(const, 0.05, 4, 2, ctx=ctx).data, 0.37, rtol=1e-6)
    # h -> 0: only identical patches get weight; a noisy image stays itself
    np.testing.assert_allclose(ds.nlm(pl, 0.0, 3, 1, ctx=ctx).data, img, atol=1e-6)


def test_nlm_reduces_noise(ctx, oracle):
    """enhance.rs:137-151 on the GPU path, with the reference's LCG."""
    from test_oracle import lcg_noise

    p = np.where(np.arange(64)[None, :] < 32, 0.3, 0.7).astype(np.float32) * np.ones((64, 1), np.float32)
    noisy = (p.ravel() + lcg_noise(64 * 64) * np.float32(0.1)).reshape(64, 64).astype(np.float32)
    s = oracle.estimate_noise(noisy)
    d = ds.nlm(ds.Plane(64, 64, noisy), s * 1.5, 3, 1, ctx=ctx).data
    assert ((d - p) ** 2).sum() < ((noisy - p) ** 2).sum() * 0.5


def test_nlm_rgb_equals_per_channel(ctx):
    img = np.random.default_rng(4).uniform(0, 1, (45, 70, 3)).astype(np.float32)
    rgb = ds.nlm(ds.Image3(70, 45, img), 0.08, 4, 2, ctx=ctx).data
    for c in range(3):
        pc = ds.nlm(ds.Plane(70, 45, img[..., c].copy()), 0.08, 4, 2, ctx=ctx).data
        np.testing.assert_array_equal(rgb[..., c], pc)


# --------------------------------------------------------- the whole path
def test_develop_u16_c1_config(ctx, oracle):
    """1024x768 RGGB 12-bit (black 256, white 4095), NLM 7x7 / 21x21, h 0.08."""
    sc = ds.Scene(seed=1, w=1024, h=768, pattern=ds.RGGB, black=256, white=4095, gain=0.5, read_sigma=3)
    raw = sc.render_host()
    white = np.full(3, 4095, np.float32)
    out, clip = ds.develop_u16(raw, ds.RGGB, 256, white, WB, 0.08, 10, 3, with_clip=True, ctx=ctx)
    cfa = oracle.normalize_u16(raw, ds.RGGB.codes(), 256, white)
    rgb = oracle.rcd(cfa, ds.RGGB.codes(), WB)
    np.testing.assert_array_equal(ds.rcd_bayer(cfa_img(cfa, ds.RGGB), WB, ctx=ctx).data, rgb)
    np.testing.assert_array_equal(clip.data, oracle.clip_plane(cfa))
    exp = oracle.nlm_rgb(rgb, 0.08, 10, 3)
    err = np.abs(out.data - exp).max()
    assert err <= NLM_TOL, err


def test_torch_device_path_matches_host_path(ctx):
    import torch

    sc = ds.Scene(seed=3, w=300, h=200, pattern=ds.BGGR, black=512, white=16383)
    raw_t = sc.render()
    raw = raw_t.cpu().numpy()
    white = np.full(3, 16383, np.float32)
    host = ds.develop_u16(raw, ds.BGGR, 512, white, WB, 0.02, 5, 2, ctx=ctx).data
    dev = ds.develop_u16(raw_t, ds.BGGR, 512, white, WB, 0.02, 5, 2).data
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy(), host)


def test_full_size_frame_matches_oracle_on_crops(ctx, oracle):
    """24 MP (6000x4000) RGGB 14-bit: the full-frame GPU result, checked on
    crops that the oracle computes with enough margin that its own borders do
    not reach the compared interior (RCD radius 10, NLM radius S+P)."""
    import torch

    sc = ds.Scene(seed=7, w=6000, h=4000, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    raw_t = sc.render()
    white = np.full(3, 16383, np.float32)
    S, P = 10, 3
    h_param = 1.5 * sc.sigma_norm()
    out = ds.develop_u16(raw_t, ds.RGGB, 512, white, WB, h_param, S, P).data
    torch.cuda.synchronize()
    out = out.cpu().numpy()
    assert np.isfinite(out).all()
    m = 10 + S + P + 2
    for (x0, y0) in [(0, 0), (3000, 2000), (6000 - 96, 4000 - 80), (1234, 3917 - 60)]:
        cw, ch = 96, 80
        ax0, ay0 = max(x0 - m, 0), max(y0 - m, 0)
        ax1, ay1 = min(x0 + cw + m, 6000), min(y0 + ch + m, 4000)
        raw = sc.render_host(ax0, ay0, ax1 - ax0, ay1 - ay0)
        pat = ds.RGGB.shifted(ax0, ay0).codes()
        cfa = oracle.normalize_u16(raw, pat, 512, white)
        rgb = oracle.rcd(cfa, pat, WB)
        exp = oracle.nlm_rgb(rgb, h_param, S, P)
        sl = (slice(y0 - ay0, y0 - ay0 + ch), slice(x0 - ax0, x0 - ax0 + cw))
        got = out[y0:y0 + ch, x0:x0 + cw]
        err = np.abs(got - exp[sl]).max()
        assert err <= NLM_TOL, ((x0, y0), err)


# ----------------------------------------------------------- error handling
def test_errors_are_status_codes(ctx):
    img = cfa_img(np.zeros((20, 20), np.float32), ds.CfaPattern(2, 2, [0, 1, 3, 2]))
    with pytest.raises(ds.DsgpuError) as e:
        ds.rcd_bayer(img, WB, ctx=ctx)
    assert e.value.status == -2
    pl = ds.Plane(20, 20, np.zeros((20, 20), np.float32))
    with pytest.raises(ds.DsgpuError) as e:
        ds.nlm(pl, 0.1, 17, 1, ctx=ctx)
    assert e.value.status == -1
    with pytest.raises(ds.DsgpuError) as e:
        ds.nlm(pl, 0.1, 3, 8, ctx=ctx)
    assert e.value.status == -1
    with pytest.raises(ds.DsgpuError) as e:
        ds.box_blur(pl, -1, ctx=ctx)
    assert e.value.status == -1
    big = ds.Plane(70000, 1, np.zeros((1, 70000), np.float32))
    with pytest.raises(ds.DsgpuError) as e:
        ds.box_blur(big, 1, ctx=ctx)
    assert e.value.status == -3
    # the context stays usable after argument errors
    assert np.all(ds.box_blur(pl, 1, ctx=ctx).data == 0)


def test_row_band_split_on_gpu(ctx):
    """The row-band split of darkslide_b200.shard on the GPU kernels: bands
    developed one after another reassemble the whole-frame result."""
    from darkslide_b200 import shard

    sc = ds.Scene(seed=21, w=640, h=480, pattern=ds.GRBG, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render_host()
    white = np.full(3, 16383, np.float32)
    S, P, h = 10, 3, 1.5 * sc.sigma_norm()
    full = ds.develop_u16(raw, ds.GRBG, 512, white, WB, h, S, P, ctx=ctx).data
    for world in (2, 3):
        parts = [shard.develop_band(raw, ds.GRBG, shard.band(480, r, world, shard.halo_rows(S, P)), 512, white, WB,
                                    h, S, P, ctx=ctx) for r in range(world)]
        got = np.concatenate(parts, axis=0)
        assert got.shape == full.shape
        # bands place the NLM tiles differently, which changes the order of
        # the FMA sums: equal to ~20 ulps
        assert np.abs(got - full).max() <= 1e-5


@pytest.mark.parametrize("hw", [(4000, 600), (37, 1201), (64, 58)])
def test_develop_host_buffers_equal_device_path(ctx, hw):
    """With host buffers the develop call runs NLM in bands of tile rows and
    copies each band back while the next one computes; the result must equal
    the device-buffer call bit for bit (RGB and clip plane)."""
    import torch

    w, h = hw
    sc = ds.Scene(seed=9, w=w, h=h, pattern=ds.GRBG, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render_host()
    white = [16383.0] * 3
    mul = [2.0, 1.0, 1.0 / 0.7]
    host, hclip = ds.develop_u16(raw, ds.GRBG, 512, white, mul, 0.02, 10, 3, with_clip=True, ctx=ctx)
    dev_img, dclip = ds.develop_u16(torch.from_numpy(raw).cuda(), ds.GRBG, 512, white, mul, 0.02, 10, 3,
                                    with_clip=True, ctx=ctx)
    np.testing.assert_array_equal(host.data, dev_img.data.cpu().numpy())
    np.testing.assert_array_equal(hclip.data, dclip.data.cpu().numpy())
