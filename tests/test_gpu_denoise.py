"""GPU parity for the denoise composite (enhance.rs:75-92) and its parts.

Oklab matrices, estimate_noise and guided_filter round every operation as the
reference does and are compared exactly. The composite goes through cbrtf
(within an ulp of the host's cbrt, not always equal) and NLM, so it is
checked to DENOISE_TOL = 2e-4 max abs.
"""
import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu
DENOISE_TOL = 2e-4


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return ds.default_context(0)


def test_oklab_matrices_match(ctx, oracle):
    ok = ds.Oklab()
    m = oracle.oklab_matrices()
    np.testing.assert_array_equal(ok.to_lms, m[0])
    np.testing.assert_array_equal(ok.from_lms, m[1])
    np.testing.assert_array_equal(ok.m2_inv, m[2])


@pytest.mark.parametrize("hw", [(3, 3), (40, 50), (480, 640), (700, 900)])
def test_estimate_noise_exact(ctx, oracle, hw):
    p = np.random.default_rng(hw[0]).normal(0.4, 0.02, hw).astype(np.float32)
    got = ds.estimate_noise(ds.Plane(hw[1], hw[0], p), ctx=ctx)
    assert got == oracle.estimate_noise(p)


@pytest.mark.parametrize("r", [1, 4, 13])
def test_guided_filter_exact(ctx, oracle, r):
    rng = np.random.default_rng(r)
    I = rng.uniform(0, 1, (90, 130)).astype(np.float32)
    p = (I * 0.5 + rng.normal(0, 0.05, I.shape)).astype(np.float32)
    got = ds.guided_filter(ds.Plane(130, 90, I), ds.Plane(130, 90, p), r, 1e-3, ctx=ctx).data
    np.testing.assert_array_equal(got, oracle.guided_filter(I, p, r, 1e-3))


def test_guided_preserves_edge(ctx):
    """image.rs:464-471 on the GPU path."""
    p = np.where(np.arange(40)[None, :] < 20, 0.1, 0.9).astype(np.float32) * np.ones((30, 1), np.float32)
    g = ds.guided_filter(ds.Plane(40, 30, p), ds.Plane(40, 30, p), 4, 1e-4, ctx=ctx).data
    assert abs(g[5, 5] - 0.1) < 0.02 and abs(g[5, 35] - 0.9) < 0.02


@pytest.mark.parametrize("amount", [0.0, 50.0, 100.0])
def test_denoise_vs_oracle(ctx, oracle, amount):
    sc = ds.Scene(seed=4, w=320, h=240, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    cfa = oracle.normalize_u16(sc.render_host(), ds.RGGB.codes(), 512, np.full(3, 16383, np.float32))
    rgb = oracle.rcd(cfa, ds.RGGB.codes(), np.array([2.0, 1.0, 1 / 0.7], np.float32))
    got = ds.denoise(ds.Image3(320, 240, rgb), amount, ctx=ctx).data
    exp, _ = oracle.denoise(rgb, amount)
    err = np.abs(got - exp).max()
    assert err <= DENOISE_TOL, err


def test_denoise_large_frame_runs_on_device(ctx):
    import torch

    sc = ds.Scene(seed=5, w=3000, h=2000, pattern=ds.RGGB, black=512, white=16383)
    img = ds.develop_u16(sc.render(), ds.RGGB, 512, np.full(3, 16383, np.float32), [2.0, 1.0, 1 / 0.7], 0.02, 3, 1)
    out = ds.denoise(img, 40)
    torch.cuda.synchronize()
    o = out.data.cpu().numpy()
    assert np.isfinite(o).all() and o.min() >= 0
