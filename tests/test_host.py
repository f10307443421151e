"""Host-side checks that need no GPU: the C-ABI library loads and exports
every symbol its headers declare, argument errors come back as status codes,
the synthetic scene generator is deterministic, and the Python mirror of the
reference types behaves like decode.rs / image.rs."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    from darkslide_b200 import build

    build.build()
    return _lib.lib()


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(dsgpu_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(L):
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTS)


def test_abi_version_and_strerror(L):
    assert L.dsgpu_abi_version() == 2
    for code in range(-8, 1):
        assert _lib.strerror(code) != "unknown status"
    assert _lib.strerror(-99) == "unknown status"


def test_null_context_is_an_argument_error(L):
    vp = ctypes.c_void_p
    assert L.dsgpu_nlm(vp(0), vp(0), 8, 8, 1, 0.1, 3, 1, vp(0), 0) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_rcd(vp(0), vp(0), 8, 8, vp(0), vp(0), vp(0), 0) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_destroy(vp(0)) == _lib.DSGPU_ERR_ARG
    assert L.dsgpu_create(0, None) == _lib.DSGPU_ERR_ARG


def test_create_without_device_reports_nodev(L):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert L.dsgpu_create(0, ctypes.byref(h)) == _lib.DSGPU_ERR_NODEV


def test_scene_host_render_is_deterministic_and_croppable(L):
    sc = ds.Scene(seed=5, w=96, h=64, pattern=ds.BGGR, black=256, white=4095, gain=0.5, read_sigma=3)
    a = sc.render_host()
    b = sc.render_host()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(sc.render_host(10, 7, 30, 20), a[7:27, 10:40])
    assert a.min() >= 0 and a.max() <= 4095
    assert not np.array_equal(a, ds.Scene(seed=6, w=96, h=64, black=256, white=4095).render_host())


def test_oracle_scene_copy_equals_library_scene(L):
    """The oracle's copy of the scene generator (what the benchmark's CPU legs
    render their input with, so that they never load the GPU library) gives
    the library's mosaic and noise-free scene exactly."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import dsref

    for seed, w, h, pat, black, white, g, s in [(1, 6000, 4000, ds.RGGB, 512, 16383, 0.5, 6.0),
                                                (9, 301, 203, ds.GRBG, 256, 4095, 0.25, 12.0)]:
        sc = ds.Scene(seed=seed, w=w, h=h, pattern=pat, black=black, white=white, gain=g, read_sigma=s)
        x0, y0 = (w - 96) // 2, (h - 64) // 2
        np.testing.assert_array_equal(
            sc.render_host(x0, y0, 96, 64),
            dsref.scene_render(seed, w, h, pat.codes(), black, white, g, s, x0, y0, 96, 64))
        np.testing.assert_array_equal(
            sc.truth_host(x0, y0, 40, 30),
            dsref.scene_truth(seed, w, h, pat.codes(), black, white, g, s, x0, y0, 40, 30))


def test_scene_noise_statistics(L):
    """Poisson-Gaussian noise: var(DN) ~ signal/g + sigma_read^2 on flat-ish areas."""
    sc = ds.Scene(seed=1, w=512, h=512, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render_host().astype(np.float64)
    truth = sc.truth_host()
    col = np.array([0, 1, 1, 2]).reshape(2, 2)[np.mgrid[0:512, 0:512][0] % 2, np.mgrid[0:512, 0:512][1] % 2]
    sig = np.take_along_axis(truth, col[..., None], axis=2)[..., 0] * (16383 - 512)
    resid = raw - 512 - sig
    assert abs(resid.mean()) < 0.5
    pred = sig / 0.5 + 36.0
    z = resid / np.sqrt(pred)
    assert 0.9 < z.std() < 1.1
    v = truth / np.array([0.5, 1.0, 0.7], np.float32)
    assert 0.05 - 1e-6 <= v.min() and v.max() <= 0.9 + 1e-6
    assert v.max() - v.min() > 0.3  # the scene is not flat


def test_scene_rejects_bad_arguments(L):
    sc = ds.Scene(seed=1, w=16, h=16)
    with pytest.raises(ds.DsgpuError):
        sc.render_host(10, 10, 10, 10)
    bad = ds.Scene(seed=1, w=16, h=16, pattern=ds.CfaPattern(2, 2, [0, 1, 3, 2]))
    with pytest.raises(ds.DsgpuError):
        bad.render_host()


def test_cfa_pattern_mirror():
    """decode.rs:24-47."""
    p = ds.RGGB
    assert [p.color_at(x, y) for y in range(2) for x in range(2)] == [0, 1, 1, 2]
    assert p.color_at(3, 5) == 2 and p.is_bayer() and not p.is_xtrans()
    assert p.shifted(1, 0).colors == [1, 0, 2, 1]  # RGGB cropped by one column is GRBG
    assert p.shifted(0, 1).colors == [1, 2, 0, 1]  # ... by one row is GBRG
    assert p.shifted(1, 1).colors == [2, 1, 1, 0]
    with pytest.raises(ds.DsgpuError):
        ds.CfaPattern(6, 6, [1] * 36).codes()
