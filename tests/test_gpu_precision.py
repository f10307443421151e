"""NLM's precision variant (DSGPU_FP16_STAGING) and the FP32 path against the
FP64 oracle of RCD+NLM, on the precision workload: an 8256x5504 (45 MP)
BGGR 14-bit mosaic (black 512, white 16383) with high noise (read noise
12 DN, gain 1.0 e/DN), patch 7x7, search 21x21, h = 1.5 x the noise sigma at
mid grey.

The GPU develops the whole frame; the oracle recomputes a central 512x512
crop in FP64 from the raw with a margin wider than the RCD + NLM receptive
field (10 + S + P), and the interior is compared; then the oracle develops
the whole frame in FP64 and every pixel is compared. Max-abs and PSNR
(peak 1) are printed (pytest -s) and bounded here."""
import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu

W45, H45 = 8256, 5504
SEARCH, PATCH = 10, 3
MUL = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
MARGIN = 10 + SEARCH + PATCH + 3


@pytest.fixture(scope="module")
def frame():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    dev = torch.device("cuda", 0)
    sc = ds.Scene(seed=45, w=W45, h=H45, pattern=ds.BGGR, black=512, white=16383, gain=1.0, read_sigma=12.0)
    raw = sc.render(dev)
    hp = 1.5 * sc.sigma_norm()
    white = [16383.0] * 3
    out32 = ds.develop_u16(raw, ds.BGGR, 512, white, MUL, hp, SEARCH, PATCH).data.cpu().numpy()
    out16 = ds.develop_u16(raw, ds.BGGR, 512, white, MUL, hp, SEARCH, PATCH, fp16_staging=True).data.cpu().numpy()
    return sc, raw.cpu().numpy(), hp, out32, out16


def oracle64(oracle, raw, hp, pattern):
    cfa = oracle.normalize_u16(raw, pattern.codes(), 512, np.full(3, 16383, np.float32))
    rgb = oracle.rcd(cfa, pattern.codes(), MUL, fp64=True)
    return oracle.nlm_rgb(rgb, hp, SEARCH, PATCH, fp64=True)


def errors(got, ref):
    d = got.astype(np.float64) - ref
    mse = float(np.mean(d * d))
    return float(np.abs(d).max()), 10.0 * np.log10(1.0 / max(mse, 1e-30))


def test_crop_512_against_fp64(frame, oracle):
    sc, raw, hp, out32, out16 = frame
    x0, y0 = (W45 // 2 - 256) & ~1, (H45 // 2 - 256) & ~1
    ox, oy = x0 - MARGIN, y0 - MARGIN  # even: the crop keeps the BGGR layout
    sub = raw[oy:oy + 512 + 2 * MARGIN, ox:ox + 512 + 2 * MARGIN]
    ref = oracle64(oracle, sub, hp, ds.BGGR)[MARGIN:MARGIN + 512, MARGIN:MARGIN + 512]
    e32 = errors(out32[y0:y0 + 512, x0:x0 + 512], ref)
    e16 = errors(out16[y0:y0 + 512, x0:x0 + 512], ref)
    print(f"\n45MP BGGR read 12 DN, 512x512 crop vs FP64: fp32 max-abs {e32[0]:.3e} PSNR {e32[1]:.1f} dB; "
          f"fp16-staged max-abs {e16[0]:.3e} PSNR {e16[1]:.1f} dB")
    # measured: 5.9e-6 for both (PSNR 145 dB)
    assert e32[0] <= 6e-5 and e16[0] <= 6e-5, (e32, e16)


def test_full_frame_against_fp64(frame, oracle):
    sc, raw, hp, out32, out16 = frame
    ref = oracle64(oracle, raw, hp, ds.BGGR)
    e32, e16 = errors(out32, ref), errors(out16, ref)
    print(f"\n45MP BGGR read 12 DN, full frame vs FP64: fp32 max-abs {e32[0]:.3e} PSNR {e32[1]:.1f} dB; "
          f"fp16-staged max-abs {e16[0]:.3e} PSNR {e16[1]:.1f} dB")
    # measured: 1.33e-4 for both (PSNR 142 dB); the maximum sits at RCD sites
    # where the FP32 demosaic differs from the FP64 one
    assert e32[0] <= 1e-3 and e16[0] <= 1e-3, (e32, e16)


def test_fp16_variant_on_small_frames(oracle):
    """Ragged sizes and all four layouts: the variant stays within the FP32
    path's bound (2e-4) of the FP64 oracle."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    for k, (w, h, pat) in enumerate([(100, 77, ds.RGGB), (257, 130, ds.GRBG), (64, 200, ds.GBRG)]):
        sc = ds.Scene(seed=70 + k, w=w, h=h, pattern=pat, black=512, white=16383, gain=0.5, read_sigma=6.0)
        raw = sc.render(torch.device("cuda", 0))
        hp = 1.5 * sc.sigma_norm()
        got = ds.develop_u16(raw, pat, 512, [16383.0] * 3, MUL, hp, SEARCH, PATCH,
                             fp16_staging=True).data.cpu().numpy()
        ref = oracle64(oracle, raw.cpu().numpy(), hp, pat)
        assert errors(got, ref)[0] <= 2e-4
