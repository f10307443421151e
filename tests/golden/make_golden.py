"""Generate the golden fixtures in this directory from the CPU oracle.

The reference (Rust) cannot run in this environment and its own tests hold
no golden vectors, so these fixtures pin the oracle (oracle/dsref.cpp, a
restatement of the reference cross-checked against an independent numpy
restatement) and give the GPU parity tests committed expectations. Inputs
come from numpy's PCG64 with fixed seeds and are stored beside the outputs.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import dsref  # noqa: E402

PATTERNS = {"RGGB": [0, 1, 1, 2], "BGGR": [2, 1, 1, 0], "GRBG": [1, 0, 2, 1], "GBRG": [1, 2, 0, 1]}


def mosaic(rng, h, w, black, white):
    """Smooth field plus an edge plus noise, quantised to u16 DN."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    base = 0.45 + 0.2 * np.sin(xx / 5.3) * np.cos(yy / 7.1) + 0.25 * (xx + 0.6 * yy > 0.55 * w)
    dn = black + base * (white - black) + rng.normal(0, 0.02 * (white - black), (h, w))
    dn[rng.random((h, w)) < 0.01] = white  # a few clipped sites
    return np.clip(np.rint(dn), 0, white).astype(np.uint16)


def main():
    dsref.build()
    rng = np.random.default_rng(20261203)
    cases = {}
    mul = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
    for name, (h, w, pat, black, white) in {
        "rggb_48x40": (40, 48, "RGGB", 256, 4095),
        "bggr_33x17": (17, 33, "BGGR", 512, 16383),
        "grbg_37x29": (29, 37, "GRBG", 512, 16383),
        "gbrg_16x16": (16, 16, "GBRG", 256, 4095),
        "rggb_12x20_mhc": (20, 12, "RGGB", 256, 4095),
    }.items():
        raw = mosaic(rng, h, w, black, white)
        white3 = np.array([white, white, white], np.float32)
        cfa = dsref.normalize_u16(raw, PATTERNS[pat], black, white3)
        rgb = dsref.rcd(cfa, PATTERNS[pat], mul)
        clip = dsref.clip_plane(cfa)
        cases[name] = dict(raw=raw, pattern=np.array(PATTERNS[pat], np.uint8), black=np.float32(black),
                           white=white3, mul=mul, cfa=cfa, rgb=rgb, clip=clip)
    # NLM on demosaiced planes
    plane = cases["rggb_48x40"]["rgb"][..., 1].copy()
    nlm_cases = {}
    for (h_param, s, p) in [(0.05, 3, 1), (0.08, 10, 3), (0.03, 2, 0), (0.05, 0, 2)]:
        nlm_cases[f"nlm_h{h_param}_s{s}_p{p}"] = dict(
            inp=plane, h=np.float32(h_param), search=np.int32(s), patch=np.int32(p),
            out=dsref.nlm(plane, h_param, s, p, nthreads=1))
    box = {f"box_r{r}": dict(inp=plane, r=np.int32(r), out=dsref.box_blur(plane, r)) for r in (1, 3, 4)}
    for k, v in {**cases, **nlm_cases, **box}.items():
        np.savez_compressed(os.path.join(HERE, f"{k}.npz"), **v)
    print("wrote", len(cases) + len(nlm_cases) + len(box), "fixtures")


if __name__ == "__main__":
    main()
