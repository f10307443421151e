"""Run one kernel of the path on a small case, for profiler captures.

    python -m darkslide_b200.profile_case nlm   # 4096x3072x3 NLM, 7x7 / 21x21
    python -m darkslide_b200.profile_case rcd   # 6000x4000 u16 -> RCD (+clip)
    python -m darkslide_b200.profile_case develop [--w W --h H]
    python -m darkslide_b200.profile_case denoise  # enhance::denoise, amount 50
    python -m darkslide_b200.profile_case cnn      # the learned stand-in (8 conv layers)
    python -m darkslide_b200.profile_case learned  # u16 -> RCD -> network + NLM fallback (committed weights)
    python -m darkslide_b200.profile_case batch --frames 8 --w 2048 --h 1536   # one batched graph launch
    python -m darkslide_b200.profile_case mma      # tcgen05 MMA issue rate vs N and commit spacing

Each case does one warm-up call and `--reps` timed calls on cuda:0 and
prints the mean device time per call (CUDA events).
"""
from __future__ import annotations

import argparse
import ctypes

import numpy as np
import torch

import darkslide_b200 as ds
from darkslide_b200 import _lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["nlm", "rcd", "develop", "denoise", "cnn", "learned", "batch", "mma"])
    ap.add_argument("--frames", type=int, default=8, help="batch: frames of w x h")
    ap.add_argument("--w", type=int, default=0)
    ap.add_argument("--h", type=int, default=0)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--search", type=int, default=10)
    ap.add_argument("--patch", type=int, default=3)
    ap.add_argument("--fp16", action="store_true", help="NLM's FP16-staging precision variant")
    a = ap.parse_args()
    if a.case == "mma":  # no frame: the microbenchmark alone
        ctx = ds.Context(0)
        commits = [0, 1, 2, 6, 12, 19, 57, 228]
        print("SM cycles per 128 x N x 16 BF16 tcgen05 MMA (4096 back to back per SM, all SMs)")
        print("commit every:" + "".join(f"{c:>8}" for c in commits))
        for n in (48, 96, 144, 256):
            row = [ctx.measure_tcgen05_mma(n, c) for c in commits]
            print(f"N = {n:3d}     :" + "".join(f"{v:8.1f}" for v in row))
        return
    xflags = _lib.DSGPU_FP16_STAGING if a.fp16 else 0
    dev = torch.device("cuda", 0)
    ctx = ds.Context(0)
    st = torch.cuda.Stream(dev)
    ctx.set_stream(st.cuda_stream)
    L = _lib.lib()
    vp = ctypes.c_void_p
    w = a.w or (4096 if a.case == "nlm" else 6000)
    h = a.h or (3072 if a.case == "nlm" else 4000)
    sc = ds.Scene(seed=1, w=w, h=h, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    white = np.full(3, 16383, np.float32)
    mul = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
    pat = ds.RGGB.codes()
    hp = 1.5 * sc.sigma_norm()
    with torch.cuda.stream(st):
        raw = sc.render(dev, ctx=ctx)
        rgb = torch.empty((h, w, 3), dtype=torch.float32, device=dev)
        out = torch.empty((h, w, 3), dtype=torch.float32, device=dev)
        clip = torch.empty((h, w), dtype=torch.float32, device=dev)
    st.synchronize()
    with torch.cuda.stream(st):  # keeps the context on stream st
        cfa = ds.normalize_u16(raw, ds.RGGB, 512, white, ctx=ctx).data
    st.synchronize()

    frames = None
    if a.case == "batch":  # a batch of equal frames, alternating CFA layouts
        pats = [ds.RGGB, ds.BGGR, ds.GRBG, ds.GBRG]
        with torch.cuda.stream(st):
            frames = [ds.BatchFrame(raw, pats[k % 4], 512, white, mul, hp,
                                    torch.empty((h, w, 3), dtype=torch.float32, device=dev))
                      for k in range(a.frames)]
        st.synchronize()

    def call():
        if a.case == "batch":
            with torch.cuda.stream(st):
                ds.develop_batch(frames, a.search, a.patch, ctx=ctx, sync=False)
            return
        if a.case == "nlm":
            r = L.dsgpu_nlm(ctx.handle, vp(rgb.data_ptr()), w, h, 3, float(hp), a.search, a.patch, vp(out.data_ptr()),
                            _lib.DSGPU_ASYNC | xflags)
        elif a.case == "rcd":
            r = L.dsgpu_demosaic(ctx.handle, vp(cfa.data_ptr()), w, h, vp(pat.ctypes.data), vp(mul.ctypes.data),
                                 _lib.DSGPU_QUALITY_FULL, vp(rgb.data_ptr()), vp(clip.data_ptr()), _lib.DSGPU_ASYNC)
        elif a.case == "cnn":
            r = L.dsgpu_cnn_infer(ctx.handle, net.handle, vp(rgb.data_ptr()), w, h, 0.5, vp(out.data_ptr()),
                                  _lib.DSGPU_ASYNC)
        elif a.case == "learned":
            r = L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, vp(raw.data_ptr()), w, h, w, vp(pat.ctypes.data), 512.0,
                                        vp(white.ctypes.data), vp(mul.ctypes.data), float(hp), a.search, a.patch, 3.0,
                                        vp(out.data_ptr()), vp(0), _lib.DSGPU_ASYNC)
        elif a.case == "denoise":
            r = L.dsgpu_denoise(ctx.handle, vp(rgb.data_ptr()), w, h, 50.0, vp(out.data_ptr()), _lib.DSGPU_ASYNC)
        else:
            r = L.dsgpu_develop_u16(ctx.handle, vp(raw.data_ptr()), w, h, w, vp(pat.ctypes.data), 512.0,
                                    vp(white.ctypes.data), vp(mul.ctypes.data), float(hp), a.search, a.patch,
                                    vp(out.data_ptr()), vp(0), _lib.DSGPU_ASYNC | xflags)
        ctx.check(r, a.case)

    net = None
    if a.case in ("cnn", "learned"):
        import os

        from darkslide_b200 import cnn

        net = cnn.ResidualCNN(ctx)
        if a.case == "learned":
            net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    if a.case in ("nlm", "denoise", "cnn"):  # input: the demosaiced frame
        ctx.check(L.dsgpu_demosaic(ctx.handle, vp(cfa.data_ptr()), w, h, vp(pat.ctypes.data), vp(mul.ctypes.data),
                                   _lib.DSGPU_QUALITY_FULL, vp(rgb.data_ptr()), vp(0), 0), "demosaic")
    call()
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(a.reps):
        call()
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    px = w * h * (a.frames if a.case == "batch" else 1)
    print(f"{a.case} {w}x{h}: {ms:.3f} ms per call, {px / ms / 1e3:.1f} Mpix/s")


if __name__ == "__main__":
    main()
