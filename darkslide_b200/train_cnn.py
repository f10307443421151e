"""Train the residual CNN to reproduce plain NLM on synthetic mosaics.

Data: seeded synthetic Bayer frames (darkslide_b200.Scene) with read noise
uniform in 2..12 DN, gain 0.25..1 e/DN, random CFA layout and 12/14-bit
levels, demosaiced on the GPU (RCD); the target is plain GPU NLM of the same
image (7x7 patch, 21x21 search, h = 1.5 x the noise sigma at mid grey).
Random crop x crop windows of (RCD output, NLM output, strength map) form the
batches. Everything runs on the GPU through the library; torch only moves
tensors.

    python -m darkslide_b200.train_cnn --crops 200000 --out darkslide_b200/weights/cnn_nlm.bin
"""
from __future__ import annotations

import argparse
import math
import time

import numpy as np

import darkslide_b200 as ds
from darkslide_b200 import cnn

PATTERNS = [ds.RGGB, ds.BGGR, ds.GRBG, ds.GBRG]
SEARCH, PATCH = 10, 3


def make_frame(seed: int, w: int, h: int, dev, ctx=None):
    """(rgb, target, h_param, scene) of one synthetic frame, device tensors."""
    rng = np.random.default_rng(seed)
    bits = 12 if rng.random() < 0.5 else 14
    black, white = (256, 4095) if bits == 12 else (512, 16383)
    sc = ds.Scene(seed=seed, w=w, h=h, pattern=PATTERNS[rng.integers(4)], black=black, white=white,
                  gain=float(rng.uniform(0.25, 1.0)), read_sigma=float(rng.uniform(2.0, 12.0)))
    raw = sc.render(dev, ctx=ctx)
    cfa = ds.normalize_u16(raw, sc.pattern, black, np.full(3, white, np.float32), ctx=ctx)
    rgb = ds.rcd_bayer(cfa, [2.0, 1.0, 1.0 / 0.7], ctx=ctx).data
    hp = 1.5 * sc.sigma_norm()
    tgt = ds.nlm(ds.Image3(w, h, rgb), hp, SEARCH, PATCH, ctx=ctx).data
    return rgb, tgt, hp, sc


def psnr(a, b, peak=1.0):
    import torch

    mse = float(torch.mean((a - b) ** 2))
    return 10.0 * math.log10(peak * peak / max(mse, 1e-20))


def train(crops=200000, batch=32, crop=128, lr=1e-3, frame=1024, crops_per_frame=256, seed=0, out=None,
          resume=None, log_every=200, verbose=True):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    ctx = ds.Context(0)
    stream = torch.cuda.Stream(dev)
    net = cnn.ResidualCNN(ctx, max_batch=batch, crop=crop, seed=seed)
    if resume:
        net.load(resume)
    steps = max(1, crops // batch)
    rng = np.random.default_rng(seed + 12345)
    pool = []
    t0 = time.time()
    losses = []
    with torch.cuda.stream(stream):
        frame_seed = seed * 100003 + 1
        for step in range(net.step, steps):
            if not pool:  # a new frame: crops_per_frame random windows
                rgb, tgt, hp, _ = make_frame(frame_seed, frame, frame, dev, ctx)
                frame_seed += 1
                ys = rng.integers(0, frame - crop + 1, crops_per_frame)
                xs = rng.integers(0, frame - crop + 1, crops_per_frame)
                pool = [(rgb, tgt, hp, int(y), int(x)) for y, x in zip(ys, xs)]
            take = [pool.pop() for _ in range(min(batch, len(pool)))]
            while len(take) < batch:
                take.append(take[len(take) % max(len(take), 1)])
            xb = torch.stack([r[y:y + crop, x:x + crop] for (r, _, _, y, x) in take]).contiguous()
            tb = torch.stack([t[y:y + crop, x:x + crop] for (_, t, _, y, x) in take]).contiguous()
            smap = torch.stack([torch.full((crop, crop), hp * cnn.STRENGTH_SCALE, device=dev)
                                for (_, _, hp, _, _) in take]).contiguous()
            cur = lr * 0.5 * (1 + math.cos(math.pi * step / steps))  # cosine decay
            want = (step % log_every == 0) or step == steps - 1
            loss = net.train_step(xb, 0.0, tb, cur, strength_map=smap, want_loss=want)
            if want:
                mse = loss / (batch * crop * crop * 3)
                losses.append((step, mse))
                if verbose:
                    print(f"step {step}/{steps} lr {cur:.2e} mse {mse:.3e} ({time.time() - t0:.1f} s)", flush=True)
    stream.synchronize()
    if out:
        net.save(out)
    return net, losses, time.time() - t0


def evaluate(net, n_frames=4, w=1024, h=1024, seed=999, verbose=True):
    """PSNR (dB) against the noise-free scene of the noisy RCD output, plain
    NLM and the CNN, and PSNR of the CNN against NLM, averaged over frames."""
    import torch

    dev = torch.device("cuda", 0)
    res = {"noisy": [], "nlm": [], "cnn": [], "cnn_vs_nlm": []}
    for k in range(n_frames):
        rgb, tgt, hp, sc = make_frame(seed + k, w, h, dev)
        out = net.infer(ds.Image3(w, h, rgb), hp).data
        truth = torch.from_numpy(sc.truth_host() * np.array([2.0, 1.0, 1.0 / 0.7], np.float32)).to(dev)
        m = 16  # ignore the frame border
        sl = (slice(m, h - m), slice(m, w - m))
        res["noisy"].append(psnr(rgb[sl], truth[sl]))
        res["nlm"].append(psnr(tgt[sl], truth[sl]))
        res["cnn"].append(psnr(out[sl], truth[sl]))
        res["cnn_vs_nlm"].append(psnr(out[sl], tgt[sl]))
    avg = {k: float(np.mean(v)) for k, v in res.items()}
    if verbose:
        print("PSNR dB:", {k: round(v, 2) for k, v in avg.items()}, flush=True)
    return avg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--crops", type=int, default=200000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--resume", default=None)
    ap.add_argument("--eval", type=int, default=4)
    a = ap.parse_args()
    net, losses, secs = train(a.crops, a.batch, a.crop, a.lr, seed=a.seed, out=a.out, resume=a.resume)
    print(f"trained {a.crops} crops in {secs:.1f} s", flush=True)
    if a.eval:
        evaluate(net, a.eval)


if __name__ == "__main__":
    main()
