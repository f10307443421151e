"""Train the residual CNN to reproduce plain NLM on synthetic mosaics.

Data: seeded synthetic Bayer frames (darkslide_b200.Scene) with read noise
uniform in 2..12 DN, gain 0.25..1 e/DN, random CFA layout and 12/14-bit
levels, demosaiced on the GPU (RCD); the target is plain GPU NLM of the same
image (7x7 patch, 21x21 search, h = 1.5 x the noise sigma at mid grey).
The data set is a fixed set of `dataset` crop x crop windows of (RCD output,
NLM output, strength map): crops_per_frame windows of each of
dataset / crops_per_frame frames, frame f drawn from seed `seed * 100003 + 1 +
f` (its scene and its window positions), so the same crops come back in every
epoch. Training runs `crops` crop visits (crops / dataset epochs); every epoch
visits the frames in a new order, `mix` frames at a time, and every batch
mixes crops of those frames (so of several noise levels). Each frame is a
512 x 512 window (at an even position) of a scene whose size is drawn
log-uniformly between 512 and 9504 px on the long side: the generator lays
its sinusoids and edges out over the whole scene, so windows of large scenes
are as smooth as a crop of a camera-size frame. The loss is plain MSE
(--relative-loss weights each pixel's squared error by 1 / strength^2). The
learning rate
warms up linearly and then follows a cosine, and the global gradient norm is
clipped at `clip_factor` x the median norm of the first batches. A logged
loss above 5x its running mean (a divergence, after which ReLU units die
and the residual collapses to zero) rolls the whole state (weights and Adam
moments) back to the last healthy snapshot and halves the learning rate. Everything
runs on the GPU through the library; torch only moves tensors.

    python -m darkslide_b200.train_cnn --dataset 200000 --crops 2000000 --out darkslide_b200/weights/cnn_nlm.bin
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


CAMERA_SIZES = [(4000, 3000), (6000, 4000), (8256, 5504), (9504, 6336)]


def draw_virtual(seed: int, w: int, h: int, scenes: str = "any"):
    """A scene size holding a w x h window at an even position: (W, H, x0,
    y0). scenes="any": log-uniform in 512..9504 px on the long side (aspect 1,
    4:3 or 3:2); scenes="camera": one of the camera sizes the path is run on."""
    rng = np.random.default_rng(seed ^ 0xF00D)
    if scenes == "camera":
        W, H = CAMERA_SIZES[int(rng.integers(len(CAMERA_SIZES)))]
    else:
        L = float(np.exp(rng.uniform(np.log(512), np.log(9504))))
        aspect = (1.0, 4 / 3, 1.5)[rng.integers(3)]
        W, H = max(w, int(L)), max(h, int(L / aspect))
    x0 = 2 * int(rng.integers(0, (W - w) // 2 + 1))
    y0 = 2 * int(rng.integers(0, (H - h) // 2 + 1))
    return W, H, x0, y0


def make_frame(seed: int, w: int, h: int, dev, ctx=None, bits=None, gain=None, read_sigma=None, virtual=None):
    """(rgb, target, h_param, scene, (x0, y0)) of a w x h synthetic frame,
    device tensors. bits / gain / read_sigma default to draws from the seed.
    virtual = (W, H, x0, y0): the frame is that window of a W x H scene (the
    generator lays its sinusoids and edges out over the whole W x H, so large
    scenes are smooth at the pixel scale); "draw" draws one (draw_virtual)."""
    rng = np.random.default_rng(seed)
    b_draw = 12 if rng.random() < 0.5 else 14
    pattern = PATTERNS[rng.integers(4)]
    g_draw, r_draw = float(rng.uniform(0.25, 1.0)), float(rng.uniform(2.0, 12.0))
    bits = bits or b_draw
    black, white = (256, 4095) if bits == 12 else (512, 16383)
    if virtual in ("draw", "camera"):
        virtual = draw_virtual(seed, w, h, "camera" if virtual == "camera" else "any")
    W, H, x0, y0 = virtual or (w, h, 0, 0)
    sc = ds.Scene(seed=seed, w=W, h=H, pattern=pattern, black=black, white=white,
                  gain=gain if gain is not None else g_draw,
                  read_sigma=read_sigma if read_sigma is not None else r_draw)
    raw = sc.render(dev, ctx=ctx, window=(x0, y0, w, h))
    # x0, y0 are even, so the window has the frame's CFA layout
    cfa = ds.normalize_u16(raw, sc.pattern, black, np.full(3, white, np.float32), ctx=ctx)
    rgb = ds.rcd_bayer(cfa, [2.0, 1.0, 1.0 / 0.7], ctx=ctx).data
    hp = 1.5 * sc.sigma_norm()
    tgt = ds.nlm(ds.Image3(w, h, rgb), hp, SEARCH, PATCH, ctx=ctx).data
    return rgb, tgt, hp, sc, (x0, y0)


def psnr(a, b, peak=1.0):
    import torch

    mse = float(torch.mean((a - b) ** 2))
    return 10.0 * math.log10(peak * peak / max(mse, 1e-20))


def train(crops=200000, batch=32, crop=128, lr=5e-4, frame=512, crops_per_frame=64, mix=8, warmup=500,
          clip_factor=3.0, seed=0, out=None, resume=None, log_every=200, verbose=True, dataset=200000,
          relative=False, scenes="any", engine="tcgen05"):
    """engine: "tcgen05" (forward, data and weight gradients on the
    5th-generation tensor cores) or "mma.sync" throughout."""
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    ctx = ds.Context(0)
    stream = torch.cuda.Stream(dev)
    net = cnn.ResidualCNN(ctx, max_batch=batch, crop=crop, seed=seed)
    net.set_engine(engine == "tcgen05")
    if resume:
        net.load(resume)
    net.set_loss(relative)
    steps = max(1, crops // batch)
    n_frames = max(mix, dataset // crops_per_frame)
    rng = np.random.default_rng(seed + 12345)
    pool = []
    t0 = time.time()
    losses = []
    queue = []  # frames still to visit in this epoch

    def refill():
        if len(queue) < mix:
            queue.extend(int(f) for f in rng.permutation(n_frames))
        for _ in range(mix):
            fseed = seed * 100003 + 1 + queue.pop()
            rgb, tgt, hp, _, _ = make_frame(fseed, frame, frame, dev, ctx,
                                            virtual="camera" if scenes == "camera" else "draw")
            pos = np.random.default_rng(fseed ^ 0x5EED).integers(0, frame - crop + 1, (crops_per_frame, 2))
            pool.extend((rgb, tgt, hp, int(y), int(x)) for y, x in pos)
        order = rng.permutation(len(pool))
        pool[:] = [pool[i] for i in order]

    def next_batch():
        if len(pool) < batch:
            pool.clear()
            refill()
        take = [pool.pop() for _ in range(batch)]
        xb = torch.stack([r[y:y + crop, x:x + crop] for (r, _, _, y, x) in take]).contiguous()
        tb = torch.stack([t[y:y + crop, x:x + crop] for (_, t, _, y, x) in take]).contiguous()
        hps = np.array([hp * cnn.STRENGTH_SCALE for (_, _, hp, _, _) in take], np.float32)
        smap = torch.from_numpy(hps).pin_memory().to(dev, non_blocking=True)
        smap = smap.view(batch, 1, 1).expand(batch, crop, crop).contiguous()
        return xb, tb, smap

    with torch.cuda.stream(stream):
        if clip_factor > 0:  # clip at a multiple of the typical gradient norm at the start
            norms = []
            for _ in range(8):
                xb, tb, smap = next_batch()
                g, _ = net.gradients(xb, 0.0, tb, strength_map=smap)
                norms.append(float(torch.linalg.vector_norm(g)))
            net.set_clip(clip_factor * float(np.median(norms)))
        scale, ema, snap, rollbacks = 1.0, None, None, 0
        step = net.step
        while step < steps:
            xb, tb, smap = next_batch()
            cur = scale * lr * 0.5 * (1 + math.cos(math.pi * step / steps))  # cosine decay
            if step < warmup:
                cur *= (step + 1) / warmup
            want = (step % log_every == 0) or step == steps - 1
            loss = net.train_step(xb, 0.0, tb, cur, strength_map=smap, want_loss=want)
            step += 1
            if want:
                mse = loss / (batch * crop * crop * 3)
                if ema is not None and mse > 5.0 * ema and snap is not None:
                    net.restore(snap)
                    step = net.step
                    scale *= 0.5
                    rollbacks += 1
                    if verbose:
                        print(f"loss spike {mse:.3e} (mean {ema:.3e}): back to step {step}, lr x{scale}", flush=True)
                    continue
                ema = mse if ema is None else 0.9 * ema + 0.1 * mse
                losses.append((step - 1, mse))
                if (step - 1) % (5 * log_every) == 0:
                    snap = net.snapshot()
                if verbose:
                    print(f"step {step - 1}/{steps} lr {cur:.2e} mse {mse:.3e} ({time.time() - t0:.1f} s)", flush=True)
    stream.synchronize()
    if out:
        net.save(out)
    return net, losses, time.time() - t0


# (bits, gain e/DN, read sigma DN, scene size) of the fixed evaluation grid:
# whole 1024 x 1024 scenes, and central windows of 6000 x 4000 scenes
EVAL_GRID = [(b, 0.5, r, sz) for sz in ((1024, 1024), (6000, 4000)) for b in (12, 14) for r in (2.0, 6.0, 12.0)]


def evaluate(net, n_frames=4, w=1024, h=1024, seed=10_000_999, verbose=True, grid=True):
    """PSNR (dB) against the noise-free scene of the noisy RCD output, plain
    NLM and the CNN, and PSNR of the CNN against NLM, averaged over n_frames
    random frames and (grid) the frames of EVAL_GRID; also the mean and the
    worst PSNR loss of the CNN against NLM. The frame seeds lie far outside
    the training set's."""
    import torch

    dev = torch.device("cuda", 0)
    res = {"noisy": [], "nlm": [], "cnn": [], "cnn_vs_nlm": []}
    cases = [dict()] * n_frames
    if grid:
        for b, g, r, (W, H) in EVAL_GRID:
            virt = (W, H, (W - w) // 2 & ~1, (H - h) // 2 & ~1)
            cases.append(dict(bits=b, gain=g, read_sigma=r, virtual=virt))
    for k, kw in enumerate(cases):
        rgb, tgt, hp, sc, (x0, y0) = make_frame(seed + k, w, h, dev, **kw)
        out = net.infer(ds.Image3(w, h, rgb), hp).data
        truth = torch.from_numpy(sc.truth_host(x0, y0, w, h) * np.array([2.0, 1.0, 1.0 / 0.7], np.float32)).to(dev)
        m = 16  # ignore the frame border
        sl = (slice(m, h - m), slice(m, w - m))
        res["noisy"].append(psnr(rgb[sl], truth[sl]))
        res["nlm"].append(psnr(tgt[sl], truth[sl]))
        res["cnn"].append(psnr(out[sl], truth[sl]))
        res["cnn_vs_nlm"].append(psnr(out[sl], tgt[sl]))
        if verbose and kw:
            print(f"  {kw['bits']}-bit read {kw['read_sigma']} scene {sc.w}x{sc.h}: nlm {res['nlm'][-1]:.2f} cnn {res['cnn'][-1]:.2f} dB", flush=True)
    avg = {k: float(np.mean(v)) for k, v in res.items()}
    loss = np.array(res["nlm"]) - np.array(res["cnn"])
    avg["loss_mean"], avg["loss_max"] = float(loss.mean()), float(loss.max())
    if verbose:
        print("PSNR dB:", {k: round(v, 3) for k, v in avg.items()}, flush=True)
    return avg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--crops", type=int, default=2000000, help="crop visits (epochs = crops / dataset)")
    ap.add_argument("--dataset", type=int, default=200000, help="distinct crops in the training set")
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--frame", type=int, default=512)
    ap.add_argument("--mix", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=500)
    ap.add_argument("--clip", type=float, default=3.0, help="clip factor x initial median gradient norm (0: off)")
    ap.add_argument("--relative-loss", action="store_true", help="weight squared errors by 1 / strength^2")
    ap.add_argument("--scenes", default="any", choices=["any", "camera"],
                    help="scene sizes the training windows come from")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--resume", default=None)
    ap.add_argument("--eval", type=int, default=4)
    ap.add_argument("--engine", default="tcgen05", choices=["tcgen05", "mma.sync"])
    a = ap.parse_args()
    net, losses, secs = train(a.crops, a.batch, a.crop, a.lr, frame=a.frame, mix=a.mix, warmup=a.warmup,
                              clip_factor=a.clip, seed=a.seed, out=a.out, resume=a.resume, dataset=a.dataset,
                              relative=a.relative_loss, scenes=a.scenes, engine=a.engine)
    print(f"trained {a.crops} crop visits of a {a.dataset}-crop set in {secs:.1f} s", flush=True)
    if a.eval:
        evaluate(net, a.eval)


if __name__ == "__main__":
    main()
