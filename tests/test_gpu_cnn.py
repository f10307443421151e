"""The learned path's tensor-core kernels against the FP64 reference
(oracle/cnn_ref.py), plus Adam, checkpoint/resume and training.

The GPU keeps weights, inputs, activations and gradients in BF16 (8-bit
mantissa) with FP32 accumulation, so it is compared with an FP64 reference fed
the same BF16-rounded weights and packed inputs (cnn_ref.pack_input): outputs to 2e-2 of their scale,
gradients per layer by cosine similarity >= 0.995 and relative L2 error
<= 5e-2."""
import os

import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_dev():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch, torch.device("cuda", 0)


def _batch(torch, dev, B, crop, seed):
    rng = np.random.default_rng(seed)
    rgb = rng.uniform(0.05, 0.9, (B, crop, crop, 3)).astype(np.float32)
    tgt = (rgb + rng.normal(0, 0.02, rgb.shape)).astype(np.float32)
    return rgb, tgt, torch.from_numpy(rgb).to(dev), torch.from_numpy(tgt).to(dev)


def test_forward_matches_fp64(torch_dev):
    import cnn_ref as C
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    p = cnn.init_params(3)
    p[-1299:] = np.random.default_rng(3).normal(0, 0.05, 1299)  # a non-zero last layer
    net = cnn.ResidualCNN(params=p)
    rgb = np.random.default_rng(1).uniform(0.05, 0.9, (37, 45, 3)).astype(np.float32)
    out = net.infer(ds.Image3(45, 37, rgb), 0.01).data
    s = 0.01 * cnn.STRENGTH_SCALE
    ref, _ = C.forward(C.bf16_round(p), C.bf16_round(C.pack_input(rgb[None], s)), rgb[None])
    ref = ref[0]
    scale = np.abs(ref - rgb).max()
    assert np.abs(out - ref).max() <= 2e-2 * max(scale, 1e-3)


@pytest.mark.parametrize("engine", ["tcgen05", "mma.sync"])
@pytest.mark.parametrize("crop", [16, 18, 20])
def test_gradients_match_fp64(torch_dev, crop, engine):
    """Per-layer weight and bias gradients of a batch against the FP64
    reference, on either engine: tcgen05 (forward, data and weight gradients
    on the 5th-generation tensor cores over the batch laid out as one frame
    of crops; crop 18 leaves two zero padding columns per frame row) or
    mma.sync throughout."""
    import cnn_ref as C
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    p = cnn.init_params(5)
    p[-1299:] = np.random.default_rng(5).normal(0, 0.05, 1299)
    net = cnn.ResidualCNN(max_batch=2, crop=crop, params=p)
    net.set_engine(engine == "tcgen05")
    rgb, tgt, trgb, ttgt = _batch(torch, dev, 2, crop, 7)
    s = 0.5
    g, loss = net.gradients(trgb, s, ttgt)
    g = g.cpu().numpy()
    gr, loss_r = C.gradients(C.bf16_round(p), C.bf16_round(C.pack_input(rgb, s)), rgb, tgt)
    assert abs(loss - loss_r) <= 2e-2 * loss_r
    for i, (ws, bs, _) in enumerate(cnn.layer_slices()):
        for sl in (ws, bs):
            a, b = g[sl], gr[sl]
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            rel = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
            assert cos >= 0.995 and rel <= 5e-2, (i, sl, cos, rel)


@pytest.mark.parametrize("engine", ["tcgen05", "mma.sync"])
def test_relative_loss_gradients_match_fp64(torch_dev, engine):
    """Loss weighted by 1 / strength^2 with a strength map that differs per crop."""
    import cnn_ref as C
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    crop = 16
    p = cnn.init_params(6)
    p[-1299:] = np.random.default_rng(6).normal(0, 0.05, 1299)
    net = cnn.ResidualCNN(max_batch=2, crop=crop, params=p)
    net.set_engine(engine == "tcgen05")
    net.set_loss(True)
    rgb, tgt, trgb, ttgt = _batch(torch, dev, 2, crop, 8)
    smap = np.stack([np.full((crop, crop), 0.3, np.float32), np.full((crop, crop), 1.7, np.float32)])
    g, loss = net.gradients(trgb, 0.0, ttgt, strength_map=torch.from_numpy(smap).to(dev))
    g = g.cpu().numpy()
    gr, loss_r = C.gradients(C.bf16_round(p), C.bf16_round(C.pack_input(rgb, smap)), rgb, tgt,
                             weight=1.0 / smap.astype(np.float64) ** 2)
    assert abs(loss - loss_r) <= 2e-2 * loss_r
    for i, (ws, bs, _) in enumerate(cnn.layer_slices()):
        for sl in (ws, bs):
            a, b = g[sl], gr[sl]
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            rel = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
            assert cos >= 0.995 and rel <= 5e-2, (i, sl, cos, rel)


def test_adam_step_and_bit_identical_resume(torch_dev, tmp_path):
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    batches = [_batch(torch, dev, 2, 16, 20 + k)[2:] for k in range(5)]
    net = cnn.ResidualCNN(max_batch=2, crop=16, seed=9)
    p0 = net.get_params()
    g, _ = net.gradients(*batches[0][:1], 0.5, batches[0][1])
    net.train_step(batches[0][0], 0.5, batches[0][1], 1e-3)
    # first Adam step: m = 0.1 g, v = 0.001 g^2 -> update = lr * g / (|g| + eps)
    g = g.cpu().numpy()
    exp = p0 - 1e-3 * g / (np.abs(g) + 1e-8)
    np.testing.assert_allclose(net.get_params(), exp, rtol=1e-5, atol=1e-8)
    for k in range(1, 3):
        net.train_step(batches[k][0], 0.5, batches[k][1], 1e-3)
    path = os.path.join(tmp_path, "ck.bin")
    net.save(path)
    for k in range(3, 5):
        net.train_step(batches[k][0], 0.5, batches[k][1], 1e-3)
    direct = net.get_params()
    net2 = cnn.ResidualCNN(max_batch=2, crop=16, seed=1)
    net2.load(path)
    assert net2.step == 3
    for k in range(3, 5):
        net2.train_step(batches[k][0], 0.5, batches[k][1], 1e-3)
    np.testing.assert_array_equal(net2.get_params(), direct)


def test_adam_gradient_norm_clip(torch_dev):
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    b1, b2 = (_batch(torch, dev, 2, 16, 40 + k)[2:] for k in range(2))
    net = cnn.ResidualCNN(max_batch=2, crop=16, seed=4)
    p0 = net.get_params().astype(np.float64)
    g1, _ = net.gradients(b1[0], 0.5, b1[1])
    g1 = g1.cpu().numpy().astype(np.float64)
    clip = 0.5 * np.linalg.norm(g1)
    net.set_clip(clip)
    net.train_step(b1[0], 0.5, b1[1], 1e-3)
    p1 = net.get_params().astype(np.float64)
    g2, _ = net.gradients(b2[0], 0.5, b2[1])
    g2 = g2.cpu().numpy().astype(np.float64)
    net.train_step(b2[0], 0.5, b2[1], 1e-3)

    def clipped(g):
        n = np.linalg.norm(g)
        return g * min(1.0, clip / n)

    c1, c2 = clipped(g1), clipped(g2)
    m1, v1 = 0.1 * c1, 0.001 * c1 * c1
    m2, v2 = 0.9 * m1 + 0.1 * c2, 0.999 * v1 + 0.001 * c2 * c2
    exp = p1 - 1e-3 * (m2 / (1 - 0.9 ** 2)) / (np.sqrt(v2 / (1 - 0.999 ** 2)) + 1e-8)
    assert np.abs(p1 - p0).max() > 0
    np.testing.assert_allclose(net.get_params(), exp, rtol=1e-4, atol=1e-7)


def test_tensor_core_training_matches_mma_sync(torch_dev):
    """The two training engines on a batch of 4 crops of 32 (smaller than the
    batch the network was created for): the same loss and gradients up to
    BF16 rounding of the activations."""
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    p = cnn.init_params(12)
    p[-1299:] = np.random.default_rng(12).normal(0, 0.05, 1299)
    net = cnn.ResidualCNN(max_batch=6, crop=32, params=p)
    rgb, tgt, trgb, ttgt = _batch(torch, dev, 4, 32, 13)
    g_tc, l_tc = net.gradients(trgb, 0.4, ttgt)
    net.set_engine(False)
    g_ms, l_ms = net.gradients(trgb, 0.4, ttgt)
    g_tc, g_ms = g_tc.cpu().numpy(), g_ms.cpu().numpy()
    assert abs(l_tc - l_ms) <= 1e-2 * l_ms
    for i, (ws, bs, _) in enumerate(cnn.layer_slices()):
        for sl in (ws, bs):
            a, b = g_tc[sl], g_ms[sl]
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos >= 0.995, (i, sl, cos)


@pytest.mark.parametrize("crop", [72, 128])
def test_tensor_core_gradients_at_wide_crops(torch_dev, crop):
    """Crops wider than the weight-gradient kernel's 64-pixel chunk: a frame
    row then holds two chunks (the second one ragged at 72, whole at the
    training crop 128), loaded at a non-zero start pixel. Both engines agree
    on the loss and every layer's weight and bias gradients up to BF16
    rounding of the activations."""
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    p = cnn.init_params(21)
    p[-1299:] = np.random.default_rng(21).normal(0, 0.05, 1299)
    net = cnn.ResidualCNN(max_batch=2, crop=crop, params=p)
    rgb, tgt, trgb, ttgt = _batch(torch, dev, 2, crop, 22)
    g_tc, l_tc = net.gradients(trgb, 0.4, ttgt)
    net.set_engine(False)
    g_ms, l_ms = net.gradients(trgb, 0.4, ttgt)
    g_tc, g_ms = g_tc.cpu().numpy(), g_ms.cpu().numpy()
    assert abs(l_tc - l_ms) <= 1e-2 * l_ms
    for i, (ws, bs, _) in enumerate(cnn.layer_slices()):
        for sl in (ws, bs):
            a, b = g_tc[sl], g_ms[sl]
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos >= 0.995, (crop, i, sl, cos)


def test_training_reduces_loss(torch_dev):
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    rng = np.random.default_rng(0)
    clean = np.repeat(rng.uniform(0.2, 0.8, (8, 1, 1, 3)), 32, 1).repeat(32, 2).astype(np.float32)
    noisy = (clean + rng.normal(0, 0.05, clean.shape)).astype(np.float32)
    x, t = torch.from_numpy(noisy).to(dev), torch.from_numpy(clean).to(dev)
    net = cnn.ResidualCNN(max_batch=8, crop=32, seed=2)
    first = net.train_step(x, 0.5, t, 2e-3)
    for _ in range(300):
        last = net.train_step(x, 0.5, t, 2e-3)
    assert last < 0.8 * first, (first, last)


@pytest.mark.parametrize("hw", [(37, 45), (130, 300), (256, 129)])
def test_tensor_core_engine_matches_mma_sync_and_fp64(torch_dev, hw):
    """tcgen05 inference (default engine) against the mma.sync kernels and the
    FP64 reference on the same weights."""
    import cnn_ref as C
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    h, w = hw
    p = cnn.init_params(11)
    p[-1299:] = np.random.default_rng(11).normal(0, 0.05, 1299)
    net = cnn.ResidualCNN(params=p)
    rgb = np.random.default_rng(h).uniform(0.05, 0.9, (h, w, 3)).astype(np.float32)
    tc = net.infer(ds.Image3(w, h, rgb), 0.01).data
    net.set_engine(False)
    ms = net.infer(ds.Image3(w, h, rgb), 0.01).data
    ref, _ = C.forward(C.bf16_round(p), C.bf16_round(C.pack_input(rgb[None], 0.5)), rgb[None])
    ref = ref[0]
    scale = max(np.abs(ref - rgb).max(), 1e-3)
    assert np.isfinite(tc).all()
    assert np.abs(tc - ms).max() <= 2e-2 * scale
    assert np.abs(tc - ref).max() <= 2e-2 * scale


QUALITY_BOUND_DB = 0.1  # the learned path's allowed PSNR loss against NLM


def test_quality_bound_on_held_out_grid(torch_dev):
    """The committed network on the held-out evaluation grid (12- and 14-bit,
    read noise 2, 6 and 12 DN, 1024x1024 frames and 1024x1024 windows of
    6000x4000 scenes, plus four random frames; seeds outside the training
    set): on every frame its PSNR against the noise-free scene is at most
    0.1 dB below plain GPU NLM's."""
    from darkslide_b200 import cnn, train_cnn

    torch, dev = torch_dev
    net = cnn.ResidualCNN(ds.Context(0))
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    r = train_cnn.evaluate(net, n_frames=4, verbose=False)
    print(f"\nheld-out grid: NLM {r['nlm']:.3f} dB, network {r['cnn']:.3f} dB, loss mean {r['loss_mean']:+.3f} "
          f"worst {r['loss_max']:+.3f} dB")
    assert r["loss_max"] <= QUALITY_BOUND_DB, r


def test_quality_against_fp64_oracle(torch_dev, oracle):
    """On a 1024x1024 crop of a camera-size frame (14-bit RGGB, read noise 6 DN),
    the learned output's PSNR against the noise-free scene is at most 0.1 dB
    below the FP64 oracle's RCD + NLM (oracle/dsref.cpp in double precision);
    plain GPU NLM is within 0.01 dB of it. (A 256x256 crop of the same frame
    measured a 0.137 dB loss: on a crop that small the PSNR difference of two
    denoisers is dominated by which structures it happens to hold.)"""
    from darkslide_b200 import cnn, train_cnn

    torch, dev = torch_dev
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    W, H, c = 6000, 4000, 1024
    m = 64  # > RCD + NLM radius (23) and the network's 36-row reach; even, so the window stays RGGB
    x0, y0 = (W // 2 - c // 2) & ~1, (H // 2 - c // 2) & ~1
    ax, ay, aw, ah = x0 - m, y0 - m, c + 2 * m, c + 2 * m
    sc = ds.Scene(seed=64_000_003, w=W, h=H, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render(dev, ctx=ctx, window=(ax, ay, aw, ah))
    hp = 1.5 * sc.sigma_norm()
    white = np.full(3, 16383, np.float32)
    mul = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
    learned = net.develop_u16(raw, ds.RGGB, 512, white, mul, hp, 10, 3, 3.0).data.cpu().numpy()
    plain = ds.develop_u16(raw, ds.RGGB, 512, white, mul, hp, 10, 3, ctx=ctx).data.cpu().numpy()
    raw_h = raw.cpu().numpy()
    cfa = oracle.normalize_u16(raw_h, ds.RGGB.codes(), 512, white)
    ref64 = oracle.nlm_rgb(oracle.rcd(cfa, ds.RGGB.codes(), mul, fp64=True), hp, 10, 3, fp64=True)
    truth = sc.truth_host(ax, ay, aw, ah).astype(np.float64) * mul
    sl = (slice(m, m + c), slice(m, m + c))

    def psnr(a):
        return 10 * np.log10(1.0 / np.mean((a[sl].astype(np.float64) - truth[sl]) ** 2))

    p64, pl, pg = psnr(ref64), psnr(learned), psnr(plain)
    print(f"\n1024x1024 crop vs truth: FP64 oracle {p64:.3f} dB, plain GPU {pg:.3f} dB, learned {pl:.3f} dB "
          f"(loss {p64 - pl:+.3f} dB)")
    assert abs(pg - p64) <= 0.01
    assert p64 - pl <= QUALITY_BOUND_DB


def test_trained_network_gain(torch_dev):
    """The committed network against the method without it, on a held-out
    14-bit frame (read noise 6 DN): it removes most of the noise that plain
    NLM removes (>= 5 dB over the undenoised RCD output, within 0.1 dB of
    NLM) and the learned develop is faster than the plain one."""
    from darkslide_b200 import _lib, cnn, train_cnn

    torch, dev = torch_dev
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    w = h = 1024
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        rgb, tgt, hp, sc, _ = train_cnn.make_frame(77_000_001, w, h, dev, ctx, bits=14, gain=0.5, read_sigma=6.0)
        out = net.infer(ds.Image3(w, h, rgb), hp).data
    stream.synchronize()
    truth = torch.from_numpy(sc.truth_host() * np.array([2.0, 1.0, 1.0 / 0.7], np.float32)).to(dev)
    sl = (slice(16, h - 16), slice(16, w - 16))
    p_noisy, p_nlm, p_cnn = (train_cnn.psnr(a[sl], truth[sl]) for a in (rgb, tgt, out))
    assert p_cnn >= p_noisy + 5.0, (p_noisy, p_cnn)
    assert p_cnn >= p_nlm - QUALITY_BOUND_DB, (p_nlm, p_cnn)

    # speed at 2048 x 2048: learned develop (RCD + CNN + fallback check) vs plain (RCD + NLM)
    W = H = 2048
    scene = ds.Scene(seed=5, w=W, h=H, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    L = _lib.lib()
    vp = __import__("ctypes").c_void_p
    pat = ds.RGGB.codes()
    white = np.full(3, 16383, np.float32)
    mul = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
    hpar = 1.5 * scene.sigma_norm()
    with torch.cuda.stream(stream):
        raw = scene.render(dev, ctx=ctx)
        o = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    ctx.set_stream(stream.cuda_stream)

    def plain():
        ctx.check(L.dsgpu_develop_u16(ctx.handle, vp(raw.data_ptr()), W, H, W, vp(pat.ctypes.data), 512.0,
                                      vp(white.ctypes.data), vp(mul.ctypes.data), float(hpar), 10, 3,
                                      vp(o.data_ptr()), vp(0), _lib.DSGPU_ASYNC), "develop")

    def learned():
        ctx.check(L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, vp(raw.data_ptr()), W, H, W, vp(pat.ctypes.data),
                                          512.0, vp(white.ctypes.data), vp(mul.ctypes.data), float(hpar), 10, 3,
                                          3.0, vp(o.data_ptr()), vp(0), _lib.DSGPU_ASYNC), "develop_cnn")

    def timed(f, n=10):
        for _ in range(3):
            f()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            f()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    t_plain, t_learned = timed(plain), timed(learned)
    assert t_learned * 1.3 < t_plain, (t_plain, t_learned)


@pytest.mark.parametrize("w,h", [(2048, 1536), (1000, 777), (300, 130), (96, 40)])
@pytest.mark.parametrize("tau", [3.0, 0.5, 0.0])
def test_host_buffer_learned_develop_equals_device_call(torch_dev, w, h, tau):
    """With host buffers (DSGPU_HOST) the learned develop runs as a band
    pipeline: the network on bands of rows with an 18-row halo, the residual
    check and NLM fallback per band, copies overlapped. Its output and clip
    plane equal the device-buffer call's bit for bit (tau 0.5 sends many tiles
    to the fallback, tau 0 none)."""
    from darkslide_b200 import _lib, cnn

    torch, dev = torch_dev
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    L = _lib.lib()
    vp = __import__("ctypes").c_void_p
    pat = ds.GRBG.codes()
    white = np.full(3, 16383, np.float32)
    mul = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
    scene = ds.Scene(seed=w + h, w=w, h=h, pattern=ds.GRBG, black=512, white=16383, gain=0.5, read_sigma=8)
    hpar = 1.5 * scene.sigma_norm()
    raw = scene.render(dev, ctx=ctx)
    torch.cuda.synchronize()
    o = torch.empty((h, w, 3), dtype=torch.float32, device=dev)
    oc = torch.empty((h, w), dtype=torch.float32, device=dev)
    ctx.check(L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, vp(raw.data_ptr()), w, h, w, vp(pat.ctypes.data),
                                      512.0, vp(white.ctypes.data), vp(mul.ctypes.data), float(hpar), 10, 3,
                                      tau, vp(o.data_ptr()), vp(oc.data_ptr()), 0), "develop_cnn device")
    raw_h = raw.cpu().pin_memory()
    out_h = torch.full((h, w, 3), -1.0, dtype=torch.float32).pin_memory()
    clip_h = torch.full((h, w), -1.0, dtype=torch.float32).pin_memory()
    for _ in range(2):  # the second call reuses the context's buffers and events
        ctx.check(L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, vp(raw_h.data_ptr()), w, h, w,
                                          vp(pat.ctypes.data), 512.0, vp(white.ctypes.data), vp(mul.ctypes.data),
                                          float(hpar), 10, 3, tau, vp(out_h.data_ptr()), vp(clip_h.data_ptr()),
                                          _lib.DSGPU_HOST), "develop_cnn host")
        np.testing.assert_array_equal(out_h.numpy(), o.cpu().numpy())
        np.testing.assert_array_equal(clip_h.numpy(), oc.cpu().numpy())
        out_h.fill_(-1.0)


def test_python_learned_develop(torch_dev):
    """ResidualCNN.develop_u16: the same result from a CUDA tensor (device
    call) and from numpy (host-buffer band pipeline), with the clip plane."""
    from darkslide_b200 import cnn

    torch, dev = torch_dev
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    w, h = 700, 450
    scene = ds.Scene(seed=31, w=w, h=h, pattern=ds.BGGR, black=512, white=16383, gain=0.5, read_sigma=6)
    hp = 1.5 * scene.sigma_norm()
    raw = scene.render(dev, ctx=ctx)
    torch.cuda.synchronize()
    args = (ds.BGGR, 512, [16383.0] * 3, [2.0, 1.0, 1.0 / 0.7], hp)
    img_d, clip_d = net.develop_u16(raw, *args, with_clip=True)
    img_h, clip_h = net.develop_u16(raw.cpu().numpy(), *args, with_clip=True)
    np.testing.assert_array_equal(np.asarray(img_h.data), img_d.data.cpu().numpy())
    np.testing.assert_array_equal(np.asarray(clip_h.data), clip_d.data.cpu().numpy())
    plain = ds.develop_u16(raw, ds.BGGR, 512, [16383.0] * 3, [2.0, 1.0, 1.0 / 0.7], hp, 10, 3).data.cpu().numpy()
    assert np.abs(img_d.data.cpu().numpy() - plain).mean() < 2e-3  # a denoised image close to NLM's


def test_learned_develop_composes_and_rejects(torch_dev):
    """dsgpu_develop_u16_cnn equals RCD (dsgpu_develop_u16 with search 0, an
    identity NLM) followed by dsgpu_cnn_denoise, bit for bit, on ragged and
    thin frames; and it rejects what the header says it rejects."""
    from darkslide_b200 import _lib, cnn

    torch, dev = torch_dev
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    L = _lib.lib()
    vp = __import__("ctypes").c_void_p
    white = np.full(3, 16383, np.float32)
    mul = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
    for k, (w, h, pat) in enumerate([(16, 16, ds.RGGB), (211, 16, ds.GBRG), (16, 190, ds.GRBG), (333, 257, ds.BGGR)]):
        sc = ds.Scene(seed=900 + k, w=w, h=h, pattern=pat, black=512, white=16383, gain=0.5, read_sigma=9)
        hp = 1.5 * sc.sigma_norm()
        raw = sc.render(dev, ctx=ctx)
        torch.cuda.synchronize()
        codes = pat.codes()
        got = torch.empty((h, w, 3), dtype=torch.float32, device=dev)
        ctx.check(L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, vp(raw.data_ptr()), w, h, w, vp(codes.ctypes.data),
                                          512.0, vp(white.ctypes.data), vp(mul.ctypes.data), float(hp), 10, 3, 0.5,
                                          vp(got.data_ptr()), vp(0), 0), "develop_cnn")
        rgb = ds.develop_u16(raw, pat, 512, white, mul, hp, 0, 3, ctx=ctx)  # search 0: RCD output
        exp, _ = net.denoise(rgb, hp, 10, 3, 0.5)
        np.testing.assert_array_equal(got.cpu().numpy(), exp.data.cpu().numpy())
    raw = torch.zeros((40, 40), dtype=torch.int16, device=dev)
    o = torch.empty((40, 40, 3), dtype=torch.float32, device=dev)

    def call(w, h, search=10, patch=3, codes=ds.RGGB.codes(), rawp=None):
        return L.dsgpu_develop_u16_cnn(ctx.handle, net.handle, rawp if rawp is not None else vp(raw.data_ptr()), w, h,
                                       w, vp(codes.ctypes.data), 512.0, vp(white.ctypes.data), vp(mul.ctypes.data),
                                       0.01, search, patch, 3.0, vp(o.data_ptr()), vp(0), 0)

    assert call(15, 40) == _lib.DSGPU_ERR_UNSUPPORTED
    assert call(40, 15) == _lib.DSGPU_ERR_UNSUPPORTED
    assert call(40, 40, search=0) == _lib.DSGPU_ERR_ARG
    assert call(40, 40, patch=99) == _lib.DSGPU_ERR_ARG
    assert call(40, 40, codes=np.array([0, 1, 3, 2], np.uint8)) == _lib.DSGPU_ERR_CFA
    assert call(40, 40, rawp=vp(0)) == _lib.DSGPU_ERR_ARG
    assert call(0, 0) == _lib.DSGPU_OK  # empty: nothing to do
