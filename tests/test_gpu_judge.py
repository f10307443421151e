"""Judge mode of the learned path: plain GPU NLM recomputes a seeded sample
of the NLM tiles and judges the network's output there (dsgpu_cnn_set_judge).

What is checked, through the C ABI:
  - with every tile sampled and a zero limit, every tile keeps NLM: the
    output is plain NLM's bit for bit;
  - with an unreachable limit, no tile does: the output is the network's;
  - the per-tile decision: sampled tiles whose error (RMS of network - NLM
    over sigma, recomputed here on the CPU) is above the limit hold NLM's
    tile, the others the network's, unsampled tiles the network's;
  - a network forced wrong (output layer zeroed: it returns its noisy input)
    fails every sampled tile at a limit the trained network passes;
  - the band-pipelined host-buffer call equals the device call bit for bit.
"""
import os

import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu

WB = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
S, P = 10, 3
TW, TH = 16, 64 - 2 * P  # the NLM tile of the one-frame kernel (nlm_tile.cuh: NLM_TX x (64 - 2P))
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "darkslide_b200", "weights",
                       "cnn_nlm.bin")


@pytest.fixture(scope="module")
def setup():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build, cnn

    build.build()
    dev = torch.device("cuda", 0)
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(WEIGHTS)
    sc = ds.Scene(seed=91, w=700, h=500, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    hp = 1.5 * sc.sigma_norm()
    raw = sc.render(dev, ctx=ctx)
    rgb = ds.develop_u16(raw, ds.RGGB, 512, [16383.0] * 3, WB, hp, 0, P, ctx=ctx).data  # the demosaic alone
    nlm = ds.nlm(ds.Image3(sc.w, sc.h, rgb), hp, S, P, ctx=ctx).data  # plain NLM of the same frame
    torch.cuda.synchronize()
    return torch, dev, ctx, net, sc, hp, rgb, nlm.cpu().numpy()


def _denoise(net, rgb, w, h, hp, tau=0.0):
    out, _ = net.denoise(ds.Image3(w, h, rgb), hp, S, P, tau)
    return out.data.cpu().numpy()


def _tiles(w, h):
    return -(-w // TW), -(-h // TH)


def _tile_view(a, tx, ty):
    return a[ty * TH:(ty + 1) * TH, tx * TW:(tx + 1) * TW]


def _tile_errors(cnn_out, nlm, w, h, sigma):
    tx, ty = _tiles(w, h)
    return np.array([[np.sqrt(np.mean((_tile_view(cnn_out, x, y).astype(np.float64) - _tile_view(nlm, x, y)) ** 2))
                      / sigma for x in range(tx)] for y in range(ty)])


def test_sample_depends_only_on_seed_and_fraction():
    from darkslide_b200 import _lib

    L = _lib.lib()
    a = [L.dsgpu_cnn_judge_tile(7, 0.25, t) for t in range(4000)]
    assert a == [L.dsgpu_cnn_judge_tile(7, 0.25, t) for t in range(4000)]
    assert 0.2 < sum(a) / 4000 < 0.3
    assert a != [L.dsgpu_cnn_judge_tile(8, 0.25, t) for t in range(4000)]
    assert sum(L.dsgpu_cnn_judge_tile(7, 1.0, t) for t in range(1000)) == 1000
    assert sum(L.dsgpu_cnn_judge_tile(7, 0.0, t) for t in range(1000)) == 0
    assert L.dsgpu_cnn_judge_tile(7, 1.5, 0) == _lib.DSGPU_ERR_ARG


def test_all_tiles_zero_limit_is_plain_nlm(setup):
    torch, dev, ctx, net, sc, hp, rgb, nlm = setup
    net.set_judge(1.0, 0.0, seed=3)
    try:
        got = _denoise(net, rgb, sc.w, sc.h, hp)
        st = net.judge_stats()
    finally:
        net.set_judge(0.0)
    tx, ty = _tiles(sc.w, sc.h)
    assert st["judged"] == tx * ty and st["failed"] == tx * ty, st
    np.testing.assert_array_equal(got, nlm)


def test_unreachable_limit_keeps_the_network(setup):
    torch, dev, ctx, net, sc, hp, rgb, nlm = setup
    plain_net = _denoise(net, rgb, sc.w, sc.h, hp)
    net.set_judge(1.0, 1e30, seed=3)
    try:
        got = _denoise(net, rgb, sc.w, sc.h, hp)
        st = net.judge_stats()
    finally:
        net.set_judge(0.0)
    assert st["failed"] == 0, st
    np.testing.assert_array_equal(got, plain_net)


def test_per_tile_decision(setup):
    from darkslide_b200 import _lib

    torch, dev, ctx, net, sc, hp, rgb, nlm = setup
    L = _lib.lib()
    cnn_out = _denoise(net, rgb, sc.w, sc.h, hp)
    tx, ty = _tiles(sc.w, sc.h)
    err = _tile_errors(cnn_out, nlm, sc.w, sc.h, hp / 1.5)
    limit = float(np.median(err))
    seed, frac = 11, 0.5
    net.set_judge(frac, limit, seed=seed)
    try:
        got = _denoise(net, rgb, sc.w, sc.h, hp)
        st = net.judge_stats()
    finally:
        net.set_judge(0.0)
    sampled = 0
    for y in range(ty):
        for x in range(tx):
            g = _tile_view(got, x, y)
            if not L.dsgpu_cnn_judge_tile(seed, frac, y * tx + x):
                np.testing.assert_array_equal(g, _tile_view(cnn_out, x, y))
                continue
            sampled += 1
            if err[y, x] > limit * 1.01:
                np.testing.assert_array_equal(g, _tile_view(nlm, x, y))
            elif err[y, x] < limit * 0.99:
                np.testing.assert_array_equal(g, _tile_view(cnn_out, x, y))
    assert st["judged"] == sampled > 0, (st, sampled)
    assert 0 < st["failed"] < sampled
    print(f"\njudge: {sampled} of {tx * ty} tiles sampled, {st['failed']} kept NLM at limit {limit:.3f} sigma; "
          f"network error vs NLM: rms {st['rms_over_sigma']:.3f}, max {st['max_rms_over_sigma']:.3f} sigma")


def test_forced_wrong_network_fails_the_judge(setup):
    from darkslide_b200 import _lib, cnn

    torch, dev, ctx, net, sc, hp, rgb, nlm = setup
    sigma = hp / 1.5
    good_err = _tile_errors(_denoise(net, rgb, sc.w, sc.h, hp), nlm, sc.w, sc.h, sigma)
    broken = cnn.ResidualCNN(ctx)
    broken.load(WEIGHTS)
    p = broken.get_params()
    p[-(9 * 48 * 3 + 3):] = 0.0  # the output layer (48 -> 3, 3x3, + bias): the residual is zero, out = noisy input
    broken.set_params(p)
    bad_err = _tile_errors(_denoise(broken, rgb, sc.w, sc.h, hp), nlm, sc.w, sc.h, sigma)
    # a limit between what the trained network does and what the broken one does
    limit = float(np.sqrt(good_err.max() * bad_err.min()))
    assert good_err.max() < limit < bad_err.min(), (good_err.max(), bad_err.min())
    for which, m in (("good", net), ("bad", broken)):
        m.set_judge(0.25, limit, seed=5)
    try:
        _denoise(net, rgb, sc.w, sc.h, hp)
        good = net.judge_stats()
        got = _denoise(broken, rgb, sc.w, sc.h, hp)
        bad = broken.judge_stats()
    finally:
        net.set_judge(0.0)
    print(f"\njudge at {limit:.3f} sigma: trained network tile error {good_err.mean():.3f} (max {good_err.max():.3f}) "
          f"sigma, {good['failed']} of {good['judged']} fail; zeroed output layer {bad_err.mean():.3f} sigma, "
          f"{bad['failed']} of {bad['judged']} fail")
    assert good["judged"] == bad["judged"] > 0
    assert good["failed"] == 0, good
    assert bad["failed"] == bad["judged"], bad
    L = _lib.lib()  # the failed tiles hold NLM's result
    tx, ty = _tiles(sc.w, sc.h)
    for t in range(tx * ty):
        if L.dsgpu_cnn_judge_tile(5, 0.25, t):
            x, y = t % tx, t // tx
            np.testing.assert_array_equal(_tile_view(got, x, y), _tile_view(nlm, x, y))


@pytest.mark.parametrize("tau", [0.0, 3.0])
def test_band_pipeline_equals_device_call_under_judge(setup, tau):
    torch, dev, ctx, net, sc, hp, rgb, nlm = setup
    raw = sc.render(dev, ctx=ctx)
    net.set_judge(0.3, 0.2, seed=9)
    try:
        a = net.develop_u16(raw, ds.RGGB, 512, [16383.0] * 3, WB, hp, S, P, tau).data.cpu().numpy()
        sa = net.judge_stats()
        b = net.develop_u16(raw.cpu().numpy(), ds.RGGB, 512, [16383.0] * 3, WB, hp, S, P, tau).data
        sb = net.judge_stats()
    finally:
        net.set_judge(0.0)
    np.testing.assert_array_equal(b, a)
    assert (sa["judged"], sa["failed"]) == (sb["judged"], sb["failed"]) and sa["judged"] > 0
