"""Batched develop (dsgpu_rcd_nlm_batch) and its autotuner on the GPU.

Every frame of a batch runs the same per-tile device code as the one-frame
path, so its output must equal dsgpu_develop_u16's bit for bit, whatever the
RCD tile shape the table chose for its size class."""
import numpy as np
import pytest

import darkslide_b200 as ds
from darkslide_b200 import _lib

pytestmark = pytest.mark.gpu

PATTERNS = [ds.RGGB, ds.BGGR, ds.GRBG, ds.GBRG]
SHAPES = [(32, 32), (64, 16), (48, 24), (24, 48), (16, 64)]
# (w, h, bits, read sigma): ragged sizes, thin frames, both bit depths
CASES = [(300, 200, 14, 6.0), (517, 333, 12, 2.0), (64, 48, 14, 12.0), (1000, 37, 12, 6.0), (129, 1025, 14, 3.0)]


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch, torch.device("cuda", 0)


def make_frames(torch, dev, cases, seed=0):
    frames = []
    for k, (w, h, bits, rs) in enumerate(cases):
        black, white = (256, 4095) if bits == 12 else (512, 16383)
        pat = PATTERNS[k % 4]
        sc = ds.Scene(seed=seed + k, w=w, h=h, pattern=pat, black=black, white=white, gain=0.5, read_sigma=rs)
        raw = sc.render(dev)
        hp = 1.5 * sc.sigma_norm()
        frames.append(ds.BatchFrame(raw=raw, pattern=pat, black=black, white=[white] * 3,
                                    mul=[2.0, 1.0, 1.0 / 0.7], h_param=hp,
                                    out=torch.empty((h, w, 3), dtype=torch.float32, device=dev),
                                    clip=torch.empty((h, w), dtype=torch.float32, device=dev)))
    torch.cuda.synchronize()
    return frames


def single(f, search, patch, ctx):
    img, clip = ds.develop_u16(f.raw, f.pattern, f.black, f.white, f.mul, f.h_param, search, patch,
                               with_clip=True, ctx=ctx)
    return img.data.cpu().numpy(), clip.data.cpu().numpy()


@pytest.mark.parametrize("shape_offset", range(len(SHAPES)))
def test_batch_equals_one_frame_path(env, shape_offset):
    torch, dev = env
    ctx = ds.Context(0)
    frames = make_frames(torch, dev, CASES)
    for k, (w, h, _, _) in enumerate(CASES):  # every frame a different tile shape
        ds.autotune_set(w, h, SHAPES[(k + shape_offset) % len(SHAPES)], 1 + (k + shape_offset) % 2, ctx=ctx)
    ds.develop_batch(frames, 10, 3, ctx=ctx)
    for f in frames:
        rgb, clip = single(f, 10, 3, ctx)
        np.testing.assert_array_equal(f.out.cpu().numpy(), rgb)
        np.testing.assert_array_equal(f.clip.cpu().numpy(), clip)


def test_graph_replay_picks_up_new_strengths_and_buffers(env):
    torch, dev = env
    ctx = ds.Context(0)
    frames = make_frames(torch, dev, CASES[:3], seed=40)
    ds.develop_batch(frames, 4, 2, ctx=ctx)
    # same layout: the captured graph is replayed with new strengths and outputs
    for f in frames:
        f.h_param *= 0.5
        f.out = torch.empty_like(f.out)
        f.clip = None
    ds.develop_batch(frames, 4, 2, ctx=ctx)
    for f in frames:
        rgb, _ = single(f, 4, 2, ctx)
        np.testing.assert_array_equal(f.out.cpu().numpy(), rgb)


def test_frame_completion_times(env):
    torch, dev = env
    ctx = ds.Context(0)
    frames = make_frames(torch, dev, CASES, seed=80)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ds.develop_batch(frames, 10, 3, ctx=ctx, sync=False)
    e1.record(stream)
    ms = ds.batch_frame_ms(len(frames), ctx=ctx)
    total = e0.elapsed_time(e1)
    assert np.all(ms > 0) and np.all(ms <= total + 0.5), (ms, total)


def test_autotune_table(env):
    torch, dev = env
    ctx = ds.Context(0)
    sizes = [(640, 480), (1000, 37)]
    ds.autotune(sizes, 10, 3, ctx=ctx)
    for w, h in sizes:
        t = ds.autotune_get(w, h, ctx=ctx)
        assert tuple(t["rcd_tile"]) in SHAPES and t["nlm_ctas_per_sm"] in (1, 2)
        assert all(v > 0 for v in t["rcd_ms"])
        assert t["rcd_ms"][SHAPES.index(tuple(t["rcd_tile"]))] == min(t["rcd_ms"])
    # a class not in the table takes the nearest one in pixel count
    assert ds.autotune_get(650, 480, ctx=ctx)["rcd_tile"] == ds.autotune_get(640, 480, ctx=ctx)["rcd_tile"]
    frames = make_frames(torch, dev, [(640, 480, 14, 6.0), (1000, 37, 12, 2.0)], seed=120)
    ds.develop_batch(frames, 10, 3, ctx=ctx)
    for f in frames:
        rgb, _ = single(f, 10, 3, ctx)
        np.testing.assert_array_equal(f.out.cpu().numpy(), rgb)


def test_batch_argument_errors(env):
    torch, dev = env
    ctx = ds.Context(0)
    frames = make_frames(torch, dev, CASES[:1])
    L = _lib.lib()
    arr = (_lib.Frame * 1)()
    assert L.dsgpu_rcd_nlm_batch(ctx.handle, arr, 0, 10, 3, 0) == _lib.DSGPU_ERR_ARG
    with pytest.raises(ds.DsgpuError):
        ds.develop_batch(frames, 0, 3, ctx=ctx)  # search 0: unsupported in a batch
    small = make_frames(torch, dev, [(15, 40, 14, 6.0)])
    with pytest.raises(ds.DsgpuError):
        ds.develop_batch(small, 10, 3, ctx=ctx)
    assert ds.autotune_get(100, 100, ctx=ds.Context(0))["rcd_tile"] == (32, 32)  # empty table: the default


def test_batch_black_patterns(env):
    """Per-frame black patterns (dsgpu_frame.black_pattern): each frame of a
    batch equals the one-frame develop under the same context pattern, bit
    for bit; a frame without one keeps its scalar black."""
    torch, dev = env
    ctx = ds.Context(0)
    frames = make_frames(torch, dev, CASES[:3], seed=300)
    pats = [([[500.0, 507.0], [503.0, 519.0]], (1, 0)), None, ([[250, 251, 252, 253], [254, 255, 256, 257]], (3, 1))]
    for f, p in zip(frames, pats):
        if p is not None:
            f.black_pattern, f.black_origin = p
    ds.develop_batch(frames, 10, 3, ctx=ctx)
    for f, p in zip(frames, pats):
        one = ds.Context(0)
        if p is not None:
            one.set_black_pattern(*p)
        rgb, clip = single(f, 10, 3, one)
        np.testing.assert_array_equal(f.out.cpu().numpy(), rgb)
        np.testing.assert_array_equal(f.clip.cpu().numpy(), clip)
    bad = make_frames(torch, dev, CASES[:1], seed=301)
    bad[0].black_pattern = [[512.0] * 5]  # 5 wide: more than 4
    with pytest.raises(ds.DsgpuError):
        ds.develop_batch(bad, 10, 3, ctx=ctx)


def test_bounded_wait_reports_timeout(env):
    """Failure detection without a fault: a work item whose frame's demosaic
    is never queued waits in vain; its bounded wait (2 s of device clock)
    gives up, the call returns DSGPU_ERR_TIMEOUT, and the same context then
    develops a batch correctly."""
    import time

    torch, dev = env
    ctx = ds.Context(0)
    L = _lib.lib()
    t0 = time.perf_counter()
    assert L.dsgpu_selftest_batch_timeout(ctx.handle) == _lib.DSGPU_ERR_TIMEOUT
    dt = time.perf_counter() - t0
    assert 1.5 < dt < 20.0, dt
    frames = make_frames(torch, dev, CASES[:2], seed=500)
    ds.develop_batch(frames, 10, 3, ctx=ctx)
    for f in frames:
        rgb, _ = single(f, 10, 3, ctx)
        np.testing.assert_array_equal(f.out.cpu().numpy(), rgb)
