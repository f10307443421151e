"""Resource hygiene: repeated calls reuse what a context holds (scratch
slots, band-pipeline events, the copy stream, the batch's graph), so device
memory stays flat across them; contexts created and destroyed in a loop
give their memory back."""
import os

import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu

MUL = [2.0, 1.0, 1.0 / 0.7]
WHITE = [16383.0] * 3
MB = 1 << 20


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch, torch.device("cuda", 0)


def _free(torch):
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_steady_state_memory(env):
    from darkslide_b200 import cnn

    torch, dev = env
    ctx = ds.Context(0)
    net = cnn.ResidualCNN(ctx)
    net.load(os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin"))
    sc = ds.Scene(seed=1, w=1024, h=768, pattern=ds.RGGB, black=512, white=16383, gain=0.5, read_sigma=6)
    hp = 1.5 * sc.sigma_norm()
    raw = sc.render(dev)
    raw_h = raw.cpu().numpy()
    frames = [ds.BatchFrame(raw, ds.RGGB, 512, WHITE, MUL, hp, torch.empty((768, 1024, 3), device=dev))]

    def round_of_calls():
        ds.develop_u16(raw, ds.RGGB, 512, WHITE, MUL, hp, 10, 3, ctx=ctx)
        ds.develop_u16(raw_h, ds.RGGB, 512, WHITE, MUL, hp, 10, 3, ctx=ctx)  # host-buffer pipeline
        net.develop_u16(raw, ds.RGGB, 512, WHITE, MUL, hp)
        net.develop_u16(raw_h, ds.RGGB, 512, WHITE, MUL, hp)
        ds.develop_batch(frames, 10, 3, ctx=ctx)

    for _ in range(2):  # warm-up: scratch, events, streams and the graph are created here
        round_of_calls()
    torch.cuda.empty_cache()
    before = _free(torch)
    for _ in range(10):
        round_of_calls()
    torch.cuda.empty_cache()
    after = _free(torch)
    assert before - after < 8 * MB, (before - after) / MB


def test_context_create_destroy(env):
    torch, dev = env
    sc = ds.Scene(seed=2, w=640, h=480, pattern=ds.BGGR, black=512, white=16383, gain=0.5, read_sigma=6)
    raw = sc.render(dev)
    raw_h = raw.cpu().numpy()

    def use_and_drop():
        ctx = ds.Context(0)
        ds.develop_u16(raw, ds.BGGR, 512, WHITE, MUL, 0.02, 10, 3, ctx=ctx)
        ds.develop_u16(raw_h, ds.BGGR, 512, WHITE, MUL, 0.02, 10, 3, ctx=ctx)
        ctx.close()

    use_and_drop()
    torch.cuda.empty_cache()
    before = _free(torch)
    for _ in range(15):
        use_and_drop()
    torch.cuda.empty_cache()
    after = _free(torch)
    assert before - after < 8 * MB, (before - after) / MB
