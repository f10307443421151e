"""One context per caller thread (the render worker, export and CLI each
hold their own): threads running develops concurrently, each on its own
context and stream, get exactly what a single thread gets."""
import os
import threading

import numpy as np
import pytest

import darkslide_b200 as ds

pytestmark = pytest.mark.gpu

MUL = [2.0, 1.0, 1.0 / 0.7]
WHITE = [16383.0] * 3


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from darkslide_b200 import build

    build.build()
    return torch, torch.device("cuda", 0)


def test_threads_with_own_contexts(env):
    from darkslide_b200 import cnn

    torch, dev = env
    weights = os.path.join(os.path.dirname(cnn.__file__), "weights", "cnn_nlm.bin")
    jobs = []
    for k, (w, h, pat) in enumerate([(640, 480, ds.RGGB), (517, 333, ds.GBRG), (800, 600, ds.BGGR)]):
        sc = ds.Scene(seed=200 + k, w=w, h=h, pattern=pat, black=512, white=16383, gain=0.5, read_sigma=6)
        jobs.append((sc.render_host(), pat, 1.5 * sc.sigma_norm()))

    def run(job, ctx, net):
        raw, pat, hp = job
        plain = ds.develop_u16(raw, pat, 512, WHITE, MUL, hp, 10, 3, ctx=ctx).data
        learned = net.develop_u16(raw, pat, 512, WHITE, MUL, hp).data
        return np.asarray(plain).copy(), np.asarray(learned).copy()

    ref_ctx = ds.Context(0)
    ref_net = cnn.ResidualCNN(ref_ctx)
    ref_net.load(weights)
    expected = [run(j, ref_ctx, ref_net) for j in jobs]

    results, errors = {}, []

    def worker(i):
        try:
            ctx = ds.Context(0)
            net = cnn.ResidualCNN(ctx)
            net.load(weights)
            for rep in range(4):
                results[(i, rep)] = run(jobs[i], ctx, net)
        except Exception as e:  # surfaced below
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for (i, rep), (plain, learned) in results.items():
        np.testing.assert_array_equal(plain, expected[i][0])
        np.testing.assert_array_equal(learned, expected[i][1])
    assert len(results) == 4 * len(jobs)
