"""Multi-process (gloo, world_size 2) check of the row-band sharding: each
rank develops its band of one frame with the halo from darkslide_b200.shard,
the bands are gathered, and the result must equal the whole-frame result.
The per-rank compute is the CPU oracle (no GPU here); the sharding logic is
the same the GPU ranks use."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from darkslide_b200 import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _develop_oracle(raw, pat, black, white, mul, h, S, P):
    """(demosaiced, denoised) of a mosaic through the oracle."""
    import dsref

    cfa = dsref.normalize_u16(raw, pat, black, white)
    rgb = dsref.rcd(cfa, pat, mul)
    return np.concatenate([rgb, dsref.nlm_rgb(rgb, h, S, P, nthreads=1)], axis=-1)


def _worker(rank, world, port, raw, args, out_q):
    import sys

    import torch
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pat, black, white, mul, h, S, P = args
    b = shard.band(raw.shape[0], rank, world, shard.halo_rows(S, P))
    pat_b = np.array([pat[((y + b.in0) % 2) * 2 + (x % 2)] for y in range(2) for x in range(2)], np.uint8)
    out = _develop_oracle(raw[b.in0:b.in1], pat_b, black, white, mul, h, S, P)[b.keep]
    # gather the kept rows on rank 0 (the only exchange of the sharded path)
    rows = torch.tensor([b.y1 - b.y0])
    sizes = [torch.zeros_like(rows) for _ in range(world)]
    dist.all_gather(sizes, rows)
    flat = torch.from_numpy(np.ascontiguousarray(out)).reshape(-1)
    maxn = int(max(s.item() for s in sizes)) * raw.shape[1] * 6
    buf = torch.zeros(maxn, dtype=flat.dtype)
    buf[: flat.numel()] = flat
    gathered = [torch.zeros(maxn, dtype=flat.dtype) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, gathered, dst=0)
    if rank == 0:
        parts = [g[: int(s.item()) * raw.shape[1] * 6].reshape(-1, raw.shape[1], 6).numpy()
                 for g, s in zip(gathered, sizes)]
        out_q.put(np.concatenate(parts, axis=0))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_row_bands_reassemble_exactly(oracle, world):
    rng = np.random.default_rng(0)
    h, w = 96, 40
    raw = rng.integers(256, 4096, (h, w), dtype=np.uint16)
    pat = [0, 1, 1, 2]
    white = np.full(3, 4095, np.float32)
    mul = np.array([2.0, 1.0, 1.4], np.float32)
    args = (pat, 256.0, white, mul, 0.05, 3, 1)
    full = _develop_oracle(raw, np.array(pat, np.uint8), 256.0, white, mul, 0.05, 3, 1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, raw, args, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # RCD is local arithmetic: bands reproduce it bit for bit. NLM's box filter
    # is a running sum down each column (image.rs:298-309), whose rounding
    # depends on the row it starts from, so bands agree to the last ulps.
    np.testing.assert_array_equal(got[..., :3], full[..., :3])
    np.testing.assert_allclose(got[..., 3:], full[..., 3:], rtol=0, atol=1e-6)


def test_band_cover_and_frames():
    for h in (17, 96, 4000):
        for world in (1, 2, 3, 8):
            bands = [shard.band(h, r, world, 27) for r in range(world)]
            assert bands[0].y0 == 0 and bands[-1].y1 == h
            for a, b in zip(bands, bands[1:]):
                assert a.y1 == b.y0
            for b in bands:
                assert b.in0 % 2 == 0 and b.in0 <= b.y0 and b.in1 >= b.y1
    assert shard.frames_for_rank(10, 1, 4) == [1, 5, 9]
    assert shard.halo_rows(10, 3) == 27
