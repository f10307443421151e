"""Multi-GPU sharding of the detail path: one process per GPU, no collective
on the data path.

The path partitions cleanly:
  - frames are independent, so a batch is split across ranks
    (``frames_for_rank``); this is what bench.py measures (weak scaling);
  - one frame can be split into row bands (``band``): each rank develops its
    band plus a halo of rows and keeps the interior. A site's demosaiced value
    depends on CFA samples within 10 rows (the RCD passes of demosaic.rs:160-341)
    and on the 4-row MHC ring at an image border (demosaic.rs:203-214), so RCD
    values at 14 or more rows from a band cut equal the whole-frame values;
    NLM (enhance.rs:36-72) then reads demosaiced values within S+P rows. A
    halo of 14 + S + P rows therefore makes every kept row identical to the
    whole-frame result.
The only exchange is the final gather of bands (or of per-frame statistics),
done with torch.distributed (NCCL between GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from dataclasses import dataclass

RCD_RADIUS = 10  # receptive radius of the RCD passes
RCD_RING = 4     # MHC ring width at an image border


def halo_rows(search: int, patch: int) -> int:
    """Rows a band needs beyond its kept rows for an exact result."""
    return RCD_RING + RCD_RADIUS + max(search, 0) + max(patch, 0)


def frames_for_rank(n_frames: int, rank: int, world: int) -> list[int]:
    """Round-robin assignment of frame indices to a rank."""
    return list(range(rank, n_frames, world))


@dataclass(frozen=True)
class Band:
    y0: int   # first kept row (frame coordinates)
    y1: int   # one past the last kept row
    in0: int  # first input row (with halo, clamped to the frame)
    in1: int  # one past the last input row

    @property
    def keep(self) -> slice:
        """Rows of the band's own output that are kept."""
        return slice(self.y0 - self.in0, self.y1 - self.in0)


def band(h: int, rank: int, world: int, halo: int, align: int = 2) -> Band:
    """Row band of `rank`: kept rows split as evenly as possible on `align`
    boundaries (2 keeps every band's CFA phase equal to the frame's), input
    rows extended by `halo` on each side and clamped to the frame."""
    units = (h + align - 1) // align
    per, extra = divmod(units, world)
    u0 = rank * per + min(rank, extra)
    u1 = u0 + per + (1 if rank < extra else 0)
    y0, y1 = min(u0 * align, h), min(u1 * align, h)
    in0 = max(y0 - halo, 0)
    in1 = min(y1 + halo, h)
    if align % 2 == 0:
        in0 -= in0 % 2  # keep the CFA phase of the band's first row
    return Band(y0, y1, in0, in1)


def develop_band(raw, pattern, b: Band, black, white, mul, h_param, search, patch, ctx=None):
    """Develop one row band of a u16 frame (device tensor or numpy array) and
    return its kept rows (the GPU side of the row-band split)."""
    from . import develop_u16

    pat = pattern.shifted(0, b.in0)
    img = develop_u16(raw[b.in0:b.in1], pat, black, white, mul, h_param, search, patch, ctx=ctx)
    return img.data[b.keep]
