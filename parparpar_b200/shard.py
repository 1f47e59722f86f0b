"""Byte-range sharding of a job across GPUs (one process per GPU).

The path partitions with no data-path collective: every rank takes a
contiguous byte range of every input slice and produces the same range of
every recovery (or restored) slice, as the reference distributes one slice
over several backends (PAR2Proc, gf16/controller.cpp:42-84, whose
checkBackendAllocation accepts exactly such a cover: no gaps, no overlaps,
offsets on 16-bit words, an odd size only for the range that ends the slice)
and as its Fenger path shards words (src/par3_engine_fenger.cc:266-290).
"""
from __future__ import annotations


def byte_ranges(slice_bytes: int, world: int, unit: int = 2) -> list[tuple[int, int]]:
    """[start, end) for each of `world` ranks: contiguous, covering the slice,
    every start a multiple of `unit` (2 for PAR2 words; 8 for PAR3 words, 16
    to keep the tensor-core kernels' 16-byte rows), sizes within one unit of
    each other; the odd tail goes to the last rank.  Ranks past the number of
    units get empty ranges."""
    if slice_bytes < 0 or world < 1 or unit < 1:
        raise ValueError("bad slice size, world size or unit")
    units = slice_bytes // unit
    out, pos = [], 0
    for r in range(world):
        n = units // world + (1 if r < units % world else 0)
        end = pos + n * unit
        if r == world - 1:
            end = slice_bytes
        out.append((pos, end))
        pos = end
    return out


def check_ranges(ranges, slice_bytes: int) -> bool:
    """The reference's acceptance rule for a backend split
    (PAR2Proc::checkBackendAllocation): the ranges cover [0, slice_bytes)
    without gaps or overlaps, start on even offsets, and only the range that
    ends the slice may have an odd size."""
    rs = sorted((s, e) for s, e in ranges if e > s)
    if not rs:
        return slice_bytes == 0
    pos = 0
    for s, e in rs:
        if s != pos or s & 1:
            return False
        if (e - s) & 1 and e != slice_bytes:
            return False
        pos = e
    return pos == slice_bytes
