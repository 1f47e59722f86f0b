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


def _ptr_of(buf):
    import ctypes
    if hasattr(buf, "data_ptr"):
        return ctypes.c_void_p(buf.data_ptr())
    return ctypes.c_void_p(buf.ctypes.data)


def _range_arrays(ranges, contexts):
    import ctypes
    n = len(ranges)
    if len(contexts) != n:
        raise ValueError("one context per range")
    ctxs = (ctypes.c_void_p * n)(*[c.follow_torch().h.value for c in contexts])
    b = (ctypes.c_size_t * n)(*[r[0] for r in ranges])
    e = (ctypes.c_size_t * n)(*[r[1] for r in ranges])
    return ctxs, b, e, n


def par2_create_split(inputs, input_idx, exps, contexts, ranges=None, out=None):
    """PAR2 create with byte range r of every slice computed on contexts[r]
    (pp_par2_create_split): each GPU reads and writes only its range, as
    PAR2Proc spreads a slice over its backends.  inputs: (N, S) uint8 host
    array or tensor; ranges default to byte_ranges(S, len(contexts), 2)."""
    import numpy as np
    from ._lib import lib
    n, s = inputs.shape
    if ranges is None:
        ranges = byte_ranges(s, len(contexts), 2)
    idx = np.ascontiguousarray(np.asarray(input_idx, dtype=np.uint16))
    ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
    if out is None:
        out = np.zeros((ex.size, s), dtype=np.uint8)
    ctxs, b, e, k = _range_arrays(ranges, contexts)
    in_stride = inputs.stride(0) if hasattr(inputs, "stride") else inputs.strides[0]
    out_stride = out.stride(0) if hasattr(out, "stride") else out.strides[0]
    contexts[0].check(lib.pp_par2_create_split(ctxs, b, e, k, _ptr_of(inputs), in_stride, n, s, _ptr_of(idx),
                                               _ptr_of(ex), ex.size, _ptr_of(out), out_stride))
    return out


def par3_create_split(inputs, num_recovery, first_input, first_recovery, contexts, ranges=None, out=None):
    """PAR3 create (Cauchy product) with byte range r of every block on
    contexts[r] (pp_gf64_compute_recovery_split).  inputs: (N, W) uint64 /
    int64; ranges default to byte_ranges(8 W, len(contexts), 16)."""
    import numpy as np
    from ._lib import lib
    n, w = inputs.shape
    if ranges is None:
        ranges = byte_ranges(8 * w, len(contexts), 16)
    if out is None:
        out = np.zeros((num_recovery, w), dtype=np.uint64)
    ctxs, b, e, k = _range_arrays(ranges, contexts)
    contexts[0].check(lib.pp_gf64_compute_recovery_split(ctxs, b, e, k, _ptr_of(inputs), n, _ptr_of(out),
                                                         num_recovery, w, first_input, first_recovery))
    return out
