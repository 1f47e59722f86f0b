"""Batches of create / repair jobs run as a few fused tensor-core launches
replayed from a CUDA graph (pp_batch_* in include/parpar_b200.h).

There is no counterpart in the reference, which runs one job at a time; each
job's result is bit-identical to the single-job calls
(par2.par2_create, par3.GF64Controller.ComputeRecoveryBlocks, par3.repair).

All buffers are torch CUDA tensors that stay bound to the batch: later
``run()`` calls read whatever the input tensors hold then.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (PP_BATCH_NO_GRAPH, PP_BATCH_TUNE, PP_JOB_GF16_MULADD, PP_JOB_PAR2_CREATE, PP_JOB_PAR3_CREATE, PP_JOB_PAR3_REPAIR,
                   PPJob, default_context, lib, ptr)


def _ctx(ctx):
    return (ctx if ctx is not None else default_context()).follow_torch()


def _rows(t):
    """(rows, row stride in bytes) of a 2-D torch tensor or numpy array with
    contiguous rows (batches need CUDA tensors; the server also takes host
    buffers)."""
    if hasattr(t, "data_ptr"):
        if t.dim() != 2 or t.stride(1) != 1:
            raise ValueError("rows must be a 2-D tensor with contiguous rows")
        return t.shape[0], t.stride(0) * t.element_size()
    if isinstance(t, np.ndarray):
        if t.ndim != 2 or t.strides[1] != t.itemsize:
            raise ValueError("rows must be a 2-D array with contiguous rows")
        return t.shape[0], t.strides[0]
    raise TypeError("job buffers are torch tensors or numpy arrays")


def _width(t):
    return t.shape[1] * (t.element_size() if hasattr(t, "element_size") else t.itemsize)


def par2_create_job(inputs, exponents, outputs, input_ids=None, slice_bytes=None):
    """PAR2 create: outputs[e] = XOR_i c(input_ids[i], exponents[e]) * inputs[i] (uint8 rows)."""
    n, istride = _rows(inputs)
    r, ostride = _rows(outputs)
    exps = np.ascontiguousarray(np.asarray(exponents, dtype=np.uint16))
    ids = None if input_ids is None else np.ascontiguousarray(np.asarray(input_ids, dtype=np.uint16))
    if exps.size != r:
        raise ValueError("one exponent per output row")
    j = PPJob(kind=PP_JOB_PAR2_CREATE, inputs=ptr(inputs), input_stride=istride, num_inputs=n,
              slice_bytes=slice_bytes if slice_bytes is not None else _width(inputs),
              input_ids=ptr(ids) if ids is not None else None, exponents=ptr(exps), num_recovery=r,
              outputs=ptr(outputs), output_stride=ostride)
    return j, (inputs, outputs, exps, ids)


def par3_create_job(inputs, outputs, first_input=0, first_recovery=None):
    """PAR3 create: outputs[r] = XOR_c inv((fI + c) ^ (fR + r)) * inputs[c] (int64 / uint64 rows)."""
    n, istride = _rows(inputs)
    r, ostride = _rows(outputs)
    fr = n if first_recovery is None else first_recovery
    j = PPJob(kind=PP_JOB_PAR3_CREATE, inputs=ptr(inputs), input_stride=istride, num_inputs=n,
              slice_bytes=_width(inputs), num_recovery=r, outputs=ptr(outputs),
              output_stride=ostride, first_input=first_input & (2**64 - 1), first_recovery=fr & (2**64 - 1))
    return j, (inputs, outputs)


def par3_repair_job(inputs, missing, recovery, restored, first_input=0, first_recovery=None,
                    recovery_present=None):
    """PAR3 repair: restored[k] = input block missing[k] from the first len(missing) recovery blocks."""
    n_in, istride = _rows(inputs)
    nrec, rstride = _rows(recovery)
    nres, ostride = _rows(restored)
    miss = np.ascontiguousarray(np.asarray(missing, dtype=np.uint64))
    if nrec < miss.size or nres < miss.size:
        raise ValueError("need one recovery row and one restored row per missing block")
    pres = None if recovery_present is None else np.ascontiguousarray(np.asarray(recovery_present, dtype=np.uint8))
    fr = n_in if first_recovery is None else first_recovery
    j = PPJob(kind=PP_JOB_PAR3_REPAIR, inputs=ptr(inputs), input_stride=istride, num_inputs=n_in,
              slice_bytes=_width(inputs), outputs=ptr(restored), output_stride=ostride,
              first_input=first_input & (2**64 - 1), first_recovery=fr & (2**64 - 1), missing=ptr(miss),
              num_missing=miss.size, recovery=ptr(recovery), recovery_stride=rstride,
              recovery_present=ptr(pres) if pres is not None else None)
    return j, (inputs, recovery, restored, miss, pres)


def gf16_muladd_job(inputs, coeffs, outputs, slice_bytes=None):
    """outputs[o] = XOR_i coeffs[o, i] * inputs[i] over GF(2^16), e.g. the PAR2
    repair decode with the factors of par2.Galois16RecMatrix."""
    n, istride = _rows(inputs)
    r, ostride = _rows(outputs)
    co = np.ascontiguousarray(np.asarray(coeffs, dtype=np.uint16))
    if co.shape != (r, n):
        raise ValueError("coeffs must be (num_outputs, num_inputs)")
    j = PPJob(kind=PP_JOB_GF16_MULADD, inputs=ptr(inputs), input_stride=istride, num_inputs=n,
              slice_bytes=slice_bytes if slice_bytes is not None else _width(inputs), num_recovery=r,
              outputs=ptr(outputs), output_stride=ostride, coeffs=ptr(co))
    return j, (inputs, outputs, co)


class Batch:
    """A batch plan over jobs made by the *_job helpers."""

    def __init__(self, jobs, tune=False, graph=True, ctx=None):
        """tune: time candidate work splits at creation (resident plans);
        graph=False: jobs seen once -- build the tables only and issue the
        fused launches directly at run() (no eager run, no capture)."""
        self.ctx = _ctx(ctx)
        self._keep = [k for _, k in jobs]
        arr = (PPJob * len(jobs))(*[j for j, _ in jobs])
        h = ctypes.c_void_p()
        flags = (PP_BATCH_TUNE if tune and graph else 0) | (0 if graph else PP_BATCH_NO_GRAPH)
        self.ctx.check(lib.pp_batch_create(self.ctx.h, arr, len(jobs), flags, ctypes.byref(h)))
        self.h = h

    @property
    def launches(self) -> int:
        return lib.pp_batch_launches(self.h)

    def run(self):
        self.ctx.check(lib.pp_batch_run(self.h))

    def close(self):
        if self.h:
            lib.pp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
