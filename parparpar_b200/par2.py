"""PAR2 (GF(2^16)) host interface over the CUDA engine.

Mirrors the reference's PAR2 operator surface so a caller of the reference
finds the same names, argument meaning and error behaviour:

* ``PAR2ProcCUDA``      — an ``IPAR2ProcBackend`` for a CUDA device
                          (reference gf16/controller.h:77-217; behaviour of
                          PAR2ProcCPU, gf16/controller_cpu.cpp): staging areas,
                          ``addInput``/``endInput``/``getOutput``.
* ``Galois16RecMatrix`` — repair-matrix inversion, ``Compute``/``GetFactor``
                          (reference gf16/gfmat_inv.h:16-50).
* ``gf16_muladd`` / ``par2_create`` / ``coeff_matrix`` — one-call forms.
* ``gfmat_coeff`` / ``gfmat_input_log`` — scalar coefficient helpers
                          (reference gf16/gfmat_coeff.c:80-101).

Buffers are numpy arrays (host) or torch tensors (host or CUDA).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PP_OK, PPError, default_context, lib, ptr


def _ctx(ctx):
    return ctx if ctx is not None else default_context()


def gfmat_coeff(input_block: int, recovery_exp: int) -> int:
    return int(lib.pp_par2_coeff(input_block, recovery_exp))


def gfmat_input_log(input_block: int) -> int:
    return int(lib.pp_par2_input_log(input_block))


def _rows(buf):
    """(n_rows, row_bytes, row_stride_bytes) of a 2-D uint8 buffer."""
    if hasattr(buf, "stride") and hasattr(buf, "data_ptr"):  # torch
        if buf.dim() != 2 or buf.element_size() != 1:
            raise TypeError("expected a 2-D uint8 tensor")
        if buf.stride(1) != 1:
            raise ValueError("rows must be contiguous")
        return buf.shape[0], buf.shape[1], buf.stride(0)
    a = buf
    if a.ndim != 2 or a.dtype.itemsize != 1:
        raise TypeError("expected a 2-D uint8 array")
    if a.strides[1] != 1:
        raise ValueError("rows must be contiguous")
    return a.shape[0], a.shape[1], a.strides[0]


def coeff_matrix(input_idx, exps, out=None, ctx=None):
    """coeffs[o, i] = gfmat_coeff(input_idx[i], exps[o]) computed on the device."""
    c = _ctx(ctx)
    idx = np.ascontiguousarray(np.asarray(input_idx, dtype=np.uint16))
    ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
    if out is None:
        out = np.zeros((ex.size, idx.size), dtype=np.uint16)
    c.check(lib.pp_par2_coeff_matrix(c.h, ptr(idx), idx.size, ptr(ex), ex.size, ptr(out)))
    return out


def gf16_muladd(inputs, coeffs, out=None, slice_bytes=None, accumulate=False, ctx=None):
    """out[o] (^)= XOR_i coeffs[o, i] * inputs[i] over GF(2^16) (LE u16 words).

    inputs: (N, S) uint8; coeffs: (R, N) uint16; out: (R, S) uint8."""
    c = _ctx(ctx)
    n, s, istride = _rows(inputs)
    if slice_bytes is None:
        slice_bytes = s
    if coeffs is None:
        raise TypeError("coeffs required")
    if hasattr(coeffs, "data_ptr"):
        r, cs = coeffs.shape[0], coeffs.stride(0)
    else:
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint16)
        r, cs = coeffs.shape[0], coeffs.shape[1]
    if coeffs.shape[1] != n:
        raise ValueError("coeffs must be (num_outputs, num_inputs)")
    if out is None:
        out = np.zeros((r, slice_bytes), dtype=np.uint8)
    ro, so, ostride = _rows(out)
    if ro != r or so < slice_bytes:
        raise ValueError("out must be (num_outputs, >= slice_bytes)")
    c.check(lib.pp_gf16_muladd(c.h, ptr(inputs), istride, n, slice_bytes, ptr(coeffs), cs, r, ptr(out), ostride,
                               1 if accumulate else 0))
    return out


def par2_create(inputs, input_idx, exps, out=None, slice_bytes=None, ctx=None):
    """PAR2 recovery slices: out[o] = XOR_i gfmat_coeff(input_idx[i], exps[o]) * inputs[i]."""
    c = _ctx(ctx)
    n, s, istride = _rows(inputs)
    if slice_bytes is None:
        slice_bytes = s
    idx = np.ascontiguousarray(np.asarray(input_idx, dtype=np.uint16))
    ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
    if idx.size != n:
        raise ValueError("input_idx length must equal the number of input slices")
    if out is None:
        out = np.zeros((ex.size, slice_bytes), dtype=np.uint8)
    ro, so, ostride = _rows(out)
    c.check(lib.pp_par2_create(c.h, ptr(inputs), istride, n, slice_bytes, ptr(idx), ptr(ex), ex.size, ptr(out),
                               ostride))
    return out


class Galois16RecMatrix:
    """Repair-matrix inversion (reference gf16/gfmat_inv.h:16-50)."""

    def __init__(self, ctx=None):
        self.ctx = _ctx(ctx)
        self.factors = None
        self.numInputs = 0

    def setNumThreads(self, threads: int):  # API parity; the device decides its own parallelism
        pass

    def Compute(self, inputValid, validCount, recovery) -> bool:
        """recovery: a Python list, sorted and truncated in place like the
        reference's std::vector<uint16_t>&."""
        v = np.ascontiguousarray(np.asarray([1 if x else 0 for x in inputValid], dtype=np.uint8))
        n = v.size
        if int(v.sum()) != validCount:
            raise ValueError("validCount does not match inputValid")
        m = n - validCount
        rec = np.ascontiguousarray(np.asarray(recovery, dtype=np.uint16)).copy()
        nrec = ctypes.c_uint(rec.size)
        f = np.zeros((max(m, 1), n), dtype=np.uint16)
        st = lib.pp_par2_invert(self.ctx.h, ptr(v), n, ptr(rec), ctypes.byref(nrec), ptr(f))
        if st == _lib.PP_ERR_NOT_INVERTIBLE:
            return False
        self.ctx.check(st)
        recovery[:] = [int(x) for x in rec[: nrec.value]]
        self.factors = f[:m]
        self.numInputs = n
        return True

    def GetFactor(self, inIdx: int, recIdx: int) -> int:
        return int(self.factors[recIdx, inIdx])


class PAR2ProcCUDA:
    """CUDA processor behind the gf16 controller interface (IPAR2ProcBackend)."""

    def __init__(self, sliceSize: int, stagingAreas: int = 2, inputBatchSize: int = 0, ctx=None):
        self.ctx = _ctx(ctx)
        h = ctypes.c_void_p()
        self.ctx.check(lib.pp_par2_proc_create(self.ctx.h, sliceSize, stagingAreas, inputBatchSize, ctypes.byref(h)))
        self.h = h
        self.numRecovery = 0

    def _chk(self, st):
        return self.ctx.check(st)

    def setCurrentSliceSize(self, size: int) -> bool:
        return lib.pp_par2_proc_set_current_slice_size(self.h, size) == PP_OK

    def setRecoverySlices(self, numSlices: int, exponents=None) -> bool:
        ex = None if exponents is None else np.ascontiguousarray(np.asarray(exponents, dtype=np.uint16))
        self.numRecovery = numSlices
        return lib.pp_par2_proc_set_recovery_slices(self.h, numSlices, ptr(ex) if ex is not None else None) == PP_OK

    def getNumRecoverySlices(self) -> int:
        return self.numRecovery

    def canAdd(self) -> int:
        return lib.pp_par2_proc_can_add(self.h)

    def waitForAdd(self):
        self._chk(lib.pp_par2_proc_wait_for_add(self.h))

    def addInput(self, buffer, size: int, inputNumOrCoeffs, flush: bool = False):
        if isinstance(inputNumOrCoeffs, (int, np.integer)):
            self._chk(lib.pp_par2_proc_add_input(self.h, ptr(buffer), size, int(inputNumOrCoeffs), 1 if flush else 0))
        else:
            co = np.ascontiguousarray(np.asarray(inputNumOrCoeffs, dtype=np.uint16))
            if co.size < self.numRecovery:
                raise ValueError("one coefficient per recovery slice required")
            self._chk(lib.pp_par2_proc_add_input_coeffs(self.h, ptr(buffer), size, ptr(co), 1 if flush else 0))

    def flush(self):
        self._chk(lib.pp_par2_proc_flush(self.h))

    def endInput(self):
        self._chk(lib.pp_par2_proc_end_input(self.h))

    def getOutput(self, index: int, output) -> bool:
        valid = ctypes.c_int(0)
        self._chk(lib.pp_par2_proc_get_output(self.h, index, ptr(output), ctypes.byref(valid)))
        return bool(valid.value)

    def discardOutput(self):
        self._chk(lib.pp_par2_proc_discard_output(self.h))

    def freeProcessingMem(self):
        self._chk(lib.pp_par2_proc_free_processing_mem(self.h))

    def getInputBatchSize(self) -> int:
        return int(lib.pp_par2_proc_input_batch_size(self.h))

    def getBatchesStarted(self) -> int:
        return int(lib.pp_par2_proc_batches_started(self.h))

    def deinit(self):
        if self.h:
            lib.pp_par2_proc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass


__all__ = ["PAR2ProcCUDA", "Galois16RecMatrix", "gf16_muladd", "par2_create", "coeff_matrix", "gfmat_coeff",
           "gfmat_input_log", "PPError"]
