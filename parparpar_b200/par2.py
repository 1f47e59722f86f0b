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
* ``block_hashes`` / ``HasherInput`` — input-slice MD5 + CRC32 (IFSC
                          entries) on the device; ``HasherInput`` mirrors the
                          reference's hasher binding (src/gf.cc:869-1060).

Buffers are numpy arrays (host) or torch tensors (host or CUDA).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PP_OK, PPError, default_context, lib, ptr


def _ctx(ctx):
    return (ctx if ctx is not None else default_context()).follow_torch()


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


def par2_create(inputs, input_idx, exps, out=None, slice_bytes=None, hashes=None, ctx=None):
    """PAR2 recovery slices: out[o] = XOR_i gfmat_coeff(input_idx[i], exps[o]) * inputs[i].

    hashes: optional (n, 20) uint8 buffer (host or CUDA) that receives the
    inputs' IFSC entries (MD5 || CRC32 of each input row), computed on the
    device in the same pass over the inputs."""
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
    if hashes is not None:
        c.check(lib.pp_par2_create_hashed(c.h, ptr(inputs), istride, n, slice_bytes, ptr(idx), ptr(ex), ex.size,
                                          ptr(out), ostride, ptr(hashes)))
        return out
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

    def Compute(self, inputValid, validCount, recovery, out=None) -> bool:
        """recovery: a Python list, sorted and truncated in place like the
        reference's std::vector<uint16_t>&.  out: optional (m, n) uint16
        buffer (host or CUDA) for the factors; default a new numpy array."""
        if isinstance(inputValid, np.ndarray) and inputValid.dtype.kind in "biu":
            v = np.ascontiguousarray(inputValid != 0, dtype=np.uint8)  # vectorised: no per-element Python loop
        else:
            v = np.ascontiguousarray(np.asarray([1 if x else 0 for x in inputValid], dtype=np.uint8))
        n = v.size
        if int(v.sum()) != validCount:
            raise ValueError("validCount does not match inputValid")
        m = n - validCount
        rec = np.ascontiguousarray(np.asarray(recovery, dtype=np.uint16)).copy()
        nrec = ctypes.c_uint(rec.size)
        f = np.zeros((max(m, 1), n), dtype=np.uint16) if out is None else out
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
        if getattr(buffer, "is_cuda", False):
            # the processor copies device slices on its own stream: the
            # producer of a CUDA tensor (torch's current stream) finishes first
            import torch
            torch.cuda.current_stream(buffer.device).synchronize()
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

    def outputDevicePtr(self, index: int) -> int:
        """Device address of recovery slice `index` in the output area (after
        endInput), for consumers that read recovery data on the device."""
        p = ctypes.c_void_p()
        self._chk(lib.pp_par2_proc_output_ptr(self.h, index, ctypes.byref(p)))
        return int(p.value)

    def setInputHashes(self, maxInputs: int):
        """Hash every slice added by input number from now on (IFSC entries:
        MD5 || CRC32le of the slice zero-padded to the slice size), on the
        device, in the processor's own pass; 0 turns it off."""
        self._chk(lib.pp_par2_proc_set_input_hashes(self.h, maxInputs))

    def getInputHashes(self, count: int, out=None):
        """Entries [0, count) as a (count, 20) uint8 array (or into `out`,
        host or CUDA), after the submitted batches finish."""
        if out is None:
            out = np.zeros((count, 20), dtype=np.uint8)
        self._chk(lib.pp_par2_proc_get_input_hashes(self.h, ptr(out), count))
        return out

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
           "gfmat_input_log", "PPError", "block_hashes", "HasherInput", "memory_checksums",
           "recovery_packet_headers"]


# ------------------------------------------------------------ block hashes
def block_hashes(blocks, slice_size=None, lengths=None, out=None, ctx=None):
    """IFSC entries of input slices on the device: row i of the (n, 20) result
    is MD5 || CRC32 (little-endian) of ``blocks[i, :lengths[i]]`` followed by
    zeros up to ``slice_size`` bytes -- HasherInput::getBlock(md5crc, zeroPad)
    (hasher/hasher_input_base.h:104-117).

    blocks: 2-D uint8 numpy array or torch tensor (host or CUDA), one slice per
    row; slice_size defaults to the row length; lengths (n,) or None (full
    rows).  out: an (n, 20) uint8 buffer (host or CUDA) or None (numpy)."""
    c = _ctx(ctx)
    n, row_bytes, stride = _rows(blocks)
    slice_size = row_bytes if slice_size is None else int(slice_size)
    if out is None:
        out = np.empty((n, 20), dtype=np.uint8)
    lens = None
    if lengths is not None:
        lens = lengths if hasattr(lengths, "data_ptr") else np.ascontiguousarray(np.asarray(lengths, dtype=np.uint64))
    c.check(lib.pp_par2_block_hashes(c.h, ptr(blocks), stride, n, slice_size, ptr(lens), ptr(out)))
    return out


class HasherInput:
    """The reference's PAR2 input hasher object (src/gf.cc:869-1060:
    ``new HasherInput(sliceSize, ifscBuf)``, ``update(buf)``, ``end(md5Buf)``,
    ``reset()``): a file's bytes are fed in order; every completed slice gets
    its 20-byte IFSC entry written into ``ifsc`` (in order, while room
    remains), the zero-padded last partial slice at ``end``, which also writes
    the whole-file MD5 into ``md5`` (16 bytes).

    Slice hashes run on the device in batches of ``batch`` slices; the file
    MD5 is one serial hash of the stream and is computed on the host as the
    bytes go by."""

    def __init__(self, slice_size: int, ifsc, batch: int = 1024, ctx=None):
        if slice_size <= 0:
            raise ValueError("Requires a size and buffer")
        self.slice = int(slice_size)
        self.ifsc = np.frombuffer(memoryview(ifsc).cast("B"), dtype=np.uint8) if not isinstance(ifsc, np.ndarray) \
            else ifsc.reshape(-1).view(np.uint8)
        # staging rows: at most `batch` slices and about 256 MiB
        self.batch = max(1, min(int(batch), (256 << 20) // self.slice))
        self.ctx = _ctx(ctx)
        self.reset()

    def reset(self):
        import hashlib

        self._md5 = hashlib.md5()
        self._rows = np.zeros((self.batch, self.slice), dtype=np.uint8)
        self._n = 0        # slices buffered in _rows (the last may be partial)
        self._pos = 0      # bytes in the current (partial) slice
        self._done = 0     # IFSC entries written
        self._ended = False

    def _flush(self, lengths=None):
        n = self._n
        if n == 0:
            return
        room = self.ifsc.size // 20 - self._done
        n_out = min(n, max(room, 0))
        if n_out:
            h = block_hashes(self._rows[:n_out], self.slice, lengths[:n_out] if lengths is not None else None,
                             ctx=self.ctx)
            self.ifsc[20 * self._done: 20 * (self._done + n_out)] = h.reshape(-1)
            self._done += n_out
        self._n = 0

    def update(self, data):
        if self._ended:
            raise RuntimeError("Process already ended")
        buf = np.frombuffer(memoryview(data).cast("B"), dtype=np.uint8)
        self._md5.update(buf)
        i = 0
        while i < buf.size:
            take = min(self.slice - self._pos, buf.size - i)
            self._rows[self._n, self._pos: self._pos + take] = buf[i: i + take]
            self._pos += take
            i += take
            if self._pos == self.slice:
                self._n += 1
                self._pos = 0
                if self._n == self.batch:
                    self._flush()

    def end(self, md5_out):
        if self._ended:
            raise RuntimeError("Process already ended")
        lengths = None
        if self._pos:
            self._rows[self._n, self._pos:] = 0
            lengths = np.full(self._n + 1, self.slice, dtype=np.uint64)
            lengths[-1] = self._pos
            self._n += 1
        self._flush(lengths)
        out = np.frombuffer(memoryview(md5_out).cast("B"), dtype=np.uint8) if not isinstance(md5_out, np.ndarray) \
            else md5_out.reshape(-1).view(np.uint8)
        if out.size < 16:
            raise ValueError("Buffer must be at least 16 bytes long")
        out[:16] = np.frombuffer(self._md5.digest(), dtype=np.uint8)
        self._ended = True


def memory_checksums(rows, slice_size=None, out=None, ctx=None):
    """PAR2 memory checksum blocks (16 bytes per row) of the staged-slice
    checksum the processor carries through the region pass
    (gf16/gf16_cksum_base.h:40-55): C = sum_j 2^(nb-1-j) * B_j over the row's
    16-byte blocks, lane-wise in GF(2^16)."""
    c = _ctx(ctx)
    n, row_bytes, stride = _rows(rows)
    slice_size = row_bytes if slice_size is None else int(slice_size)
    if out is None:
        out = np.empty((n, 16), dtype=np.uint8)
    c.check(lib.pp_par2_memory_checksums(c.h, ptr(rows), stride, n, slice_size, ptr(out)))
    return out


def recovery_packet_headers(slices, exps, set_id, slice_size=None, out=None, ctx=None):
    """68-byte PAR2 recovery packet headers with their MD5s (getRecoveryHeader
    and the packet MD5 of lib/par2.js:240-330,517-530): row i describes
    recovery slice ``slices[i]`` with exponent ``exps[i]``."""
    c = _ctx(ctx)
    n, row_bytes, stride = _rows(slices)
    slice_size = row_bytes if slice_size is None else int(slice_size)
    ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
    if ex.size != n:
        raise ValueError("one exponent per slice")
    sid = np.frombuffer(bytes(set_id), dtype=np.uint8)
    if sid.size != 16:
        raise ValueError("set_id must be 16 bytes")
    if out is None:
        out = np.empty((n, 68), dtype=np.uint8)
    c.check(lib.pp_par2_recovery_packet_headers(c.h, ptr(slices), stride, n, slice_size, ptr(sid), ptr(ex),
                                                ptr(out)))
    return out
