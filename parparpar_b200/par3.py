"""PAR3 (GF(2^64)) host interface over the CUDA engine.

Mirrors the reference's PAR3 operator surface:

* ``GF64Controller``  — static engine entry points with the reference's names
                         and argument meaning (src/par3_engine.h:11-244).
* ``compute_recovery*``, ``build_coefficient_matrix``, ``solve_and_reconstruct``,
  ``Gf64Encoder`` — the gf64_addon N-API functions (src/gf64_addon.cc:3271-3612)
  with the same argument checks (TypeError / RangeError become Python
  ``TypeError`` / ``ValueError``).
* ``gf64_region_*`` / ``gf64_inverse_batch`` — the region dispatch table
  (gf64/gf64_global.h:23-37).
* ``block_hashes`` / ``assemble_recovery_packets`` — BLAKE3 block checksums
  (lib/par3gen.js:1001-1017) and recovery packets (src/gf64_addon.cc:2784-2936)
  on the device.

Buffers: numpy uint64 arrays (host) or torch int64/uint64 tensors (host or
CUDA).  numThreads arguments are accepted for interface parity; the device
schedules itself.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PP_OK, PPError, default_context, lib, ptr


def _ctx(ctx):
    return (ctx if ctx is not None else default_context()).follow_torch()


def _u64(x) -> int:
    return int(x) & 0xFFFFFFFFFFFFFFFF


class GF64Controller:
    """Static GF(2^64) engine entry points (reference src/par3_engine.h:11-244)."""

    ctx = None

    @classmethod
    def _c(cls):
        return _ctx(cls.ctx)

    @classmethod
    def ComputeRecoveryBlocks(cls, inputs, numInputs, recovery, numRecovery, blockSize64, firstInput, firstRecovery,
                              numThreads=0, accumulate=False, kernel=_lib.PP_GF64_KERNEL_MATVEC):
        c = cls._c()
        c.check(lib.pp_gf64_compute_recovery(c.h, ptr(inputs), numInputs, ptr(recovery), numRecovery, blockSize64,
                                             _u64(firstInput), _u64(firstRecovery), 1 if accumulate else 0, kernel))

    @classmethod
    def ComputeRecoveryBlocksFull(cls, inputs, numInputs, recovery, numRecovery, blockSize64, firstInput,
                                  firstRecovery, numThreads=0, accumulate=False):
        cls.ComputeRecoveryBlocks(inputs, numInputs, recovery, numRecovery, blockSize64, firstInput, firstRecovery,
                                  numThreads, accumulate, _lib.PP_GF64_KERNEL_AUTO)

    @classmethod
    def ComputeRecoveryBlocksBarycentric(cls, inputs, numInputs, recovery, numRecovery, blockSize64, firstInput,
                                         firstRecovery, numThreads=0, accumulate=False):
        cls.ComputeRecoveryBlocks(inputs, numInputs, recovery, numRecovery, blockSize64, firstInput, firstRecovery,
                                  numThreads, accumulate, _lib.PP_GF64_KERNEL_BARYCENTRIC)

    @classmethod
    def ComputeRecoveryBlocksFenger(cls, inputs, numInputs, recovery, numRecovery, blockSize64, firstInput,
                                    firstRecovery, numThreads=0):
        cls.ComputeRecoveryBlocks(inputs, numInputs, recovery, numRecovery, blockSize64, firstInput, firstRecovery,
                                  numThreads, False, _lib.PP_GF64_KERNEL_FENGER)

    @classmethod
    def ComputeRecoveryBlocksWithCoeff(cls, inputs, numInputs, recovery, numRecovery, blockSize64, coeff,
                                       numThreads=0, accumulate=False):
        c = cls._c()
        c.check(lib.pp_gf64_compute_recovery_with_coeff(c.h, ptr(inputs), numInputs, ptr(recovery), numRecovery,
                                                        blockSize64, ptr(coeff), 1 if accumulate else 0))

    @classmethod
    def BuildCauchyMatrix(cls, coeffMatrix, numInputs, numRecovery, firstInput, firstRecovery):
        c = cls._c()
        c.check(lib.pp_gf64_build_cauchy(c.h, ptr(coeffMatrix), numInputs, numRecovery, _u64(firstInput),
                                         _u64(firstRecovery)))

    @classmethod
    def BuildCauchyMatrixAlloc(cls, numInputs, numRecovery, firstInput, firstRecovery):
        if numInputs == 0 or numRecovery == 0:
            return None
        m = np.zeros((numRecovery, numInputs), dtype=np.uint64)
        cls.BuildCauchyMatrix(m, numInputs, numRecovery, firstInput, firstRecovery)
        return m

    @classmethod
    def MultiplyAccumulate(cls, out, numOut, inp, numIn, coeffMatrix, blockSize64):
        """out[i] ^= sum_j in[j] * coeffMatrix[i*numIn + j] (accumulating form)."""
        cls.ComputeRecoveryBlocksWithCoeff(inp, numIn, out, numOut, blockSize64, coeffMatrix, 0, True)

    @classmethod
    def SolveAndReconstruct(cls, A, rhsBlocks, n, blockSize64, numThreads=0) -> int:
        """0 on success, -1 if the matrix is singular (reference return codes)."""
        c = cls._c()
        st = lib.pp_gf64_solve_and_reconstruct(c.h, ptr(A), ptr(rhsBlocks), n, blockSize64)
        if st == _lib.PP_ERR_SINGULAR:
            return -1
        c.check(st)
        return 0


# ------------------------------------------------------------- N-API mirror
def _buf_words(buf, name):
    if buf is None or not (hasattr(buf, "data_ptr") or hasattr(buf, "ctypes")):
        raise TypeError(f"{name} must be a Buffer")
    nbytes = buf.numel() * buf.element_size() if hasattr(buf, "numel") else buf.nbytes
    return nbytes


def _check_int(v, name):
    if isinstance(v, bool) or not isinstance(v, (int, np.integer)):
        raise TypeError(f"{name} must be an integer")
    return int(v)


def compute_recovery(inputs, outputs, numInputs, numRecovery, blockSize, firstInput, firstRecovery, numThreads=0,
                     accumulate=False, _kernel=_lib.PP_GF64_KERNEL_MATVEC):
    """gf64_addon compute_recovery (src/gf64_addon.cc:1266-1434): blockSize in
    BYTES, a positive multiple of 8."""
    in_bytes = _buf_words(inputs, "inputs")
    out_bytes = _buf_words(outputs, "outputs")
    numInputs = _check_int(numInputs, "numInputs")
    numRecovery = _check_int(numRecovery, "numRecovery")
    blockSize = _check_int(blockSize, "blockSize")
    if not isinstance(firstInput, (int, np.integer)) or isinstance(firstInput, bool):
        raise TypeError("firstInput must be a Number or BigInt")
    if not isinstance(firstRecovery, (int, np.integer)) or isinstance(firstRecovery, bool):
        raise TypeError("firstRecovery must be a Number or BigInt")
    if not isinstance(accumulate, bool):
        raise TypeError("accumulate must be a boolean")
    if numInputs <= 0:
        raise ValueError("numInputs must be positive")
    if numRecovery <= 0:
        raise ValueError("numRecovery must be positive")
    if blockSize <= 0 or blockSize % 8:
        raise ValueError("blockSize must be positive and a multiple of 8")
    if in_bytes < numInputs * blockSize:
        raise ValueError("inputs buffer too small for numInputs * blockSize")
    if out_bytes < numRecovery * blockSize:
        raise ValueError("outputs buffer too small for numRecovery * blockSize")
    GF64Controller.ComputeRecoveryBlocks(inputs, numInputs, outputs, numRecovery, blockSize // 8, firstInput,
                                         firstRecovery, numThreads, accumulate, _kernel)


def compute_recovery_full(*a, **k):
    compute_recovery(*a, _kernel=_lib.PP_GF64_KERNEL_AUTO, **k)


def compute_recovery_barycentric(*a, **k):
    compute_recovery(*a, _kernel=_lib.PP_GF64_KERNEL_BARYCENTRIC, **k)


def compute_recovery_fenger(inputs, outputs, numInputs, numRecovery, blockSize, firstInput, firstRecovery,
                            numThreads=0):
    compute_recovery(inputs, outputs, numInputs, numRecovery, blockSize, firstInput, firstRecovery, numThreads,
                     False, _kernel=_lib.PP_GF64_KERNEL_FENGER)


def compute_recovery_accumulate(inputs, outputs, numInputs, numRecovery, blockSize, firstInput, firstRecovery,
                                numThreads=0):
    compute_recovery(inputs, outputs, numInputs, numRecovery, blockSize, firstInput, firstRecovery, numThreads, True)


def build_coefficient_matrix(numInputs, numRecovery, firstInput, firstRecovery):
    m = GF64Controller.BuildCauchyMatrixAlloc(numInputs, numRecovery, firstInput, firstRecovery)
    return m


def compute_recovery_with_coeff(inputs, outputs, numInputs, numRecovery, blockSize, coeff, numThreads=0,
                                accumulate=False):
    if blockSize <= 0 or blockSize % 8:
        raise ValueError("blockSize must be positive and a multiple of 8")
    GF64Controller.ComputeRecoveryBlocksWithCoeff(inputs, numInputs, outputs, numRecovery, blockSize // 8, coeff,
                                                  numThreads, accumulate)


def solve_and_reconstruct(A, rhs, n, blockSize):
    """Returns the solved RHS (in place); raises on a singular matrix like the
    N-API wrapper does."""
    if blockSize <= 0 or blockSize % 8:
        raise ValueError("blockSize must be positive and a multiple of 8")
    if GF64Controller.SolveAndReconstruct(A, rhs, n, blockSize // 8) != 0:
        raise PPError(_lib.PP_ERR_SINGULAR, "singular matrix")
    return rhs


def repair(inputs, missing, recovery, block_size64, first_input, first_recovery, restored=None,
           recovery_present=None, ctx=None):
    """PAR3 repair on the device (lib/par3gen.js:3840-4010): solve for the
    lost input blocks `missing` from the first len(missing) recovery blocks.
    inputs: (N, B) words (lost rows ignored); recovery: (n, B); returns the
    restored (n, B) blocks.  Raises PPError(PP_ERR_SINGULAR) where the
    reference's solve returns -1."""
    c = _ctx(ctx)
    miss = np.ascontiguousarray(np.asarray(missing, dtype=np.uint64))
    n = miss.size
    num_inputs = inputs.shape[0]
    if restored is None:
        restored = np.zeros((n, block_size64), dtype=np.uint64)
    pres = None if recovery_present is None else np.ascontiguousarray(np.asarray(recovery_present, dtype=np.uint8))
    c.check(lib.pp_gf64_repair(c.h, ptr(inputs), num_inputs, ptr(miss), n, ptr(recovery),
                               ptr(pres) if pres is not None else None, block_size64, _u64(first_input),
                               _u64(first_recovery), ptr(restored)))
    return restored


# ------------------------------------------------------------- region table
def gf64_region_mul(out, inp, length, constant, ctx=None):
    c = _ctx(ctx)
    c.check(lib.pp_gf64_region_mul(c.h, ptr(out), ptr(inp), length, _u64(constant)))


def gf64_region_mul_arr(out, inp, coeff, length, n_coeff, ctx=None):
    c = _ctx(ctx)
    c.check(lib.pp_gf64_region_mul_arr(c.h, ptr(out), ptr(inp), ptr(coeff), length, n_coeff))


def gf64_region_muladd_arr(out, inp, coeff, length, n_coeff, ctx=None):
    c = _ctx(ctx)
    c.check(lib.pp_gf64_region_muladd_arr(c.h, ptr(out), ptr(inp), ptr(coeff), length, n_coeff))


def _ptr_array(bufs):
    arr = (ctypes.c_void_p * len(bufs))(*[ptr(b) for b in bufs])
    return arr


def gf64_region_coupled_muladd_arr(out, in_blocks, coeff_blocks, length, G, ctx=None):
    c = _ctx(ctx)
    pa = _ptr_array(in_blocks)
    c.check(lib.pp_gf64_region_coupled_muladd_arr(c.h, ptr(out), ctypes.cast(pa, ctypes.c_void_p), ptr(coeff_blocks),
                                                  length, G))


def gf64_region_fused_output_muladd_arr(outs, inp, coeff_block_starts, length, K, ctx=None):
    c = _ctx(ctx)
    po = _ptr_array(outs)
    pc = _ptr_array(coeff_block_starts)
    c.check(lib.pp_gf64_region_fused_output_muladd_arr(c.h, ctypes.cast(po, ctypes.c_void_p), ptr(inp),
                                                       ctypes.cast(pc, ctypes.c_void_p), length, K))


def gf64_region_2d_muladd_arr(outs, K, in_blocks, G, coeff_block_2d, K_stride, length, ctx=None):
    c = _ctx(ctx)
    po = _ptr_array(outs)
    pi = _ptr_array(in_blocks)
    c.check(lib.pp_gf64_region_2d_muladd_arr(c.h, ctypes.cast(po, ctypes.c_void_p), K,
                                             ctypes.cast(pi, ctypes.c_void_p), G, ptr(coeff_block_2d), K_stride,
                                             length))


def gf64_inverse_batch(out, inp, n, ctx=None):
    c = _ctx(ctx)
    c.check(lib.pp_gf64_inverse_batch(c.h, ptr(out), ptr(inp), n))


def gf64_addfft64_fwd(arr, n=None, batch=1, ld=None, ctx=None):
    """Forward additive FFT (gf64_addfft64_fwd_recursive_scratch), in place.
    1-D: one polynomial; 2-D (n, batch): one polynomial per column."""
    c = _ctx(ctx)
    n, batch, ld = _fft_shape(arr, n, batch, ld)
    c.check(lib.pp_gf64_fft_fwd(c.h, ptr(arr), n, batch, ld))
    return arr


def gf64_addfft64_inv(arr, n=None, batch=1, ld=None, ctx=None):
    """Inverse additive FFT (gf64_addfft64_inv_recursive_scratch), in place,
    not normalised."""
    c = _ctx(ctx)
    n, batch, ld = _fft_shape(arr, n, batch, ld)
    c.check(lib.pp_gf64_fft_inv(c.h, ptr(arr), n, batch, ld))
    return arr


def _fft_shape(arr, n, batch, ld):
    shape = tuple(arr.shape)
    if len(shape) == 2:
        n = shape[0] if n is None else n
        batch = shape[1]
        ld = (arr.stride(0) if hasattr(arr, "stride") and callable(arr.stride) else arr.strides[0] // 8) \
            if ld is None else ld
    else:
        n = shape[0] if n is None else n
        ld = 1 if ld is None else ld
    return n, batch, ld


class Gf64Encoder:
    """gf64_addon Gf64Encoder (src/gf64_addon.cc:446,835 and export table)."""

    def __init__(self, ctx=None):
        self.ctx = _ctx(ctx)

    def mul(self, a: int, b: int) -> int:
        x = np.array([a], dtype=np.uint64)
        o = np.zeros(1, dtype=np.uint64)
        gf64_region_mul(o, x, 1, b, self.ctx)
        return int(o[0])

    def mul_arr(self, out, inp, coeff, length, n_coeff):
        gf64_region_mul_arr(out, inp, coeff, length, n_coeff, self.ctx)

    def coupled_muladd_arr(self, out, in_blocks, coeff_blocks, G, length):
        gf64_region_coupled_muladd_arr(out, in_blocks, coeff_blocks, length, G, self.ctx)

    def fused_output_muladd_arr(self, outs, inp, coeffs, K, length):
        gf64_region_fused_output_muladd_arr(outs, inp, coeffs, length, K, self.ctx)

    def two_d_muladd_arr(self, outs, K, in_blocks, G, coeff2d, K_stride, length):
        gf64_region_2d_muladd_arr(outs, K, in_blocks, G, coeff2d, K_stride, length, self.ctx)


# ------------------------------------------------------------ block hashes
def _nbytes(buf):
    return buf.numel() * buf.element_size() if hasattr(buf, "numel") else buf.nbytes


def block_hashes(blocks, block_size, first_index, after_checksum, num_blocks=None, block_stride=None, out=None,
                 ctx=None):
    """PAR3 data-block checksums (lib/par3gen.js:1001-1017, _inlineHashBlock):
    row i of the (n, 16) result is BLAKE3(after_checksum || u64le(first_index
    + i) || block_i)[:16].  blocks: a buffer of num_blocks blocks block_stride
    bytes apart (default: contiguous); after_checksum: 24 bytes."""
    c = _ctx(ctx)
    block_size = int(block_size)
    block_stride = block_size if block_stride is None else int(block_stride)
    if num_blocks is None:
        num_blocks = _nbytes(blocks) // block_stride if block_stride else 0
    ac = np.frombuffer(bytes(after_checksum), dtype=np.uint8)
    if ac.size != 24:
        raise ValueError("after_checksum must be 24 bytes")
    if out is None:
        out = np.empty((num_blocks, 16), dtype=np.uint8)
    c.check(lib.pp_par3_block_hashes(c.h, ptr(blocks), block_stride, num_blocks, block_size, _u64(first_index),
                                     ptr(ac), ptr(out)))
    return out


def assemble_recovery_packets(recoveryBlocksBuf, inputSetIdBuf, firstRecoveryIndex, numRecovery, blockSize,
                              out=None, ctx=None):
    """gf64_addon assemble_recovery_packets (src/gf64_addon.cc:2784-2936):
    numRecovery PAR3 RECOVERY packets of 64 + blockSize bytes, concatenated,
    with their BLAKE3 checksums.  Same argument checks (TypeError / RangeError
    become TypeError / ValueError).  Returns a numpy uint8 array unless an
    output buffer (host or CUDA) is given."""
    if recoveryBlocksBuf is None or not (hasattr(recoveryBlocksBuf, "data_ptr") or
                                         hasattr(recoveryBlocksBuf, "ctypes")):
        raise TypeError("recoveryBlocksBuf must be a Buffer")
    sid = np.frombuffer(bytes(inputSetIdBuf), dtype=np.uint8) if isinstance(inputSetIdBuf, (bytes, bytearray)) \
        else np.asarray(inputSetIdBuf, dtype=np.uint8).reshape(-1)
    if sid.size != 8:
        raise TypeError("inputSetIdBuf must be a 8-byte Buffer")
    if isinstance(firstRecoveryIndex, bool) or not isinstance(firstRecoveryIndex, (int, np.integer)):
        raise TypeError("firstRecoveryIndex must be a BigInt or Number")
    numRecovery = int(numRecovery)
    blockSize = int(blockSize)
    if numRecovery <= 0:
        raise ValueError("numRecovery must be a positive integer")
    if blockSize <= 0:
        raise ValueError("blockSize must be a positive integer")
    if numRecovery > (1 << 40) // blockSize:
        raise ValueError("numRecovery * blockSize exceeds 1 TiB cap")
    if _nbytes(recoveryBlocksBuf) != numRecovery * blockSize:
        raise ValueError("recoveryBlocksBuf length must equal numRecovery * blockSize")
    if out is None:
        out = np.empty(numRecovery * (64 + blockSize), dtype=np.uint8)
    elif _nbytes(out) < numRecovery * (64 + blockSize):
        raise ValueError("output buffer too small")
    c = _ctx(ctx)
    c.check(lib.pp_par3_assemble_recovery_packets(c.h, ptr(recoveryBlocksBuf), numRecovery, blockSize, ptr(sid),
                                                  _u64(firstRecoveryIndex), ptr(out)))
    return out


def create_packets(inputs, num_inputs, block_size64, first_input, num_recovery, first_recovery, input_set_id,
                   data_after_checksum=None, data_hashes=None, packets=None, ctx=None):
    """One create pass: the recovery packets of recovery blocks
    first_recovery.. and (when data_after_checksum is given) the input blocks'
    data-packet checksums, both from one staging of the inputs.  Returns
    (packets, data_hashes) -- numpy arrays unless buffers are given."""
    c = _ctx(ctx)
    sid = np.frombuffer(bytes(input_set_id), dtype=np.uint8)
    if sid.size != 8:
        raise TypeError("inputSetIdBuf must be a 8-byte Buffer")
    bs = int(block_size64) * 8
    if packets is None:
        packets = np.empty(int(num_recovery) * (64 + bs), dtype=np.uint8)
    ac = None
    if data_after_checksum is not None:
        ac = np.frombuffer(bytes(data_after_checksum), dtype=np.uint8)
        if ac.size != 24:
            raise ValueError("data_after_checksum must be 24 bytes")
        if data_hashes is None:
            data_hashes = np.empty((int(num_inputs), 16), dtype=np.uint8)
    c.check(lib.pp_par3_create_packets(c.h, ptr(inputs), num_inputs, block_size64, _u64(first_input), num_recovery,
                                       _u64(first_recovery), ptr(ac), ptr(data_hashes) if ac is not None else 0,
                                       ptr(sid), ptr(packets)))
    return packets, data_hashes


def par3_create_streaming(sourcePath, options, callback=None, recovery=None, data_hashes=None,
                          data_after_checksum=None, ctx=None):
    """gf64_addon par3_create_streaming(sourcePath, options, callback)
    (src/gf64_create_streaming.cc:93-506): PAR3 recovery blocks of a whole
    file, read in pipelined chunks and multiplied on the device.

    options: recoverySlices (required, > 0), blockSize (required, positive
    multiple of 8), firstInput, firstRecovery (default 0), numThreads and
    useMmap (accepted for parity; the reader uses parallel preads into pinned
    memory).  Result: {recoveryBytes, throughputMBps, durationMs,
    recoveryBuffer}; with callback, callback(err, result) is called instead of
    returning / raising (the reference's async completion).  Optional
    data_hashes (+ data_after_checksum) receive the input blocks' data-packet
    checksums from the same pass."""
    if not isinstance(options, dict):
        raise TypeError("options must be an object")
    if "recoverySlices" not in options:
        raise TypeError("options.recoverySlices is required")
    if "blockSize" not in options:
        raise TypeError("options.blockSize is required")
    R, bs = options["recoverySlices"], options["blockSize"]
    if isinstance(bs, bool) or not isinstance(bs, (int, np.integer)):
        raise TypeError("blockSize must be an integer")
    if isinstance(R, bool) or not isinstance(R, (int, np.integer)) or R <= 0:
        raise ValueError("recoverySlices must be a positive integer")
    if bs <= 0 or bs % 8:
        raise ValueError("blockSize must be positive and a multiple of 8")
    fI = options.get("firstInput") or 0
    fR = options.get("firstRecovery") or 0
    for v, name in ((fI, "firstInput"), (fR, "firstRecovery")):
        if isinstance(v, bool) or not isinstance(v, (int, np.integer)):
            raise TypeError(f"{name} must be a Number or BigInt")
    c = _ctx(ctx)
    if recovery is None:
        recovery = np.zeros(int(R) * int(bs), dtype=np.uint8)
    ac = None
    if data_hashes is not None:
        ac = np.frombuffer(bytes(data_after_checksum), dtype=np.uint8)
        if ac.size != 24:
            raise ValueError("data_after_checksum must be 24 bytes")
    st = _lib.PPStreamStats()
    status = lib.pp_par3_create_streaming(c.h, str(sourcePath).encode(), int(bs), int(R), _u64(fI), _u64(fR),
                                          ptr(recovery), ptr(ac), ptr(data_hashes), ctypes.byref(st))
    if status != PP_OK:
        err = PPError(status, lib.pp_ctx_last_error(c.h).decode())
        if callback is not None:
            callback(err, None)
            return None
        raise err
    rbytes = int(R) * int(bs)
    ms = st.seconds * 1e3
    result = {"recoveryBytes": rbytes, "throughputMBps": (rbytes / 1048576.0) / st.seconds if st.seconds else 0.0,
              "durationMs": ms, "recoveryBuffer": recovery, "bytesRead": int(st.bytes_read),
              "numInputs": int(st.num_inputs), "readMs": st.read_seconds * 1e3}
    if callback is not None:
        callback(None, result)
        return None
    return result


# ------------------------------------------------------ remaining N-API exports
def mul_arr(out, inp, coeff, len_words, n_coeff, ctx=None):
    """mul_arr export (src/gf64_addon.cc:3021-3150): out[w] = in[w] * coeff[w % n_coeff]."""
    if any(b is None for b in (out, inp, coeff)):
        raise TypeError("Requires out, in, coeff, len_words, n_coeff")
    len_words, n_coeff = _check_int(len_words, "len_words"), _check_int(n_coeff, "n_coeff")
    if n_coeff <= 0 and len_words > 0:
        raise ValueError("n_coeff must be positive")
    if _nbytes(out) < 8 * len_words or _nbytes(inp) < 8 * len_words or _nbytes(coeff) < 8 * n_coeff:
        raise ValueError("buffer too small")
    gf64_region_mul_arr(out, inp, coeff, len_words, n_coeff, ctx=ctx)


def xor_buffers(dst, src, ctx=None):
    """xor_buffers export (src/gf64_addon.cc:3216-3265): dst ^= src; equal lengths required."""
    if dst is None or src is None:
        raise TypeError("Requires dst and src Buffers")
    if _nbytes(dst) != _nbytes(src):
        raise ValueError(f"xor_buffers: dst.length ({_nbytes(dst)}) must equal src.length ({_nbytes(src)})")
    c = _ctx(ctx)
    c.check(lib.pp_xor_buffers(c.h, ptr(dst), ptr(src), _nbytes(dst)))


def gf64_solve(A, b, n, ctx=None):
    """gf64_solve export (src/gf64_addon.cc:1127-1230, gf64/gf64_solve.c:39-96):
    solve A x = b for one right-hand side; A and b are left unchanged.
    Returns x (numpy uint64, n words) or None if A is singular."""
    if A is None or b is None:
        raise TypeError("Requires A, b, and n")
    n = _check_int(n, "n")
    Ac = np.array(np.frombuffer(memoryview(A).cast("B"), dtype=np.uint64)[: n * n]) if not hasattr(A, "numel") \
        else np.array(A.cpu().numpy().view(np.uint64).reshape(-1)[: n * n])
    bc = np.array(np.frombuffer(memoryview(b).cast("B"), dtype=np.uint64)[:n]) if not hasattr(b, "numel") \
        else np.array(b.cpu().numpy().view(np.uint64).reshape(-1)[:n])
    if Ac.size < n * n or bc.size < n:
        raise ValueError("buffer too small for n")
    if n == 0:
        return np.zeros(0, dtype=np.uint64)
    rhs = bc.reshape(n, 1).copy()
    if GF64Controller.SolveAndReconstruct(Ac.reshape(n, n), rhs, n, 1) != 0:
        return None
    return rhs.reshape(-1)


def gf64_info(method=0):
    """gf64_info export (src/gf64_addon.cc:89-160): the arithmetic method in use."""
    return {"method": 4, "name": "CUDA sm_100a (tcgen05 int8 bit-matrix)", "alignment": 16}


def compute_recovery_streaming(inputBatches, outputBuffer, numInputs, numRecovery, blockSize, firstInput,
                               firstRecovery, numThreads=0, ctx=None):
    """compute_recovery_streaming export (src/gf64_addon.cc:2290-2480): the
    recovery of the concatenation of inputBatches (each a whole number of
    blocks), one pass per batch accumulating into outputBuffer."""
    if not isinstance(inputBatches, (list, tuple)):
        raise TypeError("inputBatches must be an array of Buffers")
    numInputs, numRecovery = _check_int(numInputs, "numInputs"), _check_int(numRecovery, "numRecovery")
    blockSize = _check_int(blockSize, "blockSize")
    if numInputs <= 0 or numRecovery <= 0:
        raise ValueError("numInputs and numRecovery must be positive")
    if blockSize <= 0 or blockSize % 8:
        raise ValueError("blockSize must be positive and a multiple of 8")
    counts = [_nbytes(bb) // blockSize for bb in inputBatches]
    if sum(counts) != numInputs or any(_nbytes(bb) % blockSize for bb in inputBatches):
        raise ValueError("inputBatches must hold numInputs whole blocks")
    if _nbytes(outputBuffer) < numRecovery * blockSize:
        raise ValueError("outputBuffer too small for numRecovery * blockSize")
    off = 0
    for k, (bb, cnt) in enumerate(zip(inputBatches, counts)):
        if cnt:
            GF64Controller.ComputeRecoveryBlocks(bb, cnt, outputBuffer, numRecovery, blockSize // 8,
                                                 _u64(firstInput) + off, firstRecovery, numThreads, off > 0)
        off += cnt


def get_last_decomposition_path():
    """get_last_decomposition_path export: the reference's CPU engine reports
    which input decomposition its last call used; this engine never splits the
    inputs into host-side decompositions, so it is always 0."""
    return 0


def isAlignedBuffer(buf, alignment=64):
    """isAlignedBuffer export (src/gf64_addon.cc:2976-3015)."""
    if buf is None or not (hasattr(buf, "data_ptr") or hasattr(buf, "ctypes")):
        return False
    if not isinstance(alignment, (int, np.integer)) or alignment <= 0 or alignment & (alignment - 1):
        alignment = 64
    return ptr(buf) % int(alignment) == 0


def allocAlignedBuffer(size):
    """allocAlignedBuffer export: a zeroed, 64-byte aligned host buffer."""
    size = _check_int(size, "Size")
    if size <= 0:
        raise ValueError("Size must be positive")
    raw = np.zeros(size + 64, dtype=np.uint8)
    off = (-raw.ctypes.data) % 64
    return raw[off: off + size]


def get_cpu_topology():
    """get_cpu_topology export (host information; the device engine does not
    depend on it)."""
    import os
    n = os.cpu_count() or 1
    return {"logicalCpus": n, "groups": 1}


def reset_cpu_topology_cache():
    return None


def get_effective_cpu_count():
    import os
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def reset_effective_cpu_count_cache():
    return None


def Gf64Encoder_create(method=0, ctx=None):
    return Gf64Encoder(ctx)


def Gf64Encoder_destroy(encoder):
    return None
