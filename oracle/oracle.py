"""Test infrastructure only: ctypes access to the oracle and the reference build.

``Oracle`` wraps ``oracle/liboracle.so`` (the C restatement, gf_oracle.c).
``Reference`` wraps ``oracle/_ref/libppref.so`` (the reference's own sources
compiled by oracle/Makefile; present only where it was built).
``Shim`` wraps ``oracle/_ref/libppshim.so``: the reference's PAR2Proc front
controller driving the CUDA backend shim (parparpar_b200/shim), alone or
beside the reference's PAR2ProcCPU.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libppref.so")
SHIM_SO = os.path.join(HERE, "_ref", "libppshim.so")

_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_U16 = ctypes.c_uint16
_U64 = ctypes.c_uint64


def _ptr(a: np.ndarray):
    return _P(a.ctypes.data)


def reference_dir():
    """The reference source tree: $PP_REFERENCE_DIR, else a checkout named
    `reference` beside this repository; None when neither exists."""
    ref = os.environ.get("PP_REFERENCE_DIR") or os.path.join(os.path.dirname(HERE), "..", "reference")
    ref = os.path.abspath(ref)
    return ref if os.path.isdir(ref) else None


def build(ref: bool = False) -> None:
    """Compile the oracle (and, when asked and the sources exist, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    src = reference_dir() if ref else None
    if src:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={src}"], check=True)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        self.L = L
        L.or_gf16_mul.restype = _U16
        L.or_gf16_mul.argtypes = [_U16, _U16]
        L.or_gf16_inv.restype = _U16
        L.or_gf16_inv.argtypes = [_U16]
        L.or_par2_input_log.restype = _U16
        L.or_par2_input_log.argtypes = [_U16]
        L.or_par2_coeff.restype = _U16
        L.or_par2_coeff.argtypes = [_U16, _U16]
        L.or_gf64_mul.restype = _U64
        L.or_gf64_mul.argtypes = [_U64, _U64]
        L.or_gf64_inv.restype = _U64
        L.or_gf64_inv.argtypes = [_U64]
        L.or_gf64_solve_and_reconstruct.restype = ctypes.c_int
        L.or_par2_invert.restype = ctypes.c_int

    # ---- GF(2^16) / PAR2 ---------------------------------------------------
    def gf16_mul(self, a: int, b: int) -> int:
        return self.L.or_gf16_mul(a, b)

    def par2_coeff(self, input_idx: int, exp: int) -> int:
        return self.L.or_par2_coeff(input_idx, exp)

    def par2_coeff_matrix(self, input_idx, exps) -> np.ndarray:
        """coeffs[o, i] = coeff(input_idx[i], exps[o])"""
        m = np.empty((len(exps), len(input_idx)), dtype=np.uint16)
        for o, e in enumerate(exps):
            for i, ii in enumerate(input_idx):
                m[o, i] = self.L.or_par2_coeff(int(ii), int(e))
        return m

    def par2_muladd(self, inputs, slice_size: int, coeffs: np.ndarray) -> np.ndarray:
        """inputs: list of uint8 arrays (each <= slice_size bytes);
        coeffs: (R, N) uint16.  Returns (R, slice_size) uint8."""
        n = len(inputs)
        r = coeffs.shape[0]
        bufs = [np.ascontiguousarray(x, dtype=np.uint8) for x in inputs]
        ptrs = (ctypes.c_void_p * max(n, 1))(*[b.ctypes.data for b in bufs])
        sizes = (_SZ * max(n, 1))(*[b.size for b in bufs])
        c = np.ascontiguousarray(coeffs, dtype=np.uint16)
        out = np.zeros((r, slice_size), dtype=np.uint8)
        self.L.or_par2_muladd(ptrs, sizes, ctypes.c_uint(n), _SZ(slice_size), _ptr(c),
                              ctypes.c_uint(r), _ptr(out))
        return out

    def par2_invert(self, valid, recovery):
        """Returns (ok, factors (m, N) uint16, recovery_used list)."""
        v = np.ascontiguousarray(np.asarray(valid, dtype=np.uint8))
        n = v.size
        m = int(n - v.astype(bool).sum())
        rec = np.ascontiguousarray(np.asarray(recovery, dtype=np.uint16)).copy()
        nrec = ctypes.c_uint(rec.size)
        f = np.zeros((max(m, 1), n), dtype=np.uint16)
        ok = self.L.or_par2_invert(_ptr(v), ctypes.c_uint(n), _ptr(rec), ctypes.byref(nrec), _ptr(f))
        return bool(ok), f[:m], [int(x) for x in rec[: nrec.value]]

    # ---- GF(2^64) / PAR3 ---------------------------------------------------
    def gf64_mul(self, a: int, b: int) -> int:
        return self.L.or_gf64_mul(a, b)

    def gf64_inv(self, a: int) -> int:
        return self.L.or_gf64_inv(a)

    def gf64_build_cauchy(self, n_in: int, n_rec: int, first_in: int, first_rec: int) -> np.ndarray:
        m = np.zeros((n_rec, n_in), dtype=np.uint64)
        self.L.or_gf64_build_cauchy(_ptr(m), _SZ(n_in), _SZ(n_rec), _U64(first_in), _U64(first_rec))
        return m

    def gf64_matvec(self, inputs: np.ndarray, coeff: np.ndarray, out: np.ndarray | None = None,
                    accumulate: bool = False) -> np.ndarray:
        inputs = np.ascontiguousarray(inputs, dtype=np.uint64)
        n, b = inputs.shape
        r = coeff.shape[0]
        if out is None:
            out = np.zeros((r, b), dtype=np.uint64)
        c = np.ascontiguousarray(coeff, dtype=np.uint64)
        self.L.or_gf64_matvec(_ptr(inputs), _SZ(n), _ptr(out), _SZ(r), _SZ(b), _ptr(c),
                              ctypes.c_int(1 if accumulate else 0))
        return out

    def gf64_compute_recovery(self, inputs: np.ndarray, n_rec: int, first_in: int, first_rec: int,
                              out: np.ndarray | None = None, accumulate: bool = False) -> np.ndarray:
        inputs = np.ascontiguousarray(inputs, dtype=np.uint64)
        n, b = inputs.shape
        if out is None:
            out = np.zeros((n_rec, b), dtype=np.uint64)
        self.L.or_gf64_compute_recovery(_ptr(inputs), _SZ(n), _ptr(out), _SZ(n_rec), _SZ(b),
                                        _U64(first_in), _U64(first_rec),
                                        ctypes.c_int(1 if accumulate else 0))
        return out

    def gf64_solve_and_reconstruct(self, A: np.ndarray, rhs: np.ndarray) -> int:
        n = A.shape[0]
        b = rhs.shape[1] if rhs.ndim == 2 else 0
        return self.L.or_gf64_solve_and_reconstruct(_ptr(A), _ptr(rhs), _SZ(n), _SZ(b))

    def gf64_fft(self, a: np.ndarray, inverse: bool = False) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        (self.L.or_gf64_fft_inv if inverse else self.L.or_gf64_fft_fwd)(_ptr(a), _SZ(a.size))
        return a

    def gf64_region(self, op: str, inp: np.ndarray, coeff, out: np.ndarray) -> np.ndarray:
        c = np.ascontiguousarray(np.atleast_1d(np.asarray(coeff, dtype=np.uint64)))
        if op == "mul":
            self.L.or_gf64_region_mul(_ptr(out), _ptr(inp), _SZ(inp.size), _U64(int(c[0])))
        elif op == "mul_arr":
            self.L.or_gf64_region_mul_arr(_ptr(out), _ptr(inp), _ptr(c), _SZ(inp.size), _SZ(c.size))
        elif op == "muladd_arr":
            self.L.or_gf64_region_muladd_arr(_ptr(out), _ptr(inp), _ptr(c), _SZ(inp.size), _SZ(c.size))
        else:
            raise ValueError(op)
        return out


    # ---- block hashes -----------------------------------------------------
    def blake3(self, data, out_len: int = 32) -> bytes:
        a = np.frombuffer(bytes(data), dtype=np.uint8)
        out = np.zeros(out_len, dtype=np.uint8)
        self.L.or_blake3(_ptr(a) if a.size else None, _SZ(a.size), _ptr(out), _SZ(out_len))
        return out.tobytes()

    def par3_block_hashes(self, blocks: np.ndarray, first_index: int, after_checksum: bytes) -> np.ndarray:
        """blocks: (n, block_size) uint8 -> (n, 16) (lib/par3gen.js:1001-1017)."""
        blocks = np.ascontiguousarray(blocks, dtype=np.uint8)
        n, bs = blocks.shape
        ac = np.frombuffer(bytes(after_checksum), dtype=np.uint8).copy()
        out = np.zeros((n, 16), dtype=np.uint8)
        self.L.or_par3_block_hashes(_ptr(blocks), _SZ(bs), _SZ(n), _SZ(bs), _U64(first_index), _ptr(ac), _ptr(out))
        return out

    def par3_recovery_packets(self, recovery: np.ndarray, input_set_id: bytes, first_index: int) -> np.ndarray:
        """recovery: (n, block_size) uint8 -> n * (64 + block_size) bytes
        (src/gf64_addon.cc:2884-2934)."""
        recovery = np.ascontiguousarray(recovery, dtype=np.uint8)
        n, bs = recovery.shape
        sid = np.frombuffer(bytes(input_set_id), dtype=np.uint8).copy()
        out = np.zeros(n * (64 + bs), dtype=np.uint8)
        self.L.or_par3_recovery_packets(_ptr(recovery), _SZ(n), _SZ(bs), _ptr(sid), _U64(first_index), _ptr(out))
        return out


    def par2_memory_checksums(self, rows: np.ndarray, slice_size: int) -> np.ndarray:
        rows = np.ascontiguousarray(rows, dtype=np.uint8)
        out = np.zeros((rows.shape[0], 16), dtype=np.uint8)
        for r in range(rows.shape[0]):
            self.L.or_par2_mem_cksum(_ptr(rows[r]), _SZ(slice_size), _ptr(out[r]))
        return out


def par2_block_hashes(blocks: np.ndarray, slice_size: int, lengths=None) -> np.ndarray:
    """PAR2 IFSC entries, HasherInput::getBlock(md5crc, zeroPad)
    (hasher/hasher_input_base.h:104-117): MD5 of the block's data followed by
    zeroPad zero bytes, then CRC32 of the same bytes, little-endian.  MD5 is
    RFC 1321 and CRC32 the reflected 0xEDB88320 CRC with ~0 init and final
    xor, here from Python's hashlib and zlib."""
    import hashlib
    import zlib

    blocks = np.asarray(blocks, dtype=np.uint8)
    n = blocks.shape[0]
    out = np.zeros((n, 20), dtype=np.uint8)
    for i in range(n):
        ln = slice_size if lengths is None else int(lengths[i])
        msg = blocks[i, :ln].tobytes() + bytes(slice_size - ln)
        out[i, :16] = np.frombuffer(hashlib.md5(msg).digest(), dtype=np.uint8)
        out[i, 16:] = np.frombuffer((zlib.crc32(msg) & 0xFFFFFFFF).to_bytes(4, "little"), dtype=np.uint8)
    return out


def par2_recovery_packet_headers(slices: np.ndarray, exps, set_id: bytes, slice_size: int) -> np.ndarray:
    """lib/par2.js:240-330 (packet MD5 over set id, type, u32le exponent and
    the slice) and :517-530 (getRecoveryHeader: magic, u64le length, MD5, set
    id, type, exponent); MD5 from hashlib."""
    import hashlib

    n = slices.shape[0]
    out = np.zeros((n, 68), dtype=np.uint8)
    for i in range(n):
        body = bytes(set_id) + b"PAR 2.0\x00RecvSlic" + int(exps[i]).to_bytes(4, "little")
        md5 = hashlib.md5(body + slices[i, :slice_size].tobytes()).digest()
        hdr = b"PAR2\x00PKT" + (68 + slice_size).to_bytes(8, "little") + md5 + body
        out[i] = np.frombuffer(hdr, dtype=np.uint8)
    return out


def pattern_bytes(n: int, seed: int) -> np.ndarray:
    """Deterministic pseudo-random bytes (a multiplicative hash of the index),
    independent of any RNG implementation; fixtures store only outputs."""
    with np.errstate(over="ignore"):
        x = np.arange(n, dtype=np.uint64) + np.uint64(seed)
        x = x * np.uint64(0x9E3779B97F4A7C15)
        x ^= x >> np.uint64(29)
        x = x * np.uint64(0xBF58476D1CE4E5B9)
    return (x >> np.uint64(56)).astype(np.uint8)


class Reference:
    """The reference's own implementation, built from its sources (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        self.L = L
        L.ref_gf64_mul.restype = _U64
        L.ref_gf64_mul.argtypes = [_U64, _U64]
        L.ref_gf64_inverse.restype = _U64
        L.ref_gf64_inverse.argtypes = [_U64]
        L.ref_gfmat_coeff.restype = _U16
        L.ref_gfmat_coeff.argtypes = [_U16, _U16]
        L.ref_gfmat_input_log.restype = _U16
        L.ref_gfmat_input_log.argtypes = [_U16]
        L.ref_par2_method.restype = ctypes.c_char_p
        L.ref_gf64_solve_and_reconstruct.restype = ctypes.c_int

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def par2_create(self, inputs: np.ndarray, slice_size: int, input_idx, exps, last_size=None,
                    threads: int = 0) -> tuple[np.ndarray, bool]:
        """inputs: (N, slice_size) uint8 (the last row may be logically shorter)."""
        inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
        n = inputs.shape[0]
        idx = np.ascontiguousarray(np.asarray(input_idx, dtype=np.uint16))
        ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
        out = np.zeros((ex.size, slice_size), dtype=np.uint8)
        ok = self.L.ref_par2_create(_ptr(inputs), ctypes.c_uint(n), _SZ(slice_size),
                                    _SZ(slice_size if last_size is None else last_size), _ptr(idx),
                                    _ptr(ex), ctypes.c_uint(ex.size), _ptr(out), ctypes.c_int(threads))
        return out, ok == 1

    def par2_create_coeffs(self, inputs: np.ndarray, slice_size: int, coeffs: np.ndarray,
                           threads: int = 0) -> tuple[np.ndarray, bool]:
        """coeffs: (R, N); the reference takes per-input columns."""
        inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
        n = inputs.shape[0]
        r = coeffs.shape[0]
        col = np.ascontiguousarray(coeffs.T.astype(np.uint16))
        out = np.zeros((r, slice_size), dtype=np.uint8)
        ok = self.L.ref_par2_create_coeffs(_ptr(inputs), ctypes.c_uint(n), _SZ(slice_size), _ptr(col),
                                           ctypes.c_uint(r), _ptr(out), ctypes.c_int(threads))
        return out, ok == 1

    def par2_method(self) -> str:
        return self.L.ref_par2_method().decode()

    def par2_invert(self, valid, recovery, threads: int = 0):
        v = np.ascontiguousarray(np.asarray(valid, dtype=np.uint8))
        n = v.size
        m = int(n - v.astype(bool).sum())
        rec = np.ascontiguousarray(np.asarray(recovery, dtype=np.uint16)).copy()
        nrec = ctypes.c_uint(rec.size)
        f = np.zeros((max(m, 1), n), dtype=np.uint16)
        ok = self.L.ref_par2_invert(_ptr(v), ctypes.c_uint(n), _ptr(rec), ctypes.byref(nrec), _ptr(f),
                                    ctypes.c_int(threads))
        return bool(ok), f[:m], [int(x) for x in rec[: nrec.value]]

    def gf64_compute_recovery(self, kind: int, inputs: np.ndarray, n_rec: int, first_in: int,
                              first_rec: int, out: np.ndarray | None = None, accumulate=False,
                              threads: int = 0) -> np.ndarray:
        inputs = np.ascontiguousarray(inputs, dtype=np.uint64)
        n, b = inputs.shape
        if out is None:
            out = np.zeros((n_rec, b), dtype=np.uint64)
        self.L.ref_gf64_compute_recovery(ctypes.c_int(kind), _ptr(inputs), _SZ(n), _ptr(out), _SZ(n_rec),
                                         _SZ(b), _U64(first_in), _U64(first_rec), ctypes.c_int(threads),
                                         ctypes.c_int(1 if accumulate else 0))
        return out

    def gf64_build_cauchy(self, n_in, n_rec, first_in, first_rec) -> np.ndarray:
        m = np.zeros((n_rec, n_in), dtype=np.uint64)
        self.L.ref_gf64_build_cauchy(_ptr(m), _SZ(n_in), _SZ(n_rec), _U64(first_in), _U64(first_rec))
        return m

    def gf64_solve_and_reconstruct(self, A: np.ndarray, rhs: np.ndarray) -> int:
        n = A.shape[0]
        b = rhs.shape[1]
        return self.L.ref_gf64_solve_and_reconstruct(_ptr(A), _ptr(rhs), _SZ(n), _SZ(b))

    def gf64_fft_fwd(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.ref_gf64_fft_fwd(_ptr(a), _SZ(a.size))
        return a

    def gf64_fft_inv(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.ref_gf64_fft_inv(_ptr(a), _SZ(a.size))
        return a

    # ---- block hashes -----------------------------------------------------
    def par2_hasher_method(self) -> str:
        self.L.ref_par2_hasher_method.restype = ctypes.c_char_p
        return self.L.ref_par2_hasher_method().decode()

    def par2_hash_file(self, data: np.ndarray, slice_size: int):
        """One file through the reference hasher (the variant it selects for
        this CPU): (IFSC entries (n, 20), file MD5)."""
        data = np.ascontiguousarray(data, dtype=np.uint8)
        n = (data.size + slice_size - 1) // slice_size
        ifsc = np.zeros((max(n, 1), 20), dtype=np.uint8)
        md5 = np.zeros(16, dtype=np.uint8)
        self.L.ref_par2_hash_file(_ptr(data) if data.size else None, _SZ(data.size), _SZ(slice_size), _ptr(ifsc),
                                  _ptr(md5))
        return ifsc[:n], md5.tobytes()

    def blake3(self, data, out_len: int = 32) -> bytes:
        a = np.frombuffer(bytes(data), dtype=np.uint8)
        out = np.zeros(out_len, dtype=np.uint8)
        self.L.ref_blake3(_ptr(a) if a.size else None, _SZ(a.size), _ptr(out), _SZ(out_len))
        return out.tobytes()

    def par3_block_hashes(self, blocks: np.ndarray, first_index: int, after_checksum: bytes) -> np.ndarray:
        blocks = np.ascontiguousarray(blocks, dtype=np.uint8)
        n, bs = blocks.shape
        ac = np.frombuffer(bytes(after_checksum), dtype=np.uint8).copy()
        out = np.zeros((n, 16), dtype=np.uint8)
        self.L.ref_par3_block_hashes(_ptr(blocks), _SZ(n), _SZ(bs), _U64(first_index), _ptr(ac), _ptr(out))
        return out

    def par3_recovery_packets(self, recovery: np.ndarray, input_set_id: bytes, first_index: int) -> np.ndarray:
        recovery = np.ascontiguousarray(recovery, dtype=np.uint8)
        n, bs = recovery.shape
        sid = np.frombuffer(bytes(input_set_id), dtype=np.uint8).copy()
        out = np.zeros(n * (64 + bs), dtype=np.uint8)
        self.L.ref_par3_assemble_recovery_packets(_ptr(recovery), _SZ(n), _SZ(bs), _ptr(sid), _U64(first_index),
                                                  _ptr(out))
        return out


class Shim:
    """PAR2Proc (the reference's controller) over PAR2ProcCUDA: byte range
    [0, split) of every slice on the reference's PAR2ProcCPU, [split, slice)
    on the GPU (split 0: the GPU alone; split = slice: the CPU alone)."""

    def __init__(self, path: str = SHIM_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = ctypes.CDLL(path)

    @staticmethod
    def available(path: str = SHIM_SO) -> bool:
        return os.path.exists(path)

    def par2_create(self, inputs: np.ndarray, slice_size: int, input_idx, exps, split: int, last_size=None,
                    device: int = 0, threads: int = 0) -> tuple[np.ndarray, int]:
        """Returns (outputs, status): status 1 = every output valid, 0 = an
        output failed its memory checksum, < 0 = a set-up error."""
        inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
        n = inputs.shape[0]
        idx = np.ascontiguousarray(np.asarray(input_idx, dtype=np.uint16))
        ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
        out = np.zeros((ex.size, slice_size), dtype=np.uint8)
        st = self.L.shim_par2_create(_ptr(inputs), ctypes.c_uint(n), _SZ(slice_size),
                                     _SZ(slice_size if last_size is None else last_size), _ptr(idx), _ptr(ex),
                                     ctypes.c_uint(ex.size), _ptr(out), _SZ(split), ctypes.c_int(device),
                                     ctypes.c_int(threads))
        return out, st

    def par2_create_coeffs(self, inputs: np.ndarray, slice_size: int, coeffs: np.ndarray, split: int,
                           device: int = 0, threads: int = 0) -> tuple[np.ndarray, int]:
        """coeffs: (R, N) as the region product takes them."""
        inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
        n = inputs.shape[0]
        r = coeffs.shape[0]
        col = np.ascontiguousarray(coeffs.T.astype(np.uint16))
        out = np.zeros((r, slice_size), dtype=np.uint8)
        st = self.L.shim_par2_create_coeffs(_ptr(inputs), ctypes.c_uint(n), _SZ(slice_size), _ptr(col),
                                            ctypes.c_uint(r), _ptr(out), _SZ(split), ctypes.c_int(device),
                                            ctypes.c_int(threads))
        return out, st

    def par2_resize_then_create(self, inputs: np.ndarray, first_size: int, slice_size: int, input_idx, exps,
                                device: int = 0) -> tuple[np.ndarray, int]:
        inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
        n = inputs.shape[0]
        idx = np.ascontiguousarray(np.asarray(input_idx, dtype=np.uint16))
        ex = np.ascontiguousarray(np.asarray(exps, dtype=np.uint16))
        out = np.zeros((ex.size, slice_size), dtype=np.uint8)
        st = self.L.shim_par2_resize_then_create(_ptr(inputs), ctypes.c_uint(n), _SZ(first_size), _SZ(slice_size),
                                                 _ptr(idx), _ptr(ex), ctypes.c_uint(ex.size), _ptr(out),
                                                 ctypes.c_int(device))
        return out, st
