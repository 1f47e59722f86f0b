"""ctypes binding of libparpar_b200.so (the C ABI declared in include/parpar_b200.h).

The library is the product: there is no Python or CPU implementation behind
these calls.  If the shared library is missing or cannot be loaded, importing
this module raises; if no CUDA device is present, creating a context raises
``PPError(PP_ERR_NO_DEVICE)``.
"""
from __future__ import annotations

import ctypes
import os
import sys
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libparpar_b200.so")

PP_OK = 0
PP_ERR_INVALID_ARG = -1
PP_ERR_CUDA = -2
PP_ERR_NO_MEMORY = -3
PP_ERR_SINGULAR = -4
PP_ERR_NOT_INVERTIBLE = -5
PP_ERR_BUSY = -6
PP_ERR_NO_DEVICE = -7
PP_ERR_UNSUPPORTED = -8
PP_ERR_TIMEOUT = -9
PP_ERR_TOO_LARGE = -10
PP_ERR_IO = -11
PP_NOALLOC_SOLVE_MAX_N = 4096

PP_GF16_KERNEL_AUTO = 0
PP_GF16_KERNEL_LUT = 1
PP_GF16_KERNEL_TENSOR = 2

PP_PROC_ADD_OK = 0
PP_PROC_ADD_OK_BUSY = 1
PP_PROC_ADD_FULL = 2

PP_GF64_KERNEL_AUTO = 0
PP_GF64_KERNEL_MATVEC = 1
PP_GF64_KERNEL_BARYCENTRIC = 2
PP_GF64_KERNEL_FENGER = 3

# every symbol declared in include/parpar_b200.h
EXPORTS = [
    "pp_version", "pp_status_string", "pp_ctx_create", "pp_ctx_destroy", "pp_ctx_set_stream",
    "pp_ctx_get_stream", "pp_ctx_synchronize", "pp_ctx_last_error", "pp_launch_count", "pp_ctx_free_cache",
    "pp_ctx_set_gf16_kernel", "pp_ctx_set_gf64_kernel", "pp_ctx_set_kernel_timing", "pp_ctx_kernel_time",
    "pp_par2_coeff", "pp_par2_input_log", "pp_par2_coeff_matrix", "pp_gf16_muladd", "pp_par2_create",
    "pp_par2_invert", "pp_par2_proc_create", "pp_par2_proc_destroy", "pp_par2_proc_set_current_slice_size",
    "pp_par2_proc_set_recovery_slices", "pp_par2_proc_can_add", "pp_par2_proc_wait_for_add",
    "pp_par2_proc_add_input", "pp_par2_proc_add_input_coeffs", "pp_par2_proc_flush", "pp_par2_proc_end_input",
    "pp_par2_proc_get_output", "pp_par2_proc_discard_output", "pp_par2_proc_output_ptr",
    "pp_par2_proc_free_processing_mem",
    "pp_par2_proc_set_input_hashes", "pp_par2_proc_get_input_hashes",
    "pp_par2_proc_input_batch_size", "pp_par2_proc_batches_started", "pp_par2_proc_batches_done",
    "pp_par2_proc_wait_batches", "pp_gf64_build_cauchy",
    "pp_gf64_compute_recovery", "pp_gf64_compute_recovery_with_coeff", "pp_gf64_solve_and_reconstruct",
    "pp_gf64_region_mul", "pp_gf64_region_mul_arr", "pp_gf64_region_muladd_arr",
    "pp_gf64_region_coupled_muladd_arr", "pp_gf64_region_fused_output_muladd_arr",
    "pp_gf64_region_2d_muladd_arr", "pp_gf64_inverse_batch", "pp_gf64_fft_fwd", "pp_gf64_fft_inv",
    "pp_gf64_solve_and_reconstruct_noalloc", "pp_gf64_repair",
    "pp_batch_create", "pp_batch_run", "pp_batch_launches", "pp_batch_destroy",
    "pp_server_create", "pp_server_submit", "pp_server_wait", "pp_server_get_stats", "pp_server_reset_stats",
    "pp_server_last_error", "pp_server_destroy",
    "pp_par2_block_hashes", "pp_par3_block_hashes", "pp_par3_assemble_recovery_packets",
    "pp_par2_create_hashed", "pp_par3_create_packets", "pp_par2_memory_checksums", "pp_par3_create_streaming",
    "pp_par2_recovery_packet_headers", "pp_xor_buffers", "pp_par2_create_split", "pp_gf64_compute_recovery_split",
]


class PPError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"parpar_b200 error {status}: {msg}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python parparpar_b200/build.py` "
            "(the CUDA engine has no CPU fallback)")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_U = ctypes.c_uint
_I = ctypes.c_int
_U16 = ctypes.c_uint16
_U64 = ctypes.c_uint64


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)


_sig("pp_version", ctypes.c_char_p)
_sig("pp_status_string", ctypes.c_char_p, _I)
_sig("pp_ctx_create", _I, _I, ctypes.POINTER(_P))
_sig("pp_ctx_destroy", None, _P)
_sig("pp_ctx_set_stream", _I, _P, _P)
_sig("pp_ctx_get_stream", _P, _P)
_sig("pp_ctx_synchronize", _I, _P)
_sig("pp_ctx_last_error", ctypes.c_char_p, _P)
_sig("pp_launch_count", _U64)
_sig("pp_ctx_free_cache", _I, _P)
_sig("pp_ctx_set_gf16_kernel", _I, _P, _I)
_sig("pp_ctx_set_gf64_kernel", _I, _P, _I)
_sig("pp_par2_coeff", _U16, _U16, _U16)
_sig("pp_par2_input_log", _U16, _U16)
_sig("pp_par2_coeff_matrix", _I, _P, _P, _U, _P, _U, _P)
_sig("pp_gf16_muladd", _I, _P, _P, _SZ, _U, _SZ, _P, _SZ, _U, _P, _SZ, _I)
_sig("pp_par2_create", _I, _P, _P, _SZ, _U, _SZ, _P, _P, _U, _P, _SZ)
_sig("pp_par2_invert", _I, _P, _P, _U, _P, ctypes.POINTER(_U), _P)
_sig("pp_par2_proc_create", _I, _P, _SZ, _U, _U, ctypes.POINTER(_P))
_sig("pp_par2_proc_destroy", None, _P)
_sig("pp_par2_proc_set_current_slice_size", _I, _P, _SZ)
_sig("pp_par2_proc_set_recovery_slices", _I, _P, _U, _P)
_sig("pp_par2_proc_can_add", _I, _P)
_sig("pp_par2_proc_wait_for_add", _I, _P)
_sig("pp_par2_proc_add_input", _I, _P, _P, _SZ, _U16, _I)
_sig("pp_par2_proc_add_input_coeffs", _I, _P, _P, _SZ, _P, _I)
_sig("pp_par2_proc_flush", _I, _P)
_sig("pp_par2_proc_end_input", _I, _P)
_sig("pp_par2_proc_get_output", _I, _P, _U, _P, ctypes.POINTER(_I))
_sig("pp_par2_proc_discard_output", _I, _P)
_sig("pp_par2_proc_output_ptr", _I, _P, _U, ctypes.POINTER(_P))
_sig("pp_par2_proc_set_input_hashes", _I, _P, _U)
_sig("pp_par2_proc_get_input_hashes", _I, _P, _P, _U)
_sig("pp_par2_proc_free_processing_mem", _I, _P)
_sig("pp_par2_proc_input_batch_size", _U, _P)
_sig("pp_par2_proc_batches_started", _U, _P)
_sig("pp_par2_proc_batches_done", _U, _P)
_sig("pp_par2_proc_wait_batches", _I, _P, _U)
_sig("pp_gf64_build_cauchy", _I, _P, _P, _SZ, _SZ, _U64, _U64)
_sig("pp_ctx_set_kernel_timing", _I, _P, _I)
_sig("pp_ctx_kernel_time", _I, _P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_U64))
_sig("pp_gf64_compute_recovery", _I, _P, _P, _SZ, _P, _SZ, _SZ, _U64, _U64, _I, _I)
_sig("pp_par2_create_split", _I, _P, _P, _P, _U, _P, _SZ, _U, _SZ, _P, _P, _U, _P, _SZ)
_sig("pp_gf64_compute_recovery_split", _I, _P, _P, _P, _U, _P, _SZ, _P, _SZ, _SZ, _U64, _U64)
_sig("pp_gf64_compute_recovery_with_coeff", _I, _P, _P, _SZ, _P, _SZ, _SZ, _P, _I)
_sig("pp_gf64_solve_and_reconstruct", _I, _P, _P, _P, _SZ, _SZ)
_sig("pp_gf64_region_mul", _I, _P, _P, _P, _SZ, _U64)
_sig("pp_gf64_region_mul_arr", _I, _P, _P, _P, _P, _SZ, _SZ)
_sig("pp_gf64_region_muladd_arr", _I, _P, _P, _P, _P, _SZ, _SZ)
_sig("pp_gf64_region_coupled_muladd_arr", _I, _P, _P, _P, _P, _SZ, _SZ)
_sig("pp_gf64_region_fused_output_muladd_arr", _I, _P, _P, _P, _P, _SZ, _SZ)
_sig("pp_gf64_region_2d_muladd_arr", _I, _P, _P, _SZ, _P, _SZ, _P, _SZ, _SZ)
_sig("pp_gf64_inverse_batch", _I, _P, _P, _P, _SZ)
_sig("pp_gf64_fft_fwd", _I, _P, _P, _SZ, _SZ, _SZ)
_sig("pp_gf64_fft_inv", _I, _P, _P, _SZ, _SZ, _SZ)
_sig("pp_gf64_solve_and_reconstruct_noalloc", _I, _P, _P, _SZ, _SZ, _P)
_sig("pp_gf64_repair", _I, _P, _P, _SZ, _P, _SZ, _P, _P, _SZ, _U64, _U64, _P)
_sig("pp_par2_block_hashes", _I, _P, _P, _SZ, _SZ, _SZ, _P, _P)
_sig("pp_par2_memory_checksums", _I, _P, _P, _SZ, _SZ, _SZ, _P)
_sig("pp_par2_recovery_packet_headers", _I, _P, _P, _SZ, _SZ, _SZ, _P, _P, _P)
_sig("pp_xor_buffers", _I, _P, _P, _P, _SZ)


class PPStreamStats(ctypes.Structure):
    _fields_ = [("bytes_read", ctypes.c_uint64), ("num_inputs", ctypes.c_uint64), ("seconds", ctypes.c_double),
                ("read_seconds", ctypes.c_double)]


_sig("pp_par3_create_streaming", _I, _P, ctypes.c_char_p, _SZ, _SZ, _U64, _U64, _P, _P, _P,
     ctypes.POINTER(PPStreamStats))
_sig("pp_par2_create_hashed", _I, _P, _P, _SZ, _U, _SZ, _P, _P, _U, _P, _SZ, _P)
_sig("pp_par3_block_hashes", _I, _P, _P, _SZ, _SZ, _SZ, _U64, _P, _P)
_sig("pp_par3_assemble_recovery_packets", _I, _P, _P, _SZ, _SZ, _P, _U64, _P)
_sig("pp_par3_create_packets", _I, _P, _P, _SZ, _SZ, _U64, _SZ, _U64, _P, _P, _P, _P)

PP_JOB_PAR2_CREATE = 1
PP_JOB_PAR3_CREATE = 2
PP_JOB_PAR3_REPAIR = 3
PP_JOB_GF16_MULADD = 4
PP_BATCH_TUNE = 1
PP_BATCH_NO_GRAPH = 2


class PPJob(ctypes.Structure):
    """struct pp_job (include/parpar_b200.h)"""
    _fields_ = [
        ("kind", ctypes.c_int),
        ("inputs", ctypes.c_void_p),
        ("input_stride", ctypes.c_size_t),
        ("num_inputs", ctypes.c_size_t),
        ("slice_bytes", ctypes.c_size_t),
        ("input_ids", ctypes.c_void_p),
        ("exponents", ctypes.c_void_p),
        ("num_recovery", ctypes.c_size_t),
        ("outputs", ctypes.c_void_p),
        ("output_stride", ctypes.c_size_t),
        ("first_input", ctypes.c_uint64),
        ("first_recovery", ctypes.c_uint64),
        ("missing", ctypes.c_void_p),
        ("num_missing", ctypes.c_size_t),
        ("recovery", ctypes.c_void_p),
        ("recovery_stride", ctypes.c_size_t),
        ("recovery_present", ctypes.c_void_p),
        ("coeffs", ctypes.c_void_p),
    ]


class PPServerStats(ctypes.Structure):
    """struct pp_server_stats (include/parpar_b200.h)"""
    _fields_ = [
        ("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
        ("waves", ctypes.c_uint64), ("input_bytes", ctypes.c_uint64), ("elapsed_s", ctypes.c_double),
        ("gbps", ctypes.c_double), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
        ("max_ms", ctypes.c_double), ("hbm_peak_bytes", ctypes.c_uint64), ("tables_resident", ctypes.c_uint64),
        ("table_bytes", ctypes.c_uint64),
    ]


_sig("pp_batch_create", _I, _P, ctypes.POINTER(PPJob), _SZ, _I, ctypes.POINTER(_P))
_sig("pp_batch_run", _I, _P)
_sig("pp_batch_launches", _I, _P)
_sig("pp_batch_destroy", None, _P)
_sig("pp_server_create", _I, _I, _SZ, _I, _I, ctypes.POINTER(_P))
_sig("pp_server_submit", _I, _P, ctypes.POINTER(PPJob), ctypes.POINTER(_U64))
_sig("pp_server_wait", _I, _P, _U64, _I)
_sig("pp_server_get_stats", _I, _P, ctypes.POINTER(PPServerStats))
_sig("pp_server_reset_stats", None, _P)
_sig("pp_server_last_error", ctypes.c_char_p, _P)
_sig("pp_server_destroy", None, _P)


def status_string(s: int) -> str:
    return lib.pp_status_string(s).decode()


class Context:
    """One device + stream.  ``check`` turns statuses into ``PPError``.

    The library runs a context's work on its CUDA stream.  From Python that
    stream follows torch's current stream on the context's device (as a torch
    operation would), so CUDA tensors produced before a call are ready when
    its kernels read them and torch work queued after it sees its results;
    the module functions rebind before every call (``follow_torch``).
    ``set_stream`` pins an explicit stream instead."""

    def __init__(self, device: int = 0):
        h = _P()
        st = lib.pp_ctx_create(device, ctypes.byref(h))
        if st != PP_OK:
            raise PPError(st, status_string(st))
        self.h = h
        self.device = device
        self._follow = True
        self._bound = None

    def check(self, st: int) -> int:
        if st != PP_OK:
            raise PPError(st, f"{status_string(st)}: {lib.pp_ctx_last_error(self.h).decode()}")
        return st

    def synchronize(self):
        self.check(lib.pp_ctx_synchronize(self.h))

    def set_kernel_timing(self, on: bool):
        """Bracket each region product with CUDA events (measurement only)."""
        self.check(lib.pp_ctx_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_time(self):
        """(summed device ms, launches) of the bracketed region products since
        the last call; waits for them."""
        ms, n = ctypes.c_double(0), _U64(0)
        self.check(lib.pp_ctx_kernel_time(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, int(n.value)

    def set_stream(self, stream_ptr: int | None):
        """Pin the context to a CUDA stream (None: its own stream); stops
        following torch's current stream."""
        self._follow = False
        self._bound = None
        self.check(lib.pp_ctx_set_stream(self.h, _P(stream_ptr or 0)))

    def follow_torch(self):
        """Bind the context to torch's current stream on its device, if torch
        has initialised CUDA and no stream was pinned (torch's default stream
        is CUDA's legacy default stream, handle 1 in the C API)."""
        if not self._follow:
            return self
        torch = sys.modules.get("torch")
        if torch is None:
            return self
        try:
            if not torch.cuda.is_initialized():
                return self
            s = int(torch.cuda.current_stream(self.device).cuda_stream) or 1
        except Exception:
            return self
        if s != self._bound:
            self.check(lib.pp_ctx_set_stream(self.h, _P(s)))
            self._bound = s
        return self

    def set_gf16_kernel(self, kernel: int):
        """PP_GF16_KERNEL_AUTO / _LUT / _TENSOR"""
        self.check(lib.pp_ctx_set_gf16_kernel(self.h, kernel))

    def set_gf64_kernel(self, kernel: int):
        """PP_GF16_KERNEL_AUTO / _LUT / _TENSOR for the GF(2^64) region kernel"""
        self.check(lib.pp_ctx_set_gf64_kernel(self.h, kernel))

    def free_cache(self):
        self.check(lib.pp_ctx_free_cache(self.h))

    def close(self):
        if self.h:
            lib.pp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_ctx_lock = threading.Lock()
_ctxs: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    with _ctx_lock:
        c = _ctxs.get(device)
        if c is None:
            c = Context(device)
            _ctxs[device] = c
        return c


def launch_count() -> int:
    return int(lib.pp_launch_count())


def ptr(buf) -> int:
    """Address of a numpy array or torch tensor (host or device)."""
    if buf is None:
        return 0
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr())
    if hasattr(buf, "ctypes"):
        return int(buf.ctypes.data)
    if isinstance(buf, int):
        return buf
    raise TypeError(f"unsupported buffer type {type(buf)}")
