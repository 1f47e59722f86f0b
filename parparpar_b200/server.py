"""Serving loop (pp_server_* in include/parpar_b200.h): continuous batching of
create / repair jobs under a device-memory budget, with p50/p99 latency.

No counterpart in the reference.  Jobs are made with the helpers of
parparpar_b200.batch (par2_create_job, par3_create_job, par3_repair_job,
gf16_muladd_job) and may use host buffers (pinned, for copies that overlap)
or CUDA tensors; every job's result is identical to running it alone.
"""
from __future__ import annotations

import ctypes

from ._lib import PP_OK, PPError, PPJob, PPServerStats, lib


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 120 * 10**9, max_jobs_per_wave: int = 24,
                 lanes: int = 2):
        h = ctypes.c_void_p()
        st = lib.pp_server_create(device, hbm_budget_bytes, max_jobs_per_wave, lanes, ctypes.byref(h))
        if st != PP_OK:
            raise PPError(st, "pp_server_create failed")
        self.h = h
        self._keep = {}

    def submit(self, job) -> int:
        """Queue a job (a tuple from the batch helpers); returns its ticket.
        The job's buffers are kept referenced until wait() returns."""
        j, keep = job
        cuda = [b for b in (keep if isinstance(keep, (list, tuple)) else [keep]) if getattr(b, "is_cuda", False)]
        if cuda:
            # the server copies and reads device buffers on its own lanes: the
            # producer of a CUDA tensor (torch's current stream) finishes first
            import torch
            torch.cuda.current_stream(cuda[0].device).synchronize()
        t = ctypes.c_uint64()
        st = lib.pp_server_submit(self.h, ctypes.byref(j), ctypes.byref(t))
        if st != PP_OK:
            raise PPError(st, (lib.pp_server_last_error(self.h) or b"").decode())
        self._keep[t.value] = keep
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> int:
        """The job's status: PP_OK, or the error code it failed with."""
        st = lib.pp_server_wait(self.h, ticket, timeout_ms)
        self._keep.pop(ticket, None)
        return st

    def stats(self) -> dict:
        s = PPServerStats()
        lib.pp_server_get_stats(self.h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in PPServerStats._fields_}

    def reset_stats(self):
        lib.pp_server_reset_stats(self.h)

    def close(self):
        if self.h:
            lib.pp_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
