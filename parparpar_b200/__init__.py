"""parparpar_b200 — B200-native (sm_100a) engine for the GF hot paths of ParParPar.

PAR2: GF(2^16) region multiply-accumulate and repair-matrix inversion, input
      slice MD5 + CRC32 and the staging memory checksum.
PAR3: GF(2^64) Cauchy-matrix recovery, solve/reconstruct, region primitives,
      additive FFT, BLAKE3 block checksums, recovery packets, streaming create.

All data-path arithmetic runs in hand-written CUDA kernels inside
``libparpar_b200.so`` (C ABI: include/parpar_b200.h).  Importing this package
raises ImportError if that library has not been built; there is no CPU
fallback.
"""
from ._lib import (PP_ERR_BUSY, PP_ERR_CUDA, PP_ERR_INVALID_ARG, PP_ERR_NO_DEVICE, PP_ERR_NO_MEMORY,
                   PP_ERR_NOT_INVERTIBLE, PP_ERR_SINGULAR, PP_ERR_TIMEOUT, PP_ERR_TOO_LARGE, PP_ERR_IO, PP_OK, PP_PROC_ADD_FULL, PP_PROC_ADD_OK,
                   PP_PROC_ADD_OK_BUSY, Context, PPError, default_context, launch_count)
from . import batch, par2, par3, server

__all__ = ["batch", "par2", "par3", "server", "Context", "PPError", "default_context", "launch_count", "PP_OK",
           "PP_ERR_INVALID_ARG", "PP_ERR_CUDA", "PP_ERR_NO_MEMORY", "PP_ERR_SINGULAR", "PP_ERR_NOT_INVERTIBLE",
           "PP_ERR_BUSY", "PP_ERR_NO_DEVICE", "PP_ERR_TIMEOUT", "PP_ERR_TOO_LARGE", "PP_ERR_IO", "PP_PROC_ADD_OK", "PP_PROC_ADD_OK_BUSY", "PP_PROC_ADD_FULL"]
