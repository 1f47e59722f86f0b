"""The C-ABI library loads and exports every symbol include/parpar_b200.h
declares; host-side logic that needs no GPU behaves like the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "parpar_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"PP_API\s+[\w\s\*]+?\b(pp_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import parparpar_b200._lib as L
    syms = declared_symbols()
    assert len(syms) >= 40
    for s in syms:
        assert hasattr(L.lib, s), s
    assert sorted(L.EXPORTS) == syms


def test_version_and_status_strings():
    import parparpar_b200._lib as L
    assert b"sm_100a" in L.lib.pp_version()
    assert L.status_string(L.PP_ERR_SINGULAR) == "singular matrix"


def test_scalar_coeff_matches_oracle(oracle):
    from parparpar_b200 import par2
    rng = np.random.default_rng(5)
    for i, e in zip(rng.integers(0, 32768, 300), rng.integers(0, 65535, 300)):
        assert par2.gfmat_coeff(int(i), int(e)) == oracle.par2_coeff(int(i), int(e))
    for i in (0, 1, 2, 100, 32767):
        assert par2.gfmat_input_log(i) == oracle.L.or_par2_input_log(i)


def test_no_device_is_a_loud_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import parparpar_b200 as pp
    with pytest.raises(pp.PPError) as ei:
        pp.Context(0)
    assert ei.value.status == pp.PP_ERR_NO_DEVICE


def test_compute_recovery_argument_errors():
    """gf64_addon compute_recovery argument checks (src/gf64_addon.cc:1266-1405):
    TypeError for wrong types, RangeError (ValueError) for bad sizes, raised
    before any device work."""
    from parparpar_b200 import par3
    buf = np.zeros(64, dtype=np.uint64)
    with pytest.raises(TypeError):
        par3.compute_recovery(None, buf, 1, 1, 8, 0, 1)
    with pytest.raises(TypeError):
        par3.compute_recovery(buf, buf, 1.5, 1, 8, 0, 1)
    with pytest.raises(TypeError):
        par3.compute_recovery(buf, buf, 1, 1, 8, "x", 1)
    with pytest.raises(TypeError):
        par3.compute_recovery(buf, buf, 1, 1, 8, 0, 1, 0, 1)
    with pytest.raises(ValueError):
        par3.compute_recovery(buf, buf, 0, 1, 8, 0, 1)
    with pytest.raises(ValueError):
        par3.compute_recovery(buf, buf, 1, 0, 8, 0, 1)
    with pytest.raises(ValueError):
        par3.compute_recovery(buf, buf, 1, 1, 12, 0, 1)
    with pytest.raises(ValueError):
        par3.compute_recovery(buf, buf, 100, 1, 8, 0, 1)
    with pytest.raises(ValueError):
        par3.compute_recovery(buf, buf, 1, 100, 8, 0, 1)


def test_null_context_is_rejected():
    import parparpar_b200._lib as L
    assert L.lib.pp_gf64_compute_recovery(None, None, 1, None, 1, 1, 0, 1, 0, 0) == L.PP_ERR_INVALID_ARG
    assert L.lib.pp_par2_create(None, None, 0, 0, 0, None, None, 0, None, 0) == L.PP_ERR_INVALID_ARG
    # processor input hashing: a null processor is rejected before any device work
    assert L.lib.pp_par2_proc_set_input_hashes(None, 4) == L.PP_ERR_INVALID_ARG
    assert L.lib.pp_par2_proc_get_input_hashes(None, None, 0) == L.PP_ERR_INVALID_ARG


def test_assemble_recovery_packets_argument_errors():
    """The N-API argument checks of assemble_recovery_packets
    (src/gf64_addon.cc:2813-2884) run before any device work."""
    from parparpar_b200 import par3
    rec = np.zeros(64, dtype=np.uint8)
    with pytest.raises(TypeError):
        par3.assemble_recovery_packets(None, b"12345678", 0, 1, 64)
    with pytest.raises(TypeError):
        par3.assemble_recovery_packets(rec, b"1234567", 0, 1, 64)
    with pytest.raises(TypeError):
        par3.assemble_recovery_packets(rec, b"12345678", 1.5, 1, 64)
    with pytest.raises(ValueError):
        par3.assemble_recovery_packets(rec, b"12345678", 0, 0, 64)
    with pytest.raises(ValueError):
        par3.assemble_recovery_packets(rec, b"12345678", 0, 1, 0)
    with pytest.raises(ValueError):
        par3.assemble_recovery_packets(rec, b"12345678", 0, 2, 64)
    with pytest.raises(ValueError):
        par3.assemble_recovery_packets(rec, b"12345678", 0, 1 << 21, 1 << 20)


def test_create_streaming_argument_errors():
    """par3_create_streaming's option checks (src/gf64_create_streaming.cc:
    365-430) run before any device work."""
    from parparpar_b200 import par3
    with pytest.raises(TypeError):
        par3.par3_create_streaming("x", None)
    with pytest.raises(TypeError):
        par3.par3_create_streaming("x", {"blockSize": 64})
    with pytest.raises(TypeError):
        par3.par3_create_streaming("x", {"recoverySlices": 1})
    with pytest.raises(ValueError):
        par3.par3_create_streaming("x", {"recoverySlices": 0, "blockSize": 64})
    with pytest.raises(ValueError):
        par3.par3_create_streaming("x", {"recoverySlices": 1, "blockSize": 60})
    with pytest.raises(TypeError):
        par3.par3_create_streaming("x", {"recoverySlices": 1, "blockSize": 64, "firstInput": 1.5})


def test_compute_recovery_native_edge_errors():
    """test/par3-native-edge.js error scenarios: numInputs 0, numRecovery 0,
    blockSize 7 and 0, a numInputs the inputs buffer cannot hold -- all raise
    before any device work."""
    from parparpar_b200 import par3
    x = np.zeros(8, dtype=np.uint64)
    out = np.zeros(8, dtype=np.uint64)
    for args in [(0, 1, 8), (1, 0, 8), (1, 1, 7), (1, 1, 0), (2**31 - 1, 1, 8)]:
        with pytest.raises((ValueError, TypeError)):
            par3.compute_recovery(x, out, args[0], args[1], args[2], 0, 1)
    assert par3.isAlignedBuffer(par3.allocAlignedBuffer(100)) and par3.get_last_decomposition_path() == 0
