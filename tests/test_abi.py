"""The C ABI library builds for sm_100a and exports every entry point include/tdi.h declares.
No compute call is made (this runs without a GPU)."""
import ctypes
import importlib
import os


def test_library_builds_and_exports_every_declared_symbol(tdi):
    build = importlib.import_module("3di_b200.build")
    path = build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    declared = tdi.header_symbols()
    assert len(declared) >= 13
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) == set(tdi.SIGNATURES)


def test_python_front_end_binds_the_library(tdi):
    lib = tdi.load_library()
    assert lib.tdi_last_error() is not None


def test_argument_errors_come_back_as_status_codes(tdi):
    """Entry points reject bad arguments before touching the device, with a message."""
    import numpy as np
    lib = tdi.load_library()
    z = np.zeros(51, np.float32)
    st = lib.tdi_orthographic_init(0, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, None, None, None)
    assert st == 1                                  # TDI_ERR_INVALID
    assert b"orthographic" in lib.tdi_last_error()
    st = lib.tdi_orthographic_init(1, None, z.ctypes.data, z.ctypes.data, z.ctypes.data, None, None, None)
    assert st != 0
