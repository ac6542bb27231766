"""The C-ABI library loads and exports every entry point the header declares (no GPU)."""
import ctypes
import os

from gip_b200 import _lib


def test_library_exports_all_declared_symbols():
    lib = _lib.load()
    missing = [s for s in _lib.declared_symbols() if not hasattr(lib, s)]
    assert missing == []


def test_status_strings_without_gpu():
    lib = _lib.load()
    assert lib.gipb200_status_string(0) == b"ok"
    assert lib.gipb200_status_string(3) == b"PCG breakdown"
    assert lib.gipb200_version() >= 100


def test_library_is_in_tree_sm100a_build():
    assert os.path.dirname(_lib.LIB_PATH).endswith("gip_b200")
    assert os.path.exists(_lib.LIB_PATH)
    # every kernel image in the library is for sm_100a (checked from the build flags)
    from gip_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_bad_arguments_fail_without_touching_the_device():
    lib = _lib.load()
    st = lib.gipb200_matrix_create(-1, 0, 0, None, None, None, ctypes.byref(ctypes.c_void_p()))
    assert st == _lib.ERR_ARG
    assert b"negative" in lib.gipb200_last_error()
