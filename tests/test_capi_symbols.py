"""CPU: libifdda_gpu.so loads and exports every entry point declared in
include/ifdda_gpu.h (no CUDA call is made)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ifdda_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ifdda_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("ifdda_green_create", "ifdda_matvec", "ifdda_inverserig", "ifdda_inverserig_batch",
                 "ifdda_local_macro", "ifdda_cross_sections"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import ifdda._capi as capi
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding knows every exported entry point too
    assert set(declared_functions()) <= set(capi.SIGNATURES)


def test_abi_version_without_gpu():
    import ifdda._capi as capi
    assert capi.load().ifdda_abi_version() == 1


def test_product_does_not_link_the_oracle():
    import ifdda._capi as capi
    data = open(capi.LIB_PATH, "rb").read()
    assert b"orc_" not in data and b"libifdda_oracle" not in data
