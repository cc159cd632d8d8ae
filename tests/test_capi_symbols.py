"""CPU: libifdda_gpu.so loads and exports every entry point declared in
include/ifdda_gpu.h (no CUDA call is made)."""
import ctypes
import os
import re
import subprocess

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


def _nm(*flags):
    import ifdda._capi as capi
    out = subprocess.run(["nm", "-D", *flags, capi.LIB_PATH], check=True, capture_output=True, text=True).stdout
    return [ln.split()[-1] for ln in out.splitlines() if ln.strip()]


def test_product_does_not_link_the_oracle():
    """The product library neither defines nor needs an oracle symbol, and
    does not load the oracle's shared library."""
    import ifdda._capi as capi
    defined, undefined = _nm("--defined-only"), _nm("--undefined-only")
    assert not [s for s in defined + undefined if s.startswith("orc_")]
    deps = subprocess.run(["ldd", capi.LIB_PATH], check=True, capture_output=True, text=True).stdout
    assert "oracle" not in deps
    # the exported C entry points are exactly the header's
    exported = {s for s in defined if s.startswith("ifdda_")}
    assert exported == set(declared_functions())


C_PROGRAM = r"""
#include <stdio.h>
#include "ifdda_gpu.h"
int main(void) {
    ifdda_dcmplx z = {1.0, -2.0};
    ifdda_solve_options opt = {IFDDA_MIXED, 0, 0, 0.0, 0};
    int v = ifdda_abi_version();
    printf("%d %d %g\n", v, opt.precision, z.im);
    return v == IFDDA_GPU_ABI_VERSION ? 0 : 1;
}
"""


def test_header_is_c99_and_links(tmp_path):
    """include/ifdda_gpu.h compiles as strict C99 and a C program links
    against libifdda_gpu.so and calls an entry point that needs no GPU."""
    import ifdda._capi as capi
    src = tmp_path / "abi.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "abi"
    libdir = os.path.dirname(capi.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", libdir, "-lifdda_gpu", f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out == ["1", "1", "-2"]
