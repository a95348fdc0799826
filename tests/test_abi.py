"""CPU checks of the boundary: the library loads, exports every entry point the
public headers declare, and fails cleanly (no crash, a status) without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

from ct2_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def _declared_c_symbols():
    src = open(os.path.join(INC, "ct2g.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ct2g_[a-z0-9_]+)\s*\(", src)))


def _exported():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


def test_library_exports_every_c_entry_point():
    lib = _lib.load()
    declared = _declared_c_symbols()
    assert len(declared) >= 39
    exported = _exported()
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    # and the ctypes table binds exactly the declared set
    assert sorted(n for n, _, _ in _lib.SYMBOLS) == declared
    for s in declared:
        assert hasattr(lib, s)


def test_library_exports_reference_cxx_interface():
    src = open(os.path.join(INC, "ct2_cosmictiger.hpp")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = set(re.findall(r"^\s*[\w:&<>, *]+?\b(\w+)\(", src, flags=re.M))
    names -= {"ct2_error", "real", "imag"}  # constructor, inline accessors of ct2::complex
    out = subprocess.run(["nm", "-DC", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for n in sorted(names):
        assert re.search(r"\b%s\(" % re.escape(n), out), n


def test_default_options_are_the_reference_defaults():
    lib = _lib.load()
    o = _lib.Options()
    lib.ct2g_default_options(ctypes.byref(o))
    # src/options.cpp:53-58
    assert abs(o.bwidth - 3.0) < 1e-7 and abs(o.hsoft - 1.0 / 50.0) < 1e-7
    assert abs(o.eta - 0.15) < 1e-7
    assert o.order >= 1 and o.mesh >= 8


def test_create_rejects_bad_options_and_reports_status():
    lib = _lib.load()
    o = _lib.Options()
    lib.ct2g_default_options(ctypes.byref(o))
    h = ctypes.c_void_p()
    for field, bad in (("mesh", 48), ("order", 0), ("order", 99), ("bwidth", 40.0),
                       ("hsoft", 0.0), ("kernel", 7)):
        o2 = _lib.Options()
        ctypes.memmove(ctypes.byref(o2), ctypes.byref(o), ctypes.sizeof(o))
        setattr(o2, field, bad)
        assert lib.ct2g_create(ctypes.byref(o2), ctypes.byref(h)) == 1, field  # CT2G_EINVAL
    assert lib.ct2g_status_string(6).decode() == "no usable sm_100 device"


def test_create_without_gpu_returns_enodev():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    o = _lib.Options()
    lib.ct2g_default_options(ctypes.byref(o))
    h = ctypes.c_void_p()
    assert lib.ct2g_create(ctypes.byref(o), ctypes.byref(h)) == 6  # CT2G_ENODEV


def test_drop_in_program_compiles(tmp_path):
    exe = tmp_path / "drop_in"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + INC, os.path.join(ROOT, "tests", "cpp",
                    "drop_in.cpp"), "-L" + os.path.dirname(_lib.LIB_PATH), "-lct2g",
                    "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH), "-o", str(exe)], check=True)
    assert exe.exists()


def test_reference_fft_surface_signatures():
    """The C++ names of the reference's 1D FFT surface (fft.hpp:18-27) are
    exported with their argument types."""
    out = subprocess.run(["nm", "-DC", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for sig in ("fft_real(double*, int, int)", "fft_real(ct2::simd_f64*, int, int)",
                "fft_complex(ct2::complex<ct2::simd_f64>*, int, int)",
                "scramble(double*, int, int, int)", "transpose_yz(double*, int)",
                "transpose_r2c(double*, double*, int)", "transpose_c2r(double*, double*, int)",
                "cos_twiddles(int)", "sin_twiddles(int)", "inv_sin_twiddles(int)",
                "fft_r2c_3d(double*, double*, int)", "fft_c2r_3d(double*, double*, int)"):
        assert sig in out, sig
