"""Host-side parts of the reference's C++ interface, on the CPU
(tests/cpp/host_check.cpp): options from a config file and the command line
(src/options.cpp:44-115) with their derived values (:88-95), the cosmology
functions (src/cosmology.cpp) against an independent integration of the
Friedmann equation and, where oracle/_ref was built, against the reference's
own cosmology.cpp compiled from its source, and the raw SoA particle files.
"""
import json
import os
import subprocess

import numpy as np
import pytest
from scipy.integrate import quad, solve_ivp

from ct2_b200 import _lib, ics
from oracle import ref_particle as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H0 = 1e7 / 3.086e24

CONFIG = """# a config file in the reference's key = value form
hsoft = 0.01
bwidth = 2.5
Ngrid = 16
omega_m = 0.3
eta = 0.2   # overridden on the command line
mesh = 32
"""


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    d = tmp_path_factory.mktemp("host")
    exe = d / "host_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "host_check.cpp"),
                    "-L" + os.path.dirname(_lib.LIB_PATH), "-lct2g",
                    "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH), "-o", str(exe)], check=True)
    cfg = d / "run.cfg"
    cfg.write_text(CONFIG)
    soa = d / "p.soa"
    r = subprocess.run([str(exe), str(cfg), str(soa), "--eta", "0.25", "--order=3"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    return dict(json.loads(line), exe=str(exe), dir=d, soa=str(soa))


def test_config_file_and_command_line(host):
    h = host
    assert h["ok"]
    assert abs(h["hsoft"] - 0.01) < 1e-9 and abs(h["bwidth"] - 2.5) < 1e-9
    assert h["Ngrid"] == 16 and h["mesh"] == 32 and abs(h["omega_m"] - 0.3) < 1e-7
    # the command line wins over the file (program_options' first store)
    assert abs(h["eta"] - 0.25) < 1e-7 and h["order"] == 3
    # untouched keys keep the reference defaults (src/options.cpp:50-62)
    assert h["ppcell"] == 256 and abs(h["hubble"] - 0.7) < 1e-7
    # derived values (src/options.cpp:88-95)
    assert h["nparts"] == 16 ** 3 and abs(h["GM"] - 1.0 / 16 ** 3) < 1e-12
    assert np.isfinite(h["code_to_cm"]) and np.isfinite(h["code_to_s"])
    assert abs(h["code_to_s"] - h["code_to_cm"] / 2.99792458e10) <= 1e-6 * h["code_to_s"]
    assert abs(h["omega_lam"] - (1.0 - h["omega_r"] - h["omega_m"])) < 1e-6
    assert 1e-5 < h["omega_r"] < 1e-4


def test_missing_config_file_is_refused(host):
    r = subprocess.run([host["exe"], str(host["dir"] / "absent.cfg"), host["soa"]],
                       capture_output=True, text=True, timeout=60)
    assert '"ok": false' in r.stdout and "not found" in r.stdout


def _friedmann(h):
    H = H0 * np.float32(h["code_to_s"]) * np.float32(h["hubble"])
    om, orr, ol = (float(np.float32(h[k])) for k in ("omega_m", "omega_r", "omega_lam"))

    def dadt(a):
        return H * a * np.sqrt(orr / a ** 4 + om / a ** 3 + ol)

    def accel(a):
        return a * H * H * (-orr / a ** 4 - 0.5 * om / a ** 3 + ol)
    return dadt, accel


def test_cosmology_against_friedmann_integration(host):
    h = host
    dadt, accel = _friedmann(h)
    for a, v in zip((0.02, 0.1, 0.5, 1.0), h["dadt"]):
        assert abs(v - dadt(a)) <= 1e-6 * dadt(a)
    t = quad(lambda a: 1.0 / dadt(a), 0.1, 0.5, epsabs=0, epsrel=1e-11)[0]
    assert abs(h["time"] - t) <= 1e-6 * t
    tau = quad(lambda a: 1.0 / (a * dadt(a)), 0.1, 0.5, epsabs=0, epsrel=1e-11)[0]
    assert abs(h["conformal_time"] - tau) <= 1e-6 * tau
    # cosmos_update: (a, adot)' = (adot a, accel(a) a), 128 RK3 substeps
    u = h["update"]
    sol = solve_ivp(lambda s, y: [y[1] * y[0], accel(y[0]) * y[0]], (0.0, u["dt"]),
                    [0.1, dadt(0.1)], rtol=1e-12, atol=1e-15, method="DOP853")
    assert abs(u["a"] - sol.y[0, -1]) <= 1e-8 * sol.y[0, -1]
    assert abs(u["adot"] - sol.y[1, -1]) <= 1e-7 * abs(sol.y[1, -1])
    assert u["a"] > 0.1


@pytest.mark.skipif(R.lib() is None, reason="oracle/_ref not built here")
def test_cosmology_matches_reference_source(host):
    """The reference's cosmology.cpp, compiled from its source, with the same
    option values (the finite ones: the reference's own derivation overflows
    code_to_g and makes code_to_s infinite, divergence D16)."""
    h = host
    L = R.cosmology(h["omega_m"], h["omega_r"], h["omega_lam"], h["hubble"], h["code_to_s"])
    for a, v in zip((0.02, 0.1, 0.5, 1.0), h["dadt"]):
        assert abs(v - L.ref_cosmos_dadt(a)) <= 1e-13 * v
    assert abs(h["time"] - L.ref_cosmos_time(0.1, 0.5)) <= 1e-10 * h["time"]
    tr = L.ref_cosmos_conformal_time(0.1, 0.5)
    assert abs(h["conformal_time"] - tr) <= 1e-8 * tr
    import ctypes
    a, adot, add = ctypes.c_double(0.1), ctypes.c_double(h["dadt"][1]), ctypes.c_double(0.0)
    L.ref_cosmos_update(ctypes.byref(add), ctypes.byref(adot), ctypes.byref(a), h["update"]["dt"])
    u = h["update"]
    assert abs(u["a"] - a.value) <= 1e-13 * a.value
    assert abs(u["adot"] - adot.value) <= 1e-12 * abs(adot.value)
    assert abs(u["adotdot"] - add.value) <= 1e-12 * abs(add.value)


def test_soa_file_round_trip(host, tmp_path):
    h = host
    assert h["soa_round_trip"]
    # the C++ layer's file reads back in Python, and Python's in C++ terms
    d = ics.load_soa(h["soa"])
    assert len(d["x"]) == 1000
    i = np.arange(1000, dtype=np.uint64)
    assert np.array_equal(d["x"], (np.uint64(2654435761) * i % 2 ** 32).astype(np.uint32))
    assert np.array_equal(d["rung"], (i % 5).astype(np.int8))
    p = tmp_path / "q.soa"
    ics.save_soa(str(p), d)
    assert open(str(p), "rb").read() == open(h["soa"], "rb").read()
    with pytest.raises(ValueError):
        (tmp_path / "bad").write_bytes(b"notasoafile" * 3)
        ics.load_soa(str(tmp_path / "bad"))
