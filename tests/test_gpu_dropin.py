"""The reference's C++ interface end to end on the GPU (tests/cpp/drop_in.cpp)."""
import os
import subprocess

import pytest

from ct2_b200 import _lib

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_cxx_interface_runs(gpu, tmp_path):
    exe = tmp_path / "drop_in"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "drop_in.cpp"),
                    "-L" + os.path.dirname(_lib.LIB_PATH), "-lct2g",
                    "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "--Ngrid", "16", "--mesh", "32", "--order", "3", "--bwidth",
                        "2", "--hsoft", str(1.0 / 800)], capture_output=True, text=True,
                       timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
