"""include/ddcb.hpp (the C++ classes over the C-ABI) compiles warning-free, links against
libddcb.so and maps library errors to std::runtime_error (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ddc_b200", "libddcb.so")


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(LIB), reason="needs g++ and the built library")
def test_cpp_header_compiles_and_reports_errors(tmp_path):
    exe = str(tmp_path / "hpp_check")
    cmd = ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-O1", os.path.join(ROOT, "tests", "native", "hpp_check.cpp"),
           "-L" + os.path.dirname(LIB), "-lddcb", "-Wl,-rpath," + os.path.dirname(LIB), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("OK") == 2, r.stdout
