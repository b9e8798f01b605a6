"""The DDC adapter header (include/ddc_b200/spline_builder_b200.hpp): ddc::SplineBuilder with
SplineSolver::B200 and ddc_b200::SplineEvaluator, compiled against a minimal stand-in for DDC's
public surface (tests/native/ddc_mock) and run on ChunkSpans in the characteristics-advection shape
(tests/native/adapter_check.cpp): coefficients and values equal direct ddcb_build / ddcb_eval calls
bit for bit. The compile runs everywhere; the run needs a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ddc_b200", "libddcb.so")


def _compile(out):
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
           f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(ROOT, 'tests', 'native', 'ddc_mock')}",
           "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "native", "adapter_check.cpp"),
           f"-L{os.path.dirname(LIB)}", "-lddcb", "-L/usr/local/cuda/lib64", "-lcudart",
           f"-Wl,-rpath,{os.path.dirname(LIB)}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(LIB), reason="needs g++ and libddcb.so")
def test_adapter_compiles(tmp_path):
    _compile(str(tmp_path / "adapter_check"))


@pytest.mark.gpu
def test_adapter_matches_c_abi(tmp_path):
    exe = str(tmp_path / "adapter_check")
    _compile(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "ALL EQUAL" in r.stdout
