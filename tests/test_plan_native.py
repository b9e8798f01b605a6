"""Host-side check of the device solve's algorithm (no GPU): tests/native/plan_check.cpp builds
plans for degrees 1-5, uniform and non-uniform meshes, every closure pair and several sizes and
chunkings, then replays on the host exactly the steps the kernels run -- chunked banded sweeps,
the log-depth carry scan over precomputed transfer-matrix products and the periodic border
correction -- with the tables the kernels receive, for A and A^T, and compares each result with
the direct banded solve (<= 1e-12 relative)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_device_solve_emulation(tmp_path):
    exe = str(tmp_path / "plan_check")
    cuda_inc = "/usr/local/cuda/include"
    cmd = ["g++", "-std=c++17", "-O1", f"-I{cuda_inc}", "-x", "c++",
           os.path.join(ROOT, "ddc_b200", "csrc", "plan.cpp"), os.path.join(ROOT, "tests", "native", "plan_check.cpp"),
           "-x", "none", "-L/usr/local/cuda/lib64", "-lcudart", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "0 failures" in r.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_plan_matrix_equals_reference_matrix(tmp_path, oracle_mod):
    """tests/native/matrix_check.cpp: the plan's assembled system equals the oracle's restatement of
    the reference's matrix (including the symmetric storage of uniform centre blocks) entry by
    entry, for degrees 1-5, uniform and non-uniform, every closure pair and sizes 7..429."""
    exe = str(tmp_path / "matrix_check")
    obuild = os.path.join(ROOT, "oracle", "_build")
    cmd = ["g++", "-std=c++17", "-O1", "-Wno-subobject-linkage", "-I/usr/local/cuda/include", "-x", "c++",
           os.path.join(ROOT, "tests", "native", "matrix_check.cpp"), "-x", "none", f"-L{obuild}", "-loracle",
           f"-Wl,-rpath,{obuild}", "-L/usr/local/cuda/lib64", "-lcudart", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "0 failures" in r.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_plan_under_sanitizers(tmp_path):
    """The plan code compiled with AddressSanitizer and UndefinedBehaviorSanitizer: the device-solve
    emulation of every plan_check case, and a sweep of tiny grids (1-15 cells, every degree, closure
    and mesh kind) that must plan or be refused without touching memory outside its arrays."""
    cuda_inc = "/usr/local/cuda/include"
    flags = ["-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
             f"-I{cuda_inc}"]
    for name in ("plan_check", "small_grids_check"):
        exe = str(tmp_path / name)
        cmd = ["g++", *flags, "-x", "c++", os.path.join(ROOT, "ddc_b200", "csrc", "plan.cpp"),
               os.path.join(ROOT, "tests", "native", name + ".cpp"), "-x", "none", "-L/usr/local/cuda/lib64", "-lcudart",
               "-o", exe]
        subprocess.run(cmd, check=True, capture_output=True)
        env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0")
        r = subprocess.run([exe], capture_output=True, text=True, timeout=900, env=env)
        assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-3000:])
