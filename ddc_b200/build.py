"""Build the CUDA library libddcb.so in-tree for sm_100a (B200), and its bounds-checked variant
libddcb_check.so (the same sources with -DDDCB_CHECK_BOUNDS: every computed array index checked
on the device, reported by ddcb_last_device_error).

    python -m ddc_b200.build [--check-bounds]        (or ddc_b200.build.build())
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libddcb.so")
LIB_CHECK = os.path.join(HERE, "libddcb_check.so")
SOURCES = ["api.cu", "plan.cpp", "build_kernels.cu", "eval_kernels.cu", "fused_kernels.cu", "tensor2d.cu",
           "adjoint_kernels.cu", "refine_kernels.cu",
           "uneven_batch.cu", "host_pipeline.cu", "quadrature.cu", "tensornd.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "ddcb.h")]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(verbose: bool = False, force: bool = False, check_bounds: bool = False) -> str:
    """Compile every source to an object in parallel, then link libddcb.so (libddcb_check.so with
    check_bounds)."""
    lib = LIB_CHECK if check_bounds else LIB
    if not force and not needs_build(lib):
        return lib
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(HERE, "_build_check" if check_bounds else "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-ccbin", "g++",
              "--expt-relaxed-constexpr"]
    if check_bounds:
        common.append("-DDDCB_CHECK_BOUNDS")
    if verbose:
        common.append("-Xptxas=-v")

    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "ddcb.h"))
    newest_header = max(os.path.getmtime(h) for h in headers if os.path.exists(h))

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        # an object newer than its source and every header is up to date
        if not force and os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(src), newest_header):
            return src, obj, subprocess.CompletedProcess([], 0, "", "")
        cmd = [*common, "-c", "-o", obj, src]
        if src.endswith(".cpp"):
            cmd = [*common, "-x", "cu", "-c", "-o", obj, src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, sources()))
    for src, obj, r in results:
        if verbose or r.returncode:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, src)
    link = [nvcc(), *ARCH, "-shared", "-o", lib, *[o for _, o, _ in results]]
    subprocess.run(link, check=True)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True, check_bounds="--check-bounds" in sys.argv))
