"""CPU checks of the C-ABI library: it loads, exports every declared symbol, and its host-side
plan functions (bases, Greville points, integrals, grid validation) agree with the oracle.
No kernel is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "ddcb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ddcb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ddc_b200

    L = ddc_b200.load_library()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_bounds_checked_build_exports_the_same_symbols():
    """libddcb_check.so (the DDCB_CHECK_BOUNDS build) exports every declared symbol and says it is
    the checked build; the default library says it is not."""
    import ddc_b200

    path = os.path.join(ROOT, "ddc_b200", "libddcb_check.so")
    if not os.path.exists(path):
        pytest.skip("libddcb_check.so not built")
    L = C.CDLL(path)
    for n in declared_functions():
        assert hasattr(L, n), n
    L.ddcb_bounds_checked.restype = C.c_int32
    assert L.ddcb_bounds_checked() == 1
    assert ddc_b200.bounds_checked() is False


def test_bounds_site_tags_are_distinct(tmp_path):
    """The file tags that name the site of a recorded out-of-range index are distinct for every
    device source and header (check_bounds.cuh's 16-bit hash of the base name)."""
    import shutil
    import subprocess

    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    files = sorted(f for f in os.listdir(os.path.join(ROOT, "ddc_b200", "csrc")) if f.endswith((".cu", ".cuh")))
    src = tmp_path / "tags.cpp"
    src.write_text('#include <cstdio>\n#include "check_bounds.cuh"\nint main(){\n'
                   + "".join(f'std::printf("%u\\n", ddcb::bounds_file_tag("dir/{f}"));\n' for f in files) + "}\n")
    exe = str(tmp_path / "tags")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "ddc_b200", "csrc"), str(src), "-o", exe], check=True)
    tags = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert len(tags) == len(files) and len(set(tags)) == len(tags)


def test_status_strings():
    import ddc_b200

    L = ddc_b200.load_library()
    L.ddcb_status_string.restype = C.c_char_p
    assert L.ddcb_status_string(0) == b"success"
    assert L.ddcb_status_string(2) == b"invalid interpolation grid"


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("bcs", [(0, 0), (1, 1), (3, 3), (1, 3), (3, 1), (2, 2)])
def test_host_basis_matches_oracle(oracle_mod, degree, uniform, bcs):
    import ddc_b200 as D

    O = oracle_mod
    lo, hi = bcs
    periodic = lo == 0
    br = np.linspace(0.0, 2.0, 24)
    if not uniform:
        br[1:-1] += np.random.default_rng(degree).uniform(-0.02, 0.02, 22)
    if uniform:
        b = D.UniformBSplines(degree, periodic, 0.0, 2.0, 23)
        o = O.BSplines(degree, periodic, rmin=0.0, rmax=2.0, ncells=23)
    else:
        b = D.NonUniformBSplines(degree, periodic, br)
        o = O.BSplines(degree, periodic, breaks=br)
    assert (b.nbasis, b.size, b.ncells) == (o.nbasis, o.size, o.ncells)
    assert b.rmin == o.rmin and b.rmax == o.rmax
    np.testing.assert_array_equal(b.knots(), [o.knot(k) for k in range(b.ncells + 1 + 2 * degree)])
    np.testing.assert_array_equal(D.greville_points(b, lo, hi), o.greville(lo, hi))
    np.testing.assert_allclose(b.integrals(), o.integrals(), rtol=1e-15, atol=1e-17)


def test_bad_grid_is_reported():
    import ddc_b200 as D
    from ddc_b200 import _lib

    b = D.UniformBSplines(3, False, 0.0, 1.0, 10)
    pts = D.greville_points(b, 3, 3)
    with pytest.raises(_lib.DdcbError, match="Incorrect number of points"):
        D.SplineBuilder(b, pts[:-1], 3, 3)
    bad = pts.copy()
    bad[1:6] = np.linspace(0.01, 0.05, 5)
    with pytest.raises(_lib.DdcbError, match="overconstrained"):
        D.SplineBuilder(b, np.sort(bad), 3, 3)


def test_invalid_arguments():
    import ddc_b200 as D
    from ddc_b200 import _lib

    with pytest.raises(_lib.DdcbError):
        D.UniformBSplines(3, False, 1.0, 0.0, 10)
    with pytest.raises(_lib.DdcbError):
        D.NonUniformBSplines(3, False, [0.0, 0.5, 0.4, 1.0])
    with pytest.raises(_lib.DdcbError):
        D.UniformBSplines(9, False, 0.0, 1.0, 10)
