"""The C++ drop-in (include/skm_gpu_evaluator.hpp) with the reference's own boundary types.

CPU: the header compiles against the reference's headers for 2-D/3-D and double/float
ScalarType (the four builds the reference supports).  GPU: the ITK-free finite-difference
program (tests/cpp/shim_fd_test.cpp, built by tests/cpp/Makefile) runs the way
test/itkFiniteDifferenceTest.cpp drives the evaluator and must pass.
"""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle import REFERENCE as REF
BUILD = os.path.join(ROOT, "tests", "_build")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include", "cuda")) or shutil.which("g++") is None,
                    reason="reference checkout or g++ not available")
@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("single", [0, 1])
def test_shim_compiles_against_reference_headers(D, single):
    with tempfile.TemporaryDirectory() as tmp:
        cmd = ["g++", "-std=c++14", "-fsyntax-only", "-include", "cmath", "-include", "iostream",
               "-DSinglePrecisionType=%d" % single, "-DSpaceDimensions=%d" % D, "-DUSE_WENDLAND_C0=1",
               "-I" + os.path.join(REF, "include", "cuda"), "-I" + os.path.join(REF, "include"),
               "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
               os.path.join(ROOT, "tests", "cpp", "shim_fd_test.cpp")]
        r = subprocess.run(cmd, capture_output=True, text=True, cwd=tmp)
        assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.gpu
@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("metric", [0, 1])
def test_shim_finite_differences(D, metric):
    exe = os.path.join(BUILD, "shim_fd_test_d%d" % D)
    if not os.path.exists(exe):
        pytest.skip("tests/_build not built (needs the reference checkout at build time)")
    r = subprocess.run([exe, str(metric), "11"], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
