"""The mixed form's Newton reciprocal against CUDA's division.

The mixed form's FP64 p* solve and cell C2P multiply by reciprocals,
computed by Newton's method on f(y) = 1/y - d from the
hardware's approximate reciprocal (``nr_rcp`` in
hlld_ai_b200/csrc/srmhd_phys.cuh).  ``tests/host/nr_rcp_check.cu`` runs it
on a million doubles of both signs with exponents over [1e-300, 1e300] and
compares each result with the correctly rounded 1.0 / d of the same device:
every one finite and at most 2 ulp away, the two ends of its documented
domain (2^-1000 <= |d| < 2^1000) included, and a NaN gives a NaN.  Outside
the domain (inf, subnormals, |d| >= 2^1022) the seed flushes to zero; the
callers never pass such values (see the comment at nr_rcp).

The Newton square root (``nr_sqrt``: the approximate reciprocal square root
refined by Newton's method, then one Newton step on s^2 - x) is checked the
same way by ``tests/host/nr_sqrt_check.cu`` against CUDA's correctly rounded
sqrt on positive doubles over [1e-300, 1e300] and its domain ends: at most
2 ulp, 0 gives 0 and a NaN a NaN.
"""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run_check(tmp_path, name):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("needs nvcc to build the device check")
    exe = str(tmp_path / name)
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "hlld_ai_b200", "csrc"),
           os.path.join(ROOT, "tests", "host", name + ".cu"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe, "2"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.stdout, r.stderr)
    assert r.stdout.startswith("max_ulp ")
    assert "nan_ok=1" in r.stdout
    return r.stdout


def test_newton_reciprocal_within_two_ulp_of_division(tmp_path):
    _run_check(tmp_path, "nr_rcp_check")


def test_newton_sqrt_within_two_ulp_of_sqrt(tmp_path):
    out = _run_check(tmp_path, "nr_sqrt_check")
    assert "zero_ok=1" in out
