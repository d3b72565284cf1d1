"""The hand-written reverse mode of the HLLE and HLLD face solvers against
forward-mode dual numbers, on the host.

The device physics headers compile as plain C++ with a host compiler;
``tests/host/face_vjp_check.cpp`` contracts random flux adjoints with the
dual Jacobian of the forward solver (HLLD at its solved p* through the
implicit-function theorem) and with the reverse mode, over random face
states including B_n = 0 and HLLD -> HLLE fallbacks.  No GPU is needed.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    tmp_path = tmp_path_factory.mktemp("vjp")
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path / "face_vjp_check")
    cmd = [gxx, "-O1", "-std=c++17", "-x", "c++", "-I", CUDA_INC,
           "-I", os.path.join(ROOT, "hlld_ai_b200", "csrc"),
           os.path.join(HERE, "host", "face_vjp_check.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


@pytest.mark.parametrize("seed", [11, 2])
def test_face_vjp_matches_dual_jacobian(checker, seed):
    r = subprocess.run([checker, "1e-10", "6000", str(seed)], capture_output=True, text=True)
    out = r.stdout.strip()
    assert r.returncode == 0, out
    worst = [float(x) for x in out.split()[1:4]]
    assert max(worst) <= 1e-10, out
    nfail = int(out.split("failed=")[1].split()[0])
    assert 0 < nfail < 6000, out  # both the HLLD path and its fallback were exercised
