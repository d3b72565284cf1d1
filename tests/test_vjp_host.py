"""The hand-written reverse modes of the adjoint against forward-mode dual
numbers, on the host.

The device physics headers compile as plain C++ with a host compiler.
``tests/host/face_vjp_check.cpp`` contracts random flux adjoints with the
dual Jacobian of the HLLE / HLLD face solvers (HLLD at its solved p* through
the implicit-function theorem) and with their reverse mode, over random
face states including B_n = 0, HLLD -> HLLE fallbacks and degenerate
contacts; ``tests/host/c2p_vjp_check.cpp`` does the same for the Kastaun
C2P at its solved root (S-rescale, atmosphere and B = 0 cases included).
No GPU is needed.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


def _build(tmp_path_factory, name):
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path_factory.mktemp("vjp") / name)
    cmd = [gxx, "-O1", "-std=c++17", "-x", "c++", "-I", CUDA_INC,
           "-I", os.path.join(ROOT, "hlld_ai_b200", "csrc"),
           os.path.join(HERE, "host", name + ".cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    return _build(tmp_path_factory, "face_vjp_check")


@pytest.fixture(scope="module")
def c2p_checker(tmp_path_factory):
    return _build(tmp_path_factory, "c2p_vjp_check")


@pytest.mark.parametrize("seed", [11, 2])
def test_face_vjp_matches_dual_jacobian(checker, seed):
    r = subprocess.run([checker, "1e-10", "6000", str(seed)], capture_output=True, text=True)
    out = r.stdout.strip()
    assert r.returncode == 0, out
    worst = [float(x) for x in out.split()[1:4]]
    assert max(worst) <= 1e-10, out
    nfail = int(out.split("failed=")[1].split()[0])
    assert 0 < nfail < 6000, out  # both the HLLD path and its fallback were exercised


@pytest.mark.parametrize("seed", [3, 4])
def test_c2p_vjp_matches_dual_jacobian(c2p_checker, seed):
    r = subprocess.run([c2p_checker, "1e-9", "6000", str(seed)], capture_output=True, text=True)
    out = r.stdout.strip().splitlines()[-1]
    assert r.returncode == 0, r.stdout[-2000:]
    assert float(out.split()[1]) <= 1e-9, out
    nres = int(out.split("rescaled=")[1].split()[0])
    natmo = int(out.split("atmo=")[1].split()[0])
    assert nres > 0 and natmo > 0, out  # the S-rescale and atmosphere branches ran
