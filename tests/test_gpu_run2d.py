"""The run_2d drop-in (hlld_ai_b200.run_2d) end to end, after the reference's
own run tests (tests/test_high_order_2d.py:102-126 restart is bitwise,
:196-215 a non-finite run exits non-zero) and its output formats
(scripts/run_2d.py:264-287, :321-334)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def run(*args, check=True):
    r = subprocess.run([sys.executable, "-m", "hlld_ai_b200.run_2d", *args], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError(r.stdout + r.stderr)
    return r


def test_restart_is_bitwise(tmp_path):
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    common = ["--problem", "rotor", "--n", "32", "--solver", "hlld", "--tend", "1.0",
              "--restart-every", "0", "--log-every", "1"]
    run(*common, "--out", a, "--max-steps", "4")
    run(*common, "--out", b, "--max-steps", "2")
    run(*common, "--out", b, "--max-steps", "2", "--restart", os.path.join(b, "restart.npz"))
    ra, rb = np.load(os.path.join(a, "restart.npz")), np.load(os.path.join(b, "restart.npz"))
    assert int(ra["step"]) == int(rb["step"]) == 4
    assert float(ra["t"]) == float(rb["t"])
    for k in ("cons_D", "cons_Sx", "cons_Sy", "cons_Sz", "cons_tau", "cons_Bz", "Bxf", "Byf"):
        assert np.array_equal(ra[k], rb[k]), k
    assert int(rb["gen"]) == 1


def test_output_files_carry_the_reference_keys(tmp_path):
    out = str(tmp_path / "o")
    run("--problem", "orszag_tang", "--n", "32", "--solver", "hlle", "--tend", "0.01",
        "--out", out, "--nsnap", "1", "--log-every", "1")
    snap = np.load(os.path.join(out, "snap_000.npz"))
    assert set(snap.files) == {"t", "x", "y", "rho", "p", "vx", "vy", "Bx", "By", "divB",
                               "limiter", "ng", "n", "solver"}
    assert snap["rho"].shape == (32, 32)
    assert os.path.exists(os.path.join(out, "snap_fin.npz"))
    hdr = open(os.path.join(out, "diag.csv")).readline().strip().split(",")
    assert hdr == ["step", "t", "dt", "divB_max", "divB_l2", "sym_err", "rho_max", "rho_min",
                   "p_min", "W_max", "hlle_frac_x", "hlle_frac_y", "mean_iters", "c2p_bad",
                   "n_exact_x", "n_verified_x"]
    rows = open(os.path.join(out, "diag.csv")).read().strip().splitlines()[1:]
    assert len(rows) >= 1 and float(rows[-1].split(",")[3]) < 1e-10  # div B
    meta = json.load(open(os.path.join(out, "run_meta.json")))
    for k in ("problem", "n", "solver", "limiter", "ng", "cfl", "tend", "steps", "s_per_step"):
        assert k in meta


def test_non_finite_run_exits_nonzero(tmp_path):
    r = run("--problem", "rotor", "--n", "32", "--cfl", "40", "--tend", "1.0",
            "--out", str(tmp_path / "x"), "--restart-every", "0", check=False)
    assert r.returncode != 0
    assert "run failed" in (r.stdout + r.stderr)
    assert not os.path.exists(str(tmp_path / "x" / "snap_fin.npz"))
