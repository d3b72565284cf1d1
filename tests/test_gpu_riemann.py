"""Per-face HLLE/HLLD/HLLC kernels (the flux_fn plugin) against the CPU oracle.

FP64-exact build: bitwise equal to the oracle.  FP64 (FMA) build: the
tolerances of the reference's direction-genericity test
(tests/test_idir.py:104-156): same-branch faces within 1e-13 relative, and
HLLE-fallback flips rare (below 1%: contraction moves last bits, and the
multi-root p* residual turns a last-bit change into a different branch on
about 0.5% of these random faces, as rotating the input does in the
reference).
"""
import numpy as np
import pytest
import torch

from helpers import bitwise_equal, max_rel, random_face_states, to_dev, to_np
from oracle import oracle

import hlld_ai_b200 as H
from hlld_ai_b200.physics import hlld as Hh

GAMMA = 5.0 / 3.0
EOS = H.hybrid_eos(K=0.0, gamma=GAMMA, gamma_th=GAMMA)
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def states():
    sL, sR = random_face_states(4000, GAMMA)
    return to_np(sL), to_np(sR)


@pytest.mark.parametrize("solver", ["hlle", "hlld", "hllc"])
@pytest.mark.parametrize("idir", [0, 1, 2])
def test_exact_build_is_bitwise_oracle(states, solver, idir):
    nL, nR = states
    F, U, ps, err, it, fl, _ = Hh.riemann(to_dev(nL), to_dev(nR), EOS, idir, solver, "fp64_exact")
    oF, oU, ops, oerr, oit, ofl = oracle.riemann(nL, nR, idir, solver, GAMMA)
    for k in oF:
        assert bitwise_equal(F[k].cpu().numpy(), oF[k]), (solver, idir, "F", k)
        assert bitwise_equal(U[k].cpu().numpy(), oU[k]), (solver, idir, "U", k)
    assert bitwise_equal(ps.cpu().numpy(), ops)
    if solver == "hlld":
        assert np.array_equal(err.cpu().numpy(), oerr)
        assert np.array_equal(it.cpu().numpy(), oit)
        assert np.array_equal(fl.cpu().numpy(), ofl)


@pytest.mark.parametrize("solver", ["hlle", "hlld"])
@pytest.mark.parametrize("idir", [0, 1, 2])
def test_fma_build_matches_oracle(states, solver, idir):
    nL, nR = states
    F, U, ps, *_ = Hh.riemann(to_dev(nL), to_dev(nR), EOS, idir, solver, "fp64")
    oF, oU, ops, *_ = oracle.riemann(nL, nR, idir, solver, GAMMA)
    gp = ps.cpu().numpy()
    flip = (gp < 0) ^ (ops < 0)
    keep = ~flip
    for k in oF:
        assert max_rel(oF[k][keep], F[k].cpu().numpy()[keep]) < 1e-13, (solver, idir, k)
        assert max_rel(oU[k][keep], U[k].cpu().numpy()[keep]) < 1e-13, (solver, idir, k)
    assert flip.mean() < 0.01


def test_plugin_api_and_last_diag(states):
    """hlld_flux keeps the reference's return layout and LAST_DIAG keys."""
    nL, nR = states
    F, U, ps = H.hlld_flux(to_dev(nL), to_dev(nR), EOS, idir=0)
    assert set(F) == {"D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz"} == set(U)
    d = H.LAST_DIAG
    for key in ("solver", "idir", "n_interfaces", "n_not_converged", "n_wave_order_bad",
                "n_bn_zero", "n_hlle_fallback", "frac_hlle_fallback", "mean_iters",
                "max_iters"):
        assert key in d
    _, _, ops, oerr, oit, ofl = oracle.riemann(nL, nR, 0, "hlld", GAMMA)
    assert d["n_interfaces"] == 4000
    fail = (ofl & oracle.RF_FAILED) != 0
    assert abs(d["n_hlle_fallback"] - int(fail.sum())) <= 20
    conv = oerr == 0
    assert abs(d["mean_iters"] - float(oit[conv].mean())) < 0.05
    # hlle_flux leaves LAST_DIAG alone (hlld.py:1005-1044 never writes it)
    before = dict(d)
    H.hlle_flux(to_dev(nL), to_dev(nR), EOS, idir=1)
    assert H.LAST_DIAG == before


def test_rotation_equivalence():
    """flux(C P, idir=1) == C flux(P, idir=0) (reference tests/test_idir.py)."""
    sL, sR = random_face_states(2000, GAMMA, seed=7)
    cyc = lambda d: {**d, "vx": d["vz"], "vy": d["vx"], "vz": d["vy"],
                     "Bx": d["Bz"], "By": d["Bx"], "Bz": d["By"]}
    F0, U0, p0 = H.hlld_flux(to_dev(to_np(sL)), to_dev(to_np(sR)), EOS, idir=0)
    F1, U1, p1 = H.hlld_flux(to_dev(to_np(cyc(sL))), to_dev(to_np(cyc(sR))), EOS, idir=1)
    keep = ~((p0 < 0) ^ (p1 < 0))
    expect = {**F0, "Sx": F0["Sz"], "Sy": F0["Sx"], "Sz": F0["Sy"],
              "Bx": F0["Bz"], "By": F0["Bx"], "Bz": F0["By"]}
    for k in F1:
        assert max_rel(expect[k][keep].cpu().numpy(), F1[k][keep].cpu().numpy()) < 1e-13, k
    assert float((~keep).float().mean()) < 0.005


def test_cpu_tensors_are_rejected(states):
    nL, nR = states
    cpu = {k: torch.as_tensor(v) for k, v in nL.items()}
    with pytest.raises(TypeError):
        H.hlld_flux(cpu, cpu, EOS)


@pytest.mark.parametrize("idir", [0, 1, 2])
def test_hllc_matches_reference_golden(idir):
    """hllc_flux against the reference's own output (tests/golden/hllc.npz,
    a quarter of the faces with zero normal field): FP64-exact build."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "hllc.npz"))
    keys = ["rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz"]
    L = {k: torch.tensor(z[f"{idir}_L_{k}"], device="cuda") for k in keys}
    R = {k: torch.tensor(z[f"{idir}_R_{k}"], device="cuda") for k in keys}
    F, U, ps = Hh.hllc_flux(L, R, EOS, idir=idir, precision="fp64_exact")
    for k in ("D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz"):
        assert max_rel(z[f"{idir}_F_{k}"], F[k].cpu().numpy()) < 1e-12, k
        assert max_rel(z[f"{idir}_U_{k}"], U[k].cpu().numpy()) < 1e-12, k
    assert max_rel(z[f"{idir}_pstar"], ps.cpu().numpy()) < 1e-14
