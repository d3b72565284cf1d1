"""The all-FP32 form (HLLD_FP32: conserved state, staggered field,
primitives, fluxes, the HLLD p* solve and the cell C2P all in float) against
the oracle, a precision study beside the FP64 and mixed forms.

Tolerances (density and pressure L1 after five RK3 steps from the same
initial state, the oracle's dt sequence), with the values measured on a
B200 in brackets:
  * rotor (rho 10 disk at v = 0.995, W = 10): 1e-3 (2.0e-4 at 32^2,
    3.4e-4 at 64^2) -- the FP32 C2P of the rim's W = 10 cells and faces on
    the HLLD wave-order thresholds make this the worst case;
  * relativistic vortex: 1e-4 (2.1e-5 .. 3.3e-5);
  * Orszag-Tang: 1e-5 (1.7e-6 .. 2.2e-6).
No cell C2P may fail, and div B stays at FP32 round-off.
"""
import numpy as np
import pytest
import torch

from oracle import oracle

import hlld_ai_b200 as H
from hlld_ai_b200.physics.initial_data2d import b_from_potential, initial_prims
from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS

pytestmark = pytest.mark.gpu

TOL = {"rotor_tapered": 1e-3, "vortex": 1e-4, "orszag_tang": 1e-5}


def test_fp32_state_is_float32_throughout():
    g, eos, st, spec = H.setup_problem("rotor_tapered", 48, device="cuda", precision="fp32")
    assert all(st.cons[k].dtype == torch.float32 for k in EVOLVED_KEYS)
    assert all(st.prims[k].dtype == torch.float32 for k in PRIM_KEYS)
    assert st.Bxf.dtype == torch.float32 and st.Byf.dtype == torch.float32
    stp = H.Stepper2D(g, eos, bc_x="periodic", bc_y="periodic", precision="fp32")
    stp.step(st, stp.compute_dt(st, 0.4), "rk3")
    assert all(torch.isfinite(st.cons[k]).all() for k in EVOLVED_KEYS)
    g2, _, st64, _ = H.setup_problem("rotor_tapered", 48, device="cuda", precision="fp64")
    with pytest.raises(ValueError):  # an FP64 state is refused, not converted
        stp.step(st64, 1e-4, "rk3")


@pytest.mark.parametrize("problem", sorted(TOL))
@pytest.mark.parametrize("n", [32, 64])
def test_fp32_step_close_to_the_oracle(problem, n):
    g64, eos, prims, Az, spec = initial_prims(problem, n, 2, "cpu")
    np_prims = {k: v.contiguous().numpy().copy() for k, v in prims.items()}
    Bxf, Byf = b_from_potential(Az, g64.dx, g64.dy)
    cons = oracle.prim_to_cons(np_prims)
    ost = {"cons": {k: cons[k].copy() for k in EVOLVED_KEYS},
           "Bxf": Bxf.contiguous().numpy().copy(), "Byf": Byf.contiguous().numpy().copy(),
           "prims": {k: np_prims[k].copy() for k in PRIM_KEYS}}
    og = oracle.Grid2DSpec(n, n, 2, g64.dx, g64.dy, *spec["bc"], "mc", "hlld", spec["gamma"])
    oracle.sync_state(og, ost)
    g, eos, st, _ = H.setup_problem(problem, n, device="cuda", precision="fp32")
    stp = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], precision="fp32")
    for _ in range(5):
        dt = oracle.compute_dt_2d(og, ost["prims"], 0.4)
        oracle.rk_step_ct(og, ost, dt, "rk3")
        stp.step(st, dt, "rk3")
    ph = g.phys
    for key in ("rho", "p"):
        d = np.abs(st.prims[key][ph].double().cpu().numpy() - ost["prims"][key][ph])
        assert d.mean() <= TOL[problem], (key, d.mean(), d.max())
    assert stp.diag()["c2p"]["not_converged"] == 0
    div = g.div_b(st.Bxf.double(), st.Byf.double())[ph]
    bmax = float(torch.maximum(st.Bxf.abs().max(), st.Byf.abs().max()))
    assert float(div.abs().max()) < 1e-5 * bmax / g.dx
