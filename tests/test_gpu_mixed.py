"""Mixed-precision step (FP32 primitives, reconstruction, fluxes, corner EMF,
divergence and HLL-state C2P; FP64 cell C2P, HLLD p* iteration and RK
accumulation) against FP64.

Acceptance: density L1 <= 1e-5 against the FP64 solution (the CPU oracle
at small size, the FP64 kernels -- themselves bitwise equal to the oracle in
their exact build -- at larger sizes and times), and div B preserved at
round-off.
"""
import numpy as np
import pytest
import torch

from oracle import oracle

import hlld_ai_b200 as H
from hlld_ai_b200.physics.initial_data2d import b_from_potential, initial_prims
from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS

pytestmark = pytest.mark.gpu


def pair(problem, n):
    out = {}
    for prec in ("fp64", "mixed"):
        g, eos, st, spec = H.setup_problem(problem, n, limiter="mc", device="cuda", precision=prec)
        stp = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld",
                          limiter="mc", precision=prec)
        out[prec] = (g, st, stp)
    return out


def norms(g, a, b):
    ph = g.phys
    d = (a[ph].double() - b[ph].double()).abs()
    return float(d.mean()), float(d.max())


def test_mixed_prims_are_float32_and_state_float64():
    r = pair("rotor_tapered", 64)
    g, st, stp = r["mixed"]
    assert all(st.prims[k].dtype == torch.float32 for k in PRIM_KEYS)
    assert all(st.cons[k].dtype == torch.float64 for k in EVOLVED_KEYS)
    stp.step(st, stp.compute_dt(st, 0.4), "rk3")
    assert all(torch.isfinite(st.cons[k]).all() for k in EVOLVED_KEYS)


def test_rotor_density_l1_within_1e5_of_fp64():
    r = pair("rotor_tapered", 256)
    g = r["fp64"][0]
    for _ in range(20):
        dt = float(r["fp64"][2].compute_dt(r["fp64"][1], 0.4).item())
        for prec in ("fp64", "mixed"):
            r[prec][2].step(r[prec][1], dt, "rk3")
    l1, linf = norms(g, r["mixed"][1].prims["rho"], r["fp64"][1].prims["rho"])
    assert l1 <= 1e-5, (l1, linf)
    assert linf < 1e-2


def test_mixed_matches_the_oracle_on_a_small_rotor():
    n = 32
    g64, eos, prims, Az, spec = initial_prims("rotor_tapered", n, 2, "cpu")
    np_prims = {k: v.contiguous().numpy().copy() for k, v in prims.items()}
    Bxf, Byf = b_from_potential(Az, g64.dx, g64.dy)
    cons = oracle.prim_to_cons(np_prims)
    ost = {"cons": {k: cons[k].copy() for k in EVOLVED_KEYS},
           "Bxf": Bxf.contiguous().numpy().copy(), "Byf": Byf.contiguous().numpy().copy(),
           "prims": {k: np_prims[k].copy() for k in PRIM_KEYS}}
    og = oracle.Grid2DSpec(n, n, 2, g64.dx, g64.dy, *spec["bc"], "mc", "hlld", spec["gamma"])
    oracle.sync_state(og, ost)
    g, eos, st, _ = H.setup_problem("rotor_tapered", n, device="cuda", precision="mixed")
    stp = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], precision="mixed")
    for _ in range(5):
        dt = oracle.compute_dt_2d(og, ost["prims"], 0.4)
        oracle.rk_step_ct(og, ost, dt, "rk3")
        stp.step(st, dt, "rk3")
    ph = g.phys
    d = np.abs(st.prims["rho"][ph].double().cpu().numpy() - ost["prims"]["rho"][ph])
    assert d.mean() <= 1e-5, d.mean()


def test_vortex_precision_study_to_t_half():
    """The relativistic vortex (gamma 4/3) to t = 0.5: L1 of rho, p, |B|^2."""
    r = pair("vortex", 64)
    g = r["fp64"][0]
    t, tend = 0.0, 0.5
    while t < tend - 1e-14:
        dt = min(float(r["fp64"][2].compute_dt(r["fp64"][1], 0.4).item()), tend - t)
        for prec in ("fp64", "mixed"):
            r[prec][2].step(r[prec][1], dt, "rk3")
        t += dt
    a, b = r["mixed"][1].prims, r["fp64"][1].prims
    l1_rho, _ = norms(g, a["rho"], b["rho"])
    l1_p, _ = norms(g, a["p"], b["p"])
    B2 = lambda P: P["Bx"].double() ** 2 + P["By"].double() ** 2 + P["Bz"].double() ** 2
    l1_b2, _ = norms(g, B2(a), B2(b))
    assert l1_rho <= 1e-5, l1_rho
    assert l1_p <= 1e-5, l1_p
    assert l1_b2 <= 1e-5, l1_b2


def test_mixed_preserves_div_b():
    g, eos, st, spec = H.setup_problem("orszag_tang", 128, device="cuda", precision="mixed")
    stp = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], precision="mixed")
    d0 = g.div_b(st.Bxf, st.Byf)[g.phys]
    for _ in range(5):
        stp.step(st, stp.compute_dt(st, 0.4), "rk3")
    d1 = g.div_b(st.Bxf, st.Byf)[g.phys]
    bmax = float(torch.maximum(st.Bxf.abs().max(), st.Byf.abs().max()))
    assert float((d1 - d0).abs().max()) < 1e-12 * bmax / g.dx
