"""The fused 2D RK3 + CT step against the oracle, and its invariants.

The FP64-exact step must reproduce the oracle's step bit for bit (same
reconstruction, fluxes, corner EMF, combine, BCs and C2P, one rounding per
operation); the FMA step within 1e-10 relative after a few steps.  Property
checks follow the reference's own tests: div B at round-off
(tests/test_ct.py:262-289), the periodic seam (:428-462), pi-rotation
symmetry of the rotor (:351-369).
"""
import numpy as np
import pytest
import torch

from helpers import bitwise_equal, max_rel
from oracle import oracle

import hlld_ai_b200 as H
from hlld_ai_b200.physics.grid import Grid2D
from hlld_ai_b200.physics.initial_data2d import PROBLEMS, b_from_potential
from hlld_ai_b200.physics.reconstruction import ghosts_needed
from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS, State2D

pytestmark = pytest.mark.gpu


def build(problem, nx, ny, limiter="mc", solver="hlld", precision="fp64_exact", emf_mode="solver"):
    spec = PROBLEMS[problem]
    lo, hi = spec["box"]
    ng = ghosts_needed(limiter)
    gc = Grid2D(lo, hi, nx, lo, hi, ny, ng=ng, device="cpu")
    eos = H.hybrid_eos(K=0.0, gamma=spec["gamma"], gamma_th=spec["gamma"])
    prims, Az = spec["build"](gc, eos)
    prims = {k: v.contiguous().numpy().copy() for k, v in prims.items()}
    Bxf, Byf = b_from_potential(Az, gc.dx, gc.dy)
    Bxf, Byf = Bxf.contiguous().numpy().copy(), Byf.contiguous().numpy().copy()
    bc = spec["bc"]
    # oracle state
    cons = oracle.prim_to_cons(prims)
    ostate = {"cons": {k: cons[k].copy() for k in EVOLVED_KEYS}, "Bxf": Bxf.copy(),
              "Byf": Byf.copy(), "prims": {k: prims[k].copy() for k in PRIM_KEYS}}
    og = oracle.Grid2DSpec(nx, ny, ng, gc.dx, gc.dy, bc[0], bc[1], limiter, solver, spec["gamma"],
                           emf_mode=emf_mode)
    oracle.sync_state(og, ostate)
    # device state
    g = Grid2D(lo, hi, nx, lo, hi, ny, ng=ng, device="cuda")
    dev = lambda a: torch.from_numpy(a).cuda()
    gprims = {k: dev(prims[k]) for k in PRIM_KEYS}
    gcons = H.prims_to_cons_2d(gprims, g, "fp64" if precision == "mixed" else precision)
    if precision == "mixed":  # FP32 primitives (recomputed by the sync below)
        gprims = {k: v.float() for k, v in gprims.items()}
    st = State2D(cons={k: gcons[k].contiguous() for k in EVOLVED_KEYS}, Bxf=dev(Bxf),
                 Byf=dev(Byf), prims=gprims)
    stepper = H.Stepper2D(g, eos, bc_x=bc[0], bc_y=bc[1], flux_fn=solver, limiter=limiter,
                          precision=precision, emf_mode=emf_mode)
    stepper.sync(st)
    return g, eos, st, stepper, og, ostate


def compare(st, ostate, exact, tol=1e-10):
    for k in EVOLVED_KEYS:
        a, b = st.cons[k].cpu().numpy(), ostate["cons"][k]
        if exact:
            assert bitwise_equal(a, b), ("cons", k, max_rel(b, a))
        else:
            assert max_rel(b, a) < tol, ("cons", k, max_rel(b, a))
    for name in ("Bxf", "Byf"):
        a, b = getattr(st, name).cpu().numpy(), ostate[name]
        if exact:
            assert bitwise_equal(a, b), (name, max_rel(b, a))
        else:
            assert max_rel(b, a) < tol, (name, max_rel(b, a))
    for k in PRIM_KEYS:
        a, b = st.prims[k].cpu().numpy(), ostate["prims"][k]
        if exact:
            assert bitwise_equal(a, b), ("prims", k, max_rel(b, a))
        else:
            assert max_rel(b, a) < tol, ("prims", k, max_rel(b, a))


CASES = [
    ("rotor", 32, 32, "mc", "hlld"),
    ("orszag_tang", 32, 32, "mc", "hlld"),
    ("rotor_tapered", 40, 36, "mc", "hlld"),
    ("riemann2d", 33, 29, "mc", "hlld"),
    ("rotor", 32, 32, "mc", "hlle"),
    ("orszag_tang", 30, 34, "weno5z", "hlld"),
    ("riemann2d", 32, 32, "mp5", "hlld"),
    ("rotor", 24, 24, "minmod", "hlld"),
    ("orszag_tang", 24, 24, "pcm", "hlld"),
    ("orszag_tang", 24, 24, "mp7", "hlld"),
    ("rotor", 32, 32, "mc", "hllc"),
    ("orszag_tang", 28, 28, "weno5z", "hllc"),
]


@pytest.mark.parametrize("problem,nx,ny,limiter,solver", CASES)
def test_exact_step_bitwise_oracle(problem, nx, ny, limiter, solver):
    g, eos, st, stepper, og, ostate = build(problem, nx, ny, limiter, solver, "fp64_exact")
    compare(st, ostate, exact=True)
    for _ in range(3):
        dt = oracle.compute_dt_2d(og, ostate["prims"], 0.4)
        gdt = float(stepper.compute_dt(st, 0.4).item())
        assert gdt == dt
        oracle.rk_step_ct(og, ostate, dt, "rk3")
        stepper.step(st, dt, "rk3")
        compare(st, ostate, exact=True)


@pytest.mark.parametrize("problem,nx,ny,limiter,solver", CASES[:4])
def test_fma_step_close_to_oracle(problem, nx, ny, limiter, solver):
    g, eos, st, stepper, og, ostate = build(problem, nx, ny, limiter, solver, "fp64")
    for _ in range(3):
        dt = oracle.compute_dt_2d(og, ostate["prims"], 0.4)
        oracle.rk_step_ct(og, ostate, dt, "rk3")
        stepper.step(st, dt, "rk3")
    compare(st, ostate, exact=False, tol=1e-9)


@pytest.mark.parametrize("problem,limiter,solver", [
    ("rotor", "mc", "hlld"), ("orszag_tang", "mc", "hlld"), ("orszag_tang", "weno5z", "hlle"),
    ("rotor_tapered", "mc", "hllc")])
def test_hll_face_emf_exact_step_bitwise_oracle(problem, limiter, solver):
    """emf_mode "hll" (ct.py:63-96): the face EMF from the HLL average of the
    transverse-B flux, whatever the solver; bit for bit with the oracle,
    which is pinned to the reference's rk_step_ct(emf_mode="hll")."""
    g, eos, st, stepper, og, ostate = build(problem, 32, 32, limiter, solver, "fp64_exact",
                                            emf_mode="hll")
    for _ in range(3):
        dt = oracle.compute_dt_2d(og, ostate["prims"], 0.4)
        oracle.rk_step_ct(og, ostate, dt, "rk3")
        stepper.step(st, dt, "rk3")
        compare(st, ostate, exact=True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_hll_face_emf_fast_forms_close_to_oracle(precision):
    """The FMA form within 1e-9 relative; the mixed form within 1e-5 in L1
    (relative) on the faces and the density."""
    g, eos, st, stepper, og, ostate = build("rotor", 32, 32, "mc", "hlld", precision,
                                            emf_mode="hll")
    for _ in range(3):
        dt = oracle.compute_dt_2d(og, ostate["prims"], 0.4)
        oracle.rk_step_ct(og, ostate, dt, "rk3")
        stepper.step(st, dt, "rk3")
    if precision == "fp64":
        compare(st, ostate, exact=False, tol=1e-9)
        return
    for a, b in ((st.Bxf, ostate["Bxf"]), (st.Byf, ostate["Byf"]), (st.cons["D"], ostate["cons"]["D"])):
        a = a.cpu().numpy()
        assert np.abs(a - b).mean() <= 1e-5 * np.abs(b).mean()


def test_hll_face_emf_keeps_div_b_at_roundoff():
    """reference tests/test_ct.py:262-289 with emf_mode="hll"."""
    g, eos, st, stepper, og, ostate = build("orszag_tang", 128, 128, "mc", "hlld", "fp64",
                                            emf_mode="hll")
    d0 = g.div_b(st.Bxf, st.Byf)[g.phys]
    for _ in range(5):
        stepper.step(st, stepper.compute_dt(st, 0.4), "rk3")
    d1 = g.div_b(st.Bxf, st.Byf)[g.phys]
    bmax = float(torch.maximum(st.Bxf.abs().max(), st.Byf.abs().max()))
    assert float((d1 - d0).abs().max()) < 1e-12 * bmax / g.dx


def test_rk2_matches_oracle():
    g, eos, st, stepper, og, ostate = build("orszag_tang", 24, 24, "mc", "hlld", "fp64_exact")
    for _ in range(2):
        dt = oracle.compute_dt_2d(og, ostate["prims"], 0.4)
        oracle.rk_step_ct(og, ostate, dt, "rk2")
        stepper.step(st, dt, "rk2")
    compare(st, ostate, exact=True)


def test_reference_signature_step_leaves_input_untouched():
    g, eos, st, stepper, og, ostate = build("rotor", 32, 32)
    before = {k: v.clone() for k, v in st.cons.items()}
    dt = H.compute_dt_2d(st.prims, g, eos, 0.4)
    S, diag = H.rk_step_ct(st, g, eos, dt, scheme="rk3", bc_x="outflow", bc_y="outflow",
                           flux_fn=H.hlld_flux, limiter="mc", precision="fp64_exact")
    for k in before:
        assert torch.equal(before[k], st.cons[k])
    oracle.rk_step_ct(og, ostate, dt, "rk3")
    compare(S, ostate, exact=True)
    d = diag["x"]["diag"]
    assert d["n_interfaces"] == (g.nxt + 1) * g.nyt
    assert 0.0 <= d["frac_hlle_fallback"] <= 1.0


def test_div_b_and_seam_at_256():
    """div B stays at round-off and the periodic seam faces stay identical."""
    g, eos, st, stepper, og, ostate = build("orszag_tang", 256, 256, "mc", "hlld", "fp64")
    ng, n = g.ng, g.nx
    d0 = g.div_b(st.Bxf, st.Byf)[g.phys]
    for _ in range(5):
        dt = stepper.compute_dt(st, 0.4)
        stepper.step(st, dt, "rk3")
    d1 = g.div_b(st.Bxf, st.Byf)[g.phys]
    bmax = float(torch.maximum(st.Bxf.abs().max(), st.Byf.abs().max()))
    assert float((d1 - d0).abs().max()) < 1e-12 * bmax / g.dx
    assert torch.equal(st.Bxf[ng], st.Bxf[ng + n])
    assert torch.equal(st.Byf[:, ng], st.Byf[:, ng + n])
    for k in EVOLVED_KEYS:
        assert torch.isfinite(st.cons[k]).all()


def test_rotor_pi_rotation_symmetry():
    """reference tests/test_ct.py:351-369: the rotor stays pi-rotation
    symmetric (rho even, v odd, B even) to 1e-9 after 8 steps."""
    g, eos, st, stepper, og, ostate = build("rotor", 32, 32, "mc", "hlld", "fp64")
    for _ in range(8):
        stepper.step(st, stepper.compute_dt(st, 0.25), "rk3")
    ph = g.phys
    worst = 0.0
    for k, parity in (("rho", 1), ("p", 1), ("vx", -1), ("vy", -1), ("Bx", 1), ("By", 1)):
        a = st.prims[k][ph]
        b = torch.flip(a, dims=(0, 1))
        worst = max(worst, float((a - parity * b).abs().max()) / max(float(a.abs().max()), 1e-30))
    assert worst < 1e-9, worst


def test_step_rejects_bad_state():
    g, eos, st, stepper, og, ostate = build("rotor", 32, 32)
    bad = State2D(cons=dict(st.cons), Bxf=st.Bxf[:-1], Byf=st.Byf, prims=st.prims)
    with pytest.raises(ValueError):
        stepper.step(bad, 1e-3)
    cpu = State2D(cons={k: v.cpu() for k, v in st.cons.items()}, Bxf=st.Bxf, Byf=st.Byf,
                  prims=st.prims)
    with pytest.raises(TypeError):
        stepper.step(cpu, 1e-3)


def test_stepper_takes_reference_shaped_grid_and_eos():
    """A caller inside the reference passes its own Grid2D and hybrid_eos:
    the stepper reads only nx, ny, ng, dx, dy, device and K, gamma,
    gamma_th, so objects with just those attributes give the same step."""
    from types import SimpleNamespace

    g, eos, st, stepper, og, ostate = build("rotor_tapered", 48, 40, "mc", "hlld", "fp64")
    ref_grid = SimpleNamespace(nx=g.nx, ny=g.ny, ng=g.ng, dx=g.dx, dy=g.dy, device=g.device,
                               nxt=g.nxt, nyt=g.nyt)
    ref_eos = SimpleNamespace(K=0.0, gamma=eos.gamma, gamma_th=eos.gamma)
    other = H.Stepper2D(ref_grid, ref_eos, bc_x="periodic", bc_y="periodic", flux_fn="hlld",
                        limiter="mc", precision="fp64")
    twin = st.clone()
    for _ in range(2):
        dt = stepper.compute_dt(st, 0.4)
        stepper.step(st, dt, "rk3")
        other.step(twin, dt, "rk3")
    for k in EVOLVED_KEYS:
        assert bitwise_equal(st.cons[k].cpu().numpy(), twin.cons[k].cpu().numpy()), k
    assert bitwise_equal(st.Byf.cpu().numpy(), twin.Byf.cpu().numpy())
