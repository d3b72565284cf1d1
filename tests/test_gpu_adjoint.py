"""The discrete adjoint of the FP64 RK3+CT step against central finite
differences of the forward step (the same kernels, dt sequence fixed).

A gradient from the adjoint is exact for the frozen-decision linearisation
of the scheme; a central difference with h small enough not to cross a
limiter or Riemann-solver switch agrees with it to O(h^2) plus round-off.
"""
import math

import numpy as np
import pytest
import torch

import hlld_ai_b200 as H
from hlld_ai_b200.adjoint import (CheckpointedRun, RKSteps, RotorCase, gaussian_weight,
                                  magnetic_objective, prim_to_cons_vjp, rotor_forward,
                                  rotor_gradients)
from hlld_ai_b200.physics.state import CONS_KEYS, EVOLVED_KEYS, PRIM_KEYS, State2D

pytestmark = pytest.mark.gpu


def _setup(problem, n, limiter="mc"):
    g, eos, st, spec = H.setup_problem(problem, n, limiter=limiter, device="cuda")
    run = CheckpointedRun(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], limiter=limiter,
                          checkpoint_every=3)
    return g, eos, st, run


def _objective_of_final(g, w, outs):
    """A smooth objective touching every conserved variable and both faces."""
    J = 0.0
    ph = g.phys
    for i, k in enumerate(EVOLVED_KEYS):
        J = J + (w[ph] * outs[i][ph] ** 2).sum() * (0.1 * (i + 1))
    J = J + (outs[6][2:-2, 2:-2] ** 2).sum() * 1e-3 + (outs[7][2:-2, 2:-2] ** 2).sum() * 1e-3
    return J


def _inputs(st):
    return [st.cons[k].clone() for k in EVOLVED_KEYS] + [st.Bxf.clone(), st.Byf.clone()]


def _run_J(run, dts, g, w, xs):
    outs = RKSteps.apply(run, dts, *xs)
    return float(_objective_of_final(g, w, outs))


@pytest.mark.parametrize("problem,limiter", [("rotor_tapered", "mc"), ("orszag_tang", "mc"),
                                             ("rotor_tapered", "weno5z")])
def test_adjoint_directional_derivative_matches_central_difference(problem, limiter):
    n = 32
    g, eos, st, run = _setup(problem, n, limiter)
    w = gaussian_weight(g)
    dts = []
    s = st.clone()
    for _ in range(6):
        dt = float(run.stepper.compute_dt(s, 0.4).item())
        dts.append(dt)
        run.stepper.step(s, dt, "rk3")
    xs = [x.requires_grad_(True) for x in _inputs(st)]
    outs = RKSteps.apply(run, dts, *xs)
    J = _objective_of_final(g, w, outs)
    J.backward()
    grads = [x.grad.clone() for x in xs]
    gen = torch.Generator(device="cuda").manual_seed(3)
    ph = g.phys
    for trial in range(3):
        # a direction on the physical conserved cells (scaled to each field)
        d = []
        for i, x in enumerate(xs[:6]):
            di = torch.zeros_like(x)
            scale = float(x.detach()[ph].abs().mean()) + 1e-3
            di[ph] = scale * (2 * torch.rand(di[ph].shape, generator=gen, device="cuda",
                                             dtype=torch.float64) - 1)
            d.append(di)
        d += [torch.zeros_like(xs[6]), torch.zeros_like(xs[7])]
        adj = sum(float((gi * di).sum()) for gi, di in zip(grads, d))
        h = 1e-6
        xp = [x.detach() + h * di for x, di in zip(xs, d)]
        xm = [x.detach() - h * di for x, di in zip(xs, d)]
        fd = (_run_J(run, dts, g, w, xp) - _run_J(run, dts, g, w, xm)) / (2 * h)
        assert abs(adj - fd) <= 1e-5 * abs(fd) + 1e-12, (problem, trial, adj, fd)


def test_checkpoint_interval_does_not_change_the_gradient():
    n = 32
    g, eos, st, _ = _setup("rotor_tapered", n)
    w = gaussian_weight(g)
    res = []
    for every in (1, 4, 10):
        run = CheckpointedRun(g, eos, bc_x="periodic", bc_y="periodic", checkpoint_every=every)
        dts = [2e-4] * 10
        xs = [x.requires_grad_(True) for x in _inputs(st)]
        J = _objective_of_final(g, w, RKSteps.apply(run, dts, *xs))
        J.backward()
        res.append([x.grad.clone() for x in xs])
    for other in res[1:]:
        for a, b in zip(res[0], other):
            assert torch.equal(a, b)


def test_prim_to_cons_vjp_matches_central_difference():
    g, eos, st, _ = _setup("rotor_tapered", 32)
    prims = {k: st.prims[k].clone() for k in PRIM_KEYS}
    gen = torch.Generator(device="cuda").manual_seed(5)
    lam = {k: torch.randn(prims["rho"].shape, generator=gen, device="cuda", dtype=torch.float64)
           for k in CONS_KEYS}
    lp = prim_to_cons_vjp(prims, lam)
    from hlld_ai_b200.physics.driver2d import prims_to_cons_2d
    for k in ("rho", "vx", "p", "eps", "By"):
        h = 1e-7 * (float(prims[k].abs().max()) + 1.0)
        pp = dict(prims)
        pm = dict(prims)
        pp[k] = prims[k] + h
        pm[k] = prims[k] - h
        cp, cm = prims_to_cons_2d(pp, g), prims_to_cons_2d(pm, g)
        fd = sum((lam[c] * (cp[c] - cm[c]) / (2 * h)) for c in CONS_KEYS if c in cp)
        assert torch.allclose(lp[k], fd, rtol=1e-6, atol=1e-8 * float(fd.abs().max() + 1)), k


def test_rotor_gradient_study_small():
    """The rotor objective (Gaussian-weighted final magnetic energy) at 48^2
    over 30 steps, checkpointed every 10: dJ/d omega and dJ/d rho0 along
    random directions against central differences (h = 1e-6)."""
    case = RotorCase(n=48, steps=30, checkpoint_every=10)
    r = rotor_gradients(case)
    run, g, eos, w, dts = r["run"], r["grid"], r["eos"], r["weight"], r["dts"]
    h = 1e-6
    Jp = rotor_forward(run, g, eos, None, case.omega * (1 + h), dts, w)
    Jm = rotor_forward(run, g, eos, None, case.omega * (1 - h), dts, w)
    fd_w = (Jp - Jm) / (2 * h * case.omega)
    assert abs(r["grad_omega"] - fd_w) <= 1e-5 * abs(fd_w), (r["grad_omega"], fd_w)
    gen = torch.Generator(device="cuda").manual_seed(11)
    rho0 = r["rho0"]
    for trial in range(4):
        d = rho0 * (2 * torch.rand(rho0.shape, generator=gen, device="cuda",
                                   dtype=torch.float64) - 1)
        adj = float((r["grad_rho0"] * d).sum())
        Jp = rotor_forward(run, g, eos, rho0 + h * d, case.omega, dts, w)
        Jm = rotor_forward(run, g, eos, rho0 - h * d, case.omega, dts, w)
        fd = (Jp - Jm) / (2 * h)
        assert abs(adj - fd) <= 1e-5 * abs(fd), (trial, adj, fd)
