"""The discrete adjoint of the FP64 RK+CT step against central finite
differences of the forward step (the same kernels, dt sequence fixed).

A gradient from the adjoint is exact for the frozen-decision linearisation
of the scheme; a central difference agrees with it to O(h^2) plus round-off
wherever the scheme is differentiable at the state.  It is not
differentiable where a discrete choice sits exactly on its switch: a limiter
at a uniform field (a = b = 0), the HLL wave speeds max(c_L, c_R) where the
two sides tie (mirror-symmetric data such as the Orszag-Tang vortex), an
HLLD wave-order check on its threshold.  There a central difference returns
the average of two one-sided slopes, not a derivative.  The checks therefore
run on a generic smooth state (random-phase sinusoids in every field, a
divergence-free field from a random potential), where no tie occurs.
"""
import math

import numpy as np
import pytest
import torch

import hlld_ai_b200 as H
from hlld_ai_b200.adjoint import (CheckpointedRun, RKSteps, RotorCase, gaussian_weight,
                                  magnetic_objective, prim_to_cons_vjp, rotor_fd_study,
                                  rotor_forward, rotor_gradients)
from hlld_ai_b200.physics.state import CONS_KEYS, EVOLVED_KEYS, PRIM_KEYS, State2D

pytestmark = pytest.mark.gpu


def _setup(problem, n, limiter="mc"):
    g, eos, st, spec = H.setup_problem(problem, n, limiter=limiter, device="cuda")
    run = CheckpointedRun(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], limiter=limiter,
                          checkpoint_every=3)
    return g, eos, st, run


def smooth_random_state(n, limiter="mc", seed=1, solver="hlld", upwind=True, scheme="rk3"):
    """A periodic state with no symmetry: every primitive a sum of three
    random-phase sinusoids, B from a random potential plus a uniform part."""
    from hlld_ai_b200.physics.driver2d import prims_to_cons_2d
    from hlld_ai_b200.physics.grid import Grid2D
    from hlld_ai_b200.physics.initial_data2d import b_from_potential
    from hlld_ai_b200.physics.reconstruction import ghosts_needed

    eos = H.hybrid_eos(K=0.0, gamma=5.0 / 3.0, gamma_th=5.0 / 3.0)
    g = Grid2D(0.0, 1.0, n, 0.0, 1.0, n, ng=ghosts_needed(limiter), device="cuda")
    rng = np.random.default_rng(seed)

    def field(X, Y):
        s = 0.0
        for _ in range(3):
            kx, ky = rng.integers(1, 3, 2)
            s = s + rng.uniform(0.3, 1.0) * torch.sin(2 * math.pi * (kx * X + ky * Y)
                                                      + rng.uniform(0, 2 * math.pi))
        return s / 3.0

    X, Y = g.X, g.Y
    prims = {"rho": 1.0 + 0.3 * field(X, Y), "p": 1.0 + 0.3 * field(X, Y),
             "vx": 0.3 * field(X, Y), "vy": 0.3 * field(X, Y), "vz": 0.2 * field(X, Y),
             "Bz": 0.4 * field(X, Y)}
    XF, YF = g.corner_mesh()
    Az = 0.5 * YF - 0.3 * XF + 0.05 * field(XF, YF)
    Bxf, Byf = b_from_potential(Az, g.dx, g.dy)
    Bxf, Byf = Bxf.contiguous(), Byf.contiguous()
    prims["Bx"] = 0.5 * (Bxf[:-1, :] + Bxf[1:, :])
    prims["By"] = 0.5 * (Byf[:, :-1] + Byf[:, 1:])
    prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    prims = {k: v.contiguous() for k, v in prims.items()}
    c = prims_to_cons_2d(prims, g)
    st = State2D(cons={k: c[k].contiguous() for k in EVOLVED_KEYS}, Bxf=Bxf, Byf=Byf, prims={})
    run = CheckpointedRun(g, eos, bc_x="periodic", bc_y="periodic", limiter=limiter,
                          flux_fn=solver, upwind=upwind, scheme=scheme, checkpoint_every=3)
    run.stepper.sync(st)
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


@pytest.mark.parametrize("limiter,solver,upwind,scheme", [
    ("pcm", "hlle", False, "rk2"), ("mc", "hlle", True, "rk3"), ("mc", "hlld", True, "rk3"),
    ("weno5z", "hlld", True, "rk3"), ("minmod", "hlld", False, "rk2")])
def test_adjoint_directional_derivative_matches_central_difference(limiter, solver, upwind, scheme):
    """Four steps on a smooth 24^2 state: the gradient of an objective of
    every output field, along random directions in the conserved cells (and,
    in the last trial, the faces), against central differences (h = 1e-6)."""
    g, eos, st, run = smooth_random_state(24, limiter, seed=7, solver=solver, upwind=upwind,
                                          scheme=scheme)
    w = gaussian_weight(g)
    dts = []
    s = st.clone()
    for _ in range(4):
        dt = float(run.stepper.compute_dt(s, 0.4).item())
        dts.append(dt)
        run.stepper.step(s, dt, scheme)
    xs = [x.requires_grad_(True) for x in _inputs(st)]
    outs = RKSteps.apply(run, dts, *xs)
    J = _objective_of_final(g, w, outs)
    J.backward()
    grads = [x.grad.clone() for x in xs]
    gen = torch.Generator(device="cuda").manual_seed(3)
    ph = g.phys
    ng = g.ng
    for trial in range(3):
        d = []
        for i, x in enumerate(xs):
            di = torch.zeros_like(x)
            if i < 6:
                scale = float(x.detach()[ph].abs().mean()) + 1e-3
                di[ph] = scale * (2 * torch.rand(di[ph].shape, generator=gen, device="cuda",
                                                 dtype=torch.float64) - 1)
            elif trial == 2:
                # the faces too (interior faces only: the seam copies are set
                # by the boundary fill); a field perturbation need not be
                # divergence free for the derivative check
                sl = (slice(ng, -ng - 1), slice(ng, -ng)) if i == 6 else (slice(ng, -ng), slice(ng, -ng - 1))
                di[sl] = 0.3 * (2 * torch.rand(di[sl].shape, generator=gen, device="cuda",
                                               dtype=torch.float64) - 1)
            d.append(di)
        adj = sum(float((gi * di).sum()) for gi, di in zip(grads, d))
        h = 1e-6
        xp = [x.detach() + h * di for x, di in zip(xs, d)]
        xm = [x.detach() - h * di for x, di in zip(xs, d)]
        fd = (_run_J(run, dts, g, w, xp) - _run_J(run, dts, g, w, xm)) / (2 * h)
        # cells only: 1e-5; cells and faces: 5e-5 (a face perturbation also
        # moves the normal field Bn, whose HLL wave-speed ties are the
        # likeliest kinks in a generic state)
        tol = 1e-5 if trial < 2 else 5e-5
        assert abs(adj - fd) <= tol * abs(fd) + 1e-10, (limiter, solver, trial, adj, fd)


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
    """The rotor study's pipeline at 48^2 over 30 steps, checkpointed every
    10: J and the gradients are finite and independent of the checkpoint
    interval.  (No finite-difference bound here: the rotor's uniform ambient
    medium puts the limiter at its kink and its disk edge holds HLLD faces on
    the wave-order threshold, so central differences of the rotor measure
    jumps, not derivatives; the derivative check is the smooth-state test.)"""
    r1 = rotor_gradients(RotorCase(n=48, steps=30, checkpoint_every=10))
    r2 = rotor_gradients(RotorCase(n=48, steps=30, checkpoint_every=7))
    assert math.isfinite(r1["J"]) and math.isfinite(r1["grad_omega"])
    assert bool(torch.isfinite(r1["grad_rho0"]).all())
    assert r1["J"] == r2["J"]
    assert r1["grad_omega"] == r2["grad_omega"]
    assert torch.equal(r1["grad_rho0"], r2["grad_rho0"])


def test_recorded_step_and_reverse_match_the_self_contained_adjoint():
    """hlld_adjoint_record_step advances the state exactly as the production
    step does, and the reverse from its tape equals hlld_adjoint_rk_step_ct
    (which records internally) bit for bit."""
    g, eos, st, run = smooth_random_state(24, "mc", seed=5)
    dt = float(run.stepper.compute_dt(st, 0.4).item())
    a, b = st.clone(), st.clone()
    run.stepper.step(a, dt, "rk3")
    run.record_step(b, dt, 0)
    for k in EVOLVED_KEYS:
        assert torch.equal(a.cons[k], b.cons[k]), k
    assert torch.equal(a.Bxf, b.Bxf) and torch.equal(a.Byf, b.Byf)
    from hlld_ai_b200.adjoint import _zeros_state
    gen = torch.Generator(device="cuda").manual_seed(2)
    lam1 = _zeros_state(g, "cuda")
    for k in EVOLVED_KEYS:
        lam1.cons[k][g.phys] = torch.rand(lam1.cons[k][g.phys].shape, generator=gen, device="cuda",
                                          dtype=torch.float64)
    lam2 = lam1.clone()
    run.reverse_step(st, b, dt, 0, lam1)
    run.step_adjoint(st, a, dt, lam2)
    for k in EVOLVED_KEYS:
        assert torch.equal(lam1.cons[k], lam2.cons[k]), k
    assert torch.equal(lam1.Bxf, lam2.Bxf) and torch.equal(lam1.Byf, lam2.Byf)


def _direction(grid, k):
    """Direction k of tests/helpers.py gradient_directions on the physical cells."""
    from helpers import gradient_directions

    return gradient_directions(grid.X[grid.phys] - 0.5, grid.Y[grid.phys] - 0.5, k)


def test_rotor_gradient_matches_the_reference_central_differences():
    """The config-5 objective on the tapered rotor at 128^2 after four FP64
    HLLD + PLM-MC + RK3 + CT steps, with the reference's dt sequence, against
    the reference's own central differences (tests/golden/rotor_gradient.npz):
    J to 1e-12; dJ/d omega to 1e-6 (measured 8e-8 on a B200; the reference's
    differences at h = 1e-5 and 1e-6 agree); dJ/d rho0 along each seeded
    direction whose two differences (h = 1e-5, 2e-5) agree to 1e-4 -- the
    four ring modes on the rotor's taper -- to 1e-3 (measured 1e-5 .. 1e-4:
    a few hundred MC limiter branches sit on ties between their candidates
    and switch between the +h and -h runs).  The whole-domain modes'
    differences disagree with each other: they perturb the uniform ambient
    medium, where the limiter sits at its kink (a = b = 0), and measure
    jumps, not derivatives.  (The shimmed torch autograd through the
    reference recorded in the same file gives dJ/d omega = 0.630 where its
    central differences and this adjoint give 0.3362: it is not a gradient
    oracle.)"""
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "rotor_gradient.npz"))
    n, dts = int(z["n"]), [float(d) for d in z["dts"]]
    r = rotor_gradients(RotorCase(n=n, checkpoint_every=len(dts)), dts=dts)
    assert abs(r["J"] - float(z["J"])) <= 1e-12 * abs(float(z["J"]))
    fd = z["fd_omega"]
    assert abs(fd[0] - fd[1]) <= 1e-5 * abs(fd[0])
    assert abs(r["grad_omega"] - fd[0]) <= 1e-6 * abs(fd[0]), (r["grad_omega"], fd)
    checked = 0
    for k, (f1, f2) in enumerate(z["fd_dir"]):
        if abs(f1 - f2) > 1e-4 * max(abs(f1), abs(f2)):
            continue
        d = float((r["grad_rho0"] * _direction(r["grid"], k)).sum())
        assert abs(d - f1) <= 1e-3 * abs(f1), (k, d, f1, f2)
        checked += 1
    assert checked >= 4, checked


def test_rotor_gradient_matches_central_differences_on_flip_free_directions():
    """The rotor study itself (tapered rotor, FP64 HLLD + PLM-MC + CT) at
    128^2 over 10 RK3 steps: the adjoint's directional derivatives of J
    against central differences (h = 1e-5) along omega and 16 seeded density
    directions -- 8 smooth modes over the whole domain and 8 ring modes on
    the rotor's taper (tests/helpers.py gradient_directions, seeds 0..15).
    For every direction the discrete decisions the adjoint freezes (HLLE
    fallbacks, CT upwind signs, MC limiter branches) are compared between
    the +h and -h runs.  The whole-domain modes flip hundreds of fallbacks
    and thousands of upwind signs (the limiter's kink in the uniform ambient
    medium) and their differences are jumps.  Directions with no fallback or
    upwind flip must agree to 1e-3 (measured 1.6e-4 .. 3.5e-4 on a B200 for
    the four such ring modes; their remaining flips are MC limiter branches
    at ties between candidates), and at least three directions are such."""
    from helpers import gradient_directions

    dirs = [(lambda X, Y, k=k: gradient_directions(X, Y, k)) for k in range(16)]
    study = rotor_fd_study(RotorCase(n=128, steps=10, checkpoint_every=10), dirs, h=1e-5)
    free = [r for r in study["records"]
            if r["flips"]["fallback"] == 0 and r["flips"]["upwind"] == 0]
    assert len(free) >= 3, [(r["direction"], r["flips"]) for r in study["records"]]
    for r in free:
        assert r["rel_err"] <= 1e-3, r
