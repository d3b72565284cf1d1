"""Gradients through many RK+CT steps: the discrete adjoint on the GPU.

``CheckpointedRun`` runs the FP64 2D step forward for a fixed sequence of
time steps, keeping the state every ``checkpoint_every`` steps (and the
last segment's step states and tapes), and runs the adjoint backward: each
earlier segment is recomputed once from its checkpoint with
``hlld_adjoint_record_step`` (the step states and each step's tape kept),
then the steps are reversed one by one with ``hlld_adjoint_reverse_step``,
the transpose of the step's Jacobian with the
time step fixed and every discrete decision frozen at its forward outcome
(limiter branches, HLLD region and fallback, CT upwind signs); the HLLD p*
and the Kastaun C2P root are differentiated by the implicit-function
theorem.  The reference has no adjoint; its gradients would come from torch
autograd through ``src/physics/driver2d.py:221-249`` rk_step_ct, which the
same step sequence reproduces.

``RKSteps`` wraps a run in a ``torch.autograd.Function`` over the conserved
state (the six evolved cell variables and the two face fields), so a torch
objective of the final state backpropagates into the initial state.
``rotor_gradients`` is the magnetic-rotor study: the gradient of the
Gaussian-weighted final magnetic energy with respect to the initial density
field and the rotor's angular velocity.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import torch

from . import _lib
from .physics.driver2d import Stepper2D
from .physics.state import CONS_KEYS, EVOLVED_KEYS, PRIM_KEYS, State2D

_SCHEMES = {"rk2": 2, "rk3": 3}


def _zeros_state(grid, device) -> State2D:
    z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=device)
    return State2D(cons={k: z(grid.nxt, grid.nyt) for k in EVOLVED_KEYS},
                   Bxf=z(grid.nxt + 1, grid.nyt), Byf=z(grid.nxt, grid.nyt + 1),
                   prims={k: z(grid.nxt, grid.nyt) for k in PRIM_KEYS})


class CheckpointedRun:
    """Forward steps with checkpoints, and the adjoint of the whole run."""

    def __init__(self, grid, eos, *, bc_x="periodic", bc_y="periodic", flux_fn="hlld",
                 limiter="mc", scheme="rk3", upwind=True, atmo_rho=1e-10,
                 checkpoint_every=20):
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.grid, self.eos, self.scheme = grid, eos, scheme
        self.every = int(checkpoint_every)
        self.stepper = Stepper2D(grid, eos, bc_x=bc_x, bc_y=bc_y, flux_fn=flux_fn,
                                 limiter=limiter, upwind=upwind, atmo_rho=atmo_rho,
                                 precision="fp64")
        self.device = self.stepper.device
        n = ctypes.c_size_t(0)
        _lib.check(_lib.lib().hlld_adjoint_scratch_bytes(ctypes.byref(self.stepper.gc),
                                                         ctypes.byref(n)),
                   "hlld_adjoint_scratch_bytes")
        self._scratch = torch.empty(n.value + 256, dtype=torch.uint8, device=self.device)
        self._scratch_ptr = (self._scratch.data_ptr() + 255) // 256 * 256
        self._scratch_bytes = n.value
        tb, rb = ctypes.c_size_t(0), ctypes.c_size_t(0)
        _lib.check(_lib.lib().hlld_adjoint_tape_bytes(ctypes.byref(self.stepper.gc),
                                                      ctypes.byref(tb), ctypes.byref(rb)),
                   "hlld_adjoint_tape_bytes")
        self._tape_bytes = tb.value
        assert rb.value <= self._scratch_bytes
        # one tape per step of a segment, allocated up front
        self._tapes: list[torch.Tensor] = [
            torch.empty(self._tape_bytes + 256, dtype=torch.uint8, device=self.device)
            for _ in range(self.every)]
        self.checkpoints: list[State2D] = []
        self._last_states: list[State2D] = []
        self.dts: list[float] = []

    # -- forward ----------------------------------------------------------
    def forward(self, state: State2D, dts) -> State2D:
        """Advance a copy of the (synced, FP64) state through dts; returns
        the final state and keeps the checkpoints.  The last segment -- the
        one the backward pass starts with -- is recorded as it runs (its
        states and tapes kept; hlld_adjoint_record_step advances the state
        exactly as the plain step does), so the backward pass recomputes
        only the earlier segments: none when checkpoint_every >= len(dts)."""
        self.dts = [float(d) for d in dts]
        s = state.clone()
        self.checkpoints = []
        self._last_states = []
        last = ((len(self.dts) - 1) // self.every) * self.every if self.dts else 0
        for i, dt in enumerate(self.dts):
            if i % self.every == 0:
                self.checkpoints.append(s.clone())
            if i >= last:
                self.record_step(s, dt, i - last)
                self._last_states.append(s.clone())
            else:
                self.stepper.step(s, dt, self.scheme)
        self.final = s
        return s

    def step_adjoint(self, s_in: State2D, s_out: State2D, dt: float, lam: State2D) -> None:
        """lam: gradient with respect to s_out -> gradient with respect to s_in (in place)."""
        st = self.stepper
        a, b, l = st._struct(s_in), st._struct(s_out), st._struct(lam)
        with torch.cuda.device(self.device):
            rc = _lib.lib().hlld_adjoint_rk_step_ct(
                ctypes.byref(st.gc), ctypes.byref(a), ctypes.byref(b), float(dt),
                _SCHEMES[self.scheme], ctypes.byref(l), self._scratch_ptr, self._scratch_bytes,
                _lib.stream_handle(self.device))
        _lib.check(rc, "hlld_adjoint_rk_step_ct")

    def _tape(self, k: int) -> int:
        while len(self._tapes) <= k:
            self._tapes.append(torch.empty(self._tape_bytes + 256, dtype=torch.uint8,
                                           device=self.device))
        return (self._tapes[k].data_ptr() + 255) // 256 * 256

    def record_step(self, s: State2D, dt: float, k: int) -> None:
        """One forward step of s in place, recording tape k."""
        st = self.stepper
        a = st._struct(s)
        with torch.cuda.device(self.device):
            rc = _lib.lib().hlld_adjoint_record_step(
                ctypes.byref(st.gc), ctypes.byref(a), float(dt), _SCHEMES[self.scheme],
                self._tape(k), self._tape_bytes, self._scratch_ptr, self._scratch_bytes,
                _lib.stream_handle(self.device))
        _lib.check(rc, "hlld_adjoint_record_step")

    def reverse_step(self, s_in: State2D, s_out: State2D, dt: float, k: int, lam: State2D) -> None:
        """lam: gradient w.r.t. s_out -> w.r.t. s_in (in place), from tape k."""
        st = self.stepper
        a, b, l = st._struct(s_in), st._struct(s_out), st._struct(lam)
        with torch.cuda.device(self.device):
            rc = _lib.lib().hlld_adjoint_reverse_step(
                ctypes.byref(st.gc), ctypes.byref(a), ctypes.byref(b), float(dt),
                _SCHEMES[self.scheme], self._tape(k), self._tape_bytes, ctypes.byref(l),
                self._scratch_ptr, self._scratch_bytes, _lib.stream_handle(self.device))
        _lib.check(rc, "hlld_adjoint_reverse_step")

    # -- backward ---------------------------------------------------------
    def backward(self, lam: State2D) -> State2D:
        """lam: gradient of the objective with respect to the final state
        (cons, faces and prims; missing prims are zero).  Returns the
        gradient with respect to the initial state's cons and faces."""
        lam = State2D(cons={k: lam.cons[k].clone() for k in EVOLVED_KEYS}, Bxf=lam.Bxf.clone(),
                      Byf=lam.Byf.clone(),
                      prims={k: (lam.prims[k].clone() if k in lam.prims else
                                 torch.zeros_like(lam.cons["D"])) for k in PRIM_KEYS})
        nsteps = len(self.dts)
        for seg in range(len(self.checkpoints) - 1, -1, -1):
            i0 = seg * self.every
            i1 = min(i0 + self.every, nsteps)
            if seg == len(self.checkpoints) - 1 and len(self._last_states) == i1 - i0:
                # recorded by the forward pass
                states = [self.checkpoints[seg]] + self._last_states
                self._last_states = []
            else:
                states = [self.checkpoints[seg].clone()]
                for i in range(i0, i1):
                    s = states[-1].clone()
                    self.record_step(s, self.dts[i], i - i0)
                    states.append(s)
            for i in range(i1 - 1, i0 - 1, -1):
                self.reverse_step(states[i - i0], states[i - i0 + 1], self.dts[i], i - i0, lam)
            del states
        return lam


class RKSteps(torch.autograd.Function):
    """Final conserved state of a CheckpointedRun as a differentiable
    function of the initial one: inputs and outputs are the six evolved cell
    variables then Bxf and Byf."""

    @staticmethod
    def forward(ctx, run: CheckpointedRun, dts, *cons_faces):
        g = run.grid
        s = State2D(cons={k: cons_faces[i].detach().clone().contiguous()
                          for i, k in enumerate(EVOLVED_KEYS)},
                    Bxf=cons_faces[6].detach().clone().contiguous(),
                    Byf=cons_faces[7].detach().clone().contiguous(), prims={})
        run.stepper.sync(s)
        out = run.forward(s, dts)
        ctx.run = run
        return tuple([out.cons[k].clone() for k in EVOLVED_KEYS] + [out.Bxf.clone(), out.Byf.clone()])

    @staticmethod
    def backward(ctx, *grads):
        run = ctx.run
        g = run.grid
        lam = _zeros_state(g, run.device)
        for i, k in enumerate(EVOLVED_KEYS):
            if grads[i] is not None:
                lam.cons[k].copy_(grads[i])
        if grads[6] is not None:
            lam.Bxf.copy_(grads[6])
        if grads[7] is not None:
            lam.Byf.copy_(grads[7])
        lam0 = run.backward(lam)
        return (None, None, *[lam0.cons[k] for k in EVOLVED_KEYS], lam0.Bxf, lam0.Byf)


def prim_to_cons_vjp(prims: dict, lam_cons: dict) -> dict:
    """(d cons / d prims)^T lam_cons per cell (hlld.py:185-217 in reverse);
    prims: the nine FP64 primitive arrays; lam_cons: any of the eight
    conserved keys (missing ones are zero).  Returns the nine lambdas."""
    ref = prims["rho"]
    n = ref.numel()
    P = [prims[k].contiguous() for k in PRIM_KEYS]
    lc = [lam_cons[k].contiguous() if k in lam_cons else None for k in CONS_KEYS]
    out = {k: torch.empty_like(ref) for k in PRIM_KEYS}
    lc_ptrs = (ctypes.c_void_p * 8)(*[t.data_ptr() if t is not None else None for t in lc])
    with torch.cuda.device(ref.device):
        rc = _lib.lib().hlld_prim_to_cons_vjp(n, _lib.ptr_array(P), lc_ptrs,
                                              _lib.ptr_array([out[k] for k in PRIM_KEYS]),
                                              _lib.stream_handle(ref.device))
    _lib.check(rc, "hlld_prim_to_cons_vjp")
    return out


# ── the magnetic-rotor gradient study ─────────────────────────────────────

def gaussian_weight(grid, centre=(0.6, 0.5), sigma=0.1):
    X, Y = grid.X, grid.Y
    return torch.exp(-((X - centre[0]) ** 2 + (Y - centre[1]) ** 2) / (2.0 * sigma ** 2))


def magnetic_objective(grid, weight, Bxf, Byf, Bz):
    """J = sum over physical cells of w |B_c|^2 / 2, B_c the cell-centred
    field (face averages for Bx, By; the cell Bz)."""
    ph = grid.phys
    Bcx = 0.5 * (Bxf[:-1, :] + Bxf[1:, :])
    Bcy = 0.5 * (Byf[:, :-1] + Byf[:, 1:])
    e = 0.5 * (Bcx ** 2 + Bcy ** 2 + Bz ** 2)
    return (weight[ph] * e[ph]).sum()


@dataclass
class RotorCase:
    n: int = 512
    steps: int = 200
    checkpoint_every: int = 20
    omega: float = 9.95
    cfl: float = 0.4


def rotor_initial(grid, eos, rho0_phys, omega):
    """Rotor primitives with the physical cells' density replaced by
    rho0_phys (ghosts from the periodic images) and angular velocity omega,
    and their conserved state, synced."""
    from .physics.initial_data2d import b_from_potential, rotor_tapered

    prims, Az = rotor_tapered(grid, eos, omega=omega)
    prims = {k: v.to(torch.float64).contiguous() for k, v in prims.items()}
    if rho0_phys is not None:
        rho = prims["rho"].clone()
        rho[grid.phys] = rho0_phys
        prims["rho"] = rho
        prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    Bxf, Byf = b_from_potential(Az, grid.dx, grid.dy)
    return prims, Bxf.contiguous(), Byf.contiguous()


def _cons_from(prims, grid):
    from .physics.driver2d import prims_to_cons_2d

    c = prims_to_cons_2d(prims, grid, "fp64")
    return {k: c[k].contiguous() for k in EVOLVED_KEYS}


def rotor_forward(run: CheckpointedRun, grid, eos, rho0_phys, omega, dts, weight):
    """J of the rotor with the given density field and omega, the dt
    sequence fixed."""
    prims, Bxf, Byf = rotor_initial(grid, eos, rho0_phys, omega)
    s = State2D(cons=_cons_from(prims, grid), Bxf=Bxf, Byf=Byf, prims={})
    run.stepper.sync(s)
    out = run.forward(s, dts)
    return float(magnetic_objective(grid, weight, out.Bxf, out.Byf, out.cons["Bz"]))


def rotor_gradients(case: RotorCase, device="cuda", dts=None):
    """Forward + adjoint of the rotor study; returns J, dJ/d rho0 (physical
    cells), dJ/d omega, the dt sequence and timings (CUDA events).  dts, when
    given, is the frozen time-step sequence (its length overrides
    case.steps); otherwise it is the CFL sequence of the unperturbed run."""
    from .physics.eos import hybrid_eos
    from .physics.grid import Grid2D

    eos = hybrid_eos(K=0.0, gamma=5.0 / 3.0, gamma_th=5.0 / 3.0)
    grid = Grid2D(0.0, 1.0, case.n, 0.0, 1.0, case.n, ng=2, device=device)
    run = CheckpointedRun(grid, eos, bc_x="periodic", bc_y="periodic", limiter="mc",
                          checkpoint_every=case.checkpoint_every)
    weight = gaussian_weight(grid)
    prims, Bxf, Byf = rotor_initial(grid, eos, None, case.omega)
    s0 = State2D(cons=_cons_from(prims, grid), Bxf=Bxf, Byf=Byf, prims={})
    run.stepper.sync(s0)
    # the dt sequence of the unperturbed run (frozen for the gradient)
    if dts is None:
        s = s0.clone()
        dts = []
        for _ in range(case.steps):
            dt = float(run.stepper.compute_dt(s, case.cfl).item())
            dts.append(dt)
            run.stepper.step(s, dt, "rk3")
    dts = [float(d) for d in dts]
    case = RotorCase(case.n, len(dts), case.checkpoint_every, case.omega, case.cfl)
    def objective_adjoint(out):
        """J of the final state and its gradient as the adjoint's seed."""
        Bxf_o = out.Bxf.clone().requires_grad_(True)
        Byf_o = out.Byf.clone().requires_grad_(True)
        Bz_o = out.cons["Bz"].clone().requires_grad_(True)
        J = magnetic_objective(grid, weight, Bxf_o, Byf_o, Bz_o)
        J.backward()
        lam = _zeros_state(grid, run.device)
        lam.Bxf.copy_(Bxf_o.grad)
        lam.Byf.copy_(Byf_o.grad)
        lam.cons["Bz"].copy_(Bz_o.grad)
        return J, lam

    # warm-up: one whole checkpoint segment forward and back, objective
    # included, loads the kernels, starts torch's autograd engine and grows
    # the allocator's pools to the segment's states, so the timed run
    # measures the steady state
    objective_adjoint(run.forward(s0, dts[:min(case.checkpoint_every, case.steps)]))
    run.backward(_zeros_state(grid, run.device))
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    out = run.forward(s0, dts)
    e1.record()
    J, lam = objective_adjoint(out)
    lam0 = run.backward(lam)
    e2.record()
    torch.cuda.synchronize()
    # initial data: cons0 = P2C(prims0(rho0, omega)); eps = p / (rho (gamma - 1))
    lp = prim_to_cons_vjp(prims, {k: lam0.cons[k] for k in EVOLVED_KEYS})
    g_rho = lp["rho"] - lp["eps"] * prims["eps"] / prims["rho"]
    ph = grid.phys
    v_over_w = {k: prims[k] / case.omega for k in ("vx", "vy")}
    g_omega = float((lp["vx"][ph] * v_over_w["vx"][ph] + lp["vy"][ph] * v_over_w["vy"][ph]).sum())
    return {"J": float(J.detach()), "grad_rho0": g_rho[ph].contiguous(), "grad_omega": g_omega,
            "dts": dts, "run": run, "grid": grid, "eos": eos, "weight": weight,
            "forward_ms": e0.elapsed_time(e1), "adjoint_ms": e1.elapsed_time(e2),
            "rho0": prims["rho"][ph].clone()}


# ── the discrete decisions a step freezes, and the finite-difference study ──

def _tape_views(run: CheckpointedRun, k: int) -> dict:
    """Views into tape k (the layout hlld_adjoint_record_step writes: two
    stage-input states, then per stage the mass fluxes, p*, HLLE-fallback
    flags and C2P roots of the sweeps, then three step diagnostics; every
    array starts on a 256-byte boundary)."""
    g = run.grid
    nxt, nyt = g.nx + 2 * g.ng, g.ny + 2 * g.ng
    nfx, nfy, nc = (nxt + 1) * nyt, nxt * (nyt + 1), nxt * nyt
    raw = run._tapes[k]
    off = run._tape(k) - raw.data_ptr()
    views = {}

    def take(name, count, dtype, size):
        nonlocal off
        views[name] = raw[off:off + count * size].view(dtype)
        off += (count * size + 255) // 256 * 256

    for x in range(2):
        for i in range(6):
            take(("X", x, "U", i), nc, torch.float64, 8)
        take(("X", x, "Bxf"), nfx, torch.float64, 8)
        take(("X", x, "Byf"), nfy, torch.float64, 8)
        for i in range(9):
            take(("X", x, "P", i), nc, torch.float64, 8)
    for st in range(3):
        take(("FxD", st), nfx, torch.float64, 8)
        take(("FyD", st), nfy, torch.float64, 8)
        take(("psx", st), nfx, torch.float64, 8)
        take(("psy", st), nfy, torch.float64, 8)
        take(("fx", st), nfx, torch.uint8, 1)
        take(("fy", st), nfy, torch.uint8, 1)
        take(("mu", st), nc, torch.float64, 8)
    views["diag"] = raw[off:off + 3 * ctypes.sizeof(_lib.StepDiag)]
    return views


def _mc_branches(P: dict, grid) -> torch.Tensor:
    """The MC limiter's branch (0: a b <= 0, no slope; 1, 2, 3: 2|a|, 2|b| or
    |a + b| / 2 is the smallest) of every interior cell for the seven
    reconstructed variables (rho, p, W v, transverse and normal B) along
    both axes (reconstruction.py:69-77, 225-236)."""
    v2 = P["vx"] ** 2 + P["vy"] ** 2 + P["vz"] ** 2
    W = 1.0 / torch.sqrt(torch.clamp(1.0 - v2, min=1e-14))
    fields = [P["rho"], P["p"], W * P["vx"], W * P["vy"], W * P["vz"], P["Bx"], P["By"], P["Bz"]]
    codes = []
    for axis in (0, 1):
        for f in fields:
            a = torch.diff(f, dim=axis)
            lo = a.narrow(axis, 0, a.shape[axis] - 1)
            hi = a.narrow(axis, 1, a.shape[axis] - 1)
            c = 0.5 * (lo + hi)
            m = torch.stack([2 * lo.abs(), 2 * hi.abs(), c.abs()]).argmin(dim=0) + 1
            codes.append(torch.where(lo * hi > 0, m, torch.zeros_like(m)).to(torch.int8).flatten())
    return torch.cat(codes)


def step_decisions(run: CheckpointedRun, s: State2D, dt: float) -> dict:
    """Advance the synced FP64 state s by one step (recording tape 0) and
    return the discrete decisions of its three stages that the adjoint
    freezes: the HLLE fallback of every x and y face, the CT upwind sign of
    every face mass flux (ct.py:96-116, with its sweep-global deadband) and
    the MC limiter branch of every cell, variable and axis."""
    g = run.grid
    nxt, nyt = g.nx + 2 * g.ng, g.ny + 2 * g.ng
    inputs = [{k: s.prims[k].clone() for k in PRIM_KEYS}]
    run.record_step(s, dt, 0)
    v = _tape_views(run, 0)
    for x in range(2):
        inputs.append({k: v[("X", x, "P", i)].view(nxt, nyt) for i, k in enumerate(PRIM_KEYS)})
    dsz = ctypes.sizeof(_lib.StepDiag)
    out = {"fallback": [], "upwind": [], "limiter": []}
    for st in range(3):
        d = _lib.StepDiag.from_buffer_copy(bytes(v["diag"][st * dsz:(st + 1) * dsz].cpu().numpy()))
        for axis, key in ((0, "FxD"), (1, "FyD")):
            F = v[(key, st)]
            scale = ctypes.c_double.from_buffer(ctypes.c_ulonglong(d.sweep[axis].fd_max_bits)).value
            sgn = torch.where(F.abs() > 1e-9 * scale, torch.sign(F), torch.zeros_like(F))
            out["upwind"].append(sgn.to(torch.int8))
        out["fallback"] += [v[("fx", st)].clone(), v[("fy", st)].clone()]
        out["limiter"].append(_mc_branches(inputs[st], g))
    return {k: torch.cat(t) for k, t in out.items()}


def decision_flips(run: CheckpointedRun, s_plus: State2D, s_minus: State2D, dts) -> dict:
    """Count the frozen decisions that differ between two runs of the same dt
    sequence (advanced in place): HLLE fallbacks, CT upwind signs and MC
    limiter branches, summed over all steps and stages."""
    flips = {"fallback": 0, "upwind": 0, "limiter": 0}
    for dt in dts:
        a = step_decisions(run, s_plus, dt)
        b = step_decisions(run, s_minus, dt)
        for k in flips:
            flips[k] += int((a[k] != b[k]).sum())
    return flips


def rotor_fd_study(case: RotorCase, directions, h=1e-6, device="cuda"):
    """Central differences of the rotor study's J along the given density
    directions (and along omega) against the adjoint's directional
    derivatives, with the decision flips between the +h and -h runs.
    directions: callables (X, Y) -> field on the physical cells, X, Y the
    cell-centre offsets from the rotor's centre.  Returns one record per
    direction (omega first)."""
    r = rotor_gradients(case, device=device)
    run, grid, eos, w, dts = r["run"], r["grid"], r["eos"], r["weight"], r["dts"]
    rho0 = r["rho0"]
    X = grid.X[grid.phys] - 0.5
    Y = grid.Y[grid.phys] - 0.5
    records = []

    def state(rho_phys, omega):
        prims, Bxf, Byf = rotor_initial(grid, eos, rho_phys, omega)
        s = State2D(cons=_cons_from(prims, grid), Bxf=Bxf, Byf=Byf, prims={})
        run.stepper.sync(s)
        return s

    cases = [("omega", None, r["grad_omega"])]
    for i, f in enumerate(directions):
        d = f(X, Y)
        cases.append((f"rho0[{i}]", d, float((r["grad_rho0"] * d).sum())))
    for name, d, adj in cases:
        if d is None:
            sp, sm = state(rho0, case.omega + h), state(rho0, case.omega - h)
        else:
            sp, sm = state(rho0 + h * d, case.omega), state(rho0 - h * d, case.omega)
        flips = decision_flips(run, sp.clone(), sm.clone(), dts)
        for dt in dts:
            run.stepper.step(sp, dt, "rk3")
            run.stepper.step(sm, dt, "rk3")
        J = lambda s: float(magnetic_objective(grid, w, s.Bxf, s.Byf, s.cons["Bz"]))
        fd = (J(sp) - J(sm)) / (2 * h)
        records.append({"direction": name, "fd": fd, "adjoint": adj, "flips": flips,
                        "rel_err": abs(fd - adj) / max(abs(fd), 1e-300)})
    return {"J": r["J"], "records": records, "n": case.n, "steps": len(dts), "h": h}
