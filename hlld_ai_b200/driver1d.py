"""The 1D shock-tube driver on the GPU, mirroring ``src/physics/driver.py``.

``rk2_step`` is the reference's Heun step (``driver.py:192-236``:
reconstruction of all nine primitives, ``flux_fn`` on the ncells + 1
physical faces, ``F[Bx] = 0``, ``U1 = U + dt L(U)``, ``U' = 0.5 (U + U1 +
dt L(U1))`` with outflow ghosts and Bx held, C2P after each stage) and
``run`` is the reference's ``run(cfg)`` time loop (``driver.py:274-412``:
``dt = compute_dt`` -- ``cfl dx`` with the default ``run.dt_speed_of_light``
-- capped at ``t_end - t``, while ``t < t_end``).  Both go through ONE
launch of the batched-tube kernel (``hlld_tubes_run`` with a driver
flavor): ``run`` advances the whole tube to ``t_end`` inside that launch.
Snapshot files and the exact-flux / harvest options of ``run`` belong to the
reference's research stack and are not reproduced.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .physics.state import CONS_KEYS, PRIM_KEYS
from .tubes import TubeBatch, TubeStates

_HUGE_CFL = 1e300


@dataclass
class Grid1D:
    """grid.py:24-47 Grid1D (cell centres x, ghosts ng per side)."""
    xmin: float
    xmax: float
    ncells: int
    ng: int = 2
    device: str = "cuda"

    def __post_init__(self):
        self.dx = (self.xmax - self.xmin) / self.ncells
        self.ntotal = self.ncells + 2 * self.ng
        i = np.arange(self.ntotal, dtype=np.float64)
        self.x = self.xmin + (i - self.ng + 0.5) * self.dx

    @property
    def phys(self) -> slice:
        return slice(self.ng, self.ng + self.ncells)


def brio_wu():
    """initial_data.py:31-45: the relativistic Brio-Wu tube (gamma = 2)."""
    pL = dict(rho=1.0, vx=0.0, vy=0.0, vz=0.0, p=1.0, eps=1.0, Bx=0.5, By=1.0, Bz=0.0)
    pR = dict(rho=0.125, vx=0.0, vy=0.0, vz=0.0, p=0.1, eps=0.8, Bx=0.5, By=-1.0, Bz=0.0)
    return pL, pR, 0.5


def generic(primL: dict, primR: dict, x_interface: float = 0.5, gamma: float | None = None):
    """initial_data.py:78-96: user left/right states; eps from the ideal-gas
    EOS when absent (eos.py eps__press_rho with K = 0)."""
    pL, pR = dict(primL), dict(primR)
    for p in (pL, pR):
        if "eps" not in p:
            if gamma is None:
                raise ValueError("generic states without eps need the EOS gamma")
            p["eps"] = 0.0 + (p["p"] - 0.0) / (p["rho"] * (gamma - 1.0))
    return pL, pR, x_interface


def init_shocktube(grid: Grid1D, primL: dict, primR: dict, x_interface: float) -> dict:
    """initial_data.py:101-127: left state where x < x_interface."""
    mask = grid.x < x_interface
    return {k: torch.tensor(np.where(mask, primL[k], primR[k]).astype(np.float64),
                            device=grid.device) for k in PRIM_KEYS}


class _OneTube:
    """A one-tube batch that holds a caller's state."""

    def __init__(self, grid: Grid1D, gamma: float, limiter: str, solver: str, flavor: str,
                 atmo_rho: float, precision: str):
        st = TubeStates(lengths=np.array([grid.ncells]), left={k: np.zeros(1) for k in PRIM_KEYS},
                        right={k: np.zeros(1) for k in PRIM_KEYS}, Bx=np.zeros(1))
        self.b = TubeBatch(st, limiter=limiter, solver=solver, scheme="rk2", precision=precision,
                           gamma=gamma, atmo_rho=atmo_rho, device=grid.device, flavor=flavor,
                           ng=grid.ng)
        if abs(float(self.b.dx[0].item()) - grid.dx) > 0:
            self.b.dx.fill_(grid.dx)

    def load(self, prims: dict, cons: dict | None):
        for k in PRIM_KEYS:
            self.b.prims[k].copy_(prims[k].reshape(-1))
        if cons is not None:
            for j, k in enumerate(CONS_KEYS):
                self.b.cons[j].copy_(cons[k].reshape(-1))

    def out(self):
        prims = {k: self.b.prims[k].clone() for k in PRIM_KEYS}
        cons = {k: self.b.cons[j].clone() for j, k in enumerate(CONS_KEYS)}
        return cons, prims


def _eos_gamma(eos) -> float:
    return eos.kernel_gamma()


def _solver_name(flux_fn) -> str:
    from .physics.hlld import solver_name

    return solver_name(flux_fn)


def rk2_step(cons: dict, prims: dict, grid: Grid1D, eos, dt, atmo_rho: float,
             bc: str = "outflow", flux_fn="hlld", limiter: str = "pcm",
             precision: str = "fp64"):
    """driver.py:192-236: one Heun step; returns new (cons, prims) device
    dicts (the inputs are not modified)."""
    if bc != "outflow":
        raise ValueError(f"bc {bc!r}: the device driver implements outflow boundaries")
    t = _OneTube(grid, _eos_gamma(eos), limiter, _solver_name(flux_fn), "driver1d_light",
                 atmo_rho, precision)
    t.load(prims, cons)
    dt = float(dt)
    # one step of exactly dt: the cfl dx bound is made larger than dt, so
    # the step is cut to t_end - 0 = dt
    t.b.launch(tend=dt, cfl=_HUGE_CFL, max_steps=1, resume=True)
    return t.out()


def run(cfg: dict, device: str = "cuda", precision: str = "fp64"):
    """driver.py:274-412 run(cfg) for the shock-tube problems: returns
    (t, grid, prims, cons) after advancing to run.t_end in one launch."""
    from .physics.eos import hybrid_eos

    gc, ec, rc = cfg["grid"], cfg["eos"], cfg["run"]
    eos = hybrid_eos(K=ec["K"], gamma=ec["gamma"], gamma_th=ec.get("gamma_th", None))
    grid = Grid1D(gc["xmin"], gc["xmax"], gc["ncells"], ng=gc.get("ng", 2), device=device)
    problem = rc.get("problem", "brio_wu")
    if problem == "generic":
        primL, primR, x_int = generic(rc["primL"], rc["primR"], rc.get("x_interface", 0.5),
                                      gamma=ec["gamma"])
    elif problem == "brio_wu":
        primL, primR, x_int = brio_wu()
    else:
        raise ValueError(f"problem {problem!r}: brio_wu and generic are provided")
    solver = rc.get("solver", "hlld")
    if solver not in ("hlld", "hlle"):
        raise ValueError(f"solver {solver!r}: the device driver implements hlld and hlle")
    prims = init_shocktube(grid, primL, primR, x_int)
    flavor = "driver1d_light" if bool(rc.get("dt_speed_of_light", True)) else "driver1d_cfl"
    tb = _OneTube(grid, _eos_gamma(eos), rc.get("limiter", "pcm"), solver, flavor,
                  rc.get("atmo_rho", 1e-10), precision)
    tb.load(prims, None)
    tb.b.launch(tend=float(rc["t_end"]), cfl=float(rc.get("cfl", 0.4)), resume=False)
    cons, prims = tb.out()
    t = float(tb.b.t_out[0].item())
    run.last_steps = int(tb.b.steps_out[0].item())
    return t, grid, prims, cons
