"""2D initial conditions, mirroring ``src/physics/initial_data2d.py``.

Every problem returns cell primitives and a corner vector potential ``Az``;
the staggered field is its discrete curl (``initial_data2d.py:24-29``), so
div B is zero to round-off at t = 0.  Tensor arithmetic follows the
reference on the grid's device (host-side set-up, not the hot path).

Beyond the reference's problems:
  * ``rotor_tapered``: the magnetic rotor on the periodic unit square with a
    linear density/velocity taper on 0.1 < r < 0.115 (the benchmark rotor);
  * ``relativistic_vortex``: ``orszag_tang(v_max=0.99, B0=1, press=1, rho=1)``
    with gamma = 4/3 (the precision-study vortex).
"""
from __future__ import annotations

import math

import torch

from .eos import hybrid_eos
from .grid import Grid2D
from .state import EVOLVED_KEYS, State2D


def b_from_potential(Az, dx, dy):
    """initial_data2d.py:24-29"""
    Bxf = (Az[:, 1:] - Az[:, :-1]) / dy
    Byf = -(Az[1:, :] - Az[:-1, :]) / dx
    return Bxf, Byf


def _corner_mesh(grid):
    XF = grid.xf.unsqueeze(1).expand(grid.nxt + 1, grid.nyt + 1)
    YF = grid.yf.unsqueeze(0).expand(grid.nxt + 1, grid.nyt + 1)
    return XF, YF


def magnetic_rotor(grid, eos, r0=0.1, rho_in=10.0, rho_out=1.0, omega=9.95, press=1.0, B0=1.0):
    """initial_data2d.py:88-125: sharp-edged rotor on [-0.5, 0.5]^2."""
    X, Y = grid.X, grid.Y
    r2 = X**2 + Y**2
    inside = r2 <= r0 * r0 * (1.0 + 16 * torch.finfo(torch.float64).eps)
    zeros = torch.zeros(grid.shape, dtype=torch.float64, device=grid.device)
    prims = {
        "rho": torch.where(inside, torch.full_like(zeros, rho_in), torch.full_like(zeros, rho_out)),
        "p": torch.full_like(zeros, press),
        "vx": torch.where(inside, -omega * Y, zeros),
        "vy": torch.where(inside, omega * X, zeros),
        "vz": zeros.clone(),
        "Bx": torch.full_like(zeros, B0),
        "By": zeros.clone(),
        "Bz": zeros.clone(),
    }
    prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    _, YF = _corner_mesh(grid)
    return prims, B0 * YF


def rotor_tapered(grid, eos, r0=0.1, r1=0.115, rho_in=10.0, rho_out=1.0, omega=9.95,
                  press=1.0, B0=1.0, centre=(0.5, 0.5)):
    """Benchmark rotor: disk r <= r0 (rho_in, rigid rotation omega) inside an
    ambient medium (rho_out, at rest), both tapered linearly in f = (r1 - r) /
    (r1 - r0) on r0 < r < r1; uniform p and B = (B0, 0, 0) (Az = B0 y)."""
    X = grid.X - centre[0]
    Y = grid.Y - centre[1]
    r = torch.sqrt(X**2 + Y**2)
    f = torch.clamp((r1 - r) / (r1 - r0), min=0.0, max=1.0)
    zeros = torch.zeros(grid.shape, dtype=torch.float64, device=grid.device)
    prims = {
        "rho": rho_out + (rho_in - rho_out) * f,
        "p": torch.full_like(zeros, press),
        "vx": -omega * Y * f,
        "vy": omega * X * f,
        "vz": zeros.clone(),
        "Bx": torch.full_like(zeros, B0),
        "By": zeros.clone(),
        "Bz": zeros.clone(),
    }
    prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    _, YF = _corner_mesh(grid)
    return prims, B0 * YF


def riemann2d(grid, eos, B0=0.5, angle_deg=45.0, angle_z_deg=0.0):
    """initial_data2d.py:128-191: four-quadrant problem with a uniform field."""
    X, Y = grid.X, grid.Y
    zeros = torch.zeros(grid.shape, dtype=torch.float64, device=grid.device)
    right, top = X > 0.0, Y > 0.0
    full = lambda v: torch.full_like(zeros, float(v))

    def pick(tl, tr, bl, br):
        return torch.where(top, torch.where(right, full(tr), full(tl)),
                           torch.where(right, full(br), full(bl)))

    a, b = math.radians(angle_deg), math.radians(angle_z_deg)
    ca, sa = math.cos(a), math.sin(a)
    if angle_deg == 45.0:
        sa = ca
    bx, by, bz = B0 * ca * math.cos(b), B0 * sa * math.cos(b), B0 * math.sin(b)
    prims = {"rho": pick(0.1, 0.1, 0.5, 0.1), "p": pick(1.0, 0.01, 1.0, 1.0),
             "vx": pick(0.99, 0.0, 0.0, 0.0), "vy": pick(0.0, 0.0, 0.0, 0.99),
             "vz": zeros.clone(), "Bx": full(bx), "By": full(by), "Bz": full(bz)}
    prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    XF, YF = _corner_mesh(grid)
    return prims, bx * YF - by * XF


def orszag_tang(grid, eos, v_max=0.99, B0=None, press=None, rho=None):
    """initial_data2d.py:194-253"""
    if B0 is None:
        B0 = 1.0 / math.sqrt(4.0 * math.pi)
    if rho is None:
        rho = 25.0 / (36.0 * math.pi)
    if press is None:
        press = 5.0 / (12.0 * math.pi)
    amp = v_max / math.sqrt(2.0)
    X, Y = grid.X, grid.Y
    zeros = torch.zeros(grid.shape, dtype=torch.float64, device=grid.device)
    prims = {"rho": torch.full_like(zeros, rho), "p": torch.full_like(zeros, press),
             "vx": -amp * torch.sin(2 * math.pi * Y), "vy": amp * torch.sin(2 * math.pi * X),
             "vz": zeros.clone(), "Bx": -B0 * torch.sin(2 * math.pi * Y),
             "By": B0 * torch.sin(4 * math.pi * X), "Bz": zeros.clone()}
    prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    XF, YF = _corner_mesh(grid)
    Az = B0 * (torch.cos(4 * math.pi * XF) / (4 * math.pi) + torch.cos(2 * math.pi * YF) / (2 * math.pi))
    return prims, Az


def relativistic_vortex(grid, eos):
    """Precision-study vortex: v = 0.99/sqrt2 (-sin 2pi y, sin 2pi x, 0),
    B = (-sin 2pi y, sin 4pi x, 0), rho = p = 1 (use gamma = 4/3)."""
    return orszag_tang(grid, eos, v_max=0.99, B0=1.0, press=1.0, rho=1.0)


# problem -> (domain, gamma, t_end, (bc_x, bc_y), builder); the first four
# follow scripts/run_2d.py:30-41
PROBLEMS = {
    "rotor": dict(box=(-0.5, 0.5), gamma=5.0 / 3.0, tend=0.4, bc=("outflow", "outflow"),
                  build=magnetic_rotor),
    "orszag_tang": dict(box=(0.0, 1.0), gamma=4.0 / 3.0, tend=1.0, bc=("periodic", "periodic"),
                        build=orszag_tang),
    "riemann2d": dict(box=(-0.5, 0.5), gamma=5.0 / 3.0, tend=0.4, bc=("outflow", "outflow"),
                      build=riemann2d),
    "rotor_tapered": dict(box=(0.0, 1.0), gamma=5.0 / 3.0, tend=0.4, bc=("periodic", "periodic"),
                          build=rotor_tapered),
    "vortex": dict(box=(0.0, 1.0), gamma=4.0 / 3.0, tend=0.5, bc=("periodic", "periodic"),
                   build=relativistic_vortex),
}


def initial_prims(problem: str, n: int, ng: int = 2, device="cpu"):
    """(grid, eos, prims, Az, spec) of a named problem, built on `device`."""
    spec = PROBLEMS[problem]
    lo, hi = spec["box"]
    g = Grid2D(lo, hi, n, lo, hi, n, ng=ng, device=device)
    eos = hybrid_eos(K=0.0, gamma=spec["gamma"], gamma_th=spec["gamma"])
    prims, Az = spec["build"](g, eos)
    return g, eos, prims, Az, spec


def setup_problem(problem: str, n: int, *, limiter: str = "mc", device="cuda",
                  precision: str = "fp64"):
    """A synced GPU State2D of a named problem: (grid, eos, state, spec).

    Initial data are built on the CPU with the reference's tensor formulas,
    moved to the device, converted to conserved variables and synced there
    (scripts/run_2d.py:216-231)."""
    from ..physics.reconstruction import ghosts_needed
    from .driver2d import prims_to_cons_2d, sync_state

    ng = ghosts_needed(limiter)
    gc, eos, prims, Az, spec = initial_prims(problem, n, ng, device="cpu")
    g = Grid2D(gc.xmin, gc.xmax, n, gc.ymin, gc.ymax, n, ng=ng, device=device)
    prims = {k: v.contiguous().to(device) for k, v in prims.items()}
    Bxf, Byf = b_from_potential(Az.to(device), g.dx, g.dy)
    # conserved variables from the FP64 initial primitives in every precision
    c = prims_to_cons_2d(prims, g, "fp64_exact" if precision == "fp64_exact" else "fp64")
    if precision == "mixed":
        prims = {k: v.to(torch.float32).contiguous() for k, v in prims.items()}
    st = State2D(cons={k: c[k].contiguous() for k in EVOLVED_KEYS}, Bxf=Bxf.contiguous(),
                 Byf=Byf.contiguous(), prims=prims)
    st = sync_state(st, g, eos, *spec["bc"], precision=precision, limiter=limiter)
    return g, eos, st, spec
