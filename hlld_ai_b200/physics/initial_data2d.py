"""2D initial conditions of the benchmark and test problems.

Each problem is a function ``(grid, eos) -> (prims, Az)``: the nine cell
primitives on the whole ghost-inclusive cell array and the vector potential
Az at the cell corners.  The staggered field is Az's discrete curl
(``b_from_potential``), so div B vanishes to round-off at t = 0, which is
how the reference initialises its CT runs (``initial_data2d.py:24-29``).
These are host-side set-ups, not part of the hot path.

Problems:
  * ``rotor``: the magnetic rotor of the reference's ``run_2d.py`` -- a
    dense disk (r <= 0.1, rho 10, rigid rotation at omega 9.95) in a medium
    at rest (rho 1), p = 1 and B = (1, 0, 0) everywhere, on [-0.5, 0.5]^2
    with outflow boundaries;
  * ``rotor_tapered``: the same rotor centred on the periodic unit square
    with density and velocity tapered linearly over 0.1 < r < 0.115 (the
    benchmark rotor);
  * ``orszag_tang``: v = v_max / sqrt2 (-sin 2 pi y, sin 2 pi x, 0),
    B = B0 (-sin 2 pi y, sin 4 pi x, 0), uniform rho and p, periodic;
  * ``vortex``: ``orszag_tang`` with v_max = 0.99, B0 = rho = p = 1,
    gamma = 4/3 (the precision-study vortex);
  * ``riemann2d``: the four-quadrant problem of the reference with a uniform
    in-plane field B0 (cos a, sin a, 0).
"""
from __future__ import annotations

import math

import torch

from .eos import hybrid_eos
from .grid import Grid2D
from .state import EVOLVED_KEYS, State2D


def b_from_potential(Az, dx, dy):
    """Face fields of a corner potential: Bx = d Az / dy on x faces,
    By = -d Az / dx on y faces (one-cell differences)."""
    return torch.diff(Az, dim=1) / dy, -torch.diff(Az, dim=0) / dx


def _field(grid, value):
    return torch.full(grid.shape, float(value), dtype=torch.float64, device=grid.device)


def _finish(grid, eos, rho, p, v, B):
    """The nine primitives from density, pressure, velocity and field."""
    prims = {"rho": rho, "p": p, "vx": v[0], "vy": v[1], "vz": v[2],
             "Bx": B[0], "By": B[1], "Bz": B[2]}
    for k, t in prims.items():
        if not isinstance(t, torch.Tensor):
            prims[k] = _field(grid, t)
    prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
    return prims


def magnetic_rotor(grid, eos, r0=0.1, rho_in=10.0, rho_out=1.0, omega=9.95, press=1.0, B0=1.0):
    """The rotor of the reference's ``run_2d.py`` problem table, on a grid
    centred on the origin: a sharp disk edge at r0 (cells whose centres lie
    within r0, allowing 16 ulp for the radius of a centre exactly on it)."""
    X, Y = grid.X, grid.Y
    inside = X * X + Y * Y <= r0 * r0 * (1.0 + 16.0 * 2.0 ** -52)
    zero = _field(grid, 0.0)
    rho = torch.where(inside, _field(grid, rho_in), _field(grid, rho_out))
    v = (torch.where(inside, -omega * Y, zero), torch.where(inside, omega * X, zero), zero.clone())
    _, yc = grid.corner_mesh()
    return _finish(grid, eos, rho, press, v, (B0, 0.0, 0.0)), B0 * yc


def rotor_tapered(grid, eos, r0=0.1, r1=0.115, rho_in=10.0, rho_out=1.0, omega=9.95,
                  press=1.0, B0=1.0, centre=(0.5, 0.5)):
    """The benchmark rotor: the disk r <= r0 at `centre`, its density and
    angular velocity falling linearly to the ambient values over r0 < r < r1."""
    X = grid.X - centre[0]
    Y = grid.Y - centre[1]
    f = ((r1 - torch.sqrt(X * X + Y * Y)) / (r1 - r0)).clamp(0.0, 1.0)
    rho = rho_out + (rho_in - rho_out) * f
    v = (-omega * Y * f, omega * X * f, _field(grid, 0.0))
    _, yc = grid.corner_mesh()
    return _finish(grid, eos, rho, press, v, (B0, 0.0, 0.0)), B0 * yc


def riemann2d(grid, eos, B0=0.5, angle_deg=45.0, angle_z_deg=0.0):
    """Four constant quadrants on [-0.5, 0.5]^2, (rho, p, vx, vy) =
    top left (0.1, 1, 0.99, 0), top right (0.1, 0.01, 0, 0), bottom left
    (0.5, 1, 0, 0), bottom right (0.1, 1, 0, 0.99), in the uniform field
    B0 (cos a cos b, sin a cos b, sin b); at a = 45 degrees the in-plane
    components are set equal, so the problem keeps its x <-> y symmetry."""
    a, b = math.radians(angle_deg), math.radians(angle_z_deg)
    ca = math.cos(a)
    sa = ca if angle_deg == 45.0 else math.sin(a)
    bx, by, bz = B0 * ca * math.cos(b), B0 * sa * math.cos(b), B0 * math.sin(b)
    east, north = grid.X > 0.0, grid.Y > 0.0

    def quadrants(nw, ne, sw, se):
        row_n = torch.where(east, _field(grid, ne), _field(grid, nw))
        row_s = torch.where(east, _field(grid, se), _field(grid, sw))
        return torch.where(north, row_n, row_s)

    prims = _finish(grid, eos, quadrants(0.1, 0.1, 0.5, 0.1), quadrants(1.0, 0.01, 1.0, 1.0),
                    (quadrants(0.99, 0.0, 0.0, 0.0), quadrants(0.0, 0.0, 0.0, 0.99), 0.0),
                    (bx, by, bz))
    xc, yc = grid.corner_mesh()
    return prims, bx * yc - by * xc


def orszag_tang(grid, eos, v_max=0.99, B0=None, press=None, rho=None):
    """The relativistic Orszag-Tang vortex on the periodic unit square.  The
    defaults B0 = 1/sqrt(4 pi), rho = 25/(36 pi), p = 5/(12 pi) are the
    classical vortex's; the field's potential is
    Az = B0 (cos 4 pi x / (4 pi) + cos 2 pi y / (2 pi))."""
    B0 = 1.0 / math.sqrt(4.0 * math.pi) if B0 is None else B0
    rho = 25.0 / (36.0 * math.pi) if rho is None else rho
    press = 5.0 / (12.0 * math.pi) if press is None else press
    k = 2.0 * math.pi
    sx, sy = torch.sin(k * grid.X), torch.sin(k * grid.Y)
    amp = v_max / math.sqrt(2.0)
    prims = _finish(grid, eos, rho, press, (-amp * sy, amp * sx, 0.0),
                    (-B0 * sy, B0 * torch.sin(2.0 * k * grid.X), 0.0))
    xc, yc = grid.corner_mesh()
    Az = B0 * (torch.cos(2.0 * k * xc) / (2.0 * k) + torch.cos(k * yc) / k)
    return prims, Az


def relativistic_vortex(grid, eos):
    """The precision-study vortex (use gamma = 4/3)."""
    return orszag_tang(grid, eos, v_max=0.99, B0=1.0, press=1.0, rho=1.0)


# problem -> domain, adiabatic index, end time, boundaries (x, y), builder;
# the first three are the reference run_2d.py's set-ups
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
    """(grid, eos, prims, Az, spec) of a named problem on an n x n grid."""
    spec = PROBLEMS[problem]
    lo, hi = spec["box"]
    g = Grid2D(lo, hi, n, lo, hi, n, ng=ng, device=device)
    eos = hybrid_eos(K=0.0, gamma=spec["gamma"], gamma_th=spec["gamma"])
    prims, Az = spec["build"](g, eos)
    return g, eos, prims, Az, spec


def setup_problem(problem: str, n: int, *, limiter: str = "mc", device="cuda",
                  precision: str = "fp64"):
    """A synced GPU State2D of a named problem: (grid, eos, state, spec).

    The primitives and the potential are evaluated on the CPU, the staggered
    field and the conserved variables are formed on the device (in FP64 for
    every precision), then stored in the precision's types and synced, so
    that the primitives the step starts from are the C2P of its own state."""
    from ..physics.reconstruction import ghosts_needed
    from .driver2d import prims_to_cons_2d, sync_state

    ng = ghosts_needed(limiter)
    gc, eos, prims, Az, spec = initial_prims(problem, n, ng, device="cpu")
    g = Grid2D(gc.xmin, gc.xmax, n, gc.ymin, gc.ymax, n, ng=ng, device=device)
    prims = {k: v.contiguous().to(device) for k, v in prims.items()}
    Bxf, Byf = b_from_potential(Az.to(device), g.dx, g.dy)
    c = prims_to_cons_2d(prims, g, "fp64_exact" if precision == "fp64_exact" else "fp64")
    if precision in ("mixed", "fp32"):
        prims = {k: v.to(torch.float32).contiguous() for k, v in prims.items()}
    if precision == "fp32":
        c = {k: v.to(torch.float32) for k, v in c.items()}
        Bxf, Byf = Bxf.to(torch.float32), Byf.to(torch.float32)
    st = State2D(cons={k: c[k].contiguous() for k in EVOLVED_KEYS}, Bxf=Bxf.contiguous(),
                 Byf=Byf.contiguous(), prims=prims)
    st = sync_state(st, g, eos, *spec["bc"], precision=precision, limiter=limiter)
    return g, eos, st, spec
