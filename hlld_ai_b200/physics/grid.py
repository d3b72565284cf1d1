"""Grid descriptors for the B200 step.

The kernels need only a grid's sizes -- ``nx, ny, ng, dx, dy`` -- and the
device its arrays live on.  ``Stepper2D`` and ``rk_step_ct`` read nothing
else, so any object with those attributes drives them; a caller inside the
reference passes its own ``src.physics.grid.Grid2D`` unchanged.

``Grid2D`` below is this package's descriptor.  It has the reference's
array layout (``grid.py:146-207``): cells ``(nx + 2 ng, ny + 2 ng)``, x-major
with y contiguous, x faces ``(nxt + 1, nyt)`` and y faces ``(nxt, nyt + 1)``
indexed by the lower face of each cell, ghost cells ``ng`` deep on every
side.  It carries the cell-centre and face coordinates that the problem
set-ups evaluate their formulas on.  Ghost cells are filled by the step's
own kernels, so it has no boundary-condition methods.
"""
from __future__ import annotations

import torch


def _axis(lo: float, hi: float, n: int, ng: int, device):
    """Spacing, cell centres and faces of one axis, ghosts included: cell c
    (0-based, ghosts first) is centred at lo + (c - ng + 1/2) d and its lower
    face is at lo + (c - ng) d."""
    d = (hi - lo) / n
    k = torch.arange(n + 2 * ng + 1, dtype=torch.float64, device=device) - ng
    faces = lo + k * d
    centres = lo + (k[:-1] + 0.5) * d
    return d, centres, faces


class Grid1D:
    """A uniform 1D grid with ``ng`` ghost cells per side (the reference's
    ``Grid1D`` attributes: ``dx``, ``ntotal``, ``x``, ``phys``)."""

    def __init__(self, xmin, xmax, ncells, ng=2, device="cuda"):
        self.xmin, self.xmax, self.ncells, self.ng, self.device = xmin, xmax, ncells, ng, device
        self.dx, self.x, _ = _axis(xmin, xmax, ncells, ng, device)
        self.ntotal = ncells + 2 * ng
        self.phys = slice(ng, ng + ncells)

    @property
    def x_phys(self):
        return self.x[self.phys]


class Grid2D:
    """A uniform 2D grid on [xmin, xmax] x [ymin, ymax] with nx x ny cells."""

    def __init__(self, xmin, xmax, nx, ymin, ymax, ny, ng=2, device="cuda"):
        self.xmin, self.xmax, self.ymin, self.ymax = xmin, xmax, ymin, ymax
        self.nx, self.ny, self.ng, self.device = nx, ny, ng, device
        self.nxt, self.nyt = nx + 2 * ng, ny + 2 * ng
        self.dx, self.x, self.xf = _axis(xmin, xmax, nx, ng, device)
        self.dy, self.y, self.yf = _axis(ymin, ymax, ny, ng, device)
        # cell-centre coordinates on the cell array (views, no copies)
        self.X = self.x[:, None].expand(self.nxt, self.nyt)
        self.Y = self.y[None, :].expand(self.nxt, self.nyt)
        inner = lambda n: slice(ng, ng + n)
        self.phys = (inner(nx), inner(ny))

    @property
    def shape(self):
        return (self.nxt, self.nyt)

    def corner_mesh(self):
        """x and y of every cell corner, arrays of shape (nxt + 1, nyt + 1)."""
        return torch.meshgrid(self.xf, self.yf, indexing="ij")

    def div_b(self, Bxf, Byf):
        """Cell divergence of the staggered field (ct.py:196-199)."""
        return torch.diff(Bxf, dim=0) / self.dx + torch.diff(Byf, dim=1) / self.dy
