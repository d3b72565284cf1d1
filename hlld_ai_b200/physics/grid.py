"""Uniform grids with ghost cells, mirroring ``src/physics/grid.py``.

``Grid2D`` carries the layout the kernels use (``grid.py:146-207``): cells
``(nxt, nyt)`` x-major, ``Bxf`` ``(nxt+1, nyt)``, ``Byf`` ``(nxt, nyt+1)``,
lower-face indexing.  The boundary-condition methods are device-side tensor
copies (``grid.py:93-143``, ``:229-255``); the step applies its own BCs in
its kernels.
"""
from __future__ import annotations

import torch


def _sl(axis: int, s, ndim: int = 2) -> tuple:
    out = [slice(None)] * ndim
    out[axis] = s
    return tuple(out)


def _bc_cc_axis(v, axis, n, ng, kind, v_ref=None):
    """grid.py:93-113"""
    if kind == "outflow":
        first = v[_sl(axis, slice(ng, ng + 1))]
        last = v[_sl(axis, slice(ng + n - 1, ng + n))]
        v[_sl(axis, slice(None, ng))] = first
        v[_sl(axis, slice(ng + n, None))] = last
    elif kind == "periodic":
        v[_sl(axis, slice(None, ng))] = v[_sl(axis, slice(n, n + ng))]
        v[_sl(axis, slice(n + ng, None))] = v[_sl(axis, slice(ng, 2 * ng))]
    elif kind == "constant":
        if v_ref is None:
            raise ValueError("constant BC needs a reference array")
        v[_sl(axis, slice(None, ng))] = v_ref[_sl(axis, slice(None, ng))]
        v[_sl(axis, slice(ng + n, None))] = v_ref[_sl(axis, slice(ng + n, None))]
    else:
        raise ValueError(f"unknown boundary condition {kind!r}")


def _bc_face_normal_axis(v, axis, n, ng, kind):
    """grid.py:116-143 (the periodic seam face ng+n is set to face ng)"""
    if kind == "outflow":
        first = v[_sl(axis, slice(ng, ng + 1))]
        last = v[_sl(axis, slice(ng + n, ng + n + 1))]
        v[_sl(axis, slice(None, ng))] = first
        v[_sl(axis, slice(ng + n + 1, None))] = last
    elif kind == "periodic":
        v[_sl(axis, slice(ng + n, ng + n + 1))] = v[_sl(axis, slice(ng, ng + 1))]
        v[_sl(axis, slice(None, ng))] = v[_sl(axis, slice(n, n + ng))]
        v[_sl(axis, slice(ng + n + 1, None))] = v[_sl(axis, slice(ng + 1, ng + 1 + ng))]
    elif kind == "constant":
        pass
    else:
        raise ValueError(f"unknown boundary condition {kind!r}")


class Grid1D:
    """grid.py:23-87"""

    def __init__(self, xmin, xmax, ncells, ng=2, device="cuda"):
        self.xmin, self.xmax, self.ncells, self.ng, self.device = xmin, xmax, ncells, ng, device
        self.dx = (xmax - xmin) / ncells
        self.ntotal = ncells + 2 * ng
        i = torch.arange(self.ntotal, dtype=torch.float64, device=device)
        self.x = xmin + (i - ng + 0.5) * self.dx
        self.phys = slice(ng, ng + ncells)

    @property
    def x_phys(self):
        return self.x[self.phys]


class Grid2D:
    """grid.py:146-266"""

    def __init__(self, xmin, xmax, nx, ymin, ymax, ny, ng=2, device="cuda"):
        self.xmin, self.xmax, self.nx = xmin, xmax, nx
        self.ymin, self.ymax, self.ny = ymin, ymax, ny
        self.ng = ng
        self.device = device
        self.dx = (xmax - xmin) / nx
        self.dy = (ymax - ymin) / ny
        self.nxt = nx + 2 * ng
        self.nyt = ny + 2 * ng
        i = torch.arange(self.nxt, dtype=torch.float64, device=device)
        j = torch.arange(self.nyt, dtype=torch.float64, device=device)
        self.x = xmin + (i - ng + 0.5) * self.dx
        self.y = ymin + (j - ng + 0.5) * self.dy
        self.xf = xmin + (torch.arange(self.nxt + 1, dtype=torch.float64, device=device) - ng) * self.dx
        self.yf = ymin + (torch.arange(self.nyt + 1, dtype=torch.float64, device=device) - ng) * self.dy
        self.X = self.x.unsqueeze(1).expand(self.nxt, self.nyt)
        self.Y = self.y.unsqueeze(0).expand(self.nxt, self.nyt)
        self.phys = (slice(ng, ng + nx), slice(ng, ng + ny))
        self.phys_xf = (slice(ng, ng + nx + 1), slice(ng, ng + ny))
        self.phys_yf = (slice(ng, ng + nx), slice(ng, ng + ny + 1))

    @property
    def shape(self):
        return (self.nxt, self.nyt)

    def zeros(self):
        return torch.zeros(self.nxt, self.nyt, dtype=torch.float64, device=self.device)

    def zeros_xf(self):
        return torch.zeros(self.nxt + 1, self.nyt, dtype=torch.float64, device=self.device)

    def zeros_yf(self):
        return torch.zeros(self.nxt, self.nyt + 1, dtype=torch.float64, device=self.device)

    def zeros_corner(self):
        return torch.zeros(self.nxt + 1, self.nyt + 1, dtype=torch.float64, device=self.device)

    def apply_bc_cc(self, U, bc_x="outflow", bc_y="outflow", U_ref=None):
        for k, v in U.items():
            ref = None if U_ref is None else U_ref[k]
            _bc_cc_axis(v, 0, self.nx, self.ng, bc_x, ref)
            _bc_cc_axis(v, 1, self.ny, self.ng, bc_y, ref)
        return U

    def apply_bc_face(self, Bxf, Byf, bc_x="outflow", bc_y="outflow"):
        _bc_face_normal_axis(Bxf, 0, self.nx, self.ng, bc_x)
        _bc_cc_axis(Bxf, 1, self.ny, self.ng, bc_y)
        _bc_cc_axis(Byf, 0, self.nx, self.ng, bc_x)
        _bc_face_normal_axis(Byf, 1, self.ny, self.ng, bc_y)
        return Bxf, Byf

    def div_b(self, Bxf, Byf):
        return (Bxf[1:, :] - Bxf[:-1, :]) / self.dx + (Byf[:, 1:] - Byf[:, :-1]) / self.dy
