"""Riemann-solver plugins, mirroring ``src/physics/hlld.py``'s flux_fn contract.

``flux_fn(sL, sR, eos, idir) -> (F, U, p_star)``: sL/sR are dicts of
primitive tensors (rho, vx, vy, vz, p, eps, Bx, By, Bz), F/U dicts of the
eight conserved components, p_star < 0 marks an HLLE-fallback face
(``hlld.py:1531``).  The arithmetic runs in the CUDA kernels of
libhlld_b200.so (``hlld_riemann_faces``); inputs must be float64 CUDA
tensors.  ``hlld_flux`` refreshes the module-global ``LAST_DIAG`` as the
reference does (``hlld.py:1098``, ``:1516-1529``); ``hlle_flux`` and
``hllc_flux`` leave it alone, as the reference's do.
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib
from .state import CONS_KEYS, PRIM_KEYS

LAST_DIAG: dict = {}
_PSTAR_TOL = 1.0e-10  # hlld.py:1080 (built into the kernel)
_PSTAR_METHOD = "secant"  # hlld.py:1088 (the only method the kernel implements)


def _flat_inputs(sL, sR):
    tensors = [sL[k] for k in PRIM_KEYS] + [sR[k] for k in PRIM_KEYS]
    for k, t in zip(PRIM_KEYS * 2, tensors):
        _lib.require_cuda(t, f"state[{k!r}]")
    shape = torch.broadcast_shapes(*[t.shape for t in tensors])
    flat = [t.expand(shape).reshape(-1).contiguous() for t in tensors]
    return shape, flat[:9], flat[9:]


def riemann(sL, sR, eos, idir: int, solver: str, precision: str = "fp64", want_u: bool = True):
    """Run the solver; returns (F, U, p_star, err, iters, flags, diag)."""
    if idir not in (0, 1, 2):
        raise ValueError("idir must be 0, 1 or 2")
    gamma = eos.kernel_gamma()
    shape, L, R = _flat_inputs(sL, sR)
    n = L[0].numel()
    dev = L[0].device
    F = [torch.empty(n, dtype=torch.float64, device=dev) for _ in CONS_KEYS]
    U = [torch.empty(n, dtype=torch.float64, device=dev) for _ in CONS_KEYS] if want_u else None
    ps = torch.empty(n, dtype=torch.float64, device=dev)
    err = torch.empty(n, dtype=torch.int32, device=dev)
    it = torch.empty(n, dtype=torch.int32, device=dev)
    fl = torch.empty(n, dtype=torch.uint8, device=dev)
    diag = torch.zeros(ctypes.sizeof(_lib.FluxDiag), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = _lib.lib().hlld_riemann_faces(
            n, _lib.ptr_array(L), _lib.ptr_array(R), idir, _lib.SOLVERS[solver], gamma,
            _lib.PRECISIONS[precision], _lib.ptr_array(F),
            _lib.ptr_array(U) if want_u else None, ps.data_ptr(), err.data_ptr(),
            it.data_ptr(), fl.data_ptr(), diag.data_ptr(), _lib.stream_handle(dev))
    _lib.check(rc, f"{solver}_flux")
    Fd = {k: f.reshape(shape) for k, f in zip(CONS_KEYS, F)}
    Ud = {k: u.reshape(shape) for k, u in zip(CONS_KEYS, U)} if want_u else None
    return Fd, Ud, ps.reshape(shape), err.reshape(shape), it.reshape(shape), fl.reshape(shape), diag


def flux_diag_dict(raw: torch.Tensor, solver: str, idir: int) -> dict:
    """LAST_DIAG-style dict from a device FluxDiag buffer (one D2H copy)."""
    return flux_diag_from_struct(_lib.FluxDiag.from_buffer_copy(bytes(raw.cpu().numpy())),
                                 solver, idir)


def flux_diag_from_struct(d, solver: str, idir: int) -> dict:
    """hlld.py:1516-1529 LAST_DIAG keys from FluxDiag counters."""
    n = int(d.n_faces)
    return dict(solver=solver, idir=idir, n_interfaces=n,
                n_not_converged=int(d.n_not_converged),
                n_wave_order_bad=int(d.n_wave_order_bad), n_bn_zero=int(d.n_bn_zero),
                n_hlle_fallback=int(d.n_failed),
                frac_hlle_fallback=float(d.n_failed) / max(n, 1),
                mean_iters=(float(d.iters_sum_conv) / float(d.n_conv) if d.n_conv else float("nan")),
                pstar_method=_PSTAR_METHOD, pstar_cost=None, max_iters=int(d.max_iters))


def hlld_flux(sL, sR, eos, idir: int = 0, lo_fac: float = 0.1, hi_fac: float = 10,
              precision: str = "fp64"):
    """hlld.py:1202-1543.  lo_fac/hi_fac are accepted and unused, as in the
    reference (its bracket comes from p0 / p_hll, hlld.py:1300-1301)."""
    F, U, ps, err, it, fl, diag = riemann(sL, sR, eos, idir, "hlld", precision)
    LAST_DIAG.update(flux_diag_dict(diag, "hlld", idir))
    return F, U, ps


def hlle_flux(sL, sR, eos, idir: int = 0, precision: str = "fp64"):
    """hlld.py:1005-1044"""
    F, U, ps, *_ = riemann(sL, sR, eos, idir, "hlle", precision)
    return F, U, ps


def hllc_flux(sL, sR, eos, idir: int = 0, precision: str = "fp64"):
    """hlld.py:1549-1765; the third output is p_hll, as in the reference."""
    F, U, ps, *_ = riemann(sL, sR, eos, idir, "hllc", precision)
    return F, U, ps


def primitive_to_conserved(prim: dict, precision: str = "fp64") -> dict:
    """hlld.py:185-217"""
    tensors = [_lib.require_cuda(prim[k], f"prim[{k!r}]") for k in PRIM_KEYS]
    shape = torch.broadcast_shapes(*[t.shape for t in tensors])
    P = [t.expand(shape).reshape(-1).contiguous() for t in tensors]
    n = P[0].numel()
    C = [torch.empty(n, dtype=torch.float64, device=P[0].device) for _ in CONS_KEYS]
    with torch.cuda.device(P[0].device):
        rc = _lib.lib().hlld_prim_to_cons(n, _lib.ptr_array(P), _lib.PRECISIONS[precision],
                                          _lib.ptr_array(C), _lib.stream_handle(P[0].device))
    _lib.check(rc, "primitive_to_conserved")
    return {k: c.reshape(shape) for k, c in zip(CONS_KEYS, C)}


SOLVERS = {"hlld": hlld_flux, "hlle": hlle_flux, "hllc": hllc_flux}


def solver_name(flux_fn) -> str:
    """Map a flux_fn (ours, or the reference's by name) to a kernel solver."""
    if isinstance(flux_fn, str):
        name = flux_fn
    else:
        name = getattr(flux_fn, "__name__", "")
        name = {"hlld_flux": "hlld", "hlle_flux": "hlle", "hllc_flux": "hllc"}.get(name, name)
    if name not in ("hlld", "hlle", "hllc"):
        raise NotImplementedError(f"flux_fn {name!r}: the B200 step implements hlld, hlle "
                                  "and hllc")
    return name
