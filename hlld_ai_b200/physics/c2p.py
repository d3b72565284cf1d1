"""Kastaun C2P, mirroring ``src/physics/c2p.py:313-363`` conservative_to_primitive.

Runs in libhlld_b200.so (``hlld_cons_to_prim``).  The iteration limits and
tolerance are the reference's defaults, built into the kernel.
"""
from __future__ import annotations

import torch

from .. import _lib
from .state import CONS_KEYS, PRIM_KEYS


def conservative_to_primitive(cons, eos, atmo_rho: float = 1e-10, atmo_eps: float = 1e-10,
                              n_iter: int = 60, tol: float = 1e-15, return_status: bool = False,
                              n_iter_bisect: int = 200, precision: str = "fp64"):
    if (n_iter, tol, n_iter_bisect) != (60, 1e-15, 200):
        raise NotImplementedError("the kernel implements n_iter=60, tol=1e-15, n_iter_bisect=200")
    gamma = eos.kernel_gamma()
    tensors = [_lib.require_cuda(cons[k], f"cons[{k!r}]") for k in CONS_KEYS]
    shape = torch.broadcast_shapes(*[t.shape for t in tensors])
    C = [t.expand(shape).reshape(-1).contiguous() for t in tensors]
    n = C[0].numel()
    dev = C[0].device
    P = [torch.empty(n, dtype=torch.float64, device=dev) for _ in PRIM_KEYS]
    st = torch.empty(n, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = _lib.lib().hlld_cons_to_prim(n, _lib.ptr_array(C), float(gamma), float(atmo_rho),
                                          float(atmo_eps), _lib.PRECISIONS[precision],
                                          _lib.ptr_array(P), st.data_ptr(), _lib.stream_handle(dev))
    _lib.check(rc, "conservative_to_primitive")
    prims = {k: p.reshape(shape) for k, p in zip(PRIM_KEYS, P)}
    if not return_status:
        return prims
    st = st.reshape(shape)
    status = {"bracket_ok": (st & _lib.ST_BRACKET_OK) != 0,
              "converged": (st & _lib.ST_CONVERGED) != 0,
              "v_clamped": (st & _lib.ST_V_CLAMPED) != 0,
              "atmo_floored": (st & _lib.ST_ATMO) != 0}
    return prims, status
