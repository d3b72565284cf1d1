"""CPU oracle for the SRMHD finite-volume step -- TEST INFRASTRUCTURE ONLY.

Python (numpy, ctypes) face of ``srmhd_oracle.c``, a scalar C restatement of
kemi2805/HLLD-AI's FP64 hot path.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline legs may import this module, and only as the
checker or as the timed CPU baseline; the product package never does.

Arrays are numpy float64, dicts keyed like the reference's state dicts
(``src/physics/hlld.py:8-12``, ``src/physics/state.py:41``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

PRIM_KEYS = ("rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz")
CONS_KEYS = ("D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz")
EVOLVED_KEYS = ("D", "Sx", "Sy", "Sz", "tau", "Bz")
LIMITERS = {"pcm": 0, "mc": 1, "minmod": 2, "weno5z": 3, "mp5": 4, "mp7": 5}
SOLVERS = {"hlle": 0, "hlld": 1, "hllc": 2}
BCS = {"outflow": 0, "periodic": 1}

ST_BRACKET_OK, ST_CONVERGED, ST_V_CLAMPED, ST_ATMO, ST_BISECTED = 1, 2, 4, 8, 16
RF_WAVE_ORDER_BAD, RF_BN_ZERO, RF_FAILED = 1, 2, 4

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    """Compile liboracle.so in place (make); returns its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "srmhd_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        _LIB = ctypes.CDLL(path)
        _LIB.orc_compute_dt_2d.restype = ctypes.c_double
        _LIB.orc_rk_step_ct.restype = ctypes.c_int
    return _LIB


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def prim_to_cons(prim: dict) -> dict:
    """``src/physics/hlld.py:185-217`` primitive_to_conserved."""
    P = [_f64(prim[k]).ravel() for k in PRIM_KEYS]
    n = P[0].size
    C = [np.empty(n) for _ in CONS_KEYS]
    lib().orc_prim_to_cons(ctypes.c_int64(n), _ptrs(P), _ptrs(C))
    shape = np.shape(prim["rho"])
    return {k: c.reshape(shape) for k, c in zip(CONS_KEYS, C)}


def cons_to_prim(cons: dict, gamma: float, atmo_rho: float = 1e-10, atmo_eps: float = 1e-10):
    """``src/physics/c2p.py:313-363``; returns (prims, status bits)."""
    C = [_f64(cons[k]).ravel() for k in CONS_KEYS]
    n = C[0].size
    P = [np.empty(n) for _ in PRIM_KEYS]
    st = np.zeros(n, dtype=np.uint8)
    lib().orc_cons_to_prim(ctypes.c_int64(n), _ptrs(C), ctypes.c_double(gamma),
                           ctypes.c_double(atmo_rho), ctypes.c_double(atmo_eps), _ptrs(P), _p(st))
    shape = np.shape(cons["D"])
    return {k: p.reshape(shape) for k, p in zip(PRIM_KEYS, P)}, st.reshape(shape)


def riemann(sL: dict, sR: dict, idir: int, solver: str, gamma: float):
    """``hlld.py:1005-1044`` hlle_flux / ``hlld.py:1202-1543`` hlld_flux.

    Returns (F, U, p_star, err, iters, flags)."""
    L = [_f64(sL[k]).ravel() for k in PRIM_KEYS]
    R = [_f64(sR[k]).ravel() for k in PRIM_KEYS]
    n = L[0].size
    F = [np.empty(n) for _ in CONS_KEYS]
    U = [np.empty(n) for _ in CONS_KEYS]
    ps = np.empty(n)
    err = np.zeros(n, dtype=np.int32)
    it = np.zeros(n, dtype=np.int32)
    fl = np.zeros(n, dtype=np.uint8)
    lib().orc_riemann(ctypes.c_int64(n), _ptrs(L), _ptrs(R), ctypes.c_int(idir),
                      ctypes.c_int(SOLVERS[solver]), ctypes.c_double(gamma), _ptrs(F), _ptrs(U),
                      _p(ps), _p(err), _p(it), _p(fl))
    return (dict(zip(CONS_KEYS, F)), dict(zip(CONS_KEYS, U)), ps, err, it, fl)


def reconstruct(q: np.ndarray, axis: int, limiter: str):
    """``reconstruction.py:239-264`` reconstruct() of a 1D or 2D array."""
    q = _f64(q)
    q2 = q.reshape(q.shape[0], -1) if q.ndim == 1 else q
    n0, n1 = q2.shape
    shp = (n0 + 1, n1) if axis == 0 else (n0, n1 + 1)
    QL, QR = np.empty(shp), np.empty(shp)
    lib().orc_reconstruct(_p(q2), ctypes.c_int(n0), ctypes.c_int(n1), ctypes.c_int(axis),
                          ctypes.c_int(LIMITERS[limiter]), _p(QL), _p(QR))
    if q.ndim == 1:
        return QL.ravel(), QR.ravel()
    return QL, QR


def reconstruct_prims(prims: dict, axis: int, gamma: float, limiter: str = "mc",
                      vel_var: str = "Wv"):
    """``reconstruction.py:272-338`` reconstruct_prims on (n0, n1) arrays."""
    P = [_f64(prims[k]) for k in PRIM_KEYS]
    n0, n1 = P[0].shape
    shp = (n0 + 1, n1) if axis == 0 else (n0, n1 + 1)
    L = [np.empty(shp) for _ in PRIM_KEYS]
    R = [np.empty(shp) for _ in PRIM_KEYS]
    lib().orc_reconstruct_prims(_ptrs(P), ctypes.c_int(n0), ctypes.c_int(n1), ctypes.c_int(axis),
                                ctypes.c_int(LIMITERS[limiter]), ctypes.c_int(vel_var == "Wv"),
                                ctypes.c_double(gamma), _ptrs(L), _ptrs(R))
    return dict(zip(PRIM_KEYS, L)), dict(zip(PRIM_KEYS, R))


def corner_emf(Ec, Efx, Efy, Fx_rho, Fy_rho, upwind: bool = True) -> np.ndarray:
    """``ct.py:119-177`` corner_emf."""
    Ec, Efx, Efy, Fx_rho, Fy_rho = (_f64(a) for a in (Ec, Efx, Efy, Fx_rho, Fy_rho))
    n0, n1 = Ec.shape
    Ez = np.empty((n0 + 1, n1 + 1))
    lib().orc_corner_emf(ctypes.c_int(n0), ctypes.c_int(n1), _p(Ec), _p(Efx), _p(Efy),
                         _p(Fx_rho), _p(Fy_rho), ctypes.c_int(int(upwind)), _p(Ez))
    return Ez


class _Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("ng", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("bc_x", ctypes.c_int), ("bc_y", ctypes.c_int),
                ("limiter", ctypes.c_int), ("solver", ctypes.c_int),
                ("gamma", ctypes.c_double), ("atmo_rho", ctypes.c_double),
                ("upwind", ctypes.c_int), ("emf_mode", ctypes.c_int)]


EMF_MODES = {"solver": 0, "hll": 1}


class _Diag(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64 * 2) for name in
                ("n_faces", "n_not_converged", "n_wave_order_bad", "n_bn_zero", "n_failed",
                 "iters_sum_conv", "n_conv", "max_iters")] + [("fd_max", ctypes.c_double * 2)]


@dataclass
class Grid2DSpec:
    """The pieces of ``grid.py:146-207`` Grid2D the stepper needs."""
    nx: int
    ny: int
    ng: int
    dx: float
    dy: float
    bc_x: str = "outflow"
    bc_y: str = "outflow"
    limiter: str = "mc"
    solver: str = "hlld"
    gamma: float = 5.0 / 3.0
    atmo_rho: float = 1e-10
    upwind: bool = True
    emf_mode: str = "solver"  # ct.py:63-88 face EMF: "solver" or "hll"

    def c(self) -> _Grid:
        return _Grid(self.nx, self.ny, self.ng, self.dx, self.dy, BCS[self.bc_x],
                     BCS[self.bc_y], LIMITERS[self.limiter], SOLVERS[self.solver],
                     self.gamma, self.atmo_rho, int(self.upwind), EMF_MODES[self.emf_mode])


def _state_ptrs(state: dict):
    for k in EVOLVED_KEYS:
        assert state["cons"][k].dtype == np.float64 and state["cons"][k].flags.c_contiguous
    cons = _ptrs([state["cons"][k] for k in EVOLVED_KEYS])
    prim = _ptrs([state["prims"][k] for k in PRIM_KEYS])
    return cons, prim


def sync_state(g: Grid2DSpec, state: dict) -> np.ndarray:
    """``driver2d.py:196-218`` in place on numpy arrays; returns C2P status."""
    cons, prim = _state_ptrs(state)
    st = np.zeros(state["cons"]["D"].shape, dtype=np.uint8)
    gc = g.c()
    lib().orc_sync_state(ctypes.byref(gc), cons, _p(state["Bxf"]), _p(state["Byf"]), prim, _p(st))
    return st


def rk_step_ct(g: Grid2DSpec, state: dict, dt: float, scheme: str = "rk3") -> dict:
    """``driver2d.py:221-249`` in place; returns the last stage's sweep diag."""
    cons, prim = _state_ptrs(state)
    d = _Diag()
    gc = g.c()
    rc = lib().orc_rk_step_ct(ctypes.byref(gc), ctypes.c_double(dt),
                              ctypes.c_int(3 if scheme == "rk3" else 2), cons,
                              _p(state["Bxf"]), _p(state["Byf"]), prim, ctypes.byref(d))
    if rc != 0:
        raise ValueError(f"oracle rk_step_ct failed ({rc})")
    return {name: list(getattr(d, name)) for name, _ in _Diag._fields_}


def compute_dt_2d(g: Grid2DSpec, prims: dict, cfl: float) -> float:
    """``driver2d.py:52-82``."""
    P = _ptrs([_f64(prims[k]) for k in PRIM_KEYS])
    gc = g.c()
    return float(lib().orc_compute_dt_2d(ctypes.byref(gc), P, ctypes.c_double(cfl)))


def rk2_step_1d(cons: dict, prims: dict, ncells: int, ng: int, dx: float, dt: float,
                limiter: str, solver: str, gamma: float, atmo_rho: float = 1e-10) -> None:
    """``driver.py:192-236`` rk2_step, in place on 1D arrays."""
    C = _ptrs([cons[k] for k in CONS_KEYS])
    P = _ptrs([prims[k] for k in PRIM_KEYS])
    lib().orc_rk2_step_1d(ctypes.c_int(ncells), ctypes.c_int(ng), ctypes.c_double(dx),
                          ctypes.c_double(dt), ctypes.c_int(LIMITERS[limiter]),
                          ctypes.c_int(SOLVERS[solver]), ctypes.c_double(gamma),
                          ctypes.c_double(atmo_rho), C, P)


def tube_run(prims: dict, L: int, ng: int, dx: float, cfl: float, tend: float, limiter: str,
             solver: str, gamma: float, scheme: str = "rk3", max_steps: int = 1 << 30,
             atmo_rho: float = 1e-10):
    """One 1D tube to tend (driver2d.py:110-156 on a ny = 1 grid), in place
    on 9 primitive arrays of L + 2 ng cells; returns (t, steps)."""
    P = _ptrs([prims[k] for k in PRIM_KEYS])
    t = ctypes.c_double(0.0)
    steps = lib().orc_tube_run(ctypes.c_int(L), ctypes.c_int(ng), ctypes.c_double(dx),
                               ctypes.c_double(cfl), ctypes.c_double(tend),
                               ctypes.c_int(max_steps), ctypes.c_int(LIMITERS[limiter]),
                               ctypes.c_int(SOLVERS[solver]), ctypes.c_double(gamma),
                               ctypes.c_double(atmo_rho), ctypes.c_int(3 if scheme == "rk3" else 2),
                               P, ctypes.byref(t))
    return t.value, int(steps)


TUBE_FLAVORS = {"rk_step": 0, "driver1d_light": 1, "driver1d_cfl": 2}


def tube_run_ex(prims: dict, L: int, ng: int, dx: float, cfl: float, tend: float, limiter: str,
                solver: str, gamma: float, *, scheme: str = "rk3", flavor: str = "rk_step",
                cons: dict | None = None, resume: bool = False, max_steps: int = 1 << 30,
                atmo_rho: float = 1e-10):
    """orc_tube_run_ex: one tube in the given stepping flavor, in place on 9
    primitive arrays (and the 8 conserved arrays when given; with
    resume=True they are the starting state); returns (t, steps)."""
    P = _ptrs([prims[k] for k in PRIM_KEYS])
    C = _ptrs([cons[k] for k in CONS_KEYS]) if cons is not None else None
    t = ctypes.c_double(0.0)
    steps = lib().orc_tube_run_ex(ctypes.c_int(L), ctypes.c_int(ng), ctypes.c_double(dx),
                                  ctypes.c_double(cfl), ctypes.c_double(tend),
                                  ctypes.c_int(max_steps), ctypes.c_int(LIMITERS[limiter]),
                                  ctypes.c_int(SOLVERS[solver]), ctypes.c_double(gamma),
                                  ctypes.c_double(atmo_rho),
                                  ctypes.c_int(3 if scheme == "rk3" else 2),
                                  ctypes.c_int(TUBE_FLAVORS[flavor]), ctypes.c_int(int(resume)),
                                  C, P, ctypes.byref(t))
    return t.value, int(steps)
