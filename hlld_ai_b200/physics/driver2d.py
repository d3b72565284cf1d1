"""2D SRMHD driver, mirroring ``src/physics/driver2d.py``.

``rk_step_ct``, ``sync_state``, ``compute_dt_2d``, ``prims_to_cons_2d`` and
``cons_to_prims_2d`` keep the reference signatures and semantics
(``driver2d.py:52-249``); the work is done by libhlld_b200.so.  One RK
step is ``scheme`` stages of five launches each -- x sweep, y sweep (fused
reconstruction + Riemann solve), corner EMF, update (flux divergence + CT +
RK combine), sync (ghosts, C2P, ghosts) -- enqueued by ``hlld_rk_step_ct``.

``Stepper2D`` is the in-place form for production loops: it owns the
scratch buffer and accepts ``dt`` as a device scalar so a step can be
captured in a CUDA graph.
"""
from __future__ import annotations

import ctypes
from collections.abc import Mapping

import torch

from .. import _lib
from .hlld import flux_diag_from_struct, primitive_to_conserved, solver_name
from .c2p import conservative_to_primitive
from .eos import kernel_gamma
from .state import EVOLVED_KEYS, PRIM_KEYS, State2D, flat, unflat

_SCHEMES = {"rk2": 2, "rk3": 3}


def _event_handle(ev):
    """The cudaEvent_t of a torch.cuda.Event (created on its first record or
    wait), or None."""
    if ev is None:
        return None
    h = ev.cuda_event
    if not h:
        raise ValueError("the event has not been recorded or waited on yet")
    return h


class Stepper2D:
    """Device resources and the C grid descriptor of one grid + option set."""

    def __init__(self, grid, eos, *, bc_x="outflow", bc_y="outflow", flux_fn="hlld",
                 limiter="mc", vel_var="Wv", emf_mode="solver", upwind=True, atmo_rho=1e-10,
                 precision="fp64"):
        if vel_var != "Wv":
            raise NotImplementedError("the fused sweep reconstructs W v (vel_var='Wv')")
        if emf_mode not in _lib.EMF_MODES:
            raise ValueError(f"unknown emf_mode {emf_mode!r} (ct.py:63-88: 'solver' or 'hll')")
        if bc_x not in _lib.BCS or bc_y not in _lib.BCS:
            raise ValueError(f"unknown boundary condition {(bc_x, bc_y)!r}")
        if limiter not in _lib.LIMITERS:
            raise ValueError(f"unknown limiter {limiter!r}")
        if precision not in _lib.PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        self.precision = precision
        # mixed: primitives (and the step's fluxes) are float32; the conserved
        # state and the staggered field stay float64.  fp32: all float32.
        self.prim_dtype = torch.float32 if precision in ("mixed", "fp32") else torch.float64
        self.state_dtype = torch.float32 if precision == "fp32" else torch.float64
        self.grid = grid
        # the step reads only the grid's sizes and device: this package's
        # Grid2D and the reference's both qualify
        self.shape = (grid.nx + 2 * grid.ng, grid.ny + 2 * grid.ng)
        self.device = torch.device(grid.device)
        if self.device.type != "cuda":
            raise TypeError("Grid2D must live on a CUDA device (hlld_ai_b200 has no CPU path)")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.gc = _lib.Grid2DC(grid.nx, grid.ny, grid.ng, grid.dx, grid.dy, _lib.BCS[bc_x],
                               _lib.BCS[bc_y], _lib.LIMITERS[limiter],
                               _lib.SOLVERS[solver_name(flux_fn)], kernel_gamma(eos),
                               float(atmo_rho), int(bool(upwind)), _lib.PRECISIONS[precision],
                               _lib.EMF_MODES[emf_mode])
        nbytes = ctypes.c_size_t(0)
        _lib.check(_lib.lib().hlld_step2d_scratch_bytes(ctypes.byref(self.gc), ctypes.byref(nbytes)),
                   "hlld_step2d_scratch_bytes")
        self.scratch = torch.empty(nbytes.value + 256, dtype=torch.uint8, device=self.device)
        self._scratch_ptr = (self.scratch.data_ptr() + 255) // 256 * 256
        self.scratch_bytes = nbytes.value
        self.diag_buf = torch.zeros(ctypes.sizeof(_lib.StepDiag), dtype=torch.uint8,
                                    device=self.device)
        self.dt_buf = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.work = torch.zeros(2, dtype=torch.int64, device=self.device)

    # -- state plumbing ---------------------------------------------------
    def _struct(self, state: State2D) -> _lib.State2DC:
        nxt, nyt = self.shape
        cs, fx, fy = (nxt, nyt), (nxt + 1, nyt), (nxt, nyt + 1)
        s = _lib.State2DC()
        for i, k in enumerate(EVOLVED_KEYS):
            s.cons[i] = self._check(state.cons[k], cs, f"cons[{k!r}]", self.state_dtype)
        for i, k in enumerate(PRIM_KEYS):
            s.prims[i] = self._check(state.prims[k], cs, f"prims[{k!r}]", self.prim_dtype)
        s.Bxf = self._check(state.Bxf, fx, "Bxf", self.state_dtype)
        s.Byf = self._check(state.Byf, fy, "Byf", self.state_dtype)
        return s

    def _check(self, t, shape, name, dtype=torch.float64) -> int:
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.device != self.device:
            raise TypeError(f"{name} must be a CUDA tensor on {self.device}")
        if t.dtype != dtype or tuple(t.shape) != shape or not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous {dtype} {shape}, got "
                             f"{t.dtype} {tuple(t.shape)}")
        return t.data_ptr()

    def ensure_prims(self, state: State2D) -> None:
        """Allocate any primitive array the state lacks (sync fills them)."""
        for k in PRIM_KEYS:
            t = state.prims.get(k)
            if t is None or not t.is_contiguous() or tuple(t.shape) != self.shape:
                state.prims[k] = torch.zeros(self.shape, dtype=self.prim_dtype, device=self.device)
            elif t.dtype != self.prim_dtype:
                state.prims[k] = t.to(self.prim_dtype).contiguous()

    # -- operations ---------------------------------------------------------
    def step(self, state: State2D, dt, scheme: str = "rk3", cons_in=None, cons_out=None) -> None:
        """One SSP-RK step in place.  dt: float, or a 1-element CUDA tensor.

        cons_in / cons_out (torch.cuda.Event, optional; hlld_rk_step_ct_events):
        the step waits for cons_in before its first read of the conserved
        cell arrays, and records cons_out once the conserved arrays and the
        faces hold its result -- for copies of the state that run on other
        streams (HostStepper2D)."""
        s = self._struct(state)
        if isinstance(dt, torch.Tensor):
            if not dt.is_cuda or dt.dtype != torch.float64:
                raise TypeError("device dt must be a float64 CUDA tensor")
            dt_host, dt_dev = 0.0, dt.data_ptr()
        else:
            dt_host, dt_dev = float(dt), None
        with torch.cuda.device(self.device):
            if cons_in is None and cons_out is None:
                rc = _lib.lib().hlld_rk_step_ct(ctypes.byref(self.gc), ctypes.byref(s),
                                                self._scratch_ptr, self.scratch_bytes, dt_host,
                                                dt_dev, _SCHEMES[scheme], self.diag_buf.data_ptr(),
                                                _lib.stream_handle(self.device))
            else:
                rc = _lib.lib().hlld_rk_step_ct_events(
                    ctypes.byref(self.gc), ctypes.byref(s), self._scratch_ptr, self.scratch_bytes,
                    dt_host, dt_dev, _SCHEMES[scheme], self.diag_buf.data_ptr(),
                    _lib.stream_handle(self.device), _event_handle(cons_in),
                    _event_handle(cons_out))
        _lib.check(rc, "rk_step_ct")

    def sync(self, state: State2D, status: torch.Tensor | None = None) -> None:
        self.ensure_prims(state)
        s = self._struct(state)
        with torch.cuda.device(self.device):
            rc = _lib.lib().hlld_sync_state(ctypes.byref(self.gc), ctypes.byref(s),
                                            status.data_ptr() if status is not None else None,
                                            self.diag_buf.data_ptr(),
                                            _lib.stream_handle(self.device))
        _lib.check(rc, "sync_state")

    def compute_dt(self, state: State2D, cfl: float, out: torch.Tensor | None = None) -> torch.Tensor:
        """compute_dt_2d on the device; returns a 1-element float64 tensor."""
        s = self._struct(state)
        out = self.dt_buf if out is None else out
        with torch.cuda.device(self.device):
            rc = _lib.lib().hlld_compute_dt_2d(ctypes.byref(self.gc), ctypes.byref(s), float(cfl),
                                               out.data_ptr(), self.work.data_ptr(),
                                               _lib.stream_handle(self.device))
        _lib.check(rc, "compute_dt_2d")
        return out

    def diag(self) -> "StepDiag":
        return StepDiag(self.diag_buf.clone())


class StepDiag(Mapping):
    """``{"x": {"diag": ...}, "y": {"diag": ...}, "c2p": ...}`` of the last
    step (driver2d.py:242-249); the device counters are copied to the host
    on first access."""

    def __init__(self, raw: torch.Tensor):
        self._raw = raw
        self._d = None

    def _load(self):
        if self._d is None:
            d = _lib.StepDiag.from_buffer_copy(bytes(self._raw.cpu().numpy()))
            out = {}
            for axis, key in ((0, "x"), (1, "y")):
                out[key] = {"diag": flux_diag_from_struct(d.sweep[axis], "hlld", axis)}
            out["c2p"] = {"not_converged": int(d.c2p_not_converged),
                          "bisected": int(d.c2p_bisected), "atmo": int(d.c2p_atmo),
                          "bad_bracket": int(d.c2p_bad_bracket)}
            self._d = out
        return self._d

    def __getitem__(self, k):
        return self._load()[k]

    def __iter__(self):
        return iter(self._load())

    def __len__(self):
        return len(self._load())


_STEPPERS: dict = {}


def stepper_for(grid, eos, **opts) -> Stepper2D:
    """A cached Stepper2D for this grid object and option set."""
    key = (id(grid), float(eos.gamma), tuple(sorted((k, str(v)) for k, v in opts.items())))
    st = _STEPPERS.get(key)
    if st is None or st.grid is not grid:
        st = Stepper2D(grid, eos, **opts)
        _STEPPERS[key] = st
    return st


def _opts(bc_x, bc_y, flux_fn, limiter, vel_var, emf_mode, upwind, atmo_rho, precision):
    return dict(bc_x=bc_x, bc_y=bc_y, flux_fn=solver_name(flux_fn), limiter=limiter,
                vel_var=vel_var, emf_mode=emf_mode, upwind=upwind, atmo_rho=atmo_rho,
                precision=precision)


def rk_step_ct(state, grid, eos, dt, *, scheme="rk3", bc_x="outflow", bc_y="outflow",
               flux_fn="hlld", limiter="mc", vel_var="Wv", emf_mode="solver", upwind=True,
               atmo_rho=1e-10, recorder=None, precision="fp64"):
    """driver2d.py:221-249.  Returns a new State2D (the input is left as it
    was, as in the reference) and the last stage's sweep diagnostics."""
    if recorder is not None:
        raise NotImplementedError("interface-state recording is not part of the B200 step")
    if scheme not in _SCHEMES:
        raise ValueError(f"unknown scheme {scheme!r}")
    st = stepper_for(grid, eos, **_opts(bc_x, bc_y, flux_fn, limiter, vel_var, emf_mode, upwind,
                                        atmo_rho, precision))
    S = State2D(cons={k: state.cons[k].clone() for k in EVOLVED_KEYS}, Bxf=state.Bxf.clone(),
                Byf=state.Byf.clone(), prims={k: state.prims[k].clone() for k in PRIM_KEYS})
    st.step(S, dt, scheme)
    return S, st.diag()


def sync_state(state, grid, eos, bc_x="outflow", bc_y="outflow", atmo_rho=1e-10,
               return_status=False, precision="fp64", limiter="mc"):
    """driver2d.py:196-218, in place; returns the state (and C2P status)."""
    st = stepper_for(grid, eos, **_opts(bc_x, bc_y, "hlld", limiter, "Wv", "solver", True,
                                        atmo_rho, precision))
    status = (torch.zeros(grid.nxt, grid.nyt, dtype=torch.uint8, device=st.device)
              if return_status else None)
    st.sync(state, status)
    if not return_status:
        return state
    # C2P runs on the physical cells only (ghost primitives are BC copies);
    # ghost entries of the masks are False
    masks = {"bracket_ok": (status & _lib.ST_BRACKET_OK) != 0,
             "converged": (status & _lib.ST_CONVERGED) != 0,
             "v_clamped": (status & _lib.ST_V_CLAMPED) != 0,
             "atmo_floored": (status & _lib.ST_ATMO) != 0}
    return state, masks


def compute_dt_2d(prims, grid, eos, cfl, speed_of_light=False, precision="fp64") -> float:
    """driver2d.py:52-82 (one device->host read, as the reference's float())."""
    if speed_of_light:
        one = torch.ones((), dtype=torch.float64)
        return float(cfl / (one / grid.dx + one / grid.dy))
    st = stepper_for(grid, eos, **_opts("outflow", "outflow", "hlld", "mc", "Wv", "solver", True,
                                        1e-10, precision))
    # the speed kernel reads the primitives only; the other arrays of the
    # state descriptor are placeholders of the right shapes and types
    nxt, nyt = st.shape
    place = torch.empty(nxt, nyt, dtype=st.state_dtype, device=st.device)
    S = State2D(cons={k: place for k in EVOLVED_KEYS},
                Bxf=torch.empty(nxt + 1, nyt, dtype=st.state_dtype, device=st.device),
                Byf=torch.empty(nxt, nyt + 1, dtype=st.state_dtype, device=st.device), prims=prims)
    return float(st.compute_dt(S, cfl).item())


def prims_to_cons_2d(prims: dict, grid, precision="fp64") -> dict:
    """driver2d.py:97-98"""
    return unflat(primitive_to_conserved(flat(prims), precision), grid.shape)


def cons_to_prims_2d(cons: dict, grid, eos, atmo_rho: float = 1e-10, return_status=False):
    """driver2d.py:85-94"""
    out = conservative_to_primitive(flat(cons), eos, atmo_rho=atmo_rho, return_status=return_status)
    if return_status:
        prims, status = out
        return unflat(prims, grid.shape), {k: v.reshape(*grid.shape) for k, v in status.items()}
    return unflat(out, grid.shape)
