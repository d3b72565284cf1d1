"""Batched independent 1D SRMHD tubes in one persistent launch.

The B200 form of ``src/physics/tube_seed.py:93-144`` run_tubes for
thousands of tubes of uneven length: every tube runs the reference's no-CT
step (``driver2d.py:110-156`` rk_step on a ny = 1 grid, WENO5-Z / PLM,
HLLD / HLLE, SSP-RK3) with its OWN CFL time step (``driver.py:77-127``) to
``tend``.  All tubes advance in a single launch of ``hlld_tubes_run``: each
CTA takes whole tubes, longest first, from a device work counter.  The
launch can be captured in a CUDA graph (``TubeBatch.capture``), and the
CTA shape is chosen by ``TubeBatch.autotune``, which times the candidate
shapes on a sample of the batch.

Layout: tube i owns cells ``cell_off[i] .. cell_off[i] + L_i + 2 ng - 1`` of
the concatenated primitive / conserved arrays and faces
``cell_off[i] + i ..`` of the face arrays (L_i + 2 ng + 1 of them).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .physics.state import PRIM_KEYS


TubesC = _lib.TubesC
FLAVORS = {"rk_step": _lib.TUBE_RK_STEP, "driver1d_light": _lib.TUBE_DRIVER1D_LIGHT,
           "driver1d_cfl": _lib.TUBE_DRIVER1D_CFL}


@dataclass
class TubeStates:
    """Left/right states of the tubes' Riemann problems (host numpy)."""
    lengths: np.ndarray        # (n,) physical cells
    left: dict                 # primitive -> (n,) values
    right: dict
    Bx: np.ndarray             # (n,) normal field shared by both sides


def random_tubes(n: int, seed: int = 20261203, lmin: int = 256, lmax: int = 4096,
                 gamma: float = 5.0 / 3.0) -> TubeStates:
    """The batched-tube workload: lengths uniform in [lmin, lmax]; per side rho
    and p log-uniform in [0.1, 10] and [0.01, 100], each velocity component
    uniform in [-0.5, 0.5] (|v| < 0.9 enforced by redrawing), By and Bz
    uniform in [-2, 2]; Bx uniform in [-1, 1], shared by both sides."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(lmin, lmax + 1, size=n)
    sides = []
    for _ in range(2):
        v = rng.uniform(-0.5, 0.5, size=(n, 3))
        bad = np.linalg.norm(v, axis=1) >= 0.9
        while bad.any():
            v[bad] = rng.uniform(-0.5, 0.5, size=(int(bad.sum()), 3))
            bad = np.linalg.norm(v, axis=1) >= 0.9
        s = {"rho": 10.0 ** rng.uniform(-1, 1, n), "p": 10.0 ** rng.uniform(-2, 2, n),
             "vx": v[:, 0], "vy": v[:, 1], "vz": v[:, 2],
             "By": rng.uniform(-2, 2, n), "Bz": rng.uniform(-2, 2, n)}
        s["eps"] = 0.0 + (s["p"] - 0.0) / (s["rho"] * (gamma - 1.0))
        sides.append(s)
    Bx = rng.uniform(-1, 1, n)
    return TubeStates(lengths=lengths, left=sides[0], right=sides[1], Bx=Bx)


def tube_prims(states: TubeStates, i: int, ng: int) -> dict:
    """Host primitives (ghosts included) of tube i on [0, 1], jump at x = 0.5."""
    L = int(states.lengths[i])
    nt = L + 2 * ng
    x = 0.0 + (np.arange(nt, dtype=np.float64) - ng + 0.5) * (1.0 / L)
    left = x < 0.5
    out = {}
    for k in ("rho", "p", "vx", "vy", "vz", "By", "Bz", "eps"):
        out[k] = np.where(left, states.left[k][i], states.right[k][i]).astype(np.float64)
    out["Bx"] = np.full(nt, states.Bx[i], dtype=np.float64)
    return out


class TubeBatch:
    """Device state of a tube batch and the persistent launch over it."""

    def __init__(self, states: TubeStates, *, limiter: str = "weno5z", solver: str = "hlld",
                 scheme: str = "rk3", precision: str = "fp64", gamma: float = 5.0 / 3.0,
                 atmo_rho: float = 1e-10, device="cuda", flavor: str = "rk_step",
                 ng: int | None = None):
        from .physics.reconstruction import ghosts_needed

        if precision not in ("fp64", "fp64_exact", "mixed", "fp32"):
            raise ValueError(f"unknown precision {precision!r}")
        if flavor not in FLAVORS:
            raise ValueError(f"unknown flavor {flavor!r}")
        self.flavor = flavor
        self.states = states
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise TypeError("tubes run on a CUDA device only")
        self.ng = ghosts_needed(limiter) if ng is None else int(ng)
        self.limiter, self.solver, self.scheme, self.precision = limiter, solver, scheme, precision
        self.gamma, self.atmo_rho = gamma, atmo_rho
        n = len(states.lengths)
        self.n = n
        L = states.lengths.astype(np.int64)
        nt = L + 2 * self.ng
        off = np.zeros(n + 1, dtype=np.int64)
        off[1:] = np.cumsum(nt)
        self.total_cells = int(off[-1])
        self.total_faces = self.total_cells + n
        host = {k: np.empty(self.total_cells) for k in PRIM_KEYS}
        for i in range(n):
            p = tube_prims(states, i, self.ng)
            for k in PRIM_KEYS:
                host[k][off[i]:off[i + 1]] = p[k]
        self.host_init = host
        self.pdtype = torch.float32 if precision in ("mixed", "fp32") else torch.float64
        # conserved state: float32 in the all-FP32 form only
        self.sdtype = torch.float32 if precision == "fp32" else torch.float64
        dev = self.device
        self.prims = {k: torch.tensor(host[k], dtype=self.pdtype, device=dev) for k in PRIM_KEYS}
        self.cons = [torch.empty(self.total_cells, dtype=self.sdtype, device=dev) for _ in range(8)]
        self.U0 = [torch.empty(self.total_cells, dtype=self.sdtype, device=dev) for _ in range(8)]
        self.F = [torch.empty(self.total_faces, dtype=self.pdtype, device=dev) for _ in range(8)]
        self.ncells = torch.tensor(L.astype(np.int32), device=dev)
        self.cell_off = torch.tensor(off[:-1], device=dev)
        self.dx = torch.tensor(1.0 / L.astype(np.float64), device=dev)
        # longest tube first: the costliest work starts first
        self.order = torch.tensor(np.argsort(-L, kind="stable").astype(np.int32), device=dev)
        self.t_out = torch.zeros(n, dtype=torch.float64, device=dev)
        self.steps_out = torch.zeros(n, dtype=torch.int32, device=dev)
        self.next = torch.zeros(1, dtype=torch.int32, device=dev)
        self.threads, self.blocks = 0, 0
        self._graph = None

    def reset(self) -> None:
        """Restore the initial primitives."""
        for k in PRIM_KEYS:
            self.prims[k].copy_(torch.as_tensor(self.host_init[k], dtype=self.pdtype))

    def _c(self, tend: float, cfl: float, max_steps: int, resume: bool) -> TubesC:
        return TubesC(self.n, self.ng, self.ncells.data_ptr(), self.cell_off.data_ptr(),
                      self.dx.data_ptr(), self.order.data_ptr(), float(cfl), float(tend),
                      int(max_steps), _lib.LIMITERS[self.limiter], _lib.SOLVERS[self.solver],
                      3 if self.scheme == "rk3" else 2, _lib.PRECISIONS[self.precision],
                      float(self.gamma), float(self.atmo_rho), FLAVORS[self.flavor],
                      int(bool(resume)))

    def launch(self, tend: float, cfl: float = 0.4, max_steps: int = 1 << 30,
               threads: int | None = None, blocks: int | None = None,
               resume: bool = False) -> None:
        """Enqueue one persistent launch that advances every tube by tend
        (from t = 0 of this launch).  resume=False rebuilds the conserved
        state from the primitives first; resume=True continues from the
        conserved state the previous launch left (a run split into
        chunks then equals one run, apart from the step cut at each chunk
        end)."""
        self._cdesc = self._c(tend, cfl, max_steps, resume)  # kept alive for graph replays
        with torch.cuda.device(self.device):
            rc = _lib.lib().hlld_tubes_run(
                ctypes.byref(self._cdesc), _lib.ptr_array(self.cons),
                _lib.ptr_array([self.prims[k] for k in PRIM_KEYS]), _lib.ptr_array(self.U0),
                _lib.ptr_array(self.F), self.t_out.data_ptr(), self.steps_out.data_ptr(),
                self.next.data_ptr(), int(threads if threads is not None else self.threads),
                int(blocks if blocks is not None else self.blocks), _lib.stream_handle(self.device))
        _lib.check(rc, "hlld_tubes_run")

    def capture(self, tend: float, cfl: float = 0.4, max_steps: int = 1 << 30,
                resume: bool = False) -> torch.cuda.CUDAGraph:
        """Capture the launch in a CUDA graph (each replay advances the tubes
        by tend from the primitives -- or, with resume, the conserved state
        -- they hold)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.launch(tend, cfl, max_steps, resume=resume)
        torch.cuda.current_stream(self.device).wait_stream(s)
        self._graph = g
        return g

    def cell_updates(self) -> int:
        """Physical cell-updates (cells x steps) of the last run."""
        return int((self.steps_out.to(torch.int64).cpu() * torch.as_tensor(self.states.lengths)).sum())

    def tube_cons(self, i: int) -> dict:
        """Conserved variables of tube i (ghosts included), float64 numpy."""
        from .physics.state import CONS_KEYS

        a = int(self.cell_off[i].item())
        b = a + int(self.states.lengths[i]) + 2 * self.ng
        return {k: self.cons[j][a:b].cpu().numpy() for j, k in enumerate(CONS_KEYS)}

    def tube(self, i: int) -> dict:
        """Primitives of tube i (ghosts included), as float64 numpy."""
        a = int(self.cell_off[i].item())
        b = a + int(self.states.lengths[i]) + 2 * self.ng
        return {k: self.prims[k][a:b].double().cpu().numpy() for k in PRIM_KEYS}

    def autotune(self, tend: float, cfl: float = 0.4, sample: int = 256,
                 shapes=((128, 4), (256, 1), (256, 2), (384, 1), (512, 1))) -> tuple:
        """Pick (threads, CTAs per SM) by timing each candidate on a sample of
        the batch (every n/sample-th tube) to `tend`; stores and returns the
        winner as (threads, blocks)."""
        idx = np.linspace(0, self.n - 1, min(sample, self.n)).astype(int)
        sub = TubeStates(self.states.lengths[idx], {k: v[idx] for k, v in self.states.left.items()},
                         {k: v[idx] for k, v in self.states.right.items()}, self.states.Bx[idx])
        probe = TubeBatch(sub, limiter=self.limiter, solver=self.solver, scheme=self.scheme,
                          precision=self.precision, gamma=self.gamma, atmo_rho=self.atmo_rho,
                          device=self.device, flavor=self.flavor, ng=self.ng)
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        best = None
        for threads, per_sm in shapes:
            blocks = sms * per_sm
            probe.reset()
            probe.launch(tend, cfl, threads=threads, blocks=blocks)  # warm-up
            probe.reset()
            torch.cuda.synchronize(self.device)
            t0 = time.perf_counter()
            probe.launch(tend, cfl, threads=threads, blocks=blocks)
            torch.cuda.synchronize(self.device)
            el = time.perf_counter() - t0
            if best is None or el < best[0]:
                best = (el, threads, blocks)
        self.threads, self.blocks = best[1], best[2]
        self.tuned = {"threads": best[1], "blocks": best[2], "seconds": best[0]}
        return self.threads, self.blocks
