"""Run a 2D SRMHD problem on the GPU; drop-in for the reference's ``scripts/run_2d.py``.

    python -m hlld_ai_b200.run_2d --problem rotor --n 256 --solver hlld

The options are the reference CLI's (``run_2d.py:91-153``) without the
exact-flux and envelope ones, plus ``--precision``.  A run directory holds
the files the reference's analysis scripts read, with the same names, keys
and columns:

  * ``run_meta.json``  the run's options and, at the end, its step count and
    wall time;
  * ``diag.csv``       one row every ``--log-every`` steps (``run_2d.py:285-287``);
  * ``snap_NNN.npz``   ``--nsnap`` snapshots of rho, p, vx, vy, Bx, By and
    div B on the physical cells, plus ``snap_000`` and ``snap_fin``
    (``run_2d.py:264-272``);
  * ``restart.npz``    the conserved state and staggered field every
    ``--restart-every`` steps, replaced atomically (``run_2d.py:321-334``).

The step is the fused B200 step (``Stepper2D``); dt is computed on the
device and read back every step, as the reference reads its CFL dt.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import socket
import subprocess
import sys
import time

import numpy as np
import torch

from .physics.driver2d import Stepper2D
from .physics.initial_data2d import PROBLEMS, orszag_tang, setup_problem
from .physics.reconstruction import ghosts_needed
from .physics.state import EVOLVED_KEYS, State2D

SOLVERS = ("hlld", "hlle", "hllc")
LIMITERS = ("pcm", "mc", "minmod", "weno5z", "mp5", "mp7")
PRECISIONS = ("fp64", "fp64_exact", "mixed", "fp32")

# diag.csv columns (the reference's; the last two count exact-flux faces,
# which this step has none of, and are written as -1)
DIAG_COLUMNS = ("step", "t", "dt", "divB_max", "divB_l2", "sym_err", "rho_max", "rho_min",
                "p_min", "W_max", "hlle_frac_x", "hlle_frac_y", "mean_iters", "c2p_bad",
                "n_exact_x", "n_verified_x")
SNAP_FIELDS = ("rho", "p", "vx", "vy", "Bx", "By")
# options that must agree between a run directory's meta and a new run in it
SAME_RUN_KEYS = ("limiter", "n", "solver", "problem")


def _orszag_tang_bs(grid, eos):
    """The Orszag-Tang variant of Beckwith & Stone, v_max = sqrt(2)/2
    (initial_data2d.py:256-270)."""
    return orszag_tang(grid, eos, v_max=0.5 * math.sqrt(2.0))


PROBLEMS.setdefault("orszag_tang_bs", dict(box=(0.0, 1.0), gamma=5.0 / 3.0, tend=1.0,
                                           bc=("periodic", "periodic"), build=_orszag_tang_bs))


def symmetry_error(state, grid) -> float:
    """The rotor's pi-rotation invariance (run_2d.py:67-87): scalars and B map
    onto themselves and v onto -v under (x, y) -> (-x, -y); the largest
    violation over rho, p, v and B, relative to each field's maximum."""
    worst = 0.0
    for key, sign in (("rho", 1.0), ("p", 1.0), ("vx", -1.0), ("vy", -1.0), ("Bx", 1.0), ("By", 1.0)):
        f = state.prims[key][grid.phys].double()
        rotated = torch.rot90(f, 2, dims=(0, 1))
        scale = max(float(f.abs().max()), 1e-30)
        worst = max(worst, float((f - sign * rotated).abs().max()) / scale)
    return worst


def div_b(Bxf, Byf, dx, dy):
    """Cell divergence of the staggered field (ct.py:196-199)."""
    return torch.diff(Bxf, dim=0) / dx + torch.diff(Byf, dim=1) / dy


def _git_rev() -> str:
    try:
        r = subprocess.run(["git", "rev-parse", "--short", "HEAD"], capture_output=True, text=True,
                           timeout=5, cwd=os.path.dirname(os.path.abspath(__file__)))
        return r.stdout.strip() or "unknown"
    except Exception:
        return "unknown"


def _atomic_json(path, obj):
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(obj, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--problem", default="rotor", choices=sorted(PROBLEMS))
    ap.add_argument("--b0", type=float, default=0.5)
    ap.add_argument("--bz-deg", type=float, default=0.0)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--tend", type=float, default=None)
    ap.add_argument("--cfl", type=float, default=0.25)
    ap.add_argument("--solver", default="hlld", choices=SOLVERS)
    ap.add_argument("--emf-mode", default="solver", choices=["solver", "hll"])
    ap.add_argument("--limiter", default="mc", choices=LIMITERS)
    ap.add_argument("--no-upwind-emf", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=PRECISIONS)
    ap.add_argument("--out", default=None)
    ap.add_argument("--restart", default=None)
    ap.add_argument("--restart-every", type=int, default=10)
    ap.add_argument("--log-every", type=int, default=10)
    ap.add_argument("--max-steps", type=int, default=None)
    ap.add_argument("--nsnap", type=int, default=5)
    ap.add_argument("--device", default="cuda")
    return ap.parse_args(argv)


class Run:
    """One run directory: set-up or restart, the time loop and its outputs."""

    def __init__(self, args):
        self.a = args
        self.spec = PROBLEMS[args.problem]
        self.tend = args.tend if args.tend is not None else self.spec["tend"]
        suffix = "" if args.limiter == "mc" else f"_{args.limiter}"
        self.out = args.out or f"results/{args.problem}_{args.n}_{args.solver}{suffix}"
        self.bc = tuple(self.spec["bc"])
        self.t, self.step, self.next_snap, self.gen = 0.0, 0, 1, 0
        self.steps_here = 0
        self.meta = self._meta()

    # -- set-up ---------------------------------------------------------
    def _meta(self) -> dict:
        a = self.a
        rd = a.problem == "riemann2d"
        return dict(problem=a.problem, b0=a.b0 if rd else None, bz_deg=a.bz_deg if rd else None,
                    n=a.n, solver=a.solver, limiter=a.limiter, ng=ghosts_needed(a.limiter),
                    cfl=a.cfl, tend=self.tend, nsnap=a.nsnap, emf_mode=a.emf_mode,
                    upwind_emf=not a.no_upwind_emf, bc=list(self.bc), gamma=self.spec["gamma"],
                    host=socket.gethostname(), device=torch.cuda.get_device_name(),
                    precision=a.precision, git=_git_rev(),
                    started=time.strftime("%Y-%m-%dT%H:%M:%S"))

    def _check_directory(self):
        """Refuse to mix two different runs in one directory."""
        prev = os.path.join(self.out, "run_meta.json")
        if self.a.restart or not os.path.exists(prev):
            return
        with open(prev) as fh:
            old = json.load(fh)
        clash = [f"{k} {old.get(k)!r} != {self.meta[k]!r}" for k in SAME_RUN_KEYS
                 if old.get(k) != self.meta[k]]
        if clash:
            sys.exit(f"refusing to write into {self.out}: it holds a different run "
                     f"({', '.join(clash)}).  Pass --out, or --restart to continue that one.")

    def prepare(self):
        a = self.a
        os.makedirs(self.out, exist_ok=True)
        self._check_directory()
        self.grid, self.eos, self.state, _ = setup_problem(a.problem, a.n, limiter=a.limiter,
                                                           device=a.device, precision=a.precision)
        self.stepper = Stepper2D(self.grid, self.eos, bc_x=self.bc[0], bc_y=self.bc[1],
                                 flux_fn=a.solver, limiter=a.limiter, emf_mode=a.emf_mode,
                                 upwind=not a.no_upwind_emf, precision=a.precision)
        if a.restart:
            self._load_restart(a.restart)
        _atomic_json(os.path.join(self.out, "run_meta.json"), self.meta)

    def _load_restart(self, path):
        R = np.load(path)
        g, a = self.grid, self.a
        if "limiter" in R.files and str(R["limiter"]) != a.limiter:
            sys.exit(f"restart {path} was written with --limiter {R['limiter']}, "
                     f"this run says {a.limiter}")
        shape = tuple(R["cons_D"].shape)
        if shape != (g.nxt, g.nyt):
            sys.exit(f"restart {path} holds {shape} arrays, this grid is {(g.nxt, g.nyt)} "
                     f"(ng = {g.ng} for --limiter {a.limiter}): the limiter does not match")
        like = self.state.Bxf
        load = lambda key: torch.from_numpy(R[key].copy()).to(device=like.device, dtype=like.dtype)
        self.state = State2D(cons={k: load("cons_" + k) for k in EVOLVED_KEYS},
                             Bxf=load("Bxf"), Byf=load("Byf"), prims={})
        self.stepper.sync(self.state)
        self.t, self.step = float(R["t"]), int(R["step"])
        self.next_snap, self.gen = int(R["next_snap"]), int(R["gen"]) + 1

    # -- outputs ----------------------------------------------------------
    def snapshot(self, tag):
        g, st, a = self.grid, self.state, self.a
        fields = {k: st.prims[k][g.phys].double().cpu().numpy() for k in SNAP_FIELDS}
        np.savez_compressed(os.path.join(self.out, f"snap_{tag}.npz"), t=self.t,
                            x=g.x[g.phys[0]].cpu().numpy(), y=g.y[g.phys[1]].cpu().numpy(),
                            divB=div_b(st.Bxf, st.Byf, g.dx, g.dy)[g.phys].double().cpu().numpy(),
                            limiter=a.limiter, ng=g.ng, n=a.n, solver=a.solver, **fields)

    def checkpoint(self):
        st, a = self.state, self.a
        path = os.path.join(self.out, "restart.npz")
        tmp = path + ".tmp.npz"
        np.savez(tmp, t=self.t, step=self.step, next_snap=self.next_snap, gen=self.gen,
                 limiter=a.limiter, ng=self.grid.ng, n=a.n, solver=a.solver, harvest_sweeps=0,
                 Bxf=st.Bxf.cpu().numpy(), Byf=st.Byf.cpu().numpy(),
                 **{"cons_" + k: st.cons[k].cpu().numpy() for k in EVOLVED_KEYS})
        os.replace(tmp, path)

    def diag_row(self, dt, diag) -> tuple[str, dict]:
        g, P = self.grid, self.state.prims
        ph = g.phys
        d = div_b(self.state.Bxf, self.state.Byf, g.dx, g.dy)[ph].double()
        v2 = sum(P[k][ph].double() ** 2 for k in ("vx", "vy", "vz"))
        rho = P["rho"][ph]
        vals = dict(step=self.step, t=self.t, dt=dt, divB_max=float(d.abs().max()),
                    divB_l2=float(d.square().mean().sqrt()),
                    sym_err=symmetry_error(self.state, g) if self.a.problem == "rotor" else math.nan,
                    rho_max=float(rho.max()), rho_min=float(rho.min()),
                    p_min=float(P["p"][ph].min()),
                    W_max=float(torch.rsqrt(torch.clamp(1.0 - v2, min=1e-16)).max()),
                    hlle_frac_x=diag["x"]["diag"]["frac_hlle_fallback"],
                    hlle_frac_y=diag["y"]["diag"]["frac_hlle_fallback"],
                    mean_iters=diag["x"]["diag"]["mean_iters"],
                    c2p_bad=diag["c2p"]["not_converged"])
        fmt = dict(t="{:.6e}", dt="{:.3e}", divB_max="{:.3e}", divB_l2="{:.3e}", sym_err="{:.3e}",
                   rho_max="{:.4f}", rho_min="{:.4e}", p_min="{:.4e}", W_max="{:.3f}",
                   hlle_frac_x="{:.4f}", hlle_frac_y="{:.4f}", mean_iters="{:.2f}")
        cells = [fmt.get(c, "{}").format(vals[c]) if c in vals else "-1" for c in DIAG_COLUMNS]
        return ",".join(cells) + "\n", vals

    def _finish_meta(self, wall, **extra):
        self.meta.update(steps=self.step, steps_here=self.steps_here, wall_s=round(wall, 1),
                         s_per_step=round(wall / max(self.steps_here, 1), 4),
                         finished=time.strftime("%Y-%m-%dT%H:%M:%S"), **extra)
        _atomic_json(os.path.join(self.out, "run_meta.json"), self.meta)

    # -- the time loop ------------------------------------------------------
    def _fail(self, why):
        P = self.state.prims
        raise SystemExit(f"run failed at step {self.step}, t = {self.t:.6f}: {why} "
                         f"(rho_max {float(P['rho'].max()):.3e}, p_min {float(P['p'].min()):.3e}).  "
                         "No snap_fin is written and the exit status is non-zero.")

    def advance(self) -> int:
        a, tend = self.a, self.tend
        print(f"{a.problem} {a.n}^2  solver={a.solver}  emf={a.emf_mode}"
              f"{' (flux-CT)' if a.no_upwind_emf else ''}  limiter={a.limiter}  cfl={a.cfl}  "
              f"gamma={self.spec['gamma']:.4f}  bc=({self.bc[0]},{self.bc[1]})  t_end={tend}  "
              f"precision={a.precision}", flush=True)
        diag_path = os.path.join(self.out, "diag.csv")
        if a.restart:
            print(f"  restart from {a.restart}: t={self.t:.6f} step={self.step} "
                  f"generation={self.gen}", flush=True)
            log = open(diag_path, "a")
        else:
            self.snapshot("000")
            log = open(diag_path, "w")
            log.write(",".join(DIAG_COLUMNS) + "\n")
        t0 = time.time()
        done = lambda: self.t >= tend - 1e-14
        with log:
            while not done():
                dt = min(float(self.stepper.compute_dt(self.state, a.cfl).item()), tend - self.t)
                if not (math.isfinite(dt) and dt > 0.0):
                    self._fail(f"dt = {dt!r}, the state went non-finite")
                self.stepper.step(self.state, dt, "rk3")
                self.t += dt
                self.step += 1
                self.steps_here += 1
                if not math.isfinite(float(self.state.cons["D"].sum())):
                    self._fail("the conserved state is not finite")
                if self.step % max(1, a.log_every) == 0 or done():
                    row, v = self.diag_row(dt, self.stepper.diag())
                    log.write(row)
                    log.flush()
                    sym = f"sym={v['sym_err']:.2e} " if a.problem == "rotor" else ""
                    print(f"  step {self.step:5d} t={self.t:.4f} dt={dt:.2e} "
                          f"divB={v['divB_max']:.2e} {sym}rho=[{v['rho_min']:.3f},"
                          f"{v['rho_max']:.3f}] c2p_bad={v['c2p_bad']} ({time.time() - t0:.0f}s)",
                          flush=True)
                if self.next_snap <= a.nsnap and self.t >= self.next_snap * tend / a.nsnap - 1e-14:
                    self.snapshot(f"{self.next_snap:03d}")
                    self.next_snap += 1
                if done():
                    break
                if a.restart_every and self.step % a.restart_every == 0:
                    self.checkpoint()
                if a.max_steps is not None and self.steps_here >= a.max_steps:
                    self.checkpoint()
                    wall = time.time() - t0
                    self._finish_meta(wall, stopped_early=True)
                    print(f"stopped after {self.steps_here} steps at t={self.t:.6f} "
                          f"(step {self.step}); restart file written ({wall:.0f}s)", flush=True)
                    return 0
        self.snapshot("fin")
        wall = time.time() - t0
        self._finish_meta(wall)
        print(f"done in {wall:.0f}s, {self.step} steps -> {self.out}", flush=True)
        return 0


def main(argv=None):
    run = Run(parse(argv))
    run.prepare()
    return run.advance()


if __name__ == "__main__":
    sys.exit(main())
