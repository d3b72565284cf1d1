"""Run a 2D SRMHD problem on the GPU; drop-in for ``scripts/run_2d.py``.

    python -m hlld_ai_b200.run_2d --problem rotor --n 256 --solver hlld

Same options (``run_2d.py:91-153``, minus the exact-flux and envelope ones),
same outputs in ``--out``: ``run_meta.json``, ``diag.csv`` (same columns,
``run_2d.py:285-287``), ``snap_*.npz`` (same keys, ``:264-272``) and
``restart.npz`` (same keys, written atomically, ``:321-334``), so the
reference's analysis scripts read these runs.  The step is the fused B200
step (``Stepper2D``); dt is read back every step, as the reference does.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import subprocess
import sys
import time

import numpy as np
import torch

from .physics.driver2d import Stepper2D, sync_state
from .physics.initial_data2d import PROBLEMS, orszag_tang, setup_problem
from .physics.reconstruction import ghosts_needed
from .physics.state import EVOLVED_KEYS, State2D

SOLVERS = ("hlld", "hlle", "hllc")


def _bs(grid, eos):
    """Beckwith & Stone's Orszag-Tang (initial_data2d.py:256-270)."""
    import math
    return orszag_tang(grid, eos, v_max=0.5 * math.sqrt(2.0))


PROBLEMS.setdefault("orszag_tang_bs", dict(box=(0.0, 1.0), gamma=5.0 / 3.0, tend=1.0,
                                           bc=("periodic", "periodic"), build=_bs))


def _git_rev():
    try:
        return subprocess.run(["git", "rev-parse", "--short", "HEAD"], capture_output=True,
                              text=True, timeout=5,
                              cwd=os.path.dirname(os.path.abspath(__file__))).stdout.strip() or "unknown"
    except Exception:
        return "unknown"


def _write_meta(out, meta):
    tmp = os.path.join(out, "run_meta.json.tmp")
    with open(tmp, "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    os.replace(tmp, os.path.join(out, "run_meta.json"))


def symmetry_error(st, g):
    """run_2d.py:67-87: pi-rotation (with B -> -B) invariance of the rotor."""
    ph = g.phys
    worst = 0.0
    for k, parity in (("rho", +1), ("p", +1), ("vx", -1), ("vy", -1), ("Bx", +1), ("By", +1)):
        a = st.prims[k][ph].double()
        b = torch.flip(a, dims=(0, 1))
        worst = max(worst, float((a - parity * b).abs().max()) / max(float(a.abs().max()), 1e-30))
    return worst


def div_b(Bxf, Byf, dx, dy):
    """ct.py:196-199"""
    return (Bxf[1:, :] - Bxf[:-1, :]) / dx + (Byf[:, 1:] - Byf[:, :-1]) / dy


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
    ap.add_argument("--limiter", default="mc", choices=["pcm", "mc", "minmod", "weno5z", "mp5", "mp7"])
    ap.add_argument("--no-upwind-emf", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp64_exact", "mixed"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--restart", default=None)
    ap.add_argument("--restart-every", type=int, default=10)
    ap.add_argument("--log-every", type=int, default=10)
    ap.add_argument("--max-steps", type=int, default=None)
    ap.add_argument("--nsnap", type=int, default=5)
    ap.add_argument("--device", default="cuda")
    return ap.parse_args(argv)


def main(argv=None):
    a = parse(argv)
    P = PROBLEMS[a.problem]
    tend = a.tend if a.tend is not None else P["tend"]
    out = a.out or (f"results/{a.problem}_{a.n}_{a.solver}" + ("" if a.limiter == "mc" else f"_{a.limiter}"))
    bc_x, bc_y = P["bc"]
    os.makedirs(out, exist_ok=True)
    meta = dict(problem=a.problem, b0=(a.b0 if a.problem == "riemann2d" else None),
                bz_deg=(a.bz_deg if a.problem == "riemann2d" else None), n=a.n, solver=a.solver,
                limiter=a.limiter, ng=ghosts_needed(a.limiter), cfl=a.cfl, tend=tend,
                nsnap=a.nsnap, emf_mode=a.emf_mode, upwind_emf=not a.no_upwind_emf,
                bc=[bc_x, bc_y], gamma=P["gamma"], host=socket.gethostname(),
                device=torch.cuda.get_device_name(), precision=a.precision, git=_git_rev(),
                started=time.strftime("%Y-%m-%dT%H:%M:%S"))
    prev = os.path.join(out, "run_meta.json")
    if os.path.exists(prev) and not a.restart:
        old = json.load(open(prev))
        clash = {k: (old.get(k), meta[k]) for k in ("limiter", "n", "solver", "problem")
                 if old.get(k) != meta[k]}
        if clash:
            sys.exit("refusing to write into %s: it holds a different run (%s).  Pass --out, "
                     "or --restart to continue that one." % (out, ", ".join(
                         "%s %r != %r" % (k, o, n) for k, (o, n) in clash.items())))

    g, eos, st, spec = setup_problem(a.problem, a.n, limiter=a.limiter, device=a.device,
                                     precision=a.precision)
    stepper = Stepper2D(g, eos, bc_x=bc_x, bc_y=bc_y, flux_fn=a.solver, limiter=a.limiter,
                        emf_mode=a.emf_mode, upwind=not a.no_upwind_emf, precision=a.precision)
    gen = 0
    R = None
    if a.restart:
        R = np.load(a.restart)
        want = (g.nxt, g.nyt)
        got = tuple(R["cons_D"].shape)
        if "limiter" in R.files and str(R["limiter"]) != a.limiter:
            sys.exit("restart %s was written with --limiter %s, this run says %s"
                     % (a.restart, str(R["limiter"]), a.limiter))
        if got != want:
            sys.exit("restart %s holds %s arrays, this grid is %s (ng = %d for --limiter %s): "
                     "the limiter does not match" % (a.restart, got, want, g.ng, a.limiter))
        dev = st.Bxf.device
        st = State2D(cons={k: torch.from_numpy(R["cons_" + k].copy()).to(dev) for k in EVOLVED_KEYS},
                     Bxf=torch.from_numpy(R["Bxf"].copy()).to(dev),
                     Byf=torch.from_numpy(R["Byf"].copy()).to(dev), prims={})
        stepper.sync(st)
        gen = int(R["gen"]) + 1
    _write_meta(out, meta)

    def save(tag, t):
        ph = g.phys
        np.savez_compressed(
            os.path.join(out, f"snap_{tag}.npz"), t=t, x=g.x[ph[0]].cpu().numpy(),
            y=g.y[ph[1]].cpu().numpy(),
            **{k: st.prims[k][ph].double().cpu().numpy() for k in ("rho", "p", "vx", "vy", "Bx", "By")},
            divB=div_b(st.Bxf, st.Byf, g.dx, g.dy)[ph].cpu().numpy(),
            limiter=a.limiter, ng=g.ng, n=a.n, solver=a.solver)

    print(f"{a.problem} {a.n}^2  solver={a.solver}  emf={a.emf_mode}"
          f"{' (flux-CT)' if a.no_upwind_emf else ''}  limiter={a.limiter}  cfl={a.cfl}  "
          f"gamma={P['gamma']:.4f}  bc=({bc_x},{bc_y})  t_end={tend}  precision={a.precision}",
          flush=True)
    if a.restart:
        print(f"  restart from {a.restart}: t={float(R['t']):.6f} step={int(R['step'])} "
              f"generation={gen}", flush=True)
        log = open(os.path.join(out, "diag.csv"), "a")
    else:
        save("000", 0.0)
        log = open(os.path.join(out, "diag.csv"), "w")
        log.write("step,t,dt,divB_max,divB_l2,sym_err,rho_max,rho_min,p_min,"
                  "W_max,hlle_frac_x,hlle_frac_y,mean_iters,c2p_bad,"
                  "n_exact_x,n_verified_x\n")

    t, step, t0 = 0.0, 0, time.time()
    next_snap = 1
    if a.restart:
        t, step, next_snap = float(R["t"]), int(R["step"]), int(R["next_snap"])

    def save_restart():
        path = os.path.join(out, "restart.npz")
        tmp = path + ".tmp.npz"
        np.savez(tmp, t=t, step=step, next_snap=next_snap, gen=gen, limiter=a.limiter, ng=g.ng,
                 n=a.n, solver=a.solver, harvest_sweeps=0, Bxf=st.Bxf.cpu().numpy(),
                 Byf=st.Byf.cpu().numpy(),
                 **{"cons_" + k: st.cons[k].cpu().numpy() for k in EVOLVED_KEYS})
        os.replace(tmp, path)

    steps_here = 0
    diag = None
    while t < tend - 1e-14:
        dt = min(float(stepper.compute_dt(st, a.cfl).item()), tend - t)
        if not np.isfinite(dt) or dt <= 0.0:
            raise SystemExit(
                "run failed at step %d, t = %.6f: dt = %r.  The state went non-finite "
                "(rho_max %.3e, p_min %.3e); no snap_fin is written and the exit status is "
                "non-zero." % (step, t, dt, float(st.prims["rho"].max()), float(st.prims["p"].min())))
        stepper.step(st, dt, "rk3")
        diag = stepper.diag()
        t += dt
        step += 1
        if not np.isfinite(float(st.cons["D"].sum())):
            raise SystemExit("run failed at step %d, t = %.6f: the conserved state is not "
                             "finite.  No snap_fin is written and the exit status is non-zero."
                             % (step, t))
        steps_here += 1
        if step % max(1, a.log_every) == 0 or t >= tend - 1e-14:
            ph = g.phys
            d = div_b(st.Bxf, st.Byf, g.dx, g.dy)[ph]
            v2 = (st.prims["vx"][ph].double() ** 2 + st.prims["vy"][ph].double() ** 2
                  + st.prims["vz"][ph].double() ** 2)
            W = float((1.0 / torch.sqrt(torch.clamp(1 - v2, min=1e-16))).max())
            dx_, dy_ = diag["x"]["diag"], diag["y"]["diag"]
            c2p_bad = diag["c2p"]["not_converged"]
            sym = symmetry_error(st, g) if a.problem == "rotor" else float("nan")
            log.write(f"{step},{t:.6e},{dt:.3e},{float(d.abs().max()):.3e},"
                      f"{float(d.pow(2).mean().sqrt()):.3e},{sym:.3e},"
                      f"{float(st.prims['rho'][ph].max()):.4f},"
                      f"{float(st.prims['rho'][ph].min()):.4e},"
                      f"{float(st.prims['p'][ph].min()):.4e},{W:.3f},"
                      f"{dx_['frac_hlle_fallback']:.4f},{dy_['frac_hlle_fallback']:.4f},"
                      f"{dx_['mean_iters']:.2f},{c2p_bad},-1,-1\n")
            log.flush()
            extra = f"sym={sym:.2e} " if a.problem == "rotor" else ""
            print(f"  step {step:5d} t={t:.4f} dt={dt:.2e} divB={float(d.abs().max()):.2e} {extra}"
                  f"rho=[{float(st.prims['rho'][ph].min()):.3f},"
                  f"{float(st.prims['rho'][ph].max()):.3f}] c2p_bad={c2p_bad} "
                  f"({time.time()-t0:.0f}s)", flush=True)
        if t >= next_snap * tend / a.nsnap - 1e-14 and next_snap <= a.nsnap:
            save(f"{next_snap:03d}", t)
            next_snap += 1
        done = t >= tend - 1e-14
        if a.restart_every and step % a.restart_every == 0 and not done:
            save_restart()
        if a.max_steps is not None and steps_here >= a.max_steps and not done:
            save_restart()
            log.close()
            wall = time.time() - t0
            meta.update(steps=step, steps_here=steps_here, wall_s=round(wall, 1),
                        s_per_step=round(wall / max(steps_here, 1), 4), stopped_early=True,
                        finished=time.strftime("%Y-%m-%dT%H:%M:%S"))
            _write_meta(out, meta)
            print(f"stopped after {steps_here} steps at t={t:.6f} (step {step}); restart file "
                  f"written ({wall:.0f}s)", flush=True)
            return 0
    save("fin", t)
    log.close()
    wall = time.time() - t0
    meta.update(steps=step, steps_here=steps_here, wall_s=round(wall, 1),
                s_per_step=round(wall / max(steps_here, 1), 4),
                finished=time.strftime("%Y-%m-%dT%H:%M:%S"))
    _write_meta(out, meta)
    print(f"done in {wall:.0f}s, {step} steps -> {out}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
