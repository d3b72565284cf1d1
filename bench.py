"""Benchmark: 2D magnetic rotor, HLLD + PLM(MC) + SSP-RK3 + CT, zone-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 2048] [--precision mixed|fp64|fp64_exact]

One step is one full SSP-RK3 step (three stages, each: x and y sweeps, corner
EMF + update, sync) of the periodic tapered rotor on [0,1]^2 at n^2 cells,
preceded by the on-device CFL time step, with the state resident in HBM
(over 1 GB at 2048^2, far above the 126 MB L2, so no flush is needed).
`value` is the mixed-precision step (FP32 reconstruction/fluxes/update, FP64
C2P, p* iteration and RK state); the line also carries the FP64 step's rate
and the mixed-vs-FP64 density L1/Linf after the timed number of steps (same
dt sequence), the end-to-end rate through the public API with the state
copied host -> device and back every step (HostStepper2D: the copies on
their own streams, overlapped with the step), the roofline of the dominant
kernel (the fused sweep), the CPU baseline (the C oracle on the host cores)
and the SM clocks sampled during the timed region.

N > 1 (torchrun): every rank advances its own rotor replica (the reference
path has no domain decomposition; replicas only) and the rate is the sum
over ranks timed by the slowest rank.

The default line also carries, each in its own block:
  * ``fp64``: the FP64 step's rate, its share of faces without normal field
    and the 20-step density L1/Linf of the mixed run against it;
  * ``later_state``: both forms timed from the rotor at t = 0.2 (advanced
    untimed in the mixed form, then loaded into both);
  * ``fp32``: the all-FP32 step's rate and its 20-step density L1/Linf
    against FP64 at n^2 and (n/2)^2;
  * ``vortex``: the relativistic vortex (gamma 4/3) -- mixed and FP64 rates
    at n^2 and the L1/Linf of rho, p, |B|^2 at t = 0.5 at --vortex-n^2 of
    the mixed run and of a 1e-13-perturbed FP64 run against FP64;
  * ``tubes``: 4096 seeded tubes, mixed and FP64 cell-updates/s, the tube
    kernel's roofline, and the density L1 against the oracle of a seeded
    subset advanced to t = 0.3;
  * ``adjoint``: the rotor gradient study's adjoint/forward cost.

Workloads of their own (``--workload``): ``tubes`` (the tube block alone;
``--tube-shape`` fixes the launch shape), ``adjoint``, ``vortex`` (the
vortex block at --n / --vortex-n) and ``rotor_run`` (whole rotor runs to
--tend in the mixed, FP32 and FP64 forms on the FP64 dt sequence, each
form's mean rate and density L1/Linf against FP64, beside an untimed FP64
run from a 1e-13-perturbed state).

``--impl reference`` times the CPU oracle (a C restatement of the
reference's FP64 path) on the host cores with all threads, one RK3 step of
the same rotor at 1024^2 (``--cpu-n``) per step as a bounded sample.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PROBLEM = "rotor_tapered"
WORKLOAD = "magnetic rotor 2D, periodic [0,1]^2, gamma 5/3, HLLD + PLM(MC, Wv) + SSP-RK3 + CT"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "fp64_exact"])
    ap.add_argument("--no-fp64-arm", action="store_true",
                    help="skip timing the FP64 step and the mixed-vs-FP64 L1 check")
    ap.add_argument("--cfl", type=float, default=0.4)
    ap.add_argument("--t-start", type=float, default=0.0,
                    help="advance the rotor to this time (untimed) before the warm-up")
    ap.add_argument("--cpu-n", type=int, default=1024, help="grid of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint/forward cost of the 512^2 rotor gradient study")
    ap.add_argument("--workload", default="rotor",
                    choices=["rotor", "tubes", "adjoint", "vortex", "rotor_run"],
                    help="rotor: the 2D rotor step (default); tubes: the batched-tube launch; "
                         "adjoint: the rotor gradient study alone (adjoint/forward cost); "
                         "vortex: the vortex block alone (--vortex-n, --vortex-tend); "
                         "rotor_run: whole rotor runs to --tend in every precision")
    ap.add_argument("--tend", type=float, default=0.4, help="rotor_run: end time")
    ap.add_argument("--adjoint-n", type=int, default=512)
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--adjoint-every", type=int, default=20, help="checkpoint interval")
    ap.add_argument("--tubes", type=int, default=4096)
    ap.add_argument("--tube-shape", default=None,
                    help="threads,CTAs-per-SM of the tubes workload's launch instead of the "
                         "autotuner's pick (e.g. 512,1; for profiling a fixed shape)")
    ap.add_argument("--chunk", type=float, default=0.01,
                    help="tubes: simulated time every tube advances per step")
    ap.add_argument("--cpu-tubes", type=int, default=30, help="tubes of the CPU baseline sample")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the later_state, fp32, vortex and tubes blocks of the default line")
    ap.add_argument("--t-later", type=float, default=0.2, help="rotor time of the later_state block")
    ap.add_argument("--vortex-n", type=int, default=1024,
                    help="grid of the vortex block's t = 0.5 precision study")
    ap.add_argument("--vortex-tend", type=float, default=0.5)
    ap.add_argument("--tube-check", type=int, default=30,
                    help="seeded tubes of the tube block's accuracy check against the oracle")
    ap.add_argument("--tube-tend", type=float, default=0.3)
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


# ── clocks sampled during the timed region ───────────────────────────────────

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ── CPU baseline: the oracle on the host cores ───────────────────────────────

def cpu_sample(n: int, steps: int, threads: int):
    """zone-updates/s of the oracle's RK3 step on the rotor at n^2."""
    from oracle import oracle
    from hlld_ai_b200.physics.initial_data2d import b_from_potential, initial_prims
    from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS

    oracle.set_threads(threads)
    g, eos, prims, Az, spec = initial_prims(PROBLEM, n, 2, "cpu")
    prims = {k: v.contiguous().numpy().copy() for k, v in prims.items()}
    Bxf, Byf = b_from_potential(Az, g.dx, g.dy)
    cons = oracle.prim_to_cons(prims)
    st = {"cons": {k: cons[k].copy() for k in EVOLVED_KEYS},
          "Bxf": Bxf.contiguous().numpy().copy(), "Byf": Byf.contiguous().numpy().copy(),
          "prims": {k: prims[k].copy() for k in PRIM_KEYS}}
    og = oracle.Grid2DSpec(n, n, 2, g.dx, g.dy, *spec["bc"], "mc", "hlld", spec["gamma"])
    oracle.sync_state(og, st)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        dt = oracle.compute_dt_2d(og, st["prims"], 0.4)
        oracle.rk_step_ct(og, st, dt, "rk3")
        times.append(time.perf_counter() - t0)
    return times


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    cpu_sample(a.cpu_n, max(1, a.warmup), threads)  # warm-up
    times = cpu_sample(a.cpu_n, a.steps, threads)
    zu = a.cpu_n * a.cpu_n
    value = zu * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": a.n, "sample_n": a.cpu_n,
                   "l2": "inputs exceed L2"},
        "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": threads,
                         "kind": "port",
                         "sample": f"one RK3 step of the same rotor at {a.cpu_n}^2 per step "
                                   f"({zu} zone-updates), C oracle, {threads} threads"},
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ── our arm ──────────────────────────────────────────────────────────────────

def _timed_rotor(a, precision, rp, record=True):
    """Set up the rotor at a.n^2 in `precision`, run a.warmup steps, then time
    a.steps steps between CUDA events; returns a dict of results."""
    import torch

    import hlld_ai_b200 as H
    from hlld_ai_b200 import _lib, replicas

    dev = rp.device
    g, eos, st, spec = H.setup_problem(PROBLEM, a.n, limiter="mc", device=dev,
                                       precision=precision)
    stepper = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld",
                          limiter="mc", precision=precision)
    t = 0.0
    while t < a.t_start:  # untimed: a later state of the same run
        dt_t = stepper.compute_dt(st, a.cfl)
        stepper.step(st, dt_t, "rk3")
        t += float(dt_t.item())
    s = stepper._struct(st)
    gc = stepper.gc
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    # component buffers of the instrumented step (same kernels as hlld_rk_step_ct)
    nfx, nfy = (g.nxt + 1) * g.nyt, g.nxt * (g.nyt + 1)
    rdt = torch.float32 if precision == "mixed" else torch.float64
    f64 = dict(dtype=torch.float64, device=dev)
    Fx = [torch.empty(nfx, dtype=rdt, device=dev) for _ in range(7)]
    Fy = [torch.empty(nfy, dtype=rdt, device=dev) for _ in range(7)]
    Ez = torch.empty((g.nxt + 1) * (g.nyt + 1), dtype=rdt, device=dev)
    U0 = [torch.empty(g.nxt * g.nyt, **f64) for _ in range(6)]
    Bx0, By0 = torch.empty(nfx, **f64), torch.empty(nfy, **f64)
    diag = torch.zeros(ctypes.sizeof(_lib.StepDiag), dtype=torch.uint8, device=dev)
    # the mixed form's C2P roots of the step's first stage (as hlld_rk_step_ct:
    # stage 1 starts from the input primitives, stages 2 and 3 from its roots)
    mu = torch.zeros(g.nxt * g.nyt, dtype=torch.float64, device=dev) if precision == "mixed" else None
    fd_off = ctypes.sizeof(_lib.FluxDiag)
    pFx, pFy, pU0 = _lib.ptr_array(Fx), _lib.ptr_array(Fy), _lib.ptr_array(U0)
    dt = stepper.dt_buf
    sweep_events = []

    def step(rec=False):
        stepper.compute_dt(st, a.cfl, out=dt)
        for stage in range(3):
            for axis, pF in ((0, pFx), (1, pFy)):
                if rec:
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                _lib.check(L.hlld_sweep2d(ctypes.byref(gc), ctypes.byref(s), axis, pF,
                                          diag.data_ptr() + axis * fd_off, sh), "sweep2d")
                if rec:
                    e1.record(stream)
                    sweep_events.append((e0, e1))
            _lib.check(L.hlld_ct_update2d(ctypes.byref(gc), ctypes.byref(s), pFx, pFy,
                                          Ez.data_ptr(), pU0, Bx0.data_ptr(), By0.data_ptr(),
                                          diag.data_ptr(), stage, 3, 0.0, dt.data_ptr(), sh),
                       "ct_update2d")
            if mu is None:
                _lib.check(L.hlld_sync_state(ctypes.byref(gc), ctypes.byref(s), None, None, sh),
                           "sync_state")
            elif stage == 0:  # C2P started from the step's input primitives
                _lib.check(L.hlld_sync_state_from_prims(ctypes.byref(gc), ctypes.byref(s), None,
                                                        None, mu.data_ptr(), sh),
                           "sync_state_from_prims")
            else:  # started from the roots of stage 1
                _lib.check(L.hlld_sync_state_roots(ctypes.byref(gc), ctypes.byref(s), None, None,
                                                   None, mu.data_ptr(), sh),
                           "sync_state_roots")

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize(dev)
    replicas.barrier(rp)
    clocks = ClockSampler(dev.index or 0) if record else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    torch.cuda.synchronize(dev)
    replicas.barrier(rp)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(a.steps):
        step(rec=True)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    replicas.barrier(rp)
    clk = clocks.stop() if clocks else None
    value, ms = replicas.job_rate(rp, g.nx * g.ny * a.steps, t0.elapsed_time(t1))
    sweep_ms = [e0.elapsed_time(e1) for e0, e1 in sweep_events]
    # share of faces without normal field (HLLE fallback, no p* solve in the
    # mixed form) in the last timed stage's x and y sweeps
    d = _lib.StepDiag.from_buffer_copy(diag.cpu().numpy().tobytes())
    bn0 = [d.sweep[k].n_bn_zero / max(d.sweep[k].n_faces, 1) for k in (0, 1)]
    return dict(g=g, eos=eos, st=st, spec=spec, stepper=stepper, ms=ms, sweep_ms=sweep_ms,
                clocks=clk, faces=(nfx + nfy) / 2.0, value=value, bn_zero_share=bn0)


def _l1_mixed_vs_fp64(a, dev, steps):
    """Density L1 (mean |rho_mixed - rho_fp64| over physical cells) after
    `steps` RK3 steps from the same initial state with the FP64 run's dt."""
    import torch

    import hlld_ai_b200 as H

    res = {}
    runs = {}
    for prec in ("fp64", "mixed"):
        g, eos, st, spec = H.setup_problem(PROBLEM, a.n, limiter="mc", device=dev, precision=prec)
        runs[prec] = (g, st, H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1],
                                         flux_fn="hlld", limiter="mc", precision=prec))
    g = runs["fp64"][0]
    for _ in range(steps):
        dt = float(runs["fp64"][2].compute_dt(runs["fp64"][1], a.cfl).item())
        for prec in ("fp64", "mixed"):
            runs[prec][2].step(runs[prec][1], dt, "rk3")
    ph = g.phys
    r64 = runs["fp64"][1].prims["rho"][ph]
    rmx = runs["mixed"][1].prims["rho"][ph].double()
    d = (rmx - r64).abs()
    res["l1_rho"] = float(d.mean())
    res["linf_rho"] = float(d.max())
    res["l1_rho_rel"] = float(d.mean() / r64.abs().mean())
    res["steps"] = steps
    del runs
    torch.cuda.empty_cache()
    return res


# DRAM bytes (read + write) of one mixed-precision sweep launch measured by
# ncu on the rotor at 1536^2 (x: 95.11 + 44.85 MB, y: 95.37 + 42.32 MB over
# 2,373,140 faces each; profiles/sweep_kernel_rotor1536_mixed_ncu.md), per
# face; the 2048^2 launch is scaled by its faces
_SWEEP_DRAM_BYTES_PER_FACE_MIXED = (139.96e6 + 137.69e6) / 2 / 2373140
# FP64-pipe instructions (warp level) of the same two launches, per face
_SWEEP_FP64_INST_PER_FACE_MIXED = (114.87e6 + 7.05e6) / 2 / 2373140
# FP64 issue rate of one B200 SM: 2 warp instructions per cycle (64 lanes;
# an earlier capture's 126.1 M FP64 instructions at 35.0 % of peak
# sustained over 637 us at 1965 MHz on 148 SMs give 1.94)
_FP64_WARP_INST_PER_SM_CYCLE = 2


# DRAM bytes (read + write) of one mixed-precision tubes_kernel launch
# measured by ncu (2048 seeded tubes, chunk 0.0005, 512 threads x 148 CTAs:
# 3.329 + 6.225 GB over 2.129e7 cell-updates;
# profiles/tubes_kernel_2048tubes_ncu.md), per cell-update; a launch is
# scaled by its updates
_TUBES_DRAM_BYTES_PER_UPDATE_MIXED = (3.329e9 + 6.225e9) / 2.129e7


def _sweep_traffic(a):
    if a.precision != "mixed":
        return None
    nt = a.n + 4
    return _SWEEP_DRAM_BYTES_PER_FACE_MIXED * (nt + 1) * nt


def _time_public(stepper, st, steps, warmup, cfl, rp):
    """Mean ms per step of the on-device CFL dt + one RK3 step through the
    public Stepper2D, after `warmup` steps (CUDA events on the current
    stream, the slowest rank's time); also the share of faces without normal
    field in the last stage's x and y sweeps."""
    import torch

    from hlld_ai_b200 import _lib, replicas

    dev = stepper.device
    for _ in range(warmup):
        stepper.step(st, stepper.compute_dt(st, cfl), "rk3")
    torch.cuda.synchronize(dev)
    replicas.barrier(rp)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        stepper.step(st, stepper.compute_dt(st, cfl), "rk3")
    e1.record(stream)
    torch.cuda.synchronize(dev)
    (ms,) = replicas.max_over_ranks(rp, e0.elapsed_time(e1))
    d = _lib.StepDiag.from_buffer_copy(stepper.diag_buf.cpu().numpy().tobytes())
    bn0 = [d.sweep[k].n_bn_zero / max(d.sweep[k].n_faces, 1) for k in (0, 1)]
    return ms / steps, bn0


def _stepper(problem, n, precision, dev):
    import hlld_ai_b200 as H

    g, eos, st, spec = H.setup_problem(problem, n, limiter="mc", device=dev, precision=precision)
    stp = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld",
                      limiter="mc", precision=precision)
    return g, st, stp


def _l1_vs_fp64(a, dev, steps, n, precision):
    """Density L1 / Linf (mean / max |rho - rho_fp64| over physical cells) of
    `precision` against FP64 after `steps` RK3 steps of the rotor from the
    same initial state with the FP64 run's dt, and the C2P and fallback
    counters of the last step."""
    import torch

    runs = {p: _stepper(PROBLEM, n, p, dev) for p in ("fp64", precision)}
    for _ in range(steps):
        dt = float(runs["fp64"][2].compute_dt(runs["fp64"][1], a.cfl).item())
        for p in runs:
            runs[p][2].step(runs[p][1], dt, "rk3")
    g = runs["fp64"][0]
    r64 = runs["fp64"][1].prims["rho"][g.phys]
    d = (runs[precision][1].prims["rho"][g.phys].double() - r64).abs()
    diag = runs[precision][2].diag()
    out = {"n": n, "steps": steps, "l1_rho": float(d.mean()), "linf_rho": float(d.max()),
           "l1_rho_rel": float(d.mean() / r64.abs().mean()),
           "c2p_not_converged": diag["c2p"]["not_converged"], "c2p_atmo": diag["c2p"]["atmo"],
           "hlle_fallback_frac": {"x": diag["x"]["diag"]["frac_hlle_fallback"],
                                  "y": diag["y"]["diag"]["frac_hlle_fallback"]}}
    del runs
    torch.cuda.empty_cache()
    return out


def _later_state_block(a, rp, dev):
    """Both forms timed from the rotor at t = a.t_later: the mixed run is
    advanced there untimed, its FP64 conserved state and staggered field are
    loaded into an FP64 stepper, then each form is timed a.steps steps."""
    import torch

    from hlld_ai_b200.physics.state import EVOLVED_KEYS, State2D

    g, st, stp = _stepper(PROBLEM, a.n, "mixed", dev)
    t, nsteps = 0.0, 0
    while t < a.t_later:
        dt = stp.compute_dt(st, a.cfl)
        stp.step(st, dt, "rk3")
        t += float(dt.item())
        nsteps += 1
    snap = State2D(cons={k: st.cons[k].clone() for k in EVOLVED_KEYS}, Bxf=st.Bxf.clone(),
                   Byf=st.Byf.clone(), prims={})
    ms_mx, bn_mx = _time_public(stp, st, a.steps, a.warmup, a.cfl, rp)
    del st, stp
    torch.cuda.empty_cache()
    g64, st64, stp64 = _stepper(PROBLEM, a.n, "fp64", dev)
    del st64
    stp64.sync(snap)
    ms_64, bn_64 = _time_public(stp64, snap, a.steps, a.warmup, a.cfl, rp)
    del snap, stp64
    torch.cuda.empty_cache()
    zones = a.n * a.n * rp.world
    return {"t": t, "steps_to_reach": nsteps,
            "mixed": {"ms_per_step": ms_mx, "value": zones / (ms_mx * 1e-3),
                      "bn_zero_face_share": {"x": bn_mx[0], "y": bn_mx[1]}},
            "fp64": {"ms_per_step": ms_64, "value": zones / (ms_64 * 1e-3),
                     "bn_zero_face_share": {"x": bn_64[0], "y": bn_64[1]}},
            "mixed_speedup": ms_64 / ms_mx,
            "note": "both forms from the same state at t (the mixed run's), each timed through "
                    "Stepper2D.step + compute_dt"}


def _fp32_block(a, rp, dev):
    import torch

    g, st, stp = _stepper(PROBLEM, a.n, "fp32", dev)
    ms, bn0 = _time_public(stp, st, a.steps, a.warmup, a.cfl, rp)
    del st, stp
    torch.cuda.empty_cache()
    zones = a.n * a.n * rp.world
    return {"ms_per_step": ms, "value": zones / (ms * 1e-3),
            "bn_zero_face_share": {"x": bn0[0], "y": bn0[1]},
            "vs_fp64": [_l1_vs_fp64(a, dev, 20, n, "fp32") for n in (a.n, a.n // 2)]}


def _vortex_block(a, rp, dev):
    """Config 3: the relativistic vortex.  Rates of the mixed and FP64 steps
    at a.n^2; at a.vortex_n^2 to t = a.vortex_tend the L1 / Linf of rho, p
    and |B|^2 of the mixed run and of an FP64 run whose initial D and tau
    carry 1e-13 relative noise, both against FP64 (same dt sequence)."""
    import torch

    zones = a.n * a.n * rp.world
    rates = {}
    for prec in ("mixed", "fp64"):
        g, st, stp = _stepper("vortex", a.n, prec, dev)
        ms, _ = _time_public(stp, st, max(5, a.steps // 2), a.warmup, a.cfl, rp)
        rates[prec] = {"ms_per_step": ms, "value": zones / (ms * 1e-3)}
        del st, stp
        torch.cuda.empty_cache()
    n = a.vortex_n
    runs = {p: _stepper("vortex", n, p, dev) for p in ("fp64", "mixed")}
    g, pert, sp = _perturbed_fp64("vortex", n, dev)
    t, steps = 0.0, 0
    while t < a.vortex_tend - 1e-14:
        dt = min(float(runs["fp64"][2].compute_dt(runs["fp64"][1], a.cfl).item()), a.vortex_tend - t)
        for p in runs:
            runs[p][2].step(runs[p][1], dt, "rk3")
        sp.step(pert, dt, "rk3")
        t += dt
        steps += 1
    ph = g.phys
    fields = {"rho": lambda P: P["rho"][ph].double(), "p": lambda P: P["p"][ph].double(),
              "B2": lambda P: sum(P[k][ph].double() ** 2 for k in ("Bx", "By", "Bz"))}
    ref = runs["fp64"][1].prims

    def norms(P):
        out = {}
        for name, f in fields.items():
            d = (f(P) - f(ref)).abs()
            out[name] = {"l1": float(d.mean()), "linf": float(d.max())}
        return out

    res = {"n_rates": a.n, "mixed": rates["mixed"], "fp64": rates["fp64"],
           "mixed_speedup": rates["fp64"]["ms_per_step"] / rates["mixed"]["ms_per_step"],
           "study": {"n": n, "t": t, "steps": steps,
                     "mixed_vs_fp64": norms(runs["mixed"][1].prims),
                     "fp64_perturbed_1e-13_vs_fp64": norms(pert.prims)}}
    del runs, pert, sp
    torch.cuda.empty_cache()
    return res


def _oracle_tubes(states, idx, tend, threads):
    """Primitives of tubes `idx` advanced to tend by the oracle (one tube per
    host thread; the C call releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle
    from hlld_ai_b200.tubes import tube_prims

    def one(i):
        p = tube_prims(states, i, 3)
        L = int(states.lengths[i])
        oracle.tube_run(p, L, 3, 1.0 / L, 0.4, tend, "weno5z", "hlld", 5.0 / 3.0)
        return p

    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(one, idx))


def _tubes_block(a, rp, dev):
    """Config 4: 4096 seeded tubes.  Mixed and FP64 cell-updates/s (graph
    replays advancing every tube by a.chunk) and the L1 of rho against the
    oracle on a seeded subset of a.tube_check tubes advanced to a.tube_tend."""
    import numpy as np
    import torch

    from hlld_ai_b200 import replicas
    from hlld_ai_b200.tubes import TubeBatch, TubeStates, random_tubes

    states = random_tubes(a.tubes, seed=replicas.replica_seed(20261203, rp))
    L = torch.as_tensor(states.lengths, dtype=torch.int64, device=dev)
    peak, kind = peaks()
    out = {"workload": TUBES_WORKLOAD, "tubes": a.tubes, "chunk": a.chunk}
    for prec in ("mixed", "fp64"):
        b = TubeBatch(states, limiter="weno5z", solver="hlld", scheme="rk3", precision=prec,
                      device=dev)
        tuned = b.autotune(tend=a.chunk / 4, sample=512)
        g = b.capture(tend=a.chunk)
        b.reset()
        g.replay()  # warm-up
        torch.cuda.synchronize(dev)
        reps = 3 if prec == "mixed" else 2
        stream = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        acc = torch.zeros(a.tubes, dtype=torch.int64, device=dev)
        e0.record(stream)
        for _ in range(reps):
            g.replay()
            acc += b.steps_out
        e1.record(stream)
        torch.cuda.synchronize(dev)
        (ms,) = replicas.max_over_ranks(rp, e0.elapsed_time(e1))
        (updates,) = replicas.sum_over_ranks(rp, float((acc * L).sum().item()))
        rb = 4 if prec == "mixed" else 8
        per_launch = updates / rp.world / reps
        bytes_per_update = 3 * (14 * rb + 14 * 8) + 2 * 7 * 8
        achieved = bytes_per_update * per_launch / (ms / reps * 1e-3) / 1e9
        out[prec] = {"value": updates / (ms * 1e-3), "unit": "cell-updates/s",
                     "ms_per_launch": ms / reps, "threads": tuned[0], "blocks": tuned[1],
                     "roofline": {"bound": "hbm", "achieved": achieved, "unit": "GB/s",
                                  "peak": peak, "peak_kind": kind, "frac": achieved / peak,
                                  "bytes_per_cell_update": bytes_per_update}}
        del b, g
        torch.cuda.empty_cache()
    out["mixed"]["roofline"]["traffic_per_cell_update"] = _TUBES_DRAM_BYTES_PER_UPDATE_MIXED
    out["mixed"]["roofline"]["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                                  "of the mixed launch on 2048 tubes")
    out["mixed_speedup"] = out["mixed"]["value"] / out["fp64"]["value"]
    # accuracy: a seeded subset to t = a.tube_tend against the oracle
    rng = np.random.default_rng(7)
    idx = sorted(rng.choice(a.tubes, size=min(a.tube_check, a.tubes), replace=False).tolist())
    sub = TubeStates(states.lengths[idx], {k: v[idx] for k, v in states.left.items()},
                     {k: v[idx] for k, v in states.right.items()}, states.Bx[idx])
    ref = _oracle_tubes(sub, list(range(len(idx))), a.tube_tend, os.cpu_count() or 1)
    check = {"tubes": len(idx), "t": a.tube_tend, "seed": 7}
    for prec in ("mixed", "fp64"):
        b = TubeBatch(sub, limiter="weno5z", solver="hlld", scheme="rk3", precision=prec,
                      device=dev)
        b.launch(tend=a.tube_tend)
        torch.cuda.synchronize(dev)
        errs = []
        for i in range(len(idx)):
            got, want = b.tube(i)["rho"][3:-3], ref[i]["rho"][3:-3]
            errs.append(float(np.abs(got - want).mean() / np.abs(want).mean()))
        check[prec] = {"l1_rho_rel_median": float(np.median(errs)),
                       "l1_rho_rel_max": float(np.max(errs))}
        del b
    out["vs_oracle"] = check
    return out


def run_ours(a):
    import torch

    import hlld_ai_b200 as H
    from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS

    from hlld_ai_b200 import replicas

    rp = replicas.from_env("cuda")
    world, rank, local, dev = rp.world, rp.rank, rp.local, rp.device
    torch.cuda.set_device(local)
    replicas.init(rp)

    main = _timed_rotor(a, a.precision, rp, record=True)
    g, st, stepper = main["g"], main["st"], main["stepper"]
    ms, zones = main["ms"], g.nx * g.ny
    value = main["value"]
    clk = main["clocks"]
    bn0 = main["bn_zero_share"]
    launches_per_step = 2 + 3 * 9  # speed + dt; per stage 2 sweeps, emf, update, 2 face ghosts, cons ghosts, c2p, prim ghosts

    # roofline of the dominant kernel (fused sweep), timed inside the region
    sweep_ms = main["sweep_ms"]
    sweep_avg_s = 1e-3 * sum(sweep_ms) / len(sweep_ms)
    rb = 4 if a.precision == "mixed" else 8
    # algorithmic bytes per face: 6 primitives (R) + 2 face-B words (FP64)
    # read per cell, 7 flux words (R) written per face
    bytes_per_face = 6 * rb + 2 * 8 + 7 * rb
    achieved = bytes_per_face * main["faces"] / sweep_avg_s / 1e9
    peak, peak_kind = peaks()
    sweep_share = sum(sweep_ms) / ms
    # the compute side: FP64-pipe instructions per launch (ncu, scaled by
    # faces) over the launch time, against the SMs' FP64 issue rate at the
    # median SM clock sampled during the timed region
    fp64_pipe = None
    if a.precision == "mixed" and clk and clk.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        inst = _SWEEP_FP64_INST_PER_FACE_MIXED * main["faces"]
        rate = inst / sweep_avg_s
        peak_rate = sms * _FP64_WARP_INST_PER_SM_CYCLE * clk["sm_mhz"] * 1e6
        fp64_pipe = {"inst_per_launch": inst, "achieved_inst_per_s": rate,
                     "peak_inst_per_s": peak_rate, "frac": rate / peak_rate,
                     "source": "ncu sm__inst_executed_pipe_fp64.sum of the mixed sweeps at "
                               "1536^2 scaled by faces; peak 2 FP64 warp instructions per SM "
                               "cycle at the sampled SM clock"}

    fp64_arm = None
    if a.precision == "mixed" and not a.no_fp64_arm:
        del main
        torch.cuda.empty_cache()
        r64 = _timed_rotor(a, "fp64", rp, record=False)
        fp64_arm = {"value": r64["value"], "ms_per_step": r64["ms"] / a.steps,
                    "mixed_speedup": value / r64["value"],
                    "bn_zero_face_share": {"x": r64["bn_zero_share"][0],
                                           "y": r64["bn_zero_share"][1]}}
        del r64
        torch.cuda.empty_cache()
        fp64_arm.update(_l1_mixed_vs_fp64(a, dev, a.steps))
        g, eos, st, spec = H.setup_problem(PROBLEM, a.n, limiter="mc", device=dev,
                                           precision=a.precision)
        stepper = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld",
                              limiter="mc", precision=a.precision)
    stream = torch.cuda.current_stream(dev)

    # end to end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        from hlld_ai_b200 import HostStepper2D
        from hlld_ai_b200.physics.state import State2D

        host = State2D(cons={k: st.cons[k].cpu().pin_memory() for k in EVOLVED_KEYS},
                       Bxf=st.Bxf.cpu().pin_memory(), Byf=st.Byf.cpu().pin_memory(),
                       prims={k: st.prims[k].cpu().pin_memory() for k in PRIM_KEYS})
        hs = HostStepper2D(stepper, host)
        h2d, d2h = hs.bytes_per_step()
        ke = max(3, min(a.steps, 8))
        torch.cuda.synchronize(dev)
        replicas.barrier(rp)
        # Every step copies the whole state (faces, primitives, conserved
        # arrays) from pinned host memory and the whole result back, through
        # HostStepper2D: the copies run on their own streams, the step starts
        # once the faces and primitives are in, and the copy-in of an array
        # for step k + 1 follows the copy-out of the same array from step k.
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ke):
            hs.step(a.cfl, "rk3")
        hs.synchronize()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_rate, ems = replicas.job_rate(rp, zones * ke, e0.elapsed_time(e1))
        e2e = {"value": e2e_rate, "unit": "zone-updates/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "steps": ke, "path": "HostStepper2D.step (Stepper2D.step + compute_dt) on a pinned "
                       "host state; copies on their own streams, overlapped with the step"}
        del hs, host

    # the adjoint's cost against the forward (the rotor gradient study: 512^2,
    # 200 FP64 SSP-RK3 steps, checkpoints every 20, J = sum w |B|^2 / 2)
    adj = None
    if not a.no_adjoint:
        torch.cuda.empty_cache()
        runs = _adjoint_runs(a, dev, 3)
        ratios = [r["adjoint_ms"] / r["forward_ms"] for r in runs]
        mid = runs[ratios.index(statistics.median(ratios))]
        adj = {"workload": _adjoint_workload(a) + " (the run with the median ratio of 3)",
               "forward_ms": mid["forward_ms"], "adjoint_ms": mid["adjoint_ms"],
               "adjoint_over_forward": statistics.median(ratios),
               "J": mid["J"], "dJ_domega": mid["grad_omega"]}

    extra = {}
    if not a.no_extra:
        del st, stepper
        torch.cuda.empty_cache()
        extra["later_state"] = _later_state_block(a, rp, dev)
        extra["fp32"] = _fp32_block(a, rp, dev)
        extra["vortex"] = _vortex_block(a, rp, dev)
        extra["tubes"] = _tubes_block(a, rp, dev)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cpu_sample(a.cpu_n, 1, threads)
        times = cpu_sample(a.cpu_n, 6, threads)  # ~10 s of CPU work at 1024^2
        cpu = {"value": a.cpu_n ** 2 * len(times) / sum(times), "unit": "zone-updates/s",
               "cores": threads, "kind": "port",
               "sample": f"{len(times)} RK3 steps of the same rotor at {a.cpu_n}^2, after one "
                         f"untimed step (C oracle, FP64, {threads} threads)"}

    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": a.n, "precision": a.precision,
                       "t_start": a.t_start,
                       "parallelism": f"replicas x{world}", "cfl": a.cfl,
                       "l2": "inputs exceed L2 (state >1 GB at 2048^2), no flush",
                       "bn_zero_face_share": {"x": bn0[0], "y": bn0[1]}},
            "fp64": fp64_arm,
            **extra,
            "adjoint": adj,
            "e2e": e2e,
            "gpu_launches": launches_per_step * a.steps,
            "roofline": {"bound": "hbm", "kernel": "sweep_kernel (x and y)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": _sweep_traffic(a), "traffic_unit": "bytes per launch",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of the mixed sweep at 1536^2, scaled by faces",
                         "bytes_per_face": bytes_per_face,
                         "avg_launch_ms": sweep_avg_s * 1e3, "share_of_step": sweep_share,
                         "fp64_pipe": fp64_pipe},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    replicas.finish(rp)
    return 0


# ── batched tubes ────────────────────────────────────────────────────────────

TUBES_WORKLOAD = ("batched 1D SRMHD tubes, lengths uniform in [256, 4096], seeded left/right "
                  "states, gamma 5/3, WENO5-Z + HLLD + SSP-RK3, per-tube CFL 0.4 dt")


def tubes_cpu_sample(states, ntubes, chunk):
    """cell-updates/s of the oracle advancing a seeded subset of the tubes by
    `chunk` (one tube at a time, one thread)."""
    from oracle import oracle
    from hlld_ai_b200.tubes import tube_prims

    idx = list(range(0, len(states.lengths), max(1, len(states.lengths) // ntubes)))[:ntubes]
    work, secs = 0, 0.0
    for i in idx:
        p = tube_prims(states, i, 3)
        L = int(states.lengths[i])
        t0 = time.perf_counter()
        _, steps = oracle.tube_run(p, L, 3, 1.0 / L, 0.4, chunk, "weno5z", "hlld", 5.0 / 3.0)
        secs += time.perf_counter() - t0
        work += L * steps
    return work / secs, len(idx), work


def run_tubes(a):
    """One step = one replay of the CUDA graph holding the persistent launch,
    which advances every tube by `chunk` of simulated time (each tube with its
    own CFL steps).  value = physical cell-updates (cells x RK3 steps summed
    over tubes) per second."""
    import torch

    from hlld_ai_b200 import replicas
    from hlld_ai_b200.tubes import TubeBatch, random_tubes

    rp = replicas.from_env("cuda")
    world, rank, local, dev = rp.world, rp.rank, rp.local, rp.device
    torch.cuda.set_device(local)
    replicas.init(rp)
    # tubes are independent units: each rank runs its own seeded batch
    states = random_tubes(a.tubes, seed=replicas.replica_seed(20261203, rp))
    precision = "mixed" if a.precision == "mixed" else a.precision
    b = TubeBatch(states, limiter="weno5z", solver="hlld", scheme="rk3", precision=precision,
                  device=dev)
    if a.tube_shape:
        threads, per_sm = (int(v) for v in a.tube_shape.split(","))
        b.threads = threads
        b.blocks = per_sm * torch.cuda.get_device_properties(dev).multi_processor_count
    else:
        b.autotune(tend=a.chunk / 4, sample=1024)
    g = b.capture(tend=a.chunk)
    b.reset()
    L = torch.as_tensor(states.lengths, dtype=torch.int64, device=dev)
    acc = torch.zeros(a.tubes, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(a.warmup):
        g.replay()
    torch.cuda.synchronize(dev)
    replicas.barrier(rp)
    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    e0.record(stream)
    for _ in range(a.steps):
        k0.record(stream)
        g.replay()
        k1.record(stream)
        acc += b.steps_out
        k1.synchronize()
        kernel_ms.append(k0.elapsed_time(k1))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    replicas.barrier(rp)
    clk = clocks.stop()
    # the batches differ per rank: total work over the slowest rank's time
    (ms,) = replicas.max_over_ranks(rp, e0.elapsed_time(e1))
    (updates,) = replicas.sum_over_ranks(rp, float((acc * L).sum().item()))
    updates = int(updates)
    value = updates / (ms * 1e-3)
    # algorithmic bytes per cell-update: per stage read P (7 words, storage
    # precision) and U (7 FP64), write both; stages 2 and 3 also read U0
    rb = 4 if precision == "mixed" else 8
    bytes_per_update = 3 * (14 * rb + 14 * 8) // 1 + 2 * 7 * 8
    kernel_s = 1e-3 * sum(kernel_ms) / len(kernel_ms)
    achieved = bytes_per_update * (updates / world / a.steps) / kernel_s / 1e9
    peak, peak_kind = peaks()

    # end to end: host primitives -> device, the launch, primitives -> host
    host = {k: torch.empty_like(v, device="cpu").pin_memory() for k, v in b.prims.items()}
    for k, v in b.prims.items():
        host[k].copy_(v)
    nbytes = sum(h.numel() * h.element_size() for h in host.values())
    ke = max(1, min(a.steps, 3))
    acc.zero_()
    torch.cuda.synchronize(dev)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(ke):
        for k, v in b.prims.items():
            v.copy_(host[k], non_blocking=True)
        b.launch(tend=a.chunk)
        acc += b.steps_out
        for k, v in b.prims.items():
            host[k].copy_(v, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize(dev)
    (e2e_updates,) = replicas.sum_over_ranks(rp, float((acc * L).sum().item()))
    (e2e_ms,) = replicas.max_over_ranks(rp, f0.elapsed_time(f1))
    e2e = {"value": e2e_updates / (e2e_ms * 1e-3), "unit": "cell-updates/s",
           "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": ke,
           "path": "TubeBatch.launch with pinned host primitives"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, nt, work = tubes_cpu_sample(states, a.cpu_tubes, a.chunk)
        cpu = {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"{nt} of the tubes advanced by {a.chunk} ({work} cell-updates), "
                         "C oracle, one thread"}
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": TUBES_WORKLOAD, "tubes": a.tubes, "chunk": a.chunk,
                       "precision": precision, "threads": b.threads, "blocks": b.blocks,
                       "total_cells": b.total_cells, "parallelism": f"replicas x{world}",
                       "l2": "state of the batch above L2 (~0.7 GB), no flush"},
            "e2e": e2e,
            "gpu_launches": a.steps,
            "roofline": {"bound": "hbm", "kernel": "tubes_kernel", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind,
                         "traffic": (_TUBES_DRAM_BYTES_PER_UPDATE_MIXED * updates / world / a.steps
                                     if precision == "mixed" else None),
                         "traffic_unit": "bytes per launch",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                                           "the mixed launch on 2048 tubes, scaled by "
                                           "cell-updates",
                         "bytes_per_cell_update": bytes_per_update,
                         "avg_launch_ms": kernel_s * 1e3},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    replicas.finish(rp)
    return 0


def _adjoint_runs(a, dev, count):
    """`count` runs of the rotor gradient study; the numbers of each (its
    checkpoints and tapes are freed before the next run allocates its own)."""
    import torch
    from hlld_ai_b200.adjoint import RotorCase, rotor_gradients

    case = RotorCase(n=a.adjoint_n, steps=a.adjoint_steps, checkpoint_every=a.adjoint_every)
    runs = []
    for _ in range(count):
        r = rotor_gradients(case, device=dev)
        runs.append({k: r[k] for k in ("forward_ms", "adjoint_ms", "J", "grad_omega")})
        del r
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
    return runs


def _adjoint_workload(a):
    return (f"rotor {a.adjoint_n}^2, FP64 HLLD + PLM(MC) + CT, {a.adjoint_steps} SSP-RK3 steps, "
            f"checkpoint every {a.adjoint_every}, J = sum w |B_c|^2 / 2")


def run_adjoint(a):
    """The rotor gradient study alone: J and dJ/d(rho0, omega) by the
    checkpointed discrete adjoint; the line reports the median over --steps
    runs of the adjoint's time over the forward run's (both timed with CUDA
    events inside rotor_gradients).
    Replicas under torchrun; rank 0 prints."""
    import torch

    from hlld_ai_b200 import replicas

    rp = replicas.from_env("cuda")
    world, rank, dev = rp.world, rp.rank, rp.device
    torch.cuda.set_device(dev)
    replicas.init(rp)
    runs = _adjoint_runs(a, dev, max(1, a.steps))
    ratios = [r["adjoint_ms"] / r["forward_ms"] for r in runs]
    replicas.finish(rp)
    if rank == 0:
        line = {"metric": "adjoint time / forward time", "value": statistics.median(ratios),
                "unit": "x",
                "n_gpus": world, "steps": len(runs), "warmup": 0, "higher_is_better": False,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": _adjoint_workload(a)},
                "runs": [{"forward_ms": r["forward_ms"], "adjoint_ms": r["adjoint_ms"]} for r in runs],
                "J": runs[0]["J"], "dJ_domega": runs[0]["grad_omega"]}
        print(json.dumps(line), flush=True)
    return 0


def run_vortex(a):
    """The vortex block alone (config 3) as its own line."""
    import torch

    from hlld_ai_b200 import replicas

    rp = replicas.from_env("cuda")
    torch.cuda.set_device(rp.local)
    replicas.init(rp)
    res = _vortex_block(a, rp, rp.device)
    replicas.finish(rp)
    if rp.rank == 0:
        print(json.dumps({"metric": "zone-updates/s", "value": res["mixed"]["value"],
                          "unit": "zone-updates/s", "n_gpus": rp.world, "higher_is_better": True,
                          "dtype": "f32+f64", "data": "synthetic",
                          "config": {"workload": "relativistic vortex 2D, periodic [0,1]^2, "
                                                 "gamma 4/3, HLLD + PLM(MC, Wv) + SSP-RK3 + CT",
                                     "n": a.n},
                          "vortex": res}), flush=True)
    return 0


def _perturbed_fp64(problem, n, dev):
    """An FP64 stepper whose initial D and tau carry seeded relative noise of
    1e-13, resynced: the spread of FP64 itself under round-off."""
    import torch

    g, pert, sp = _stepper(problem, n, "fp64", dev)
    gen = torch.Generator(device=dev).manual_seed(1)
    for k in ("D", "tau"):
        noise = 2 * torch.rand(pert.cons[k].shape, generator=gen, device=dev, dtype=torch.float64) - 1
        pert.cons[k].mul_(1 + 1e-13 * noise)
    sp.sync(pert)
    return g, pert, sp


def run_rotor_whole(a):
    """Whole rotor runs from t = 0 to a.tend at a.n^2 in the mixed, FP32 and
    FP64 forms, all with the FP64 run's CFL dt sequence: each form's mean
    zone-updates/s over the run (CUDA events around every step, the dt
    computation of the FP64 run excluded) and the density L1/Linf of the
    mixed and FP32 runs against FP64 at a.tend, beside those of an untimed
    FP64 run from an initial state perturbed by 1e-13."""
    import torch

    from hlld_ai_b200 import replicas

    rp = replicas.from_env("cuda")
    dev = rp.device
    torch.cuda.set_device(rp.local)
    replicas.init(rp)
    runs = {p: _stepper(PROBLEM, a.n, p, dev) for p in ("fp64", "mixed", "fp32")}
    _, pert, psp = _perturbed_fp64(PROBLEM, a.n, dev)
    stream = torch.cuda.current_stream(dev)
    ms = {p: 0.0 for p in runs}
    t, steps = 0.0, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    while t < a.tend - 1e-14:
        dt = min(float(runs["fp64"][2].compute_dt(runs["fp64"][1], a.cfl).item()), a.tend - t)
        for p, (g, st, stp) in runs.items():
            e0.record(stream)
            stp.step(st, dt, "rk3")
            e1.record(stream)
            e1.synchronize()
            ms[p] += e0.elapsed_time(e1)
        psp.step(pert, dt, "rk3")
        t += dt
        steps += 1
    ph = runs["fp64"][0].phys
    ref = runs["fp64"][1].prims["rho"][ph]
    zones = a.n * a.n * rp.world
    out = {"n": a.n, "t": t, "steps": steps}
    for p in runs:
        (m,) = replicas.max_over_ranks(rp, ms[p])
        out[p] = {"ms_per_step": m / steps, "value": zones * steps / (m * 1e-3)}
        if p != "fp64":
            d = (runs[p][1].prims["rho"][ph].double() - ref).abs()
            out[p].update(l1_rho=float(d.mean()), linf_rho=float(d.max()))
    d = (pert.prims["rho"][ph].double() - ref).abs()
    out["fp64_perturbed_1e-13"] = {"l1_rho": float(d.mean()), "linf_rho": float(d.max())}
    replicas.finish(rp)
    if rp.rank == 0:
        print(json.dumps({"metric": "zone-updates/s", "value": out["mixed"]["value"],
                          "unit": "zone-updates/s", "n_gpus": rp.world, "higher_is_better": True,
                          "dtype": "f32+f64", "data": "synthetic",
                          "config": {"workload": WORKLOAD + f", whole run to t = {a.tend}",
                                     "n": a.n},
                          "rotor_run": out}), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "tubes":
        return run_tubes(a)
    if a.workload == "adjoint":
        return run_adjoint(a)
    if a.workload == "vortex":
        return run_vortex(a)
    if a.workload == "rotor_run":
        return run_rotor_whole(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
