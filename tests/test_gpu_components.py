"""The step's components through the C ABI -- hlld_sweep2d, hlld_ct_update2d,
hlld_sync_state(_roots) -- reproduce hlld_rk_step_ct bit for bit, in every
precision.  (A host that schedules the components itself, the bench's
per-kernel timing among them, runs exactly the production step.  In the
mixed form that includes the started C2P root solves: stage 1 starts from
the step's input primitives, stages 2 and 3 from the roots of stage 1.)"""
import ctypes

import pytest
import torch

import hlld_ai_b200 as H
from hlld_ai_b200 import _lib
from hlld_ai_b200.physics.state import EVOLVED_KEYS

pytestmark = pytest.mark.gpu


def _component_step(stepper, st, dt, scheme, precision):
    g, L = stepper.grid, _lib.lib()
    gc, s = stepper.gc, stepper._struct(st)
    dev = stepper.device
    nfx, nfy = (g.nxt + 1) * g.nyt, g.nxt * (g.nyt + 1)
    rdt = torch.float32 if precision == "mixed" else torch.float64
    f64 = dict(dtype=torch.float64, device=dev)
    Fx = [torch.empty(nfx, dtype=rdt, device=dev) for _ in range(7)]
    Fy = [torch.empty(nfy, dtype=rdt, device=dev) for _ in range(7)]
    Ez = torch.empty((g.nxt + 1) * (g.nyt + 1), dtype=rdt, device=dev)
    U0 = [torch.empty(g.nxt * g.nyt, **f64) for _ in range(6)]
    Bx0, By0 = torch.empty(nfx, **f64), torch.empty(nfy, **f64)
    diag = torch.zeros(ctypes.sizeof(_lib.StepDiag), dtype=torch.uint8, device=dev)
    fd_off = ctypes.sizeof(_lib.FluxDiag)
    mixed = precision == "mixed"
    mu = torch.zeros(g.nxt * g.nyt, **f64) if mixed else None
    pFx, pFy, pU0 = _lib.ptr_array(Fx), _lib.ptr_array(Fy), _lib.ptr_array(U0)
    dt_dev = torch.tensor([dt], **f64)
    sh = _lib.stream_handle(dev)
    nst = 3 if scheme == "rk3" else 2
    for stage in range(nst):
        for axis, pF in ((0, pFx), (1, pFy)):
            _lib.check(L.hlld_sweep2d(ctypes.byref(gc), ctypes.byref(s), axis, pF,
                                      diag.data_ptr() + axis * fd_off, sh), "sweep")
        _lib.check(L.hlld_ct_update2d(ctypes.byref(gc), ctypes.byref(s), pFx, pFy, Ez.data_ptr(),
                                      pU0, Bx0.data_ptr(), By0.data_ptr(), diag.data_ptr(), stage,
                                      nst, 0.0, dt_dev.data_ptr(), sh), "ct_update2d")
        if mixed and stage == 0:
            rc = L.hlld_sync_state_from_prims(ctypes.byref(gc), ctypes.byref(s), None, None,
                                              mu.data_ptr(), sh)
        elif mixed:
            rc = L.hlld_sync_state_roots(ctypes.byref(gc), ctypes.byref(s), None, None, None,
                                         mu.data_ptr(), sh)
        else:
            rc = L.hlld_sync_state(ctypes.byref(gc), ctypes.byref(s), None, None, sh)
        _lib.check(rc, "sync")


@pytest.mark.parametrize("precision", ["mixed", "fp64", "fp64_exact"])
@pytest.mark.parametrize("scheme", ["rk3", "rk2"])
def test_components_reproduce_the_production_step(precision, scheme):
    g, eos, st, spec = H.setup_problem("rotor_tapered", 96, limiter="mc", device="cuda",
                                       precision=precision)
    stepper = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld",
                          limiter="mc", precision=precision)
    dt = float(stepper.compute_dt(st, 0.4).item())
    a, b = st.clone(), st.clone()
    for _ in range(3):
        stepper.step(a, dt, scheme)
        _component_step(stepper, b, dt, scheme, precision)
    torch.cuda.synchronize()
    for k in EVOLVED_KEYS:
        assert torch.equal(a.cons[k], b.cons[k]), k
    assert torch.equal(a.Bxf, b.Bxf) and torch.equal(a.Byf, b.Byf)
    for k in a.prims:
        assert torch.equal(a.prims[k], b.prims[k]), k
