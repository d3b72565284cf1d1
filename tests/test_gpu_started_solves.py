"""The mixed form's shortcuts give the answers of the solves they replace.

* ``hlld_sync_state_from_prims`` starts every cell's Kastaun root search from
  the root 1/(hW) of the primitives the state holds; the result is the
  bracketed solve's (c2p.py:188-236) to the solver's tolerance, checked here
  against ``hlld_sync_state_roots`` on an evolved rotor state whose conserved
  variables were moved away from its primitives.
* Faces without normal field take the HLLE fallback (hlld.py:1512-1531)
  whatever p* is, so the mixed sweep does not solve p* there: on the rotor
  at t = 0 (B = (1, 0, 0), so B_y = 0 on every y face) the HLLD y sweep
  returns the HLLE y sweep's fluxes, counts every face as B_n = 0 and
  fallback, and solves none.
"""
import ctypes

import pytest
import torch

import hlld_ai_b200 as H
from hlld_ai_b200 import _lib

pytestmark = pytest.mark.gpu

N = 256


def _rotor(solver="hlld"):
    g, eos, st, spec = H.setup_problem("rotor_tapered", N, limiter="mc", device="cuda",
                                       precision="mixed")
    stepper = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn=solver,
                          limiter="mc", precision="mixed")
    return g, st, stepper


def _sweep(stepper, st, axis):
    g, L = stepper.grid, _lib.lib()
    nf = (g.nxt + 1) * g.nyt if axis == 0 else g.nxt * (g.nyt + 1)
    F = [torch.empty(nf, dtype=torch.float32, device="cuda") for _ in range(7)]
    diag = torch.zeros(ctypes.sizeof(_lib.FluxDiag), dtype=torch.uint8, device="cuda")
    s = stepper._struct(st)
    _lib.check(L.hlld_sweep2d(ctypes.byref(stepper.gc), ctypes.byref(s), axis,
                              _lib.ptr_array(F), diag.data_ptr(), _lib.stream_handle(stepper.device)),
               "sweep2d")
    torch.cuda.synchronize()
    return F, _lib.FluxDiag.from_buffer_copy(diag.cpu().numpy().tobytes())


def test_c2p_started_from_the_primitives_gives_the_bracketed_roots():
    g, st, stepper = _rotor()
    for _ in range(3):
        stepper.step(st, stepper.compute_dt(st, 0.4), "rk3")
    L, sh = _lib.lib(), _lib.stream_handle(stepper.device)
    cold, warm = st.clone(), st.clone()
    # an evolved, synced state; perturb its conserved variables so that every
    # root moves away from the one its primitives give
    for x in (cold, warm):
        for k in ("D", "tau"):
            x.cons[k].mul_(1.0 + 1e-4)
    mu_c = torch.zeros(g.nxt * g.nyt, dtype=torch.float64, device="cuda")
    mu_w = torch.zeros_like(mu_c)
    _lib.check(L.hlld_sync_state_roots(ctypes.byref(stepper.gc), ctypes.byref(stepper._struct(cold)),
                                       None, None, mu_c.data_ptr(), None, sh), "cold")
    _lib.check(L.hlld_sync_state_from_prims(ctypes.byref(stepper.gc),
                                            ctypes.byref(stepper._struct(warm)), None, None,
                                            mu_w.data_ptr(), sh), "from_prims")
    torch.cuda.synchronize()
    ph = g.phys
    mc, mw = mu_c.view(g.nxt, g.nyt)[ph], mu_w.view(g.nxt, g.nyt)[ph]
    assert float(((mw - mc).abs() / mc).max()) < 1e-12
    for k in ("rho", "p", "vx", "vy", "vz", "eps"):
        a, b = warm.prims[k][ph].double(), cold.prims[k][ph].double()
        scale = float(b.abs().max())
        assert float((a - b).abs().max()) <= 2e-7 * scale, k  # FP32 storage


def test_y_sweep_without_normal_field_returns_the_hlle_fluxes():
    g, st, hlld = _rotor("hlld")
    _, _, hlle = _rotor("hlle")
    assert float(st.Byf.abs().max()) == 0.0
    Fd, dd = _sweep(hlld, st, 1)
    Fe, _ = _sweep(hlle, st, 1)
    for k in range(7):
        a, b = Fd[k].double(), Fe[k].double()
        scale = max(float(b.abs().max()), 1e-30)
        assert float((a - b).abs().max()) <= 1e-6 * scale, k
    assert dd.n_bn_zero == dd.n_faces and dd.n_failed == dd.n_faces
    assert dd.n_conv == 0 and dd.iters_sum_conv == 0 and dd.n_not_converged == 0
    # the x sweep (B_x = 1) solves every face
    _, dx = _sweep(hlld, st, 0)
    assert dx.n_bn_zero == 0 and dx.n_conv > 0
