"""hlld_rk_step_ct_static: the RK + CT step for callers that cannot allocate
device memory -- hosts whose device memory belongs to someone else's pool,
plugin hosts that hand a solver only its inputs and outputs, loops that
cannot afford a cudaMalloc's device-wide synchronisation.  It keeps its
scratch in a fixed array inside the library instead of taking a
caller-allocated buffer.

Called through the C ABI on two steps in a row, it must give exactly what
hlld_rk_step_ct with caller-allocated scratch gives on the same state (the
tolerance of the step tests for the same kernels: bitwise), in every
precision of the 2D step -- the mixed form also keeps the C2P roots of its
first stage in the array -- and it must refuse a grid whose scratch does not
fit with HLLD_ERR_SCRATCH.  The test builds its own state, so it passes alone
in a fresh process and after the other tests (which leave their own data in
the shared array).
"""
import ctypes

import pytest
import torch

import hlld_ai_b200 as H
from hlld_ai_b200 import _lib
from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS, State2D

pytestmark = pytest.mark.gpu


def _copy(st):
    return State2D(cons={k: v.clone() for k, v in st.cons.items()}, Bxf=st.Bxf.clone(),
                   Byf=st.Byf.clone(), prims={k: v.clone() for k, v in st.prims.items()})


@pytest.mark.parametrize("precision", ["fp64", "fp64_exact", "mixed", "fp32"])
def test_static_scratch_step_matches_allocated_step_twice(precision):
    g, eos, st, spec = H.setup_problem("rotor_tapered", 96, limiter="mc", device="cuda",
                                       precision=precision)
    a, b = _copy(st), _copy(st)
    stepper = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld",
                          limiter="mc", precision=precision)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    dt_a = torch.zeros(1, dtype=torch.float64, device="cuda")
    diag_b = torch.zeros(ctypes.sizeof(_lib.StepDiag), dtype=torch.uint8, device="cuda")
    for _ in range(2):
        stepper.compute_dt(a, 0.4, out=dt_a)
        dt = float(dt_a.item())
        stepper.step(a, dt, "rk3")  # caller-allocated scratch (hlld_rk_step_ct)
        sb = stepper._struct(b)
        rc = L.hlld_rk_step_ct_static(ctypes.byref(stepper.gc), ctypes.byref(sb), dt, None, 3,
                                      diag_b.data_ptr(), stream)
        _lib.check(rc, "hlld_rk_step_ct_static")
        torch.cuda.synchronize()
        for k in EVOLVED_KEYS:
            assert torch.equal(a.cons[k], b.cons[k]), k
        for k in PRIM_KEYS:
            assert torch.equal(a.prims[k], b.prims[k]), k
        assert torch.equal(a.Bxf, b.Bxf) and torch.equal(a.Byf, b.Byf)
    d = _lib.StepDiag.from_buffer_copy(bytes(diag_b.cpu().numpy()))
    assert d.sweep[0].n_faces == (g.nxt + 1) * g.nyt


@pytest.mark.parametrize("precision,n_max", [("fp64", 599), ("mixed", 708), ("fp32", 849)])
def test_static_scratch_refuses_a_grid_that_does_not_fit(precision, n_max):
    L = _lib.lib()
    code = _lib.PRECISIONS[precision]
    for n, fits in ((n_max, True), (n_max + 1, False)):
        gc = _lib.Grid2DC(n, n, 2, 1.0 / n, 1.0 / n, 1, 1, 1, 1, 5.0 / 3.0, 1e-10, 1, code, 0)
        need = ctypes.c_size_t(0)
        assert L.hlld_step2d_scratch_bytes(ctypes.byref(gc), ctypes.byref(need)) == 0
        assert (need.value <= 64 << 20) == fits, (n, need.value)
    s = _lib.State2DC()
    rc = L.hlld_rk_step_ct_static(ctypes.byref(gc), ctypes.byref(s), 1e-3, None, 3, None, None)
    assert rc == -4  # HLLD_ERR_SCRATCH
    assert b"static array" in L.hlld_last_error_detail()
