"""HostStepper2D: a state held in pinned host memory, stepped on the device
with its copies in and out overlapping the steps (hlld_rk_step_ct_events'
two events, chunked copies on two streams, several steps in flight), must
hold after the last step exactly what Stepper2D.step gives on a device copy
of the same state with the same CFL dt -- bitwise, in every precision of the
2D step, since the kernels and their order are the same.
"""
import pytest
import torch

import hlld_ai_b200 as H
from hlld_ai_b200.physics.state import EVOLVED_KEYS, PRIM_KEYS, State2D

pytestmark = pytest.mark.gpu


def _pinned(st):
    return State2D(cons={k: v.cpu().pin_memory() for k, v in st.cons.items()},
                   Bxf=st.Bxf.cpu().pin_memory(), Byf=st.Byf.cpu().pin_memory(),
                   prims={k: v.cpu().pin_memory() for k, v in st.prims.items()})


@pytest.mark.parametrize("precision,problem", [("fp64", "rotor_tapered"), ("mixed", "rotor_tapered"),
                                               ("fp32", "rotor_tapered"), ("mixed", "rotor")])
def test_host_stepper_matches_device_steps(precision, problem):
    g, eos, st, spec = H.setup_problem(problem, 160, device="cuda", precision=precision)
    host = _pinned(st)
    kw = dict(bc_x=spec["bc"][0], bc_y=spec["bc"][1], flux_fn="hlld", limiter="mc",
              precision=precision)
    dev_stepper = H.Stepper2D(g, eos, **kw)
    hs = H.HostStepper2D(H.Stepper2D(g, eos, **kw), host, chunks=3)
    for _ in range(3):
        dev_stepper.step(st, dev_stepper.compute_dt(st, 0.4), "rk3")
        hs.step(0.4, "rk3")  # no synchronisation between the steps
    hs.synchronize()
    torch.cuda.synchronize()
    for k in EVOLVED_KEYS:
        assert torch.equal(host.cons[k], st.cons[k].cpu()), k
    for k in PRIM_KEYS:
        assert torch.equal(host.prims[k], st.prims[k].cpu()), k
    assert torch.equal(host.Bxf, st.Bxf.cpu()) and torch.equal(host.Byf, st.Byf.cpu())
    h2d, d2h = hs.bytes_per_step()
    assert h2d == d2h == sum(t.numel() * t.element_size() for t in
                             [*host.cons.values(), *host.prims.values(), host.Bxf, host.Byf])


def test_host_stepper_refuses_unpinned_host_tensors():
    g, eos, st, spec = H.setup_problem("rotor_tapered", 32, device="cuda", precision="fp64")
    host = _pinned(st)
    host.cons["D"] = host.cons["D"].clone()  # pageable
    stepper = H.Stepper2D(g, eos, bc_x=spec["bc"][0], bc_y=spec["bc"][1], precision="fp64")
    with pytest.raises(TypeError, match="pinned"):
        H.HostStepper2D(stepper, host)
