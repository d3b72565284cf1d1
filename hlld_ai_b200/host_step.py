"""Stepping a 2D state that lives in host memory.

``HostStepper2D`` advances a ``State2D`` whose tensors are pinned CPU
tensors -- the form a caller of the reference's ``rk_step_ct``
(src/physics/driver2d.py:221-249) holds on a machine without a GPU -- on the
device, one ``rk_step_ct`` per call with the on-device CFL dt
(driver2d.py:52-82), and leaves each step's result back in the host tensors.

Every step copies the whole state in and out, so the host link is the bound
(at 2048^2 in the mixed form, 421 MB each way per step).  The copies run on
two streams of their own and overlap the step:

* copy-in, in the order the step reads: the faces and the primitives (the
  dt and the sweeps read them first), then the conserved cell arrays, which
  the first stage's update waits for (``hlld_rk_step_ct_events`` cons_in);
* copy-out of the faces and the conserved arrays as soon as the step
  records that they hold its result (cons_out), before its last C2P; the
  primitives after the step;
* the copy-in of an array for step k + 1 starts once the copy-out of the
  same array from step k has landed in its host buffer (and step k has
  finished with the device arrays), so the two directions overlap.  An
  array may also move in ``chunks`` pieces, each following its own
  copy-out; on a B200 (54.8 GB/s in, 56.6 GB/s out) whole arrays were the
  fastest: 13.98 ms per mixed 2048^2 step, against 15.24 ms with 4 pieces
  and 17.12 ms with 16.

The device state and the host state are the same numbers after every
``synchronize()``: the steps are ``Stepper2D.step``'s, bit for bit.
"""
from __future__ import annotations

import torch

from .physics.state import EVOLVED_KEYS, PRIM_KEYS, State2D


class HostStepper2D:
    """One device copy of a pinned host state and the pipelined steps over it."""

    def __init__(self, stepper, host: State2D, chunks: int = 1):
        if chunks < 1:
            raise ValueError("chunks must be at least 1")
        self.stepper = stepper
        self.host = host
        dev = stepper.device
        self.device = dev
        tensors = [("Bxf", host.Bxf), ("Byf", host.Byf)]
        tensors += [(f"prims.{k}", host.prims[k]) for k in PRIM_KEYS]
        tensors += [(f"cons.{k}", host.cons[k]) for k in EVOLVED_KEYS]
        for name, t in tensors:
            if t.device.type != "cpu" or not t.is_pinned() or not t.is_contiguous():
                raise TypeError(f"host {name} must be a contiguous pinned CPU tensor")
        self.dev = State2D(cons={k: torch.empty_like(host.cons[k], device=dev) for k in EVOLVED_KEYS},
                           Bxf=torch.empty_like(host.Bxf, device=dev),
                           Byf=torch.empty_like(host.Byf, device=dev),
                           prims={k: torch.empty_like(host.prims[k], device=dev) for k in PRIM_KEYS})
        # (validates shapes and dtypes against the stepper's grid and precision)
        stepper._struct(self.dev)

        def pieces(h, d):
            hv, dv = h.view(-1), d.view(-1)
            n = hv.numel()
            step = -(-n // chunks)
            return [(hv[a:a + step], dv[a:a + step]) for a in range(0, n, step)]

        faces = pieces(host.Bxf, self.dev.Bxf) + pieces(host.Byf, self.dev.Byf)
        prims = [p for k in PRIM_KEYS for p in pieces(host.prims[k], self.dev.prims[k])]
        cons = [p for k in EVOLVED_KEYS for p in pieces(host.cons[k], self.dev.cons[k])]
        self.groups = {"faces": faces, "prims": prims, "cons": cons}
        self.s_in = torch.cuda.Stream(dev)
        self.s_out = torch.cuda.Stream(dev)
        self.out_done = {g: [torch.cuda.Event() for _ in v] for g, v in self.groups.items()}
        self.ev_read = torch.cuda.Event()  # faces and primitives are on the device
        self.ev_cons_in = torch.cuda.Event()
        self.ev_cons_out = torch.cuda.Event()
        self.ev_end = torch.cuda.Event()
        main = torch.cuda.current_stream(dev)
        for ev in (self.ev_read, self.ev_cons_in, self.ev_cons_out, self.ev_end):
            ev.record(main)  # creates the CUDA events
        self.steps = 0

    def _copy_in(self, group: str) -> None:
        for (h, d), done in zip(self.groups[group], self.out_done[group]):
            if self.steps:
                self.s_in.wait_event(done)
            d.copy_(h, non_blocking=True)

    def _copy_out(self, group: str) -> None:
        for (h, d), done in zip(self.groups[group], self.out_done[group]):
            h.copy_(d, non_blocking=True)
            done.record(self.s_out)

    def step(self, cfl: float, scheme: str = "rk3") -> None:
        """Enqueue one step of the host state (returns before it runs)."""
        main = torch.cuda.current_stream(self.device)
        with torch.cuda.stream(self.s_in):
            if self.steps:
                self.s_in.wait_event(self.ev_end)  # the last step is done with the device arrays
            self._copy_in("faces")
            self._copy_in("prims")
            self.ev_read.record(self.s_in)
            self._copy_in("cons")
            self.ev_cons_in.record(self.s_in)
        main.wait_event(self.ev_read)
        dt = self.stepper.compute_dt(self.dev, cfl)
        self.stepper.step(self.dev, dt, scheme, cons_in=self.ev_cons_in, cons_out=self.ev_cons_out)
        self.ev_end.record(main)
        with torch.cuda.stream(self.s_out):
            self.s_out.wait_event(self.ev_cons_out)
            self._copy_out("faces")
            self.s_out.wait_event(self.ev_end)
            self._copy_out("prims")
            self._copy_out("cons")
        self.steps += 1

    def synchronize(self) -> None:
        """Make the current stream wait for the last step's copy-out."""
        main = torch.cuda.current_stream(self.device)
        for evs in self.out_done.values():
            for ev in evs:
                main.wait_event(ev)

    def bytes_per_step(self) -> tuple[int, int]:
        """(host -> device, device -> host) bytes of one step."""
        n = sum(h.numel() * h.element_size() for g in self.groups.values() for h, _ in g)
        return n, n
