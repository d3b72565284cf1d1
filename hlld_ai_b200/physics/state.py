"""State containers, mirroring ``src/physics/state.py``.

``State2D`` holds the cell-centred conserved variables (``EVOLVED_KEYS``),
the staggered field and the primitives, each a contiguous CUDA tensor with
the reference's shapes (``state.py:54-74``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, Sequence

import torch

# state.py:41
EVOLVED_KEYS = ["D", "Sx", "Sy", "Sz", "tau", "Bz"]
PRIM_KEYS = ["rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz"]
CONS_KEYS = ["D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz"]


def flat(d: dict) -> dict:
    """state.py:44-46"""
    return {k: v.reshape(-1) for k, v in d.items()}


def unflat(d: dict, shape: Sequence[int]) -> dict:
    """state.py:49-51"""
    return {k: v.reshape(*shape) for k, v in d.items()}


@dataclass
class State2D:
    cons: dict
    Bxf: torch.Tensor
    Byf: torch.Tensor
    prims: dict = field(default_factory=dict)

    def clone(self) -> "State2D":
        return State2D(cons={k: v.clone() for k, v in self.cons.items()},
                       Bxf=self.Bxf.clone(), Byf=self.Byf.clone(),
                       prims={k: v.clone() for k, v in self.prims.items()})


def combine(states: Iterable[State2D], weights: Sequence[float]) -> State2D:
    """state.py:77-103: the affine combination with identical weights on the
    cell variables and the faces (same operation order)."""
    states = list(states)
    if len(states) != len(weights):
        raise ValueError(f"{len(states)} states but {len(weights)} weights")
    if not states:
        raise ValueError("combine() needs at least one state")
    w0, s0 = weights[0], states[0]
    cons = {k: w0 * s0.cons[k] for k in s0.cons}
    Bxf = w0 * s0.Bxf
    Byf = w0 * s0.Byf
    for w, s in zip(weights[1:], states[1:]):
        for k in cons:
            cons[k] = cons[k] + w * s.cons[k]
        Bxf = Bxf + w * s.Bxf
        Byf = Byf + w * s.Byf
    return State2D(cons=cons, Bxf=Bxf, Byf=Byf)
