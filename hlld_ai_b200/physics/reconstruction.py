"""Reconstruction settings, mirroring ``src/physics/reconstruction.py``.

The reconstruction itself runs inside the fused sweep kernel (PCM, PLM with
the MC or minmod limiter, WENO5-Z, MP5, MP7; W v velocity variable; PCM
fallback at the density/pressure floors; EOS-consistent eps).
"""
from __future__ import annotations

# reconstruction.py:85-86
_STENCIL = {"pcm": 0, "mc": 1, "minmod": 1, "weno5z": 2, "mp5": 2, "mp7": 3}
HIGH_ORDER = ("weno5z", "mp5", "mp7")


def ghosts_needed(limiter: str) -> int:
    """reconstruction.py:89-98"""
    if limiter not in _STENCIL:
        raise ValueError(f"unknown limiter {limiter!r}")
    return max(2, _STENCIL[limiter] + 1)
