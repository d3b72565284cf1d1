"""Shared test helpers: seeded state generators and comparisons."""
from __future__ import annotations

import math

import numpy as np
import torch

PRIM_KEYS = ("rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz")


def ideal_eps(p, rho, gamma):
    """eps from p for hybrid_eos(K=0, gamma, gamma_th=gamma) (eos.py:41-46 order)."""
    return 0.0 + (p - 0.0) / (rho * (gamma - 1.0))


def random_face_states(n: int, gamma: float, max_W: float = 5.0, seed: int = 20260824):
    """Admissible random left/right primitive states with a shared normal
    field, drawn like tests/test_idir.py:60-96 of the reference."""
    g = torch.Generator().manual_seed(seed)

    def u(lo, hi):
        return torch.empty(n, dtype=torch.float64).uniform_(lo, hi, generator=g)

    def one():
        rho = 10.0 ** u(-1.0, 1.0)
        p = 10.0 ** u(-1.5, 1.0)
        W = 1.0 + 10.0 ** u(-3.0, math.log10(max_W - 1.0))
        speed = torch.sqrt(1.0 - 1.0 / W**2)
        th, ph = u(0, math.pi), u(0, 2 * math.pi)
        B = torch.stack([u(-3.0, 3.0) for _ in range(3)])
        s = {"rho": rho, "p": p, "vx": speed * torch.sin(th) * torch.cos(ph),
             "vy": speed * torch.sin(th) * torch.sin(ph), "vz": speed * torch.cos(th),
             "Bx": B[0], "By": B[1], "Bz": B[2]}
        s["eps"] = ideal_eps(s["p"], s["rho"], gamma)
        return s

    sL, sR = one(), one()
    for k in ("Bx", "By", "Bz"):
        sR[k] = sL[k].clone()
    return sL, sR


def random_prims(n: int, gamma: float, W_range=(1.0, 2.0), rho_range=(1e-3, 1e2),
                 B_mag=1.0, zero_B=False, seed=0):
    """Sub-luminal primitive states drawn like tests/test_c2p.py:64-125 of the
    reference, with the ideal-gas EOS (p proportional to rho, hot)."""
    g = torch.Generator().manual_seed(seed)
    r = lambda: torch.rand(n, dtype=torch.float64, generator=g)
    lo, hi = math.log10(rho_range[0]), math.log10(rho_range[1])
    rho = 10.0 ** (lo + (hi - lo) * r())
    p = rho * (0.01 + r())
    W = W_range[0] + (W_range[1] - W_range[0]) * r()
    v = torch.sqrt(1.0 - 1.0 / W**2)
    cos_t = 2.0 * r() - 1.0
    sin_t = torch.sqrt(torch.clamp(1.0 - cos_t**2, min=0.0))
    phi = 2.0 * math.pi * r()
    if zero_B:
        Bx = By = Bz = torch.zeros(n, dtype=torch.float64)
    else:
        Bm = B_mag * r()
        cb = 2.0 * r() - 1.0
        sb = torch.sqrt(torch.clamp(1.0 - cb**2, min=0.0))
        pb = 2.0 * math.pi * r()
        Bx, By, Bz = Bm * sb * torch.cos(pb), Bm * sb * torch.sin(pb), Bm * cb
    s = {"rho": rho, "vx": v * sin_t * torch.cos(phi), "vy": v * sin_t * torch.sin(phi),
         "vz": v * cos_t, "p": p, "Bx": Bx, "By": By, "Bz": Bz}
    s["eps"] = ideal_eps(p, rho, gamma)
    return s


def to_np(d):
    return {k: (v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v))
            for k, v in d.items()}


def to_dev(d, device="cuda"):
    return {k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64).to(device)
            for k, v in d.items()}


def max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.abs(a).max()) if a.size else 0.0, 1e-300)
    return float(np.abs(a - b).max() / scale) if a.size else 0.0


def bitwise_equal(a, b) -> bool:
    """Equal as values, NaN == NaN (signed zeros compare equal)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def gradient_directions(X, Y, k):
    """Seeded density perturbation directions of the gradient fixture, as
    functions of the cell-centre offsets (X, Y) from the rotor's centre:
    k = 0..3 (and even k >= 8) a sum of three random-phase sinusoids over
    the whole domain, k = 4..7 (and odd k >= 8) a random-phase ring mode
    cos(m theta + phi) on the rotor's
    taper (0.1 < r < 0.115, where the density varies and the limiter is away
    from its kink).  tests/golden/make_golden.py evaluates them on the CPU for
    the reference's central differences, the GPU tests on the device."""
    import math

    rng = np.random.default_rng(1000 + k)
    if k < 4 or (k >= 8 and k % 2 == 0):
        d = 0.0
        for _ in range(3):
            kx, ky = rng.integers(1, 4, 2)
            ph = rng.uniform(0, 2 * math.pi)
            d = d + (2 * math.pi * (kx * X + ky * Y) + ph).cos()
        return d / 3.0
    m = int(rng.integers(1, 6))
    ph = rng.uniform(0, 2 * math.pi)
    r = (X * X + Y * Y).sqrt()
    theta = Y.atan2(X)
    ring = ((r - 0.1) * (0.115 - r)).clamp(min=0.0) / (0.0075 ** 2)
    return (m * theta + ph).cos() * ring
