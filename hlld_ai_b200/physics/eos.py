"""Equation of state, mirroring ``src/physics/eos.py`` (hybrid_eos).

The kernels implement the hot path's EOS, ``hybrid_eos(K=0, gamma,
gamma_th=gamma)`` (an ideal gas, ``scripts/run_2d.py:213``).  The tensor
methods below are host-side helpers for building initial data; they follow
the reference formulas (``eos.py:15-76``) on any device.
"""
from __future__ import annotations

import torch


class hybrid_eos:
    def __init__(self, K, gamma, gamma_th=None):
        self.K = K
        self.gamma = gamma
        self.gamma_th = gamma_th
        self.is_cold = gamma_th is None or gamma_th == 1.0

    def kernel_gamma(self) -> float:
        """The adiabatic index the CUDA kernels use (see ``kernel_gamma``)."""
        return kernel_gamma(self)

    # eos.py:19-76, element-wise on tensors
    def press_cold_eps_cold__rho(self, rho):
        press_cold = self.K * rho**self.gamma
        eps_cold = press_cold / (rho * (self.gamma - 1))
        return press_cold, eps_cold

    def press__eps_rho(self, eps, rho):
        press_cold, eps_cold = self.press_cold_eps_cold__rho(rho)
        eps = torch.maximum(eps, eps_cold)
        if self.is_cold:
            return press_cold
        return press_cold + (eps - eps_cold) * rho * (self.gamma_th - 1)

    def eps__press_rho(self, press, rho):
        press_cold, eps_cold = self.press_cold_eps_cold__rho(rho)
        if self.is_cold:
            return eps_cold
        return eps_cold + (press - press_cold) / (rho * (self.gamma_th - 1))

    def press_and_cs2(self, eps, rho):
        press = self.press__eps_rho(eps, rho)
        h = 1.0 + eps + press / rho
        if self.is_cold:
            cs2 = self.gamma * press / (rho * h)
        else:
            press_cold, _ = self.press_cold_eps_cold__rho(rho)
            cs2 = (self.gamma * press_cold + self.gamma_th * (press - press_cold)) / (rho * h)
        return press, cs2


def kernel_gamma(eos) -> float:
    """The adiabatic index of an ideal-gas ``hybrid_eos(K=0, gamma,
    gamma_th=gamma)``, the only EOS the kernels implement.  Any object with
    the attributes ``K``, ``gamma`` and ``gamma_th`` is accepted, so the
    reference's own ``hybrid_eos`` instances drive the step unchanged."""
    K, gamma, gth = (getattr(eos, a, None) for a in ("K", "gamma", "gamma_th"))
    if K != 0 or gamma is None or gth is None or gth == 1.0 or gth != gamma:
        raise NotImplementedError(
            "hlld_ai_b200 kernels implement hybrid_eos(K=0, gamma, gamma_th=gamma) only")
    return float(gamma)
