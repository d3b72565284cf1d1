"""hlld_ai_b200: B200-native (sm_100a) special-relativistic MHD finite-volume step.

A from-scratch B200 implementation of kemi2805/HLLD-AI's hot path -- HLLE/HLLD/HLLC
Riemann fluxes, Kastaun C2P, PLM/WENO5-Z/MP5 reconstruction, constrained
transport and SSP-RK2/3, with its discrete adjoint -- behind the reference's flux_fn and rk_step_ct
interfaces.  The kernels live in libhlld_b200.so (C ABI: include/hlld_b200.h);
``hlld_ai_b200.physics`` mirrors the reference's ``src/physics`` modules.
"""
from . import _lib
from .physics import *  # noqa: F401,F403
from .host_step import HostStepper2D  # noqa: F401

__version__ = "0.1.0"
