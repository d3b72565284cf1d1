"""B200 counterparts of kemi2805/HLLD-AI's ``src/physics`` hot-path modules."""
from .eos import hybrid_eos
from .grid import Grid1D, Grid2D
from .state import EVOLVED_KEYS, State2D, combine, flat, unflat
from .hlld import LAST_DIAG, hllc_flux, hlld_flux, hlle_flux, primitive_to_conserved
from .c2p import conservative_to_primitive
from .reconstruction import ghosts_needed
from .driver2d import (Stepper2D, compute_dt_2d, cons_to_prims_2d, prims_to_cons_2d,
                       rk_step_ct, sync_state)
from .initial_data2d import (PROBLEMS, b_from_potential, magnetic_rotor, orszag_tang,
                             relativistic_vortex, riemann2d, rotor_tapered, setup_problem)

__all__ = ["hybrid_eos", "Grid1D", "Grid2D", "EVOLVED_KEYS", "State2D", "combine", "flat",
           "unflat", "LAST_DIAG", "hlld_flux", "hlle_flux", "hllc_flux", "primitive_to_conserved",
           "conservative_to_primitive", "ghosts_needed", "Stepper2D", "compute_dt_2d",
           "cons_to_prims_2d", "prims_to_cons_2d", "rk_step_ct", "sync_state", "PROBLEMS",
           "b_from_potential", "magnetic_rotor", "orszag_tang", "relativistic_vortex",
           "riemann2d", "rotor_tapered", "setup_problem"]
