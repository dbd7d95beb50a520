"""moldy_b200 -- B200-native (sm_100a) MOLDY Fe EAM hot path.

A from-scratch CUDA implementation of the short-range MD force hot path of
MOLDY (gjackland/moldy): link cells, the hybrid Verlet half list, the
two-pass Finnis-Sinclair/EAM evaluation over the lookup tables, the virial
used by Parrinello-Rahman and the velocity-Verlet update.  The C ABI is in
``include/moldy_gpu.h``; :class:`MoldySystem` mirrors the reference's
routine names on top of it.
"""
from ._lib import MoldyError, load  # noqa: F401
from .potentials import FE_FE, FeFeCoefficients, read_pot_file  # noqa: F401
from .system import MoldySystem  # noqa: F401
from .batch import MoldyBatch  # noqa: F401

__all__ = ["MoldySystem", "MoldyBatch", "MoldyError", "FE_FE", "FeFeCoefficients", "read_pot_file", "load"]
