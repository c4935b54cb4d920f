"""B200-native explicit finite-volume step of the Schemi multicomponent gas-dynamics solver.

Host-side mirror of the reference's step/flux/limiter/EOS interfaces over the C-ABI in
``include/fvstep.h`` (implemented by ``schemi_b200/csrc``).  The CUDA library is required:
importing :mod:`schemi_b200.fv` raises when it is missing; there is no CPU fallback.
"""

from .case import Case, Species, BC, fv_config_t  # noqa: F401

__all__ = ["Case", "Species", "BC", "fv_config_t"]
