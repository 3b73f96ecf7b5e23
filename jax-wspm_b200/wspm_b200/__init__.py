"""wspm_b200: B200-native (sm_100a) runtime of the JAX-WSPM implicit P1-FEM Picard step.

Host logic (mesh generators, SELL-32 pattern builder, Picard time loop) is
Python; every numerical kernel runs in libwspm.so (hand-written CUDA for
sm_100a) called through the C ABI in include/wspm.h.  Importing
``wspm_b200.device`` or ``wspm_b200.engine`` loads the library and fails
loudly if it is missing.
"""
from . import mesh, pattern  # noqa: F401  (host-only modules)

__all__ = ["mesh", "pattern"]
