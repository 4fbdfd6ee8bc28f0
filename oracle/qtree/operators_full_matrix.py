"""Placeholder for qtree's full-matrix gate module.

Oracle restatement, test infrastructure only.  QTensor only assigns
``ZZFull`` into this module at import time (``qtensor/OpFactory.py:41-42``)
for its ``QtreeFullBuilder``, which no path measured here uses; the compact
gates are re-exported so attribute lookups resolve.
"""
from .operators import (Gate, ParametricGate, M, I, H, X, Y, Z, T,  # noqa: F401
                        cX, cZ, ZPhase, XPhase, YPhase)
