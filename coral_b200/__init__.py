"""B200 (sm_100a) implementation of Coral's plane-layer IMEX timestep.

The product is the C-ABI shared library ``libcoral_b200.so`` (declared in
include/coral_b200.h); ``PlaneLayer`` is a thin ctypes mirror of the
reference's data-structure procedures for Python callers and tests.
"""
import os

CONFIG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs")


def __getattr__(name):
    if name in ("PlaneLayer", "CoralError"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
