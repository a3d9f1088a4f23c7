"""rbmd_b200 -- B200-native (sm_100a) RBE + LJ/erfc-Coulomb force engine.

A drop-in for RBMD 2.0's LJ/CUT/COUL/LONG force plugin with RBE k-space and
RBL / Verlet neighbor lists.  The engine is C++/CUDA behind the C ABI of
include/rbx.h (librbx.so); ``rbmd_b200.rbx`` is the ctypes binding and
``rbmd_b200.systems`` builds the seeded benchmark systems.
"""
from . import systems  # noqa: F401

__all__ = ["systems", "rbx", "build"]
