"""B200-native (sm_100a) explicit SPH step of MCM 2.07 behind a C ABI.

The CUDA library (libmcm_gpu.so, built from csrc/) is the product; this
package holds the ctypes binding of its C ABI (include/mcm_gpu.h), the host
loop that mirrors MCM's mcm_solution, and generators for the synthetic decks.
"""
from .deck import Deck, MaterialCard, taylor_bar, fluid_column  # noqa: F401

__all__ = ["Deck", "MaterialCard", "taylor_bar", "fluid_column"]
