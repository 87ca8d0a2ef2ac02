"""B200-native volumetric cloud march for PedalSky (sm_100a).

A drop-in for the reference's `ps-clouds` march + composite pass.  The hot
path is CUDA (`csrc/`), reached through the C ABI in `include/psclouds.h`
(`libpsclouds.so`).  This package holds the ctypes binding (`capi`), the
host-side mirror of the reference's subsystem API (`subsystem`) and the
seeded scene builders used by tests and the benchmark (`scenes`).
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
