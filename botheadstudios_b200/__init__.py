"""B200-native SPH giant-impact step (drop-in for the Integrity engine's GpuSph path).

The compute lives in ``libsph_b200.so`` (hand-written sm_100a CUDA behind the C ABI of
``include/sph_b200.h``). This package holds the ctypes binding (``_lib``), the host-side mirror of the
engine's ``GpuSph`` interface (``gpusph``), material tables (``materials``) and the synthetic initial
conditions (``ic``). Importing the package does not load the library; the first call that needs it does,
and it raises if the library is missing — there is no CPU fallback.
"""
from .materials import MAT_BASALT, MAT_IRON, MAX_MATERIALS  # noqa: F401

__version__ = "0.1.0"
