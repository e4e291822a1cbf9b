"""B200-native density-and-potential stage of the PGalF galaxy finder.

The CUDA kernels and the C ABI live in ``libgf.so`` (sources under ``csrc/``,
declarations in ``include/gf.h``); this package holds the ctypes binding, the
host-side mirror of the reference's entry points and the synthetic inputs.
"""
from ._lib import GFError, lib  # noqa: F401
