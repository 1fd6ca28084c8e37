"""irs_b200: B200-native microlensing magnification maps (IRS and IPM).

The compute path is hand-written CUDA for sm_100a behind a C ABI
(include/lib_ipm.h, include/lib_irs.h); this package holds the ctypes
interface. Build the libraries with `python -m irs_b200.build`.
"""
from .adaptive import AdaptiveIPM, LevelNet  # noqa: F401
from .batch import BatchIPM  # noqa: F401
from .ccf import CCF  # noqa: F401
from .mapmaker import IPM, IRS  # noqa: F401
from .ncc import NCC  # noqa: F401

__all__ = ["IPM", "IRS", "BatchIPM", "AdaptiveIPM", "LevelNet", "CCF", "NCC"]
