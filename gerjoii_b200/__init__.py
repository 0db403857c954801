"""gerjoii_b200 — B200-native (sm_100a) radar full-waveform gradient path and
2.5D DC-resistivity solves, behind a C ABI (include/gerjoii_gpu.h).

The compute path is the CUDA library built by ``gerjoii_b200.build``; the
Python modules are thin host-side mirrors of the reference's MATLAB interface.
"""
from .geometry import WGrid, Shot, ricker, w_wavelet, w_M, surface_acquisition  # noqa: F401

__version__ = "0.1.0"


def native():
    """The loaded CUDA library (raises ImportError if it is not built)."""
    from . import _native
    return _native.load()
