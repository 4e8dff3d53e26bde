"""B200-native (sm_100a) engine for the dense acoustic FDTD path of sangderenard/spectral-analyzer.

``AcousticFDTD`` is the drop-in for ``_spectral_kernels.AcousticFDTD``; the C ABI
(include/acoustic_fdtd_b200.h) is the drop-in for ``acoustic_fdtd.h``.
"""
from .fdtd import AcousticFDTD  # noqa: F401

__all__ = ["AcousticFDTD"]
