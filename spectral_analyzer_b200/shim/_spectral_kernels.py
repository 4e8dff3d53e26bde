"""Import shim: ``from _spectral_kernels import AcousticFDTD`` resolves to the CUDA engine.

Put this directory first on ``sys.path`` (or PYTHONPATH) and the reference's
acoustic_fdtd_bridge.py (``from _spectral_kernels import AcousticFDTD``,
acoustic_fdtd_bridge.py:81-86) builds its solver on the GPU engine, and
``from _spectral_kernels import AcousticAMR`` (acoustic_amr.py:329) its AMR
stepper.  Only these two classes are provided; the reference module's other
classes are not part of this engine, so importing them raises ImportError as
the bridge's try/except blocks expect.
"""
import os
import sys

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from spectral_analyzer_b200.amr import AcousticAMR  # noqa: E402,F401
from spectral_analyzer_b200.fdtd import AcousticFDTD  # noqa: E402,F401

FDTD_AIR, FDTD_WALL, FDTD_PLATE, FDTD_PML = 0, 1, 2, 3
