"""Drop-in replacement for SMILI's f2py ``fortlib`` module surface.

``image`` holds the host-side regularizer initialisers; ``fftim2d`` and
``fftlib`` call the CUDA library through its C ABI.
"""
from . import image  # noqa: F401
from . import fftim2d  # noqa: F401
from . import fftlib  # noqa: F401
from . import fftim3d  # noqa: F401
