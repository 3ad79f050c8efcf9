"""Drop-in replacement for SMILI's f2py ``fortlib`` module surface.

``image`` holds the host-side regularizer initialisers and image moments
(totalflux, xy_cen, sigma, check_sm_character); ``coord`` the uvw
computation; ``fftim2d``, ``fftim3d`` and ``fftlib`` call the CUDA library
through its C ABI.
"""
from . import coord  # noqa: F401
from . import image  # noqa: F401
from . import fftim2d  # noqa: F401
from . import fftlib  # noqa: F401
from . import fftim3d  # noqa: F401
