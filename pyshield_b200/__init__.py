"""B200-native GFDL cloud microphysics and physics-to-dynamics coupling.

A drop-in for pySHiELD's ``Microphysics`` step and its column coupling
stencils, running hand-written sm_100a CUDA kernels through a C-ABI shared
library (``libshield_mp.so``) loaded with ctypes.
"""

from ._config import PHYSICS_PACKAGES, PhysicsConfig  # noqa: F401

__version__ = "0.1.0"
