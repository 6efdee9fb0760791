"""The physical constants, taken from the same module the oracle and kernels use."""
from pyshield_b200.constants import *  # noqa: F401,F403

X_DIM = "x"
Y_DIM = "y"
Z_DIM = "z"
X_INTERFACE_DIM = "x_interface"
Y_INTERFACE_DIM = "y_interface"
Z_INTERFACE_DIM = "z_interface"
