import numpy as np

from ndsl.quantity import Quantity


class QuantityFactory:
    """zeros() on the (nx+2h+1, ny+2h+1, nz+1) storage the translate tests use."""

    def __init__(self, nx, ny, nz, n_halo=3):
        self.nx, self.ny, self.nz, self.h = nx, ny, nz, n_halo

    def zeros(self, dims, units, dtype=np.float64):
        h = self.h
        shape = []
        origin = []
        extent = []
        for d in dims:
            if d.startswith("x"):
                shape.append(self.nx + 2 * h + 1); origin.append(h); extent.append(self.nx)
            elif d.startswith("y"):
                shape.append(self.ny + 2 * h + 1); origin.append(h); extent.append(self.ny)
            else:
                shape.append(self.nz + 1); origin.append(0)
                extent.append(self.nz + 1 if d.endswith("interface") else self.nz)
        return Quantity(np.zeros(shape, dtype=dtype), dims, units, origin, extent)
