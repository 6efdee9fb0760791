import numpy as np


class Quantity:
    def __init__(self, data, dims, units, origin=None, extent=None):
        self.data = data
        self.dims = tuple(dims)
        self.units = units
        self.origin = tuple(origin) if origin is not None else (0,) * np.ndim(data)
        self.extent = tuple(extent) if extent is not None else np.shape(data)
