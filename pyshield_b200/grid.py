"""Stand-ins for the NDSL objects the ``Microphysics`` constructor takes.

pySHiELD's constructor is ``Microphysics(stencil_factory, quantity_factory,
grid_data, namelist)``. This package only reads
``stencil_factory.grid_indexing.domain`` (nx, ny, nz) and ``grid_data.area``,
so an NDSL ``StencilFactory`` / ``GridData`` works as is; callers without
NDSL can use the small classes below, which allocate torch CUDA storage with
NDSL's layout conventions (compute domain plus halo, one extra point per
dimension, i-fastest memory order as on GT4Py GPU backends).
"""

from .quantity import Quantity

X_DIM, Y_DIM, Z_DIM = "x", "y", "z"
X_INTERFACE_DIM, Y_INTERFACE_DIM, Z_INTERFACE_DIM = "x_interface", "y_interface", "z_interface"


class GridIndexing:
    def __init__(self, nx, ny, nz, n_halo=3):
        self.nx, self.ny, self.nz, self.n_halo = nx, ny, nz, n_halo
        self.domain = (nx, ny, nz)

    def origin_compute(self, add=(0, 0, 0)):
        return (self.n_halo + add[0], self.n_halo + add[1], add[2])

    def domain_compute(self, add=(0, 0, 0)):
        return (self.nx + add[0], self.ny + add[1], self.nz + add[2])

    def origin_full(self, add=(0, 0, 0)):
        return tuple(add)

    def domain_full(self, add=(0, 0, 0)):
        h = self.n_halo
        return (self.nx + 2 * h + add[0], self.ny + 2 * h + add[1], self.nz + add[2])


class SubtileGridSizer:
    """The NDSL grid sizer the reference's ``PhysicsState.init_from_storages``
    takes (``sizer.get_origin(dims)``, ``sizer.get_extent(dims)``): a rank's
    subtile of ``nx x ny`` points and ``nz`` levels inside a storage with
    ``n_halo`` halo points on each horizontal side."""

    def __init__(self, nx, ny, nz, n_halo=3, extra_dim_lengths=None):
        self.nx, self.ny, self.nz, self.n_halo = int(nx), int(ny), int(nz), int(n_halo)
        self.extra_dim_lengths = dict(extra_dim_lengths or {})

    @classmethod
    def from_tile_params(cls, nx_tile, ny_tile, nz, n_halo, extra_dim_lengths, layout, **_):
        """A cube tile of ``nx_tile x ny_tile`` split over a ``layout`` of
        ranks (the subtile is nx_tile / layout[1] by ny_tile / layout[0])."""
        return cls(int(nx_tile / layout[1]), int(ny_tile / layout[0]), nz, n_halo, extra_dim_lengths)

    def get_origin(self, dims):
        return tuple(self.n_halo if d.startswith(("x", "y")) else 0 for d in dims)

    def get_extent(self, dims):
        out = []
        for d in dims:
            inc = 1 if d.endswith("interface") else 0
            if d.startswith("x"):
                out.append(self.nx + inc)
            elif d.startswith("y"):
                out.append(self.ny + inc)
            elif d.startswith("z"):
                out.append(self.nz + inc)
            else:
                out.append(self.extra_dim_lengths[d])
        return tuple(out)


class StencilFactory:
    def __init__(self, grid_indexing):
        self.grid_indexing = grid_indexing


class GridData:
    def __init__(self, area, ptop=None):
        self.area = area
        self.ptop = ptop


def empty_storage(shape, device="cuda", ifirst=True):
    """float64 torch storage of ``shape`` (i, j, k); i-fastest memory order
    by default (the GT4Py GPU layout), C order otherwise."""
    import torch

    if ifirst:
        return torch.zeros(tuple(reversed(shape)), dtype=torch.float64, device=device).permute(
            *reversed(range(len(shape)))
        )
    return torch.zeros(shape, dtype=torch.float64, device=device)


class QuantityFactory:
    """``zeros(dims, units)`` on NDSL's (nx+2h+1, ny+2h+1, nz+1) storage."""

    def __init__(self, grid_indexing, device="cuda", ifirst=True):
        self.gi = grid_indexing
        self.device = device
        self.ifirst = ifirst

    def zeros(self, dims, units, dtype=None):
        gi = self.gi
        h = gi.n_halo
        shape, origin, extent = [], [], []
        for d in dims:
            if d.startswith("x"):
                shape.append(gi.nx + 2 * h + 1)
                origin.append(h)
                extent.append(gi.nx + (1 if d.endswith("interface") else 0))
            elif d.startswith("y"):
                shape.append(gi.ny + 2 * h + 1)
                origin.append(h)
                extent.append(gi.ny + (1 if d.endswith("interface") else 0))
            else:
                shape.append(gi.nz + 1)
                origin.append(0)
                extent.append(gi.nz + (1 if d.endswith("interface") else 0))
        return Quantity(empty_storage(tuple(shape), self.device, self.ifirst), dims, units, origin, extent)
