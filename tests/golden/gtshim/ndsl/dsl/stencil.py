"""StencilFactory / GridIndexing over the numpy executor."""
from _gtexec import Stencil


class GridIndexing:
    def __init__(self, nx, ny, nz, n_halo=3, edges=(True, True, True, True)):
        self.nx, self.ny, self.nz, self.n_halo = nx, ny, nz, n_halo
        self.domain = (nx, ny, nz)
        self.isc, self.iec = n_halo, n_halo + nx - 1
        self.jsc, self.jec = n_halo, n_halo + ny - 1
        self.south_edge, self.north_edge, self.west_edge, self.east_edge = edges

    def origin_compute(self, add=(0, 0, 0)):
        return (self.n_halo + add[0], self.n_halo + add[1], add[2])

    def domain_compute(self, add=(0, 0, 0)):
        return (self.nx + add[0], self.ny + add[1], self.nz + add[2])

    def origin_full(self, add=(0, 0, 0)):
        return (add[0], add[1], add[2])

    def domain_full(self, add=(0, 0, 0)):
        h = self.n_halo
        return (self.nx + 2 * h + add[0], self.ny + 2 * h + add[1], self.nz + add[2])

    @property
    def max_shape(self):
        return self.domain_full(add=(1, 1, 1))


class _Cfg:
    dace_config = None


class StencilFactory:
    def __init__(self, grid_indexing):
        self.grid_indexing = grid_indexing
        self.config = _Cfg()
        self.backend = "numpy"

    def from_origin_domain(self, func, origin, domain, externals=None, **kwargs):
        return Stencil(func, externals=externals, origin=origin, domain=domain)

    def from_dims_halo(self, func, compute_dims, compute_halos=(0, 0), externals=None, **kwargs):
        """NDSL's from_dims_halo: the compute domain along ``compute_dims``
        (an interface dimension has one more point) widened by
        ``compute_halos`` in x and y."""
        gi = self.grid_indexing
        hx, hy = compute_halos
        n = (gi.nx, gi.ny, gi.nz)
        domain = tuple(n[d] + (1 if compute_dims[d].endswith("interface") else 0) for d in range(3))
        domain = (domain[0] + 2 * hx, domain[1] + 2 * hy, domain[2])
        origin = (gi.n_halo - hx, gi.n_halo - hy, 0)
        return Stencil(func, externals=externals, origin=origin, domain=domain)
