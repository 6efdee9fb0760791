"""``AGrid2DGridPhysics``: the physics wind tendencies from the A grid onto
the D-grid winds, over the B200 kernels.

Mirrors ``pySHiELD/update/update_dwind_phys.py``: same constructor
``AGrid2DGridPhysics(stencil_factory, quantity_factory, partitioner, rank,
namelist, grid_info)`` and call ``(u, v, u_dt, v_dt)``. The constructor
works out, as the reference's does (:171-463), which parts of this rank's
subtile edges lie on the cube tile's edges and on which side of the edge's
midpoint, and the call runs the whole update as two launches
(``shield_agrid_to_dgrid``).

What the caller provides, as for the reference:

* ``u_dt`` / ``v_dt`` with one filled halo point (the reference's
  ``ApplyPhysicsToDycore`` exchanges them before this call);
* ``grid_info`` with ``grid_type`` and the vectors ``vlon1..3``,
  ``vlat1..3``, ``es1_1..3``, ``ew2_1..3``, ``edge_vect_w`` /
  ``edge_vect_e`` (2-D) and ``edge_vect_s`` / ``edge_vect_n`` (1-D along
  x), as float64 CUDA arrays in the storage layout;
* ``partitioner.subtile_index(rank)`` = (y, x) of the rank's subtile and
  the grid indexing's ``south_edge`` ... ``east_edge`` flags.
"""

import ctypes

from ._lib import ShieldDwindGeometry, ShieldEdgePlan, ShieldField2D, check, load
from .microphysics import _current_stream
from .quantity import _unpack, field3d

EDGES = ("south", "north", "west", "east")


def edge_plan(nx, ny, n_halo, npx, npy, layout, subtile_index, edges):
    """Edge regions of this rank's subtile, in storage indices (the
    arithmetic of update_dwind_phys.py:232-440): for each of south, north,
    west, east a list of (line, lo, hi, dir) in the order the reference runs
    them (the part below the edge midpoint, then the part above)."""
    south, north, west, east = edges
    h = n_halo
    isc, iec, jsc, jec = h, h + nx - 1, h, h + ny - 1
    im2 = int((npx - 1) / 2) + 2
    jm2 = int((npy - 1) / 2) + 2
    wx, wy = int((npx - 1) / layout[0]), int((npy - 1) / layout[1])
    sy, sx = subtile_index
    gis, gjs, gie, gje = isc + sx * wx, jsc + sy * wy, iec + sx * wx, jec + sy * wy
    shape_i, shape_j = nx + 2 * h + 1, ny + 2 * h + 1
    plan = {}
    for name, on, line in (("west", west, h), ("east", east, shape_i - h - 1)):
        regs = []
        if on:
            n_lo = (min(jm2, gje) - sy * wy) - jsc + 1
            if gjs <= jm2 and n_lo > 0:
                regs.append((line, h, h + n_lo, 1))
            if gje > jm2:
                js_up = max(jm2 + 1, gjs) - sy * wy
                n_up = jec - js_up + 1
                if n_up > 0:
                    regs.append((line, js_up, js_up + n_up, -1))
        plan[name] = regs
    for name, on, line in (("south", south, h), ("north", north, shape_j - h - 1)):
        regs = []
        if on:
            n_lo = (min(im2, gie) - sx * wx) - isc + 1
            lower = (gis <= im2) if name == "south" else (gis < im2)
            upper = (gie > im2) if name == "south" else (gie >= im2)
            if lower and n_lo > 0:
                regs.append((line, h, h + n_lo, 1))
            if upper:
                is_up = max(im2 + 1, gis) - sx * wx
                n_up = iec - is_up + 1
                if n_up > 0:
                    regs.append((line, is_up, is_up + n_up, -1))
        plan[name] = regs
    return plan


def _origin_ptr(q, h, ndim):
    """Pointer to the compute-domain origin of a grid field: its ``origin``
    when it is a quantity, else (h, h) of a full storage array."""
    ptr, st, shape, org = _unpack(q)
    if len(shape) != ndim:
        raise ValueError(f"expected a {ndim}-D grid field, got shape {shape}")
    if not hasattr(q, "origin"):
        org = (h,) * ndim
    return ptr + 8 * sum(o * s for o, s in zip(org, st)), st


class AGrid2DGridPhysics:
    """AGrid2DGridPhysics (update_dwind_phys.py:166-701) on the GPU."""

    def __init__(self, stencil_factory, quantity_factory, partitioner, rank, namelist, grid_info):
        gi = stencil_factory.grid_indexing
        self.nx, self.ny, self.nz = (int(v) for v in gi.domain)
        self.n_halo = h = int(getattr(gi, "n_halo", 3))
        self._dt5 = 0.5 * namelist.dt_atmos
        self._grid_type = int(grid_info.grid_type)
        self._plan = None
        self._geom = None
        if self._grid_type <= 3:
            edges = tuple(bool(getattr(gi, f"{e}_edge")) for e in EDGES)
            plan = edge_plan(self.nx, self.ny, h, namelist.npx, namelist.npy, tuple(namelist.layout),
                             tuple(partitioner.subtile_index(rank)), edges)
            P = ShieldEdgePlan()
            for s, name in enumerate(EDGES):
                regs = plan[name]
                P.n[s] = len(regs)
                for q, (line, lo, hi, d) in enumerate(regs):
                    P.r[s][q].line, P.r[s][q].lo, P.r[s][q].hi, P.r[s][q].dir = line - h, lo - h, hi - h, d
            self._plan = P
            G = ShieldDwindGeometry()
            # the geometry table holds raw device pointers: keep the arrays
            # alive as long as this object (a caller may drop grid_info)
            self._geom_arrays = [getattr(grid_info, name) for name in (
                "vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1", "ew2_2",
                "ew2_3", "edge_vect_w", "edge_vect_e", "edge_vect_s", "edge_vect_n")]
            for name in ("vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1",
                         "ew2_2", "ew2_3", "edge_vect_w", "edge_vect_e"):
                ptr, st = _origin_ptr(getattr(grid_info, name), h, 2)
                setattr(G, name, ShieldField2D(ptr, st[0], st[1]))
            strides = set()
            for name in ("edge_vect_s", "edge_vect_n"):
                ptr, st = _origin_ptr(getattr(grid_info, name), h, 1)
                setattr(G, name, ptr)
                strides.add(st[0])
            if len(strides) != 1:
                raise ValueError("edge_vect_s and edge_vect_n must have the same stride")
            G.edge_stride = strides.pop()
            self._geom = G
        load()

    def _winds(self, u, v, u_dt, v_dt):
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.n_halo
        # u: j in [0, ny]; v: i in [0, nx]; the tendencies: one halo point
        fu = field3d(u, (nx, ny + 1, nz))
        fv = field3d(v, (nx + 1, ny, nz))
        for q in (u_dt, v_dt):
            org = tuple(getattr(q, "origin", (h, h, 0)))
            if org[0] < 1 or org[1] < 1:
                raise ValueError("u_dt / v_dt need one halo point around the compute domain")
        fudt = field3d(u_dt, (nx + 1, ny + 1, nz))
        fvdt = field3d(v_dt, (nx + 1, ny + 1, nz))
        return fu, fv, fudt, fvdt

    def __call__(self, u, v, u_dt, v_dt, stream=None):
        nx, ny, nz = self.nx, self.ny, self.nz
        fu, fv, fudt, fvdt = self._winds(u, v, u_dt, v_dt)
        plan = ctypes.byref(self._plan) if self._plan is not None else None
        geom = ctypes.byref(self._geom) if self._geom is not None else None
        rc = load().shield_agrid_to_dgrid(nx, ny, nz, self._grid_type, float(self._dt5), plan, geom, fu, fv, fudt, fvdt,
                                          ctypes.c_void_p(_current_stream(stream)))
        check(rc, None, "shield_agrid_to_dgrid")


def agrid_to_dgrid_tiles(calls, stream=None):
    """Several ``AGrid2DGridPhysics.__call__`` at once: ``calls`` is a list
    of (a2d, u, v, u_dt, v_dt), one per tile this GPU holds (1 to 6,
    cube-sphere grids). Two launches in all (``shield_agrid_to_dgrid_tiles``)
    instead of two per tile; every tile's results are its own call's."""
    from ._lib import ShieldDwindTile

    if not 1 <= len(calls) <= 6:
        raise ValueError("1 to 6 tiles")
    arr = (ShieldDwindTile * len(calls))()
    for T, (a2d, u, v, u_dt, v_dt) in zip(arr, calls):
        if a2d._grid_type > 3:
            raise ValueError("agrid_to_dgrid_tiles takes cube-sphere tiles (grid_type <= 3)")
        T.nx, T.ny, T.nz, T.grid_type, T.dt5 = a2d.nx, a2d.ny, a2d.nz, a2d._grid_type, float(a2d._dt5)
        T.plan, T.geometry = a2d._plan, a2d._geom
        T.u, T.v, T.u_dt, T.v_dt = a2d._winds(u, v, u_dt, v_dt)
    rc = load().shield_agrid_to_dgrid_tiles(len(calls), arr, ctypes.c_void_p(_current_stream(stream)))
    check(rc, None, "shield_agrid_to_dgrid_tiles")
