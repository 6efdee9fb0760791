"""AGrid2DGridPhysics (pySHiELD/update/update_dwind_phys.py).

CPU: the package's edge plan (which parts of a rank's subtile edges lie on
the cube tile's edges, and on which side of the midpoint) equals the plan of
the oracle, which reproduces the reference's output bit for bit
(test_oracle_golden.py), over many layouts, ranks and tile sizes.

GPU: the kernels against the reference's own result (golden fixtures) for a
whole tile, two subtiles of a 2 x 2 layout and the doubly periodic grid,
every storage compared whole; and against the oracle on domains that span
several of the update kernel's tiles in i, j and k.
"""
import numpy as np
import pytest

DWIND_CASES = ("dwind_tile", "dwind_sub0", "dwind_sub3", "dwind_periodic")


@pytest.mark.parametrize("n", [6, 7, 12, 13, 48])
def test_edge_plan_matches_oracle(n):
    from oracle.dwind import edge_plan as oracle_plan
    from pyshield_b200.dwind import edge_plan

    for layout in ((1, 1), (2, 2), (3, 3), (2, 1), (1, 3)):
        if n % layout[0] or n % layout[1]:
            continue
        nx, ny = n // layout[0], n // layout[1]
        for rank in range(layout[0] * layout[1]):
            sy, sx = rank // layout[0], rank % layout[0]
            edges = (sy == 0, sy == layout[1] - 1, sx == 0, sx == layout[0] - 1)
            got = edge_plan(nx, ny, 3, n + 1, n + 1, layout, (sy, sx), edges)
            ref = oracle_plan(nx, ny, 3, n + 1, n + 1, layout, (sy, sx), edges)
            for name in ("south", "north", "west", "east"):
                # the oracle keeps the reference's empty upper south region; it changes nothing
                r = [x for x in ref[name] if x[2] > x[1]]
                assert got[name] == r, (n, layout, rank, name, got[name], r)


@pytest.mark.gpu
@pytest.mark.parametrize("name", DWIND_CASES)
def test_agrid_to_dgrid_matches_reference(name):
    from types import SimpleNamespace

    import torch

    from golden_io import load
    from pyshield_b200.dwind import AGrid2DGridPhysics
    from pyshield_b200.grid import GridIndexing, StencilFactory

    z, m = load(name)
    nx, ny, L, h = m["nx"], m["ny"], m["L"], m["halo"]

    def dev(a):
        a = np.ascontiguousarray(a.T)
        return torch.from_numpy(a).cuda().permute(*reversed(range(a.ndim)))

    gi = GridIndexing(nx, ny, L, h)
    gi.south_edge, gi.north_edge, gi.west_edge, gi.east_edge = m["edges"]
    sy, sx = m["subtile_index"]
    part = SimpleNamespace(subtile_index=lambda rank: (sy, sx))
    namelist = SimpleNamespace(dt_atmos=m["dt"], npx=m["npx"], npy=m["npy"], layout=tuple(m["layout"]))
    geom = {k[5:]: dev(z[k]) for k in z.files if k.startswith("geom_")}
    grid_info = SimpleNamespace(grid_type=m["grid_type"], **geom)
    f = {k: dev(z["in_" + k]) for k in ("u", "v", "u_dt", "v_dt")}
    from pyshield_b200.quantity import Quantity

    q = {k: Quantity(t, ("x", "y", "z"), "", (h, h, 0), (nx, ny, L)) for k, t in f.items()}
    a2d = AGrid2DGridPhysics(StencilFactory(gi), None, part, m["rank"], namelist, grid_info)
    a2d(q["u"], q["v"], q["u_dt"], q["v_dt"])
    torch.cuda.synchronize()
    for k, t in f.items():
        np.testing.assert_array_equal(t.cpu().numpy(), z["out_" + k], err_msg=f"{name} {k}")


# Domains that span several of the update kernel's tiles (32 x 8 points by 8
# levels) in i, j and k, with ragged last tiles: (tile size n, layout, rank,
# levels, storage layout)
TILED_CASES = [
    (70, (1, 1), 0, 11, "ifirst"),
    (70, (1, 1), 0, 11, "kfirst"),
    (66, (2, 2), 3, 9, "ifirst"),
    (66, (2, 2), 0, 17, "ifirst"),
    (48, (2, 1), 1, 8, "ifirst"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("n,layout,rank,L,order", TILED_CASES)
def test_agrid_to_dgrid_across_tiles_matches_oracle(n, layout, rank, L, order):
    """The kernels against the oracle (pinned bit for bit to the reference's
    own class by the golden fixtures) on domains larger than one tile of the
    update kernel: every storage compared whole, bit for bit."""
    from types import SimpleNamespace

    import torch

    from oracle.dwind import agrid_to_dgrid as oracle_a2d
    from pyshield_b200.dwind import AGrid2DGridPhysics, edge_plan
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.quantity import Quantity

    h = 3
    nx, ny = n // layout[0], n // layout[1]
    sy, sx = rank // layout[0], rank % layout[0]
    edges = (sy == 0, sy == layout[1] - 1, sx == 0, sx == layout[0] - 1)
    rng = np.random.default_rng(100 + n + rank + L)
    shape3 = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
    shape2 = shape3[:2]
    f = {"u": rng.uniform(-30.0, 30.0, shape3), "v": rng.uniform(-30.0, 30.0, shape3),
         "u_dt": rng.normal(0.0, 1e-3, shape3), "v_dt": rng.normal(0.0, 1e-3, shape3)}
    g = {name: rng.uniform(-1.0, 1.0, shape2) for name in
         ("vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1", "ew2_2", "ew2_3")}
    g["edge_vect_w"] = rng.uniform(0.0, 1.0, shape2)
    g["edge_vect_e"] = rng.uniform(0.0, 1.0, shape2)
    g["edge_vect_s"] = rng.uniform(0.0, 1.0, shape3[0])
    g["edge_vect_n"] = rng.uniform(0.0, 1.0, shape3[0])
    dt = 180.0

    def dev(a):
        if order == "ifirst" or a.ndim < 3:
            return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().permute(*reversed(range(a.ndim)))
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    gi = GridIndexing(nx, ny, L, h)
    gi.south_edge, gi.north_edge, gi.west_edge, gi.east_edge = edges
    part = SimpleNamespace(subtile_index=lambda r: (sy, sx))
    namelist = SimpleNamespace(dt_atmos=dt, npx=n + 1, npy=n + 1, layout=layout)
    grid_info = SimpleNamespace(grid_type=0, **{k: dev(v) for k, v in g.items()})
    t = {k: dev(v) for k, v in f.items()}
    q = {k: Quantity(v, ("x", "y", "z"), "", (h, h, 0), (nx, ny, L)) for k, v in t.items()}
    AGrid2DGridPhysics(StencilFactory(gi), None, part, rank, namelist, grid_info)(q["u"], q["v"], q["u_dt"], q["v_dt"])
    torch.cuda.synchronize()

    plan = edge_plan(nx, ny, h, n + 1, n + 1, layout, (sy, sx), edges)
    ref = {k: v.copy() for k, v in f.items()}
    oracle_a2d(ref["u"], ref["v"], ref["u_dt"], ref["v_dt"], g, nx, ny, L, h, 0.5 * dt, plan)
    assert any(len(plan[s]) for s in plan)  # the corrections are exercised
    for k in f:
        np.testing.assert_array_equal(t[k].cpu().numpy(), ref[k], err_msg=f"{n} {layout} {rank} {k}")


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["ifirst", "kfirst"])
def test_doubly_periodic_matches_oracle(order):
    """grid_type > 3 (doubly_periodic_wind_update) against the oracle on a
    domain of several blocks and lines, bit for bit."""
    from types import SimpleNamespace

    import torch

    from oracle.dwind import doubly_periodic
    from pyshield_b200.dwind import AGrid2DGridPhysics
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.quantity import Quantity

    nx, ny, L, h, dt = 150, 37, 11, 3, 180.0
    rng = np.random.default_rng(4)
    shape3 = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
    f = {"u": rng.uniform(-30.0, 30.0, shape3), "v": rng.uniform(-30.0, 30.0, shape3),
         "u_dt": rng.normal(0.0, 1e-3, shape3), "v_dt": rng.normal(0.0, 1e-3, shape3)}

    def dev(a):
        if order == "ifirst":
            return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().permute(2, 1, 0)
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    t = {k: dev(v) for k, v in f.items()}
    q = {k: Quantity(v, ("x", "y", "z"), "", (h, h, 0), (nx, ny, L)) for k, v in t.items()}
    namelist = SimpleNamespace(dt_atmos=dt, npx=nx + 1, npy=ny + 1, layout=(1, 1))
    a2d = AGrid2DGridPhysics(StencilFactory(GridIndexing(nx, ny, L, h)), None, None, 0, namelist,
                             SimpleNamespace(grid_type=4))
    a2d(q["u"], q["v"], q["u_dt"], q["v_dt"])
    torch.cuda.synchronize()
    ref = {k: v.copy() for k, v in f.items()}
    doubly_periodic(ref["u"], ref["v"], ref["u_dt"], ref["v_dt"], nx, ny, L, h, 0.5 * dt)
    for k in f:
        np.testing.assert_array_equal(t[k].cpu().numpy(), ref[k], err_msg=k)


@pytest.mark.gpu
def test_tiles_in_one_launch_equal_separate_calls():
    """agrid_to_dgrid_tiles (two launches for all tiles) leaves every
    storage of every tile bit for bit as each tile's own call does: six
    tiles of unequal size, layouts and ranks (whole tiles and subtiles)."""
    from types import SimpleNamespace

    import torch

    from pyshield_b200.dwind import AGrid2DGridPhysics, agrid_to_dgrid_tiles
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.quantity import Quantity

    h, L = 3, 9
    cases = [(40, (1, 1), 0), (34, (1, 1), 0), (66, (2, 2), 3), (66, (2, 2), 0), (48, (2, 1), 1), (20, (1, 1), 0)]

    def build(seed):
        rng = np.random.default_rng(seed)
        out = []
        for t, (n, layout, rank) in enumerate(cases):
            nx, ny = n // layout[0], n // layout[1]
            sy, sx = rank // layout[0], rank % layout[0]
            gi = GridIndexing(nx, ny, L, h)
            gi.south_edge, gi.north_edge = sy == 0, sy == layout[1] - 1
            gi.west_edge, gi.east_edge = sx == 0, sx == layout[0] - 1
            shape3 = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
            dev3 = lambda a: torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda().permute(2, 1, 0)  # noqa: E731
            dev2 = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()  # noqa: E731
            geom = {g: dev2(rng.uniform(-1.0, 1.0, shape3[:2])) for g in (
                "vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1", "ew2_2",
                "ew2_3")}
            geom["edge_vect_w"] = dev2(rng.uniform(0.0, 1.0, shape3[:2]))
            geom["edge_vect_e"] = dev2(rng.uniform(0.0, 1.0, shape3[:2]))
            geom["edge_vect_s"] = torch.from_numpy(rng.uniform(0.0, 1.0, shape3[0])).cuda()
            geom["edge_vect_n"] = torch.from_numpy(rng.uniform(0.0, 1.0, shape3[0])).cuda()
            part = SimpleNamespace(subtile_index=lambda r, s=(sy, sx): s)
            nl = SimpleNamespace(dt_atmos=225.0, npx=n + 1, npy=n + 1, layout=layout)
            a2d = AGrid2DGridPhysics(StencilFactory(gi), None, part, rank, nl, SimpleNamespace(grid_type=0, **geom))
            q = {k: Quantity(dev3(rng.normal(0.0, s, shape3)), ("x", "y", "z"), "", (h, h, 0), (nx, ny, L))
                 for k, s in (("u", 20.0), ("v", 20.0), ("u_dt", 1e-3), ("v_dt", 1e-3))}
            out.append((a2d, q))
        return out

    sep, bat = build(7), build(7)
    for a2d, q in sep:
        a2d(q["u"], q["v"], q["u_dt"], q["v_dt"])
    agrid_to_dgrid_tiles([(a2d, q["u"], q["v"], q["u_dt"], q["v_dt"]) for a2d, q in bat])
    torch.cuda.synchronize()
    for t, ((_, qa), (_, qb)) in enumerate(zip(sep, bat)):
        for k in ("u", "v", "u_dt", "v_dt"):
            np.testing.assert_array_equal(qa[k].data.cpu().numpy(), qb[k].data.cpu().numpy(), err_msg=f"tile {t} {k}")


@pytest.mark.gpu
def test_wind_update_with_periodic_halo():
    """DGridWindUpdate on one rank of a doubly periodic plane: the halo
    exchange fills the one-point halo of u_dt / v_dt from the opposite edges
    (this rank is its own neighbour), then the doubly periodic D-grid update
    runs; against the oracle's update on storages whose halos were filled by
    hand, bit for bit."""
    from types import SimpleNamespace

    import torch

    from oracle.dwind import doubly_periodic
    from pyshield_b200.coupling import DGridWindUpdate
    from pyshield_b200.dwind import AGrid2DGridPhysics
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.halo import doubly_periodic as periodic_table
    from pyshield_b200.quantity import Quantity

    nx, ny, L, h, dt = 40, 24, 7, 3, 180.0
    rng = np.random.default_rng(9)
    shape3 = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
    f = {"u": rng.uniform(-30.0, 30.0, shape3), "v": rng.uniform(-30.0, 30.0, shape3),
         "u_dt": rng.normal(0.0, 1e-3, shape3), "v_dt": rng.normal(0.0, 1e-3, shape3)}
    t = {k: torch.from_numpy(np.ascontiguousarray(a.T)).cuda().permute(2, 1, 0) for k, a in f.items()}
    q = {k: Quantity(v, ("x", "y", "z"), "", (h, h, 0), (nx, ny, L)) for k, v in t.items()}
    namelist = SimpleNamespace(dt_atmos=dt, npx=nx + 1, npy=ny + 1, layout=(1, 1))
    a2d = AGrid2DGridPhysics(StencilFactory(GridIndexing(nx, ny, L, h)), None, None, 0, namelist,
                             SimpleNamespace(grid_type=4))
    DGridWindUpdate(a2d, periodic_table((1, 1)), 0)(q["u"], q["v"], q["u_dt"], q["v_dt"])
    torch.cuda.synchronize()
    ref = {k: v.copy() for k, v in f.items()}
    for k in ("u_dt", "v_dt"):  # the periodic one-point halo, corners excluded
        a = ref[k]
        a[h - 1, h:h + ny, :L] = a[h + nx - 1, h:h + ny, :L]
        a[h + nx, h:h + ny, :L] = a[h, h:h + ny, :L]
        a[h:h + nx, h - 1, :L] = a[h:h + nx, h + ny - 1, :L]
        a[h:h + nx, h + ny, :L] = a[h:h + nx, h, :L]
    doubly_periodic(ref["u"], ref["v"], ref["u_dt"], ref["v_dt"], nx, ny, L, h, 0.5 * dt)
    for k in f:
        np.testing.assert_array_equal(t[k].cpu().numpy(), ref[k], err_msg=k)
