"""The one-point halo exchange of u_dt / v_dt (pyshield_b200.halo), on the
CPU with gloo ranks.

* The cubed-sphere edge table is checked against the geometry of a cube:
  each face is a gnomonic grid of n x n cells with its own centre and
  (i, j) axes (chosen so that every table entry holds; the table does not
  depend on them), and every halo cell of every tile must be the cell of
  the neighbouring tile that lies nearest, on the sphere, to the point one
  cell beyond the edge.
* The exchange itself runs over gloo: 2 ranks on a periodic plane (each
  also its own neighbour in y) and 6 ranks, one per cube tile; every halo
  point must hold its neighbour's value, with strips reversed where the
  table says so, and the rest of each storage must be untouched.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from pyshield_b200.halo import EAST, NORTH, SOUTH, WEST, check_table, cubed_sphere, doubly_periodic  # noqa: E402

# face centre, i axis, j axis of each tile (unit vectors)
X, Y, Z = np.eye(3)
FRAMES = [(X, Y, Z), (Y, -X, Z), (Z, -X, -Y), (-X, -Z, -Y), (-Y, -Z, X), (-Z, Y, X)]


def _point(t, x, y):
    c, a, b = FRAMES[t]
    v = c + x * a + y * b
    return v / np.linalg.norm(v)


def _coord(i, n):
    return -1.0 + (i + 0.5) * 2.0 / n


def _outside(e, p, n):
    """Face coordinates of the halo cell p (along the edge) beyond edge e."""
    out = 1.0 + 1.0 / n
    s = _coord(p, n)
    return {WEST: (-out, s), EAST: (out, s), SOUTH: (s, -out), NORTH: (s, out)}[e]


def _interior_cell(e, q, n):
    """(i, j) of point q of the compute-domain strip along edge e."""
    return {WEST: (0, q), EAST: (n - 1, q), SOUTH: (q, 0), NORTH: (q, n - 1)}[e]


def test_cube_table_is_consistent():
    check_table(cubed_sphere())
    check_table(doubly_periodic((2, 3)))


@pytest.mark.parametrize("n", [4, 7, 12])
def test_cube_table_matches_the_geometry(n):
    table = cubed_sphere()
    cells = [(t, i, j) for t in range(6) for i in range(n) for j in range(n)]
    pts = np.array([_point(t, _coord(i, n), _coord(j, n)) for t, i, j in cells])
    for t in range(6):
        for e, b in table[t].items():
            for p in range(n):
                v = _point(t, *_outside(e, p, n))
                nearest = cells[int(np.argmax(pts @ v))]
                q = n - 1 - p if b.reverse else p
                assert nearest == (b.rank, *_interior_cell(b.edge, q, n)), (t, e, p)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _value(rank, f, i, j, k):
    # exact in FP64: distinct per rank, field, point and level
    return rank * 1.0e6 + f * 1.0e5 + i * 1.0e3 + j + k * 1.0e-3


def _rank_main(rank, world, port, table_name, n, nz, out):
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from pyshield_b200.halo import HaloExchange, cubed_sphere, doubly_periodic
    from pyshield_b200.quantity import Quantity

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        table = cubed_sphere() if table_name == "cube" else doubly_periodic((1, 2))
        h = 3
        qs = []
        for f in range(2):  # u_dt, v_dt
            d = torch.full((n + 2 * h + 1, n + 2 * h + 1, nz + 1), -7.0, dtype=torch.float64)
            for i in range(n):
                for j in range(n):
                    for k in range(nz):
                        d[h + i, h + j, k] = _value(rank, f, i, j, k)
            qs.append(Quantity(d, ("x", "y", "z"), "", (h, h, 0), (n, n, nz)))
        ex = HaloExchange(qs, table, rank)
        ex.start()
        ex.wait()
        out.put((rank, [q.data.numpy().copy() for q in qs]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(table_name, world, n=5, nz=3):
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, table_name, n, nz, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def _check(res, table, n, nz, h=3):
    for a, fields in res.items():
        for f, d in enumerate(fields):
            expect = np.full_like(d, -7.0)
            for i in range(n):
                for j in range(n):
                    for k in range(nz):
                        expect[h + i, h + j, k] = _value(a, f, i, j, k)
            for e, b in table[a].items():
                for p in range(n):
                    q = n - 1 - p if b.reverse else p
                    bi, bj = _interior_cell(b.edge, q, n)
                    hi, hj = {WEST: (-1, p), EAST: (n, p), SOUTH: (p, -1), NORTH: (p, n)}[e]
                    for k in range(nz):
                        expect[h + hi, h + hj, k] = _value(b.rank, f, bi, bj, k)
            np.testing.assert_array_equal(d, expect, err_msg=f"rank {a} field {f}")


def test_two_ranks_periodic_exchange():
    res = _run("periodic", 2)
    _check(res, doubly_periodic((1, 2)), 5, 3)


def test_six_cube_tiles_exchange():
    res = _run("cube", 6)
    _check(res, cubed_sphere(), 5, 3)
