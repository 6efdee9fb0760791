"""One-point halo exchange of the wind tendencies between tile-owning ranks.

``ApplyPhysicsToDycore`` (pySHiELD/update/fv_update_phys.py:134-147,
173-188) fills a one-point halo of ``u_dt`` and ``v_dt`` from the
neighbouring ranks before ``AGrid2DGridPhysics`` reads them: it starts the
exchange, runs ``update_pressure_and_surface_winds``, then waits. The
reference does this with NDSL's halo updater over its communicator. Here it
is point-to-point messages over ``torch.distributed`` -- NCCL between GPUs,
gloo on the CPU -- with the same ``start()`` / ``wait()`` split, so the
transfer overlaps the column work launched between the two calls.

What travels: for every edge of a rank's domain, the row or column of
compute-domain points along that edge (all levels) goes to the neighbour that
edge touches, which writes it into its halo along its own touching edge. The
halo's corner points are not exchanged (``AGrid2DGridPhysics`` reads the
tendencies at i - 1 and j - 1 of edge points only).

The neighbours come from an edge table (``EdgeTable``): for each of a rank's
four edges, the rank on the other side, which of that rank's edges touches
it, and whether the edge's points run the other way there. ``cubed_sphere``
gives the table of the six cube tiles, one rank per tile, in the cubed-sphere
tile numbering the FV3 family uses (even tiles: east and south neighbours
unrotated, west and north ones rotated; odd tiles the other way round);
``doubly_periodic`` that of ranks laid out on a periodic plane.
"""

from typing import Dict, List, NamedTuple, Sequence

WEST, EAST, SOUTH, NORTH = 0, 1, 2, 3
EDGE_NAMES = ("west", "east", "south", "north")


class Boundary(NamedTuple):
    """The neighbour across one edge: its rank, the edge of its own domain
    that touches ours, and whether its points along that edge run the other
    way (so that a strip must be reversed)."""

    rank: int
    edge: int
    reverse: bool


EdgeTable = Dict[int, Dict[int, Boundary]]  # rank -> edge -> Boundary


def cubed_sphere(ntiles=6) -> EdgeTable:
    """Edge table of the six cubed-sphere tiles, rank = tile (0 .. 5).

    Even tile t: east -> t + 1 (its west edge, same direction), south ->
    t - 1 (its north edge, same direction), north -> t + 2 (its west edge,
    reversed), west -> t - 2 (its north edge, reversed). Odd tile t: west ->
    t - 1, north -> t + 1 (unrotated), east -> t + 2 (its south edge,
    reversed), south -> t - 2 (its east edge, reversed). Tile numbers mod 6.
    """
    if ntiles != 6:
        raise ValueError("a cube has six tiles")
    table = {}
    for t in range(6):
        if t % 2 == 0:
            table[t] = {
                EAST: Boundary((t + 1) % 6, WEST, False),
                SOUTH: Boundary((t - 1) % 6, NORTH, False),
                NORTH: Boundary((t + 2) % 6, WEST, True),
                WEST: Boundary((t - 2) % 6, NORTH, True),
            }
        else:
            table[t] = {
                WEST: Boundary((t - 1) % 6, EAST, False),
                NORTH: Boundary((t + 1) % 6, SOUTH, False),
                EAST: Boundary((t + 2) % 6, SOUTH, True),
                SOUTH: Boundary((t - 2) % 6, EAST, True),
            }
    return table


def doubly_periodic(layout) -> EdgeTable:
    """Ranks on a periodic plane of layout (ny_ranks, nx_ranks), rank =
    y * nx_ranks + x; every edge touches the facing edge of its neighbour,
    in the same direction."""
    ny_r, nx_r = layout
    table = {}
    for r in range(ny_r * nx_r):
        y, x = divmod(r, nx_r)
        table[r] = {
            WEST: Boundary(y * nx_r + (x - 1) % nx_r, EAST, False),
            EAST: Boundary(y * nx_r + (x + 1) % nx_r, WEST, False),
            SOUTH: Boundary(((y - 1) % ny_r) * nx_r + x, NORTH, False),
            NORTH: Boundary(((y + 1) % ny_r) * nx_r + x, SOUTH, False),
        }
    return table


def check_table(table: EdgeTable):
    """Every boundary is answered by its neighbour's: A's edge e touches B's
    edge f (reversed or not) exactly when B's edge f touches A's edge e the
    same way."""
    for a, edges in table.items():
        for e, b in edges.items():
            back = table[b.rank][b.edge]
            if back != Boundary(a, e, b.reverse):
                raise ValueError(f"rank {a} {EDGE_NAMES[e]} -> {b}, but its answer is {back}")


def _interior(q, e):
    """The compute-domain strip along edge e of quantity q: (points along
    the edge, levels)."""
    h0, h1, k0 = q.origin
    nx, ny, nz = q.extent
    d = q.data
    if e == WEST:
        return d[h0, h1:h1 + ny, k0:k0 + nz]
    if e == EAST:
        return d[h0 + nx - 1, h1:h1 + ny, k0:k0 + nz]
    if e == SOUTH:
        return d[h0:h0 + nx, h1, k0:k0 + nz]
    return d[h0:h0 + nx, h1 + ny - 1, k0:k0 + nz]


def _halo(q, e):
    """The halo strip just outside edge e (corners excluded)."""
    h0, h1, k0 = q.origin
    nx, ny, nz = q.extent
    d = q.data
    if e == WEST:
        return d[h0 - 1, h1:h1 + ny, k0:k0 + nz]
    if e == EAST:
        return d[h0 + nx, h1:h1 + ny, k0:k0 + nz]
    if e == SOUTH:
        return d[h0:h0 + nx, h1 - 1, k0:k0 + nz]
    return d[h0:h0 + nx, h1 + ny, k0:k0 + nz]


class HaloExchange:
    """One-point halo exchange of ``quantities`` (Quantity-likes with torch
    ``.data``, ``.origin``, ``.extent`` and at least one halo point) between
    the ranks of ``table``, over ``group`` (the default process group when
    None). ``start()`` posts the messages; ``wait()`` completes them and
    writes the halos. Every rank of the table must call both, in the same
    order as every other exchange it takes part in.

    Messages between two ranks are posted in the order of the receiving
    edge on both sides (and tagged with it), so that ranks sharing more
    than one edge pair them correctly on NCCL, which matches by order, as
    on gloo, which matches by tag."""

    def __init__(self, quantities: Sequence, table: EdgeTable, rank: int, group=None):
        import torch

        check_table(table)
        self.q = list(quantities)
        self.table = table
        self.rank = rank
        self.group = group
        self.edges = table[rank]
        for q in self.q:
            if q.origin[0] < 1 or q.origin[1] < 1:
                raise ValueError("the exchange needs at least one halo point on each side")
        dev = self.q[0].data.device
        self._send = {e: None for e in self.edges}
        self._recv = {e: None for e in self.edges}
        self._reqs: List = []
        self._torch = torch
        self._device = dev

    def _pack(self, e, reverse):
        t = self._torch
        parts = [_interior(q, e) for q in self.q]
        if reverse:
            parts = [p.flip(0) for p in parts]
        return t.cat([p.reshape(-1) for p in parts]).contiguous()

    def start(self):
        import torch.distributed as dist

        ops = []
        remote = {e: b for e, b in self.edges.items() if b.rank != self.rank}
        # sends, ordered by (neighbour, the neighbour's receiving edge)
        for e, b in sorted(remote.items(), key=lambda kv: (kv[1].rank, kv[1].edge)):
            buf = self._pack(e, b.reverse)
            self._send[e] = buf
            ops.append(dist.P2POp(dist.isend, buf, b.rank, group=self.group, tag=b.edge))
        # receives, ordered by (neighbour, our receiving edge)
        for e, b in sorted(remote.items(), key=lambda kv: (kv[1].rank, kv[0])):
            n = sum(_halo(q, e).numel() for q in self.q)
            buf = self._torch.empty(n, dtype=self.q[0].data.dtype, device=self._device)
            self._recv[e] = buf
            ops.append(dist.P2POp(dist.irecv, buf, b.rank, group=self.group, tag=e))
        # an edge that touches this rank's own domain (a periodic direction
        # with one rank) is a local copy
        for e, b in self.edges.items():
            if b.rank == self.rank:
                self._recv[b.edge] = self._pack(e, b.reverse)
        self._reqs = dist.batch_isend_irecv(ops) if ops else []

    def wait(self):
        for r in self._reqs:
            r.wait()
        self._reqs = []
        for e, buf in self._recv.items():
            if buf is None:
                continue
            off = 0
            for q in self.q:
                h = _halo(q, e)
                n = h.numel()
                h.copy_(buf[off:off + n].view(h.shape))
                off += n
        for e in self._send:
            self._send[e] = None
