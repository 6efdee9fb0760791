"""Ensembles: many microphysics domains advanced by one persistent launch.

pySHiELD advances each domain with its own ``Microphysics.__call__``
(``pySHiELD/stencils/microphysics.py:1981-2263``). ``MicrophysicsEnsemble``
takes a list of members -- each a ``MicrophysicsState`` with its own domain
size, cell area and timestep, all sharing one ``PhysicsConfig`` and level
count -- and advances all of them with a single kernel launch whose blocks
walk the members' columns. The launch shape (columns per block, resident
blocks per SM) is chosen by ``autotune``; ``capture`` records the step in a
CUDA graph that ``replay`` re-runs with one call.

Each member's results are the ones its own ``Microphysics`` would produce
(the same kernel body and constants); the persistent cloud-fraction
accumulator of each member lives in the plan.
"""

import ctypes

from . import _lib
from ._lib import SHIELD_MP_MIXED, SHIELD_MP_PLAIN, ShieldMpFields, ShieldMpMember, check, load, make_config
from .microphysics import _current_stream
from .quantity import field2d, field3d

_PRECISION = {"plain": SHIELD_MP_PLAIN, "fp64": SHIELD_MP_PLAIN, "mixed": SHIELD_MP_MIXED}

# (columns per block, blocks per SM) launch shapes the autotuner times, by
# level count: 65..80 levels pack two columns per group of 5 warps, so a
# block holds 2, 4, 6 or 8 columns (shield_mp_ensemble_step)
CANDIDATES = ((1, 4), (1, 5), (2, 2), (2, 3), (4, 1), (4, 2))
CANDIDATES_PACKED = ((2, 4), (2, 5), (4, 2), (6, 1), (8, 1), (8, 2))


def launch_shapes(nz):
    """The launch shapes ``autotune`` tries for ``nz`` levels."""
    return CANDIDATES_PACKED if nz <= 80 else CANDIDATES


class MicrophysicsEnsemble:
    def __init__(self, namelist, states, areas, timesteps, precision="mixed"):
        """``states``: MicrophysicsState per member (fields with compute-domain
        extents (nx_m, ny_m, nz)); ``areas``: the members' cell areas (2-D
        quantities); ``timesteps``: the members' steps."""
        import torch

        if not (len(states) == len(areas) == len(timesteps)) or not states:
            raise ValueError("states, areas and timesteps must be non-empty lists of equal length")
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        lib = load()
        self.precision = precision
        self.states = list(states)
        self.areas = list(areas)
        ext0 = tuple(getattr(states[0].pt, "extent"))
        self.nz = int(ext0[2])
        nm = len(states)
        self._members = (ShieldMpMember * nm)()
        self._precip = []
        dev = None
        for m, (st, area, dt) in enumerate(zip(states, areas, timesteps)):
            nx, ny, nz = (int(v) for v in getattr(st.pt, "extent"))
            if nz != self.nz:
                raise ValueError("all members must have the same number of levels")
            F = ShieldMpFields()
            for name in _lib.MP_STATE_FIELDS + _lib.MP_TENDENCY_FIELDS:
                setattr(F, name, field3d(getattr(st, name), (nx, ny, nz)))
            F.land = field2d(st.land, (nx, ny))
            if dev is None:
                dev = st.pt.data.device
            pr = torch.zeros((4, ny, nx), dtype=torch.float64, device=dev)
            self._precip.append(pr)
            base, plane = pr.data_ptr(), nx * ny * 8
            F.rain, F.snow, F.ice, F.graupel = base, base + plane, base + 2 * plane, base + 3 * plane
            M = self._members[m]
            M.fields = F
            M.nx, M.ny, M.timestep = nx, ny, float(dt)
            M.area = field2d(area, (nx, ny))
        self._cfg = make_config(namelist)
        h = ctypes.c_void_p()
        check(
            lib.shield_mp_ensemble_create(ctypes.byref(self._cfg), self.nz, nm, self._members, _PRECISION[precision], ctypes.byref(h)),
            None,
            "shield_mp_ensemble_create",
        )
        self._plan = h
        self.tuned = (2, 2)
        self.timings = {}
        self.graph = None

    def precip(self, m):
        """(rain, snow, ice, graupel) of member m's last step, (nx, ny) each."""
        pr = self._precip[m]
        return tuple(pr[i].t() for i in range(4))

    def qaz(self, m):
        """Member m's persistent cloud-fraction accumulator, (nz, ny, nx)."""
        import torch

        M = self._members[m]
        out = torch.empty((self.nz, M.ny, M.nx), dtype=torch.float64, device=self._precip[m].device)
        rc = load().shield_mp_ensemble_qaz(self._plan, m, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(_current_stream(None)))
        check(rc, None, "shield_mp_ensemble_qaz")
        return out

    def step(self, cols_per_block=None, blocks_per_sm=None, stream=None):
        G, b = self.tuned
        if cols_per_block is not None:
            G = cols_per_block
        if blocks_per_sm is not None:
            b = blocks_per_sm
        rc = load().shield_mp_ensemble_step(self._plan, int(G), int(b), ctypes.c_void_p(_current_stream(stream)))
        check(rc, None, "shield_mp_ensemble_step")

    def autotune(self, candidates=None, reps=2):
        """Time each launch shape (by default ``launch_shapes(nz)``) with CUDA
        events (after one warm-up launch) and keep the fastest. Note that
        each timed launch advances the members' state, as a real step does."""
        import torch

        stream = torch.cuda.current_stream()
        best = None
        for G, b in candidates or launch_shapes(self.nz):
            self.step(G, b)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                self.step(G, b)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            self.timings[(G, b)] = ms
            if best is None or ms < best[0]:
                best = (ms, (G, b))
        self.tuned = best[1]
        return self.tuned, self.timings

    def capture(self):
        """Record one tuned step in a CUDA graph (replay() re-runs it)."""
        import torch

        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.step()  # warm (first-launch attribute setting happens outside the graph)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def __del__(self):
        p = getattr(self, "_plan", None)
        if p is not None and p.value:
            try:
                self.graph = None
                load().shield_mp_ensemble_destroy(p)
            except Exception:
                pass
            self._plan = None
