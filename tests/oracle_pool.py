"""The FP64 oracle over a whole domain on every host core, for the parity
tests at full size (tens of thousands of columns, which one core would take
minutes to step).

The columns of a domain are independent, so the domain is cut into
contiguous slices, one per worker process. Inputs and outputs travel through
file-backed memory maps in a temporary directory rather than through pipes.
The workers are spawned (never forked), so the pool may start after CUDA has
been initialised in the parent.
"""
import multiprocessing as mp
import os
import shutil
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
IN_FIELDS = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi", "delz",
             "wmp")
TENDENCIES = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")
PRECIP = ("rain", "snow", "ice", "graupel")


def _map(path, name, shape, mode, dtype=np.float64):
    return np.memmap(os.path.join(path, name), dtype=dtype, mode=mode, shape=shape)


def _slice(args):
    """One worker's columns [lo, hi): read the inputs, run the oracle's step
    from the given accumulator (zero incoming tendencies, as the physics
    driver zeroes them before the microphysics), write the outputs."""
    path, L, n, lo, hi, cfg_kwargs, dt, ntimes = args
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200._config import PhysicsConfig

    m = hi - lo
    s = {f: np.array(_map(path, f, (L, n), "r")[:, lo:hi]) for f in IN_FIELDS}
    for t in TENDENCIES:
        s[t] = np.zeros((L, m))
    s["land"] = np.array(_map(path, "land", (n,), "r")[lo:hi])
    area = np.array(_map(path, "area", (n,), "r")[lo:hi])
    orc = OracleMicrophysics(PhysicsConfig(**cfg_kwargs), m, L, area)
    orc.qaz = np.array(_map(path, "qaz", (L, n), "r")[:, lo:hi])
    precip = orc(s, dt)
    for f in TENDENCIES + ("wmp",):
        out = _map(path, "out_" + f, (L, n), "r+")
        out[:, lo:hi] = s[f]
        out.flush()
    out = _map(path, "out_qaz", (L, n), "r+")
    out[:, lo:hi] = orc.qaz
    out.flush()
    out = _map(path, "out_precip", (4, n), "r+")
    for i, p in enumerate(PRECIP):
        out[i, lo:hi] = precip[p]
    out.flush()
    out = _map(path, "out_flags", (ntimes, n), "r+", np.int32)
    out[:, lo:hi] = orc.flags
    out.flush()


class OraclePool:
    """``run(inputs, land, area, qaz, cfg_kwargs, dt, ntimes)`` steps a whole
    domain with the oracle on ``procs`` processes and returns its outputs as
    numpy arrays: the ten tendencies and wmp (L, n), qaz (L, n), the four
    surface totals (n,) and the column flags (ntimes, n)."""

    def __init__(self, procs=None):
        self.procs = procs or os.cpu_count() or 1
        self.pool = mp.get_context("spawn").Pool(self.procs)
        self.dir = tempfile.mkdtemp(prefix="oracle_pool_")

    def run(self, inputs, land, area, qaz, cfg_kwargs, dt, ntimes):
        L, n = inputs["pt"].shape
        path = self.dir
        for f in IN_FIELDS:
            mm = _map(path, f, (L, n), "w+")
            mm[:] = inputs[f]
            mm.flush()
        for name, arr, shape in (("land", land, (n,)), ("area", area, (n,)), ("qaz", qaz, (L, n))):
            mm = _map(path, name, shape, "w+")
            mm[:] = arr
            mm.flush()
        for f in TENDENCIES + ("wmp", "qaz"):
            _map(path, "out_" + f, (L, n), "w+").flush()
        _map(path, "out_precip", (4, n), "w+").flush()
        _map(path, "out_flags", (ntimes, n), "w+", np.int32).flush()
        bounds = np.linspace(0, n, self.procs + 1).astype(int)
        work = [(path, L, n, int(a), int(b), cfg_kwargs, dt, ntimes) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
        self.pool.map(_slice, work)
        out = {f: np.array(_map(path, "out_" + f, (L, n), "r")) for f in TENDENCIES + ("wmp", "qaz")}
        pr = np.array(_map(path, "out_precip", (4, n), "r"))
        for i, p in enumerate(PRECIP):
            out[p] = pr[i]
        out["flags"] = np.array(_map(path, "out_flags", (ntimes, n), "r", np.int32))
        return out

    def close(self):
        self.pool.close()
        self.pool.join()
        shutil.rmtree(self.dir, ignore_errors=True)
