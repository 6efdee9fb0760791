"""Full-size parity of the plain FP64 step and its column branch flags.

* The column flags of every sub-step -- which species fall (the reference's
  column-wide ``no_fall``, microphysics.py:349-368 and :773-1168) and the
  melting level (the first level whose ``stop_k`` is 1, :706-724) -- are
  compared bit for bit with the oracle's, on states where species are absent
  from some columns, with one and two sub-steps.
* The C96 L127 rollout: 6 x 96 x 96 = 55,296 columns x 127 levels, 10 steps
  of 180 s. Between steps the state takes the step's tendencies
  (``update_physics_state_with_tendencies``, physics.py:151-194), and the
  tendencies are zeroed before each step, as the physics driver's
  ``prepare_microphysics`` does (physics.py:133-143). Every step is checked
  against the oracle run on all host cores from the same input state and
  the same cloud-fraction accumulator.

The gate is the plain relative bound max|gpu - oracle| <= 1e-12 max|oracle|
per field, with no absolute floor, for the ten tendencies, wmp and the
accumulator. The four surface totals are compared relative to the column's
condensate (``mp_helpers.precip_scale``): the reference sums the surface flux
as a running difference that cancels to its last digits when little mass
reaches the ground, while the kernels use the telescoped flux.
"""
import time

import numpy as np
import pytest

from golden_io import MP_TENDENCIES
from mp_helpers import TOL_PLAIN, device_state, from_storage_np, precip_scale

pytestmark = pytest.mark.gpu

PLAIN_FIELDS = MP_TENDENCIES + ("wmp", "qaz")
PRECIP = ("rain", "snow", "ice", "graupel")
STATE_FIELDS = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi",
                "delz", "wmp")
STATE_UPDATE = (("qvapor", "qv_dt"), ("qliquid", "ql_dt"), ("qrain", "qr_dt"), ("qice", "qi_dt"),
                ("qsnow", "qs_dt"), ("qgraupel", "qg_dt"), ("qcld", "qa_dt"), ("pt", "pt_dt"), ("ua", "udt"),
                ("va", "vdt"))


def _host(q, nx, ny, L):
    """(L, n) numpy copy of an i-fastest storage's compute domain."""
    arr = q.data.permute(2, 1, 0).contiguous().cpu().numpy().transpose(2, 1, 0)
    return from_storage_np(arr, nx, ny, L)


def _gpu_outputs(mp, ms, nx, ny, L):
    o = {t: _host(getattr(ms, t), nx, ny, L) for t in MP_TENDENCIES + ("wmp",)}
    for p in PRECIP:
        o[p] = getattr(mp, p).t().contiguous().cpu().numpy().reshape(-1)
    o["qaz"] = mp.get_qaz().cpu().numpy().reshape(L, -1)
    return o


def _knock_out(state, seed):
    """Remove species from random columns (each species from about a third
    of the columns), so that the no_fall flags take both values."""
    rng = np.random.default_rng(seed)
    n = state["pt"].shape[1]
    for f in ("qrain", "qice", "qsnow", "qgraupel", "qliquid"):
        cols = rng.random(n) < 0.35
        state[f][:, cols] = 0.0
    return state


def _plain_errors(gpu, ref, state, dt):
    """Per field: (max |gpu - oracle|, allowance). Plain 1e-12 relative for
    the tendencies, wmp and qaz; the column-condensate scale for the
    surface totals."""
    out = {}
    for f in PLAIN_FIELDS:
        out[f] = (float(np.max(np.abs(gpu[f] - ref[f]))), TOL_PLAIN * float(np.max(np.abs(ref[f]))))
    ps = precip_scale(state, dt)
    for p in PRECIP:
        out[p] = (float(np.max(np.abs(gpu[p] - ref[p]))), TOL_PLAIN * max(ps, float(np.max(np.abs(ref[p])))))
    return out


@pytest.mark.parametrize("dt,mp_time,extra", [(150.0, 150.0, {}), (225.0, 150.0, {}),
                                              (180.0, 150.0, {"vi_fac": 1.0e-6, "do_sedi_heat": True})])
def test_branch_flags_match_oracle(dt, mp_time, extra):
    import torch

    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import copy_state, make_state
    from pyshield_b200.microphysics import Microphysics, flag_fields

    nx, ny, L = 24, 18, 79
    n = nx * ny
    state, area = make_state(n, L, seed=31, n_cube=nx, sat_fraction=0.1)
    state = _knock_out(state, 5)
    cfg = PhysicsConfig(dt_atmos=dt, mp_time=mp_time, **extra)
    # the flag-recording launch and the production launch on two copies
    ms_f, sf, qf, gd = device_state(state, area, nx, ny)
    ms_p = device_state(state, area, nx, ny)[0]
    mp_f = Microphysics(sf, qf, gd, cfg)
    mp_p = Microphysics(sf, qf, gd, cfg)
    flags = mp_f.step_with_flags(ms_f, dt)
    mp_p(ms_p, dt)
    torch.cuda.synchronize()
    got_f, got_p = _gpu_outputs(mp_f, ms_f, nx, ny, L), _gpu_outputs(mp_p, ms_p, nx, ny, L)
    for f in got_p:
        assert np.array_equal(got_f[f], got_p[f]), f"flag-recording launch changed {f}"
    orc = OracleMicrophysics(cfg, n, L, area)
    orc(copy_state(state), dt)
    gf = flags.cpu().numpy().reshape(flags.shape[0], -1)
    assert gf.shape == orc.flags.shape
    bad = {k: int(np.sum(v != flag_fields(orc.flags)[k])) for k, v in flag_fields(gf).items()}
    assert gf.tobytes() == orc.flags.tobytes(), f"column flags differ from the oracle's: {bad}"
    ff = flag_fields(gf)
    for k in ("rain_falls_1", "ice_falls", "snow_falls", "graupel_falls"):
        if k == "ice_falls" and extra.get("vi_fac", 1.0) < 1e-5:
            assert not ff[k].any()
        else:
            assert 0 < ff[k].mean() < 1, k  # both values occur


def test_c96_l127_ten_steps():
    """C96 L127, 10 steps of 180 s, every step against the oracle
    on all host cores."""
    import torch

    from oracle_pool import OraclePool
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200._lib import load
    from pyshield_b200.coupling import update_physics_state_with_tendencies
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import Microphysics

    n_cube, L, dt, nsteps = 96, 127, 180.0, 10
    nx, ny = n_cube, 6 * n_cube
    n = nx * ny
    cfg_kwargs = {"dt_atmos": dt}
    cfg = PhysicsConfig(**cfg_kwargs)
    pool = OraclePool()
    try:
        state, area = make_state(n, L, seed=2024, n_cube=n_cube)
        ms, sf, qf, gd = device_state(state, area, nx, ny)
        mp = Microphysics(sf, qf, gd, cfg)
        land = state["land"]
        ntimes = load().shield_mp_substeps(mp._handle, dt)
        worst = {}
        t_orc = 0.0
        for step in range(nsteps):
            for t in MP_TENDENCIES:
                getattr(ms, t).data.zero_()
            inputs = {f: _host(getattr(ms, f), nx, ny, L) for f in STATE_FIELDS}
            qaz0 = mp.get_qaz().cpu().numpy().reshape(L, n)
            mp(ms, dt)
            torch.cuda.synchronize()
            got = _gpu_outputs(mp, ms, nx, ny, L)
            t0 = time.perf_counter()
            ref = pool.run(inputs, land, area, qaz0, cfg_kwargs, dt, ntimes)
            t_orc += time.perf_counter() - t0
            errs = _plain_errors(got, ref, inputs, dt)
            for f, (d, allow) in errs.items():
                w = worst.get(f, (0.0, 0.0, -1))
                r = d / allow if allow > 0 else (0.0 if d == 0 else float("inf"))
                if r >= w[0]:
                    worst[f] = (r, d / max(allow / TOL_PLAIN, 1e-300), step)
            # the state update between steps, in place: X = X + X_dt dt
            upd = [getattr(ms, x) for x, _ in STATE_UPDATE]
            tnd = [getattr(ms, t) for _, t in STATE_UPDATE]
            update_physics_state_with_tendencies(*upd, *tnd, *upd, dt)
        torch.cuda.synchronize()
    finally:
        pool.close()
    table = ", ".join(f"{f} {v[1]:.2e} (step {v[2]})" for f, v in worst.items())
    print(f"\nC96 L127 x {nsteps} steps, worst relative error per field: {table}; "
          f"oracle {t_orc:.1f} s on {pool.procs} processes")
    bad = {f: v for f, v in worst.items() if v[0] > 1.0}
    assert not bad, f"fields above the 1e-12 gate (allowance multiple, relative error, step): {bad}"
