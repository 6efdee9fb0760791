"""GPU parity of the microphysics step against the FP64 oracle.

The oracle is pinned bit-for-bit to the reference's own source by
tests/test_oracle_golden.py, so agreement here is agreement with pySHiELD.
Tolerance of the plain FP64 form, per field f:
    max |gpu - oracle| <= 1e-12 * max |oracle|
for the ten tendencies, wmp, qice, qsnow and the accumulator (no absolute
floor unless mp_helpers.TENDENCY_FLOOR names the field with its reason), and
    max |gpu - oracle| <= 1e-12 * max(max |oracle|, column condensate in mm/day)
for a surface precipitation total: the reference sums the surface flux as a
running difference that cancels to its last digits when little mass reaches
the ground, while the kernels use the telescoped flux.
"""
import numpy as np
import pytest

from golden_io import MP_CASES, MP_TENDENCIES, PRECIP, load, mp_inputs
from mp_helpers import TOL_PLAIN, assert_close, field_errors, gpu_floors as floors, run_gpu

pytestmark = pytest.mark.gpu

FIELDS = MP_TENDENCIES + ("wmp", "qice", "qsnow", "qaz") + PRECIP


def _golden_step(z, step):
    out = {}
    for f in FIELDS:
        out[f] = np.array(z[f"s{step}_{f}"])
    return out


@pytest.mark.parametrize("layout", ["ifirst", "kfirst"])
@pytest.mark.parametrize("name", MP_CASES)
def test_golden_cases(name, layout):
    from pyshield_b200._config import PhysicsConfig

    z, meta = load(name)
    cfg = PhysicsConfig(**meta["config"])
    state, area = mp_inputs(z)
    outs = run_gpu(cfg, state, area, meta["nx"], meta["ny"], meta["dt"], meta["nsteps"], layout=layout)
    for step, o in enumerate(outs):
        ref = _golden_step(z, step)
        assert_close(o, ref, FIELDS, TOL_PLAIN, ctx=f"{name}/{layout}/step{step}", fl=floors(state, ref, meta["dt"]))


def _oracle(cfg, state, area, n, L, dt, nsteps):
    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200.inputs import copy_state

    s = copy_state(state)
    mp = OracleMicrophysics(cfg, n, L, area)
    outs = []
    for _ in range(nsteps):
        pr = mp(s, dt)
        o = {f: s[f].copy() for f in MP_TENDENCIES + ("wmp", "qice", "qsnow")}
        o.update(pr)
        o["qaz"] = mp.qaz.copy()
        outs.append(o)
    return outs


CONFIGS = {
    "default": {},
    "sedi_heat_bigg": dict(do_sedi_heat=True, fast_sat_adj=False, do_qa=False),
    "hydrostatic_noslope": dict(hydrostatic=True, z_slope_ice=False, z_slope_liq=False, sedi_transport=False),
}


@pytest.mark.parametrize("cname", sorted(CONFIGS))
@pytest.mark.parametrize("nlev,dt", [(79, 150.0), (127, 180.0), (63, 450.0), (30, 150.0), (90, 180.0), (160, 150.0)])
def test_c12_vs_oracle(cname, nlev, dt):
    """C12 (6 x 12 x 12 = 864 columns) synthetic state, one step; every launch
    shape of the level ranges (up to 32, 64, 80, 96, 128 and 256 levels)."""
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import make_state

    nx, ny = 36, 24
    n = nx * ny
    state, area = make_state(n, nlev, seed=nlev + len(cname), n_cube=12)
    cfg = PhysicsConfig(dt_atmos=dt, **CONFIGS[cname])
    ref = _oracle(cfg, state, area, n, nlev, dt, 1)[0]
    got = run_gpu(cfg, state, area, nx, ny, dt, 1)[0]
    assert_close(got, ref, FIELDS, TOL_PLAIN, ctx=f"C12 L{nlev} {cname}", fl=floors(state, ref, dt))


def test_saturation_threshold_columns():
    """Columns sitting on the saturation-adjustment thresholds (RH ~ 1)."""
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import make_state

    nx, ny, L, dt = 24, 16, 79, 150.0
    n = nx * ny
    state, area = make_state(n, L, seed=7, n_cube=12, sat_fraction=1.0)
    cfg = PhysicsConfig(dt_atmos=dt)
    ref = _oracle(cfg, state, area, n, L, dt, 2)
    got = run_gpu(cfg, state, area, nx, ny, dt, 2)
    for s in range(2):
        errs = field_errors(got[s], ref[s], FIELDS, TOL_PLAIN, floors(state, ref[s], dt))
        assert max(e[0] for e in errs.values()) <= 1.0, errs


def test_timestep_change_recomputes_substeps():
    """A new timestep re-derives ntimes/dts (``_update_timestep_if_needed``)."""
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import make_state

    nx, ny, L = 12, 12, 40
    n = nx * ny
    state, area = make_state(n, L, seed=3, n_cube=12)
    cfg = PhysicsConfig(dt_atmos=150.0)
    for dt in (150.0, 225.0, 600.0):
        ref = _oracle(cfg, state, area, n, L, dt, 1)[0]
        got = run_gpu(cfg, state, area, nx, ny, dt, 1)[0]
        assert_close(got, ref, FIELDS, TOL_PLAIN, ctx=f"dt={dt}", fl=floors(state, ref, dt))


def test_column_water_budget():
    """Total water is conserved: the column water tendency plus the surface
    precipitation flux vanishes (to round-off) in every column."""
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import make_state
    from pyshield_b200 import constants as C

    nx, ny, L, dt = 48, 32, 79, 150.0
    n = nx * ny
    state, area = make_state(n, L, seed=11, n_cube=48)
    cfg = PhysicsConfig(dt_atmos=dt, fix_negative=False)
    got = run_gpu(cfg, state, area, nx, ny, dt, 1)[0]
    dp = state["delprsi"]
    qsum_dt = sum(got[f] for f in ("qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt"))
    # tendencies are of moist mixing ratios on the moist mass dp; precip in mm/day
    water_dt = np.sum(qsum_dt * dp, axis=0) * C.RGRAV  # kg m-2 s-1
    precip = (got["rain"] + got["snow"] + got["ice"] + got["graupel"]) / 86400.0
    scale = np.max(np.abs(precip)) + 1e-30
    assert np.max(np.abs(water_dt + precip)) / scale < 1e-9
