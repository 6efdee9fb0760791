"""Mixed-precision form (FP32 process rates, FP64 saturation adjustment,
sedimentation, budgets) against the FP64 oracle.

Its error is stated, not hidden: per field the max and rms of
|mixed - oracle| / max|oracle| are printed (run pytest with -s) and bounded.
Total water is conserved to FP64 round-off: every transfer is applied to its
two species in FP64."""
import numpy as np
import pytest

from golden_io import MP_TENDENCIES, PRECIP
from mp_helpers import floors, run_gpu

pytestmark = pytest.mark.gpu

FIELDS = MP_TENDENCIES + ("wmp", "qaz") + PRECIP
# bound on max |mixed - oracle| / max|oracle| per field (FP32 rates: ~1e-7
# relative per rate, amplified where a rate crosses a process threshold)
TOL_MIXED = 5e-5


def _oracle(cfg, state, area, n, L, dt):
    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200.inputs import copy_state

    s = copy_state(state)
    mp = OracleMicrophysics(cfg, n, L, area)
    pr = mp(s, dt)
    out = {f: s[f] for f in MP_TENDENCIES + ("wmp",)}
    out.update(pr)
    out["qaz"] = mp.qaz
    return out


def _errors(got, ref, state, dt):
    fl = floors(state, ref, dt)
    res = {}
    for f in FIELDS:
        scale = max(float(np.max(np.abs(ref[f]))), fl.get(f, 0.0) / 1e-12 if f in PRECIP else 0.0)
        d = np.abs(got[f] - ref[f]) / (scale if scale > 0 else 1.0)
        res[f] = (float(d.max()), float(np.sqrt(np.mean(d * d))))
    return res


@pytest.mark.parametrize("nlev,dt,sat", [(79, 150.0, 0.0), (79, 180.0, 0.1), (127, 180.0, 0.0)])
def test_mixed_error_vs_fp64_oracle(nlev, dt, sat):
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import make_state

    nx, ny = 36, 24
    n = nx * ny
    state, area = make_state(n, nlev, seed=31 + nlev, n_cube=12, sat_fraction=sat)
    cfg = PhysicsConfig(dt_atmos=dt)
    ref = _oracle(cfg, state, area, n, nlev, dt)
    got = run_gpu(cfg, state, area, nx, ny, dt, 1, precision="mixed")[0]
    errs = _errors(got, ref, state, dt)
    print(f"\nmixed vs FP64 oracle, C12-sized L{nlev} dt {dt:g} sat_fraction {sat}: field max rms")
    for f, (mx, rms) in errs.items():
        print(f"  {f:8s} {mx:.2e} {rms:.2e}")
    bad = {f: e for f, e in errs.items() if e[0] > TOL_MIXED}
    assert not bad, bad


def test_mixed_conserves_water():
    from pyshield_b200 import constants as C
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import make_state

    nx, ny, L, dt = 48, 32, 79, 150.0
    n = nx * ny
    state, area = make_state(n, L, seed=11, n_cube=48)
    cfg = PhysicsConfig(dt_atmos=dt, fix_negative=False)
    got = run_gpu(cfg, state, area, nx, ny, dt, 1, precision="mixed")[0]
    dp = state["delprsi"]
    qsum_dt = sum(got[f] for f in ("qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt"))
    water_dt = np.sum(qsum_dt * dp, axis=0) * C.RGRAV
    precip = (got["rain"] + got["snow"] + got["ice"] + got["graupel"]) / 86400.0
    # relative to the column's total water tendency scale (vapour + condensate)
    col_water = np.sum((state["qvapor"] + state["qliquid"] + state["qrain"] + state["qice"] + state["qsnow"]
                        + state["qgraupel"]) * dp, axis=0) * C.RGRAV / dt
    assert np.max(np.abs(water_dt + precip) / col_water) < 1e-12
