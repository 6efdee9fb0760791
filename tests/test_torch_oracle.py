"""The torch transcription of the step (tests/torch_oracle.py) on the CPU.

Its forward equals the numpy oracle's to round-off. torch's CPU exp, log and
pow differ from numpy's in the last place, so the check is not bit for bit.
Its forward-mode derivatives (torch.autograd.forward_ad) equal the exact
Jacobian of the dual-number column reference (tests/adjoint/column.h).
These are two independent automatic differentiations of the same pinned
step, and the GPU adjoint is checked against the first in
test_adjoint_torch_gpu.py.
"""
import numpy as np
import pytest

TOL_FWD = 1.0e-12
TOL_JVP = 1.0e-9
# The oracle sums the surface flux as the reference does, a running sum
# m1_k = m1_{k-1} + q_k - qm_k that cancels to its last digits when little
# mass reaches the ground; the column reference (like the kernels) uses the
# telescoped form. A surface total below this fraction of the column's
# condensate (in mm/day) is round-off in the oracle, value and derivative,
# and is not compared.
SURFACE_RES = 1.0e-12


def precip_columns(state, dt):
    """Per column, the surface total [mm/day] its whole condensate would make."""
    from pyshield_b200 import constants as C

    cond = sum(np.abs(state[f]) for f in ("qliquid", "qrain", "qice", "qsnow", "qgraupel"))
    return np.sum(cond * state["delprsi"], axis=0) * 86400.0 / (dt * C.GRAV)


@pytest.mark.parametrize("kw,dt", [({}, 150.0), ({"mp_time": 150.0}, 225.0)])
def test_torch_transcription_forward_matches_oracle(kw, dt):
    import torch

    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import copy_state, make_state
    from mp_helpers import floors
    from torch_oracle import OUTPUTS, TorchOracle

    n, L = 864, 79
    state, area = make_state(n, L, seed=21, n_cube=12, sat_fraction=0.1)
    cfg = PhysicsConfig(dt_atmos=int(dt), **kw)
    qaz0 = np.random.default_rng(2).uniform(0.0, 2.0, (L, n))
    s = copy_state(state)
    ref = OracleMicrophysics(cfg, n, L, area)
    ref.qaz = qaz0.copy()
    pr = ref(s, dt)
    expect = {o: s[o] for o in OUTPUTS[:11]}
    expect["qaz"] = ref.qaz
    expect.update(pr)
    got = TorchOracle(cfg, n, L, area, dt)({k: torch.as_tensor(v) for k, v in state.items()}, torch.as_tensor(qaz0))
    # the GPU gate's allowance: 1e-12 of the field's size plus the round-off
    # floor of a tendency (or of a surface total's column sum)
    fl = floors(state, expect, dt)
    for o in OUTPUTS:
        e, g = np.asarray(expect[o]), got[o].numpy()
        assert np.abs(g - e).max() <= TOL_FWD * float(np.abs(e).max()) + fl.get(o, 0.0), o


def test_forward_mode_jvp_matches_dual_column_reference():
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200._lib import make_config
    from pyshield_b200.inputs import make_state
    from test_adjoint_pointwise import build_harness, column_ref
    from torch_oracle import OUTPUTS, STATE, jvp_per_input

    lib = build_harness()
    n, L, dt = 6, 79, 150.0
    state, area = make_state(n, L, seed=23, n_cube=12, sat_fraction=0.3)
    rng = np.random.default_rng(3)
    qaz0 = rng.uniform(0.0, 2.0, (L, n))
    X = np.stack([state[f] for f in STATE[:-1]] + [qaz0])
    floor = np.array([0.0] * 7 + [1e-2, 1.0, 1.0, 0.0, 0.0, 0.1, 0.1])[:, None, None]
    DX = rng.normal(size=X.shape) * (np.abs(X) + floor)
    pc = PhysicsConfig(dt_atmos=int(dt))
    Y, T = jvp_per_input(pc, dt, X, state["land"], area, DX)
    cfg_c = make_config(pc)
    n3 = len(OUTPUTS) - 4
    pscale = precip_columns(state, dt)
    entries = fails = 0
    for c in range(n):
        YB = rng.normal(size=n3 * L + 4)
        JD, JS, Yc = column_ref(lib, cfg_c, dt, X[:, :, c], state["land"][c], area[c], DX[:, :, c], YB)
        for o in range(len(OUTPUTS)):
            yb = YB[o * L:(o + 1) * L] if o < n3 else YB[n3 * L + (o - n3)]
            if o >= n3 and abs(Yc[n3 * L + (o - n3)]) <= SURFACE_RES * pscale[c]:
                continue  # a surface total below the oracle's resolution
            for f in range(len(STATE)):
                if JS[o, f] == 0.0:
                    assert np.all(T[OUTPUTS[o]][f][..., c] == 0.0), (OUTPUTS[o], STATE[f], c)
                    continue
                entries += 1
                jd = float(np.sum(yb * T[OUTPUTS[o]][f][..., c]))
                if abs(jd - JD[o, f]) > TOL_JVP * JS[o, f]:
                    fails += 1
    assert entries > 0
    assert fails <= 0.005 * entries, f"{fails} of {entries} entries"
