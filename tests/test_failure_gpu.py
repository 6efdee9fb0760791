"""Failure detection of the microphysics step, without a GPU fault.

The kernel records the first column whose outputs hold a NaN or an infinity
in a device error word; ``Microphysics.check()`` (``shield_mp_check``) waits
for the stream, raises naming the column and clears the word. The bad value
is planted on the host, in one column's input; nothing traps or hangs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(nx=12, ny=6, nz=79):
    from mp_helpers import device_state
    from pyshield_b200.inputs import make_state

    state, area = make_state(nx * ny, nz, seed=17, n_cube=12)
    return device_state(state, area, nx, ny)


def _setup(dt=150.0):
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.microphysics import Microphysics

    ms, sf, qf, gd = _state()
    mp = Microphysics(sf, qf, gd, PhysicsConfig(dt_atmos=int(dt)))
    return ms, mp, dt


def test_clean_step_checks_clean():
    ms, mp, dt = _setup()
    mp(ms, dt)
    assert mp.check() == -1


@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_nonfinite_input_column_is_reported(bad):
    from pyshield_b200._lib import ShieldError

    ms, mp, dt = _setup()
    i, j = 5, 3
    good = float(ms.pt.view[i, j, 40])
    ms.pt.view[i, j, 40] = bad
    mp(ms, dt)
    with pytest.raises(ShieldError) as exc:
        mp.check()
    col = i + mp.nx * j
    assert f"column {col} " in str(exc.value) and f"i = {i}, j = {j}" in str(exc.value)
    # the record is cleared: the same handle on a clean state (the bad step
    # also left NaN in that column's wmp and cloud-fraction accumulator)
    ms2 = _state()[0]
    assert float(ms2.pt.view[i, j, 40]) == good
    mp.set_qaz(mp.get_qaz().nan_to_num(0.0, posinf=0.0, neginf=0.0))
    mp(ms2, dt)
    assert mp.check() == -1
    assert np.isfinite(ms2.pt_dt.view.cpu().numpy()).all()
