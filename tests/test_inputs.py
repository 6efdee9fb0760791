"""The synthetic state generator follows the stated distributions."""
import numpy as np

from pyshield_b200 import constants as C
from pyshield_b200.inputs import cube_area, make_state


def test_distributions():
    s, area = make_state(2000, 79, seed=5, n_cube=12)
    t = s["pt"]
    assert np.all(s["delz"] < 0) and np.all(s["delprsi"] > 0)
    ps = s["delprsi"].sum(axis=0) + 100.0
    assert ps.min() >= 980e2 - 1 and ps.max() <= 1030e2 + 1
    warm = t > C.TICE
    assert np.all(s["qrain"][~warm] == 0) and np.all(s["qice"][warm] == 0)
    assert np.all((s["qliquid"] == 0) | (t > 253.0))
    cond = s["qliquid"] + s["qrain"] + s["qice"] + s["qsnow"] + s["qgraupel"]
    assert np.array_equal(s["qcld"], np.where(cond > 1e-6, 1.0, 0.0))
    assert 0.2 < s["land"].mean() < 0.4
    assert np.allclose(area, cube_area(12))
    for k in ("pt_dt", "qv_dt", "udt"):
        assert not s[k].any()


def test_seeded():
    a, _ = make_state(50, 20, seed=3)
    b, _ = make_state(50, 20, seed=3)
    for k in a:
        assert np.array_equal(a[k], b[k])
