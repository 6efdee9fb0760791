"""Hand-written adjoints of the pointwise microphysics routines, on the CPU.

The routines of mp_physics.cuh are templates on their real type. The harness
(tests/adjoint/harness.cpp, built here with g++) runs each routine with
forward-mode dual numbers, which gives the exact Jacobian on the branch the
double evaluation takes, and compares J^T ybar with the hand-written adjoint
of mp_adjoint.cuh at many random points. The tolerance is relative to the
size of the terms that make up each component: the routine is run once more
with magnitude duals, which accumulate every derivative contribution in
absolute value, and the scale of component j is sum_i |ybar_i| |J|_ij. A
derivative that cancels to zero in exact arithmetic is then judged against
the size of its cancelling terms.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "adjoint", "harness.cpp")
OUT = os.path.join(HERE, "adjoint", "_build", "libadjh.so")
TOL = 1.0e-12
N = 4000


def build_harness():
    """Compile (when stale) and load the CPU harness."""
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    deps = [SRC, os.path.join(HERE, "adjoint", "dual.h"), os.path.join(HERE, "adjoint", "column.h")] + [
        os.path.join(ROOT, "pyshield_b200", "csrc", f) for f in ("mp_physics.cuh", "mp_adjoint.cuh", "mp_setup.h", "mp_params.h")
    ]
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(ROOT, "pyshield_b200", "csrc"),
               "-I", os.path.join(HERE, "adjoint"), SRC, "-o", OUT + ".tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-4000:]
        os.replace(OUT + ".tmp", OUT)
    return ctypes.CDLL(OUT)


@pytest.fixture(scope="module")
def harness():
    return build_harness()


def _cfg(**kw):
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200._lib import make_config

    return make_config(PhysicsConfig(dt_atmos=150, **kw))


def run(lib, name, X, YB, cfg=None, ts=150.0):
    dims = (ctypes.c_int * 3)()
    getattr(lib, f"adj_{name}_dims")(dims)
    nin, nd, nout = dims
    X = np.ascontiguousarray(X, dtype=np.float64)
    YB = np.ascontiguousarray(YB, dtype=np.float64)
    n = X.shape[0]
    assert X.shape == (n, nin) and YB.shape == (n, nout)
    xbh = np.zeros((n, nd))
    xbd = np.zeros((n, nd))
    xbs = np.zeros((n, nd))
    y = np.zeros((n, nout))
    c = cfg if cfg is not None else _cfg()
    P = ctypes.POINTER(ctypes.c_double)
    f = getattr(lib, f"adj_{name}")
    f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, P, P, P, P, P, P]
    p = lambda a: a.ctypes.data_as(P)  # noqa: E731
    assert f(ctypes.byref(c), ts, n, p(X), p(YB), p(xbh), p(xbd), p(y), p(xbs)) == 0
    return xbh, xbd, xbs, y


def check(xbh, xbd, xbs, what):
    err = np.abs(xbh - xbd)
    assert np.all(np.isfinite(xbd)), f"{what}: non-finite dual VJP"
    bad = err > TOL * xbs + 1e-300
    if bad.any():
        i, j = np.argwhere(bad)[0]
        raise AssertionError(
            f"{what}: {bad.sum()} components beyond {TOL:g}; first at point {i}, input {j}: "
            f"hand {xbh[i, j]:.17g} dual {xbd[i, j]:.17g} scale {xbs[i, j]:.3g}"
        )


def logu(rng, lo, hi, n):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def cond(rng, n, zero_frac=0.15, lo=1e-9, hi=3e-3):
    q = logu(rng, lo, hi, n)
    q[rng.random(n) < zero_frac] = 0.0
    return q


def qsat_w(t, den):
    # a smooth approximation of the liquid saturation mixing ratio
    es = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
    return es / (461.5 * t * den)


def test_saturation(harness):
    rng = np.random.default_rng(1)
    for name in ("wqs2", "iqs2"):
        ta = np.concatenate([rng.uniform(150.0, 400.0, N), rng.uniform(160.0, 185.0, N // 4)])
        den = rng.uniform(0.05, 1.5, ta.size)
        X = np.stack([ta, den], 1)
        YB = rng.normal(size=(ta.size, 2))
        xbh, xbd, xbs, _ = run(harness, name, X, YB)
        check(xbh, xbd, xbs, name)


def test_revap_racc(harness):
    rng = np.random.default_rng(2)
    tz = rng.uniform(240.0, 305.0, N)
    den = rng.uniform(0.3, 1.3, N)
    rh = rng.uniform(0.3, 1.1, N)
    qv = rh * qsat_w(tz, den)
    X = np.stack([cond(rng, N), cond(rng, N), cond(rng, N), cond(rng, N, 0.05), cond(rng, N), qv, tz, den,
                  np.sqrt(1.2 / den), np.full(N, 37.5), rng.uniform(0.01, 0.2, N)], 1)
    YB = rng.normal(size=(N, 7)) * np.array([1, 1, 1, 1, 1, 1, 1e-3])
    xbh, xbd, xbs, y = run(harness, "revap_racc", X, YB)
    changed = np.any(y != X[:, :7], axis=1)
    assert changed.mean() > 0.3
    check(xbh, xbd, xbs, "revap_racc")


def test_fall_speeds(harness):
    rng = np.random.default_rng(3)
    den = rng.uniform(0.05, 1.4, N)
    X = np.stack([cond(rng, N, 0.1, 1e-10, 1e-2), den], 1)
    xbh, xbd, xbs, _ = run(harness, "rain_fspeed", X, rng.normal(size=(N, 1)))
    check(xbh, xbd, xbs, "rain_fspeed")
    X = np.stack([cond(rng, N, 0.1, 1e-10, 1e-2), cond(rng, N, 0.1, 1e-10, 1e-2), cond(rng, N, 0.1, 1e-10, 1e-2),
                  rng.uniform(200.0, 300.0, N), den], 1)
    xbh, xbd, xbs, _ = run(harness, "fall_speed", X, rng.normal(size=(N, 3)))
    check(xbh, xbd, xbs, "fall_speed")
    for kw in ({"const_vi": True, "const_vs": True, "const_vg": True, "const_vr": True},):
        xbh, xbd, xbs, _ = run(harness, "fall_speed", X, rng.normal(size=(N, 3)), cfg=_cfg(**kw))
        check(xbh, xbd, xbs, "fall_speed const")


@pytest.mark.parametrize("prog_ccn", [False, True])
def test_autoconversion(harness, prog_ccn):
    rng = np.random.default_rng(4)
    ql = cond(rng, N, 0.05, 1e-7, 3e-3)
    den = rng.uniform(0.3, 1.3, N)
    ccn = rng.uniform(50e6, 300e6, N) / (den if not prog_ccn else 1.0)
    cpr = rng.uniform(1e-3, 5e-2, N)
    X = np.stack([ql, cond(rng, N), rng.uniform(230.0, 300.0, N), den, ccn, cpr, ql * rng.uniform(0.0, 1.2, N)], 1)
    cfg = _cfg(prog_ccn=prog_ccn)
    xbh, xbd, xbs, _ = run(harness, "autoconv_subgrid_var", X, rng.normal(size=(N, 2)), cfg=cfg)
    check(xbh, xbd, xbs, "autoconv_subgrid_var")
    xbh, xbd, xbs, _ = run(harness, "autoconv_no_subgrid_var", X[:, :6], rng.normal(size=(N, 2)), cfg=cfg)
    check(xbh, xbd, xbs, "autoconv_no_subgrid_var")


def test_collection_and_melt_kernels(harness):
    rng = np.random.default_rng(5)
    X = np.stack([rng.uniform(0.1, 10.0, N), rng.uniform(0.1, 10.0, N), cond(rng, N, 0.0), cond(rng, N, 0.0),
                  rng.uniform(0.3, 1.3, N), rng.uniform(1.0, 100.0, N), rng.uniform(0.1, 5.0, N),
                  rng.uniform(0.1, 5.0, N), rng.uniform(0.1, 5.0, N)], 1)
    xbh, xbd, xbs, _ = run(harness, "acr3d", X, rng.normal(size=(N, 1)))
    check(xbh, xbd, xbs, "acr3d")
    c = rng.uniform(0.1, 5.0, (N, 5))
    X = np.concatenate([np.stack([rng.uniform(-5.0, 10.0, N), rng.normal(0, 1e-3, N), cond(rng, N, 0.0),
                                  cond(rng, N, 0.0), cond(rng, N, 0.0), rng.uniform(0.3, 1.3, N),
                                  rng.uniform(0.8, 2.0, N)], 1), c], 1)
    xbh, xbd, xbs, _ = run(harness, "smlt", X, rng.normal(size=(N, 1)))
    check(xbh, xbd, xbs, "smlt")
    X = np.concatenate([X[:, :6], c], 1)
    xbh, xbd, xbs, _ = run(harness, "gmlt", X, rng.normal(size=(N, 1)))
    check(xbh, xbd, xbs, "gmlt")


def _rho_state(rng, n, tlo, thi):
    tz = rng.uniform(tlo, thi, n)
    den = rng.uniform(0.05, 1.4, n)
    rh = rng.uniform(0.1, 1.2, n)
    return tz, den, rh * qsat_w(tz, den)


@pytest.mark.parametrize("band", [(262.0, 292.0), (200.0, 262.0)])
def test_icloud_processes(harness, band):
    rng = np.random.default_rng(6)
    tz, den, qv = _rho_state(rng, N, *band)
    qg, qi, ql, qr, qs = (cond(rng, N, 0.1, 1e-9, 3e-3) for _ in range(5))
    q_liq, q_sol = ql + qr, qi + qs + qg
    cvm = 717.55 + qv * 1384.5 + q_liq * 4185.5 + q_sol * 1972.0
    p1 = den * 287.05 * tz
    p1[rng.random(N) < 0.02] = 50.0
    X = np.stack([qg, qi, ql, qr, qs, qv, tz, den, np.sqrt(1.2 / den), rng.uniform(0.1, 8.0, N),
                  rng.uniform(0.1, 8.0, N), rng.uniform(0.1, 2.0, N), p1, qi * rng.uniform(0.0, 1.0, N), q_liq, q_sol,
                  cvm], 1)
    YB = rng.normal(size=(N, 6)) * np.array([1, 1, 1, 1, 1, 1e-3])
    xbh, xbd, xbs, y = run(harness, "icloud_processes", X, YB)
    assert np.any(y != X[:, [0, 1, 2, 3, 4, 6]], axis=1).mean() > 0.3
    check(xbh, xbd, xbs, f"icloud_processes {band}")


@pytest.mark.parametrize("fast_sat_adj", [True, False])
@pytest.mark.parametrize("band", [(170.0, 240.0), (235.0, 275.0), (270.0, 310.0)])
def test_subgrid_z_proc(harness, band, fast_sat_adj):
    rng = np.random.default_rng(7)
    tz, den, qv = _rho_state(rng, N, *band)
    qg, qi, ql, qr, qs = (cond(rng, N, 0.15, 1e-9, 3e-3) for _ in range(5))
    p1 = den * 287.05 * tz
    h_var = rng.uniform(0.01, 0.2, N)
    rh_adj = 1.0 - h_var - 0.2
    X = np.stack([qg, qi, ql, qr, qs, qv, tz, den, np.sqrt(1.2 / den), p1, rng.uniform(0.0, 2.0, N), h_var, rh_adj,
                  np.maximum(0.35, rh_adj - 0.3)], 1)
    YB = rng.normal(size=(N, 8)) * np.array([1e-2, 1, 1, 1, 1, 1, 1, 1e-3])
    cfg = _cfg(fast_sat_adj=fast_sat_adj)
    xbh, xbd, xbs, y = run(harness, "subgrid_z_proc", X, YB, cfg=cfg)
    assert np.any(y[:, 1:] != X[:, [0, 1, 2, 3, 4, 5, 6]], axis=1).mean() > 0.3
    check(xbh, xbd, xbs, f"subgrid_z_proc {band} fast={fast_sat_adj}")


@pytest.mark.parametrize("band", [(262.0, 292.0), (220.0, 245.0)])
def test_step_blocks(harness, band):
    rng = np.random.default_rng(8)
    tz, den, qv = _rho_state(rng, N, *band)
    qg, qi, ql, qr, qs = (cond(rng, N, 0.15, 1e-9, 3e-3) for _ in range(5))
    X = np.stack([qv, ql, qr, qi, qs, qg, tz], 1)
    YB = rng.normal(size=(N, 7)) * np.array([1, 1, 1, 1, 1, 1, 1e-3])
    xbh, xbd, xbs, _ = run(harness, "sedi_ice_melt", X, YB)
    check(xbh, xbd, xbs, "sedi_ice_melt")
    YB10 = np.concatenate([YB, rng.normal(size=(N, 3)) * np.array([1, 1, 1e-6])], 1)
    xbh, xbd, xbs, y = run(harness, "icloud_melt_freeze", np.concatenate([X, den[:, None]], 1), YB10)
    check(xbh, xbd, xbs, "icloud_melt_freeze")
    # negative values for the fix_negative chain
    Xn = X.copy()
    for j in range(1, 6):
        neg = rng.random(N) < 0.3
        Xn[neg, j] = -rng.uniform(0, 1e-4, neg.sum())
    xbh, xbd, xbs, y = run(harness, "fix_negative_point", Xn, YB)
    assert (y[:, 1:6] == 0).any()
    check(xbh, xbd, xbs, "fix_negative_point")


# ---------------------------------------------------------------- the column
STATE_ROWS = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi", "delz",
              "wmp", "qaz")
OUT_ROWS = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt", "wmp", "qaz")
NXR, NYR = len(STATE_ROWS), len(OUT_ROWS)
SFC = ("rain", "snow", "ice", "graupel")


def column_ref(lib, cfg, ts, X, land, area, DX=None, YB=None):
    """Run the dual-number column step (tests/adjoint/column.h) on one column:
    X (14, L) input rows, DX a direction per row, YB the output cotangents
    (12 rows of L, then the 4 surface totals). Returns JD (16, 14): for
    output o and input row f, <ybar_o, J dx_f>; JS the size of its terms;
    Y the output values (laid out as YB)."""
    L = X.shape[1]
    X = np.ascontiguousarray(X, dtype=np.float64)
    DX = np.ascontiguousarray(np.zeros_like(X) if DX is None else DX, dtype=np.float64)
    YB = np.ascontiguousarray(np.zeros(NYR * L + 4) if YB is None else YB, dtype=np.float64)
    JD = np.zeros((NYR + 4, NXR))
    JS = np.zeros((NYR + 4, NXR))
    Y = np.zeros(NYR * L + 4)
    P = ctypes.POINTER(ctypes.c_double)
    f = lib.adj_column
    f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, P, P, P, P, P, P]
    p = lambda a: a.ctypes.data_as(P)  # noqa: E731
    assert f(ctypes.byref(cfg), ts, L, float(land), float(area), p(X), p(DX), p(YB), p(JD), p(JS), p(Y)) == 0
    return JD, JS, Y


@pytest.mark.parametrize("kw", [{}, {"mp_time": 75.0}, {"fix_negative": False, "z_slope_liq": False},
                                {"irain_f": 1, "prog_ccn": True, "do_qa": True},
                                {"do_sedi_w": False, "sedi_transport": False, "fast_sat_adj": False},
                                {"do_sedi_heat": True}])
def test_column_reference_matches_oracle(harness, kw):
    """The sequential column step that serves as the exact reference for the
    adjoint computes the oracle's step: every output within the plain-form
    tolerance of the GPU tests."""
    import sys

    sys.path.insert(0, HERE)
    from mp_helpers import TOL_PLAIN, floors

    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200._lib import make_config
    from pyshield_b200.inputs import copy_state, make_state

    n, L, dt = 6, 79, 150.0
    pc = PhysicsConfig(dt_atmos=int(dt), **kw)
    state, area = make_state(n, L, seed=21, n_cube=1, sat_fraction=0.2)
    s = copy_state(state)
    fl = None
    om = OracleMicrophysics(pc, n, L, area)
    state["qaz"] = np.zeros((L, n))
    pr = om(s, dt)
    s["qaz"] = om.qaz
    fl = floors(state, s, dt)
    for c in range(n):
        X = np.stack([state[r][:, c] for r in STATE_ROWS])
        _, _, Y = column_ref(harness, make_config(pc), dt, X, state["land"][c], area[c])
        for o, name in enumerate(OUT_ROWS):
            ref = s[name][:, c]
            got = Y[o * L:(o + 1) * L]
            allow = TOL_PLAIN * np.abs(s[name]).max() + fl.get(name, 0.0) + 1e-300
            assert np.abs(got - ref).max() <= allow, (name, c, np.abs(got - ref).max(), allow)
        for i, name in enumerate(SFC):
            allow = TOL_PLAIN * np.abs(pr[name]).max() + fl.get(name, 0.0) + 1e-300
            assert abs(Y[NYR * L + i] - pr[name][c]) <= allow, (name, c)


def column_window_ref(lib, cfg, ts, X, land, area, nsteps, DX, XB):
    """The dual-number window of ``nsteps`` steps (tests/adjoint/harness.cpp
    adj_column_window): JD, JS (14,) per input row, and the final state."""
    L = X.shape[1]
    X, DX, XB = (np.ascontiguousarray(a, dtype=np.float64) for a in (X, DX, XB))
    JD, JS, XF = np.zeros(NXR), np.zeros(NXR), np.zeros((NXR, L))
    P = ctypes.POINTER(ctypes.c_double)
    f = lib.adj_column_window
    f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                  P, P, P, P, P, P]
    p = lambda a: a.ctypes.data_as(P)  # noqa: E731
    assert f(ctypes.byref(cfg), ts, L, float(land), float(area), nsteps, p(X), p(DX), p(XB), p(JD), p(JS), p(XF)) == 0
    return JD, JS, XF
