"""GPU checks of the microphysics adjoint against finite differences.

For an input field x_f, an output field y_o, random cotangents ybar_o and a
random direction dx_f, per column c

    AD = <J_of^T ybar_o, dx_f>_c       (shield_mp_step_vjp, ybar only on y_o)
    FD = <ybar_o, dy_o / d(eps)>_c      (the CUDA forward step itself)

must agree to 1e-6 of the size of the terms of FD. Checking every pair
(input field, output field) separately keeps a small output's error from
hiding behind a large one.

FD is the Richardson extrapolation (4 D(eps/2) - D(eps)) / 3 of central
differences D at relative steps eps = 1e-4 and eps / 2: its truncation error
is O(eps^4) and its rounding error ~1e-12 of the outputs, where a single
central difference at 1e-6 would carry ~1e-10 (too much for outputs that
depend weakly on the perturbed field). The water species are perturbed
purely relatively, so a species that is zero stays zero (a negative
excursion would be clipped by fix_negative, a kink at the base point). A
column where a branch flips inside +-eps dx is not differentiable there: its
two central differences disagree, and it is skipped. Columns whose terms are
below 1e-9 of the largest column's carry only rounding and are not judged.
Cotangents are N(0, 1) divided by the output field's standard deviation.
"""
import pytest

pytestmark = pytest.mark.gpu

EPS = 1.0e-4
TOL = 1.0e-6
SMOOTH = 1.0e-3  # |D(eps) - D(eps/2)| allowed for a smooth column (curvature)
# relative perturbation floors per input field (added to |x|)
FLOOR = {"pt": 0.0, "qvapor": 0.0, "qliquid": 0.0, "qrain": 0.0, "qice": 0.0, "qsnow": 0.0, "qgraupel": 0.0,
         "qcld": 1e-2, "ua": 1.0, "va": 1.0, "delprsi": 0.0, "delz": 0.0, "wmp": 0.1}


def _setup(nx, ny, nz, dt, seed, **cfg):
    import torch

    from mp_helpers import device_state
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.adjoint import STATE
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import Microphysics

    state, area = make_state(nx * ny, nz, seed=seed, n_cube=nx, sat_fraction=0.1)
    ms, sf, qf, gd = device_state(state, area, nx, ny)
    mp = Microphysics(sf, qf, gd, PhysicsConfig(dt_atmos=int(dt), **cfg))
    x = [getattr(ms, n).view.clone() for n in STATE]
    land = ms.land.view.clone()
    zero_qaz = torch.zeros((nz, ny, nx), dtype=torch.float64, device="cuda")
    return mp, x, land, zero_qaz


def _f(mp, x, land, dt, zero_qaz):
    from pyshield_b200.adjoint import step_forward

    mp.set_qaz(zero_qaz)
    return step_forward(mp, x, land, dt)


def _col(t):
    return t.sum(2) if t.dim() == 3 else t


def check_adjoint(nx, ny, nz, dt, seed, fields=None, **cfg):
    """{(input, output): (smooth fraction, worst relative error)}"""
    import torch

    from pyshield_b200.adjoint import OUTPUTS, STATE, step_vjp

    mp, x, land, zq = _setup(nx, ny, nz, dt, seed, **cfg)
    y0 = _f(mp, x, land, dt, zq)
    g = torch.Generator(device="cuda").manual_seed(seed + 1)
    ybar = []
    for v in y0:
        sd = float(v.std())
        ybar.append(torch.randn(v.shape, generator=g, device="cuda", dtype=torch.float64) / (sd if sd > 0 else 1.0))
    xbar = []
    for o in range(len(OUTPUTS)):
        yb = [None] * len(OUTPUTS)
        yb[o] = ybar[o]
        xbar.append(step_vjp(mp, x, land, yb, dt))
    torch.cuda.synchronize()
    report = {}
    for fi, name in enumerate(STATE):
        if fields is not None and name not in fields:
            continue
        d = torch.randn(x[fi].shape, generator=g, device="cuda", dtype=torch.float64) * (x[fi].abs() + FLOOR[name])

        def central(eps):
            xp = [t.clone() for t in x]
            xm = [t.clone() for t in x]
            xp[fi] = x[fi] + eps * d
            xm[fi] = x[fi] - eps * d
            yp = _f(mp, xp, land, dt, zq)
            ym = _f(mp, xm, land, dt, zq)
            return [(a - b) / (2.0 * eps) for a, b in zip(yp, ym)]

        D1, D2 = central(EPS), central(EPS / 2.0)
        for o, oname in enumerate(OUTPUTS):
            t1 = ybar[o] * D1[o]
            fd1, fd2 = _col(t1), _col(ybar[o] * D2[o])
            scale = _col(t1.abs())
            if float(scale.max()) == 0.0:
                continue  # the output does not depend on this input
            judged = scale >= 1e-9 * float(scale.max())
            scale = scale + 1e-300
            smooth = ((fd1 - fd2).abs() <= SMOOTH * scale) & judged
            fd = (4.0 * fd2 - fd1) / 3.0
            ad = (xbar[o][fi] * d).sum(2)
            err = (ad - fd).abs() / scale
            n_j = float(judged.double().sum())
            frac = float(smooth.double().sum()) / max(n_j, 1.0)
            worst = float(err[smooth].max()) if smooth.any() else 0.0
            report[(name, oname)] = (frac, worst)
    return report


def _assert_report(report, min_smooth=0.5):
    bad = {k: v for k, v in report.items() if v[1] > TOL or v[0] < min_smooth}
    assert not bad, "adjoint vs finite differences, (input, output): (smooth fraction, worst rel. error): " + str(bad)


def test_adjoint_default_one_substep():
    _assert_report(check_adjoint(12, 12, 79, 150.0, 11))


def test_adjoint_two_substeps():
    _assert_report(check_adjoint(12, 8, 79, 225.0, 12, mp_time=150.0))


@pytest.mark.parametrize("cfg", [{"fix_negative": False, "z_slope_liq": False, "z_slope_ice": False},
                                 {"irain_f": 1, "prog_ccn": True, "do_qa": True},
                                 {"do_sedi_w": False, "sedi_transport": False, "fast_sat_adj": False}])
def test_adjoint_config_variants(cfg):
    _assert_report(check_adjoint(8, 8, 79, 150.0, 13, **cfg))


def test_adjoint_short_column():
    _assert_report(check_adjoint(8, 6, 31, 150.0, 14))


def test_autograd_function_matches_vjp():
    """torch.autograd through MicrophysicsStep gives step_vjp's adjoint."""
    import torch

    from pyshield_b200.adjoint import STATE, MicrophysicsStep, step_vjp

    mp, x, land, zq = _setup(8, 8, 79, 150.0, 15)
    xs = [t.clone().requires_grad_(True) for t in x]
    mp.set_qaz(zq)
    outs = MicrophysicsStep.apply(mp, 150.0, land, *xs)
    g = torch.Generator(device="cuda").manual_seed(3)
    ybar = [torch.randn(o.shape, generator=g, device="cuda", dtype=torch.float64) for o in outs]
    loss = sum((o * yb).sum() for o, yb in zip(outs, ybar))
    grads = torch.autograd.grad(loss, xs)
    ref = step_vjp(mp, x, land, ybar, 150.0)
    for name, a, b in zip(STATE, grads, ref):
        assert torch.equal(a, b), name
