"""GPU checks of the microphysics adjoint (shield_mp_step_vjp).

Primary check, exact: the same step written as a sequential column in C++
(tests/adjoint/column.h, whose values are pinned to the oracle by
tests/test_adjoint_pointwise.py) and run with dual numbers gives, for every
output y_o, input field x_f, cotangents ybar_o and direction dx_f,
<ybar_o, J dx_f> on the branches the input takes. The adjoint's
<J^T ybar_o, dx_f> must agree to 1e-9 of the size of the terms (from
magnitude duals). Pairs are checked separately, so that a small output's
error cannot hide behind a large one. The two evaluations round differently
(another summation order, another exp/log), so a branch decision that sits
within rounding of its threshold may go the other way in one of them: at most
0.5% of the (column, pair) entries may differ.

Secondary check, finite differences of the CUDA forward itself: central
differences at relative steps 1e-6, 5e-7 and 2.5e-7; their disagreement is
the rounding allowance. The step is piecewise smooth with min/max branches at
every level, so a column whose input lies closer to a branch point than the
step cannot be judged by differences (the two sides average); such columns
are a minority (at most 20% of a pair's judged columns, pairs with at least
10 of them), and the median error must still be below 1e-6.

Cotangents are N(0, 1) divided by each output field's standard deviation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXACT_TOL = 1.0e-9
EXACT_MAX_FAIL = 0.005
EPS = 1.0e-6
FD_TOL = 1.0e-6
FD_MAX_FAIL = 0.2
SMOOTH = 1.0e-3
# relative perturbation floors per input field (added to |x|); the water
# species are perturbed purely relatively, so a zero species stays zero (a
# negative excursion would be clipped by fix_negative)
FLOOR = {"pt": 0.0, "qvapor": 0.0, "qliquid": 0.0, "qrain": 0.0, "qice": 0.0, "qsnow": 0.0, "qgraupel": 0.0,
         "qcld": 1e-2, "ua": 1.0, "va": 1.0, "delprsi": 0.0, "delz": 0.0, "wmp": 0.1, "qaz": 0.1}


def _setup(nx, ny, nz, dt, seed, **cfg):
    import torch

    from mp_helpers import device_state
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.adjoint import STATE
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import Microphysics

    state, area = make_state(nx * ny, nz, seed=seed, n_cube=nx, sat_fraction=0.1)
    ms, sf, qf, gd = device_state(state, area, nx, ny)
    pc = PhysicsConfig(dt_atmos=int(dt), **cfg)
    mp = Microphysics(sf, qf, gd, pc)
    x = [getattr(ms, n).view.clone() for n in STATE[:-1]]
    g = torch.Generator(device="cuda").manual_seed(seed + 7)
    x.append(torch.rand((nx, ny, nz), generator=g, device="cuda", dtype=torch.float64) * 2.0)  # qaz
    land = ms.land.view.clone()
    area_h = gd.area.view.cpu().numpy()
    return mp, pc, x, land, area_h


def _cotangents(y, seed):
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    out = []
    for v in y:
        sd = float(v.std())
        out.append(torch.randn(v.shape, generator=g, device="cuda", dtype=torch.float64) / (sd if sd > 0 else 1.0))
    return out


def _per_output_vjps(mp, x, land, ybar, dt):
    from pyshield_b200.adjoint import OUTPUTS, step_vjp

    res = []
    for o in range(len(OUTPUTS)):
        yb = [None] * len(OUTPUTS)
        yb[o] = ybar[o]
        res.append([t.cpu().numpy() for t in step_vjp(mp, x, land, yb, dt)])
    return res


def exact_check(nx, ny, nz, dt, seed, **cfg):
    """(entries, failing entries, worst {(input, output): rel. error})"""
    from pyshield_b200._lib import make_config
    from pyshield_b200.adjoint import OUTPUTS, STATE, step_forward
    from test_adjoint_pointwise import build_harness, column_ref

    lib = build_harness()
    mp, pc, x, land, area = _setup(nx, ny, nz, dt, seed, **cfg)
    y0 = step_forward(mp, x, land, dt)
    ybar = _cotangents(y0, seed + 1)
    xbar = _per_output_vjps(mp, x, land, ybar, dt)
    X = np.stack([t.cpu().numpy() for t in x])
    YB = [t.cpu().numpy() for t in ybar]
    lnd = land.cpu().numpy()
    cfg_c = make_config(pc)
    floor = np.array([FLOOR[n] for n in STATE])[:, None]
    rng = np.random.default_rng(seed)
    n3 = len(OUTPUTS) - 4
    entries = fails = 0
    worst = {}
    for i in range(nx):
        for j in range(ny):
            Xc = X[:, i, j, :]
            DX = rng.normal(size=Xc.shape) * (np.abs(Xc) + floor)
            ybc = np.concatenate([np.stack([YB[o][i, j, :] for o in range(n3)]).ravel(),
                                  [YB[n3 + s][i, j] for s in range(4)]])
            JD, JS, _ = column_ref(lib, cfg_c, dt, Xc, lnd[i, j], area[i, j], DX, ybc)
            for o in range(len(OUTPUTS)):
                for f in range(len(STATE)):
                    if JS[o, f] == 0.0:
                        continue
                    entries += 1
                    ad = float((xbar[o][f][i, j, :] * DX[f]).sum())
                    e = abs(ad - JD[o, f]) / JS[o, f]
                    if e > EXACT_TOL:
                        fails += 1
                        key = (STATE[f], OUTPUTS[o])
                        worst[key] = max(worst.get(key, 0.0), e)
    return entries, fails, worst


def _assert_exact(res):
    entries, fails, worst = res
    assert entries > 0
    assert fails <= EXACT_MAX_FAIL * entries, (f"{fails} of {entries} (column, input, output) entries differ from "
                                               f"the exact column derivative; worst per pair: {worst}")


def test_exact_default_one_substep():
    _assert_exact(exact_check(12, 4, 79, 150.0, 11))


def test_exact_two_substeps():
    _assert_exact(exact_check(8, 4, 79, 225.0, 12, mp_time=150.0))


@pytest.mark.parametrize("cfg", [{"fix_negative": False, "z_slope_liq": False, "z_slope_ice": False},
                                 {"irain_f": 1, "prog_ccn": True, "do_qa": True},
                                 {"do_sedi_w": False, "sedi_transport": False, "fast_sat_adj": False},
                                 {"do_sedi_heat": True}])
def test_exact_config_variants(cfg):
    _assert_exact(exact_check(8, 3, 79, 150.0, 13, **cfg))


@pytest.mark.parametrize("nz", [31, 90, 127])
def test_exact_column_heights(nz):
    _assert_exact(exact_check(6, 3, nz, 150.0, 14))


@pytest.mark.parametrize("nx,ny,nz", [(5, 5, 127), (5, 3, 79)])
def test_exact_partly_filled_block(nx, ny, nz):
    """Column counts that are not a multiple of the columns per block (3 at
    L127, 4 at L79): the last block holds columns past the domain's end,
    which must neither be computed into the domain nor disturb the block's
    column exchanges."""
    _assert_exact(exact_check(nx, ny, nz, 150.0, 15))


def test_window_matches_exact_column():
    """A 3-step window through torch.autograd (MicrophysicsStep per step,
    the state update between steps, each step's inputs as its checkpoint)
    against the dual-number window of the same steps."""
    import torch

    from pyshield_b200._lib import make_config
    from pyshield_b200.adjoint import STATE, rollout
    from test_adjoint_pointwise import build_harness, column_window_ref

    lib = build_harness()
    nx, ny, nz, dt, nsteps = 6, 4, 79, 150.0, 3
    mp, pc, x, land, area = _setup(nx, ny, nz, dt, 16)
    xs = [t.clone().requires_grad_(True) for t in x]
    final, _ = rollout(mp, dict(zip(STATE, xs)), land, dt, nsteps)
    g = torch.Generator(device="cuda").manual_seed(4)
    xb = []
    for n in STATE:
        sd = float(final[n].detach().std())
        xb.append(torch.randn(final[n].shape, generator=g, device="cuda", dtype=torch.float64) / (sd if sd > 0 else 1.0))
    loss = sum((final[n] * b).sum() for n, b in zip(STATE, xb))
    grads = [t.cpu().numpy() for t in torch.autograd.grad(loss, xs)]
    X = np.stack([t.cpu().numpy() for t in x])
    XB = np.stack([b.cpu().numpy() for b in xb])
    lnd = land.cpu().numpy()
    floor = np.array([FLOOR[n] for n in STATE])[:, None]
    rng = np.random.default_rng(5)
    entries = fails = 0
    worst = {}
    for i in range(nx):
        for j in range(ny):
            Xc = X[:, i, j, :]
            DX = rng.normal(size=Xc.shape) * (np.abs(Xc) + floor)
            JD, JS, _ = column_window_ref(lib, make_config(pc), dt, Xc, lnd[i, j], area[i, j], nsteps, DX,
                                          XB[:, i, j, :])
            for f, name in enumerate(STATE):
                if JS[f] == 0.0:
                    continue
                entries += 1
                e = abs(float((grads[f][i, j, :] * DX[f]).sum()) - JD[f]) / JS[f]
                if e > EXACT_TOL:
                    fails += 1
                    worst[name] = max(worst.get(name, 0.0), e)
    assert fails <= EXACT_MAX_FAIL * entries + 1, f"{fails} of {entries} differ; worst per input: {worst}"


def test_finite_differences_default():
    """The adjoint against central differences of the CUDA forward step."""
    import torch

    from pyshield_b200.adjoint import OUTPUTS, STATE, step_forward

    nx, ny, nz, dt, seed = 12, 12, 79, 150.0, 17
    mp, pc, x, land, area = _setup(nx, ny, nz, dt, seed)
    y0 = step_forward(mp, x, land, dt)
    ybar = _cotangents(y0, seed + 1)
    xbar = _per_output_vjps(mp, x, land, ybar, dt)
    g = torch.Generator(device="cuda").manual_seed(seed + 2)
    bad = {}
    for fi, name in enumerate(STATE):
        d = torch.randn(x[fi].shape, generator=g, device="cuda", dtype=torch.float64) * (x[fi].abs() + FLOOR[name])

        def central(eps):
            xp = [t.clone() for t in x]
            xm = [t.clone() for t in x]
            xp[fi] = x[fi] + eps * d
            xm[fi] = x[fi] - eps * d
            return [(a - b) / (2.0 * eps) for a, b in zip(step_forward(mp, xp, land, dt), step_forward(mp, xm, land, dt))]

        D = [central(EPS), central(EPS / 2.0), central(EPS / 4.0)]
        dn = d.cpu().numpy()
        for o, oname in enumerate(OUTPUTS):
            yb = ybar[o]
            col = (lambda t: t.sum(2)) if yb.dim() == 3 else (lambda t: t)
            fd = [col(yb * Dk[o]).cpu().numpy() for Dk in D]
            scale = col((yb * D[2][o]).abs()).cpu().numpy()
            if scale.max() == 0.0:
                continue
            judged = scale >= 1e-9 * scale.max()
            noise = np.abs(fd[0] - fd[1]) + np.abs(fd[1] - fd[2])
            smooth = judged & (noise <= SMOOTH * scale)
            ad = (xbar[o][fi] * dn).sum(2)
            err = np.maximum(np.abs(ad - fd[2]) - 2.0 * noise, 0.0) / (scale + 1e-300)
            if smooth.sum() < 10:
                continue  # too few differentiable columns to judge the pair by differences
            fail = float((err[smooth] > FD_TOL).mean())
            med = float(np.median(err[smooth]))
            if fail > FD_MAX_FAIL or med > FD_TOL:
                bad[(name, oname)] = (fail, med)
    assert not bad, "adjoint vs finite differences, (input, output): (failing fraction, median error): " + str(bad)


def test_autograd_function_matches_vjp():
    """torch.autograd through MicrophysicsStep gives step_vjp's adjoint."""
    import torch

    from pyshield_b200.adjoint import STATE, MicrophysicsStep, step_vjp

    mp, pc, x, land, area = _setup(8, 8, 79, 150.0, 15)
    xs = [t.clone().requires_grad_(True) for t in x]
    outs = MicrophysicsStep.apply(mp, 150.0, land, *xs)
    g = torch.Generator(device="cuda").manual_seed(3)
    ybar = [torch.randn(o.shape, generator=g, device="cuda", dtype=torch.float64) for o in outs]
    loss = sum((o * yb).sum() for o, yb in zip(outs, ybar))
    grads = torch.autograd.grad(loss, xs)
    ref = step_vjp(mp, x, land, ybar, 150.0)
    for name, a, b in zip(STATE, grads, ref):
        assert torch.equal(a, b), name


def test_workspace_grows_with_the_substeps():
    """A handle's adjoint workspace, allocated for one sub-step by a first
    call, grows for a later call with three sub-steps: the result equals a
    fresh handle's, and a repeated call gives the same bits again."""
    import torch

    from pyshield_b200.adjoint import OUTPUTS, STATE, step_forward, step_vjp

    mp, pc, x, land, area = _setup(6, 4, 79, 150.0, 21, mp_time=150.0)
    y = step_forward(mp, x, land, 150.0)
    ybar = _cotangents(y, 22)
    step_vjp(mp, x, land, ybar, 150.0)  # one sub-step: the first workspace
    y3 = step_forward(mp, x, land, 450.0)
    ybar3 = _cotangents(y3, 23)
    got = step_vjp(mp, x, land, ybar3, 450.0)  # three sub-steps on the same handle
    again = step_vjp(mp, x, land, ybar3, 450.0)
    fresh_mp = _setup(6, 4, 79, 450.0, 21, mp_time=150.0)[0]
    ref = step_vjp(fresh_mp, x, land, ybar3, 450.0)
    assert len(got) == len(STATE) and len(ybar3) == len(OUTPUTS)
    for name, a, b, c in zip(STATE, got, again, ref):
        assert torch.equal(a, c), name
        assert torch.equal(a, b), name


def test_de_ice_composes_with_the_step():
    """de_ice (microphysics.py:110-120) with incoming qi_dt: the adjoint equals
    the adjoint of the step without de_ice taken at the de-iced state, chained
    with de_ice's own derivative. Where qi becomes qi0_max, the input qi
    reaches the outputs through qs (qs + qi - qi0_max) and through the
    tendencies de_ice sets (qi_dt = dqi, qs_dt += qi_dt - dqi with
    dqi = (qi0_max - qi + dt qi_dt) / dt); elsewhere qi and qs pass through.
    With zero incoming tendencies de_ice changes nothing."""
    import torch

    from pyshield_b200.adjoint import OUTPUTS, STATE, step_forward, step_vjp

    dt = 150.0
    mp, pc, x, land, area = _setup(6, 4, 79, dt, 23, de_ice=True)
    iqi, iqs = STATE.index("qice"), STATE.index("qsnow")
    qi = x[iqi]
    g = torch.Generator(device="cuda").manual_seed(5)
    # half the points with ice above qi0_max lose it to the floor, a quarter
    # keep qi - dt qi_dt, the rest get no tendency
    u = torch.rand(qi.shape, generator=g, device="cuda", dtype=torch.float64)
    qi_dt = torch.where(u < 0.5, (qi + 1e-4) / dt, torch.where(u < 0.75, 0.2 * qi / dt, torch.zeros_like(qi)))
    x[iqi] = torch.where(qi > pc.qi0_max, qi, qi + 2.0 * pc.qi0_max)  # plenty of points above the threshold
    qi = x[iqi]
    tend = {"qi_dt": qi_dt}
    y = step_forward(mp, x, land, dt, tendencies=tend)
    ybar = _cotangents(y, 31)
    got = step_vjp(mp, x, land, ybar, dt, tendencies=tend)
    # the step without de_ice at the de-iced state
    qio = qi - dt * qi_dt
    qin = torch.maximum(qio, torch.full_like(qio, pc.qi0_max))
    hit = qi > qin
    floor = hit & ~(qio >= pc.qi0_max)
    assert int(floor.sum()) > 100 and int((hit & ~floor).sum()) > 100
    xd = [t.clone() for t in x]
    xd[iqs] = torch.where(hit, x[iqs] + qi - qin, x[iqs])
    xd[iqi] = torch.where(hit, qin, qi)
    mp0 = _setup(6, 4, 79, dt, 23)[0]  # the same domain without de_ice
    ref = list(step_vjp(mp0, xd, land, ybar, dt))
    c_qi, c_qs = ybar[OUTPUTS.index("qi_dt")], ybar[OUTPUTS.index("qs_dt")]
    ref[iqi] = torch.where(floor, ref[iqs] + (c_qs - c_qi) / dt, ref[iqi])
    for name, a, b in zip(STATE, got, ref):
        scale = float(b.abs().max()) or 1.0
        assert float((a - b).abs().max()) <= 1e-12 * scale, name
    # zero incoming tendencies: de_ice leaves the step alone
    plain = step_vjp(mp0, x, land, ybar, dt)
    for name, a, b in zip(STATE, step_vjp(mp, x, land, ybar, dt), plain):
        assert torch.equal(a, b), name


def test_exact_five_substeps():
    # dt = 750 s with mp_time = 150 s: five sub-steps, whose records the
    # workspace holds like any other count
    _assert_exact(exact_check(6, 4, 79, 750.0, 19, mp_time=150.0))
