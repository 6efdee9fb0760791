"""The adjoint at C48 (6 x 48 x 48 = 13,824 columns x L79, FP64, dt 150 s)
against central finite differences of the CUDA forward, one step and an
8-step window with per-step checkpointing.

Columns and levels. Central differences of a piecewise-smooth step only
measure its derivative where no branch point lies within the step. The test
therefore draws 1,000 random columns of the domain and perturbs, in each, only
the levels whose input state lies more than 5 % (relative) from every
threshold the scheme compares it with: T from tice and t_wfr, the vapour
from saturation over water and over ice, each species from QRMIN (and cloud
water and ice from QCMIN), cloud ice from qi0_crt / den and the ice
generation limit qi_crt, snow from qs0_crt / den, cloud water from ql_mlt and
qs_mlt. Other levels keep a zero perturbation. Columns are independent, so
every column's difference quotient is its own.

Judging. Per (column, input field, output) entry the adjoint's
<xbar_o,f, dx_f> is compared with the central difference
<ybar_o, (y(x + eps dx) - y(x - eps dx)) / 2 eps> at eps = 1e-6 (relative),
in units of the size of the difference's terms sum |ybar_o dy_o|, after
subtracting twice the quotient's rounding noise (how much the quotients at
eps, eps/2 and eps/4 differ: the forward's last-place rounding divided by
eps). An entry is judged when those quotients agree to 1e-3 of that size: entries whose neighbourhood still holds a branch point of an
intermediate quantity (a min/max of two rates, a saturation test after the
first process) do not, and there a difference is not a derivative.
Cotangents are N(0, 1) divided by each output field's standard deviation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_CUBE, NZ, DT = 48, 79, 150.0
NCOLS = 1000
EPS = 1.0e-6
FD_TOL = 1.0e-6
SMOOTH = 1.0e-3
FLOOR = {"pt": 0.0, "qvapor": 0.0, "qliquid": 0.0, "qrain": 0.0, "qice": 0.0, "qsnow": 0.0, "qgraupel": 0.0,
         "qcld": 1e-2, "ua": 1.0, "va": 1.0, "delprsi": 0.0, "delz": 0.0, "wmp": 0.1, "qaz": 0.1}
MARGIN = 0.05


def _far(x, thr):
    """|x / thr - 1| > MARGIN (thr may be an array)."""
    return np.abs(x / thr - 1.0) > MARGIN


def safe_levels(st, cfg):
    """(L, n) mask of levels whose input state is more than 5 % from every
    threshold the step compares it with (see the module docstring)."""
    from oracle.microphysics import QCMIN, QRMIN, iqs1, wqs1
    from pyshield_b200 import constants as C

    T, qv, ql, qr = st["pt"], st["qvapor"], st["qliquid"], st["qrain"]
    qi, qs, qg = st["qice"], st["qsnow"], st["qgraupel"]
    dp1 = st["delprsi"] * (1.0 - qv)
    den = -dp1 / (C.GRAV * st["delz"])
    tice, t_wfr = cfg.tice, cfg.tice - 40.0
    ok = _far(T, tice) & _far(T, t_wfr)
    with np.errstate(all="ignore"):
        ok &= _far(qv, wqs1(T, den)) & _far(qv, iqs1(T, den))
        for q in (qr, qi, qs, qg):
            ok &= (q == 0.0) | _far(q, QRMIN)
        for q in (ql, qi):
            ok &= (q == 0.0) | _far(q, QCMIN)
        ok &= (qi == 0.0) | _far(qi * den, cfg.qi0_crt)
        qi_crt = cfg.qi_gen * np.minimum(cfg.qi_lim, 0.1 * (tice - T)) / den
        ok &= (qi == 0.0) | (T >= tice) | _far(qi, qi_crt)
        ok &= (qs == 0.0) | _far(qs * den, cfg.qs0_crt)
        ok &= (ql == 0.0) | (_far(ql, cfg.ql_mlt) & _far(ql, cfg.qs_mlt))
    return ok


def _setup(seed):
    import torch

    from mp_helpers import device_state
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.adjoint import STATE
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import Microphysics

    nx, ny = N_CUBE, 6 * N_CUBE
    n = nx * ny
    state, area = make_state(n, NZ, seed=seed, n_cube=N_CUBE)
    ms, sf, qf, gd = device_state(state, area, nx, ny)
    cfg = PhysicsConfig(dt_atmos=int(DT))
    mp = Microphysics(sf, qf, gd, cfg)
    x = [getattr(ms, f).view.clone() for f in STATE[:-1]]
    g = torch.Generator(device="cuda").manual_seed(seed + 7)
    x.append(torch.rand((nx, ny, NZ), generator=g, device="cuda", dtype=torch.float64) * 2.0)  # qaz
    land = ms.land.view.clone()
    # the 1,000 columns and their perturbed levels
    rng = np.random.default_rng(seed)
    ok = safe_levels(state, cfg)  # (L, n), column c = j nx + i
    cols = rng.choice(n, NCOLS, replace=False)
    mask = np.zeros((NZ, n), dtype=bool)
    mask[:, cols] = ok[:, cols]
    # (L, n) -> (nx, ny, L)
    mask3 = torch.from_numpy(mask.reshape(NZ, ny, nx).transpose(2, 1, 0).copy()).cuda()
    dx = []
    for f, name in enumerate(STATE):
        d = torch.randn(x[f].shape, generator=g, device="cuda", dtype=torch.float64) * (x[f].abs() + FLOOR[name])
        dx.append(torch.where(mask3, d, torch.zeros_like(d)))
    ci, cj = cols % nx, cols // nx
    return mp, cfg, x, land, dx, (ci, cj), state, area, mask


def _judge(ad, fds, scale):
    """Entries (per column) of one pair: the error at EPS beyond the
    difference quotient's own rounding (estimated by how much the quotients
    at EPS, EPS/2 and EPS/4 differ), the raw error, and the judged mask."""
    noise = np.abs(fds[0] - fds[1]) + np.abs(fds[1] - fds[2])
    judged = (scale > 0.0) & (noise <= SMOOTH * scale)
    sc = np.where(scale > 0.0, scale, 1.0)
    raw = np.abs(ad - fds[0]) / sc
    err = np.maximum(np.abs(ad - fds[0]) - 2.0 * noise, 0.0) / sc
    return err, raw, judged


def test_one_step_finite_differences_c48():
    import torch

    from pyshield_b200.adjoint import OUTPUTS, STATE, step_forward, step_vjp

    mp, cfg, x, land, dx, (ci, cj), state, _, mask = _setup(41)
    assert mask.any(axis=0).sum() >= 0.9 * NCOLS, "too few perturbable columns"
    y0 = step_forward(mp, x, land, DT)
    g = torch.Generator(device="cuda").manual_seed(43)
    ybar = []
    for v in y0:
        sd = float(v.std())
        ybar.append(torch.randn(v.shape, generator=g, device="cuda", dtype=torch.float64) / (sd if sd > 0 else 1.0))
    # one VJP per output, so that every (input, output) pair is judged alone
    xbar = []
    for o in range(len(OUTPUTS)):
        yb = [None] * len(OUTPUTS)
        yb[o] = ybar[o]
        xbar.append(step_vjp(mp, x, land, yb, DT))
    total = judged_n = good = raw_good = 0
    per_pair = {}
    for f, name in enumerate(STATE):
        def central(eps):
            xp = [t.clone() for t in x]
            xm = [t.clone() for t in x]
            xp[f] = x[f] + eps * dx[f]
            xm[f] = x[f] - eps * dx[f]
            return [(a - b) / (2.0 * eps) for a, b in zip(step_forward(mp, xp, land, DT),
                                                          step_forward(mp, xm, land, DT))]

        D = [central(EPS), central(EPS / 2.0), central(EPS / 4.0)]
        for o, oname in enumerate(OUTPUTS):
            yb = ybar[o]
            red = (lambda t: t.sum(2)) if yb.dim() == 3 else (lambda t: t)
            fds = [red(yb * Dk[o]).cpu().numpy()[ci, cj] for Dk in D]
            scale = red((yb * D[0][o]).abs()).cpu().numpy()[ci, cj]
            ad = (xbar[o][f] * dx[f]).sum(2).cpu().numpy()[ci, cj]
            if not np.any(scale > 0.0):
                continue
            err, raw, judged = _judge(ad, fds, scale)
            total += int((scale > 0).sum())
            judged_n += int(judged.sum())
            good += int((err[judged] <= FD_TOL).sum())
            raw_good += int((raw[judged] <= FD_TOL).sum())
            if judged.sum():
                per_pair[(name, oname)] = (float(np.median(err[judged])), float((err[judged] <= FD_TOL).mean()),
                                           int(judged.sum()))
    frac = good / judged_n
    worst = sorted(per_pair.items(), key=lambda kv: kv[1][1])[:5]
    print(f"\nC48 one step, {NCOLS} columns: {judged_n} of {total} (column, input, output) entries judged, "
          f"{frac:.4%} within {FD_TOL:g} beyond the quotients' rounding ({raw_good / judged_n:.4%} without "
          f"subtracting it); lowest pairs (median, within, judged): {worst}")
    assert judged_n >= 0.8 * total, "too few entries away from branch points"
    assert frac >= 0.99, f"only {frac:.4%} of judged entries agree to {FD_TOL:g}"
    bad = {k: v for k, v in per_pair.items() if v[0] > FD_TOL}
    assert not bad, f"pairs whose median error exceeds {FD_TOL:g}: {bad}"


def test_eight_step_window_c48():
    """The 8-step window through torch.autograd (per-step checkpointing)
    against central differences of the 8-step rollout, per column, and on 24
    of the columns against the dual-number window (exact derivative)."""
    import torch

    from pyshield_b200._lib import make_config
    from pyshield_b200.adjoint import STATE, rollout
    from test_adjoint_pointwise import build_harness, column_window_ref

    nsteps = 8
    mp, cfg, x, land, dx, (ci, cj), state, area, mask = _setup(51)
    xs = [t.clone().requires_grad_(True) for t in x]
    final, _ = rollout(mp, dict(zip(STATE, xs)), land, DT, nsteps)
    g = torch.Generator(device="cuda").manual_seed(52)
    xb = []
    for name in STATE:
        sd = float(final[name].detach().std())
        xb.append(torch.randn(final[name].shape, generator=g, device="cuda", dtype=torch.float64) / (sd if sd > 0 else 1.0))
    loss = sum((final[n] * b).sum() for n, b in zip(STATE, xb))
    grads = torch.autograd.grad(loss, xs)
    ad = sum((gr * d).sum(2) for gr, d in zip(grads, dx)).cpu().numpy()[ci, cj]

    def central(eps):
        with torch.no_grad():
            fp, _ = rollout(mp, dict(zip(STATE, [t + eps * d for t, d in zip(x, dx)])), land, DT, nsteps)
            fm, _ = rollout(mp, dict(zip(STATE, [t - eps * d for t, d in zip(x, dx)])), land, DT, nsteps)
            terms = [b * (fp[n] - fm[n]) / (2.0 * eps) for n, b in zip(STATE, xb)]
            return sum(t.sum(2) for t in terms), sum(t.abs().sum(2) for t in terms)

    fds, scales = zip(*[central(e) for e in (EPS, EPS / 2.0, EPS / 4.0)])
    fds = [t.cpu().numpy()[ci, cj] for t in fds]
    scale = scales[0].cpu().numpy()[ci, cj]
    err, raw, judged = _judge(ad, fds, scale)
    frac = float((err[judged] <= FD_TOL).mean())
    print(f"\nC48 8-step window, {NCOLS} columns: {int(judged.sum())} judged, {frac:.4%} within {FD_TOL:g}, "
          f"median {np.median(err[judged]):.2e}")
    assert judged.sum() >= 0.7 * NCOLS
    assert frac >= 0.98 and np.median(err[judged]) <= FD_TOL

    # exact: the dual-number window on 24 of the columns
    lib = build_harness()
    X = np.stack([t.cpu().numpy() for t in x])
    XB = np.stack([b.cpu().numpy() for b in xb])
    DX = np.stack([d.cpu().numpy() for d in dx])
    G = np.stack([t.cpu().numpy() for t in grads])
    lnd = land.cpu().numpy()
    area2 = area.reshape(6 * N_CUBE, N_CUBE).T
    fails = 0
    for i, j in list(zip(ci, cj))[:24]:
        JD, JS, _ = column_window_ref(lib, make_config(cfg), DT, X[:, i, j, :], lnd[i, j], area2[i, j], nsteps,
                                      DX[:, i, j, :], XB[:, i, j, :])
        for f in range(len(STATE)):
            if JS[f] == 0.0:
                continue
            if abs(float((G[f, i, j, :] * DX[f, i, j, :]).sum()) - JD[f]) > 1e-9 * JS[f]:
                fails += 1
    assert fails <= 2, f"{fails} (column, input) entries of the window differ from the exact derivative"
