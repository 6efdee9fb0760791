"""The GPU adjoint against torch.autograd on the FP64 torch transcription, C12.

tests/torch_oracle.py runs the oracle's step on torch FP64 tensors. That
step is pinned to the reference's own source, and the transcription matches
the numpy oracle (test_torch_oracle.py). Forward-mode torch.autograd
differentiates it along one random direction DX_f per input field f; the
GPU's vector-Jacobian products, one per output o, must satisfy

    <ybar_o, J_of DX_f> = <J_of^T ybar_o, DX_f>

per column, for every (output, input) pair, to 1e-9 of the size of the
terms. The term size comes from the magnitude duals of the dual-number
column reference (tests/adjoint/column.h). The two sides round differently,
so a branch decision within rounding of its threshold may go either way: at
most 0.5 % of the (column, pair) entries may differ. A surface total below
the oracle's resolution is skipped (see test_torch_oracle.SURFACE_RES).

C12 is 6 x 12 x 12 = 864 columns, laid out as nx = 12, ny = 72 (the six
tiles side by side), 79 levels, dt 150 s.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1.0e-9
MAX_FAIL = 0.005


@pytest.mark.parametrize("kw,dt", [({}, 150.0), ({"mp_time": 150.0}, 225.0)])
def test_vjp_matches_torch_autograd_c12(kw, dt):
    from pyshield_b200._lib import make_config
    from pyshield_b200.adjoint import OUTPUTS, STATE, step_forward
    from test_adjoint_gpu import FLOOR, _cotangents, _per_output_vjps, _setup
    from test_adjoint_pointwise import build_harness, column_ref
    from test_torch_oracle import SURFACE_RES, precip_columns
    from torch_oracle import jvp_per_input

    nx, ny, nz = 12, 72, 79
    n = nx * ny
    mp, pc, x, land, area = _setup(nx, ny, nz, dt, 31, **kw)
    y0 = step_forward(mp, x, land, dt)
    ybar = _cotangents(y0, 32)
    xbar = _per_output_vjps(mp, x, land, ybar, dt)  # [o][f] (nx, ny, nz)

    # oracle layout: (L, n), column c = j * nx + i
    X = np.stack([t.permute(2, 1, 0).reshape(nz, n).cpu().numpy() for t in x])
    lnd = land.t().reshape(n).cpu().numpy()
    ar = area.T.reshape(n)
    rng = np.random.default_rng(33)
    floor = np.array([FLOOR[f] for f in STATE])[:, None, None]
    DX = rng.normal(size=X.shape) * (np.abs(X) + floor)
    _, T = jvp_per_input(pc, dt, X, lnd, ar, DX)

    lib = build_harness()
    cfg_c = make_config(pc)
    n3 = len(OUTPUTS) - 4
    YB = [t.permute(2, 1, 0).reshape(nz, n).cpu().numpy() if t.dim() == 3 else t.t().reshape(n).cpu().numpy()
          for t in ybar]
    XB = [[g.transpose(2, 1, 0).reshape(nz, n) for g in per_o] for per_o in xbar]
    pscale = precip_columns({f: X[i] for i, f in enumerate(STATE[:-1])}, dt)
    entries = fails = skipped = 0
    worst = {}
    for c in range(n):
        ybc = np.concatenate([np.stack([YB[o][:, c] for o in range(n3)]).ravel(), [YB[n3 + s][c] for s in range(4)]])
        _, JS, Yc = column_ref(lib, cfg_c, dt, X[:, :, c], lnd[c], ar[c], DX[:, :, c], ybc)
        for o in range(len(OUTPUTS)):
            if o >= n3 and abs(Yc[n3 * nz + (o - n3)]) <= SURFACE_RES * pscale[c]:
                skipped += 1
                continue
            for f in range(len(STATE)):
                if JS[o, f] == 0.0:
                    continue
                entries += 1
                torch_ad = float(np.sum(YB[o][..., c] * T[OUTPUTS[o]][f][..., c]))
                gpu_ad = float(np.sum(XB[o][f][:, c] * DX[f][:, c]))
                e = abs(torch_ad - gpu_ad) / JS[o, f]
                if e > TOL:
                    fails += 1
                    key = (STATE[f], OUTPUTS[o])
                    worst[key] = max(worst.get(key, 0.0), e)
    assert entries > 10000
    assert fails <= MAX_FAIL * entries, f"{fails} of {entries} entries (skipped {skipped}); worst per pair: {worst}"
