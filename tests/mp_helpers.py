"""Helpers shared by the GPU parity tests: build reference-layout states on the
device, run the CUDA step through the public API, compare with the oracle."""
import numpy as np

from golden_io import MP_TENDENCIES, PRECIP

# per-field relative tolerance of the plain FP64 form against the FP64
# oracle: max |gpu - oracle| / max |oracle| over the field
TOL_PLAIN = 1.0e-12


def to_storage_np(arr_ln, nx, ny, h=3):
    L = arr_ln.shape[0]
    out = np.zeros((nx + 2 * h + 1, ny + 2 * h + 1, L + 1))
    out[h : h + nx, h : h + ny, :L] = arr_ln.reshape(L, ny, nx).transpose(2, 1, 0)
    return out


def from_storage_np(st, nx, ny, L, h=3):
    return st[h : h + nx, h : h + ny, :L].transpose(2, 1, 0).reshape(L, nx * ny).copy()


def device_quantity(arr_ln, nx, ny, layout, h=3):
    """NDSL-style storage on the GPU holding (L, n) data in the compute domain.
    layout 'ifirst' (GT4Py GPU order) or 'kfirst' (C-order numpy storage)."""
    import torch

    from pyshield_b200.quantity import Quantity

    L = arr_ln.shape[0]
    st = to_storage_np(arr_ln, nx, ny, h)
    if layout == "ifirst":
        t = torch.from_numpy(np.ascontiguousarray(st.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
    else:
        t = torch.from_numpy(np.ascontiguousarray(st)).cuda()
    return Quantity(t, ("x", "y", "z"), "", (h, h, 0), (nx, ny, L))


def device_quantity2d(arr_n, nx, ny, h=3):
    import torch

    from pyshield_b200.quantity import Quantity

    st = np.zeros((nx + 2 * h + 1, ny + 2 * h + 1))
    st[h : h + nx, h : h + ny] = arr_n.reshape(ny, nx).T
    return Quantity(torch.from_numpy(st).cuda(), ("x", "y"), "", (h, h), (nx, ny))


def device_state(state, area, nx, ny, layout="ifirst"):
    """MicrophysicsState with NDSL-layout device storages holding ``state``;
    returns (state, stencil_factory, quantity_factory, grid_data)."""
    from pyshield_b200.grid import GridData, GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.microphysics import MicrophysicsState

    L = state["pt"].shape[0]
    gi = GridIndexing(nx, ny, L)
    qf = QuantityFactory(gi)
    q = {k: device_quantity(v, nx, ny, layout) for k, v in state.items() if k != "land"}
    land = device_quantity2d(state["land"], nx, ny)
    ms = MicrophysicsState(
        q["pt"], q["qvapor"], q["qliquid"], q["qrain"], q["qice"], q["qsnow"], q["qgraupel"], q["qcld"], q["ua"],
        q["va"], qf.zeros(["x", "y", "z"], ""), q["delz"], qf.zeros(["x", "y", "z"], ""), q["delprsi"], q["wmp"],
        qf.zeros(["x", "y", "z"], ""), qf.zeros(["x", "y", "z"], ""), land,
    )
    for t in MP_TENDENCIES:
        setattr(ms, t, q[t])
    return ms, StencilFactory(gi), qf, GridData(device_quantity2d(area, nx, ny))


def read_state(ms, nx, ny, L, layout="ifirst"):
    o = {}
    for t in MP_TENDENCIES + ("wmp", "qice", "qsnow"):
        data = getattr(ms, t).data
        if layout == "ifirst":
            arr = data.permute(2, 1, 0).contiguous().cpu().numpy().transpose(2, 1, 0)
        else:
            arr = data.cpu().numpy()
        o[t] = from_storage_np(arr, nx, ny, L)
    return o


def run_gpu(cfg, state, area, nx, ny, dt, nsteps=1, layout="ifirst", precision="plain", qaz0=None):
    """Run the CUDA step ``nsteps`` times; return per-step outputs as (L, n)
    numpy arrays (tendencies, wmp, qice, qsnow, qaz) and (n,) precip."""
    import torch

    from pyshield_b200.grid import GridData, GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.microphysics import Microphysics, MicrophysicsState

    L = state["pt"].shape[0]
    gi = GridIndexing(nx, ny, L)
    sf = StencilFactory(gi)
    qf = QuantityFactory(gi)
    q = {k: device_quantity(v, nx, ny, layout) for k, v in state.items() if k != "land"}
    land = device_quantity2d(state["land"], nx, ny)
    tend = qf.zeros(["x", "y", "z"], "")
    ms = MicrophysicsState(
        q["pt"], q["qvapor"], q["qliquid"], q["qrain"], q["qice"], q["qsnow"], q["qgraupel"], q["qcld"], q["ua"],
        q["va"], qf.zeros(["x", "y", "z"], ""), q["delz"], qf.zeros(["x", "y", "z"], ""), q["delprsi"], q["wmp"],
        qf.zeros(["x", "y", "z"], ""), tend, land,
    )
    for t in MP_TENDENCIES:
        setattr(ms, t, q[t])
    mp = Microphysics(sf, qf, GridData(device_quantity2d(area, nx, ny)), cfg, precision=precision)
    if qaz0 is not None:
        mp.set_qaz(torch.from_numpy(qaz0).cuda())
    outs = []
    for _ in range(nsteps):
        mp(ms, dt)
        torch.cuda.synchronize()
        o = {}
        for t in MP_TENDENCIES + ("wmp", "qice", "qsnow"):
            data = getattr(ms, t).data
            if layout == "ifirst":
                arr = data.permute(2, 1, 0).contiguous().cpu().numpy().transpose(2, 1, 0)
            else:
                arr = data.cpu().numpy()
            o[t] = from_storage_np(arr, nx, ny, L)
        for p in PRECIP:
            o[p] = getattr(mp, p).t().contiguous().cpu().numpy().reshape(-1)
        o["qaz"] = mp.get_qaz().cpu().numpy().reshape(L, -1)
        outs.append(o)
    return outs


def rel_err(a, b):
    """Per-field relative error: max |a - b| / max |b| (0 when both vanish)."""
    scale = float(np.max(np.abs(b)))
    d = float(np.max(np.abs(a - b)))
    if scale == 0.0:
        return d
    return d / scale


def precip_scale(state, dt):
    """Surface precipitation [mm/day] that the step's whole column condensate
    would make: the scale of the terms the reference sums to get the surface
    flux. The reference's running flux sum cancels to its last digits when
    little mass reaches the ground, so precipitation totals are compared
    relative to this scale (and to their own magnitude, whichever is larger)."""
    from pyshield_b200 import constants as C

    cond = sum(state[f] for f in ("qliquid", "qrain", "qice", "qsnow", "qgraupel"))
    col = np.sum(np.abs(cond) * state["delprsi"], axis=0)
    return float(np.max(col)) * 86400.0 / (dt * C.GRAV)


def rel_err_scaled(a, b, floor):
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b))) / scale if scale > 0 else float(np.max(np.abs(a - b)))


# Round-off floor of a tendency: X_dt = (X_new - X_old) / dt cannot be
# reproduced more closely than the round-off of X itself, whatever the size
# of X_dt, so each tendency may also differ by NOISE * max|X| / dt
# (about 45 ulps of the state it changes).
NOISE = 1.0e-14
TENDENCY_STATE = {
    "pt_dt": "pt", "qv_dt": "qvapor", "ql_dt": "qliquid", "qr_dt": "qrain", "qi_dt": "qice", "qs_dt": "qsnow",
    "qg_dt": "qgraupel", "qa_dt": "qcld", "udt": "ua", "vdt": "va",
}


def floors(state, ref, dt):
    """Absolute slack per field: the tendency round-off floor above, and for
    the precipitation totals the column-condensate scale of precip_scale."""
    fl = {}
    for f, x in TENDENCY_STATE.items():
        if f in ref:
            xin = state[x]
            xout = xin + ref[f] * dt
            fl[f] = NOISE * max(float(np.max(np.abs(xin))), float(np.max(np.abs(xout)))) / dt
    ps = precip_scale(state, dt)
    for p in PRECIP:
        fl[p] = TOL_PLAIN * ps
    return fl


# Tendencies that the GPU gate lets exceed the plain 1e-12 relative bound by
# the round-off floor above, each with its reason. Every other field of the
# plain form is held to max |gpu - oracle| <= 1e-12 max |oracle|.
TENDENCY_FLOOR = {
    # (u1 - u0) / dt of winds of order 10 m/s that the falling mass changes
    # by about a thousandth: the momentum recurrence u1_k = (dp0 u0_k +
    # m1_{k-1} u1_{k-1}) / (dp0 + m1_{k-1}) is evaluated as a parallel scan,
    # whose rounding of u1 (1e-15 of u) is 1e-12 of the difference
    "udt": "momentum transport: round-off of u1 against a small u1 - u0",
    "vdt": "momentum transport: round-off of v1 against a small v1 - v0",
}


def gpu_floors(state, ref, dt):
    """Absolute slack of the GPU-against-oracle gate: none for the
    tendencies, wmp and the accumulator (except the fields named in
    TENDENCY_FLOOR); the column-condensate scale for the four surface totals,
    which the reference sums as a running difference that cancels to its last
    digits when little mass reaches the ground (the kernels use the
    telescoped flux)."""
    full = floors(state, ref, dt)
    return {f: v for f, v in full.items() if f in PRECIP or f in TENDENCY_FLOOR}


def field_errors(gpu, ref, fields, tol, fl=None):
    """Per-field error in units of the allowance: max |gpu - ref| divided by
    (tol * max|ref| + floor); a value <= 1 passes. Also the plain relative
    error max |gpu - ref| / max |ref| for reporting."""
    fl = fl or {}
    out = {}
    for f in fields:
        d = float(np.max(np.abs(gpu[f] - ref[f])))
        allow = tol * float(np.max(np.abs(ref[f]))) + fl.get(f, 0.0)
        if not np.all(np.isfinite(gpu[f])) and np.all(np.isfinite(ref[f])):
            out[f] = (float("inf"), float("inf"))
        else:
            out[f] = (d / allow if allow > 0 else (0.0 if d == 0 else float("inf")), rel_err(gpu[f], ref[f]))
    return out


def assert_close(gpu, ref, fields, tol, ctx="", fl=None):
    errs = field_errors(gpu, ref, fields, tol, fl)
    bad = [f"{f}: {e[0]:.2f}x allowance (plain relative {e[1]:.2e})" for f, e in errs.items() if e[0] > 1.0]
    assert not bad, f"{ctx} error above tolerance {tol:g}: " + ", ".join(bad)
