"""``Physics.__call__`` on the GPU: the fused driver pre-step kernel
(statein, get_prs_fv3, get_phi_fv3, prepare_microphysics), the microphysics
step and the state update, against the reference's own result (golden
fixtures, equal bit for bit to the oracle) and against the oracle at C12.

Every output storage is compared whole, halo and extra level included, so a
write outside a stencil's domain would show. Per field:
max |gpu - ref| <= 1e-12 * max |ref|, with an absolute floor only for the
surface precipitation totals (the column-condensate scale of the plain-form
gate, mp_helpers.gpu_floors) and for any tendency named in
mp_helpers.TENDENCY_FLOOR (carried through ``physics_updated_X = X + X_dt * dt``).
"""
import numpy as np
import pytest

from golden_io import MP_TENDENCIES, PHYS_CASES, PRECIP, load, physics_inputs
from mp_helpers import NOISE, TENDENCY_FLOOR, TOL_PLAIN, precip_scale

pytestmark = pytest.mark.gpu

H = 3
UPDATED = {
    "physics_updated_specific_humidity": ("qvapor", "qv_dt"), "physics_updated_qliquid": ("qliquid", "ql_dt"),
    "physics_updated_qrain": ("qrain", "qr_dt"), "physics_updated_qice": ("qice", "qi_dt"),
    "physics_updated_qsnow": ("qsnow", "qs_dt"), "physics_updated_qgraupel": ("qgraupel", "qg_dt"),
    "physics_updated_cloud_fraction": ("qcld", "qa_dt"), "physics_updated_pt": ("pt", "pt_dt"),
    "physics_updated_ua": ("ua", "udt"), "physics_updated_va": ("va", "vdt"),
}
TEND_STATE = {t: x for x, t in UPDATED.values()}


def _dev3(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda().permute(2, 1, 0)


def _host3(t):
    return t.permute(2, 1, 0).contiguous().cpu().numpy().transpose(2, 1, 0)


def run_physics_gpu(cfg, st, area, nx, ny, L, dt, ptop, dycore=None, fused=False):
    """Physics on device copies of the storages ``st``; returns the storages
    after the call (plus '_prsik', '_dm3d', '_del_gz') and the precipitation.
    With ``dycore`` (storages of DycoreToPhysics' 16 fields), DycoreToPhysics
    runs first: as its own call, or (``fused``) inside the pre-step launch."""
    import torch

    from pyshield_b200.grid import GridData, GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.inputs import PHYSICS_3D, PHYSICS_INTERFACE
    from pyshield_b200.physics import Physics, PhysicsState
    from pyshield_b200.quantity import Quantity

    gi = GridIndexing(nx, ny, L, H)
    qf = QuantityFactory(gi)
    q = {}
    for nm in PHYSICS_3D:
        dims = ("x", "y", "z_interface" if nm in PHYSICS_INTERFACE else "z")
        q[nm] = Quantity(_dev3(st[nm]), dims, "", (H, H, 0), (nx, ny, L + 1 if nm in PHYSICS_INTERFACE else L))
    q["land"] = Quantity(torch.from_numpy(np.ascontiguousarray(st["land"].T)).cuda().t(), ("x", "y"), "", (H, H), (nx, ny))
    ps = PhysicsState(**q, quantity_factory=qf, schemes=cfg.schemes)
    for t in MP_TENDENCIES:
        getattr(ps.microphysics, t).data.copy_(_dev3(st[t]))
    area_st = np.zeros(st["land"].shape)
    area_st[H:H + nx, H:H + ny] = area.reshape(ny, nx).T
    area_q = Quantity(torch.from_numpy(np.ascontiguousarray(area_st.T)).cuda().t(), ("x", "y"), "m^2", (H, H), (nx, ny))
    phys = Physics(StencilFactory(gi), qf, GridData(area_q, ptop), cfg)
    dyc = None
    if dycore is not None:
        import types

        from pyshield_b200.coupling import D2P_FIELDS, DycoreToPhysics

        dyc = types.SimpleNamespace(**{f: Quantity(_dev3(dycore[f]), ("x", "y", "z"), "", (H, H, 0), (nx, ny, L))
                                       for f in D2P_FIELDS})
        if not fused:
            DycoreToPhysics(StencilFactory(gi), qf, None, False, False)(dyc, ps)
    phys(ps, dt, dycore_state=dyc if fused else None)
    torch.cuda.synchronize()
    if dyc is not None:
        for f in D2P_FIELDS:
            assert np.array_equal(_host3(getattr(dyc, f).data), dycore[f]), f"the dycore's {f} changed"
    out = {nm: _host3(getattr(ps, nm).data) for nm in PHYSICS_3D}
    for t in MP_TENDENCIES:
        out[t] = _host3(getattr(ps.microphysics, t).data)
    out["_prsik"] = _host3(phys._prsik.data)
    out["_dm3d"] = _host3(phys._dm3d.data)
    out["_del_gz"] = _host3(phys._del_gz.data)
    pr = {p: getattr(phys._microphysics, p).t().contiguous().cpu().numpy().reshape(-1) for p in PRECIP}
    return out, pr


def _floors(st_in, ref, dt, nx, ny, L):
    """Round-off floors of the microphysics outputs (the plain-form gate's)."""
    ci, cj = slice(H, H + nx), slice(H, H + ny)
    fl = {}
    for t, x in TEND_STATE.items():
        if t not in TENDENCY_FLOOR:
            continue
        xin = ref[x][ci, cj, :L]
        xout = xin + ref[t][ci, cj, :L] * dt
        fl[t] = NOISE * max(float(np.max(np.abs(xin))), float(np.max(np.abs(xout)))) / dt
    for u, (x, t) in UPDATED.items():
        if t in fl:
            fl[u] = fl[t] * dt
    ln = {f: ref[f][ci, cj, :L].transpose(2, 1, 0).reshape(L, nx * ny)
          for f in ("qliquid", "qrain", "qice", "qsnow", "qgraupel", "delprsi")}
    ps = precip_scale(ln, dt)
    for p in PRECIP:
        fl[p] = TOL_PLAIN * ps
    return fl


def _compare(got, gpr, ref, rpr, fl, ctx):
    bad = {}
    for k, r in list(ref.items()) + list(rpr.items()):
        g = got[k] if k in got else gpr[k]
        d = float(np.max(np.abs(g - r)))
        allow = TOL_PLAIN * float(np.max(np.abs(r))) + fl.get(k, 0.0)
        if not d <= allow:
            bad[k] = (d, allow)
    assert not bad, f"{ctx}: {bad}"


@pytest.mark.parametrize("name", PHYS_CASES)
def test_physics_matches_reference_golden(name):
    from pyshield_b200._config import PhysicsConfig

    z, m = load(name)
    nx, ny, L, dt = m["nx"], m["ny"], m["L"], m["dt"]
    cfg = PhysicsConfig(**{k: v for k, v in m["config"].items() if k in PhysicsConfig.__dataclass_fields__})
    st, area = physics_inputs(z)
    got, gpr = run_physics_gpu(cfg, st, area, nx, ny, L, dt, m["ptop"])
    ref = {k[4:]: z[k] for k in z.files if k.startswith("out_") and k[4:] not in PRECIP}
    rpr = {p: z["out_" + p] for p in PRECIP}
    _compare(got, gpr, ref, rpr, _floors(st, ref, dt, nx, ny, L), name)


@pytest.mark.parametrize("kw,dt,nx,ny,L", [({}, 180.0, 12, 72, 79), ({"mp_time": 90.0, "do_qa": True}, 180.0, 12, 72, 79),
                                           ({}, 180.0, 6, 36, 127)])
def test_physics_matches_oracle_c12(kw, dt, nx, ny, L):
    """Against the oracle at C12 L79, and on 216 columns at L127 (the
    pre-step kernel's instantiation for more than 95 levels)."""
    from oracle.physics import OraclePhysics
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import PTOP, make_physics_state

    st, area = make_physics_state(nx, ny, L, seed=51, halo=H)
    cfg = PhysicsConfig(dt_atmos=int(dt), **kw)
    got, gpr = run_physics_gpu(cfg, st, area, nx, ny, L, dt, PTOP)
    ref = {k: np.array(v, copy=True) for k, v in st.items()}
    oracle = OraclePhysics(cfg, nx, ny, L, area, PTOP, H)
    rpr = oracle(ref, dt)
    ref.pop("land")
    ref["_prsik"], ref["_dm3d"], ref["_del_gz"] = oracle.prsik, oracle.dm3d, oracle.del_gz
    _compare(got, gpr, ref, rpr, _floors(st, ref, dt, nx, ny, L), f"{nx}x{ny} L{L} {kw}")


@pytest.mark.parametrize("L,dt", [(79, 180.0), (127, 150.0)])
def test_fused_dycore_copy_equals_copy_then_physics(L, dt):
    """Physics.__call__ with dycore_state (DycoreToPhysics' copy inside the
    pre-step launch) leaves every storage -- halo, interface points and the
    extra level included -- bit for bit as DycoreToPhysics.__call__ followed
    by Physics.__call__ does; the dycore storages are not written."""
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.coupling import D2P_FIELDS
    from pyshield_b200.inputs import PTOP, make_physics_state

    nx, ny = 12, 18
    st, area = make_physics_state(nx, ny, L, seed=61, halo=H)
    dyn, _ = make_physics_state(nx, ny, L, seed=62, halo=H)
    dycore = {f: dyn[f] for f in D2P_FIELDS}
    cfg = PhysicsConfig(dt_atmos=int(dt))
    a, apr = run_physics_gpu(cfg, st, area, nx, ny, L, dt, PTOP, dycore=dycore, fused=False)
    b, bpr = run_physics_gpu(cfg, st, area, nx, ny, L, dt, PTOP, dycore=dycore, fused=True)
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    for k in apr:
        assert np.array_equal(apr[k], bpr[k]), k
    # the copy did reach the physics storages: the dycore's winds
    np.testing.assert_array_equal(b["ua"][H:H + nx + 1, H:H + ny + 1, :L], dyn["ua"][H:H + nx + 1, H:H + ny + 1, :L])
