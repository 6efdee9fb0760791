"""GPU parity of the coupling kernels against the reference's own stencils
(golden fixtures from tests/golden/make_golden.py; the CPU oracle matches
them bit for bit). Tolerance: 1e-12 relative per field (these kernels are
elementwise or short column sweeps with no cancellation-prone sums)."""
import types

import numpy as np
import pytest

from golden_io import load

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _dev(a, layout):
    import torch

    if layout == "ifirst" and a.ndim == 3:
        return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
    if layout == "ifirst" and a.ndim == 2:
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _q(a, nx, ny, L, h, layout):
    from pyshield_b200.quantity import Quantity

    if a.ndim == 3:
        return Quantity(_dev(a, layout), ("x", "y", "z"), "", (h, h, 0), (nx, ny, L))
    return Quantity(_dev(a, layout), ("x", "y"), "", (h, h), (nx, ny))


def _close(got, ref, what):
    scale = float(np.max(np.abs(ref)))
    err = float(np.max(np.abs(got - ref)))
    assert err <= TOL * max(scale, 1e-300), f"{what}: {err / max(scale, 1e-300):.3e}"


@pytest.mark.parametrize("layout", ["ifirst", "kfirst"])
@pytest.mark.parametrize("name", ["cpl_small", "cpl_stress"])
def test_update_physics_state(name, layout):
    from pyshield_b200.coupling import update_physics_state_with_tendencies

    z, m = load(name)
    nx, ny, L, dt, h = m["nx"], m["ny"], m["L"], m["dt"], m["halo"]
    names = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "pt", "ua", "va")
    tends = ("qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "pt_dt", "udt", "vdt")
    s = [_q(z["upd_in_" + n], nx, ny, L, h, layout) for n in names]
    t = [_q(z["upd_in_" + n], nx, ny, L, h, layout) for n in tends]
    o = [_q(np.zeros_like(z["upd_in_qvapor"]), nx, ny, L, h, layout) for _ in names]
    update_physics_state_with_tendencies(*s, *t, *o, dt)
    cs = (slice(h, h + nx), slice(h, h + ny), slice(0, L))
    for n, q in zip(names, o):
        _close(q.data.cpu().numpy()[cs], z["upd_out_" + n][cs], n)


@pytest.mark.parametrize("layout", ["ifirst", "kfirst"])
def test_update_atmos_state_chain(layout):
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.coupling import UpdateAtmosphereState
    from pyshield_b200.grid import GridIndexing, StencilFactory

    z, m = load("cpl_chain")
    nx, ny, L, dt, h = m["nx"], m["ny"], m["L"], m["dt"], m["halo"]
    f = {k[3:]: np.array(z[k]) for k in z.files if k.startswith("in_")}
    Q = {k: _q(v, nx, ny, L, h, layout) for k, v in f.items()}
    ps = np.zeros(f["pe"].shape[:2])
    d = types.SimpleNamespace(
        qvapor=Q["dy_qvapor"], qliquid=Q["dy_qliquid"], qrain=Q["dy_qrain"], qsnow=Q["dy_qsnow"],
        qice=Q["dy_qice"], qgraupel=Q["dy_qgraupel"], delp=Q["dy_delp"], pt=Q["dy_pt"], pe=Q["pe"],
        peln=Q["peln"], pk=Q["pk"], ua=Q["dy_ua"], va=Q["dy_va"], ps=_q(ps, nx, ny, L, h, layout),
    )
    p = types.SimpleNamespace(
        physics_updated_ua=Q["pu_ua"], physics_updated_va=Q["pu_va"], physics_updated_pt=Q["pu_pt"],
        physics_updated_specific_humidity=Q["pu_qvapor"], physics_updated_qliquid=Q["pu_qliquid"],
        physics_updated_qrain=Q["pu_qrain"], physics_updated_qsnow=Q["pu_qsnow"], physics_updated_qice=Q["pu_qice"],
        physics_updated_qgraupel=Q["pu_qgraupel"], ua=Q["ph_ua"], va=Q["ph_va"], pt=Q["ph_pt"], prsi=Q["prsi"],
    )
    cfg = PhysicsConfig(dt_atmos=dt)
    uas = UpdateAtmosphereState(StencilFactory(GridIndexing(nx, ny, L, h)), None, cfg)
    uas(d, p, Q["u_dt"], Q["v_dt"], Q["pt_dt"], dt)
    import torch

    torch.cuda.synchronize()
    full = (slice(0, nx + 2 * h), slice(0, ny + 2 * h))
    cd = (slice(h, h + nx), slice(h, h + ny))
    for k, q in Q.items():
        got = q.data.cpu().numpy()
        ref = z["out_" + k]
        if k == "pu_qvapor":
            _close(got[full], ref[full], k)
        elif k in ("peln", "pk"):
            _close(got[cd][..., 1:], ref[cd][..., 1:], k)
        else:
            _close(got[cd], ref[cd], k)
    _close(d.ps.data.cpu().numpy()[cd], z["out_ps"][cd], "ps")
    _close(uas.u_srf.cpu().numpy(), z["out_u_srf"][cd], "u_srf")
    _close(uas.v_srf.cpu().numpy(), z["out_v_srf"][cd], "v_srf")


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["ifirst", "kfirst"])
def test_dycore_to_physics_matches_reference(layout):
    """DycoreToPhysics' copy against the reference's own result (golden):
    every storage whole, so nothing outside the interface-extended compute
    domain and levels 0 .. nz - 1 may change."""
    import numpy as np
    import torch

    from golden_io import load
    from pyshield_b200.coupling import D2P_FIELDS, DycoreToPhysics
    from pyshield_b200.grid import GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.quantity import Quantity

    z, m = load("d2p_copy")
    nx, ny, L, h = m["nx"], m["ny"], m["L"], m["halo"]

    def dev(a):
        if layout == "ifirst":
            return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    class State:
        pass

    ds, ps = State(), State()
    for f in D2P_FIELDS:
        setattr(ds, f, Quantity(dev(z["in_dycore_" + f]), ("x", "y", "z"), "", (h, h, 0), (nx, ny, L)))
        setattr(ps, f, Quantity(dev(z["in_physics_" + f]), ("x", "y", "z"), "", (h, h, 0), (nx, ny, L)))
    gi = GridIndexing(nx, ny, L, h)
    DycoreToPhysics(StencilFactory(gi), QuantityFactory(gi), None, False, False)(ds, ps)
    torch.cuda.synchronize()
    for f in D2P_FIELDS:
        got = getattr(ps, f).data.cpu().numpy()
        np.testing.assert_array_equal(got, z["out_physics_" + f], err_msg=f)


@pytest.mark.parametrize("L", [79, 127])
def test_update_atmos_state_tall_columns_match_oracle(L):
    """UpdateAtmosphereState on 390 columns of L79 and L127 (the kernel's
    instantiations for up to 95 and up to 128 levels) against the oracle,
    with negative physics-updated vapour at 5 % of the points so that
    fill_gfs_delp borrows."""
    import torch

    from oracle import coupling as OC
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.coupling import UpdateAtmosphereState
    from pyshield_b200.grid import GridIndexing, StencilFactory

    nx, ny, h, dt = 20, 9, 3, 180.0
    shape = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
    rng = np.random.default_rng(700 + L)
    f = {}
    for n in ("u_dt", "v_dt", "pt_dt"):
        f[n] = rng.normal(0.0, 1e-4, shape)
    for n in ("pu_ua", "pu_va", "ph_ua", "ph_va", "dy_ua", "dy_va"):
        f[n] = rng.uniform(-30.0, 30.0, shape)
    for n in ("pu_pt", "ph_pt", "dy_pt"):
        f[n] = rng.uniform(200.0, 300.0, shape)
    for n in ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel"):
        f["pu_" + n] = rng.uniform(0.0, 2e-3, shape)
        f["dy_" + n] = rng.uniform(0.0, 2e-3, shape)
    neg = rng.random(shape) < 0.05
    f["pu_qvapor"][neg] = -rng.uniform(0.0, 1e-6, int(neg.sum()))
    f["prsi"] = np.cumsum(rng.uniform(50.0, 2000.0, shape), axis=2)
    f["dy_delp"] = rng.uniform(50.0, 2000.0, shape)
    f["pe"] = np.zeros(shape)
    f["pe"][..., 0] = 100.0
    f["peln"] = np.zeros(shape)
    f["pk"] = np.zeros(shape)
    ref = {k: v.copy() for k, v in f.items()}
    rps, rus, rvs = OC.update_atmos_state_columns(ref, dt, nx, ny, h)

    Q = {k: _q(v, nx, ny, L, h, "ifirst") for k, v in f.items()}
    ps = np.zeros(shape[:2])
    d = types.SimpleNamespace(
        qvapor=Q["dy_qvapor"], qliquid=Q["dy_qliquid"], qrain=Q["dy_qrain"], qsnow=Q["dy_qsnow"],
        qice=Q["dy_qice"], qgraupel=Q["dy_qgraupel"], delp=Q["dy_delp"], pt=Q["dy_pt"], pe=Q["pe"],
        peln=Q["peln"], pk=Q["pk"], ua=Q["dy_ua"], va=Q["dy_va"], ps=_q(ps, nx, ny, L, h, "ifirst"),
    )
    p = types.SimpleNamespace(
        physics_updated_ua=Q["pu_ua"], physics_updated_va=Q["pu_va"], physics_updated_pt=Q["pu_pt"],
        physics_updated_specific_humidity=Q["pu_qvapor"], physics_updated_qliquid=Q["pu_qliquid"],
        physics_updated_qrain=Q["pu_qrain"], physics_updated_qsnow=Q["pu_qsnow"], physics_updated_qice=Q["pu_qice"],
        physics_updated_qgraupel=Q["pu_qgraupel"], ua=Q["ph_ua"], va=Q["ph_va"], pt=Q["ph_pt"], prsi=Q["prsi"],
    )
    uas = UpdateAtmosphereState(StencilFactory(GridIndexing(nx, ny, L, h)), None, PhysicsConfig(dt_atmos=int(dt)))
    uas(d, p, Q["u_dt"], Q["v_dt"], Q["pt_dt"], dt)
    torch.cuda.synchronize()
    full = (slice(0, nx + 2 * h), slice(0, ny + 2 * h))
    cd = (slice(h, h + nx), slice(h, h + ny))
    for k, q in Q.items():
        got = q.data.cpu().numpy()
        if k == "pu_qvapor":
            _close(got[full], ref[k][full], k)
        elif k in ("peln", "pk"):
            _close(got[cd][..., 1:L + 1], ref[k][cd][..., 1:L + 1], k)
        else:
            _close(got[cd], ref[k][cd], k)
    _close(d.ps.data.cpu().numpy()[cd], rps, "ps")
    _close(uas.u_srf.cpu().numpy(), rus, "u_srf")
    _close(uas.v_srf.cpu().numpy(), rvs, "v_srf")
