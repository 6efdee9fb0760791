"""The oracle reproduces the reference's own source bit for bit.

The fixtures were produced by running pySHiELD's ``Microphysics`` class and
coupling stencils (their unmodified source) through a GT4Py-semantics numpy
executor; see tests/golden/make_golden.py.
"""
import numpy as np
import pytest

from golden_io import CPL_CASES, MP_CASES, MP_TENDENCIES, PHYS_CASES, PRECIP, load, mp_inputs, physics_inputs
from oracle import coupling as OC
from oracle.microphysics import OracleMicrophysics
from pyshield_b200 import constants as C
from pyshield_b200._config import PhysicsConfig


@pytest.mark.parametrize("name", MP_CASES)
def test_microphysics_bitexact(name):
    z, meta = load(name)
    cfg = PhysicsConfig(**meta["config"])
    state, area = mp_inputs(z)
    L, n = meta["L"], meta["nx"] * meta["ny"]
    mp = OracleMicrophysics(cfg, n, L, area)
    for step in range(meta["nsteps"]):
        precip = mp(state, meta["dt"])
        for f in MP_TENDENCIES + ("wmp", "qice", "qsnow"):
            np.testing.assert_array_equal(state[f], z[f"s{step}_{f}"], err_msg=f"{name} step{step} {f}")
        for f in PRECIP:
            np.testing.assert_array_equal(precip[f], z[f"s{step}_{f}"], err_msg=f"{name} {f}")
        np.testing.assert_array_equal(mp.qaz, z[f"s{step}_qaz"])


def _coupling(name):
    z, m = load(name)
    nx, ny, L, dt, h = m["nx"], m["ny"], m["L"], m["dt"], m["halo"]
    return z, nx, ny, L, dt, h


@pytest.mark.parametrize("name", CPL_CASES)
def test_update_physics_state_bitexact(name):
    z, nx, ny, L, dt, h = _coupling(name)
    cs = (slice(h, h + nx), slice(h, h + ny), slice(0, L))
    st = {k[7:]: z[k][cs] for k in z.files if k.startswith("upd_in_")}
    res = OC.update_physics_state_with_tendencies(st, st, dt)
    for k, v in res.items():
        np.testing.assert_array_equal(v, z["upd_out_" + k][cs])


@pytest.mark.parametrize("name", CPL_CASES)
def test_fill_gfs_delp_bitexact(name):
    z, nx, ny, L, dt, h = _coupling(name)
    fd = (slice(0, nx + 2 * h), slice(0, ny + 2 * h))
    q = z["fill_in_q"][fd].copy()
    OC.fill_gfs_delp(z["fill_in_delp"][fd], q, 1.0e-9)
    np.testing.assert_array_equal(q, z["fill_out_q"][fd])


PREP_RENAME = {"pu_pt": "physics_updated_pt", "pu_qvapor": "physics_updated_specific_humidity"}
for _nm in ("qliquid", "qrain", "qice", "qsnow", "qgraupel"):
    PREP_RENAME["pu_" + _nm] = "physics_updated_" + _nm


@pytest.mark.parametrize("name", CPL_CASES)
def test_prepare_tendencies_bitexact(name):
    z, nx, ny, L, dt, h = _coupling(name)
    cs = (slice(h, h + nx), slice(h, h + ny))
    a = {PREP_RENAME.get(k[8:], k[8:]): z[k][cs].copy() for k in z.files if k.startswith("prep_in_")}
    OC.prepare_tendencies_and_update_tracers(a, 1.0 / dt)
    for k in [f for f in z.files if f.startswith("prep_out_")]:
        np.testing.assert_array_equal(a[k[9:]], z[k][cs], err_msg=k)


@pytest.mark.parametrize("name", CPL_CASES)
def test_moist_cv_and_pressure_bitexact(name):
    z, nx, ny, L, dt, h = _coupling(name)
    cs = (slice(h, h + nx), slice(h, h + ny))
    m = {k[7:]: z[k][cs].copy() for k in z.files if k.startswith("mcv_in_")}
    OC.moist_cv(m["qvapor"], m["qliquid"], m["qrain"], m["qsnow"], m["qice"], m["qgraupel"], m["pt"], m["t_dt"], C.CP_AIR, dt)
    np.testing.assert_array_equal(m["pt"], z["mcv_out_pt"][cs])
    np.testing.assert_array_equal(m["t_dt"], z["mcv_out_t_dt"][cs])
    pe = z["ups_in_pe"][cs].copy()
    peln = np.zeros_like(pe)
    pk = np.zeros_like(pe)
    ps, us, vs = OC.update_pressure_and_surface_winds(
        pe, z["ups_in_delp"][cs], peln, pk, C.KAPPA, z["ups_in_ua"][cs], z["ups_in_va"][cs]
    )
    np.testing.assert_array_equal(pe, z["ups_out_pe"][cs])
    np.testing.assert_array_equal(peln[..., 1:], z["ups_out_peln"][cs][..., 1:])
    np.testing.assert_array_equal(pk[..., 1:], z["ups_out_pk"][cs][..., 1:])
    np.testing.assert_array_equal(ps, z["ups_out_ps"][cs])
    np.testing.assert_array_equal(us, z["ups_out_u_srf"][cs])
    np.testing.assert_array_equal(vs, z["ups_out_v_srf"][cs])


def test_update_atmos_state_chain_bitexact():
    """fill_gfs_delp -> prepare_tendencies_and_update_tracers -> moist_cv ->
    update_pressure_and_surface_winds on one state, as UpdateAtmosphereState
    runs them."""
    z, m = load("cpl_chain")
    nx, ny, h, dt = m["nx"], m["ny"], m["halo"], m["dt"]
    f = {k[3:]: np.array(z[k]) for k in z.files if k.startswith("in_")}
    ps, us, vs = OC.update_atmos_state_columns(f, dt, nx, ny, h)
    full = (slice(0, nx + 2 * h), slice(0, ny + 2 * h))
    cd = (slice(h, h + nx), slice(h, h + ny))
    for k, v in f.items():
        ref = z["out_" + k]
        if k == "pu_qvapor":
            np.testing.assert_array_equal(v[full], ref[full], err_msg=k)
        elif k in ("peln", "pk"):
            np.testing.assert_array_equal(v[cd][..., 1:], ref[cd][..., 1:], err_msg=k)
        else:
            np.testing.assert_array_equal(v[cd], ref[cd], err_msg=k)
    np.testing.assert_array_equal(ps, z["out_ps"][cd])
    np.testing.assert_array_equal(us, z["out_u_srf"][cd])
    np.testing.assert_array_equal(vs, z["out_v_srf"][cd])


@pytest.mark.parametrize("name", PHYS_CASES)
def test_physics_call_bitexact(name):
    """Physics.__call__: the driver pre-steps on the compute and full
    domains, the microphysics step and the state update."""
    from oracle.physics import OraclePhysics

    z, m = load(name)
    cfg = PhysicsConfig(**{k: v for k, v in m["config"].items() if k in PhysicsConfig.__dataclass_fields__})
    st, area = physics_inputs(z)
    ph = OraclePhysics(cfg, m["nx"], m["ny"], m["L"], area, m["ptop"], m["halo"])
    precip = ph(st, m["dt"])
    for k in [f[4:] for f in z.files if f.startswith("out_")]:
        if k.startswith("_"):
            got = {"_prsik": ph.prsik, "_dm3d": ph.dm3d, "_del_gz": ph.del_gz}[k]
        elif k in PRECIP:
            got = precip[k]
        else:
            got = st[k]
        np.testing.assert_array_equal(got, z["out_" + k], err_msg=f"{name} {k}")


def test_copy_dycore_to_physics_bitexact():
    """DycoreToPhysics' 16-field copy on the interface-extended domain."""
    z, m = load("d2p_copy")
    dy = {k[10:]: z[k] for k in z.files if k.startswith("in_dycore_")}
    ph = {k[11:]: np.array(z[k]) for k in z.files if k.startswith("in_physics_")}
    OC.copy_dycore_to_physics(dy, ph, m["nx"], m["ny"], m["L"], m["halo"])
    for f, v in ph.items():
        np.testing.assert_array_equal(v, z["out_physics_" + f], err_msg=f)


DWIND_CASES = ("dwind_tile", "dwind_sub0", "dwind_sub3", "dwind_periodic")


@pytest.mark.parametrize("name", DWIND_CASES)
def test_agrid_to_dgrid_bitexact(name):
    """AGrid2DGridPhysics on one rank's subtile: prep, reset, edge
    corrections of the rank's cube edges, D-grid update."""
    from oracle import dwind as OD

    z, m = load(name)
    nx, ny, L, h = m["nx"], m["ny"], m["L"], m["halo"]
    f = {k: np.array(z["in_" + k]) for k in ("u", "v", "u_dt", "v_dt")}
    g = {k[5:]: z[k] for k in z.files if k.startswith("geom_")}
    dt5 = 0.5 * m["dt"]
    if m["grid_type"] > 3:
        OD.doubly_periodic(f["u"], f["v"], f["u_dt"], f["v_dt"], nx, ny, L, h, dt5)
    else:
        plan = OD.edge_plan(nx, ny, h, m["npx"], m["npy"], m["layout"], m["subtile_index"], m["edges"])
        OD.agrid_to_dgrid(f["u"], f["v"], f["u_dt"], f["v_dt"], g, nx, ny, L, h, dt5, plan)
    for k, v in f.items():
        np.testing.assert_array_equal(v, z["out_" + k], err_msg=f"{name} {k}")
