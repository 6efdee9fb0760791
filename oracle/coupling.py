"""CPU oracle for the physics-to-dynamics column coupling stencils.

TEST INFRASTRUCTURE ONLY (see ``oracle/microphysics.py``).

Restates, with GT4Py semantics and the reference's operand order:

* ``update_physics_state_with_tendencies`` -- ``pySHiELD/stencils/physics.py:146-194``
* ``fill_gfs_delp`` -- ``pySHiELD/update/update_atmos_state.py:21-37``
* ``prepare_tendencies_and_update_tracers`` -- ``pySHiELD/update/update_atmos_state.py:40-92``
* ``moist_cv`` -- ``pySHiELD/update/fv_update_phys.py:20-51``
* ``update_pressure_and_surface_winds`` -- ``pySHiELD/update/fv_update_phys.py:54-75``
* ``copy_dycore_to_physics`` -- ``pySHiELD/update/update_atmos_state.py:95-142``

Arrays carry k on the LAST axis and are already restricted to the stencil's
domain (``nk`` is the domain's level count: L for the compute domain, L+1
where the reference builds the stencil with ``add=(0, 0, 1)``).
"""

import numpy as np

from pyshield_b200 import constants as C

W = np.where


def update_physics_state_with_tendencies(state, tend, dt):
    """``physics_updated_X = X + X_dt * dt`` for the ten pairs (physics.py:187-194).
    ``state``/``tend`` map the reference argument names to arrays; returns
    the ten ``physics_updated_*`` arrays keyed by the input name."""
    pairs = (
        ("qvapor", "qv_dt"), ("qliquid", "ql_dt"), ("qrain", "qr_dt"), ("qice", "qi_dt"),
        ("qsnow", "qs_dt"), ("qgraupel", "qg_dt"), ("qcld", "qa_dt"), ("pt", "pt_dt"),
        ("ua", "udt"), ("va", "vdt"),
    )
    return {x: state[x] + tend[t] * dt for x, t in pairs}


def fill_gfs_delp(delp, q, q_min):
    """In place on ``q`` (domain of nk = L+1 levels)."""
    nk = q.shape[-1]
    for k in range(nk - 3, -1, -1):  # BACKWARD interval(0, -2)
        q[..., k] = W(
            q[..., k + 1] < q_min,
            q[..., k] + (q[..., k + 1] - q_min) * delp[..., k + 1] / delp[..., k],
            q[..., k],
        )
    inner = q[..., 1 : nk - 1]  # PARALLEL interval(1, -1)
    q[..., 1 : nk - 1] = W(inner < q_min, q_min, inner)
    for k in range(1, nk - 1):  # FORWARD interval(1, -1)
        q[..., k] = W(
            q[..., k - 1] < 0.0,
            q[..., k] + q[..., k - 1] * (delp[..., k - 1]) / (delp[..., k]),
            q[..., k],
        )
    for k in range(0, nk - 1):  # FORWARD interval(0, -1)
        q[..., k] = W(q[..., k] < 0.0, 0.0, q[..., k])
    return q


def prepare_tendencies_and_update_tracers(a, rdt):
    """In place on ``a`` (a dict with the reference argument names; 3-D
    arrays on a domain of nk = L+1 levels, ``prsi`` included)."""
    nk = a["prsi"].shape[-1]
    s = slice(0, nk - 1)
    g = {k: v[..., s] for k, v in a.items() if k != "prsi"}
    prsi = a["prsi"]
    a["u_dt"][..., s] = g["u_dt"] + (g["u_t1"] - g["u_t0"]) * rdt
    a["v_dt"][..., s] = g["v_dt"] + (g["v_t1"] - g["v_t0"]) * rdt
    a["pt_dt"][..., s] = g["pt_dt"] + (g["physics_updated_pt"] - g["pt_t0"]) * rdt
    dp = prsi[..., 1:nk] - prsi[..., 0 : nk - 1]
    qwat_qv = dp * g["physics_updated_specific_humidity"]
    qwat_ql = dp * g["physics_updated_qliquid"]
    qwat_qr = dp * g["physics_updated_qrain"]
    qwat_qs = dp * g["physics_updated_qsnow"]
    qwat_qi = dp * g["physics_updated_qice"]
    qwat_qg = dp * g["physics_updated_qgraupel"]
    qt = qwat_qv + qwat_ql + qwat_qr + qwat_qs + qwat_qi + qwat_qg
    q_sum = (
        g["qvapor_t0"] + g["qliquid_t0"] + g["qrain_t0"] + g["qsnow_t0"] + g["qice_t0"] + g["qgraupel_t0"]
    )
    q0 = g["delp"] * (1.0 - q_sum) + qt
    a["delp"][..., s] = q0
    a["qvapor_t0"][..., s] = qwat_qv / q0
    a["qliquid_t0"][..., s] = qwat_ql / q0
    a["qrain_t0"][..., s] = qwat_qr / q0
    a["qsnow_t0"][..., s] = qwat_qs / q0
    a["qice_t0"][..., s] = qwat_qi / q0
    a["qgraupel_t0"][..., s] = qwat_qg / q0
    return a


def moist_cv(qvapor, qliquid, qrain, qsnow, qice, qgraupel, pt, t_dt, con_cp, dt):
    """In place on ``pt`` and ``t_dt`` over their whole (domain) extent."""
    ql = qliquid + qrain
    qs = qice + qsnow + qgraupel
    gz = ql + qs
    cvm = (
        (1.0 - (qvapor + gz)) * C.CV_AIR
        + qvapor * C.CV_VAP
        + ql * C.C_LIQ
        + qs * C.C_ICE
    )
    pt[...] = pt + t_dt * dt * con_cp / cvm
    t_dt[...] = 0.0
    return pt, t_dt


def update_pressure_and_surface_winds(pe, delp, peln, pk, kappa, ua, va):
    """In place on pe/peln/pk (domain of nk = L+1 levels); returns
    ``(ps, u_srf, v_srf)``."""
    nk = pe.shape[-1]
    for k in range(1, nk):
        pe[..., k] = pe[..., k - 1] + delp[..., k - 1]
    peln[..., 1:] = np.log(pe[..., 1:])
    pk[..., 1:] = np.exp(kappa * peln[..., 1:])
    return pe[..., nk - 1].copy(), ua[..., nk - 2].copy(), va[..., nk - 2].copy()


def update_atmos_state_columns(f, dt, nx, ny, h, dycore_only=False, apply_tendencies=True):
    """The column part of ``UpdateAtmosphereState.__call__``
    (update_atmos_state.py:301-349, fv_update_phys.py:170-186), in place on
    NDSL storages (ni, nj, L+1) keyed as in tests/golden/make_golden.py:
    ``pu_*`` physics-updated fields, ``ph_*`` physics-state fields, ``dy_*``
    dycore fields, ``u_dt``/``v_dt``/``pt_dt``, ``prsi``, ``pe``/``peln``/``pk``.
    fill_gfs_delp runs on the full domain [0, nx+2h) x [0, ny+2h); the others
    on the compute domain. Returns (ps, u_srf, v_srf) on the compute domain,
    or None when the tendencies are not applied."""
    full = (slice(0, nx + 2 * h), slice(0, ny + 2 * h))
    cd = (slice(h, h + nx), slice(h, h + ny))
    if dycore_only:
        q = f["dy_qvapor"][full]
        fill_gfs_delp(f["dy_delp"][full], q, 1.0e-9)
    else:
        q = f["pu_qvapor"][full]
        fill_gfs_delp(f["dy_delp"][full], q, 1.0e-9)
        a = {
            "u_dt": f["u_dt"][cd], "v_dt": f["v_dt"][cd], "pt_dt": f["pt_dt"][cd],
            "u_t1": f["pu_ua"][cd], "v_t1": f["pu_va"][cd], "physics_updated_pt": f["pu_pt"][cd],
            "physics_updated_specific_humidity": f["pu_qvapor"][cd],
            "physics_updated_qliquid": f["pu_qliquid"][cd], "physics_updated_qrain": f["pu_qrain"][cd],
            "physics_updated_qsnow": f["pu_qsnow"][cd], "physics_updated_qice": f["pu_qice"][cd],
            "physics_updated_qgraupel": f["pu_qgraupel"][cd],
            "u_t0": f["ph_ua"][cd], "v_t0": f["ph_va"][cd], "pt_t0": f["ph_pt"][cd],
            "qvapor_t0": f["dy_qvapor"][cd], "qliquid_t0": f["dy_qliquid"][cd], "qrain_t0": f["dy_qrain"][cd],
            "qsnow_t0": f["dy_qsnow"][cd], "qice_t0": f["dy_qice"][cd], "qgraupel_t0": f["dy_qgraupel"][cd],
            "prsi": f["prsi"][cd], "delp": f["dy_delp"][cd],
        }
        prepare_tendencies_and_update_tracers(a, 1.0 / dt)
    if not apply_tendencies:
        return None
    moist_cv(
        f["dy_qvapor"][cd], f["dy_qliquid"][cd], f["dy_qrain"][cd], f["dy_qsnow"][cd], f["dy_qice"][cd],
        f["dy_qgraupel"][cd], f["dy_pt"][cd], f["pt_dt"][cd], C.CP_AIR, dt,
    )
    return update_pressure_and_surface_winds(
        f["pe"][cd], f["dy_delp"][cd], f["peln"][cd], f["pk"][cd], C.KAPPA, f["dy_ua"][cd], f["dy_va"][cd]
    )


D2P_FIELDS = ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "qo3mr", "qsgs_tke", "qcld", "pt", "delp",
              "delz", "ua", "va", "w", "omga")


def copy_dycore_to_physics(dycore, physics, nx, ny, nz, h=3):
    """update_atmos_state.py:95-142 as DycoreToPhysics builds it
    (:160-167): the compute domain extended by one interface point in x and
    y, PARALLEL interval(0, -1) of nz + 1 levels. In place on ``physics``."""
    box = (slice(h, h + nx + 1), slice(h, h + ny + 1), slice(0, nz))
    for f in D2P_FIELDS:
        physics[f][box] = dycore[f][box]
