"""CPU oracle for pySHiELD's physics driver: ``Physics.__call__``.

TEST INFRASTRUCTURE ONLY (see ``oracle/microphysics.py``).

Restates, with GT4Py semantics and the reference's operand order:

* ``atmos_phys_driver_statein`` -- ``pySHiELD/stencils/physics.py:26-102``
* ``prepare_microphysics``      -- ``pySHiELD/stencils/physics.py:105-143``
* ``get_prs_fv3``               -- ``pySHiELD/stencils/get_prs_fv3.py:7-20``
* ``get_phi_fv3``               -- ``pySHiELD/stencils/get_phi_fv3.py:7-25``
* ``Physics.__init__`` scalars and ``Physics.__call__`` -- ``physics.py:197-366``:
  statein on the compute domain with nz + 1 levels, get_prs_fv3 and
  get_phi_fv3 on the full (halo) domain with nz + 1 levels,
  prepare_microphysics on the compute domain, the microphysics step,
  update_physics_state_with_tendencies.

Arrays carry k on the LAST axis and are views restricted to the stencil's
horizontal domain; the functions update them in place.
"""

import numpy as np

from pyshield_b200 import constants as C

from .coupling import update_physics_state_with_tendencies
from .microphysics import OracleMicrophysics

TRACERS = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr")
TENDENCIES = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")
P00 = 1.0e5  # Physics._setup_statein (physics.py:270-274)
NWAT = 6


def atmos_phys_driver_statein(f, prsik, dm, nwat, ptop, pk0inv, pktop):
    """physics.py:26-102 on nk = nz + 1 levels. ``f`` maps the argument names
    (phii, prsi, delz, delp, the seven tracers, qsgs_tke, pt) to views."""
    phii, prsi, delz, delp, pt = f["phii"], f["prsi"], f["delz"], f["delp"], f["pt"]
    nk = phii.shape[-1]
    s, s1 = slice(0, nk - 1), slice(1, nk)
    # BACKWARD interval(...) then BACKWARD interval(0, -1)
    phii[...] = 0.0
    for k in range(nk - 2, -1, -1):
        phii[..., k] = phii[..., k + 1] - delz[..., k] * C.GRAV
    # PARALLEL interval(...)
    prsik[...] = 1.0e25
    for q in TRACERS:
        f[q][...] = f[q] * delp
    if nwat == 6:
        delp[...] = delp - f["qliquid"] - f["qrain"] - f["qice"] - f["qsnow"] - f["qgraupel"]
    prsi[..., 0] = ptop
    for k in range(1, nk):  # FORWARD interval(1, None)
        prsi[..., k] = prsi[..., k - 1] + delp[..., k - 1]
    # PARALLEL interval(0, -1)
    prsik[..., s] = np.log(prsi[..., s])
    for q in TRACERS + ("qsgs_tke",):
        f[q][..., s] = f[q][..., s] / delp[..., s]
    prsik[..., nk - 1] = np.log(prsi[..., nk - 1])  # interval(-1, None)
    prsik[..., 0] = np.log(ptop)  # interval(0, 1)
    # PARALLEL interval(0, -1): the layer thickness from the geopotential
    qgrs_rad = np.maximum(1.0e-10, f["qvapor"][..., s])
    rTv = C.RDGAS * pt[..., s] * (1.0 + C.ZVIR * qgrs_rad)
    dm[..., s] = delp[..., s]
    d = dm[..., s] * rTv / (phii[..., s] - phii[..., s1])
    d = np.minimum(d, prsi[..., s1] - 0.01 * dm[..., s])
    delp[..., s] = np.maximum(d, prsi[..., s] + 0.01 * dm[..., s])
    prsik[..., nk - 1] = np.exp(C.KAPPA * prsik[..., nk - 1]) * pk0inv
    prsik[..., 0] = pktop


def get_prs_fv3(phii, prsi, tgrs, qgrs, del_, del_gz):
    """get_prs_fv3.py:7-20, interval(0, -1) of nk = nz + 1 levels."""
    nk = phii.shape[-1]
    s, s1 = slice(0, nk - 1), slice(1, nk)
    del_[..., s] = prsi[..., s1] - prsi[..., s]
    del_gz[..., s] = (phii[..., s] - phii[..., s1]) / (tgrs[..., s] * (1.0 + C.ZVIR * np.maximum(0.0, qgrs[..., s])))


def get_phi_fv3(gt0, gq0, del_gz, phii, phil):
    """get_phi_fv3.py:7-25 on nk = nz + 1 levels. ``phil`` is the reference's
    ``0.5 * (phii[k + 1] + phii[k + 1] + del_gz)`` (the level below taken
    twice), kept as written."""
    nk = phii.shape[-1]
    s = slice(0, nk - 1)
    del_gz[..., s] = del_gz[..., s] * gt0[..., s] * (1.0 + C.ZVIR * np.maximum(0.0, gq0[..., s]))
    phii[..., nk - 1] = 0.0
    for k in range(nk - 2, -1, -1):  # BACKWARD interval(-2, -1), interval(0, -2)
        phil[..., k] = 0.5 * (phii[..., k + 1] + phii[..., k + 1] + del_gz[..., k])
        phii[..., k] = phii[..., k + 1] + del_gz[..., k]


def prepare_microphysics(dz, phii, wmp, omga, qvapor, pt, delp, tend):
    """physics.py:105-143 on nz levels (``phii`` carries nz + 1)."""
    nz = dz.shape[-1]
    dz[...] = (phii[..., 1:nz + 1] - phii[..., 0:nz]) * C.RGRAV
    wmp[...] = -omga * (1.0 + C.ZVIR * qvapor) * pt / delp * (C.RDGAS * C.RGRAV)
    for t in tend:
        t[...] = 0.0


class OraclePhysics:
    """``Physics`` (physics.py:197-366) on full NDSL-layout storages.

    ``st`` maps the PhysicsState attribute names to arrays of shape
    (nx + 2h + 1, ny + 2h + 1, nz + 1) (``land`` 2-D), plus the ten
    tendencies of ``physics_state.microphysics`` under their own names
    (``pt_dt``, ...). The Physics-owned scratch (``_prsik``, ``_dm3d``,
    ``_del_gz``) lives on this object."""

    def __init__(self, cfg, nx, ny, nz, area, ptop, halo=3):
        self.cfg = cfg
        self.nx, self.ny, self.nz, self.h = nx, ny, nz, halo
        self.ptop = float(ptop)
        self.pktop = (self.ptop / P00) ** C.KAPPA
        self.pk0inv = (1.0 / P00) ** C.KAPPA
        shape = (nx + 2 * halo + 1, ny + 2 * halo + 1, nz + 1)
        self.prsik = np.zeros(shape)
        self.dm3d = np.zeros(shape)
        self.del_gz = np.zeros(shape)
        self.mp = OracleMicrophysics(cfg, nx * ny, nz, area)
        self.precip = None

    def __call__(self, st, timestep):
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.h
        ci, cj = slice(h, h + nx), slice(h, h + ny)
        fi, fj = slice(0, nx + 2 * h), slice(0, ny + 2 * h)
        cv = {k: v[ci, cj] for k, v in st.items() if v.ndim == 3}
        atmos_phys_driver_statein(cv, self.prsik[ci, cj], self.dm3d[ci, cj], NWAT, self.ptop, self.pk0inv, self.pktop)
        get_prs_fv3(st["phii"][fi, fj], st["prsi"][fi, fj], st["pt"][fi, fj], st["qvapor"][fi, fj],
                    st["delprsi"][fi, fj], self.del_gz[fi, fj])
        get_phi_fv3(st["pt"][fi, fj], st["qvapor"][fi, fj], self.del_gz[fi, fj], st["phii"][fi, fj],
                    st["phil"][fi, fj])
        k3 = slice(0, nz)
        tend = [st[t][ci, cj, k3] for t in TENDENCIES]
        prepare_microphysics(st["dz"][ci, cj, k3], st["phii"][ci, cj], st["wmp"][ci, cj, k3], st["omga"][ci, cj, k3],
                             st["qvapor"][ci, cj, k3], st["pt"][ci, cj, k3], st["delp"][ci, cj, k3], tend)
        # the microphysics step on the compute domain, (L, n) arrays
        def to_ln(a):
            return np.ascontiguousarray(a[ci, cj, k3].transpose(2, 1, 0).reshape(nz, nx * ny))

        def from_ln(a, dst):
            dst[ci, cj, k3] = a.reshape(nz, ny, nx).transpose(2, 1, 0)

        names = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi",
                 "delz", "wmp")
        s = {k: to_ln(st[k]) for k in names}
        for t in TENDENCIES:
            s[t] = to_ln(st[t])
        s["land"] = np.ascontiguousarray(st["land"][ci, cj].T.reshape(nx * ny))
        self.precip = self.mp(s, timestep)
        for t in TENDENCIES:
            from_ln(s[t], st[t])
        for k in ("wmp", "qice", "qsnow"):
            from_ln(s[k], st[k])
        # update_physics_state_with_tendencies on the compute domain
        state = {k: st[k][ci, cj, k3] for k in ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld",
                                                 "pt", "ua", "va")}
        tnd = {t: st[t][ci, cj, k3] for t in TENDENCIES}
        res = update_physics_state_with_tendencies(state, tnd, timestep)
        out_name = {"qvapor": "physics_updated_specific_humidity", "qcld": "physics_updated_cloud_fraction"}
        for k, v in res.items():
            st[out_name.get(k, "physics_updated_" + k)][ci, cj, k3] = v
        return self.precip
