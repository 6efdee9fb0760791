"""Physics-to-dynamics column coupling over the B200 kernels.

* ``update_physics_state_with_tendencies`` -- the stencil of
  ``pySHiELD/stencils/physics.py:151-194`` with the same argument order:
  ``physics_updated_X = X + X_dt * dt`` for the ten prognostic fields.
* ``UpdateAtmosphereState`` -- ``pySHiELD/update/update_atmos_state.py:235-349``:
  ``fill_gfs_delp`` then ``prepare_tendencies_and_update_tracers`` and, with
  ``apply_tendencies``, ``ApplyPhysicsToDycore``'s column stencils
  ``moist_cv`` and ``update_pressure_and_surface_winds``
  (``pySHiELD/update/fv_update_phys.py:152-188``), fused in one kernel.

* ``DycoreToPhysics`` -- ``pySHiELD/update/update_atmos_state.py:145-232``:
  the 16-field copy of the dycore state into the physics state, on the
  compute domain plus one interface point in x and y, levels 0 .. nz - 1.

The horizontal part of ``ApplyPhysicsToDycore`` (the halo exchange of
``u_dt``/``v_dt``, ``AGrid2DGridPhysics`` and ``CubedToLatLon``) needs cubed-
sphere edge geometry and a communicator; it is not part of this package, and
``UpdateAtmosphereState`` leaves ``u_dt``/``v_dt`` (updated by the column
stencils) for the caller's horizontal step.
"""

import ctypes

from . import constants as C
from ._lib import SHIELD_UAS_APPLY, SHIELD_UAS_DYCORE_ONLY, ShieldField3D, check, load
from .microphysics import _current_stream
from .quantity import field3d


def _domain(q):
    ext = tuple(getattr(q, "extent", q.data.shape if hasattr(q, "data") else q.shape))
    return ext


def update_physics_state_with_tendencies(
    qvapor, qliquid, qrain, qice, qsnow, qgraupel, qcld, pt, ua, va,
    qv_dt, ql_dt, qr_dt, qi_dt, qs_dt, qg_dt, qa_dt, pt_dt, udt, vdt,
    physics_updated_specific_humidity, physics_updated_qliquid, physics_updated_qrain, physics_updated_qice,
    physics_updated_qsnow, physics_updated_qgraupel, physics_updated_cloud_fraction, physics_updated_pt,
    physics_updated_ua, physics_updated_va, dt, stream=None,
):
    """Forward-Euler update of the ten prognostic fields on the compute
    domain of ``qvapor`` (its ``extent``)."""
    nx, ny, nz = _domain(qvapor)[:3]
    ext = (nx, ny, nz)
    state = (qvapor, qliquid, qrain, qice, qsnow, qgraupel, qcld, pt, ua, va)
    tend = (qv_dt, ql_dt, qr_dt, qi_dt, qs_dt, qg_dt, qa_dt, pt_dt, udt, vdt)
    out = (
        physics_updated_specific_humidity, physics_updated_qliquid, physics_updated_qrain, physics_updated_qice,
        physics_updated_qsnow, physics_updated_qgraupel, physics_updated_cloud_fraction, physics_updated_pt,
        physics_updated_ua, physics_updated_va,
    )
    arr = ShieldField3D * 10
    s = arr(*[field3d(q, ext) for q in state])
    t = arr(*[field3d(q, ext) for q in tend])
    o = arr(*[field3d(q, ext) for q in out])
    rc = load().shield_update_physics_state(nx, ny, nz, s, t, o, float(dt), ctypes.c_void_p(_current_stream(stream)))
    check(rc, None, "shield_update_physics_state")


class UpdateAtmosphereState:
    """Column part of ``UpdateAtmosphereState`` (update_atmos_state.py:235-349).

    Same constructor arguments as the reference; ``comm``, ``grid_info``,
    ``state``, ``quantity_factory`` and ``tendency_state`` are accepted for
    signature compatibility and only needed by the horizontal step, which
    this class does not run. ``rdt`` for the tendencies is ``1 / dt_atmos``
    (``namelist.dt_atmos``), as in the reference (:262).
    """

    def __init__(
        self, stencil_factory, grid_data, namelist, comm=None, grid_info=None, state=None, quantity_factory=None,
        dycore_only=False, apply_tendencies=True, tendency_state=None,
    ):
        gi = stencil_factory.grid_indexing
        self.nx, self.ny, self.nz = (int(v) for v in gi.domain)
        self.n_halo = int(getattr(gi, "n_halo", 3))
        self.namelist = namelist
        self._rdt = 1.0 / float(namelist.dt_atmos)
        self._dycore_only = bool(dycore_only)
        self._apply_tendencies = bool(apply_tendencies)
        # surface winds of the last call (the reference's ApplyPhysicsToDycore
        # keeps them as private (nx, ny) fields)
        self.u_srf = None
        self.v_srf = None
        load()

    def __call__(self, dycore_state, phy_state, u_dt, v_dt, pt_dt, dt, stream=None, winds=None):
        """The column stencils in one launch; then, with ``apply_tendencies``
        and ``winds`` (a ``DGridWindUpdate``; not in the reference's
        signature, whose ``ApplyPhysicsToDycore`` owns these steps), the halo
        exchange of u_dt / v_dt and the D-grid wind update on
        ``dycore_state.u`` / ``.v``."""
        self._columns(dycore_state, phy_state, u_dt, v_dt, pt_dt, dt, stream)
        if winds is not None and self._apply_tendencies:
            winds(dycore_state.u, dycore_state.v, u_dt, v_dt, stream=stream)

    def _columns(self, dycore_state, phy_state, u_dt, v_dt, pt_dt, dt, stream=None):
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.n_halo
        ext = (nx, ny, nz + 1)
        d, p = dycore_state, phy_state
        fields = (
            u_dt, v_dt, pt_dt, p.physics_updated_ua, p.physics_updated_va, p.physics_updated_pt,
            p.physics_updated_specific_humidity, p.physics_updated_qliquid, p.physics_updated_qrain,
            p.physics_updated_qsnow, p.physics_updated_qice, p.physics_updated_qgraupel, p.ua, p.va, p.pt,
            d.qvapor, d.qliquid, d.qrain, d.qsnow, d.qice, d.qgraupel, p.prsi, d.delp, d.pt, d.pe, d.peln, d.pk,
            d.ua, d.va,
        )
        arr = (ShieldField3D * len(fields))(*[field3d(q, ext) for q in fields])
        # halo reach of fill_gfs_delp: the full domain around the compute domain
        for q in (p.physics_updated_specific_humidity, d.qvapor, d.delp):
            org = tuple(getattr(q, "origin", (0, 0, 0)))
            if org[0] < h or org[1] < h:
                raise ValueError("fill_gfs_delp needs the halo of the full domain on every side")
        mode = 0
        if self._apply_tendencies:
            mode |= SHIELD_UAS_APPLY
        if self._dycore_only:
            mode |= SHIELD_UAS_DYCORE_ONLY
        if self.u_srf is None:
            import torch

            dev = d.ps.data.device
            self.u_srf = torch.zeros((nx, ny), dtype=torch.float64, device=dev)
            self.v_srf = torch.zeros((nx, ny), dtype=torch.float64, device=dev)
        ps = field3d(_as3d(d.ps), (nx, ny, 1))
        us = field3d(_as3d(self.u_srf), (nx, ny, 1))
        vs = field3d(_as3d(self.v_srf), (nx, ny, 1))
        rc = load().shield_update_atmos_state(
            nx, ny, nz, h, mode, arr, ps, us, vs, self._rdt, float(dt), C.KAPPA, C.CP_AIR,
            ctypes.c_void_p(_current_stream(stream)),
        )
        check(rc, None, "shield_update_atmos_state")


class _View3:
    """A 2-D quantity seen as 3-D with one level (the kernels ignore its k)."""

    def __init__(self, q):
        data = q.data
        self.data = data.unsqueeze(-1) if hasattr(data, "unsqueeze") else data[..., None]
        self.origin = tuple(getattr(q, "origin", (0, 0))) + (0,)
        self.extent = tuple(getattr(q, "extent", data.shape)) + (1,)


def _as3d(q):
    return _View3(q)


D2P_FIELDS = ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "qo3mr", "qsgs_tke", "qcld", "pt", "delp",
              "delz", "ua", "va", "w", "omga")


class DycoreToPhysics:
    """``DycoreToPhysics`` (update_atmos_state.py:145-232): same constructor
    and call. The dry convective adjustment (``do_dry_convective_adjust``)
    is pyFV3's ``DryConvectiveAdjustment``, which is not part of this
    package; asking for it raises ``NotImplementedError``."""

    def __init__(self, stencil_factory, quantity_factory, dycore_config, do_dry_convective_adjust, dycore_only):
        if do_dry_convective_adjust:
            raise NotImplementedError("the dry convective adjustment (pyFV3 fv_subgridz) is not part of pyshield_b200")
        gi = stencil_factory.grid_indexing
        self.nx, self.ny, self.nz = (int(v) for v in gi.domain)
        self._dycore_only = bool(dycore_only)
        load()

    def __call__(self, dycore_state, physics_state, tendency_state=None, timestep=None, stream=None):
        if self._dycore_only:
            return
        ext = (self.nx + 1, self.ny + 1, self.nz)
        arr = ShieldField3D * len(D2P_FIELDS)
        src = arr(*[field3d(getattr(dycore_state, f), ext) for f in D2P_FIELDS])
        dst = arr(*[field3d(getattr(physics_state, f), ext) for f in D2P_FIELDS])
        rc = load().shield_copy_dycore_to_physics(self.nx, self.ny, self.nz, src, dst,
                                                  ctypes.c_void_p(_current_stream(stream)))
        check(rc, None, "shield_copy_dycore_to_physics")


class DGridWindUpdate:
    """The horizontal half of ``ApplyPhysicsToDycore`` that follows its column
    stencils (fv_update_phys.py:134-147, 173-195): the one-point halo
    exchange of ``u_dt`` and ``v_dt`` with the neighbouring ranks
    (``halo.HaloExchange`` over the edge ``table``; this rank is ``rank``),
    then ``AGrid2DGridPhysics`` (``agrid_to_dgrid``). ``CubedToLatLon``,
    which the reference runs next, is NDSL's and stays with the caller.

    The reference starts the exchange before ``update_pressure_and_surface_
    winds`` and waits after it; here that stencil runs inside
    ``UpdateAtmosphereState``'s single column launch, which also produces
    the tendencies, so the exchange starts after that launch."""

    def __init__(self, agrid_to_dgrid, table, rank, group=None):
        from .halo import check_table

        check_table(table)
        self.agrid_to_dgrid = agrid_to_dgrid
        self.table = table
        self.rank = rank
        self.group = group

    def __call__(self, u, v, u_dt, v_dt, stream=None):
        from .halo import HaloExchange

        ex = HaloExchange([u_dt, v_dt], self.table, self.rank, self.group)
        ex.start()
        ex.wait()
        self.agrid_to_dgrid(u, v, u_dt, v_dt, stream=stream)
