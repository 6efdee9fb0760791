"""``Physics`` and ``PhysicsState``: pySHiELD's physics driver over the B200
kernels.

Mirrors ``pySHiELD/stencils/physics.py:197-366`` and
``pySHiELD/physics_state.py:17-330``:

* ``PhysicsState`` has the reference's fields, in the reference's order,
  and builds ``.microphysics`` (a ``MicrophysicsState`` sharing its
  quantities, with its own zeroed tendency fields) when
  ``GFS_microphysics`` is among the schemes.
* ``Physics(stencil_factory, quantity_factory, grid_data, namelist)`` and
  ``__call__(physics_state, timestep)`` run, in the reference's order:
  ``atmos_phys_driver_statein`` (compute domain, nz + 1 levels),
  ``get_prs_fv3`` and ``get_phi_fv3`` (full domain, nz + 1 levels),
  ``prepare_microphysics``, the microphysics step and
  ``update_physics_state_with_tendencies``. The first four are one fused
  kernel (``shield_physics_prestep``); the microphysics and the update are
  the kernels behind ``Microphysics`` and
  ``update_physics_state_with_tendencies``.

Differences: fields are float64 CUDA arrays (see ``quantity``), the work
runs on the current torch stream (or the ``stream`` passed), and
``Physics`` takes the microphysics ``precision`` ("plain" FP64 or
"mixed").
"""

import ctypes
import dataclasses
from dataclasses import InitVar
from typing import Any, List

from . import _lib
from . import constants as C
from ._config import PHYSICS_PACKAGES
from ._lib import SHIELD_PHYS_PREPARE_MICROPHYSICS, ShieldPhysicsFields, check, load
from .coupling import update_physics_state_with_tendencies
from .grid import X_DIM, Y_DIM, Z_DIM, Z_INTERFACE_DIM
from .microphysics import Microphysics, MicrophysicsState, _current_stream
from .quantity import field3d

_INTERFACE = ("phii", "prsi", "prsik")


@dataclasses.dataclass
class PhysicsState:
    """pySHiELD's ``PhysicsState`` (physics_state.py:17-330): the same fields
    in the same order; ``phii``, ``prsi`` and ``prsik`` are interface (nz + 1
    level) fields, ``land`` is 2-D."""

    qvapor: Any
    qliquid: Any
    qice: Any
    qrain: Any
    qsnow: Any
    qgraupel: Any
    qo3mr: Any
    qsgs_tke: Any
    qcld: Any
    pt: Any
    delp: Any
    delz: Any
    ua: Any
    va: Any
    w: Any
    omga: Any
    physics_updated_specific_humidity: Any
    physics_updated_qliquid: Any
    physics_updated_qice: Any
    physics_updated_qrain: Any
    physics_updated_qsnow: Any
    physics_updated_qgraupel: Any
    physics_updated_cloud_fraction: Any
    physics_updated_pt: Any
    physics_updated_ua: Any
    physics_updated_va: Any
    delprsi: Any
    phii: Any
    phil: Any
    dz: Any
    wmp: Any
    prsi: Any
    prsik: Any
    land: Any
    quantity_factory: InitVar[Any]
    schemes: InitVar[List]

    def __post_init__(self, quantity_factory, schemes):
        if "GFS_microphysics" in [getattr(s, "value", s) for s in schemes]:
            tendency = quantity_factory.zeros([X_DIM, Y_DIM, Z_DIM], "unknown")
            self.microphysics = MicrophysicsState(
                pt=self.pt, qvapor=self.qvapor, qliquid=self.qliquid, qrain=self.qrain, qice=self.qice,
                qsnow=self.qsnow, qgraupel=self.qgraupel, qcld=self.qcld, ua=self.ua, va=self.va, delp=self.delp,
                delz=self.delz, omga=self.omga, delprsi=self.delprsi, wmp=self.wmp, dz=self.dz, tendency=tendency,
                land=self.land,
            )
        else:
            self.microphysics = None

    @classmethod
    def init_zeros(cls, quantity_factory, schemes):
        """Every field zero, allocated by ``quantity_factory`` (physics_state.py:327-343)."""
        arrays = {}
        for f in dataclasses.fields(cls):
            if f.name == "land":
                arrays[f.name] = quantity_factory.zeros([X_DIM, Y_DIM], "")
            else:
                dims = [X_DIM, Y_DIM, Z_INTERFACE_DIM if f.name in _INTERFACE else Z_DIM]
                arrays[f.name] = quantity_factory.zeros(dims, "")
        return cls(**arrays, quantity_factory=quantity_factory, schemes=schemes)


class Physics:
    """pySHiELD's ``Physics`` (physics.py:197-366) on the GPU."""

    def __init__(self, stencil_factory, quantity_factory, grid_data, namelist, precision="plain"):
        schemes = [getattr(s, "value", s) for s in namelist.schemes]
        for scheme in schemes:
            if scheme not in PHYSICS_PACKAGES:
                raise NotImplementedError(f"{scheme} is not an implemented physics parameterization")
        gi = stencil_factory.grid_indexing
        self.nx, self.ny, self.nz = (int(v) for v in gi.domain)
        self.n_halo = int(getattr(gi, "n_halo", 3))
        self._setup_statein()
        self._ptop = float(grid_data.ptop)
        # the statein externals (physics.py:219-221); the library computes
        # the same two values from ptop
        self._pktop = (self._ptop / self._p00) ** C.KAPPA
        self._pk0inv = (1.0 / self._p00) ** C.KAPPA
        self._prsik = quantity_factory.zeros([X_DIM, Y_DIM, Z_DIM], "unknown")
        self._dm3d = quantity_factory.zeros([X_DIM, Y_DIM, Z_DIM], "unknown")
        self._del_gz = quantity_factory.zeros([X_DIM, Y_DIM, Z_DIM], "unknown")
        self._gfs_microphysics = "GFS_microphysics" in schemes
        if self._gfs_microphysics:
            self._microphysics = Microphysics(stencil_factory, quantity_factory, grid_data, namelist,
                                              precision=precision)
        self._fields = ShieldPhysicsFields()
        self._key = None
        load()

    def _setup_statein(self):
        self._NQ = 8
        self._dnats = 1
        self._nwat = 6
        self._p00 = 1.0e5

    def _build_fields(self, ps):
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.n_halo
        ext = (nx, ny, nz + 1)
        F = self._fields
        mp = ps.microphysics
        src = {
            "prsik": self._prsik, "dm": self._dm3d, "del_gz": self._del_gz,
        }
        for name in _lib.PHYS_FIELDS:
            if name in src:
                q = src[name]
            elif name in _lib.MP_TENDENCY_FIELDS:
                if mp is None:
                    setattr(F, name, _lib.ShieldField3D())
                    continue
                q = getattr(mp, name)
            elif name in ("omga", "dz", "wmp") and not self._gfs_microphysics:
                setattr(F, name, _lib.ShieldField3D())
                continue
            else:
                q = getattr(ps, name)
            if name in ("phii", "prsi", "delprsi", "del_gz", "phil", "pt", "qvapor"):
                # read or written on the full domain by get_prs_fv3 / get_phi_fv3
                org = tuple(getattr(q, "origin", (0, 0, 0)))
                if org[0] < h or org[1] < h:
                    raise ValueError(f"{name}: get_prs_fv3/get_phi_fv3 need the halo of the full domain")
            setattr(F, name, field3d(q, ext))
        return F

    def prestep(self, physics_state, stream=None):
        """The driver steps before the microphysics (physics.py:277-330):
        statein, get_prs_fv3, get_phi_fv3 and, with GFS_microphysics,
        prepare_microphysics, as one kernel launch."""
        ps = physics_state
        key = tuple(id(getattr(ps, f.name).data) for f in dataclasses.fields(ps))
        if ps.microphysics is not None:
            key += tuple(id(getattr(ps.microphysics, t).data) for t in _lib.MP_TENDENCY_FIELDS)
        if key != self._key:
            self._build_fields(ps)
            self._key = key
        flags = SHIELD_PHYS_PREPARE_MICROPHYSICS if self._gfs_microphysics else 0
        rc = load().shield_physics_prestep(self.nx, self.ny, self.nz, self.n_halo, self._nwat, self._ptop, flags,
                                           ctypes.byref(self._fields), ctypes.c_void_p(_current_stream(stream)))
        check(rc, None, "shield_physics_prestep")

    def __call__(self, physics_state, timestep, stream=None):
        ps = physics_state
        self.prestep(ps, stream)
        if self._gfs_microphysics:
            m = ps.microphysics
            self._microphysics(m, timestep, stream=stream)
            update_physics_state_with_tendencies(
                ps.qvapor, ps.qliquid, ps.qrain, ps.qice, ps.qsnow, ps.qgraupel, ps.qcld, ps.pt, ps.ua, ps.va,
                m.qv_dt, m.ql_dt, m.qr_dt, m.qi_dt, m.qs_dt, m.qg_dt, m.qa_dt, m.pt_dt, m.udt, m.vdt,
                ps.physics_updated_specific_humidity, ps.physics_updated_qliquid, ps.physics_updated_qrain,
                ps.physics_updated_qice, ps.physics_updated_qsnow, ps.physics_updated_qgraupel,
                ps.physics_updated_cloud_fraction, ps.physics_updated_pt, ps.physics_updated_ua,
                ps.physics_updated_va, timestep, stream=stream,
            )
