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

import numpy as np
from dataclasses import InitVar
from typing import Any, List

from . import _lib
from . import constants as C
from ._config import PHYSICS_PACKAGES
from ._lib import SHIELD_PHYS_PREPARE_MICROPHYSICS, ShieldPhysicsFields, check, load
from .coupling import D2P_FIELDS, update_physics_state_with_tendencies
from .grid import X_DIM, Y_DIM, Z_DIM, Z_INTERFACE_DIM
from .microphysics import Microphysics, MicrophysicsState, _current_stream
from .quantity import Quantity, field3d

_XYZ = [X_DIM, Y_DIM, Z_DIM]
_XYZI = [X_DIM, Y_DIM, Z_INTERFACE_DIM]
_XY = [X_DIM, Y_DIM]


def _field(name, dims, units):
    """A state field with the reference's metadata (physics_state.py:17-288)."""
    return dataclasses.field(metadata={"name": name, "dims": list(dims), "units": units})


@dataclasses.dataclass
class PhysicsState:
    """pySHiELD's ``PhysicsState`` (physics_state.py:17-330): the same fields
    in the same order, each with the reference's metadata (long name, dims,
    units); ``phii``, ``prsi`` and ``prsik`` are interface (nz + 1 level)
    fields, ``land`` is 2-D."""

    qvapor: Any = _field("specific_humidity", _XYZ, "kg/kg")
    qliquid: Any = _field("cloud_water_mixing_ratio", _XYZ, "kg/kg")
    qice: Any = _field("cloud_ice_mixing_ratio", _XYZ, "kg/kg")
    qrain: Any = _field("rain_mixing_ratio", _XYZ, "kg/kg")
    qsnow: Any = _field("snow_mixing_ratio", _XYZ, "kg/kg")
    qgraupel: Any = _field("graupel_mixing_ratio", _XYZ, "kg/kg")
    qo3mr: Any = _field("ozone_mixing_ratio", _XYZ, "kg/kg")
    qsgs_tke: Any = _field("turbulent_kinetic_energy", _XYZ, "m**2/s**2")
    qcld: Any = _field("cloud_fraction", _XYZ, "")
    pt: Any = _field("air_temperature", _XYZ, "degK")
    delp: Any = _field("pressure_thickness_of_atmospheric_layer", _XYZ, "Pa")
    delz: Any = _field("vertical_thickness_of_atmospheric_layer", _XYZ, "m")
    ua: Any = _field("eastward_wind", _XYZ, "m/s")
    va: Any = _field("northward_wind", _XYZ, "m/s")
    w: Any = _field("vertical_wind", _XYZ, "m/s")
    omga: Any = _field("vertical_pressure_velocity", _XYZ, "Pa/s")
    physics_updated_specific_humidity: Any = _field("physics_updated_specific_humidity", _XYZ, "kg/kg")
    physics_updated_qliquid: Any = _field("physics_updated_liquid_water_mixing_ratio", _XYZ, "kg/kg")
    physics_updated_qice: Any = _field("physics_updated_ice_water_mixing_ratio", _XYZ, "kg/kg")
    physics_updated_qrain: Any = _field("physics_updated_rain_water_mixing_ratio", _XYZ, "kg/kg")
    physics_updated_qsnow: Any = _field("physics_updated_snow_mixing_ratio", _XYZ, "kg/kg")
    physics_updated_qgraupel: Any = _field("physics_updated_graupel_mixing_ratio", _XYZ, "kg/kg")
    physics_updated_cloud_fraction: Any = _field("physics_cloud_fraction", _XYZ, "")
    physics_updated_pt: Any = _field("physics_air_temperature", _XYZ, "degK")
    physics_updated_ua: Any = _field("physics_eastward_wind", _XYZ, "m/s")
    physics_updated_va: Any = _field("physics_northward_wind", _XYZ, "m/s")
    delprsi: Any = _field("model_level_pressure_thickness_in_physics", _XYZ, "Pa")
    phii: Any = _field("interface_geopotential_height", _XYZI, "m")
    phil: Any = _field("layer_geopotential_height", _XYZ, "m")
    dz: Any = _field("geopotential_height_thickness", _XYZ, "m")
    wmp: Any = _field("layer_mean_vertical_velocity_microph", _XYZ, "m/s")
    prsi: Any = _field("interface_pressure", _XYZI, "Pa")
    prsik: Any = _field("log_interface_pressure", _XYZI, "Pa")
    land: Any = _field("land_mask", _XY, "-")
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
        arrays = {f.name: quantity_factory.zeros(f.metadata["dims"], f.metadata["units"]) for f in cls._state_fields()}
        return cls(**arrays, quantity_factory=quantity_factory, schemes=schemes)

    @classmethod
    def init_from_storages(cls, storages, sizer, quantity_factory, schemes):
        """Wrap existing storages (physics_state.py:344-364): ``storages[name]``
        is each field's full array; its compute domain is
        ``sizer.get_origin(dims)`` / ``sizer.get_extent(dims)``. The arrays
        are used in place, not copied."""
        inputs = {}
        for f in cls._state_fields():
            dims = f.metadata["dims"]
            inputs[f.name] = Quantity(storages[f.name], dims, f.metadata["units"], origin=sizer.get_origin(dims),
                                      extent=sizer.get_extent(dims))
        return cls(**inputs, quantity_factory=quantity_factory, schemes=schemes)

    @classmethod
    def _state_fields(cls):
        return [f for f in dataclasses.fields(cls) if "dims" in f.metadata]

    @property
    def xr_dataset(self):
        """The state as a dataset (physics_state.py:366-383): one variable per
        field holding its full storage, with dims ``f"{dim}_{name}"`` and
        attrs ``long_name`` and ``units``. An ``xarray.Dataset`` when xarray
        is importable; otherwise a ``StateDataset`` with the same variables,
        dims and attrs (host numpy copies of the storages)."""
        data_vars = {}
        for f in self._state_fields():
            data = getattr(self, f.name).data
            if hasattr(data, "detach"):
                data = data.detach().cpu().numpy()
            data_vars[f.name] = StateVariable(
                np.asarray(data), [f"{d}_{f.name}" for d in f.metadata["dims"]],
                {"long_name": f.metadata["name"], "units": f.metadata.get("units", "unknown")},
            )
        try:
            import xarray as xr
        except ImportError:
            return StateDataset(data_vars)
        return xr.Dataset(
            data_vars={n: xr.DataArray(v.values, dims=v.dims, attrs=v.attrs) for n, v in data_vars.items()})


class StateVariable:
    """One variable of ``PhysicsState.xr_dataset`` without xarray: ``values``
    (numpy), ``dims`` (names, one per axis) and ``attrs``."""

    def __init__(self, values, dims, attrs):
        if len(dims) != values.ndim:
            raise ValueError(f"{len(dims)} dims for a {values.ndim}-D array")
        self.values, self.dims, self.attrs = values, tuple(dims), dict(attrs)

    @property
    def sizes(self):
        return dict(zip(self.dims, self.values.shape))


class StateDataset:
    """``PhysicsState.xr_dataset`` without xarray: ``data_vars`` maps each
    field's name to its ``StateVariable``; ``ds[name]`` and ``ds.dims`` work
    as in xarray."""

    def __init__(self, data_vars):
        self.data_vars = dict(data_vars)

    def __getitem__(self, name):
        return self.data_vars[name]

    def __contains__(self, name):
        return name in self.data_vars

    def __iter__(self):
        return iter(self.data_vars)

    @property
    def dims(self):
        out = {}
        for v in self.data_vars.values():
            out.update(v.sizes)
        return out


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

    def prestep(self, physics_state, stream=None, dycore_state=None):
        """The driver steps before the microphysics (physics.py:277-330):
        statein, get_prs_fv3, get_phi_fv3 and, with GFS_microphysics,
        prepare_microphysics, as one kernel launch. With ``dycore_state``,
        the same launch first does ``DycoreToPhysics``' copy of its 16
        fields into ``physics_state`` (update_atmos_state.py:196-232): the
        pre-step reads the dycore storages and writes each copied field
        once, with the results of the copy followed by the pre-step."""
        ps = physics_state
        # rebuilt on every call from the storages themselves (see
        # Microphysics.__call__), never cached by object identity
        self._build_fields(ps)
        flags = SHIELD_PHYS_PREPARE_MICROPHYSICS if self._gfs_microphysics else 0
        st = ctypes.c_void_p(_current_stream(stream))
        if dycore_state is None:
            rc = load().shield_physics_prestep(self.nx, self.ny, self.nz, self.n_halo, self._nwat, self._ptop, flags,
                                               ctypes.byref(self._fields), st)
            check(rc, None, "shield_physics_prestep")
            return
        ext = (self.nx + 1, self.ny + 1, self.nz)
        arr = _lib.ShieldField3D * len(D2P_FIELDS)
        src = arr(*[field3d(getattr(dycore_state, f), ext) for f in D2P_FIELDS])
        dst = arr(*[field3d(getattr(ps, f), ext) for f in D2P_FIELDS])
        rc = load().shield_physics_prestep_from_dycore(self.nx, self.ny, self.nz, self.n_halo, self._nwat, self._ptop,
                                                       flags, ctypes.byref(self._fields), src, dst, st)
        check(rc, None, "shield_physics_prestep_from_dycore")

    def __call__(self, physics_state, timestep, stream=None, dycore_state=None):
        """``Physics.__call__`` (physics.py:276-366). ``dycore_state``
        (optional, not in the reference's signature): run
        ``DycoreToPhysics``' copy from it inside the pre-step launch, in
        place of a separate ``DycoreToPhysics.__call__`` before this call
        (same results; measured slower at C96 L79 than the separate copy,
        whose launch runs near the HBM bandwidth)."""
        ps = physics_state
        self.prestep(ps, stream, dycore_state)
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
