"""``Microphysics`` and ``MicrophysicsState``: the reference's call signatures
over the B200 kernels.

Mirrors ``pySHiELD/stencils/microphysics.py:1556-2263``:

* ``MicrophysicsState(pt, qvapor, ..., tendency, land)`` keeps the same
  attribute names; the ten tendencies are independent copies of
  ``tendency`` (deep copies in the reference, :1607-1616).
* ``Microphysics(stencil_factory, quantity_factory, grid_data, namelist)``
  reads the domain from ``stencil_factory.grid_indexing.domain`` and the cell
  area from ``grid_data.area``; ``__call__(state, timestep)`` accumulates the
  tendencies in place (and updates ``wmp``, plus ``qice``/``qsnow`` with
  ``de_ice``), exactly like the reference.

What differs: every field must be a float64 CUDA array (torch tensor or any
``__cuda_array_interface__`` object) and the work runs on the current torch
stream (or the ``stream`` passed). The surface precipitation of the last
step, which the reference keeps in private 3-D fields, is available as the
(nx, ny) arrays ``rain``, ``snow``, ``ice`` and ``graupel`` (mm/day).
"""

import copy
import ctypes

from . import _lib
from ._lib import SHIELD_MP_MIXED, SHIELD_MP_PLAIN, ShieldMpFields, check, load, make_config
from .quantity import field2d, field3d

_PRECISION = {"plain": SHIELD_MP_PLAIN, "fp64": SHIELD_MP_PLAIN, "mixed": SHIELD_MP_MIXED}


def _clone(q):
    data = q.data.clone() if hasattr(q.data, "clone") else copy.deepcopy(q.data)
    out = copy.copy(q)
    out.data = data
    return out


class MicrophysicsState:
    """Same constructor and attributes as the reference (:1556-1620)."""

    def __init__(
        self, pt, qvapor, qliquid, qrain, qice, qsnow, qgraupel, qcld, ua, va, delp, delz, omga, delprsi, wmp, dz,
        tendency, land,
    ):
        self.pt = pt
        self.qvapor = qvapor
        self.qliquid = qliquid
        self.qrain = qrain
        self.qice = qice
        self.qsnow = qsnow
        self.qgraupel = qgraupel
        self.qcld = qcld
        self.ua = ua
        self.va = va
        self.delp = delp
        self.delz = delz
        self.omga = omga
        self.qv_dt = _clone(tendency)
        self.ql_dt = _clone(tendency)
        self.qr_dt = _clone(tendency)
        self.qi_dt = _clone(tendency)
        self.qs_dt = _clone(tendency)
        self.qg_dt = _clone(tendency)
        self.qa_dt = _clone(tendency)
        self.udt = _clone(tendency)
        self.vdt = _clone(tendency)
        self.pt_dt = _clone(tendency)
        self.delprsi = delprsi
        self.wmp = wmp
        self.dz = dz
        self.land = land


def _current_stream(stream):
    if stream is not None:
        return int(getattr(stream, "cuda_stream", stream))
    import torch

    return torch.cuda.current_stream().cuda_stream


class Microphysics:
    """GFDL cloud microphysics on the GPU (reference :1623-2263)."""

    def __init__(self, stencil_factory, quantity_factory, grid_data, namelist, precision="plain"):
        import torch

        self.namelist = namelist
        nx, ny, nz = stencil_factory.grid_indexing.domain
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        self.precision = precision
        lib = load()
        if not torch.cuda.is_available():
            raise _lib.ShieldError("no CUDA device: the microphysics step has no CPU fallback")
        self._area = grid_data.area
        self._cfg = make_config(namelist)
        h = ctypes.c_void_p()
        check(
            lib.shield_mp_create(ctypes.byref(self._cfg), self.nx, self.ny, self.nz, field2d(self._area, (self.nx, self.ny)), ctypes.byref(h)),
            None,
            "shield_mp_create",
        )
        self._handle = h
        dev = torch.device("cuda", torch.cuda.current_device())
        self._precip = torch.zeros((4, self.ny, self.nx), dtype=torch.float64, device=dev)
        self._fields = ShieldMpFields()

    # surface precipitation of the last call, (nx, ny) views, mm/day
    @property
    def rain(self):
        return self._precip[0].t()

    @property
    def snow(self):
        return self._precip[1].t()

    @property
    def ice(self):
        return self._precip[2].t()

    @property
    def graupel(self):
        return self._precip[3].t()

    def _build_fields(self, state):
        F = self._fields
        ext3 = (self.nx, self.ny, self.nz)
        for name in _lib.MP_STATE_FIELDS + _lib.MP_TENDENCY_FIELDS:
            setattr(F, name, field3d(getattr(state, name), ext3))
        F.land = field2d(state.land, (self.nx, self.ny))
        base = self._precip.data_ptr()
        plane = self.nx * self.ny * 8
        F.rain, F.snow, F.ice, F.graupel = base, base + plane, base + 2 * plane, base + 3 * plane
        return F

    def __call__(self, state, timestep, stream=None):
        # the field table (pointer at the domain origin and element strides
        # of every storage) is rebuilt from the storages on every call, so a
        # state whose arrays were freed and reallocated is never stepped
        # through stale pointers
        self._build_fields(state)
        lib = load()
        rc = lib.shield_mp_step(
            self._handle, ctypes.byref(self._fields), float(timestep), _PRECISION[self.precision], ctypes.c_void_p(_current_stream(stream))
        )
        check(rc, self._handle, "shield_mp_step")

    def step_with_flags(self, state, timestep, stream=None):
        """``__call__`` (plain FP64 form) that also returns the step's column
        branch flags: an int32 tensor (ntimes, ny, nx) whose bits are the
        reference's column-wide decisions in each sub-step -- bit 0/1 rain
        falls in the first/second warm_rain pass, bit 2/3/4 ice/snow/graupel
        fall (no_fall == 0), bits 16-23 the melting level (the first level
        with stop_k == 1). See ``flag_fields`` to unpack them."""
        import torch

        self._build_fields(state)
        lib = load()
        nt = check(lib.shield_mp_substeps(self._handle, float(timestep)), self._handle, "shield_mp_substeps")
        flags = torch.empty((nt, self.ny, self.nx), dtype=torch.int32, device=self._precip.device)
        rc = lib.shield_mp_step_flags(self._handle, ctypes.byref(self._fields), float(timestep),
                                      ctypes.c_void_p(flags.data_ptr()), flags.numel(),
                                      ctypes.c_void_p(_current_stream(stream)))
        check(rc, self._handle, "shield_mp_step_flags")
        return flags

    def check(self, stream=None):
        """Wait for the steps queued so far and raise ``ShieldError`` naming
        the column if one of them produced a NaN or an infinity (the kernel
        records the first such column; the record is cleared here). Returns
        -1 when every step was clean."""
        bad = ctypes.c_int64(-1)
        rc = load().shield_mp_check(self._handle, ctypes.byref(bad), ctypes.c_void_p(_current_stream(stream)))
        check(rc, self._handle, "microphysics step")
        return bad.value

    # persistent cloud-fraction accumulator (the reference's self._qaz)
    def get_qaz(self):
        import torch

        out = torch.empty((self.nz, self.ny, self.nx), dtype=torch.float64, device=self._precip.device)
        check(load().shield_mp_get_qaz(self._handle, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(_current_stream(None))), self._handle)
        return out

    def set_qaz(self, qaz):
        check(load().shield_mp_set_qaz(self._handle, ctypes.c_void_p(qaz.contiguous().data_ptr()), ctypes.c_void_p(_current_stream(None))), self._handle)

    def constants(self, timestep):
        buf = (ctypes.c_double * 512)()
        n = check(load().shield_mp_constants(self._handle, float(timestep), buf, 512), self._handle)
        return list(buf[:n])

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                load().shield_mp_destroy(h)
            except Exception:
                pass
            self._handle = None


def flag_fields(flags):
    """Unpack ``Microphysics.step_with_flags`` words into named arrays of
    the same shape: rain_falls_1, rain_falls_2, ice_falls, snow_falls,
    graupel_falls (0/1) and melt_level (level index)."""
    return {
        "rain_falls_1": flags & 1,
        "rain_falls_2": (flags >> 1) & 1,
        "ice_falls": (flags >> 2) & 1,
        "snow_falls": (flags >> 3) & 1,
        "graupel_falls": (flags >> 4) & 1,
        "melt_level": (flags >> 16) & 255,
    }
