"""Physics configuration: the field names and meaning of ``pySHiELD/_config.py``.

``PhysicsConfig`` keeps every field of the reference dataclass
(``pySHiELD/_config.py:22-109``) with the same name, type and meaning, so a
caller's config object carries over unchanged. The reference takes its
defaults from ``ndsl.namelist.NamelistDefaults``, which cannot be imported
here; the defaults below are this project's explicit choice (the GFDL
microphysics namelist values of the C12 test cases that the pace/NDSL
defaults were drawn from, as far as they are known here). They are not
verified against NDSL. Every value is also written out in the C-ABI's
``ShieldMpConfig`` by ``to_c_config``.

Differences from the reference, all deliberate:

* ``from_f90nml`` / ``namelist_override`` need ``f90nml``, which is absent;
  ``from_namelist`` accepts any object with the same attribute names.
* ``schemes`` accepts strings or ``PHYSICS_PACKAGES`` members, and an unknown
  scheme raises ``NotImplementedError`` as in ``_config.py:111-119``.
"""

import dataclasses
from enum import Enum, unique
from typing import List, Optional, Tuple

DEFAULT_INT = 0
DEFAULT_BOOL = False
DEFAULT_SCHEMES = ["GFS_microphysics"]


class _MetaEnumStr(type(Enum)):
    """``"name" in Enum`` membership by value string, like ``ndsl.utils.MetaEnumStr``."""

    def __contains__(cls, item):
        if isinstance(item, cls):
            return True
        return item in {m.value for m in cls}


@unique
class PHYSICS_PACKAGES(Enum, metaclass=_MetaEnumStr):
    GFS_microphysics = "GFS_microphysics"


@dataclasses.dataclass
class PhysicsConfig:
    dt_atmos: int = DEFAULT_INT
    hydrostatic: bool = DEFAULT_BOOL
    npx: int = DEFAULT_INT
    npy: int = DEFAULT_INT
    npz: int = DEFAULT_INT
    nwat: int = DEFAULT_INT
    schemes: List = None
    do_qa: bool = DEFAULT_BOOL
    c_cracw: float = 0.8
    c_paut: float = 0.5
    c_pgacs: float = 0.01
    c_psaci: float = 0.05
    ccn_l: float = 300.0
    ccn_o: float = 100.0
    const_vg: bool = False
    const_vi: bool = False
    const_vr: bool = False
    const_vs: bool = False
    vs_fac: float = 1.0
    vg_fac: float = 1.0
    vi_fac: float = 1.0
    vr_fac: float = 1.0
    de_ice: bool = False
    layout: Tuple[int, int] = (1, 1)
    tau_imlt: float = 600.0  # cloud ice melting
    tau_i2s: float = 1000.0  # cloud ice to snow auto-conversion
    tau_g2v: float = 900.0  # graupel sublimation
    tau_v2g: float = 21600.0  # graupel deposition -- a slow process
    ql_mlt: float = 2.0e-3  # max cloud water allowed from melted cloud ice
    qs_mlt: float = 1.0e-6  # max cloud water due to snow melt
    t_sub: float = 184.0  # min temperature for sublimation of cloud ice
    qi_gen: float = 1.82e-6  # max cloud ice generation
    qi_lim: float = 1.0  # cloud ice limiter
    qi0_max: float = 1.0e-4  # max cloud ice value (by other sources)
    rad_snow: bool = True  # snow in the cloud fraction
    rad_rain: bool = True  # rain in the cloud fraction
    dw_ocean: float = 0.10  # base subgrid variability over ocean
    dw_land: float = 0.15  # base subgrid variability over land
    tau_l2v: float = 300.0  # cloud water to water vapour (evaporation)
    c2l_ord: int = 4
    do_sedi_heat: bool = False
    do_sedi_w: bool = True
    fast_sat_adj: bool = True
    qc_crt: float = 5.0e-8
    fix_negative: bool = True
    irain_f: int = 0
    mp_time: float = 150.0
    prog_ccn: bool = False
    qi0_crt: float = 8.0e-5
    qs0_crt: float = 3.0e-3
    rh_inc: float = 0.2
    rh_inr: float = 0.3
    rthresh: float = 1.0e-5
    sedi_transport: bool = True
    use_ppm: bool = False
    vg_max: float = 12.0
    vi_max: float = 1.0
    vr_max: float = 12.0
    vs_max: float = 2.0
    z_slope_ice: bool = True
    z_slope_liq: bool = True
    tice: float = 273.16
    alin: float = 842.0
    clin: float = 4.8
    namelist_override: Optional[str] = None

    def __post_init__(self):
        if self.schemes is None:
            self.schemes = DEFAULT_SCHEMES
        package_schemes = []
        for scheme in self.schemes:
            if isinstance(scheme, PHYSICS_PACKAGES):
                package_schemes.append(scheme)
                continue
            if scheme not in PHYSICS_PACKAGES:
                raise NotImplementedError(f"{scheme} physics scheme not implemented")
            package_schemes.append(PHYSICS_PACKAGES[scheme])
        self.schemes = package_schemes
        if self.namelist_override is not None:
            raise NotImplementedError(
                "namelist_override needs f90nml, which this build does not ship; "
                "build the config with from_namelist() instead"
            )

    @classmethod
    def from_namelist(cls, namelist) -> "PhysicsConfig":
        """Copy every field that ``namelist`` carries (``_config.py:135-200``)."""
        kwargs = {}
        for f in dataclasses.fields(cls):
            if f.name in ("schemes", "namelist_override"):
                continue
            if hasattr(namelist, f.name):
                kwargs[f.name] = getattr(namelist, f.name)
        return cls(**kwargs)

    def replace(self, **changes) -> "PhysicsConfig":
        return dataclasses.replace(self, **changes)
