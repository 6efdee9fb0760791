"""Physical constants used by the GFDL cloud-microphysics step and its coupling.

pySHiELD takes these from ``ndsl.constants`` (NDSL is a third-party package,
``ndsl @ git+https://github.com/NOAA-GFDL/NDSL.git@main``, no pinned commit,
``setup.py:17``). The symbols used on the microphysics path are imported at
``pySHiELD/stencils/microphysics.py:14`` and
``pySHiELD/functions/microphysics_funcs.py:4``.

NDSL cannot be imported here, so the values below are a choice made by this
project: the GFS constant set that the GFDL microphysics Fortran scheme
(``gfdl_cloud_microphys.F90``) declares, with the derived constants computed
by the same formulas that scheme documents. They are not verified against
NDSL's own module. This one module feeds the oracle, the host code and (as
kernel parameters) the CUDA kernels, so every implementation sees identical
double-precision values.
"""

GRAV = 9.80665  # acceleration due to gravity [m/s^2]
RGRAV = 1.0 / GRAV
RDGAS = 287.05  # gas constant for dry air [J/kg/K]
RVGAS = 461.50  # gas constant for water vapour [J/kg/K]
HLV = 2.5e6  # latent heat of evaporation [J/kg]
HLF = 3.3358e5  # latent heat of fusion [J/kg]
CP_AIR = 1004.6  # heat capacity of dry air at constant pressure
KAPPA = RDGAS / CP_AIR
CP_VAP = 4.0 * RVGAS  # heat capacity of water vapour at constant pressure
CV_AIR = CP_AIR - RDGAS  # heat capacity of dry air at constant volume
CV_VAP = 3.0 * RVGAS  # heat capacity of water vapour at constant volume
C_ICE = 1972.0  # heat capacity of ice at -15 C
C_LIQ = 4.1855e3  # heat capacity of water at 15 C
TICE = 273.16  # freezing temperature
E00 = 611.21  # saturation vapour pressure at 0 C [Pa]
DC_VAP = CP_VAP - C_LIQ  # isobaric heating / cooling
DC_ICE = C_LIQ - C_ICE
D2ICE = DC_VAP + DC_ICE
LV0 = HLV - DC_VAP * TICE  # evaporation latent heat coefficient at 0 K
LI00 = HLF - DC_ICE * TICE  # fusion latent heat coefficient at 0 K
LI2 = LV0 + LI00  # sublimation latent heat coefficient at 0 K
EPS = RDGAS / RVGAS
ZVIR = RVGAS / RDGAS - 1.0
T_MIN = 178.0  # minimum temperature to freeze-dry all water vapour
T_SAT_MIN = TICE - 160.0
LAT2 = (HLV + HLF) ** 2  # used in the ice deposition rate

# Order in which the constants are packed into the kernel parameter block.
# The C header ``include/shield_mp.h`` declares the same order.
PACKED_ORDER = (
    "GRAV", "RGRAV", "RDGAS", "RVGAS", "HLV", "HLF", "CP_AIR", "KAPPA",
    "CP_VAP", "CV_AIR", "CV_VAP", "C_ICE", "C_LIQ", "TICE", "E00", "DC_VAP",
    "DC_ICE", "D2ICE", "LV0", "LI00", "LI2", "EPS", "ZVIR", "T_MIN",
    "T_SAT_MIN", "LAT2",
)


def packed():
    """The constants as a tuple in ``PACKED_ORDER``."""
    g = globals()
    return tuple(float(g[n]) for n in PACKED_ORDER)
