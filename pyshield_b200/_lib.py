"""ctypes binding of libshield_mp.so (the C-ABI in include/shield_mp.h).

The library is built in place by ``pyshield_b200.build``; loading fails
loudly when it is missing. There is no CPU fallback.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SHIELD_MP_LIB") or os.path.join(HERE, "libshield_mp.so")

SHIELD_OK = 0
SHIELD_MP_PLAIN = 0
SHIELD_MP_MIXED = 1
SHIELD_UAS_APPLY = 1
SHIELD_UAS_DYCORE_ONLY = 2


class ShieldField3D(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("si", ctypes.c_int64), ("sj", ctypes.c_int64), ("sk", ctypes.c_int64)]


class ShieldField2D(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("si", ctypes.c_int64), ("sj", ctypes.c_int64)]


_CFG_FIELDS = [
    ("dt_atmos", ctypes.c_double),
    ("hydrostatic", ctypes.c_int),
    ("do_qa", ctypes.c_int),
    ("c_cracw", ctypes.c_double),
    ("c_paut", ctypes.c_double),
    ("c_pgacs", ctypes.c_double),
    ("c_psaci", ctypes.c_double),
    ("ccn_l", ctypes.c_double),
    ("ccn_o", ctypes.c_double),
    ("const_vg", ctypes.c_int),
    ("const_vi", ctypes.c_int),
    ("const_vr", ctypes.c_int),
    ("const_vs", ctypes.c_int),
    ("vs_fac", ctypes.c_double),
    ("vg_fac", ctypes.c_double),
    ("vi_fac", ctypes.c_double),
    ("vr_fac", ctypes.c_double),
    ("de_ice", ctypes.c_int),
    ("tau_imlt", ctypes.c_double),
    ("tau_i2s", ctypes.c_double),
    ("tau_g2v", ctypes.c_double),
    ("tau_v2g", ctypes.c_double),
    ("ql_mlt", ctypes.c_double),
    ("qs_mlt", ctypes.c_double),
    ("t_sub", ctypes.c_double),
    ("qi_gen", ctypes.c_double),
    ("qi_lim", ctypes.c_double),
    ("qi0_max", ctypes.c_double),
    ("rad_snow", ctypes.c_int),
    ("rad_rain", ctypes.c_int),
    ("dw_ocean", ctypes.c_double),
    ("dw_land", ctypes.c_double),
    ("tau_l2v", ctypes.c_double),
    ("do_sedi_heat", ctypes.c_int),
    ("do_sedi_w", ctypes.c_int),
    ("fast_sat_adj", ctypes.c_int),
    ("qc_crt", ctypes.c_double),
    ("fix_negative", ctypes.c_int),
    ("irain_f", ctypes.c_int),
    ("mp_time", ctypes.c_double),
    ("prog_ccn", ctypes.c_int),
    ("qi0_crt", ctypes.c_double),
    ("qs0_crt", ctypes.c_double),
    ("rh_inc", ctypes.c_double),
    ("rh_inr", ctypes.c_double),
    ("rthresh", ctypes.c_double),
    ("sedi_transport", ctypes.c_int),
    ("use_ppm", ctypes.c_int),
    ("vg_max", ctypes.c_double),
    ("vi_max", ctypes.c_double),
    ("vr_max", ctypes.c_double),
    ("vs_max", ctypes.c_double),
    ("z_slope_ice", ctypes.c_int),
    ("z_slope_liq", ctypes.c_int),
    ("tice", ctypes.c_double),
    ("alin", ctypes.c_double),
    ("clin", ctypes.c_double),
]


class ShieldMpConfig(ctypes.Structure):
    _fields_ = _CFG_FIELDS


MP_STATE_FIELDS = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi", "delz", "wmp")
MP_TENDENCY_FIELDS = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")


class ShieldMpFields(ctypes.Structure):
    _fields_ = (
        [(n, ShieldField3D) for n in MP_STATE_FIELDS]
        + [(n, ShieldField3D) for n in MP_TENDENCY_FIELDS]
        + [("land", ShieldField2D)]
        + [(n, ctypes.c_void_p) for n in ("rain", "snow", "ice", "graupel")]
    )


class ShieldMpCotangents(ctypes.Structure):
    _fields_ = [(n, ShieldField3D) for n in MP_TENDENCY_FIELDS + ("wmp", "qaz")] + [
        (n, ctypes.c_void_p) for n in ("rain", "snow", "ice", "graupel")
    ]


class ShieldMpGradients(ctypes.Structure):
    _fields_ = [(n, ShieldField3D) for n in MP_STATE_FIELDS + ("qaz",)]


class ShieldMpMember(ctypes.Structure):
    _fields_ = [
        ("fields", ShieldMpFields),
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("timestep", ctypes.c_double),
        ("area", ShieldField2D),
    ]


PHYS_FIELDS = (
    "phii", "prsi", "prsik", "delz", "delp", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr",
    "qsgs_tke", "pt", "dm", "delprsi", "del_gz", "phil", "omga", "dz", "wmp",
) + MP_TENDENCY_FIELDS
SHIELD_PHYS_PREPARE_MICROPHYSICS = 1


class ShieldPhysicsFields(ctypes.Structure):
    _fields_ = [(n, ShieldField3D) for n in PHYS_FIELDS]


class ShieldEdgeRegion(ctypes.Structure):
    _fields_ = [("line", ctypes.c_int), ("lo", ctypes.c_int), ("hi", ctypes.c_int), ("dir", ctypes.c_int)]


class ShieldEdgePlan(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 4), ("r", (ShieldEdgeRegion * 2) * 4)]


DWIND_GEOM_2D = ("vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1", "ew2_2",
                 "ew2_3", "edge_vect_w", "edge_vect_e")


class ShieldDwindGeometry(ctypes.Structure):
    _fields_ = [(n, ShieldField2D) for n in DWIND_GEOM_2D] + [
        ("edge_vect_s", ctypes.c_void_p), ("edge_vect_n", ctypes.c_void_p), ("edge_stride", ctypes.c_int64)]


class ShieldDwindTile(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("grid_type", ctypes.c_int),
                ("dt5", ctypes.c_double), ("plan", ShieldEdgePlan), ("geometry", ShieldDwindGeometry),
                ("u", ShieldField3D), ("v", ShieldField3D), ("u_dt", ShieldField3D), ("v_dt", ShieldField3D)]


EXPORTS = (
    "shield_mp_create",
    "shield_mp_step",
    "shield_mp_destroy",
    "shield_mp_last_error",
    "shield_mp_constants",
    "shield_mp_get_qaz",
    "shield_mp_set_qaz",
    "shield_update_physics_state",
    "shield_update_atmos_state",
    "shield_last_error",
    "shield_mp_setup_constants",
    "shield_mp_ensemble_create",
    "shield_mp_ensemble_step",
    "shield_mp_ensemble_qaz",
    "shield_mp_ensemble_destroy",
    "shield_mp_step_noalloc",
    "shield_mp_step_vjp",
    "shield_physics_prestep",
    "shield_copy_dycore_to_physics",
    "shield_agrid_to_dgrid",
    "shield_mp_check",
    "shield_mp_check_noalloc",
    "shield_mp_step_flags",
    "shield_mp_substeps",
    "shield_physics_prestep_from_dycore",
    "shield_agrid_to_dgrid_tiles",
)

_lib = None


class ShieldError(RuntimeError):
    pass


def load():
    """Load the library (once). Raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ShieldError(
            f"{LIB_PATH} is missing; build it with `python -m pyshield_b200.build` "
            "(this package has no CPU fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.shield_mp_create.argtypes = [ctypes.POINTER(ShieldMpConfig), i32, i32, i32, ShieldField2D, ctypes.POINTER(vp)]
    lib.shield_mp_step.argtypes = [vp, ctypes.POINTER(ShieldMpFields), dbl, i32, vp]
    lib.shield_mp_destroy.argtypes = [vp]
    lib.shield_mp_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.shield_mp_constants.argtypes = [vp, dbl, ctypes.POINTER(ctypes.c_double), i32]
    lib.shield_mp_get_qaz.argtypes = [vp, vp, vp]
    lib.shield_mp_set_qaz.argtypes = [vp, vp, vp]
    lib.shield_update_physics_state.argtypes = [
        i32, i32, i32, ctypes.POINTER(ShieldField3D), ctypes.POINTER(ShieldField3D), ctypes.POINTER(ShieldField3D), dbl, vp,
    ]
    lib.shield_update_atmos_state.argtypes = [
        i32, i32, i32, i32, i32, ctypes.POINTER(ShieldField3D), ShieldField3D, ShieldField3D, ShieldField3D, dbl, dbl, dbl, dbl, vp,
    ]
    lib.shield_mp_setup_constants.argtypes = [ctypes.POINTER(ShieldMpConfig), dbl, ctypes.POINTER(ctypes.c_double), i32]
    lib.shield_mp_ensemble_create.argtypes = [ctypes.POINTER(ShieldMpConfig), i32, i32, ctypes.POINTER(ShieldMpMember), i32, ctypes.POINTER(vp)]
    lib.shield_mp_ensemble_step.argtypes = [vp, i32, i32, vp]
    lib.shield_mp_ensemble_qaz.argtypes = [vp, i32, vp, vp]
    lib.shield_mp_ensemble_destroy.argtypes = [vp]
    lib.shield_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.shield_mp_step_vjp.argtypes = [
        vp, ctypes.POINTER(ShieldMpFields), ctypes.POINTER(ShieldMpCotangents), ctypes.POINTER(ShieldMpGradients), dbl, vp,
    ]
    lib.shield_mp_step_noalloc.argtypes = [
        ctypes.POINTER(ShieldMpConfig), i32, i32, i32, ShieldField2D, ctypes.POINTER(ShieldMpFields), dbl, i32, i32, vp,
    ]
    lib.shield_mp_check.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), vp]
    lib.shield_mp_check_noalloc.argtypes = [i32, ctypes.POINTER(ctypes.c_int64), vp]
    lib.shield_mp_step_flags.argtypes = [vp, ctypes.POINTER(ShieldMpFields), dbl, vp, ctypes.c_int64, vp]
    lib.shield_mp_substeps.argtypes = [vp, dbl]
    lib.shield_agrid_to_dgrid.argtypes = [
        i32, i32, i32, i32, dbl, ctypes.POINTER(ShieldEdgePlan), ctypes.POINTER(ShieldDwindGeometry), ShieldField3D,
        ShieldField3D, ShieldField3D, ShieldField3D, vp,
    ]
    lib.shield_agrid_to_dgrid_tiles.argtypes = [i32, ctypes.POINTER(ShieldDwindTile), vp]
    lib.shield_copy_dycore_to_physics.argtypes = [i32, i32, i32, ctypes.POINTER(ShieldField3D), ctypes.POINTER(ShieldField3D), vp]
    lib.shield_physics_prestep.argtypes = [i32, i32, i32, i32, i32, dbl, i32, ctypes.POINTER(ShieldPhysicsFields), vp]
    lib.shield_physics_prestep_from_dycore.argtypes = [
        i32, i32, i32, i32, i32, dbl, i32, ctypes.POINTER(ShieldPhysicsFields), ctypes.POINTER(ShieldField3D),
        ctypes.POINTER(ShieldField3D), vp,
    ]
    for name in EXPORTS:
        getattr(lib, name).restype = i32
    _lib = lib
    return lib


def last_error(handle=None):
    lib = load()
    buf = ctypes.create_string_buffer(512)
    if handle is None:
        lib.shield_last_error(buf, 512)
    else:
        lib.shield_mp_last_error(handle, buf, 512)
    return buf.value.decode(errors="replace")


def check(rc, handle=None, what="call"):
    if rc < 0:
        raise ShieldError(f"{what} failed ({rc}): {last_error(handle)}")
    return rc


def make_config(cfg):
    """ShieldMpConfig from a PhysicsConfig-like object."""
    c = ShieldMpConfig()
    for name, ctype in _CFG_FIELDS:
        v = getattr(cfg, name)
        setattr(c, name, float(v) if ctype is ctypes.c_double else int(bool(v)) if isinstance(v, bool) else int(v))
    return c
