"""Loading helpers for the golden fixtures written by tests/golden/make_golden.py."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MP_CASES = ("mp_default", "mp_substeps", "mp_flags_a", "mp_flags_b", "mp_prog_ccn_off_ice")
CPL_CASES = ("cpl_small", "cpl_stress")
PHYS_CASES = ("phys_default", "phys_substeps")
MP_TENDENCIES = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")
PRECIP = ("rain", "snow", "ice", "graupel")


def load(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    return z, meta


def mp_inputs(z):
    state = {k[3:]: np.array(z[k]) for k in z.files if k.startswith("in_")}
    area = state.pop("area")
    return state, area


def physics_inputs(z):
    """The PhysicsState storages plus the ten tendencies of
    ``physics_state.microphysics`` (random outside the compute domain,
    which prepare_microphysics zeroes), and the (n,) cell area."""
    st = {k[3:]: np.array(z[k]) for k in z.files if k.startswith("in_")}
    area = st.pop("area")
    return st, area
