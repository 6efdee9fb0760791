"""PhysicsConfig keeps the reference's field names (pySHiELD/_config.py:22-109)."""
import dataclasses

import pytest

from pyshield_b200._config import PHYSICS_PACKAGES, PhysicsConfig

REFERENCE_FIELDS = (
    "dt_atmos hydrostatic npx npy npz nwat schemes do_qa c_cracw c_paut c_pgacs c_psaci ccn_l ccn_o const_vg "
    "const_vi const_vr const_vs vs_fac vg_fac vi_fac vr_fac de_ice layout tau_imlt tau_i2s tau_g2v tau_v2g ql_mlt "
    "qs_mlt t_sub qi_gen qi_lim qi0_max rad_snow rad_rain dw_ocean dw_land tau_l2v c2l_ord do_sedi_heat do_sedi_w "
    "fast_sat_adj qc_crt fix_negative irain_f mp_time prog_ccn qi0_crt qs0_crt rh_inc rh_inr rthresh "
    "sedi_transport use_ppm vg_max vi_max vr_max vs_max z_slope_ice z_slope_liq tice alin clin namelist_override"
).split()


def test_same_fields_same_order():
    assert [f.name for f in dataclasses.fields(PhysicsConfig)] == REFERENCE_FIELDS


def test_schemes_validation():
    assert PhysicsConfig().schemes == [PHYSICS_PACKAGES.GFS_microphysics]
    with pytest.raises(NotImplementedError):
        PhysicsConfig(schemes=["unknown_scheme"])


def test_from_namelist_copies_known_fields():
    class NL:
        dt_atmos = 225
        mp_time = 90.0
        do_qa = True
        unrelated = 3

    c = PhysicsConfig.from_namelist(NL())
    assert c.dt_atmos == 225 and c.mp_time == 90.0 and c.do_qa is True
