// Host-side constants of the microphysics step: Microphysics.setupm and
// _set_timestep as plain C++ (no CUDA), shared by the C-ABI and the CPU
// adjoint tests.
#pragma once

#include <cmath>
#include <string>

#include "../../include/shield_mp.h"
#include "mp_params.h"

namespace shield {

// Microphysics.setupm (pySHiELD/stencils/microphysics.py:1813-1953) and the
// scalars of __init__ / gfdl_cloud_microphys_init (:1643-1658, :1806-1811).
inline void setupm(const ShieldMpConfig& c, MpConst& K) {
  // physical constants: the values of pyshield_b200/constants.py, with the
  // derived ones computed by the same formulas
  K.GRAV = 9.80665;
  K.RGRAV = 1.0 / K.GRAV;
  K.RDGAS = 287.05;
  K.RVGAS = 461.50;
  K.HLV = 2.5e6;
  K.HLF = 3.3358e5;
  K.CP_AIR = 1004.6;
  K.KAPPA = K.RDGAS / K.CP_AIR;
  K.CP_VAP = 4.0 * K.RVGAS;
  K.CV_AIR = K.CP_AIR - K.RDGAS;
  K.CV_VAP = 3.0 * K.RVGAS;
  K.C_ICE = 1972.0;
  K.C_LIQ = 4.1855e3;
  K.TICE = 273.16;
  K.E00 = 611.21;
  K.DC_VAP = K.CP_VAP - K.C_LIQ;
  K.DC_ICE = K.C_LIQ - K.C_ICE;
  K.D2ICE = K.DC_VAP + K.DC_ICE;
  K.LV0 = K.HLV - K.DC_VAP * K.TICE;
  K.LI00 = K.HLF - K.DC_ICE * K.TICE;
  K.LI2 = K.LV0 + K.LI00;
  K.EPS = K.RDGAS / K.RVGAS;
  K.ZVIR = K.RVGAS / K.RDGAS - 1.0;
  K.T_MIN = 178.0;
  K.T_SAT_MIN = K.TICE - 160.0;
  K.LAT2 = std::pow(K.HLV + K.HLF, 2.0);

  const double RHOS = 1.0e2, RHOG = 4.0e2, RHOR = 1.0e3, SFCRHO = 1.2;
  const double gam263 = 1.456943, gam275 = 1.608355, gam290 = 1.827363, gam325 = 2.54925, gam350 = 3.323363,
               gam380 = 4.694155;
  const double rnzs = 3.0e6, rnzr = 8.0e6, rnzg = 4.0e6;
  const double acc[3] = {5.0, 2.0, 0.5};
  const double pie = 4.0 * std::atan(1.0);
  const double fac_rc = (4.0 / 3.0) * pie * RHOR * std::pow(c.rthresh, 3.0);
  const double vdifu = 2.11e-5, tcond = 2.36e-2, visk = 1.259e-5, hlts = 2.8336e6, hltc = 2.5e6, hltf = 3.336e5,
               ch2o = 4.1855e3;
  const double pisq = pie * pie;
  const double scm3 = std::pow(visk / vdifu, 1.0 / 3.0);
  K.cracs = pisq * rnzr * rnzs * RHOS;
  K.csacr = pisq * rnzr * rnzs * RHOR;
  K.cgacr = pisq * rnzr * rnzg * RHOR;
  K.cgacs = pisq * rnzg * rnzs * RHOS;
  K.cgacs = K.cgacs * c.c_pgacs;
  double act[8];
  act[0] = pie * rnzs * RHOS;
  act[1] = pie * rnzr * RHOR;
  act[5] = pie * rnzg * RHOG;
  act[2] = act[1];
  act[3] = act[0];
  act[4] = act[1];
  act[6] = act[0];
  act[7] = act[5];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 4; ++k)
      K.acco[i][k] =
          acc[i] / (std::pow(act[2 * k], (6 - i) * 0.25) * std::pow(act[2 * k + 1], (i + 1) * 0.25));
  const double gcon = 40.74 * std::sqrt(SFCRHO);
  K.csacw = pie * rnzs * c.clin * gam325 / (4.0 * std::pow(act[0], 0.8125));
  const double craci = pie * rnzr * c.alin * gam380 / (4.0 * std::pow(act[1], 0.95));
  K.csaci = K.csacw * c.c_psaci;
  K.cgacw = pie * rnzg * gam350 * gcon / (4.0 * std::pow(act[5], 0.875));
  K.cgaci = K.cgacw * 0.05;
  K.cracw = c.c_cracw * craci;
  K.cssub[0] = 2.0 * pie * vdifu * tcond * K.RVGAS * rnzs;
  K.cssub[1] = 0.78 / std::sqrt(act[0]);
  K.cssub[2] = 0.31 * scm3 * gam263 * std::sqrt(c.clin / visk) / std::pow(act[0], 0.65625);
  K.cssub[3] = tcond * K.RVGAS;
  K.cssub[4] = std::pow(hlts, 2.0) * vdifu;
  const double cgsub_1 = 0.78 / std::sqrt(act[5]);
  const double cgsub_2 = 0.31 * scm3 * gam275 * std::sqrt(gcon / visk) / std::pow(act[5], 0.6875);
  K.crevp[0] = 2.0 * pie * vdifu * tcond * K.RVGAS * rnzr;
  K.crevp[1] = 0.78 / std::sqrt(act[1]);
  K.crevp[2] = 0.31 * scm3 * gam290 * std::sqrt(c.alin / visk) / std::pow(act[1], 0.725);
  K.crevp[3] = K.cssub[3];
  K.crevp[4] = std::pow(hltc, 2.0) * vdifu;
  K.cgfr[0] = 20.0e2 * pisq * rnzr * RHOR / std::pow(act[1], 1.75);
  K.cgfr[1] = 0.66;
  K.csmlt[0] = 2.0 * pie * tcond * rnzs / hltf;
  K.csmlt[1] = 2.0 * pie * vdifu * rnzs * hltc / hltf;
  K.csmlt[2] = K.cssub[1];
  K.csmlt[3] = K.cssub[2];
  K.csmlt[4] = ch2o / hltf;
  K.cgmlt[0] = 2.0 * pie * tcond * rnzg / hltf;
  K.cgmlt[1] = 2.0 * pie * vdifu * rnzg * hltc / hltf;
  K.cgmlt[2] = cgsub_1;
  K.cgmlt[3] = cgsub_2;
  K.cgmlt[4] = ch2o / hltf;
  const double es0 = 6.107799961e2;
  K.fac_rc = fac_rc;
  K.ces0 = K.EPS * es0;
  K.iqs_lo_num = K.E00 * std::exp((K.D2ICE * std::log(1.0 - 160.0 / K.TICE) - K.LI2 * 160.0 / (K.T_SAT_MIN * K.TICE)) /
                                  K.RVGAS);
  K.log_10 = std::log(10.0);
  K.tice0 = c.tice - 0.01;
  K.t_wfr = c.tice - 40.0;
  K.c_air = K.CP_AIR;
  K.c_vap = K.CP_VAP;
  K.d0_vap = K.c_vap - K.C_LIQ;
  K.lv00 = K.HLV - K.d0_vap * K.TICE;
  K.cpaut = c.c_paut * 0.104 * K.GRAV / 1.717e-5;
  K.so3 = 7.0 / 3.0;
  K.zs = 0.0;
  // namelist values baked in as stencil externals
  K.tice = c.tice;
  K.ql_mlt = c.ql_mlt;
  K.qs_mlt = c.qs_mlt;
  K.t_sub = c.t_sub;
  K.qi_gen = c.qi_gen;
  K.qi_lim = c.qi_lim;
  K.qi0_max = c.qi0_max;
  K.dw_ocean = c.dw_ocean;
  K.dw_land = c.dw_land;
  K.qc_crt = c.qc_crt;
  K.qi0_crt = c.qi0_crt;
  K.qs0_crt = c.qs0_crt;
  K.rh_inc = c.rh_inc;
  K.rh_inr = c.rh_inr;
  K.vi_fac = c.vi_fac;
  K.vs_fac = c.vs_fac;
  K.vg_fac = c.vg_fac;
  K.vr_fac = c.vr_fac;
  K.vi_max = c.vi_max;
  K.vs_max = c.vs_max;
  K.vg_max = c.vg_max;
  K.vr_max = c.vr_max;
  K.ccn_l = c.ccn_l;
  K.ccn_o = c.ccn_o;
  K.do_qa = c.do_qa != 0;
  K.const_vg = c.const_vg != 0;
  K.const_vi = c.const_vi != 0;
  K.const_vr = c.const_vr != 0;
  K.const_vs = c.const_vs != 0;
  K.rad_snow = c.rad_snow != 0;
  K.rad_rain = c.rad_rain != 0;
  K.do_sedi_heat = c.do_sedi_heat != 0;
  K.do_sedi_w = c.hydrostatic ? 0 : (c.do_sedi_w != 0);
  K.fast_sat_adj = c.fast_sat_adj != 0;
  K.fix_negative = c.fix_negative != 0;
  K.irain_f = c.irain_f;
  K.prog_ccn = c.prog_ccn != 0;
  K.use_ccn = c.prog_ccn ? 0 : 1;
  K.sedi_transport = c.sedi_transport != 0;
  K.z_slope_ice = c.z_slope_ice != 0;
  K.z_slope_liq = c.z_slope_liq != 0;
  K.de_ice = c.de_ice != 0;
}

// Microphysics._set_timestep (microphysics.py:1964-1979).
inline int set_timestep(const ShieldMpConfig& c, MpConst& K, double timestep, std::string& why) {
  if (!(timestep > 0.0) || !std::isfinite(timestep)) {
    why = "timestep must be positive and finite";
    return SHIELD_EINVAL;
  }
  const double mpdt = std::fmin(timestep, c.mp_time);
  if (!(mpdt > 0.0)) {
    why = "mp_time must be positive";
    return SHIELD_EINVAL;
  }
  K.rdt = 1.0 / timestep;
  // Python's round(): halves go to the even neighbour, as nearbyint does in
  // the default rounding mode
  const double nt = std::nearbyint(timestep / mpdt);
  if (nt < 1.0 || nt > 1.0e6) {
    why = "timestep / mp_time gives an unusable number of sub-steps";
    return SHIELD_EINVAL;
  }
  K.ntimes = (int)nt;
  K.timestep = timestep;
  K.dts = timestep / K.ntimes;
  K.dt_rain = K.dts * 0.5;
  K.rdts = 1.0 / K.dts;
  K.dt_evap = c.fast_sat_adj ? 0.5 * K.dts : K.dts;
  K.fac_i2s = 1.0 - std::exp(-K.dts / c.tau_i2s);
  K.fac_g2v = 1.0 - std::exp(-K.dts / c.tau_g2v);
  K.fac_v2g = 1.0 - std::exp(-K.dts / c.tau_v2g);
  K.fac_imlt = 1.0 - std::exp(-0.5 * K.dts / c.tau_imlt);
  K.fac_l2v = 1.0 - std::exp(-K.dt_evap / c.tau_l2v);
  return SHIELD_OK;
}

// FP32 copies of the constants used by the mixed form's process rates.
inline MpConstF to_float(const MpConst& K) {
  MpConstF F;
  F.qs_e00 = K.E00 / K.RVGAS;
  F.qw_c1 = K.DC_VAP / K.RVGAS;
  F.qw_c2 = K.LV0 / K.RVGAS;
  F.qw_c3 = F.qw_c2 / K.TICE - F.qw_c1 * std::log(K.TICE);
  F.qi_c1 = K.D2ICE / K.RVGAS;
  F.qi_c2 = K.LI2 / K.RVGAS;
  F.qi_c3 = F.qi_c2 / K.TICE - F.qi_c1 * std::log(K.TICE);
  F.qs_t0 = K.TICE;
  F.qs_tmin = K.T_SAT_MIN;
  F.qs_thi = K.TICE + 102.0;
  F.qi_lo = K.iqs_lo_num / (K.RVGAS * K.T_SAT_MIN);
  F.qi_lo_dq = (K.D2ICE + K.LI2 / K.T_SAT_MIN) / (K.RVGAS * K.T_SAT_MIN);
  F.qs_rtw = 1.0 / (K.tice - K.t_wfr);
  F.E00 = (float)K.E00;
  F.DC_VAP = (float)K.DC_VAP;
  F.LV0 = (float)K.LV0;
  F.D2ICE = (float)K.D2ICE;
  F.LI2 = (float)K.LI2;
  F.RVGAS = (float)K.RVGAS;
  F.TICE = (float)K.TICE;
  F.T_SAT_MIN = (float)K.T_SAT_MIN;
  F.iqs_lo_num = (float)K.iqs_lo_num;
  F.LAT2 = (float)K.LAT2;
  F.cracs = (float)K.cracs;
  F.csacr = (float)K.csacr;
  F.cgacr = (float)K.cgacr;
  F.cgacs = (float)K.cgacs;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 4; ++k) F.acco[i][k] = (float)K.acco[i][k];
  F.csacw = (float)K.csacw;
  F.csaci = (float)K.csaci;
  F.cgacw = (float)K.cgacw;
  F.cgaci = (float)K.cgaci;
  F.cracw = (float)K.cracw;
  for (int i = 0; i < 5; ++i) {
    F.cssub[i] = (float)K.cssub[i];
    F.crevp[i] = (float)K.crevp[i];
    F.csmlt[i] = (float)K.csmlt[i];
    F.cgmlt[i] = (float)K.cgmlt[i];
  }
  F.cgfr[0] = (float)K.cgfr[0];
  F.cgfr[1] = (float)K.cgfr[1];
  F.ces0 = (float)K.ces0;
  F.log_10 = (float)K.log_10;
  F.fac_rc = (float)K.fac_rc;
  F.so3 = (float)K.so3;
  F.dt_rain = (float)K.dt_rain;
  F.dts = (float)K.dts;
  F.rdts = (float)K.rdts;
  F.fac_i2s = (float)K.fac_i2s;
  return F;
}

}  // namespace shield
