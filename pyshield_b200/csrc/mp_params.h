// Kernel parameter block of the microphysics step (host and device).
#pragma once

#include <cstdint>

namespace shield {

// Every scalar the step reads: the physical constants, the process constants
// of Microphysics.setupm (pySHiELD/stencils/microphysics.py:1813-1953), the
// sub-step scalars of _set_timestep (:1964-1979) and the namelist values the
// stencils bake in as externals (:1715-1804).
struct MpConst {
  // physical constants (pyshield_b200/constants.py order)
  double GRAV, RGRAV, RDGAS, RVGAS, HLV, HLF, CP_AIR, KAPPA, CP_VAP, CV_AIR, CV_VAP, C_ICE, C_LIQ, TICE, E00,
      DC_VAP, DC_ICE, D2ICE, LV0, LI00, LI2, EPS, ZVIR, T_MIN, T_SAT_MIN, LAT2;
  // Microphysics.__init__ scalars (:1643-1658, :1712-1713) and init (:1806-1811)
  double c_air, c_vap, d0_vap, lv00, cpaut, so3, zs, log_10, tice0, t_wfr;
  // setupm
  double fac_rc, cracs, csacr, cgacr, cgacs, acco[3][4], csacw, csaci, cgacw, cgaci, cracw, cssub[5], crevp[5],
      cgfr[2], csmlt[5], cgmlt[5], ces0;
  double iqs_lo_num;  // E00 * exp(...) of iqs1's below-T_SAT_MIN branch
  // _set_timestep
  double timestep, rdt, dts, dt_rain, rdts, dt_evap, fac_i2s, fac_g2v, fac_v2g, fac_imlt, fac_l2v;
  int ntimes;
  // namelist values
  double tice, ql_mlt, qs_mlt, t_sub, qi_gen, qi_lim, qi0_max, dw_ocean, dw_land, qc_crt, qi0_crt, qs0_crt, rh_inc,
      rh_inr, vi_fac, vs_fac, vg_fac, vr_fac, vi_max, vs_max, vg_max, vr_max, ccn_l, ccn_o;
  int do_qa, const_vg, const_vi, const_vr, const_vs, rad_snow, rad_rain, do_sedi_heat, do_sedi_w, fast_sat_adj,
      fix_negative, irain_f, prog_ccn, use_ccn, sedi_transport, z_slope_ice, z_slope_liq, de_ice;
};

// FP32 copies of the constants the mixed form's process rates use.
struct MpConstF {
  // FP64 constants of the mixed form's saturation adjustment (qsat_m)
  double qs_e00, qw_c1, qw_c2, qw_c3, qi_c1, qi_c2, qi_c3, qs_t0, qs_tmin, qs_thi, qi_lo, qi_lo_dq;
  double qs_rtw;  // 1 / (tice - t_wfr) of the saturation adjustment
  float E00, DC_VAP, LV0, D2ICE, LI2, RVGAS, TICE, T_SAT_MIN, iqs_lo_num, LAT2;
  float cracs, csacr, cgacr, cgacs, acco[3][4], csacw, csaci, cgacw, cgaci, cracw, cssub[5], crevp[5], cgfr[2],
      csmlt[5], cgmlt[5], ces0, log_10, fac_rc, so3, dt_rain, dts, rdts, fac_i2s;
};

// A strided 3-D field; ptr addresses the compute-domain origin.
struct Fld3 {
  double* p;
  int64_t si, sj, sk;
};
struct Fld2 {
  const double* p;
  int64_t si, sj;
};

// Input tiles staged in shared memory, in this order.
enum InField {
  IN_PT = 0, IN_QV, IN_QL, IN_QR, IN_QI, IN_QS, IN_QG, IN_QA, IN_UA, IN_VA, IN_DELP, IN_DELZ, IN_W, IN_QAZ,
  N_IN
};
// Output slots (tendency increments, then assigned fields), same tiles reused.
enum OutField {
  OUT_PT_DT = 0, OUT_QV_DT, OUT_QL_DT, OUT_QR_DT, OUT_QI_DT, OUT_QS_DT, OUT_QG_DT, OUT_QA_DT, OUT_UDT, OUT_VDT,
  OUT_W, OUT_QAZ, N_OUT
};

struct MpArgs {
  MpConst K;
  MpConstF KF;
  int nx, ny, nz;
  int64_t ncol;
  Fld3 in[N_IN];
  Fld3 out[N_OUT];
  Fld2 land, area;
  double *rain, *snow, *ice, *graupel;  // (ncol,) surface precipitation [mm/day]; may be null
  int* err;                             // device error word
  // column flags of each sub-step (ntimes x ncol, see MpFlagBits), written
  // only by the flag-recording launch; null otherwise
  int* flags;
};

// Bits of the per-column, per-sub-step flags word: which species fall (the
// reference's column-wide no_fall == 0, microphysics.py:349-368 for rain in
// each warm_rain pass, :773-1168 for ice, snow and graupel; ice also needs
// vi_fac >= 1e-5) and the melting level, the first level whose stop_k is 1
// (:706-724; the bottom level when no level is warmer than tice).
enum MpFlagBits : unsigned {
  FLAG_RAIN_FALLS_1 = 1u << 0,
  FLAG_RAIN_FALLS_2 = 1u << 1,
  FLAG_ICE_FALLS = 1u << 2,
  FLAG_SNOW_FALLS = 1u << 3,
  FLAG_GRAUPEL_FALLS = 1u << 4,
  FLAG_MELT_SHIFT = 16u,  // melting level in bits 16..23
};

// Parameter block of the adjoint (vector-Jacobian product) launch. in: the
// step's input state (the first 13 input fields, in the order of InField);
// cot: cotangents of the outputs in the order of OutField (the 10
// tendencies, wmp, the cloud-fraction accumulator); grad: the input
// adjoints written by the launch, in the order of InField (the 13 state
// fields, then the accumulator). A null field pointer is a zero cotangent or
// a gradient that is not written. rain_b .. graupel_b: cotangents of the
// surface totals, ncol each, or null.
constexpr int N_VJP_IN = 13;
constexpr int N_VJP_COT = 12;
constexpr int N_VJP_GRAD = 14;
struct VjpArgs {
  MpConst K;
  MpConstF KF;
  int nx, ny, nz;
  int64_t ncol;
  Fld3 in[N_VJP_IN];
  Fld3 cot[N_VJP_COT];
  Fld3 grad[N_VJP_GRAD];
  Fld2 land, area;
  const double *rain_b, *snow_b, *ice_b, *graupel_b;
  // workspace of mp_vjp_workspace_doubles(ntimes, nz * ncol, ncol) doubles
  double* ws;
  // the incoming qi_dt that de_ice reads (null: zero)
  Fld3 de_ice_qi_dt;
};

}  // namespace shield
