// Pointwise GFDL microphysics processes for one model level, on the device.
//
// Each function restates one function of pySHiELD's
// pySHiELD/functions/microphysics_funcs.py (line ranges cited per function)
// or one pointwise block of pySHiELD/stencils/microphysics.py, with the
// operand order of the reference expression so that the same IEEE operations
// are performed (the plain form is compiled with -fmad=false).
//
// The real type R is double for the plain FP64 form. The mixed form
// instantiates the process-rate functions with R = float and keeps
// saturation adjustment, sedimentation and the budgets in double.
#pragma once

#include <cstdint>

#include "mp_params.h"

namespace shield {

// microphysics_funcs.py:7-42 (numeric table kept identical)
constexpr double VCONS = 6.6280504;
constexpr double VCONG = 87.2382675;
constexpr double NORMS = 942477796.076938;
constexpr double NORMG = 5026548245.74367;
constexpr double VCONR = 2503.23638966667;
constexpr double NORMR = 25132741228.7183;
constexpr double THR = 1.0e-8;
constexpr double THI = 1.0e-8;
constexpr double THG = 1.0e-8;
constexpr double THS = 1.0e-8;
constexpr double AA = -4.14122e-5;
constexpr double BB = -0.00538922;
constexpr double CC = -0.0516344;
constexpr double DD_FS = 0.00216078;
constexpr double EE = 1.9714;
constexpr double VR_MIN = 1.0e-3;
constexpr double VF_MIN = 1.0e-5;
constexpr double P_MIN = 100.0;
constexpr double DT_FR = 8.0;
constexpr double SFCRHO = 1.2;
constexpr double RHOS = 1.0e2;
constexpr double RHOG = 4.0e2;
constexpr double RHOR = 1.0e3;
constexpr double QCMIN = 1.0e-12;
constexpr double QRMIN = 1.0e-8;
constexpr double QVMIN = 1.0e-20;

#define SHD __device__ __forceinline__

// The FP64 exp/log/pow sequences are large; called through these
// out-of-line wrappers they exist once in the kernel instead of at every one
// of their call sites, which keeps the kernel within the instruction cache.
#ifndef SHIELD_INLINE_MATH
#define SHIELD_MATH_ATTR static __device__ __noinline__
#else
#define SHIELD_MATH_ATTR __device__ __forceinline__
#endif
SHIELD_MATH_ATTR double xexp(double x) { return exp(x); }
SHIELD_MATH_ATTR double xlog(double x) { return log(x); }
SHIELD_MATH_ATTR double xpow(double x, double y) { return pow(x, y); }

SHD double dim(double x, double y) {
  double d = x - y;
  return d > 0.0 ? d : 0.0;
}
SHD double sq(double x) { return x * x; }

// ---------------------------------------------------- microphysics_funcs.py:52-145
SHIELD_MATH_ATTR double wqs1(const MpConst& K, double ta, double den) {
  return (K.E00 * xexp((K.DC_VAP * xlog(ta / K.TICE) + K.LV0 * (ta - K.TICE) / (ta * K.TICE)) / K.RVGAS)) /
         (K.RVGAS * ta * den);
}
SHD double wqs2(const MpConst& K, double ta, double den, double& dqdt) {
  double tmp = wqs1(K, ta, den);
  dqdt = tmp * (K.DC_VAP + K.LV0 / ta) / (K.RVGAS * ta);
  return tmp;
}
SHIELD_MATH_ATTR double iqs1(const MpConst& K, double ta, double den) {
  if (ta < K.TICE) {
    if (ta >= K.T_SAT_MIN) {
      return (K.E00 * xexp((K.D2ICE * xlog(ta / K.TICE) + K.LI2 * (ta - K.TICE) / (ta * K.TICE)) / K.RVGAS)) /
             (K.RVGAS * ta * den);
    }
    return K.iqs_lo_num / (K.RVGAS * K.T_SAT_MIN * den);
  }
  if (ta <= K.TICE + 102.0) return wqs1(K, ta, den);
  return wqs1(K, K.TICE + 102.0, den);
}
SHD double iqs2(const MpConst& K, double ta, double den, double& dqdt) {
  double tmp = iqs1(K, ta, den);
  if (ta < K.TICE) {
    if (ta >= K.T_SAT_MIN)
      dqdt = tmp * (K.D2ICE + K.LI2 / ta) / (K.RVGAS * ta);
    else
      dqdt = tmp * (K.D2ICE + K.LI2 / K.T_SAT_MIN) / (K.RVGAS * K.T_SAT_MIN);
  } else {
    if (ta <= K.TICE + 102.0)
      dqdt = tmp * (K.DC_VAP + K.LV0 / ta) / (K.RVGAS * ta);
    else
      dqdt = tmp * (K.DC_VAP + K.LV0 / (K.TICE + 102.0)) / (K.RVGAS * (K.TICE + 102.0));
  }
  return tmp;
}

// ---------------------------------------------------- microphysics_funcs.py:148-179
template <typename R>
SHD R acr3d(R v1, R v2, R q1, R q2, R c, R cac_ik, R cac_i1k, R cac_i2k, R rho) {
  R t1 = sqrt(q1 * rho);
  R s1 = sqrt(q2 * rho);
  R s2 = sqrt(s1);
  return c * fabs(v1 - v2) * q1 * s2 * (cac_ik * t1 + cac_i1k * sqrt(t1) * s2 + cac_i2k * s1);
}
template <typename R>
SHD R smlt(R tc, R dqs, R qsrho, R psacw, R psacr, R c_0, R c_1, R c_2, R c_3, R c_4, R rho, R rhofac) {
  return (c_0 * tc / rho - c_1 * dqs) * (c_2 * sqrt(qsrho) + c_3 * xpow(qsrho, R(0.65625)) * sqrt(rhofac)) +
         c_4 * tc * (psacw + psacr);
}
template <typename R>
SHD R gmlt(R tc, R dqs, R qgrho, R pgacw, R pgacr, R c_0, R c_1, R c_2, R c_3, R c_4, R rho) {
  return (c_0 * tc / rho - c_1 * dqs) * (c_2 * sqrt(qgrho) + c_3 * xpow(qgrho, R(0.6875)) / xpow(rho, R(0.25))) +
         c_4 * tc * (pgacw + pgacr);
}

SHD double cvm_of(const MpConst& K, double qv, double q_liq, double q_sol) {
  return K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
}

// ---------------------------------------------------- microphysics_funcs.py:182-265
SHD void revap_racc(const MpConst& K, double dt, double h_var, double& qg, double& qi, double& ql, double& qr,
                    double& qs, double& qv, double& tz, double den, double denfac) {
  if ((tz > K.t_wfr) && (qr > QRMIN)) {
    double lhl = K.lv00 + K.d0_vap * tz;
    double q_liq = ql + qr;
    double q_sol = qi + qs + qg;
    double cvm = cvm_of(K, qv, q_liq, q_sol);
    double lcpk = lhl / cvm;
    double tin = tz - lcpk * ql;
    double qpz = qv + ql;
    double dqsdt;
    double qsat = wqs2(K, tin, den, dqsdt);
    double dqh = fmax(ql, h_var * fmax(qpz, QCMIN));
    dqh = fmin(dqh, 0.2 * qpz);
    double dqv = qsat - qv;
    double q_minus = qpz - dqh;
    double q_plus = qpz + dqh;
    if ((dqv > QVMIN) && (qsat > q_minus)) {
      double dq;
      if (qsat > q_plus)
        dq = qsat - qpz;
      else
        dq = 0.25 * sq(q_minus - qsat) / dqh;
      double qden = qr * den;
      double t2 = tin * tin;
      double evap = K.crevp[0] * t2 * dq * (K.crevp[1] * sqrt(qden) + K.crevp[2] * xexp(0.725 * xlog(qden))) /
                    (K.crevp[3] * t2 + K.crevp[4] * qsat * den);
      evap = fmin(qr, fmin(dt * evap, dqv / (1.0 + lcpk * dqsdt)));
      qr = qr - evap;
      qv = qv + evap;
      q_liq = q_liq - evap;
      cvm = cvm_of(K, qv, q_liq, q_sol);
      tz = tz - evap * lhl / cvm;
    }
    if ((qr > QRMIN) && (ql > 1.0e-6) && (qsat < q_minus)) {
      double sink = dt * denfac * K.cracw * xexp(0.95 * xlog(qr * den));
      sink = sink / (1.0 + sink) * ql;
      ql = ql - sink;
      qr = qr + sink;
    }
  }
}

// ---------------------------------------------------- microphysics_funcs.py:268-341
SHD void fall_speed(const MpConst& K, double qg, double qi, double qs, double tk, double den, double& vtg,
                    double& vti, double& vts) {
  double rhof = sqrt(fmin(10.0, SFCRHO / den));
  if (K.const_vi) {
    vti = K.vi_fac;
  } else {
    double vi0 = 0.01 * K.vi_fac;
    if (qi < THI) {
      vti = VF_MIN;
    } else {
      double tc = tk - K.tice;
      vti = (3.0 + xlog(qi * den) / K.log_10) * (tc * (AA * tc + BB) + CC) + DD_FS * tc + EE;
      vti = vi0 * xexp(K.log_10 * vti) * 0.8;
      vti = fmin(K.vi_max, fmax(VF_MIN, vti));
    }
  }
  if (K.const_vs) {
    vts = K.vs_fac;
  } else {
    if (qs < THS) {
      vts = VF_MIN;
    } else {
      vts = K.vs_fac * VCONS * rhof * xexp(0.0625 * xlog(qs * den / NORMS));
      vts = fmin(K.vs_max, fmax(VF_MIN, vts));
    }
  }
  if (K.const_vg) {
    vtg = K.vg_fac;
  } else {
    if (qg < THG) {
      vtg = VF_MIN;
    } else {
      vtg = K.vg_fac * VCONG * rhof * sqrt(sqrt(sqrt(qg * den / NORMG)));
      vtg = fmin(K.vg_max, fmax(VF_MIN, vtg));
    }
  }
}

// microphysics_funcs.py:344-372 (the no_fall == 0 branch)
SHD double rain_fspeed(const MpConst& K, double qrz, double den) {
  if (K.const_vr) return K.vr_fac;
  double qden = qrz * den;
  if (qrz < THR) return VR_MIN;
  double v = K.vr_fac * VCONR * sqrt(fmin(10.0, SFCRHO / den)) * xexp(0.2 * xlog(qden / NORMR));
  return fmin(K.vr_max, fmax(VR_MIN, v));
}

// ---------------------------------------------------- microphysics_funcs.py:375-428
SHD void autoconv_no_subgrid_var(const MpConst& K, double& qlz, double& qrz, double tz, double den, double ccn,
                                 double c_praut) {
  double qc0 = K.fac_rc * ccn;
  if (tz > K.t_wfr) {
    double qc = K.use_ccn ? qc0 : qc0 / den;
    double dq = qlz - qc;
    if (dq > 0.0) {
      double sink = fmin(dq, K.dt_rain * c_praut * den * xexp(K.so3 * xlog(qlz)));
      qlz = qlz - sink;
      qrz = qrz + sink;
    }
  }
}
SHD void autoconv_subgrid_var(const MpConst& K, double& qlz, double& qrz, double tz, double den, double ccn,
                              double c_praut, double dl) {
  double qc0 = K.fac_rc * ccn;
  if (tz > K.t_wfr + DT_FR) {
    dl = fmin(fmax(1.0e-6, dl), 0.5 * qlz);
    double qc = K.use_ccn ? qc0 : qc0 / den;
    double dq = 0.5 * (qlz + dl - qc);
    if (dq > 0.0) {
      double sink = fmin(1.0, dq / dl) * K.dt_rain * c_praut * den * xexp(K.so3 * xlog(qlz));
      qlz = qlz - sink;
      qrz = qrz + sink;
    }
  }
}

// ---------------------------------------------------- microphysics_funcs.py:431-850
SHD void subgrid_z_proc(const MpConst& K, double h_var, double rh_adj, double rh_rain, double& qaz, double& qgz,
                        double& qiz, double& qlz, double& qrz, double& qsz, double& qvz, double& tz, double den,
                        double denfac, double p1) {
  const double tice = K.tice, t_wfr = K.t_wfr, t_sub = K.t_sub;
  double lhl = K.lv00 + K.d0_vap * tz;
  double lhi = K.LI00 + K.DC_ICE * tz;
  double q_liq = qlz + qrz;
  double q_sol = qiz + qsz + qgz;
  double cvm = cvm_of(K, qvz, q_liq, q_sol);
  double lcpk = lhl / cvm;
  double icpk = lhi / cvm;
  double tcpk = lcpk + icpk;
  double tcp3 = lcpk + icpk * fmin(1.0, dim(tice, tz) / (tice - t_wfr));
  (void)tcpk;
  if (!(p1 >= P_MIN)) return;
  if (tz < K.T_MIN) {
    double sink = dim(1.0e-7, qvz);
    qvz = qvz - sink;
    qiz = qiz + sink;
    q_sol = q_sol + sink;
    cvm = cvm_of(K, qvz, q_liq, q_sol);
    tz = tz + sink * (lhl + lhi) / cvm;
    if (!K.do_qa) qaz = qaz + 1.0;
    return;
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = lhl / cvm;
  icpk = lhi / cvm;
  tcpk = lcpk + icpk;
  tcp3 = lcpk + icpk * fmin(1.0, dim(tice, tz) / (tice - t_wfr));
  double qpz = qvz + qlz + qiz;
  double tin = tz - (lhl * (qlz + qiz) + lhi * qiz) / (K.c_air + qpz * K.c_vap + qrz * K.C_LIQ + (qsz + qgz) * K.C_ICE);
  bool warm = tin > t_sub + 6.0;
  if (warm) {
    double rh = qpz / iqs1(K, tin, den);
    if (rh < rh_adj) {
      tz = tin;
      qvz = qpz;
      qlz = 0.0;
      qiz = 0.0;
      return;  // the adjustment block below requires rh >= rh_adj
    }
  }
  // cloud water <-> vapour adjustment (:531-554)
  double dwsdt;
  double qsw = wqs2(K, tz, den, dwsdt);
  double dq0 = qsw - qvz;
  double evap;
  if (dq0 > 0.0) {
    double factor = fmin(1.0, K.fac_l2v * (10.0 * dq0 / qsw));
    evap = fmin(qlz, factor * dq0 / (1.0 + tcp3 * dwsdt));
  } else {
    evap = dq0 / (1.0 + tcp3 * dwsdt);
  }
  qvz = qvz + evap;
  qlz = qlz - evap;
  q_liq = q_liq - evap;
  cvm = cvm_of(K, qvz, q_liq, q_sol);
  tz = tz - evap * lhl / cvm;
  lhi = K.LI00 + K.DC_ICE * tz;
  icpk = lhi / cvm;
  // forced freezing below t_wfr (:560-575)
  double dtmp = t_wfr - tz;
  if ((dtmp > 0.0) && (qlz > QCMIN)) {
    double sink = fmin(qlz, fmin(qlz * dtmp * 0.125, dtmp / icpk));
    qlz = qlz - sink;
    qiz = qiz + sink;
    q_liq = q_liq - sink;
    q_sol = q_sol + sink;
    cvm = cvm_of(K, qvz, q_liq, q_sol);
    tz = tz + sink * lhi / cvm;
  }
  lhi = K.LI00 + K.DC_ICE * tz;
  icpk = lhi / cvm;
  // Bigg mechanism (:581-605)
  double dt_pisub;
  if (K.fast_sat_adj) {
    dt_pisub = 0.5 * K.dts;
  } else {
    dt_pisub = K.dts;
    double tc = tice - tz;
    if ((qlz > QRMIN) && (tc > 0.0)) {
      double sink = 3.3333e-10 * K.dts * (xexp(0.66 * tc) - 1.0) * den * qlz * qlz;
      sink = fmin(qlz, fmin(tc / icpk, sink));
      qlz = qlz - sink;
      qiz = qiz + sink;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz + sink * lhi / cvm;
    }
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = lhl / cvm;
  icpk = lhi / cvm;
  tcpk = lcpk + icpk;
  // ice deposition / sublimation (:614-661)
  if (tz < tice) {
    double dqsdt;
    double qsi = iqs2(K, tz, den, dqsdt);
    double dq = qvz - qsi;
    double sink = dq / (1.0 + tcpk * dqsdt);
    double pidep;
    if (qiz > QRMIN) {
      pidep = dt_pisub * dq * 349138.78 * xexp(0.875 * xlog(qiz * den)) /
              (qsi * den * K.LAT2 / (0.0243 * K.RVGAS * sq(tz)) + 4.42478e4);
    } else {
      pidep = 0.0;
    }
    if (dq > 0.0) {
      double tmp = tice - tz;
      double qi_crt = K.qi_gen * fmin(K.qi_lim, 0.1 * tmp) / den;
      sink = fmin(sink, fmin(fmax(qi_crt - qiz, pidep), tmp / tcpk));
    } else {
      pidep = pidep * fmin(1.0, dim(tz, t_sub) * 0.2);
      sink = fmax(pidep, fmax(sink, -qiz));
    }
    qvz = qvz - sink;
    qiz = qiz + sink;
    q_sol = q_sol + sink;
    cvm = cvm_of(K, qvz, q_liq, q_sol);
    tz = tz + sink * (lhl + lhi) / cvm;
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = lhl / cvm;
  icpk = lhi / cvm;
  tcpk = lcpk + icpk;
  // snow sublimation / deposition (:670-706)
  if (qsz > QRMIN) {
    double dqsdt;
    double qsi = iqs2(K, tz, den, dqsdt);
    double qden = qsz * den;
    double tmp = xexp(0.65625 * xlog(qden));
    double tsq = tz * tz;
    double dq = (qsi - qvz) / (1.0 + tcpk * dqsdt);
    double pssub = K.cssub[0] * tsq * (K.cssub[1] * sqrt(qden) + K.cssub[2] * tmp * sqrt(denfac)) /
                   (K.cssub[3] * tsq + K.cssub[4] * qsi * den);
    pssub = (qsi - qvz) * K.dts * pssub;
    if (pssub > 0.0) {
      pssub = fmin(pssub * fmin(1.0, dim(tz, t_sub) * 0.2), qsz);
    } else {
      if (tz > tice)
        pssub = 0.0;
      else
        pssub = fmax(pssub, fmax(dq, (tz - tice) / tcpk));
    }
    qsz = qsz - pssub;
    qvz = qvz + pssub;
    q_sol = q_sol - pssub;
    cvm = cvm_of(K, qvz, q_liq, q_sol);
    tz = tz - pssub * (lhl + lhi) / cvm;
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = lhl / cvm;
  icpk = lhi / cvm;
  tcpk = lcpk + icpk;
  // graupel sublimation / deposition (:715-746)
  if (qgz > QRMIN) {
    double dqsdt;
    double qsi = iqs2(K, tz, den, dqsdt);
    double dq = (qvz - qsi) / (1.0 + tcpk * dqsdt);
    double pgsub = (qvz / qsi - 1.0) * qgz;
    if (pgsub > 0.0) {
      if (tz > tice)
        pgsub = 0.0;
      else
        pgsub = fmin(fmin(K.fac_v2g * pgsub, 0.2 * dq), fmin(qlz + qrz, (tice - tz) / tcpk));
    } else {
      pgsub = fmax(K.fac_g2v * pgsub, dq) * fmin(1.0, dim(tz, t_sub) * 0.1);
    }
    qgz = qgz + pgsub;
    qvz = qvz - pgsub;
    q_sol = q_sol + pgsub;
    cvm = cvm_of(K, qvz, q_liq, q_sol);
    tz = tz + pgsub * (lhl + lhi) / cvm;
  }
  // minimum evaporation of rain (:751-769)
  lhl = K.lv00 + K.d0_vap * tz;
  lcpk = lhl / cvm;
  if (qrz > QCMIN) {
    double dqsdt;
    double qsw2 = wqs2(K, tz, den, dqsdt);
    double sink = fmin(qrz, dim(rh_rain * qsw2, qvz) / (1.0 + lcpk * dqsdt));
    qvz = qvz + sink;
    qrz = qrz - sink;
    q_liq = q_liq - sink;
    cvm = cvm_of(K, qvz, q_liq, q_sol);
    tz = tz - sink * lhl / cvm;
  }
  // cloud fraction (:774-848)
  lhl = K.lv00 + K.d0_vap * tz;
  cvm = K.c_air + (qvz + q_liq + q_sol) * K.c_vap;
  lcpk = lhl / cvm;
  if (!K.do_qa) {
    q_sol = K.rad_snow ? qiz + qsz : qiz;
    q_liq = K.rad_rain ? qlz + qrz : qlz;
    double q_cond = q_liq + q_sol;
    double qpz2 = qvz + q_cond;
    double tin2 = tz - (lcpk * q_cond + icpk * q_sol);
    double qstar;
    if (tin2 <= t_wfr) {
      qstar = iqs1(K, tin2, den);
    } else if (tin2 >= tice) {
      qstar = wqs1(K, tin2, den);
    } else {
      double qsi = iqs1(K, tin2, den);
      double qsw3 = wqs1(K, tin2, den);
      double rqi;
      if (q_cond > 3.0e-6)
        rqi = q_sol / q_cond;
      else
        rqi = (tice - tin2) / (tice - t_wfr);
      qstar = rqi * qsi + (1.0 - rqi) * qsw3;
    }
    if (qpz2 > QRMIN) {
      double dq = fmax(QCMIN, h_var * qpz2);
      double q_plus = qpz2 + dq;
      double q_minus = qpz2 - dq;
      if (qstar < q_minus)
        qaz = qaz + 1.0;
      else if ((qstar < q_plus) && (q_cond > K.qc_crt))
        qaz = qaz + (q_plus - qstar) / (dq + dq);
    }
  }
}

// ---------------------------------------------------- microphysics_funcs.py:853-1227
// Ice-phase processes before the saturation adjustment; the caller runs
// subgrid_z_proc afterwards (icloud_main's tail call, :1229-1258).
SHD void icloud_processes(const MpConst& K, double& qgz, double& qiz, double& qlz, double& qrz, double& qsz,
                          double qvz, double& tz, double den, double denfac, double vtgz, double vtrz, double vtsz,
                          double p1, double di, double q_liq, double q_sol, double cvm) {
  const double tice = K.tice, dts = K.dts, rdts = K.rdts;
  double lhi = K.LI00 + K.DC_ICE * tz;
  double icpk = lhi / cvm;
  if (!(p1 >= P_MIN)) return;
  double pgacr = 0.0;
  double pgacw = 0.0;
  double tc = tz - tice;
  if (tc >= 0.0) {
    double dqs0 = K.ces0 / p1 - qvz;
    if (qsz > QCMIN) {
      double psacw, psacr, pracs;
      if (qlz > QRMIN) {
        double factor = denfac * K.csacw * xexp(0.8125 * xlog(qsz * den));
        psacw = factor / (1.0 + dts * factor) * qlz;
      } else {
        psacw = 0.0;
      }
      if (qrz > QRMIN) {
        psacr = fmin(acr3d<double>(vtsz, vtrz, qrz, qsz, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den),
                     qrz * rdts);
        pracs = acr3d<double>(vtrz, vtsz, qsz, qrz, K.cracs, K.acco[0][0], K.acco[1][0], K.acco[2][0], den);
      } else {
        psacr = 0.0;
        pracs = 0.0;
      }
      double psmlt = fmax(0.0, smlt<double>(tc, dqs0, qsz * den, psacw, psacr, K.csmlt[0], K.csmlt[1], K.csmlt[2],
                                             K.csmlt[3], K.csmlt[4], den, denfac));
      double sink = fmin(qsz, fmin(dts * (psmlt + pracs), tc / icpk));
      qsz = qsz - sink;
      double tmp = fmin(sink, dim(K.qs_mlt, qlz));
      qlz = qlz + tmp;
      qrz = qrz + sink - tmp;
      q_liq = q_liq + sink;
      q_sol = q_sol - sink;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz - sink * lhi / cvm;
      tc = tz - tice;
    }
    lhi = K.LI00 + K.DC_ICE * tz;
    icpk = lhi / cvm;
    if ((qgz > QCMIN) && (tc > 0.0)) {
      if (qrz > QRMIN) {
        pgacr = fmin(acr3d<double>(vtgz, vtrz, qrz, qgz, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den),
                     rdts * qrz);
      }
      double qden = qgz * den;
      if (qlz > QRMIN) {
        double factor = K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
        pgacw = factor / (1.0 + dts * factor) * qlz;
      }
      double pgmlt = dts * gmlt<double>(tc, dqs0, qden, pgacw, pgacr, K.cgmlt[0], K.cgmlt[1], K.cgmlt[2],
                                        K.cgmlt[3], K.cgmlt[4], den);
      pgmlt = fmin(fmax(0.0, pgmlt), fmin(qgz, tc / icpk));
      qgz = qgz - pgmlt;
      qrz = qrz + pgmlt;
      q_liq = q_liq + pgmlt;
      q_sol = q_sol - pgmlt;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz - pgmlt * lhi / cvm;
    }
  } else {
    if (qiz > 3.0e-7) {
      double psaci;
      if (qsz > 1.0e-7) {
        double factor = dts * denfac * K.csaci * xexp(0.05 * tc + 0.8125 * xlog(qsz * den));
        psaci = factor / (1.0 + factor) * qiz;
      } else {
        psaci = 0.0;
      }
      double qim = K.qi0_crt / den;
      double tmp = K.const_vi ? K.fac_i2s : K.fac_i2s * xexp(0.025 * tc);
      di = fmax(di, QRMIN);
      double q_plus = qiz + di;
      double psaut;
      if (q_plus > (qim + QRMIN)) {
        double dq;
        if (qim > (qiz - di))
          dq = (0.25 * sq(q_plus - qim)) / di;
        else
          dq = qiz - qim;
        psaut = tmp * dq;
      } else {
        psaut = 0.0;
      }
      double sink = fmin(0.75 * qiz, psaci + psaut);
      qiz = qiz - sink;
      qsz = qsz + sink;
      if (qgz > 1.0e-6) {
        double factor = dts * K.cgaci * sqrt(den) * qgz;
        double pgaci = factor / (1.0 + factor) * qiz;
        qiz = qiz - pgaci;
        qgz = qgz + pgaci;
      }
    }
    tc = tz - tice;
    if ((qrz > 1e-7) && (tc < 0.0)) {
      double psacr;
      if (qsz > 1.0e-7)
        psacr = dts * acr3d<double>(vtsz, vtrz, qrz, qsz, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den);
      else
        psacr = 0.0;
      double pgfr = dts * K.cgfr[0] / den * (xexp(-K.cgfr[1] * tc) - 1.0) * xexp(1.75 * xlog(qrz * den));
      double sink = psacr + pgfr;
      double factor = fmin(sink, fmin(qrz, -tc / icpk)) / fmax(sink, QRMIN);
      psacr = factor * psacr;
      pgfr = factor * pgfr;
      sink = psacr + pgfr;
      qrz = qrz - sink;
      qsz = qsz + psacr;
      qgz = qgz + pgfr;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz + sink * lhi / cvm;
    }
    lhi = K.LI00 + K.DC_ICE * tz;
    icpk = lhi / cvm;
    if (qsz > 1.0e-7) {
      double sink;
      if (qgz > QRMIN)
        sink = dts * acr3d<double>(vtgz, vtsz, qsz, qgz, K.cgacs, K.acco[0][3], K.acco[1][3], K.acco[2][3], den);
      else
        sink = 0.0;
      double qsm = K.qs0_crt / den;
      if (qsz > qsm) {
        double factor = dts * 1.0e-3 * xexp(0.09 * (tz - tice));
        sink = sink + factor / (1.0 + factor) * (qsz - qsm);
      }
      sink = fmin(qsz, sink);
      qsz = qsz - sink;
      qgz = qgz + sink;
    }
    if ((qgz > 1.0e-7) && (tz < K.tice0)) {
      if (qlz > 1.0e-6) {
        double qden = qgz * den;
        double factor = dts * K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
        pgacw = factor / (1.0 + factor) * qlz;
      } else {
        pgacw = 0.0;
      }
      if (qrz > 1.0e-6) {
        pgacr = fmin(dts * acr3d<double>(vtgz, vtrz, qrz, qgz, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den),
                     qrz);
      } else {
        pgacr = 0.0;
      }
      double sink = pgacr + pgacw;
      double factor = fmin(sink, dim(tice, tz) / icpk) / fmax(sink, QRMIN);
      pgacr = factor * pgacr;
      pgacw = factor * pgacw;
      sink = pgacr + pgacw;
      qgz = qgz + sink;
      qrz = qrz - pgacr;
      qlz = qlz - pgacw;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz + sink * lhi / cvm;
    }
  }
}

}  // namespace shield
