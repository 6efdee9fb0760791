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
#ifndef __CUDACC__
#include <cmath>
#include <type_traits>
#endif

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

#ifdef __CUDACC__
#define SHD __device__ __forceinline__
// pointwise physics: also compiled for the host, where the adjoint tests
// instantiate it with a dual-number type
#define SHP __host__ __device__ __forceinline__
#else
#define SHD inline
#define SHP inline
#endif

// The FP64 exp/log/pow sequences are large; called through these
// out-of-line wrappers they exist once in the kernel instead of at every one
// of their call sites, which keeps the kernel within the instruction cache.
#if defined(__CUDACC__) && !defined(SHIELD_INLINE_MATH)
#define SHIELD_MATH_ATTR static __host__ __device__ __noinline__
#elif defined(__CUDACC__)
#define SHIELD_MATH_ATTR __host__ __device__ __forceinline__
#else
#define SHIELD_MATH_ATTR static inline
#endif
SHIELD_MATH_ATTR double xexp(double x) { return exp(x); }
SHIELD_MATH_ATTR double xlog(double x) { return log(x); }
SHIELD_MATH_ATTR double xpow(double x, double y) { return pow(x, y); }

SHP double dim(double x, double y) {
  double d = x - y;
  return d > 0.0 ? d : 0.0;
}
SHP double sq(double x) { return x * x; }

// ---------------------------------------------------- microphysics_funcs.py:52-145
template <typename T>
SHIELD_MATH_ATTR T wqs1(const MpConst& K, T ta, T den) {
  return (K.E00 * xexp((K.DC_VAP * xlog(ta / K.TICE) + K.LV0 * (ta - K.TICE) / (ta * K.TICE)) / K.RVGAS)) /
         (K.RVGAS * ta * den);
}
template <typename T>
SHP T wqs2(const MpConst& K, T ta, T den, T& dqdt) {
  T tmp = wqs1(K, ta, den);
  dqdt = tmp * (K.DC_VAP + K.LV0 / ta) / (K.RVGAS * ta);
  return tmp;
}
template <typename T>
SHIELD_MATH_ATTR T iqs1(const MpConst& K, T ta, T den) {
  if (ta < K.TICE) {
    if (ta >= K.T_SAT_MIN) {
      return (K.E00 * xexp((K.D2ICE * xlog(ta / K.TICE) + K.LI2 * (ta - K.TICE) / (ta * K.TICE)) / K.RVGAS)) /
             (K.RVGAS * ta * den);
    }
    return K.iqs_lo_num / (K.RVGAS * K.T_SAT_MIN * den);
  }
  if (ta <= K.TICE + 102.0) return wqs1<T>(K, ta, den);
  return wqs1<T>(K, T(K.TICE + 102.0), den);
}
template <typename T>
SHP T iqs2(const MpConst& K, T ta, T den, T& dqdt) {
  T tmp = iqs1(K, ta, den);
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
SHP R acr3d(R v1, R v2, R q1, R q2, R c, R cac_ik, R cac_i1k, R cac_i2k, R rho) {
  R t1 = sqrt(q1 * rho);
  R s1 = sqrt(q2 * rho);
  R s2 = sqrt(s1);
  return c * fabs(v1 - v2) * q1 * s2 * (cac_ik * t1 + cac_i1k * sqrt(t1) * s2 + cac_i2k * s1);
}
template <typename R>
SHP R smlt(R tc, R dqs, R qsrho, R psacw, R psacr, R c_0, R c_1, R c_2, R c_3, R c_4, R rho, R rhofac) {
  return (c_0 * tc / rho - c_1 * dqs) * (c_2 * sqrt(qsrho) + c_3 * xpow(qsrho, R(0.65625)) * sqrt(rhofac)) +
         c_4 * tc * (psacw + psacr);
}
template <typename R>
SHP R gmlt(R tc, R dqs, R qgrho, R pgacw, R pgacr, R c_0, R c_1, R c_2, R c_3, R c_4, R rho) {
  return (c_0 * tc / rho - c_1 * dqs) * (c_2 * sqrt(qgrho) + c_3 * xpow(qgrho, R(0.6875)) / xpow(rho, R(0.25))) +
         c_4 * tc * (pgacw + pgacr);
}

template <typename T>
SHP T cvm_of(const MpConst& K, T qv, T q_liq, T q_sol) {
  return K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
}

// ---------------------------------------------------- microphysics_funcs.py:182-265
template <typename T>
SHP void revap_racc(const MpConst& K, double dt, double h_var, T& qg, T& qi, T& ql, T& qr, T& qs, T& qv, T& tz,
                    T den, T denfac) {
  if ((tz > K.t_wfr) && (qr > QRMIN)) {
    T lhl = K.lv00 + K.d0_vap * tz;
    T q_liq = ql + qr;
    T q_sol = qi + qs + qg;
    T cvm = cvm_of(K, qv, q_liq, q_sol);
    T lcpk = lhl / cvm;
    T tin = tz - lcpk * ql;
    T qpz = qv + ql;
    T dqsdt;
    T qsat = wqs2(K, tin, den, dqsdt);
    T dqh = fmax(ql, h_var * fmax(qpz, QCMIN));
    dqh = fmin(dqh, 0.2 * qpz);
    T dqv = qsat - qv;
    T q_minus = qpz - dqh;
    T q_plus = qpz + dqh;
    if ((dqv > QVMIN) && (qsat > q_minus)) {
      T dq;
      if (qsat > q_plus)
        dq = qsat - qpz;
      else
        dq = 0.25 * sq(q_minus - qsat) / dqh;
      T qden = qr * den;
      T t2 = tin * tin;
      T evap = K.crevp[0] * t2 * dq * (K.crevp[1] * sqrt(qden) + K.crevp[2] * xexp(0.725 * xlog(qden))) /
                    (K.crevp[3] * t2 + K.crevp[4] * qsat * den);
      evap = fmin(qr, fmin(dt * evap, dqv / (1.0 + lcpk * dqsdt)));
      qr = qr - evap;
      qv = qv + evap;
      q_liq = q_liq - evap;
      cvm = cvm_of(K, qv, q_liq, q_sol);
      tz = tz - evap * lhl / cvm;
    }
    if ((qr > QRMIN) && (ql > 1.0e-6) && (qsat < q_minus)) {
      T sink = dt * denfac * K.cracw * xexp(0.95 * xlog(qr * den));
      sink = sink / (1.0 + sink) * ql;
      ql = ql - sink;
      qr = qr + sink;
    }
  }
}

// ---------------------------------------------------- microphysics_funcs.py:268-341
template <typename T>
SHP void fall_speed(const MpConst& K, T qg, T qi, T qs, T tk, T den, T& vtg, T& vti, T& vts) {
  T rhof = sqrt(fmin(10.0, SFCRHO / den));
  if (K.const_vi) {
    vti = K.vi_fac;
  } else {
    T vi0 = 0.01 * K.vi_fac;
    if (qi < THI) {
      vti = VF_MIN;
    } else {
      T tc = tk - K.tice;
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
template <typename T>
SHP T rain_fspeed(const MpConst& K, T qrz, T den) {
  if (K.const_vr) return K.vr_fac;
  T qden = qrz * den;
  if (qrz < THR) return VR_MIN;
  T v = K.vr_fac * VCONR * sqrt(fmin(10.0, SFCRHO / den)) * xexp(0.2 * xlog(qden / NORMR));
  return fmin(K.vr_max, fmax(VR_MIN, v));
}

// ---------------------------------------------------- microphysics_funcs.py:375-428
template <typename T>
SHP void autoconv_no_subgrid_var(const MpConst& K, T& qlz, T& qrz, T tz, T den, T ccn, T c_praut) {
  T qc0 = K.fac_rc * ccn;
  if (tz > K.t_wfr) {
    T qc = K.use_ccn ? qc0 : qc0 / den;
    T dq = qlz - qc;
    if (dq > 0.0) {
      T sink = fmin(dq, K.dt_rain * c_praut * den * xexp(K.so3 * xlog(qlz)));
      qlz = qlz - sink;
      qrz = qrz + sink;
    }
  }
}
template <typename T>
SHP void autoconv_subgrid_var(const MpConst& K, T& qlz, T& qrz, T tz, T den, T ccn, T c_praut, T dl) {
  T qc0 = K.fac_rc * ccn;
  if (tz > K.t_wfr + DT_FR) {
    dl = fmin(fmax(1.0e-6, dl), 0.5 * qlz);
    T qc = K.use_ccn ? qc0 : qc0 / den;
    T dq = 0.5 * (qlz + dl - qc);
    if (dq > 0.0) {
      T sink = fmin(1.0, dq / dl) * K.dt_rain * c_praut * den * xexp(K.so3 * xlog(qlz));
      qlz = qlz - sink;
      qrz = qrz + sink;
    }
  }
}

// exp / log in the rate type R of subgrid_z_proc: the FP64 wrappers (and the
// dual-number overloads found by argument-dependent lookup) by default,
// single precision for R = float
template <typename R>
SHP R rexp(R x) { return xexp(x); }
template <typename R>
SHP R rlog(R x) { return xlog(x); }
template <>
SHP float rexp<float>(float x) { return expf(x); }
template <>
SHP float rlog<float>(float x) { return logf(x); }
SHP float sq(float x) { return x * x; }

// The heat capacity of the saturation adjustment's latent-heat steps. The
// FP64 step divides by it at every use, as the reference does; the mixed
// form keeps its reciprocal and multiplies (FP64 either way).
template <typename T, bool RECIPROCAL>
struct HeatCap {
  T cvm, rc;
  SHP void set(T c) {
    cvm = c;
    if constexpr (RECIPROCAL) rc = T(1.0) / c;
  }
  SHP T div(T a) const {
    if constexpr (RECIPROCAL)
      return a * rc;
    else
      return a / cvm;
  }
};

// The mixed form's saturation humidities, still in FP64: wqs1/wqs2 (ice =
// 0) and iqs1/iqs2 (ice = 1) of microphysics_funcs.py:52-145 restated. With
// c1 = Dc / Rv, c2 = L / Rv and c3 = c2 / T0 - c1 ln T0,
//   exp((Dc ln(T / T0) + L (T - T0) / (T T0)) / Rv) = exp(c1 ln T + c3 - c2 / T),
//   qs = (E00 / Rv) exp(...) / (T den),   dqs/dT = qs (c1 + c2 / T) / T,
// so one reciprocal of T replaces the four divisions (the caller supplies
// 1 / den). The ice form's branches are iqs1's: below T_SAT_MIN the fixed
// value, above T0 the water form at min(T, T0 + 102). Equal to the
// reference's expressions to FP64 round-off (not bit for bit).
struct QsM {
  double q, dq;
};
SHIELD_MATH_ATTR QsM qsat_m(const MpConstF& F, int ice, double ta, double rden) {
  double c1 = F.qw_c1, c2 = F.qw_c2, c3 = F.qw_c3;
  if (ice) {
    if (ta < F.qs_t0) {
      if (!(ta >= F.qs_tmin)) {
        const double q = F.qi_lo * rden;
        return QsM{q, q * F.qi_lo_dq};
      }
      c1 = F.qi_c1;
      c2 = F.qi_c2;
      c3 = F.qi_c3;
    } else if (!(ta <= F.qs_thi)) {
      ta = F.qs_thi;
    }
  }
  const double r = 1.0 / ta;
  const double q = F.qs_e00 * exp(c1 * log(ta) + c3 - c2 * r) * r * rden;
  return QsM{q, q * r * (c1 + c2 * r)};
}

// ---------------------------------------------------- microphysics_funcs.py:431-850
// R is the type of the deposition/sublimation and Bigg-freezing rate
// expressions (T for the FP64 step; float for the mixed form). Every
// saturation humidity, latent-heat temperature step and state update stays
// in T. The mixed form (R = float, which passes KF) evaluates the saturation
// humidities with qsat_m and the latent-heat steps with the heat capacity's
// reciprocal, both FP64.
template <typename T, typename R = T>
SHP void subgrid_z_proc(const MpConst& K, double h_var, double rh_adj, double rh_rain, T& qaz, T& qgz, T& qiz,
                        T& qlz, T& qrz, T& qsz, T& qvz, T& tz, T den, T denfac, T p1,
                        const MpConstF* KF = nullptr) {
  constexpr bool FAST = std::is_same<R, float>::value;
  const T tice = K.tice, t_wfr = K.t_wfr, t_sub = K.t_sub;
  T rden = T(0.0);
  if constexpr (FAST) rden = 1.0 / den;
  // the saturation humidities (and derivatives) over water and ice
  auto qs_w = [&](T ta, T* dqdt) -> T {
    if constexpr (FAST) {
      const QsM r = qsat_m(*KF, 0, ta, rden);
      if (dqdt) *dqdt = r.dq;
      return r.q;
    } else {
      return dqdt ? wqs2(K, ta, den, *dqdt) : wqs1(K, ta, den);
    }
  };
  auto qs_i = [&](T ta, T* dqdt) -> T {
    if constexpr (FAST) {
      const QsM r = qsat_m(*KF, 1, ta, rden);
      if (dqdt) *dqdt = r.dq;
      return r.q;
    } else {
      return dqdt ? iqs2(K, ta, den, *dqdt) : iqs1(K, ta, den);
    }
  };
  HeatCap<T, FAST> H;
  // x / (tice - t_wfr): a product with the reciprocal in the mixed form
  auto over_tw = [&](T x) -> T {
    if constexpr (FAST)
      return x * KF->qs_rtw;
    else
      return x / (tice - t_wfr);
  };
  T lhl = K.lv00 + K.d0_vap * tz;
  T lhi = K.LI00 + K.DC_ICE * tz;
  T q_liq = qlz + qrz;
  T q_sol = qiz + qsz + qgz;
  H.set(cvm_of(K, qvz, q_liq, q_sol));
  T lcpk = H.div(lhl);
  T icpk = H.div(lhi);
  T tcpk = lcpk + icpk;
  T tcp3 = lcpk + icpk * fmin(1.0, over_tw(dim(tice, tz)));
  (void)tcpk;
  if (!(p1 >= P_MIN)) return;
  if (tz < K.T_MIN) {
    T sink = dim(1.0e-7, qvz);
    qvz = qvz - sink;
    qiz = qiz + sink;
    q_sol = q_sol + sink;
    H.set(cvm_of(K, qvz, q_liq, q_sol));
    tz = tz + H.div(sink * (lhl + lhi));
    if (!K.do_qa) qaz = qaz + 1.0;
    return;
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = H.div(lhl);
  icpk = H.div(lhi);
  tcpk = lcpk + icpk;
  tcp3 = lcpk + icpk * fmin(1.0, over_tw(dim(tice, tz)));
  T qpz = qvz + qlz + qiz;
  T tin = tz - (lhl * (qlz + qiz) + lhi * qiz) / (K.c_air + qpz * K.c_vap + qrz * K.C_LIQ + (qsz + qgz) * K.C_ICE);
  bool warm = tin > t_sub + 6.0;
  if (warm) {
    bool dry;
    if constexpr (FAST)
      dry = qpz < rh_adj * qs_i(tin, nullptr);  // qs > 0: rh < rh_adj without the division
    else
      dry = qpz / qs_i(tin, nullptr) < rh_adj;
    if (dry) {
      tz = tin;
      qvz = qpz;
      qlz = 0.0;
      qiz = 0.0;
      return;  // the adjustment block below requires rh >= rh_adj
    }
  }
  // cloud water <-> vapour adjustment (:531-554)
  T dwsdt;
  T qsw = qs_w(tz, &dwsdt);
  T dq0 = qsw - qvz;
  T evap;
  if (dq0 > 0.0) {
    T factor = fmin(1.0, K.fac_l2v * (10.0 * dq0 / qsw));
    evap = fmin(qlz, factor * dq0 / (1.0 + tcp3 * dwsdt));
  } else {
    evap = dq0 / (1.0 + tcp3 * dwsdt);
  }
  qvz = qvz + evap;
  qlz = qlz - evap;
  q_liq = q_liq - evap;
  H.set(cvm_of(K, qvz, q_liq, q_sol));
  tz = tz - H.div(evap * lhl);
  lhi = K.LI00 + K.DC_ICE * tz;
  icpk = H.div(lhi);
  // forced freezing below t_wfr (:560-575)
  T dtmp = t_wfr - tz;
  if ((dtmp > 0.0) && (qlz > QCMIN)) {
    T sink = fmin(qlz, fmin(qlz * dtmp * 0.125, dtmp / icpk));
    qlz = qlz - sink;
    qiz = qiz + sink;
    q_liq = q_liq - sink;
    q_sol = q_sol + sink;
    H.set(cvm_of(K, qvz, q_liq, q_sol));
    tz = tz + H.div(sink * lhi);
  }
  lhi = K.LI00 + K.DC_ICE * tz;
  icpk = H.div(lhi);
  // Bigg mechanism (:581-605)
  T dt_pisub;
  if (K.fast_sat_adj) {
    dt_pisub = 0.5 * K.dts;
  } else {
    dt_pisub = K.dts;
    T tc = tice - tz;
    if ((qlz > QRMIN) && (tc > 0.0)) {
      T sink = T(R(3.3333e-10) * R(K.dts) * (rexp(R(0.66) * R(tc)) - R(1.0)) * R(den) * R(qlz) * R(qlz));
      sink = fmin(qlz, fmin(tc / icpk, sink));
      qlz = qlz - sink;
      qiz = qiz + sink;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      H.set(cvm_of(K, qvz, q_liq, q_sol));
      tz = tz + H.div(sink * lhi);
    }
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = H.div(lhl);
  icpk = H.div(lhi);
  tcpk = lcpk + icpk;
  // ice deposition / sublimation (:614-661)
  if (tz < tice) {
    T dqsdt;
    T qsi = qs_i(tz, &dqsdt);
    T dq = qvz - qsi;
    T sink = dq / (1.0 + tcpk * dqsdt);
    T pidep;
    if (qiz > QRMIN) {
      pidep = T(R(dt_pisub) * R(dq) * R(349138.78) * rexp(R(0.875) * rlog(R(qiz) * R(den))) /
                (R(qsi) * R(den) * R(K.LAT2) / (R(0.0243) * R(K.RVGAS) * sq(R(tz))) + R(4.42478e4)));
    } else {
      pidep = 0.0;
    }
    if (dq > 0.0) {
      T tmp = tice - tz;
      T qi_crt = K.qi_gen * fmin(K.qi_lim, 0.1 * tmp);
      if constexpr (FAST)
        qi_crt = qi_crt * rden;
      else
        qi_crt = qi_crt / den;
      sink = fmin(sink, fmin(fmax(qi_crt - qiz, pidep), tmp / tcpk));
    } else {
      pidep = pidep * fmin(1.0, dim(tz, t_sub) * 0.2);
      sink = fmax(pidep, fmax(sink, -qiz));
    }
    qvz = qvz - sink;
    qiz = qiz + sink;
    q_sol = q_sol + sink;
    H.set(cvm_of(K, qvz, q_liq, q_sol));
    tz = tz + H.div(sink * (lhl + lhi));
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = H.div(lhl);
  icpk = H.div(lhi);
  tcpk = lcpk + icpk;
  // snow sublimation / deposition (:670-706)
  if (qsz > QRMIN) {
    T dqsdt;
    T qsi = qs_i(tz, &dqsdt);
    T qden = qsz * den;
    const R qdr = R(qden);
    const R tmp = rexp(R(0.65625) * rlog(qdr));
    T tsq = tz * tz;
    T dq = (qsi - qvz) / (1.0 + tcpk * dqsdt);
    const R tsr = R(tsq);
    T pssub = T(R(K.cssub[0]) * tsr * (R(K.cssub[1]) * sqrt(qdr) + R(K.cssub[2]) * tmp * sqrt(R(denfac))) /
                (R(K.cssub[3]) * tsr + R(K.cssub[4]) * R(qsi) * R(den)));
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
    H.set(cvm_of(K, qvz, q_liq, q_sol));
    tz = tz - H.div(pssub * (lhl + lhi));
  }
  lhl = K.lv00 + K.d0_vap * tz;
  lhi = K.LI00 + K.DC_ICE * tz;
  lcpk = H.div(lhl);
  icpk = H.div(lhi);
  tcpk = lcpk + icpk;
  // graupel sublimation / deposition (:715-746)
  if (qgz > QRMIN) {
    T dqsdt;
    T qsi = qs_i(tz, &dqsdt);
    T dq = (qvz - qsi) / (1.0 + tcpk * dqsdt);
    T pgsub = (qvz / qsi - 1.0) * qgz;
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
    H.set(cvm_of(K, qvz, q_liq, q_sol));
    tz = tz + H.div(pgsub * (lhl + lhi));
  }
  // minimum evaporation of rain (:751-769)
  lhl = K.lv00 + K.d0_vap * tz;
  lcpk = H.div(lhl);
  if (qrz > QCMIN) {
    T dqsdt;
    T qsw2 = qs_w(tz, &dqsdt);
    T sink = fmin(qrz, dim(rh_rain * qsw2, qvz) / (1.0 + lcpk * dqsdt));
    qvz = qvz + sink;
    qrz = qrz - sink;
    q_liq = q_liq - sink;
    H.set(cvm_of(K, qvz, q_liq, q_sol));
    tz = tz - H.div(sink * lhl);
  }
  // cloud fraction (:774-848)
  lhl = K.lv00 + K.d0_vap * tz;
  H.set(K.c_air + (qvz + q_liq + q_sol) * K.c_vap);
  lcpk = H.div(lhl);
  if (!K.do_qa) {
    q_sol = K.rad_snow ? qiz + qsz : qiz;
    q_liq = K.rad_rain ? qlz + qrz : qlz;
    T q_cond = q_liq + q_sol;
    T qpz2 = qvz + q_cond;
    T tin2 = tz - (lcpk * q_cond + icpk * q_sol);
    T qstar;
    if (tin2 <= t_wfr) {
      qstar = qs_i(tin2, nullptr);
    } else if (tin2 >= tice) {
      qstar = qs_w(tin2, nullptr);
    } else {
      T qsi = qs_i(tin2, nullptr);
      T qsw3 = qs_w(tin2, nullptr);
      T rqi;
      if (q_cond > 3.0e-6)
        rqi = q_sol / q_cond;
      else
        rqi = over_tw(tice - tin2);
      qstar = rqi * qsi + (1.0 - rqi) * qsw3;
    }
    if (qpz2 > QRMIN) {
      T dq = fmax(QCMIN, h_var * qpz2);
      T q_plus = qpz2 + dq;
      T q_minus = qpz2 - dq;
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
template <typename T>
SHP void icloud_processes(const MpConst& K, T& qgz, T& qiz, T& qlz, T& qrz, T& qsz, T qvz, T& tz, T den, T denfac,
                          T vtgz, T vtrz, T vtsz, T p1, T di, T q_liq, T q_sol, T cvm) {
  const T tice = K.tice, dts = K.dts, rdts = K.rdts;
  T lhi = K.LI00 + K.DC_ICE * tz;
  T icpk = lhi / cvm;
  if (!(p1 >= P_MIN)) return;
  T pgacr = 0.0;
  T pgacw = 0.0;
  T tc = tz - tice;
  if (tc >= 0.0) {
    T dqs0 = K.ces0 / p1 - qvz;
    if (qsz > QCMIN) {
      T psacw, psacr, pracs;
      if (qlz > QRMIN) {
        T factor = denfac * K.csacw * xexp(0.8125 * xlog(qsz * den));
        psacw = factor / (1.0 + dts * factor) * qlz;
      } else {
        psacw = 0.0;
      }
      if (qrz > QRMIN) {
        psacr = fmin(acr3d<T>(vtsz, vtrz, qrz, qsz, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den),
                     qrz * rdts);
        pracs = acr3d<T>(vtrz, vtsz, qsz, qrz, K.cracs, K.acco[0][0], K.acco[1][0], K.acco[2][0], den);
      } else {
        psacr = 0.0;
        pracs = 0.0;
      }
      T psmlt = fmax(0.0, smlt<T>(tc, dqs0, qsz * den, psacw, psacr, K.csmlt[0], K.csmlt[1], K.csmlt[2],
                                             K.csmlt[3], K.csmlt[4], den, denfac));
      T sink = fmin(qsz, fmin(dts * (psmlt + pracs), tc / icpk));
      qsz = qsz - sink;
      T tmp = fmin(sink, dim(K.qs_mlt, qlz));
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
        pgacr = fmin(acr3d<T>(vtgz, vtrz, qrz, qgz, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den),
                     rdts * qrz);
      }
      T qden = qgz * den;
      if (qlz > QRMIN) {
        T factor = K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
        pgacw = factor / (1.0 + dts * factor) * qlz;
      }
      T pgmlt = dts * gmlt<T>(tc, dqs0, qden, pgacw, pgacr, K.cgmlt[0], K.cgmlt[1], K.cgmlt[2],
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
      T psaci;
      if (qsz > 1.0e-7) {
        T factor = dts * denfac * K.csaci * xexp(0.05 * tc + 0.8125 * xlog(qsz * den));
        psaci = factor / (1.0 + factor) * qiz;
      } else {
        psaci = 0.0;
      }
      T qim = K.qi0_crt / den;
      T tmp = K.const_vi ? K.fac_i2s : K.fac_i2s * xexp(0.025 * tc);
      di = fmax(di, QRMIN);
      T q_plus = qiz + di;
      T psaut;
      if (q_plus > (qim + QRMIN)) {
        T dq;
        if (qim > (qiz - di))
          dq = (0.25 * sq(q_plus - qim)) / di;
        else
          dq = qiz - qim;
        psaut = tmp * dq;
      } else {
        psaut = 0.0;
      }
      T sink = fmin(0.75 * qiz, psaci + psaut);
      qiz = qiz - sink;
      qsz = qsz + sink;
      if (qgz > 1.0e-6) {
        T factor = dts * K.cgaci * sqrt(den) * qgz;
        T pgaci = factor / (1.0 + factor) * qiz;
        qiz = qiz - pgaci;
        qgz = qgz + pgaci;
      }
    }
    tc = tz - tice;
    if ((qrz > 1e-7) && (tc < 0.0)) {
      T psacr;
      if (qsz > 1.0e-7)
        psacr = dts * acr3d<T>(vtsz, vtrz, qrz, qsz, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den);
      else
        psacr = 0.0;
      T pgfr = dts * K.cgfr[0] / den * (xexp(-K.cgfr[1] * tc) - 1.0) * xexp(1.75 * xlog(qrz * den));
      T sink = psacr + pgfr;
      T factor = fmin(sink, fmin(qrz, -tc / icpk)) / fmax(sink, QRMIN);
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
      T sink;
      if (qgz > QRMIN)
        sink = dts * acr3d<T>(vtgz, vtsz, qsz, qgz, K.cgacs, K.acco[0][3], K.acco[1][3], K.acco[2][3], den);
      else
        sink = 0.0;
      T qsm = K.qs0_crt / den;
      if (qsz > qsm) {
        T factor = dts * 1.0e-3 * xexp(0.09 * (tz - tice));
        sink = sink + factor / (1.0 + factor) * (qsz - qsm);
      }
      sink = fmin(qsz, sink);
      qsz = qsz - sink;
      qgz = qgz + sink;
    }
    if ((qgz > 1.0e-7) && (tz < K.tice0)) {
      if (qlz > 1.0e-6) {
        T qden = qgz * den;
        T factor = dts * K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
        pgacw = factor / (1.0 + factor) * qlz;
      } else {
        pgacw = 0.0;
      }
      if (qrz > 1.0e-6) {
        pgacr = fmin(dts * acr3d<T>(vtgz, vtrz, qrz, qgz, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den),
                     qrz);
      } else {
        pgacr = 0.0;
      }
      T sink = pgacr + pgacw;
      T factor = fmin(sink, dim(tice, tz) / icpk) / fmax(sink, QRMIN);
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

// -------------------------------------- pointwise blocks of the step body
// Cloud ice melting at and below the first level warmer than tice, at the
// start of sedimentation (microphysics.py:706-746).
template <typename T>
SHP void sedi_ice_melt(const MpConst& K, T qv, T& ql, T& qr, T& qi, T qs, T qg, T& tz) {
  const T lhi = K.LI00 + K.DC_ICE * tz;
  T q_liq = ql + qr;
  T q_sol = qi + qs + qg;
  T cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
  const T icpk = lhi / cvm;
  const T tc = tz - K.tice;
  if ((qi > QCMIN) && (tc > 0.0)) {
    const T sink = fmin(qi, K.fac_imlt * tc / icpk);
    const T tmp = fmin(sink, dim(K.ql_mlt, ql));
    ql = ql + tmp;
    qr = qr + sink - tmp;
    qi = qi - sink;
    q_liq = q_liq + sink;
    q_sol = q_sol - sink;
    cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
    tz = tz - sink * lhi / cvm;
  }
}

// Instant melting of cloud ice above tice, or freezing of cloud water below
// t_wfr, at the start of icloud (microphysics.py:1298-1339); returns the
// liquid and solid totals and cvm that icloud_processes starts from.
template <typename T>
SHP void icloud_melt_freeze(const MpConst& K, T qv, T& ql, T& qr, T& qi, T& qs, T qg, T& tz, T den, T& q_liq,
                            T& q_sol, T& cvm) {
  const T lhi = K.LI00 + K.DC_ICE * tz;
  q_liq = ql + qr;
  q_sol = qi + qs + qg;
  cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
  const T icpk = lhi / cvm;
  if ((tz > K.tice) && (qi > QCMIN)) {
    const T melt = fmin(qi, K.fac_imlt * (tz - K.tice) / icpk);
    const T tmp = fmin(melt, dim(K.ql_mlt, ql));
    ql = ql + tmp;
    qr = qr + melt - tmp;
    qi = qi - melt;
    q_liq = q_liq + melt;
    q_sol = q_sol - melt;
    cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
    tz = tz - melt * lhi / cvm;
  } else if ((tz < K.t_wfr) && (ql > QCMIN)) {
    const T dtmp = K.t_wfr - tz;
    const T factor = fmin(1.0, dtmp / DT_FR);
    const T sink = fmin(ql * factor, dtmp / icpk);
    const T qi_crt = K.qi_gen * fmin(K.qi_lim, 0.1 * (K.tice - tz)) / den;
    const T tmp = fmin(sink, dim(qi_crt, qi));
    ql = ql - sink;
    qs = qs + sink - tmp;
    qi = qi + tmp;
    q_liq = q_liq - sink;
    q_sol = q_sol + sink;
    cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
    tz = tz + sink * lhi / cvm;
  }
}

// The pointwise part of fix_negative (microphysics.py:202-240): negative
// species borrow from the next one in the chain ice -> snow -> graupel ->
// rain -> cloud water -> vapour, with the latent heat.
template <typename T>
SHP void fix_negative_point(const MpConst& K, T& qv, T& ql, T& qr, T& qi, T& qs, T& qg, T& tz) {
  const T cvm = K.c_air + qv * K.c_vap + (qr + ql) * K.C_LIQ + (qi + qs + qg) * K.C_ICE;
  const T lcpk = (K.lv00 + K.d0_vap * tz) / cvm;
  const T icpk = (K.LI00 + K.DC_ICE * tz) / cvm;
  if (qi < 0.0) {
    qs = qs + qi;
    qi = 0.0;
  }
  if (qs < 0.0) {
    qg = qg + qs;
    qs = 0.0;
  }
  if (qg < 0.0) {
    qr = qr + qg;
    tz = tz - qg * icpk;
    qg = 0.0;
  }
  if (qr < 0.0) {
    ql = ql + qr;
    qr = 0.0;
  }
  if (ql < 0.0) {
    qv = qv + ql;
    tz = tz - ql * lcpk;
    ql = 0.0;
  }
}

}  // namespace shield
