// Hand-written adjoints (vector-Jacobian products) of the pointwise GFDL
// microphysics processes in mp_physics.cuh, in FP64.
//
// Convention: f_b(primal inputs..., adjoints...) receives the primal values
// at the ENTRY of the forward routine. For every state variable the routine
// updates in place, the adjoint argument holds d(loss)/d(output) on entry
// and d(loss)/d(input) on return; for inputs the routine only reads
// (density, fall speeds, ...), the adjoint argument is accumulated (+=).
//
// Each adjoint first re-runs its forward routine, keeping the intermediate
// values, then walks the statements backwards. Branch decisions are those of
// the forward at the given point (the VJP of the piecewise-smooth map on the
// branch it takes). Ties of fmin/fmax go to the first argument when
// a <= b (fmin) or a >= b (fmax); the derivative there is one-sided.
#pragma once

#include "mp_physics.cuh"

// The larger adjoints are inlined into their (out-of-line) stage reverses;
// SHIELD_ADJ_NOINLINE makes them calls instead (measured slower: the call
// sequences cost more than the instruction-cache footprint they save).
#if defined(__CUDACC__) && defined(SHIELD_ADJ_NOINLINE)
#define SHB static __host__ __device__ __noinline__
#elif defined(__CUDACC__)
#define SHB static __host__ __device__ __forceinline__
#else
#define SHB static inline
#endif

namespace shield {

SHP bool min_first(double a, double b) { return a <= b; }
SHP bool max_first(double a, double b) { return a >= b; }

// --------------------------------------------------- saturation (:52-145)
// q = wqs1(ta, den), dqdt from wqs2; accumulate ta_b, den_b from the
// adjoints of q and dqdt.
SHP void wqs2_b(const MpConst& K, double ta, double den, double q, double dqdt, double q_b, double dqdt_b,
                double& ta_b, double& den_b) {
  (void)dqdt;
  const double g = (K.DC_VAP + K.LV0 / ta) / (K.RVGAS * ta);
  const double gp = -(K.DC_VAP + 2.0 * K.LV0 / ta) / (K.RVGAS * ta * ta);
  const double qb = q_b + dqdt_b * g;
  ta_b += dqdt_b * q * gp + qb * q * (g - 1.0 / ta);
  den_b -= qb * q / den;
}

SHP void iqs2_b(const MpConst& K, double ta, double den, double q, double dqdt, double q_b, double dqdt_b,
                double& ta_b, double& den_b) {
  if (ta < K.TICE) {
    if (ta >= K.T_SAT_MIN) {
      const double g = (K.D2ICE + K.LI2 / ta) / (K.RVGAS * ta);
      const double gp = -(K.D2ICE + 2.0 * K.LI2 / ta) / (K.RVGAS * ta * ta);
      const double qb = q_b + dqdt_b * g;
      ta_b += dqdt_b * q * gp + qb * q * (g - 1.0 / ta);
      den_b -= qb * q / den;
    } else {
      const double c = (K.D2ICE + K.LI2 / K.T_SAT_MIN) / (K.RVGAS * K.T_SAT_MIN);
      den_b -= (q_b + dqdt_b * c) * q / den;
    }
  } else if (ta <= K.TICE + 102.0) {
    wqs2_b(K, ta, den, q, dqdt, q_b, dqdt_b, ta_b, den_b);
  } else {
    const double tt = K.TICE + 102.0;
    const double c = (K.DC_VAP + K.LV0 / tt) / (K.RVGAS * tt);
    den_b -= (q_b + dqdt_b * c) * q / den;
  }
}
SHP void iqs1_b(const MpConst& K, double ta, double den, double q, double q_b, double& ta_b, double& den_b) {
  iqs2_b(K, ta, den, q, 0.0, q_b, 0.0, ta_b, den_b);
}
SHP void wqs1_b(const MpConst& K, double ta, double den, double q, double q_b, double& ta_b, double& den_b) {
  wqs2_b(K, ta, den, q, 0.0, q_b, 0.0, ta_b, den_b);
}

// cvm = c_air + qv c_vap + q_liq C_LIQ + q_sol C_ICE
SHP void cvm_b(const MpConst& K, double cvm_bar, double& qv_b, double& q_liq_b, double& q_sol_b) {
  qv_b += cvm_bar * K.c_vap;
  q_liq_b += cvm_bar * K.C_LIQ;
  q_sol_b += cvm_bar * K.C_ICE;
}

// ------------------------------------------ acr3d, smlt, gmlt (:148-179)
SHP void acr3d_b(double v1, double v2, double q1, double q2, double c, double cac_ik, double cac_i1k, double cac_i2k,
                 double rho, double y_b, double& v1_b, double& v2_b, double& q1_b, double& q2_b, double& rho_b) {
  const double t1 = sqrt(q1 * rho);
  const double s1 = sqrt(q2 * rho);
  const double s2 = sqrt(s1);
  const double st1 = sqrt(t1);
  const double dv = v1 - v2;
  const double adv = fabs(dv);
  const double B = cac_ik * t1 + cac_i1k * st1 * s2 + cac_i2k * s1;
  const double pre = c * adv * q1 * s2;  // y = pre * B
  const double pre_b = y_b * B;
  const double B_b = y_b * pre;
  const double adv_b = pre_b * c * q1 * s2;
  q1_b += pre_b * c * adv * s2;
  double s2_b = pre_b * c * adv * q1;
  double t1_b = B_b * cac_ik;
  const double st1_b = B_b * cac_i1k * s2;
  s2_b += B_b * cac_i1k * st1;
  double s1_b = B_b * cac_i2k;
  const double sgn = dv >= 0.0 ? 1.0 : -1.0;
  v1_b += adv_b * sgn;
  v2_b -= adv_b * sgn;
  t1_b += st1_b * 0.5 / st1;
  s1_b += s2_b * 0.5 / s2;
  const double x1_b = t1_b * 0.5 / t1;  // x1 = q1 rho
  const double x2_b = s1_b * 0.5 / s1;  // x2 = q2 rho
  q1_b += x1_b * rho;
  q2_b += x2_b * rho;
  rho_b += x1_b * q1 + x2_b * q2;
}

// y = (c0 tc / rho - c1 dqs) (c2 sqrt(x) + c3 x^0.65625 sqrt(rhofac)) + c4 tc (psacw + psacr)
SHP void smlt_b(double tc, double dqs, double qsrho, double psacw, double psacr, double c_0, double c_1, double c_2,
                double c_3, double c_4, double rho, double rhofac, double y_b, double& tc_b, double& dqs_b,
                double& qsrho_b, double& psacw_b, double& psacr_b, double& rho_b, double& rhofac_b) {
  const double A = c_0 * tc / rho - c_1 * dqs;
  const double sx = sqrt(qsrho);
  const double px = xpow(qsrho, 0.65625);
  const double sr = sqrt(rhofac);
  const double Bv = c_2 * sx + c_3 * px * sr;
  const double A_b = y_b * Bv;
  const double B_b = y_b * A;
  tc_b += A_b * c_0 / rho + y_b * c_4 * (psacw + psacr);
  rho_b -= A_b * c_0 * tc / (rho * rho);
  dqs_b -= A_b * c_1;
  qsrho_b += B_b * (c_2 * 0.5 / sx + c_3 * sr * 0.65625 * px / qsrho);
  rhofac_b += B_b * c_3 * px * 0.5 / sr;
  psacw_b += y_b * c_4 * tc;
  psacr_b += y_b * c_4 * tc;
}

// y = (c0 tc / rho - c1 dqs) (c2 sqrt(x) + c3 x^0.6875 / rho^0.25) + c4 tc (pgacw + pgacr)
SHP void gmlt_b(double tc, double dqs, double qgrho, double pgacw, double pgacr, double c_0, double c_1, double c_2,
                double c_3, double c_4, double rho, double y_b, double& tc_b, double& dqs_b, double& qgrho_b,
                double& pgacw_b, double& pgacr_b, double& rho_b) {
  const double A = c_0 * tc / rho - c_1 * dqs;
  const double sx = sqrt(qgrho);
  const double px = xpow(qgrho, 0.6875);
  const double pr = xpow(rho, 0.25);
  const double Bv = c_2 * sx + c_3 * px / pr;
  const double A_b = y_b * Bv;
  const double B_b = y_b * A;
  tc_b += A_b * c_0 / rho + y_b * c_4 * (pgacw + pgacr);
  rho_b += -A_b * c_0 * tc / (rho * rho) - B_b * c_3 * px * 0.25 / (pr * rho);
  dqs_b -= A_b * c_1;
  qgrho_b += B_b * (c_2 * 0.5 / sx + c_3 * 0.6875 * px / (qgrho * pr));
  pgacw_b += y_b * c_4 * tc;
  pgacr_b += y_b * c_4 * tc;
}

// ------------------------------------------------ revap_racc (:182-265)
SHB void revap_racc_b(const MpConst& K, double dt, double h_var, double qg, double qi, double ql, double qr, double qs,
                      double qv, double tz, double den, double denfac, double& qg_b, double& qi_b, double& ql_b,
                      double& qr_b, double& qs_b, double& qv_b, double& tz_b, double& den_b, double& denfac_b) {
  if (!((tz > K.t_wfr) && (qr > QRMIN))) return;
  // forward
  const double lhl = K.lv00 + K.d0_vap * tz;
  const double q_liq = ql + qr;
  const double q_sol = qi + qs + qg;
  const double cvm = cvm_of(K, qv, q_liq, q_sol);
  const double lcpk = lhl / cvm;
  const double tin = tz - lcpk * ql;
  const double qpz = qv + ql;
  double dqsdt;
  const double qsat = wqs2(K, tin, den, dqsdt);
  const double mq = fmax(qpz, QCMIN);
  const double hq = h_var * mq;
  const double dqh0 = fmax(ql, hq);
  const double dqh = fmin(dqh0, 0.2 * qpz);
  const double dqv = qsat - qv;
  const double q_minus = qpz - dqh;
  const double q_plus = qpz + dqh;
  const bool cb = (dqv > QVMIN) && (qsat > q_minus);
  bool c_plus = false;
  int sel = 0;
  double dq = 0.0, qden = 0.0, t2 = 0.0, sq1 = 0.0, p725 = 0.0, P = 0.0, num = 0.0, den2 = 0.0, evap0 = 0.0;
  double e2d = 1.0, e2 = 0.0, evap = 0.0, qr1 = qr, qv1 = qv, q_liq1 = q_liq, cvm1 = cvm;
  if (cb) {
    c_plus = qsat > q_plus;
    dq = c_plus ? qsat - qpz : 0.25 * sq(q_minus - qsat) / dqh;
    qden = qr * den;
    t2 = tin * tin;
    sq1 = sqrt(qden);
    p725 = xexp(0.725 * xlog(qden));
    P = K.crevp[1] * sq1 + K.crevp[2] * p725;
    num = K.crevp[0] * t2 * dq * P;
    den2 = K.crevp[3] * t2 + K.crevp[4] * qsat * den;
    evap0 = num / den2;
    const double e1 = dt * evap0;
    e2d = 1.0 + lcpk * dqsdt;
    e2 = dqv / e2d;
    const double m12 = fmin(e1, e2);
    sel = min_first(qr, m12) ? 0 : (min_first(e1, e2) ? 1 : 2);
    evap = fmin(qr, m12);
    qr1 = qr - evap;
    qv1 = qv + evap;
    q_liq1 = q_liq - evap;
    cvm1 = cvm_of(K, qv1, q_liq1, q_sol);
  }
  const bool cc = (qr1 > QRMIN) && (ql > 1.0e-6) && (qsat < q_minus);
  // reverse: accretion
  double qr1_b = qr_b, ql0_b = ql_b;
  if (cc) {
    const double x = qr1 * den;
    const double px = xexp(0.95 * xlog(x));
    const double s0 = dt * denfac * K.cracw * px;
    const double f = s0 / (1.0 + s0);
    const double sink_b = qr_b - ql_b;
    ql0_b = ql_b + sink_b * f;
    const double s0_b = sink_b * ql / ((1.0 + s0) * (1.0 + s0));
    denfac_b += s0_b * dt * K.cracw * px;
    const double x_b = s0_b * s0 * 0.95 / x;
    qr1_b = qr_b + x_b * den;
    den_b += x_b * qr1;
  }
  // reverse: evaporation
  double qv0_b = qv_b, qr0_b = qr1_b, tz0_b = tz_b;
  double lhl_b = 0.0, q_liq_b = 0.0, q_sol_b = 0.0, lcpk_b = 0.0, tin_b = 0.0, qsat_b = 0.0, dqsdt_b = 0.0;
  double qpz_b = 0.0, dqh_b = 0.0, qm_b = 0.0, dqv_b = 0.0;
  if (cb) {
    const double tz1_b = tz_b;
    double evap_b = -tz1_b * lhl / cvm1;
    lhl_b -= tz1_b * evap / cvm1;
    const double cvm1_b = tz1_b * evap * lhl / (cvm1 * cvm1);
    double qv1_b = qv_b, q_liq1_b = 0.0;
    cvm_b(K, cvm1_b, qv1_b, q_liq1_b, q_sol_b);
    q_liq_b += q_liq1_b;
    evap_b -= q_liq1_b;
    qv0_b = qv1_b;
    evap_b += qv1_b;
    qr0_b = qr1_b;
    evap_b -= qr1_b;
    double e1_b = 0.0, e2_b = 0.0;
    if (sel == 0)
      qr0_b += evap_b;
    else if (sel == 1)
      e1_b = evap_b;
    else
      e2_b = evap_b;
    dqv_b += e2_b / e2d;
    const double e2d_b = -e2_b * e2 / e2d;
    lcpk_b += e2d_b * dqsdt;
    dqsdt_b += e2d_b * lcpk;
    const double evap0_b = dt * e1_b;
    const double num_b = evap0_b / den2;
    const double den2_b = -evap0_b * evap0 / den2;
    double t2_b = den2_b * K.crevp[3];
    qsat_b += den2_b * K.crevp[4] * den;
    den_b += den2_b * K.crevp[4] * qsat;
    t2_b += num_b * K.crevp[0] * dq * P;
    const double dq_b = num_b * K.crevp[0] * t2 * P;
    const double P_b = num_b * K.crevp[0] * t2 * dq;
    const double qden_b = P_b * (K.crevp[1] * 0.5 / sq1 + K.crevp[2] * 0.725 * p725 / qden);
    qr0_b += qden_b * den;
    den_b += qden_b * qr;
    tin_b += 2.0 * tin * t2_b;
    if (c_plus) {
      qsat_b += dq_b;
      qpz_b -= dq_b;
    } else {
      const double g = dq_b * 0.5 * (q_minus - qsat) / dqh;
      qm_b += g;
      qsat_b -= g;
      dqh_b -= dq_b * dq / dqh;
    }
  }
  // reverse: common part
  qpz_b += qm_b;
  dqh_b -= qm_b;
  qsat_b += dqv_b;
  qv0_b -= dqv_b;
  double dqh0_b = 0.0;
  if (min_first(dqh0, 0.2 * qpz))
    dqh0_b = dqh_b;
  else
    qpz_b += 0.2 * dqh_b;
  if (max_first(ql, hq)) {
    ql0_b += dqh0_b;
  } else if (max_first(qpz, QCMIN)) {
    qpz_b += dqh0_b * h_var;
  }
  wqs2_b(K, tin, den, qsat, dqsdt, qsat_b, dqsdt_b, tin_b, den_b);
  qv0_b += qpz_b;
  ql0_b += qpz_b;
  tz0_b += tin_b;
  lcpk_b -= tin_b * ql;
  ql0_b -= tin_b * lcpk;
  lhl_b += lcpk_b / cvm;
  const double cvm_bar = -lcpk_b * lcpk / cvm;
  cvm_b(K, cvm_bar, qv0_b, q_liq_b, q_sol_b);
  qi_b += q_sol_b;
  qs_b += q_sol_b;
  qg_b += q_sol_b;
  ql0_b += q_liq_b;
  qr0_b += q_liq_b;
  tz0_b += lhl_b * K.d0_vap;
  qv_b = qv0_b;
  ql_b = ql0_b;
  qr_b = qr0_b;
  tz_b = tz0_b;
}

// ------------------------------------------------------- fall speeds
// vtr = rain_fspeed(qr, den) (:344-372)
SHP void rain_fspeed_b(const MpConst& K, double qrz, double den, double v_b, double& qr_b, double& den_b) {
  if (K.const_vr) return;
  if (qrz < THR) return;
  const double qden = qrz * den;
  const double r = fmin(10.0, SFCRHO / den);
  const double sr = sqrt(r);
  const double e = xexp(0.2 * xlog(qden / NORMR));
  const double v = K.vr_fac * VCONR * sr * e;
  // fmin(vr_max, fmax(VR_MIN, v))
  const double m = fmax(VR_MIN, v);
  if (min_first(K.vr_max, m)) return;
  if (max_first(VR_MIN, v)) return;
  const double sr_b = v_b * K.vr_fac * VCONR * e;
  const double e_b = v_b * K.vr_fac * VCONR * sr;
  const double qden_b = e_b * 0.2 * e / qden;
  qr_b += qden_b * den;
  den_b += qden_b * qrz;
  if (min_first(10.0, SFCRHO / den)) return;
  const double r_b = sr_b * 0.5 / sr;
  den_b -= r_b * SFCRHO / (den * den);
}

// fall_speed (:268-341): vtg, vti, vts from qg, qi, qs, tk, den
SHB void fall_speed_b(const MpConst& K, double qg, double qi, double qs, double tk, double den, double vtg_b,
                      double vti_b, double vts_b, double& qg_b, double& qi_b, double& qs_b, double& tk_b,
                      double& den_b) {
  const double rr = SFCRHO / den;
  const bool rcap = min_first(10.0, rr);
  const double rhof = sqrt(fmin(10.0, rr));
  double rhof_b = 0.0;
  if (!K.const_vi && !(qi < THI)) {
    const double vi0 = 0.01 * K.vi_fac;
    const double tc = tk - K.tice;
    const double x = qi * den;
    const double lx = xlog(x);
    const double a = 3.0 + lx / K.log_10;
    const double bpoly = tc * (AA * tc + BB) + CC;
    const double u = a * bpoly + DD_FS * tc + EE;
    const double eu = xexp(K.log_10 * u);
    const double v = vi0 * eu * 0.8;
    const double m = fmax(VF_MIN, v);
    if (!min_first(K.vi_max, m) && !max_first(VF_MIN, v)) {
      const double u_b = vti_b * vi0 * 0.8 * eu * K.log_10;
      const double a_b = u_b * bpoly;
      const double bp_b = u_b * a;
      // bpoly = tc (AA tc + BB) + CC: d/dtc = 2 AA tc + BB
      const double tc_b = bp_b * (AA * tc + BB + tc * AA) + u_b * DD_FS;
      tk_b += tc_b;
      const double x_b = a_b / (K.log_10 * x);
      qi_b += x_b * den;
      den_b += x_b * qi;
    }
  }
  if (!K.const_vs && !(qs < THS)) {
    const double x = qs * den / NORMS;
    const double e = xexp(0.0625 * xlog(x));
    const double v = K.vs_fac * VCONS * rhof * e;
    const double m = fmax(VF_MIN, v);
    if (!min_first(K.vs_max, m) && !max_first(VF_MIN, v)) {
      rhof_b += vts_b * K.vs_fac * VCONS * e;
      const double e_b = vts_b * K.vs_fac * VCONS * rhof;
      const double x_b = e_b * 0.0625 * e / x;
      qs_b += x_b * den / NORMS;
      den_b += x_b * qs / NORMS;
    }
  }
  if (!K.const_vg && !(qg < THG)) {
    const double x = qg * den / NORMG;
    const double r2 = sqrt(x), r4 = sqrt(r2), r8 = sqrt(r4);
    const double v = K.vg_fac * VCONG * rhof * r8;
    const double m = fmax(VF_MIN, v);
    if (!min_first(K.vg_max, m) && !max_first(VF_MIN, v)) {
      rhof_b += vtg_b * K.vg_fac * VCONG * r8;
      const double r8_b = vtg_b * K.vg_fac * VCONG * rhof;
      // r8 = x^(1/8) through three square roots
      const double r4_b = r8_b * 0.5 / r8;
      const double r2_b = r4_b * 0.5 / r4;
      const double x_b = r2_b * 0.5 / r2;
      qg_b += x_b * den / NORMG;
      den_b += x_b * qg / NORMG;
    }
  }
  if (rhof_b != 0.0 && !rcap) {
    const double rr_b = rhof_b * 0.5 / rhof;
    den_b -= rr_b * SFCRHO / (den * den);
  }
}

// -------------------------------------------------- autoconversion (:375-428)
SHB void autoconv_no_subgrid_var_b(const MpConst& K, double qlz, double qrz, double tz, double den, double ccn,
                                   double c_praut, double& ql_b, double& qr_b, double& den_b, double& ccn_b,
                                   double& c_praut_b) {
  (void)qrz;
  if (!(tz > K.t_wfr)) return;
  const double qc0 = K.fac_rc * ccn;
  const double qc = K.use_ccn ? qc0 : qc0 / den;
  const double dq = qlz - qc;
  if (!(dq > 0.0)) return;
  const double pw = xexp(K.so3 * xlog(qlz));
  const double rate = K.dt_rain * c_praut * den * pw;
  // sink = fmin(dq, rate); ql -= sink; qr += sink
  const double sink_b = qr_b - ql_b;
  if (min_first(dq, rate)) {
    ql_b += sink_b;
    const double qc_b = -sink_b;
    if (K.use_ccn) {
      ccn_b += qc_b * K.fac_rc;
    } else {
      ccn_b += qc_b * K.fac_rc / den;
      den_b -= qc_b * qc / den;
    }
  } else {
    c_praut_b += sink_b * K.dt_rain * den * pw;
    den_b += sink_b * K.dt_rain * c_praut * pw;
    ql_b += sink_b * rate * K.so3 / qlz;
  }
}

SHB void autoconv_subgrid_var_b(const MpConst& K, double qlz, double qrz, double tz, double den, double ccn,
                                double c_praut, double dl, double& ql_b, double& qr_b, double& den_b, double& ccn_b,
                                double& c_praut_b, double& dl_b) {
  (void)qrz;
  if (!(tz > K.t_wfr + DT_FR)) return;
  const double dl1 = fmax(1.0e-6, dl);
  const double hq = 0.5 * qlz;
  const double dl2 = fmin(dl1, hq);
  const double qc0 = K.fac_rc * ccn;
  const double qc = K.use_ccn ? qc0 : qc0 / den;
  const double dq = 0.5 * (qlz + dl2 - qc);
  if (!(dq > 0.0)) return;
  const double r = dq / dl2;
  const double f = fmin(1.0, r);
  const double pw = xexp(K.so3 * xlog(qlz));
  const double g = K.dt_rain * c_praut * den * pw;  // sink = f * g (evaluated as ((f dt) c) den pw)
  const double sink_b = qr_b - ql_b;
  const double g_b = sink_b * f;
  const double f_b = sink_b * g;
  double dq_b = 0.0, dl2_b = 0.0;
  if (!min_first(1.0, r)) {
    dq_b += f_b / dl2;
    dl2_b -= f_b * r / dl2;
  }
  c_praut_b += g_b * K.dt_rain * den * pw;
  den_b += g_b * K.dt_rain * c_praut * pw;
  ql_b += g_b * g * K.so3 / qlz;
  // dq = 0.5 (qlz + dl2 - qc)
  ql_b += 0.5 * dq_b;
  dl2_b += 0.5 * dq_b;
  const double qc_b = -0.5 * dq_b;
  if (K.use_ccn) {
    ccn_b += qc_b * K.fac_rc;
  } else {
    ccn_b += qc_b * K.fac_rc / den;
    den_b -= qc_b * qc / den;
  }
  if (min_first(dl1, hq)) {
    if (max_first(1.0e-6, dl)) return;
    dl_b += dl2_b;
  } else {
    ql_b += 0.5 * dl2_b;
  }
}

// ---------------------------------------------- icloud_processes (:853-1227)
// The routine is a sequence of process blocks, each updating the state
// (qg, qi, ql, qr, qs, tz, q_liq, q_sol, cvm). The adjoint replays the
// blocks to obtain each block's entry state, then reverses them in order.
struct IcState {
  double qg, qi, ql, qr, qs, tz, q_liq, q_sol, cvm;
};
// adjoints of the read-only inputs of the routine
struct IcIn {
  double qv, den, denfac, vtg, vtr, vts, p1, di;
};

// d fac / d(qden, den) of fac = C qden / sqrt(den sqrt(sqrt(qden))), given fac_b
SHP void riming_fac_b(double C, double qden, double den, double fac, double fac_b, double& qden_b, double& den_b) {
  const double r2 = sqrt(qden), r4 = sqrt(r2);
  const double sD = sqrt(den * r4);
  qden_b += fac_b * C / sD;
  const double sD_b = -fac_b * fac / sD;
  const double D_b = sD_b * 0.5 / sD;
  den_b += D_b * r4;
  const double r4_b = D_b * den;
  const double r2_b = r4_b * 0.5 / r4;
  qden_b += r2_b * 0.5 / r2;
}

// cvm' = cvm_of(qv, q_liq', q_sol') and tz' = tz + sgn * s * lh / cvm' (the
// closing statements of every transfer block): adjoint, given the block's
// output adjoints Zb (overwritten with the adjoints of q_liq', q_sol' and
// of the entry tz; cvm's entry adjoint is cleared). Returns s_b.
SHP double close_transfer_b(const MpConst& K, double sgn, double s, double lh, double cvm1, IcState& Zb, double& qv_b,
                            double& lh_b) {
  const double s_b = sgn * Zb.tz * lh / cvm1;
  lh_b += sgn * Zb.tz * s / cvm1;
  const double cvm1_b = Zb.cvm - sgn * Zb.tz * s * lh / (cvm1 * cvm1);
  qv_b += cvm1_b * K.c_vap;
  Zb.q_liq += cvm1_b * K.C_LIQ;
  Zb.q_sol += cvm1_b * K.C_ICE;
  Zb.cvm = 0.0;
  return s_b;
}

// snow melting and accretion above freezing (:932-1000)
SHP void ic_snow_melt(const MpConst& K, IcState& Z, double qv, double den, double denfac, double vtr, double vts,
                      double dqs0, double lhi0, double icpk0) {
  const double tc = Z.tz - K.tice;
  double psacw = 0.0, psacr = 0.0, pracs = 0.0;
  if (Z.ql > QRMIN) {
    const double factor = denfac * K.csacw * xexp(0.8125 * xlog(Z.qs * den));
    psacw = factor / (1.0 + K.dts * factor) * Z.ql;
  }
  if (Z.qr > QRMIN) {
    psacr = fmin(acr3d<double>(vts, vtr, Z.qr, Z.qs, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den),
                 Z.qr * K.rdts);
    pracs = acr3d<double>(vtr, vts, Z.qs, Z.qr, K.cracs, K.acco[0][0], K.acco[1][0], K.acco[2][0], den);
  }
  const double psmlt = fmax(0.0, smlt<double>(tc, dqs0, Z.qs * den, psacw, psacr, K.csmlt[0], K.csmlt[1], K.csmlt[2],
                                              K.csmlt[3], K.csmlt[4], den, denfac));
  const double sink = fmin(Z.qs, fmin(K.dts * (psmlt + pracs), tc / icpk0));
  Z.qs = Z.qs - sink;
  const double tmp = fmin(sink, dim(K.qs_mlt, Z.ql));
  Z.ql = Z.ql + tmp;
  Z.qr = Z.qr + sink - tmp;
  Z.q_liq = Z.q_liq + sink;
  Z.q_sol = Z.q_sol - sink;
  Z.cvm = cvm_of(K, qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz - sink * lhi0 / Z.cvm;
}
SHP void ic_snow_melt_b(const MpConst& K, const IcState& Z, const IcIn& I, double dqs0, double lhi0, double icpk0,
                        IcState& Zb, IcIn& Ib, double& dqs0_b, double& lhi0_b, double& icpk0_b) {
  const double den = I.den, denfac = I.denfac;
  const double tc = Z.tz - K.tice;
  const double xs = Z.qs * den;
  double psacw = 0.0, psacr = 0.0, pracs = 0.0, a1 = 0.0, fac = 0.0, e8 = 0.0;
  if (Z.ql > QRMIN) {
    e8 = xexp(0.8125 * xlog(xs));
    fac = denfac * K.csacw * e8;
    psacw = fac / (1.0 + K.dts * fac) * Z.ql;
  }
  if (Z.qr > QRMIN) {
    a1 = acr3d<double>(I.vts, I.vtr, Z.qr, Z.qs, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den);
    psacr = fmin(a1, Z.qr * K.rdts);
    pracs = acr3d<double>(I.vtr, I.vts, Z.qs, Z.qr, K.cracs, K.acco[0][0], K.acco[1][0], K.acco[2][0], den);
  }
  const double sm = smlt<double>(tc, dqs0, xs, psacw, psacr, K.csmlt[0], K.csmlt[1], K.csmlt[2], K.csmlt[3],
                                 K.csmlt[4], den, denfac);
  const double psmlt = fmax(0.0, sm);
  const double r1 = K.dts * (psmlt + pracs);
  const double r2 = tc / icpk0;
  const double m = fmin(r1, r2);
  const double sink = fmin(Z.qs, m);
  const double dm = dim(K.qs_mlt, Z.ql);
  const double cvm1 = cvm_of(K, I.qv, Z.q_liq + sink, Z.q_sol - sink);
  // reverse
  double sink_b = close_transfer_b(K, -1.0, sink, lhi0, cvm1, Zb, Ib.qv, lhi0_b);
  sink_b += Zb.q_liq - Zb.q_sol;
  sink_b += Zb.qr;
  double tmp_b = -Zb.qr + Zb.ql;
  if (min_first(sink, dm)) {
    sink_b += tmp_b;
  } else if (K.qs_mlt - Z.ql > 0.0) {
    Zb.ql -= tmp_b;
  }
  sink_b -= Zb.qs;
  double m_b = 0.0;
  if (min_first(Z.qs, m))
    Zb.qs += sink_b;
  else
    m_b = sink_b;
  double r1_b = 0.0, tc_b = 0.0;
  if (min_first(r1, r2)) {
    r1_b = m_b;
  } else {
    tc_b += m_b / icpk0;
    icpk0_b -= m_b * r2 / icpk0;
  }
  const double psmlt_b = K.dts * r1_b;
  const double pracs_b = K.dts * r1_b;
  double xs_b = 0.0, psacw_b = 0.0, psacr_b = 0.0;
  if (!max_first(0.0, sm))
    smlt_b(tc, dqs0, xs, psacw, psacr, K.csmlt[0], K.csmlt[1], K.csmlt[2], K.csmlt[3], K.csmlt[4], den, denfac,
           psmlt_b, tc_b, dqs0_b, xs_b, psacw_b, psacr_b, Ib.den, Ib.denfac);
  if (Z.qr > QRMIN) {
    acr3d_b(I.vtr, I.vts, Z.qs, Z.qr, K.cracs, K.acco[0][0], K.acco[1][0], K.acco[2][0], den, pracs_b, Ib.vtr, Ib.vts,
            Zb.qs, Zb.qr, Ib.den);
    if (min_first(a1, Z.qr * K.rdts))
      acr3d_b(I.vts, I.vtr, Z.qr, Z.qs, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den, psacr_b, Ib.vts,
              Ib.vtr, Zb.qr, Zb.qs, Ib.den);
    else
      Zb.qr += psacr_b * K.rdts;
  }
  if (Z.ql > QRMIN) {
    const double d1 = 1.0 + K.dts * fac;
    Zb.ql += psacw_b * fac / d1;
    const double fac_b = psacw_b * Z.ql / (d1 * d1);
    Ib.denfac += fac_b * K.csacw * e8;
    xs_b += fac_b * denfac * K.csacw * 0.8125 * e8 / xs;
  }
  Zb.qs += xs_b * den;
  Ib.den += xs_b * Z.qs;
  Zb.tz += tc_b;
}

// graupel melting above freezing (:1002-1035); lhi, icpk from the entry tz, cvm
SHP void ic_graupel_melt(const MpConst& K, IcState& Z, double qv, double den, double vtg, double vtr, double dqs0) {
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  const double tc = Z.tz - K.tice;
  double pgacr = 0.0, pgacw = 0.0;
  if (Z.qr > QRMIN)
    pgacr = fmin(acr3d<double>(vtg, vtr, Z.qr, Z.qg, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den),
                 K.rdts * Z.qr);
  const double qden = Z.qg * den;
  if (Z.ql > QRMIN) {
    const double factor = K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
    pgacw = factor / (1.0 + K.dts * factor) * Z.ql;
  }
  double pgmlt = K.dts * gmlt<double>(tc, dqs0, qden, pgacw, pgacr, K.cgmlt[0], K.cgmlt[1], K.cgmlt[2], K.cgmlt[3],
                                      K.cgmlt[4], den);
  pgmlt = fmin(fmax(0.0, pgmlt), fmin(Z.qg, tc / icpk));
  Z.qg = Z.qg - pgmlt;
  Z.qr = Z.qr + pgmlt;
  Z.q_liq = Z.q_liq + pgmlt;
  Z.q_sol = Z.q_sol - pgmlt;
  Z.cvm = cvm_of(K, qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz - pgmlt * lhi / Z.cvm;
}
SHP void ic_graupel_melt_b(const MpConst& K, const IcState& Z, const IcIn& I, double dqs0, IcState& Zb, IcIn& Ib,
                           double& dqs0_b) {
  const double den = I.den;
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  const double tc = Z.tz - K.tice;
  double pgacr = 0.0, pgacw = 0.0, a2 = 0.0, fac = 0.0;
  if (Z.qr > QRMIN) {
    a2 = acr3d<double>(I.vtg, I.vtr, Z.qr, Z.qg, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den);
    pgacr = fmin(a2, K.rdts * Z.qr);
  }
  const double qden = Z.qg * den;
  if (Z.ql > QRMIN) {
    fac = K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
    pgacw = fac / (1.0 + K.dts * fac) * Z.ql;
  }
  const double gm = gmlt<double>(tc, dqs0, qden, pgacw, pgacr, K.cgmlt[0], K.cgmlt[1], K.cgmlt[2], K.cgmlt[3],
                                 K.cgmlt[4], den);
  const double pg0 = K.dts * gm;
  const double A = fmax(0.0, pg0);
  const double r = tc / icpk;
  const double B = fmin(Z.qg, r);
  const double pgmlt = fmin(A, B);
  const double cvm1 = cvm_of(K, I.qv, Z.q_liq + pgmlt, Z.q_sol - pgmlt);
  // reverse
  double lhi_b = 0.0;
  double pg_b = close_transfer_b(K, -1.0, pgmlt, lhi, cvm1, Zb, Ib.qv, lhi_b);
  pg_b += Zb.q_liq - Zb.q_sol + Zb.qr - Zb.qg;
  double pg0_b = 0.0, tc_b = 0.0, icpk_b = 0.0;
  if (min_first(A, B)) {
    if (!max_first(0.0, pg0)) pg0_b = pg_b;
  } else if (min_first(Z.qg, r)) {
    Zb.qg += pg_b;
  } else {
    tc_b += pg_b / icpk;
    icpk_b -= pg_b * r / icpk;
  }
  double qden_b = 0.0, pgacw_b = 0.0, pgacr_b = 0.0;
  gmlt_b(tc, dqs0, qden, pgacw, pgacr, K.cgmlt[0], K.cgmlt[1], K.cgmlt[2], K.cgmlt[3], K.cgmlt[4], den, K.dts * pg0_b,
         tc_b, dqs0_b, qden_b, pgacw_b, pgacr_b, Ib.den);
  if (Z.ql > QRMIN) {
    const double d1 = 1.0 + K.dts * fac;
    Zb.ql += pgacw_b * fac / d1;
    riming_fac_b(K.cgacw, qden, den, fac, pgacw_b * Z.ql / (d1 * d1), qden_b, Ib.den);
  }
  Zb.qg += qden_b * den;
  Ib.den += qden_b * Z.qg;
  if (Z.qr > QRMIN) {
    if (min_first(a2, K.rdts * Z.qr))
      acr3d_b(I.vtg, I.vtr, Z.qr, Z.qg, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den, pgacr_b, Ib.vtg,
              Ib.vtr, Zb.qr, Zb.qg, Ib.den);
    else
      Zb.qr += pgacr_b * K.rdts;
  }
  Zb.tz += tc_b;
  const double lhi_t = lhi_b + icpk_b / Z.cvm;
  Zb.cvm -= icpk_b * icpk / Z.cvm;
  Zb.tz += lhi_t * K.DC_ICE;
}

// cloud ice to snow (psaci, psaut) and graupel collecting ice (pgaci) below freezing (:1036-1072)
SHP void ic_ice_to_snow(const MpConst& K, IcState& Z, double den, double denfac, double di) {
  const double tc = Z.tz - K.tice;
  double psaci = 0.0;
  if (Z.qs > 1.0e-7) {
    const double factor = K.dts * denfac * K.csaci * xexp(0.05 * tc + 0.8125 * xlog(Z.qs * den));
    psaci = factor / (1.0 + factor) * Z.qi;
  }
  const double qim = K.qi0_crt / den;
  const double tmp = K.const_vi ? K.fac_i2s : K.fac_i2s * xexp(0.025 * tc);
  const double di1 = fmax(di, QRMIN);
  const double q_plus = Z.qi + di1;
  double psaut = 0.0;
  if (q_plus > (qim + QRMIN)) {
    double dq;
    if (qim > (Z.qi - di1))
      dq = (0.25 * sq(q_plus - qim)) / di1;
    else
      dq = Z.qi - qim;
    psaut = tmp * dq;
  }
  const double sink = fmin(0.75 * Z.qi, psaci + psaut);
  Z.qi = Z.qi - sink;
  Z.qs = Z.qs + sink;
  if (Z.qg > 1.0e-6) {
    const double factor = K.dts * K.cgaci * sqrt(den) * Z.qg;
    const double pgaci = factor / (1.0 + factor) * Z.qi;
    Z.qi = Z.qi - pgaci;
    Z.qg = Z.qg + pgaci;
  }
}
SHP void ic_ice_to_snow_b(const MpConst& K, const IcState& Z, const IcIn& I, IcState& Zb, IcIn& Ib) {
  const double den = I.den, denfac = I.denfac;
  const double tc = Z.tz - K.tice;
  double psaci = 0.0, fac = 0.0, ex = 0.0, xs = 0.0;
  if (Z.qs > 1.0e-7) {
    xs = Z.qs * den;
    ex = xexp(0.05 * tc + 0.8125 * xlog(xs));
    fac = K.dts * denfac * K.csaci * ex;
    psaci = fac / (1.0 + fac) * Z.qi;
  }
  const double qim = K.qi0_crt / den;
  const double tmpc = K.const_vi ? K.fac_i2s : K.fac_i2s * xexp(0.025 * tc);
  const double di1 = fmax(I.di, QRMIN);
  const double q_plus = Z.qi + di1;
  const bool aut = q_plus > (qim + QRMIN);
  const bool quad = qim > (Z.qi - di1);
  double dq = 0.0, psaut = 0.0;
  if (aut) {
    dq = quad ? (0.25 * sq(q_plus - qim)) / di1 : Z.qi - qim;
    psaut = tmpc * dq;
  }
  const double sx = psaci + psaut;
  const double sink = fmin(0.75 * Z.qi, sx);
  const double qi1 = Z.qi - sink;
  // reverse
  double qi1_b = Zb.qi;
  if (Z.qg > 1.0e-6) {
    const double sden = sqrt(den);
    const double fg = K.dts * K.cgaci * sden * Z.qg;
    const double d1 = 1.0 + fg;
    const double pga_b = Zb.qg - Zb.qi;
    qi1_b += pga_b * fg / d1;
    const double fg_b = pga_b * qi1 / (d1 * d1);
    Ib.den += fg_b * K.dts * K.cgaci * Z.qg * 0.5 / sden;
    Zb.qg += fg_b * K.dts * K.cgaci * sden;
  }
  const double sink_b = Zb.qs - qi1_b;
  Zb.qi = qi1_b;
  double sx_b = 0.0;
  if (min_first(0.75 * Z.qi, sx))
    Zb.qi += 0.75 * sink_b;
  else
    sx_b = sink_b;
  double tc_b = 0.0;
  if (aut) {
    const double tmpc_b = sx_b * dq;
    const double dq_b = sx_b * tmpc;
    double qim_b = 0.0, di1_b = 0.0;
    if (quad) {
      const double qp_b = dq_b * 0.5 * (q_plus - qim) / di1;
      qim_b -= qp_b;
      di1_b -= dq_b * dq / di1;
      Zb.qi += qp_b;
      di1_b += qp_b;
    } else {
      Zb.qi += dq_b;
      qim_b -= dq_b;
    }
    if (!K.const_vi) tc_b += tmpc_b * 0.025 * tmpc;
    if (max_first(I.di, QRMIN)) Ib.di += di1_b;
    Ib.den -= qim_b * qim / den;
  }
  if (Z.qs > 1.0e-7) {
    const double d1 = 1.0 + fac;
    Zb.qi += sx_b * fac / d1;
    const double fac_b = sx_b * Z.qi / (d1 * d1);
    Ib.denfac += fac_b * K.dts * K.csaci * ex;
    const double ex_b = fac_b * K.dts * denfac * K.csaci;
    tc_b += ex_b * ex * 0.05;
    const double xs_b = ex_b * ex * 0.8125 / xs;
    Zb.qs += xs_b * den;
    Ib.den += xs_b * Z.qs;
  }
  Zb.tz += tc_b;
}

// rain freezing (psacr, pgfr) below freezing (:1074-1099); lhi0, icpk0 of the routine's entry
SHP void ic_rain_freeze(const MpConst& K, IcState& Z, double qv, double den, double vtr, double vts, double lhi0,
                        double icpk0) {
  const double tc = Z.tz - K.tice;
  double psacr = 0.0;
  if (Z.qs > 1.0e-7)
    psacr = K.dts * acr3d<double>(vts, vtr, Z.qr, Z.qs, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den);
  double pgfr = K.dts * K.cgfr[0] / den * (xexp(-K.cgfr[1] * tc) - 1.0) * xexp(1.75 * xlog(Z.qr * den));
  double sink = psacr + pgfr;
  const double factor = fmin(sink, fmin(Z.qr, -tc / icpk0)) / fmax(sink, QRMIN);
  psacr = factor * psacr;
  pgfr = factor * pgfr;
  sink = psacr + pgfr;
  Z.qr = Z.qr - sink;
  Z.qs = Z.qs + psacr;
  Z.qg = Z.qg + pgfr;
  Z.q_liq = Z.q_liq - sink;
  Z.q_sol = Z.q_sol + sink;
  Z.cvm = cvm_of(K, qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz + sink * lhi0 / Z.cvm;
}
SHP void ic_rain_freeze_b(const MpConst& K, const IcState& Z, const IcIn& I, double lhi0, double icpk0, IcState& Zb,
                          IcIn& Ib, double& lhi0_b, double& icpk0_b) {
  const double den = I.den;
  const double tc = Z.tz - K.tice;
  double psacr0 = 0.0;
  if (Z.qs > 1.0e-7)
    psacr0 = K.dts * acr3d<double>(I.vts, I.vtr, Z.qr, Z.qs, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den);
  const double C1 = K.dts * K.cgfr[0] / den;
  const double e1 = xexp(-K.cgfr[1] * tc);
  const double xr = Z.qr * den;
  const double e2 = xexp(1.75 * xlog(xr));
  const double pgfr0 = C1 * (e1 - 1.0) * e2;
  const double s0 = psacr0 + pgfr0;
  const double r = -tc / icpk0;
  const double mm = fmin(Z.qr, r);
  const double m = fmin(s0, mm);
  const double M = fmax(s0, QRMIN);
  const double factor = m / M;
  const double psacr = factor * psacr0, pgfr = factor * pgfr0;
  const double sink = psacr + pgfr;
  const double cvm1 = cvm_of(K, I.qv, Z.q_liq - sink, Z.q_sol + sink);
  // reverse
  double sink_b = close_transfer_b(K, 1.0, sink, lhi0, cvm1, Zb, Ib.qv, lhi0_b);
  sink_b += -Zb.q_liq + Zb.q_sol - Zb.qr;
  double pgfr_b = Zb.qg + sink_b;
  double psacr_b = Zb.qs + sink_b;
  const double factor_b = psacr_b * psacr0 + pgfr_b * pgfr0;
  double psacr0_b = psacr_b * factor;
  double pgfr0_b = pgfr_b * factor;
  const double m_b = factor_b / M;
  const double M_b = -factor_b * factor / M;
  double s0_b = 0.0, tc_b = 0.0;
  if (max_first(s0, QRMIN)) s0_b += M_b;
  if (min_first(s0, mm)) {
    s0_b += m_b;
  } else if (min_first(Z.qr, r)) {
    Zb.qr += m_b;
  } else {
    tc_b -= m_b / icpk0;
    icpk0_b -= m_b * r / icpk0;
  }
  psacr0_b += s0_b;
  pgfr0_b += s0_b;
  Ib.den -= pgfr0_b * pgfr0 / den;
  const double e1_b = pgfr0_b * C1 * e2;
  const double e2_b = pgfr0_b * C1 * (e1 - 1.0);
  tc_b -= e1_b * e1 * K.cgfr[1];
  const double xr_b = e2_b * 1.75 * e2 / xr;
  Zb.qr += xr_b * den;
  Ib.den += xr_b * Z.qr;
  if (Z.qs > 1.0e-7)
    acr3d_b(I.vts, I.vtr, Z.qr, Z.qs, K.csacr, K.acco[0][1], K.acco[1][1], K.acco[2][1], den, K.dts * psacr0_b, Ib.vts,
            Ib.vtr, Zb.qr, Zb.qs, Ib.den);
  Zb.tz += tc_b;
}

// snow to graupel (pgacs, psaut of snow) below freezing (:1103-1121)
SHP void ic_snow_to_graupel(const MpConst& K, IcState& Z, double den, double vtg, double vts) {
  double sink = 0.0;
  if (Z.qg > QRMIN)
    sink = K.dts * acr3d<double>(vtg, vts, Z.qs, Z.qg, K.cgacs, K.acco[0][3], K.acco[1][3], K.acco[2][3], den);
  const double qsm = K.qs0_crt / den;
  if (Z.qs > qsm) {
    const double factor = K.dts * 1.0e-3 * xexp(0.09 * (Z.tz - K.tice));
    sink = sink + factor / (1.0 + factor) * (Z.qs - qsm);
  }
  sink = fmin(Z.qs, sink);
  Z.qs = Z.qs - sink;
  Z.qg = Z.qg + sink;
}
SHP void ic_snow_to_graupel_b(const MpConst& K, const IcState& Z, const IcIn& I, IcState& Zb, IcIn& Ib) {
  const double den = I.den;
  double s1 = 0.0;
  if (Z.qg > QRMIN)
    s1 = K.dts * acr3d<double>(I.vtg, I.vts, Z.qs, Z.qg, K.cgacs, K.acco[0][3], K.acco[1][3], K.acco[2][3], den);
  const double qsm = K.qs0_crt / den;
  double s2 = s1, fac = 0.0;
  const bool big = Z.qs > qsm;
  if (big) {
    fac = K.dts * 1.0e-3 * xexp(0.09 * (Z.tz - K.tice));
    s2 = s1 + fac / (1.0 + fac) * (Z.qs - qsm);
  }
  const double sink_b = Zb.qg - Zb.qs;
  double s2_b = 0.0;
  if (min_first(Z.qs, s2))
    Zb.qs += sink_b;
  else
    s2_b = sink_b;
  const double s1_b = s2_b;
  if (big) {
    const double d1 = 1.0 + fac;
    Zb.qs += s2_b * fac / d1;
    const double qsm_b = -s2_b * fac / d1;
    const double fac_b = s2_b * (Z.qs - qsm) / (d1 * d1);
    Zb.tz += fac_b * fac * 0.09;
    Ib.den -= qsm_b * qsm / den;
  }
  if (Z.qg > QRMIN)
    acr3d_b(I.vtg, I.vts, Z.qs, Z.qg, K.cgacs, K.acco[0][3], K.acco[1][3], K.acco[2][3], den, K.dts * s1_b, Ib.vtg,
            Ib.vts, Zb.qs, Zb.qg, Ib.den);
}

// graupel riming (pgacw, pgacr) below tice0 (:1123-1160); lhi, icpk from the entry tz, cvm
SHP void ic_graupel_rime(const MpConst& K, IcState& Z, double qv, double den, double vtg, double vtr) {
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  double pgacw = 0.0, pgacr = 0.0;
  if (Z.ql > 1.0e-6) {
    const double qden = Z.qg * den;
    const double factor = K.dts * K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
    pgacw = factor / (1.0 + factor) * Z.ql;
  }
  if (Z.qr > 1.0e-6)
    pgacr = fmin(K.dts * acr3d<double>(vtg, vtr, Z.qr, Z.qg, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den),
                 Z.qr);
  double sink = pgacr + pgacw;
  const double factor = fmin(sink, dim(K.tice, Z.tz) / icpk) / fmax(sink, QRMIN);
  pgacr = factor * pgacr;
  pgacw = factor * pgacw;
  sink = pgacr + pgacw;
  Z.qg = Z.qg + sink;
  Z.qr = Z.qr - pgacr;
  Z.ql = Z.ql - pgacw;
  Z.q_liq = Z.q_liq - sink;
  Z.q_sol = Z.q_sol + sink;
  Z.cvm = cvm_of(K, qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz + sink * lhi / Z.cvm;
}
SHP void ic_graupel_rime_b(const MpConst& K, const IcState& Z, const IcIn& I, IcState& Zb, IcIn& Ib) {
  const double den = I.den;
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  double pgacw0 = 0.0, pgacr0 = 0.0, fac = 0.0, qden = 0.0, a = 0.0;
  if (Z.ql > 1.0e-6) {
    qden = Z.qg * den;
    fac = K.dts * K.cgacw * qden / sqrt(den * sqrt(sqrt(qden)));
    pgacw0 = fac / (1.0 + fac) * Z.ql;
  }
  if (Z.qr > 1.0e-6) {
    a = K.dts * acr3d<double>(I.vtg, I.vtr, Z.qr, Z.qg, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den);
    pgacr0 = fmin(a, Z.qr);
  }
  const double s0 = pgacr0 + pgacw0;
  const double dm = dim(K.tice, Z.tz);
  const double r = dm / icpk;
  const double m = fmin(s0, r);
  const double M = fmax(s0, QRMIN);
  const double factor = m / M;
  const double pgacr = factor * pgacr0, pgacw = factor * pgacw0;
  const double sink = pgacr + pgacw;
  const double cvm1 = cvm_of(K, I.qv, Z.q_liq - sink, Z.q_sol + sink);
  // reverse
  double lhi_b = 0.0;
  double sink_b = close_transfer_b(K, 1.0, sink, lhi, cvm1, Zb, Ib.qv, lhi_b);
  sink_b += -Zb.q_liq + Zb.q_sol + Zb.qg;
  const double pgacw_b = sink_b - Zb.ql;
  const double pgacr_b = sink_b - Zb.qr;
  const double factor_b = pgacr_b * pgacr0 + pgacw_b * pgacw0;
  double pgacr0_b = pgacr_b * factor;
  double pgacw0_b = pgacw_b * factor;
  const double m_b = factor_b / M;
  const double M_b = -factor_b * factor / M;
  double s0_b = 0.0, icpk_b = 0.0;
  if (max_first(s0, QRMIN)) s0_b += M_b;
  if (min_first(s0, r)) {
    s0_b += m_b;
  } else {
    const double dm_b = m_b / icpk;
    icpk_b -= m_b * r / icpk;
    if (K.tice - Z.tz > 0.0) Zb.tz -= dm_b;
  }
  pgacr0_b += s0_b;
  pgacw0_b += s0_b;
  if (Z.qr > 1.0e-6) {
    if (min_first(a, Z.qr))
      acr3d_b(I.vtg, I.vtr, Z.qr, Z.qg, K.cgacr, K.acco[0][2], K.acco[1][2], K.acco[2][2], den, K.dts * pgacr0_b,
              Ib.vtg, Ib.vtr, Zb.qr, Zb.qg, Ib.den);
    else
      Zb.qr += pgacr0_b;
  }
  if (Z.ql > 1.0e-6) {
    const double d1 = 1.0 + fac;
    Zb.ql += pgacw0_b * fac / d1;
    double qden_b = 0.0;
    riming_fac_b(K.dts * K.cgacw, qden, den, fac, pgacw0_b * Z.ql / (d1 * d1), qden_b, Ib.den);
    Zb.qg += qden_b * den;
    Ib.den += qden_b * Z.qg;
  }
  const double lhi_t = lhi_b + icpk_b / Z.cvm;
  Zb.cvm -= icpk_b * icpk / Z.cvm;
  Zb.tz += lhi_t * K.DC_ICE;
}

// The whole routine. Outputs: qg qi ql qr qs tz (q_liq, q_sol, cvm are
// inputs only: the routine works on copies). On entry Zb holds the output
// adjoints (its q_liq, q_sol, cvm fields are ignored); on return, the input
// adjoints. Ib is accumulated.
SHB void icloud_processes_b(const MpConst& K, const IcState& Z0, const IcIn& I, IcState& Zb, IcIn& Ib) {
  Zb.q_liq = 0.0;
  Zb.q_sol = 0.0;
  Zb.cvm = 0.0;
  if (!(I.p1 >= P_MIN)) return;
  const double lhi0 = K.LI00 + K.DC_ICE * Z0.tz;
  const double icpk0 = lhi0 / Z0.cvm;
  double lhi0_b = 0.0, icpk0_b = 0.0;
  const double tc0 = Z0.tz - K.tice;
  if (tc0 >= 0.0) {
    const double dqs0 = K.ces0 / I.p1 - I.qv;
    double dqs0_b = 0.0;
    const bool s_on = Z0.qs > QCMIN;
    IcState Z1 = Z0;
    if (s_on) ic_snow_melt(K, Z1, I.qv, I.den, I.denfac, I.vtr, I.vts, dqs0, lhi0, icpk0);
    if ((Z1.qg > QCMIN) && (Z1.tz - K.tice > 0.0)) ic_graupel_melt_b(K, Z1, I, dqs0, Zb, Ib, dqs0_b);
    if (s_on) ic_snow_melt_b(K, Z0, I, dqs0, lhi0, icpk0, Zb, Ib, dqs0_b, lhi0_b, icpk0_b);
    Ib.p1 -= dqs0_b * K.ces0 / (I.p1 * I.p1);
    Ib.qv -= dqs0_b;
  } else {
    const bool i_on = Z0.qi > 3.0e-7;
    IcState Z1 = Z0;
    if (i_on) ic_ice_to_snow(K, Z1, I.den, I.denfac, I.di);
    const bool r_on = (Z1.qr > 1e-7) && (Z1.tz - K.tice < 0.0);
    IcState Z2 = Z1;
    if (r_on) ic_rain_freeze(K, Z2, I.qv, I.den, I.vtr, I.vts, lhi0, icpk0);
    const bool sg_on = Z2.qs > 1.0e-7;
    IcState Z3 = Z2;
    if (sg_on) ic_snow_to_graupel(K, Z3, I.den, I.vtg, I.vts);
    if ((Z3.qg > 1.0e-7) && (Z3.tz < K.tice0)) ic_graupel_rime_b(K, Z3, I, Zb, Ib);
    if (sg_on) ic_snow_to_graupel_b(K, Z2, I, Zb, Ib);
    if (r_on) ic_rain_freeze_b(K, Z1, I, lhi0, icpk0, Zb, Ib, lhi0_b, icpk0_b);
    if (i_on) ic_ice_to_snow_b(K, Z0, I, Zb, Ib);
  }
  const double lhi_t = lhi0_b + icpk0_b / Z0.cvm;
  Zb.cvm -= icpk0_b * icpk0 / Z0.cvm;
  Zb.tz += lhi_t * K.DC_ICE;
}

// --------------------------------------------- subgrid_z_proc (:431-850)
// State blocks of the saturation adjustment. The state carries the running
// liquid and solid totals and cvm exactly as the routine updates them.
struct SgState {
  double qv, ql, qr, qi, qs, qg, tz, q_liq, q_sol, cvm;
};

// closing statements of a transfer: cvm' from the updated totals, then
// tz' = tz + sgn s lh / cvm'. Zb: output adjoints in, entry ones out (the
// entry cvm's adjoint is cleared); returns s_b.
SHP double sg_close_b(const MpConst& K, double sgn, double s, double lh, double cvm1, SgState& Zb, double& lh_b) {
  const double s_b = sgn * Zb.tz * lh / cvm1;
  lh_b += sgn * Zb.tz * s / cvm1;
  const double cvm1_b = Zb.cvm - sgn * Zb.tz * s * lh / (cvm1 * cvm1);
  Zb.qv += cvm1_b * K.c_vap;
  Zb.q_liq += cvm1_b * K.C_LIQ;
  Zb.q_sol += cvm1_b * K.C_ICE;
  Zb.cvm = 0.0;
  return s_b;
}
// adjoints of lhl = lv00 + d0_vap tz, lhi = LI00 + DC_ICE tz and
// tcpk = lhl / cvm + lhi / cvm at a block entry
SHP void sg_lat_b(const MpConst& K, const SgState& Z, double lh_b, double tcpk_b, SgState& Zb) {
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  const double l_b = lh_b + tcpk_b / Z.cvm;
  Zb.cvm -= tcpk_b * tcpk / Z.cvm;
  Zb.tz += l_b * K.d0_vap + l_b * K.DC_ICE;
}

// cloud water <-> vapour adjustment (:531-554); lhl0, tcp3 of the routine's entry
SHP void sg_cloud_water(const MpConst& K, SgState& Z, double den, double lhl0, double tcp3) {
  double dwsdt;
  const double qsw = wqs2(K, Z.tz, den, dwsdt);
  const double dq0 = qsw - Z.qv;
  double evap;
  if (dq0 > 0.0) {
    const double factor = fmin(1.0, K.fac_l2v * (10.0 * dq0 / qsw));
    evap = fmin(Z.ql, factor * dq0 / (1.0 + tcp3 * dwsdt));
  } else {
    evap = dq0 / (1.0 + tcp3 * dwsdt);
  }
  Z.qv = Z.qv + evap;
  Z.ql = Z.ql - evap;
  Z.q_liq = Z.q_liq - evap;
  Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz - evap * lhl0 / Z.cvm;
}
SHP void sg_cloud_water_b(const MpConst& K, const SgState& Z, double den, double lhl0, double tcp3, SgState& Zb,
                          double& den_b, double& lhl0_b, double& tcp3_b) {
  double dwsdt;
  const double qsw = wqs2(K, Z.tz, den, dwsdt);
  const double dq0 = qsw - Z.qv;
  const double D = 1.0 + tcp3 * dwsdt;
  double f0 = 0.0, factor = 0.0, e = 0.0, evap;
  if (dq0 > 0.0) {
    f0 = K.fac_l2v * (10.0 * dq0 / qsw);
    factor = fmin(1.0, f0);
    e = factor * dq0 / D;
    evap = fmin(Z.ql, e);
  } else {
    evap = dq0 / D;
  }
  const double cvm1 = cvm_of(K, Z.qv + evap, Z.q_liq - evap, Z.q_sol);
  double evap_b = sg_close_b(K, -1.0, evap, lhl0, cvm1, Zb, lhl0_b);
  evap_b += Zb.qv - Zb.ql - Zb.q_liq;
  double dq0_b = 0.0, D_b = 0.0, qsw_b = 0.0;
  if (dq0 > 0.0) {
    if (min_first(Z.ql, e)) {
      Zb.ql += evap_b;
    } else {
      const double factor_b = evap_b * dq0 / D;
      dq0_b += evap_b * factor / D;
      D_b -= evap_b * e / D;
      if (!min_first(1.0, f0)) {
        dq0_b += factor_b * K.fac_l2v * 10.0 / qsw;
        qsw_b -= factor_b * f0 / qsw;
      }
    }
  } else {
    dq0_b += evap_b / D;
    D_b -= evap_b * evap / D;
  }
  tcp3_b += D_b * dwsdt;
  const double dwsdt_b = D_b * tcp3;
  qsw_b += dq0_b;
  Zb.qv -= dq0_b;
  wqs2_b(K, Z.tz, den, qsw, dwsdt, qsw_b, dwsdt_b, Zb.tz, den_b);
}

// forced freezing below t_wfr (:560-575)
SHP void sg_freeze(const MpConst& K, SgState& Z) {
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  const double dtmp = K.t_wfr - Z.tz;
  if ((dtmp > 0.0) && (Z.ql > QCMIN)) {
    const double sink = fmin(Z.ql, fmin(Z.ql * dtmp * 0.125, dtmp / icpk));
    Z.ql = Z.ql - sink;
    Z.qi = Z.qi + sink;
    Z.q_liq = Z.q_liq - sink;
    Z.q_sol = Z.q_sol + sink;
    Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
    Z.tz = Z.tz + sink * lhi / Z.cvm;
  }
}
SHP void sg_freeze_b(const MpConst& K, const SgState& Z, SgState& Zb) {
  const double dtmp = K.t_wfr - Z.tz;
  if (!((dtmp > 0.0) && (Z.ql > QCMIN))) return;
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  const double a = Z.ql * dtmp * 0.125, b = dtmp / icpk;
  const double m = fmin(a, b);
  const double sink = fmin(Z.ql, m);
  const double cvm1 = cvm_of(K, Z.qv, Z.q_liq - sink, Z.q_sol + sink);
  double lhi_b = 0.0;
  double sink_b = sg_close_b(K, 1.0, sink, lhi, cvm1, Zb, lhi_b);
  sink_b += -Zb.ql + Zb.qi - Zb.q_liq + Zb.q_sol;
  double dtmp_b = 0.0, icpk_b = 0.0;
  if (min_first(Z.ql, m)) {
    Zb.ql += sink_b;
  } else if (min_first(a, b)) {
    Zb.ql += sink_b * dtmp * 0.125;
    dtmp_b += sink_b * Z.ql * 0.125;
  } else {
    dtmp_b += sink_b / icpk;
    icpk_b -= sink_b * b / icpk;
  }
  Zb.tz -= dtmp_b;
  const double l_b = lhi_b + icpk_b / Z.cvm;
  Zb.cvm -= icpk_b * icpk / Z.cvm;
  Zb.tz += l_b * K.DC_ICE;
}

// Bigg freezing (:581-605), only without fast_sat_adj
SHP void sg_bigg(const MpConst& K, SgState& Z, double den) {
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  const double tc = K.tice - Z.tz;
  if ((Z.ql > QRMIN) && (tc > 0.0)) {
    double sink = 3.3333e-10 * K.dts * (xexp(0.66 * tc) - 1.0) * den * Z.ql * Z.ql;
    sink = fmin(Z.ql, fmin(tc / icpk, sink));
    Z.ql = Z.ql - sink;
    Z.qi = Z.qi + sink;
    Z.q_liq = Z.q_liq - sink;
    Z.q_sol = Z.q_sol + sink;
    Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
    Z.tz = Z.tz + sink * lhi / Z.cvm;
  }
}
SHP void sg_bigg_b(const MpConst& K, const SgState& Z, double den, SgState& Zb, double& den_b) {
  const double tc = K.tice - Z.tz;
  if (!((Z.ql > QRMIN) && (tc > 0.0))) return;
  const double lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double icpk = lhi / Z.cvm;
  const double e = xexp(0.66 * tc);
  const double C0 = 3.3333e-10 * K.dts;
  const double s0 = C0 * (e - 1.0) * den * Z.ql * Z.ql;
  const double r = tc / icpk;
  const double m = fmin(r, s0);
  const double sink = fmin(Z.ql, m);
  const double cvm1 = cvm_of(K, Z.qv, Z.q_liq - sink, Z.q_sol + sink);
  double lhi_b = 0.0;
  double sink_b = sg_close_b(K, 1.0, sink, lhi, cvm1, Zb, lhi_b);
  sink_b += -Zb.ql + Zb.qi - Zb.q_liq + Zb.q_sol;
  double tc_b = 0.0, icpk_b = 0.0;
  if (min_first(Z.ql, m)) {
    Zb.ql += sink_b;
  } else if (min_first(r, s0)) {
    tc_b += sink_b / icpk;
    icpk_b -= sink_b * r / icpk;
  } else {
    tc_b += sink_b * C0 * den * Z.ql * Z.ql * 0.66 * e;
    den_b += sink_b * C0 * (e - 1.0) * Z.ql * Z.ql;
    Zb.ql += sink_b * 2.0 * C0 * (e - 1.0) * den * Z.ql;
  }
  Zb.tz -= tc_b;
  const double l_b = lhi_b + icpk_b / Z.cvm;
  Zb.cvm -= icpk_b * icpk / Z.cvm;
  Zb.tz += l_b * K.DC_ICE;
}

// cloud ice deposition / sublimation (:614-661)
SHP void sg_ice(const MpConst& K, SgState& Z, double den, double dt_pisub) {
  if (!(Z.tz < K.tice)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  double dqsdt;
  const double qsi = iqs2(K, Z.tz, den, dqsdt);
  const double dq = Z.qv - qsi;
  double sink = dq / (1.0 + tcpk * dqsdt);
  double pidep = 0.0;
  if (Z.qi > QRMIN)
    pidep = dt_pisub * dq * 349138.78 * xexp(0.875 * xlog(Z.qi * den)) /
            (qsi * den * K.LAT2 / (0.0243 * K.RVGAS * sq(Z.tz)) + 4.42478e4);
  if (dq > 0.0) {
    const double tmp = K.tice - Z.tz;
    const double qi_crt = K.qi_gen * fmin(K.qi_lim, 0.1 * tmp) / den;
    sink = fmin(sink, fmin(fmax(qi_crt - Z.qi, pidep), tmp / tcpk));
  } else {
    pidep = pidep * fmin(1.0, dim(Z.tz, K.t_sub) * 0.2);
    sink = fmax(pidep, fmax(sink, -Z.qi));
  }
  Z.qv = Z.qv - sink;
  Z.qi = Z.qi + sink;
  Z.q_sol = Z.q_sol + sink;
  Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz + sink * (lhl + lhi) / Z.cvm;
}
SHP void sg_ice_b(const MpConst& K, const SgState& Z, double den, double dt_pisub, SgState& Zb, double& den_b) {
  if (!(Z.tz < K.tice)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  double dqsdt;
  const double qsi = iqs2(K, Z.tz, den, dqsdt);
  const double dq = Z.qv - qsi;
  const double D = 1.0 + tcpk * dqsdt;
  const double sink0 = dq / D;
  double pidep0 = 0.0, x = 0.0, ex = 0.0, num = 0.0, W = 0.0, dd = 1.0;
  if (Z.qi > QRMIN) {
    x = Z.qi * den;
    ex = xexp(0.875 * xlog(x));
    num = dt_pisub * dq * 349138.78 * ex;
    W = 0.0243 * K.RVGAS * sq(Z.tz);
    dd = qsi * den * K.LAT2 / W + 4.42478e4;
    pidep0 = num / dd;
  }
  const double lh = lhl + lhi;
  double sink;
  double tmp = 0.0, qlim = 0.0, qi_crt = 0.0, A = 0.0, B = 0.0, M1 = 0.0, g = 0.0, fmn = 0.0, pidep = 0.0, Mx = 0.0;
  if (dq > 0.0) {
    tmp = K.tice - Z.tz;
    qlim = fmin(K.qi_lim, 0.1 * tmp);
    qi_crt = K.qi_gen * qlim / den;
    A = fmax(qi_crt - Z.qi, pidep0);
    B = tmp / tcpk;
    M1 = fmin(A, B);
    sink = fmin(sink0, M1);
  } else {
    g = dim(Z.tz, K.t_sub) * 0.2;
    fmn = fmin(1.0, g);
    pidep = pidep0 * fmn;
    Mx = fmax(sink0, -Z.qi);
    sink = fmax(pidep, Mx);
  }
  const double cvm1 = cvm_of(K, Z.qv - sink, Z.q_liq, Z.q_sol + sink);
  double lh_b = 0.0;
  double s_b = sg_close_b(K, 1.0, sink, lh, cvm1, Zb, lh_b);
  s_b += -Zb.qv + Zb.qi + Zb.q_sol;
  double sink0_b = 0.0, pidep0_b = 0.0, tcpk_b = 0.0;
  if (dq > 0.0) {
    if (min_first(sink0, M1)) {
      sink0_b += s_b;
    } else if (min_first(A, B)) {
      if (max_first(qi_crt - Z.qi, pidep0)) {
        Zb.qi -= s_b;
        const double qlim_b = s_b * K.qi_gen / den;
        den_b -= s_b * qi_crt / den;
        if (!min_first(K.qi_lim, 0.1 * tmp)) Zb.tz -= 0.1 * qlim_b;
      } else {
        pidep0_b += s_b;
      }
    } else {
      Zb.tz -= s_b / tcpk;
      tcpk_b -= s_b * B / tcpk;
    }
  } else {
    if (max_first(pidep, Mx)) {
      pidep0_b += s_b * fmn;
      const double fmn_b = s_b * pidep0;
      if (!min_first(1.0, g) && (Z.tz - K.t_sub > 0.0)) Zb.tz += fmn_b * 0.2;
    } else if (max_first(sink0, -Z.qi)) {
      sink0_b += s_b;
    } else {
      Zb.qi -= s_b;
    }
  }
  double dq_b = 0.0, qsi_b = 0.0;
  if (Z.qi > QRMIN) {
    const double num_b = pidep0_b / dd;
    const double dd_b = -pidep0_b * pidep0 / dd;
    dq_b += num_b * dt_pisub * 349138.78 * ex;
    const double ex_b = num_b * dt_pisub * dq * 349138.78;
    const double x_b = ex_b * 0.875 * ex / x;
    Zb.qi += x_b * den;
    den_b += x_b * Z.qi;
    const double t1 = qsi * den * K.LAT2;
    qsi_b += dd_b * den * K.LAT2 / W;
    den_b += dd_b * qsi * K.LAT2 / W;
    const double W_b = -dd_b * (t1 / W) / W;
    Zb.tz += W_b * 0.0243 * K.RVGAS * 2.0 * Z.tz;
  }
  dq_b += sink0_b / D;
  const double D_b = -sink0_b * sink0 / D;
  tcpk_b += D_b * dqsdt;
  const double dqsdt_b = D_b * tcpk;
  Zb.qv += dq_b;
  qsi_b -= dq_b;
  iqs2_b(K, Z.tz, den, qsi, dqsdt, qsi_b, dqsdt_b, Zb.tz, den_b);
  sg_lat_b(K, Z, lh_b, tcpk_b, Zb);
}

// snow sublimation / deposition (:670-706)
SHP void sg_snow(const MpConst& K, SgState& Z, double den, double denfac) {
  if (!(Z.qs > QRMIN)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  double dqsdt;
  const double qsi = iqs2(K, Z.tz, den, dqsdt);
  const double qden = Z.qs * den;
  const double tmp = xexp(0.65625 * xlog(qden));
  const double tsq = Z.tz * Z.tz;
  const double dq = (qsi - Z.qv) / (1.0 + tcpk * dqsdt);
  double pssub = K.cssub[0] * tsq * (K.cssub[1] * sqrt(qden) + K.cssub[2] * tmp * sqrt(denfac)) /
                 (K.cssub[3] * tsq + K.cssub[4] * qsi * den);
  pssub = (qsi - Z.qv) * K.dts * pssub;
  if (pssub > 0.0) {
    pssub = fmin(pssub * fmin(1.0, dim(Z.tz, K.t_sub) * 0.2), Z.qs);
  } else {
    if (Z.tz > K.tice)
      pssub = 0.0;
    else
      pssub = fmax(pssub, fmax(dq, (Z.tz - K.tice) / tcpk));
  }
  Z.qs = Z.qs - pssub;
  Z.qv = Z.qv + pssub;
  Z.q_sol = Z.q_sol - pssub;
  Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz - pssub * (lhl + lhi) / Z.cvm;
}
SHP void sg_snow_b(const MpConst& K, const SgState& Z, double den, double denfac, SgState& Zb, double& den_b,
                   double& denfac_b) {
  if (!(Z.qs > QRMIN)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  double dqsdt;
  const double qsi = iqs2(K, Z.tz, den, dqsdt);
  const double qden = Z.qs * den;
  const double tmp = xexp(0.65625 * xlog(qden));
  const double tsq = Z.tz * Z.tz;
  const double D = 1.0 + tcpk * dqsdt;
  const double dq = (qsi - Z.qv) / D;
  const double sqq = sqrt(qden), sd = sqrt(denfac);
  const double Pp = K.cssub[1] * sqq + K.cssub[2] * tmp * sd;
  const double N1 = K.cssub[0] * tsq * Pp;
  const double D1 = K.cssub[3] * tsq + K.cssub[4] * qsi * den;
  const double ps0 = N1 / D1;
  const double ps1 = (qsi - Z.qv) * K.dts * ps0;
  double g = 0.0, fmn = 0.0, a = 0.0, r = 0.0, Mx = 0.0, pssub;
  if (ps1 > 0.0) {
    g = dim(Z.tz, K.t_sub) * 0.2;
    fmn = fmin(1.0, g);
    a = ps1 * fmn;
    pssub = fmin(a, Z.qs);
  } else if (Z.tz > K.tice) {
    pssub = 0.0;
  } else {
    r = (Z.tz - K.tice) / tcpk;
    Mx = fmax(dq, r);
    pssub = fmax(ps1, Mx);
  }
  const double cvm1 = cvm_of(K, Z.qv + pssub, Z.q_liq, Z.q_sol - pssub);
  double lh_b = 0.0;
  double p_b = sg_close_b(K, -1.0, pssub, lhl + lhi, cvm1, Zb, lh_b);
  p_b += Zb.qv - Zb.qs - Zb.q_sol;
  double ps1_b = 0.0, dq_b = 0.0, tcpk_b = 0.0;
  if (ps1 > 0.0) {
    if (min_first(a, Z.qs)) {
      ps1_b += p_b * fmn;
      const double fmn_b = p_b * ps1;
      if (!min_first(1.0, g) && (Z.tz - K.t_sub > 0.0)) Zb.tz += fmn_b * 0.2;
    } else {
      Zb.qs += p_b;
    }
  } else if (!(Z.tz > K.tice)) {
    if (max_first(ps1, Mx)) {
      ps1_b += p_b;
    } else if (max_first(dq, r)) {
      dq_b += p_b;
    } else {
      Zb.tz += p_b / tcpk;
      tcpk_b -= p_b * r / tcpk;
    }
  }
  double qsi_b = ps1_b * K.dts * ps0;
  Zb.qv -= ps1_b * K.dts * ps0;
  const double ps0_b = ps1_b * (qsi - Z.qv) * K.dts;
  const double N1_b = ps0_b / D1;
  const double D1_b = -ps0_b * ps0 / D1;
  double tsq_b = D1_b * K.cssub[3];
  qsi_b += D1_b * K.cssub[4] * den;
  den_b += D1_b * K.cssub[4] * qsi;
  tsq_b += N1_b * K.cssub[0] * Pp;
  const double P_b = N1_b * K.cssub[0] * tsq;
  double qden_b = P_b * K.cssub[1] * 0.5 / sqq;
  const double tmp_b = P_b * K.cssub[2] * sd;
  denfac_b += P_b * K.cssub[2] * tmp * 0.5 / sd;
  qden_b += tmp_b * 0.65625 * tmp / qden;
  Zb.qs += qden_b * den;
  den_b += qden_b * Z.qs;
  Zb.tz += tsq_b * 2.0 * Z.tz;
  qsi_b += dq_b / D;
  Zb.qv -= dq_b / D;
  const double D_b = -dq_b * dq / D;
  tcpk_b += D_b * dqsdt;
  iqs2_b(K, Z.tz, den, qsi, dqsdt, qsi_b, D_b * tcpk, Zb.tz, den_b);
  sg_lat_b(K, Z, lh_b, tcpk_b, Zb);
}

// graupel sublimation / deposition (:715-746)
SHP void sg_graupel(const MpConst& K, SgState& Z, double den) {
  if (!(Z.qg > QRMIN)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  double dqsdt;
  const double qsi = iqs2(K, Z.tz, den, dqsdt);
  const double dq = (Z.qv - qsi) / (1.0 + tcpk * dqsdt);
  double pgsub = (Z.qv / qsi - 1.0) * Z.qg;
  if (pgsub > 0.0) {
    if (Z.tz > K.tice)
      pgsub = 0.0;
    else
      pgsub = fmin(fmin(K.fac_v2g * pgsub, 0.2 * dq), fmin(Z.ql + Z.qr, (K.tice - Z.tz) / tcpk));
  } else {
    pgsub = fmax(K.fac_g2v * pgsub, dq) * fmin(1.0, dim(Z.tz, K.t_sub) * 0.1);
  }
  Z.qg = Z.qg + pgsub;
  Z.qv = Z.qv - pgsub;
  Z.q_sol = Z.q_sol + pgsub;
  Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
  Z.tz = Z.tz + pgsub * (lhl + lhi) / Z.cvm;
}
SHP void sg_graupel_b(const MpConst& K, const SgState& Z, double den, SgState& Zb, double& den_b) {
  if (!(Z.qg > QRMIN)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz, lhi = K.LI00 + K.DC_ICE * Z.tz;
  const double tcpk = lhl / Z.cvm + lhi / Z.cvm;
  double dqsdt;
  const double qsi = iqs2(K, Z.tz, den, dqsdt);
  const double D = 1.0 + tcpk * dqsdt;
  const double dq = (Z.qv - qsi) / D;
  const double ratio = Z.qv / qsi;
  const double pg0 = (ratio - 1.0) * Z.qg;
  double a1 = 0.0, a2 = 0.0, A = 0.0, b1 = 0.0, b2 = 0.0, B = 0.0, c1 = 0.0, Mx = 0.0, g = 0.0, fmn = 0.0, pg;
  if (pg0 > 0.0) {
    if (Z.tz > K.tice) {
      pg = 0.0;
    } else {
      a1 = K.fac_v2g * pg0;
      a2 = 0.2 * dq;
      A = fmin(a1, a2);
      b1 = Z.ql + Z.qr;
      b2 = (K.tice - Z.tz) / tcpk;
      B = fmin(b1, b2);
      pg = fmin(A, B);
    }
  } else {
    c1 = K.fac_g2v * pg0;
    Mx = fmax(c1, dq);
    g = dim(Z.tz, K.t_sub) * 0.1;
    fmn = fmin(1.0, g);
    pg = Mx * fmn;
  }
  const double cvm1 = cvm_of(K, Z.qv - pg, Z.q_liq, Z.q_sol + pg);
  double lh_b = 0.0;
  double pg_b = sg_close_b(K, 1.0, pg, lhl + lhi, cvm1, Zb, lh_b);
  pg_b += Zb.qg - Zb.qv + Zb.q_sol;
  double pg0_b = 0.0, dq_b = 0.0, tcpk_b = 0.0;
  if (pg0 > 0.0) {
    if (!(Z.tz > K.tice)) {
      if (min_first(A, B)) {
        if (min_first(a1, a2))
          pg0_b += pg_b * K.fac_v2g;
        else
          dq_b += 0.2 * pg_b;
      } else if (min_first(b1, b2)) {
        Zb.ql += pg_b;
        Zb.qr += pg_b;
      } else {
        Zb.tz -= pg_b / tcpk;
        tcpk_b -= pg_b * b2 / tcpk;
      }
    }
  } else {
    const double Mx_b = pg_b * fmn;
    const double fmn_b = pg_b * Mx;
    if (max_first(c1, dq))
      pg0_b += Mx_b * K.fac_g2v;
    else
      dq_b += Mx_b;
    if (!min_first(1.0, g) && (Z.tz - K.t_sub > 0.0)) Zb.tz += fmn_b * 0.1;
  }
  Zb.qg += pg0_b * (ratio - 1.0);
  const double r_b = pg0_b * Z.qg;
  Zb.qv += r_b / qsi;
  double qsi_b = -r_b * ratio / qsi;
  Zb.qv += dq_b / D;
  qsi_b -= dq_b / D;
  const double D_b = -dq_b * dq / D;
  tcpk_b += D_b * dqsdt;
  iqs2_b(K, Z.tz, den, qsi, dqsdt, qsi_b, D_b * tcpk, Zb.tz, den_b);
  sg_lat_b(K, Z, lh_b, tcpk_b, Zb);
}

// minimum evaporation of rain (:751-769)
SHP void sg_rain_evap(const MpConst& K, SgState& Z, double den, double rh_rain) {
  const double lhl = K.lv00 + K.d0_vap * Z.tz;
  const double lcpk = lhl / Z.cvm;
  if (Z.qr > QCMIN) {
    double dqsdt;
    const double qsw2 = wqs2(K, Z.tz, den, dqsdt);
    const double sink = fmin(Z.qr, dim(rh_rain * qsw2, Z.qv) / (1.0 + lcpk * dqsdt));
    Z.qv = Z.qv + sink;
    Z.qr = Z.qr - sink;
    Z.q_liq = Z.q_liq - sink;
    Z.cvm = cvm_of(K, Z.qv, Z.q_liq, Z.q_sol);
    Z.tz = Z.tz - sink * lhl / Z.cvm;
  }
}
SHP void sg_rain_evap_b(const MpConst& K, const SgState& Z, double den, double rh_rain, SgState& Zb, double& den_b) {
  if (!(Z.qr > QCMIN)) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz;
  const double lcpk = lhl / Z.cvm;
  double dqsdt;
  const double qsw = wqs2(K, Z.tz, den, dqsdt);
  const double D = 1.0 + lcpk * dqsdt;
  const double dm = dim(rh_rain * qsw, Z.qv);
  const double e = dm / D;
  const double sink = fmin(Z.qr, e);
  const double cvm1 = cvm_of(K, Z.qv + sink, Z.q_liq - sink, Z.q_sol);
  double lhl_b = 0.0;
  double s_b = sg_close_b(K, -1.0, sink, lhl, cvm1, Zb, lhl_b);
  s_b += Zb.qv - Zb.qr - Zb.q_liq;
  double lcpk_b = 0.0, qsw_b = 0.0, dqsdt_b = 0.0;
  if (min_first(Z.qr, e)) {
    Zb.qr += s_b;
  } else {
    const double dm_b = s_b / D;
    const double D_b = -s_b * e / D;
    if (rh_rain * qsw - Z.qv > 0.0) {
      qsw_b += dm_b * rh_rain;
      Zb.qv -= dm_b;
    }
    lcpk_b += D_b * dqsdt;
    dqsdt_b += D_b * lcpk;
  }
  wqs2_b(K, Z.tz, den, qsw, dqsdt, qsw_b, dqsdt_b, Zb.tz, den_b);
  const double l_b = lhl_b + lcpk_b / Z.cvm;
  Zb.cvm -= lcpk_b * lcpk / Z.cvm;
  Zb.tz += l_b * K.d0_vap;
}

// cloud fraction increment (:774-848): d(qa increment) only on the partial
// cloud branch; icpk8 is the value from the entry of the graupel block
SHP void sg_cloud_frac_b(const MpConst& K, const SgState& Z, double den, double h_var, double icpk8, double qa_b,
                         SgState& Zb, double& den_b, double& icpk8_b) {
  if (K.do_qa) return;
  const double lhl = K.lv00 + K.d0_vap * Z.tz;
  const double cvm2 = K.c_air + (Z.qv + Z.q_liq + Z.q_sol) * K.c_vap;
  const double lcpk = lhl / cvm2;
  const double qsp = K.rad_snow ? Z.qi + Z.qs : Z.qi;
  const double qlp = K.rad_rain ? Z.ql + Z.qr : Z.ql;
  const double qc = qlp + qsp;
  const double qpz = Z.qv + qc;
  const double tin = Z.tz - (lcpk * qc + icpk8 * qsp);
  double qstar, qsi = 0.0, qsw = 0.0, rqi = 0.0;
  const int br = (tin <= K.t_wfr) ? 0 : ((tin >= K.tice) ? 1 : 2);
  if (br == 0) {
    qstar = iqs1(K, tin, den);
  } else if (br == 1) {
    qstar = wqs1(K, tin, den);
  } else {
    qsi = iqs1(K, tin, den);
    qsw = wqs1(K, tin, den);
    rqi = (qc > 3.0e-6) ? qsp / qc : (K.tice - tin) / (K.tice - K.t_wfr);
    qstar = rqi * qsi + (1.0 - rqi) * qsw;
  }
  if (!(qpz > QRMIN)) return;
  const double hq = h_var * qpz;
  const double dq = fmax(QCMIN, hq);
  const double q_plus = qpz + dq;
  const double q_minus = qpz - dq;
  if (qstar < q_minus) return;
  if (!((qstar < q_plus) && (qc > K.qc_crt))) return;
  const double Dd = dq + dq;
  const double F = (q_plus - qstar) / Dd;
  const double qp_b = qa_b / Dd;
  const double qstar_b = -qa_b / Dd;
  double dq_b = 2.0 * (-qa_b * F / Dd) + qp_b;
  double qpz_b = qp_b;
  if (!max_first(QCMIN, hq)) qpz_b += dq_b * h_var;
  double tin_b = 0.0, qsp_b = 0.0, qc_b = 0.0;
  if (br == 0) {
    iqs1_b(K, tin, den, qstar, qstar_b, tin_b, den_b);
  } else if (br == 1) {
    wqs1_b(K, tin, den, qstar, qstar_b, tin_b, den_b);
  } else {
    const double rqi_b = qstar_b * (qsi - qsw);
    iqs1_b(K, tin, den, qsi, qstar_b * rqi, tin_b, den_b);
    wqs1_b(K, tin, den, qsw, qstar_b * (1.0 - rqi), tin_b, den_b);
    if (qc > 3.0e-6) {
      qsp_b += rqi_b / qc;
      qc_b -= rqi_b * rqi / qc;
    } else {
      tin_b -= rqi_b / (K.tice - K.t_wfr);
    }
  }
  Zb.tz += tin_b;
  const double lcpk_b = -tin_b * qc;
  qc_b -= tin_b * lcpk;
  icpk8_b -= tin_b * qsp;
  qsp_b -= tin_b * icpk8;
  Zb.qv += qpz_b;
  qc_b += qpz_b;
  const double qlp_b = qc_b;
  qsp_b += qc_b;
  Zb.ql += qlp_b;
  if (K.rad_rain) Zb.qr += qlp_b;
  Zb.qi += qsp_b;
  if (K.rad_snow) Zb.qs += qsp_b;
  const double lhl_b = lcpk_b / cvm2;
  const double cvm2_b = -lcpk_b * lcpk / cvm2;
  Zb.qv += cvm2_b * K.c_vap;
  Zb.q_liq += cvm2_b * K.c_vap;
  Zb.q_sol += cvm2_b * K.c_vap;
  Zb.tz += lhl_b * K.d0_vap;
}

// The whole routine. X = (qv ql qr qi qs qg tz) entry values; Xb holds the
// output adjoints on entry and the input adjoints on return; qa_b is the
// adjoint of the cloud-fraction accumulator (unchanged: qa only grows by
// increments). den_b, denfac_b are accumulated.
SHB void subgrid_z_proc_b(const MpConst& K, double h_var, double rh_adj, double rh_rain, double qa_b, double qg,
                          double qi, double ql, double qr, double qs, double qv, double tz, double den, double denfac,
                          double p1, double& qg_b, double& qi_b, double& ql_b, double& qr_b, double& qs_b,
                          double& qv_b, double& tz_b, double& den_b, double& denfac_b) {
  if (!(p1 >= P_MIN)) return;
  const double tice = K.tice, t_wfr = K.t_wfr;
  SgState Z0{qv, ql, qr, qi, qs, qg, tz, ql + qr, qi + qs + qg, 0.0};
  Z0.cvm = cvm_of(K, qv, Z0.q_liq, Z0.q_sol);
  const double lhl0 = K.lv00 + K.d0_vap * tz;
  const double lhi0 = K.LI00 + K.DC_ICE * tz;
  const double lcpk0 = lhl0 / Z0.cvm;
  const double icpk0 = lhi0 / Z0.cvm;
  const double dt3 = dim(tice, tz);
  const double fr3 = dt3 / (tice - t_wfr);
  const double fm = fmin(1.0, fr3);
  const double tcp3 = lcpk0 + icpk0 * fm;
  SgState Zb{qv_b, ql_b, qr_b, qi_b, qs_b, qg_b, tz_b, 0.0, 0.0, 0.0};
  double lhl0_b = 0.0, lhi0_b = 0.0, tcp3_b = 0.0;
  if (tz < K.T_MIN) {
    // instant deposition (:488-499)
    const double sink = dim(1.0e-7, qv);
    SgState Z1 = Z0;
    Z1.qv = qv - sink;
    Z1.qi = qi + sink;
    Z1.q_sol = Z0.q_sol + sink;
    Z1.cvm = cvm_of(K, Z1.qv, Z1.q_liq, Z1.q_sol);
    double lh_b = 0.0;
    double s_b = sg_close_b(K, 1.0, sink, lhl0 + lhi0, Z1.cvm, Zb, lh_b);
    s_b += -Zb.qv + Zb.qi + Zb.q_sol;
    if (1.0e-7 - qv > 0.0) Zb.qv -= s_b;
    lhl0_b += lh_b;
    lhi0_b += lh_b;
  } else {
    const double qpz = qv + ql + qi;
    const double Dn = K.c_air + qpz * K.c_vap + qr * K.C_LIQ + (qs + qg) * K.C_ICE;
    const double N = lhl0 * (ql + qi) + lhi0 * qi;
    const double tin = tz - N / Dn;
    bool dry = false;
    if (tin > K.t_sub + 6.0) dry = qpz / iqs1(K, tin, den) < rh_adj;
    if (dry) {
      // tz = tin, qv = qpz, ql = qi = 0
      const double tin_b = Zb.tz;
      double qpz_b = Zb.qv;
      const double N_b = -tin_b / Dn;
      const double Dn_b = tin_b * N / (Dn * Dn);
      lhl0_b += N_b * (ql + qi);
      lhi0_b += N_b * qi;
      Zb.ql = N_b * lhl0;
      Zb.qi = N_b * (lhl0 + lhi0);
      qpz_b += Dn_b * K.c_vap;
      Zb.qr += Dn_b * K.C_LIQ;
      Zb.qs += Dn_b * K.C_ICE;
      Zb.qg += Dn_b * K.C_ICE;
      Zb.qv = qpz_b;
      Zb.ql += qpz_b;
      Zb.qi += qpz_b;
      Zb.tz = tin_b;
    } else {
      const double dt_pisub = K.fast_sat_adj ? 0.5 * K.dts : K.dts;
      SgState Z3 = Z0;
      sg_cloud_water(K, Z3, den, lhl0, tcp3);
      SgState Z4 = Z3;
      sg_freeze(K, Z4);
      SgState Z5 = Z4;
      if (!K.fast_sat_adj) sg_bigg(K, Z5, den);
      SgState Z6 = Z5;
      sg_ice(K, Z6, den, dt_pisub);
      SgState Z7 = Z6;
      sg_snow(K, Z7, den, denfac);
      SgState Z8 = Z7;
      sg_graupel(K, Z8, den);
      SgState Z9 = Z8;
      sg_rain_evap(K, Z9, den, rh_rain);
      const double icpk7 = (K.LI00 + K.DC_ICE * Z7.tz) / Z7.cvm;
      double icpk7_b = 0.0;
      sg_cloud_frac_b(K, Z9, den, h_var, icpk7, qa_b, Zb, den_b, icpk7_b);
      sg_rain_evap_b(K, Z8, den, rh_rain, Zb, den_b);
      sg_graupel_b(K, Z7, den, Zb, den_b);
      Zb.tz += icpk7_b * K.DC_ICE / Z7.cvm;
      Zb.cvm -= icpk7_b * icpk7 / Z7.cvm;
      sg_snow_b(K, Z6, den, denfac, Zb, den_b, denfac_b);
      sg_ice_b(K, Z5, den, dt_pisub, Zb, den_b);
      if (!K.fast_sat_adj) sg_bigg_b(K, Z4, den, Zb, den_b);
      sg_freeze_b(K, Z3, Zb);
      sg_cloud_water_b(K, Z0, den, lhl0, tcp3, Zb, den_b, lhl0_b, tcp3_b);
    }
  }
  // prelude: q_liq, q_sol, cvm, lhl, lhi, lcpk, icpk, tcp3 from the entry state
  const double lcpk0_b = tcp3_b;
  const double icpk0_b = tcp3_b * fm;
  const double fm_b = tcp3_b * icpk0;
  if (!min_first(1.0, fr3) && (tice - tz > 0.0)) Zb.tz -= fm_b / (tice - t_wfr);
  lhl0_b += lcpk0_b / Z0.cvm;
  lhi0_b += icpk0_b / Z0.cvm;
  const double cvm0_b = Zb.cvm - lcpk0_b * lcpk0 / Z0.cvm - icpk0_b * icpk0 / Z0.cvm;
  Zb.tz += lhl0_b * K.d0_vap + lhi0_b * K.DC_ICE;
  Zb.qv += cvm0_b * K.c_vap;
  const double qliq_b = Zb.q_liq + cvm0_b * K.C_LIQ;
  const double qsol_b = Zb.q_sol + cvm0_b * K.C_ICE;
  Zb.ql += qliq_b;
  Zb.qr += qliq_b;
  Zb.qi += qsol_b;
  Zb.qs += qsol_b;
  Zb.qg += qsol_b;
  qv_b = Zb.qv;
  ql_b = Zb.ql;
  qr_b = Zb.qr;
  qi_b = Zb.qi;
  qs_b = Zb.qs;
  qg_b = Zb.qg;
  tz_b = Zb.tz;
}

// ------------------------------------------ pointwise blocks of the step
// sedi_ice_melt: state (qv ql qr qi qs qg tz); qv qs qg are read only
SHB void sedi_ice_melt_b(const MpConst& K, double qv, double ql, double qr, double qi, double qs, double qg, double tz,
                         double& qv_b, double& ql_b, double& qr_b, double& qi_b, double& qs_b, double& qg_b,
                         double& tz_b) {
  const double lhi = K.LI00 + K.DC_ICE * tz;
  const double q_liq = ql + qr;
  const double q_sol = qi + qs + qg;
  const double cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
  const double icpk = lhi / cvm;
  const double tc = tz - K.tice;
  if (!((qi > QCMIN) && (tc > 0.0))) return;
  const double r = K.fac_imlt * tc / icpk;
  const double sink = fmin(qi, r);
  const double dm = dim(K.ql_mlt, ql);
  const double q_liq1 = q_liq + sink, q_sol1 = q_sol - sink;
  const double cvm1 = K.c_air + qv * K.c_vap + q_liq1 * K.C_LIQ + q_sol1 * K.C_ICE;
  // tz' = tz - sink lhi / cvm1
  double sink_b = -tz_b * lhi / cvm1;
  double lhi_b = -tz_b * sink / cvm1;
  const double cvm1_b = tz_b * sink * lhi / (cvm1 * cvm1);
  qv_b += cvm1_b * K.c_vap;
  const double q_liq_b = cvm1_b * K.C_LIQ, q_sol_b = cvm1_b * K.C_ICE;  // q_liq1, q_sol1 adjoints
  sink_b += q_liq_b - q_sol_b;
  sink_b -= qi_b;
  sink_b += qr_b;
  const double tmp_b = ql_b - qr_b;
  if (min_first(sink, dm))
    sink_b += tmp_b;
  else if (K.ql_mlt - ql > 0.0)
    ql_b -= tmp_b;
  double tc_b = 0.0, icpk_b = 0.0;
  if (min_first(qi, r)) {
    qi_b += sink_b;
  } else {
    tc_b += sink_b * K.fac_imlt / icpk;
    icpk_b -= sink_b * r / icpk;
  }
  tz_b += tc_b;
  // icpk = lhi / cvm, cvm from the entry totals
  lhi_b += icpk_b / cvm;
  const double cvm_b = -icpk_b * icpk / cvm;
  qv_b += cvm_b * K.c_vap;
  const double ql0_b = q_liq_b + cvm_b * K.C_LIQ, qs0_b = q_sol_b + cvm_b * K.C_ICE;
  ql_b += ql0_b;
  qr_b += ql0_b;
  qi_b += qs0_b;
  qs_b += qs0_b;
  qg_b += qs0_b;
  tz_b += lhi_b * K.DC_ICE;
}

// icloud_melt_freeze: state (qv ql qr qi qs qg tz) and den; outputs also the
// totals q_liq, q_sol and cvm, whose adjoints come in q_liq_b, q_sol_b, cvm_b
SHB void icloud_melt_freeze_b(const MpConst& K, double qv, double ql, double qr, double qi, double qs, double qg,
                              double tz, double den, double q_liq_b, double q_sol_b, double cvm_b, double& qv_b,
                              double& ql_b, double& qr_b, double& qi_b, double& qs_b, double& qg_b, double& tz_b,
                              double& den_b) {
  const double lhi = K.LI00 + K.DC_ICE * tz;
  const double q_liq = ql + qr;
  const double q_sol = qi + qs + qg;
  const double cvm = K.c_air + qv * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
  const double icpk = lhi / cvm;
  double lhi_b = 0.0, icpk_b = 0.0, qliq_b = q_liq_b, qsol_b = q_sol_b, cvm0_b = cvm_b;
  if ((tz > K.tice) && (qi > QCMIN)) {
    const double r = K.fac_imlt * (tz - K.tice) / icpk;
    const double melt = fmin(qi, r);
    const double dm = dim(K.ql_mlt, ql);
    const double q_liq1 = q_liq + melt, q_sol1 = q_sol - melt;
    const double cvm1 = K.c_air + qv * K.c_vap + q_liq1 * K.C_LIQ + q_sol1 * K.C_ICE;
    double melt_b = -tz_b * lhi / cvm1;
    lhi_b -= tz_b * melt / cvm1;
    const double cvm1_b = cvm_b + tz_b * melt * lhi / (cvm1 * cvm1);
    qv_b += cvm1_b * K.c_vap;
    qliq_b += cvm1_b * K.C_LIQ;
    qsol_b += cvm1_b * K.C_ICE;
    melt_b += qliq_b - qsol_b - qi_b + qr_b;
    const double tmp_b = ql_b - qr_b;
    if (min_first(melt, dm))
      melt_b += tmp_b;
    else if (K.ql_mlt - ql > 0.0)
      ql_b -= tmp_b;
    if (min_first(qi, r)) {
      qi_b += melt_b;
    } else {
      tz_b += melt_b * K.fac_imlt / icpk;
      icpk_b -= melt_b * r / icpk;
    }
    cvm0_b = 0.0;
  } else if ((tz < K.t_wfr) && (ql > QCMIN)) {
    const double dtmp = K.t_wfr - tz;
    const double fr = dtmp / DT_FR;
    const double factor = fmin(1.0, fr);
    const double a = ql * factor, b = dtmp / icpk;
    const double sink = fmin(a, b);
    const double lim = fmin(K.qi_lim, 0.1 * (K.tice - tz));
    const double qi_crt = K.qi_gen * lim / den;
    const double dm = dim(qi_crt, qi);
    const double tmp = fmin(sink, dm);
    const double q_liq1 = q_liq - sink, q_sol1 = q_sol + sink;
    const double cvm1 = K.c_air + qv * K.c_vap + q_liq1 * K.C_LIQ + q_sol1 * K.C_ICE;
    double sink_b = tz_b * lhi / cvm1;
    lhi_b += tz_b * sink / cvm1;
    const double cvm1_b = cvm_b - tz_b * sink * lhi / (cvm1 * cvm1);
    qv_b += cvm1_b * K.c_vap;
    qliq_b += cvm1_b * K.C_LIQ;
    qsol_b += cvm1_b * K.C_ICE;
    sink_b += -qliq_b + qsol_b - ql_b + qs_b;
    const double tmp_b = qi_b - qs_b;
    double dtmp_b = 0.0;
    if (min_first(sink, dm)) {
      sink_b += tmp_b;
    } else if (qi_crt - qi > 0.0) {
      qi_b -= tmp_b;
      const double lim_b = tmp_b * K.qi_gen / den;
      den_b -= tmp_b * qi_crt / den;
      if (!min_first(K.qi_lim, 0.1 * (K.tice - tz))) tz_b -= 0.1 * lim_b;
    }
    (void)tmp;
    if (min_first(a, b)) {
      ql_b += sink_b * factor;
      if (!min_first(1.0, fr)) dtmp_b += sink_b * ql / DT_FR;
    } else {
      dtmp_b += sink_b / icpk;
      icpk_b -= sink_b * b / icpk;
    }
    tz_b -= dtmp_b;
    cvm0_b = 0.0;
  }
  lhi_b += icpk_b / cvm;
  cvm0_b -= icpk_b * icpk / cvm;
  qv_b += cvm0_b * K.c_vap;
  qliq_b += cvm0_b * K.C_LIQ;
  qsol_b += cvm0_b * K.C_ICE;
  ql_b += qliq_b;
  qr_b += qliq_b;
  qi_b += qsol_b;
  qs_b += qsol_b;
  qg_b += qsol_b;
  tz_b += lhi_b * K.DC_ICE;
}

// fix_negative_point: state (qv ql qr qi qs qg tz)
SHB void fix_negative_point_b(const MpConst& K, double qv, double ql, double qr, double qi, double qs, double qg,
                              double tz, double& qv_b, double& ql_b, double& qr_b, double& qi_b, double& qs_b,
                              double& qg_b, double& tz_b) {
  const double cvm = K.c_air + qv * K.c_vap + (qr + ql) * K.C_LIQ + (qi + qs + qg) * K.C_ICE;
  const double lhl = K.lv00 + K.d0_vap * tz, lhi = K.LI00 + K.DC_ICE * tz;
  const double lcpk = lhl / cvm, icpk = lhi / cvm;
  // replay, keeping the branch decisions and the values they read
  const bool bi = qi < 0.0;
  const double qs1 = bi ? qs + qi : qs;
  const bool bs = qs1 < 0.0;
  const double qg1 = bs ? qg + qs1 : qg;
  const bool bg = qg1 < 0.0;
  const double qr1 = bg ? qr + qg1 : qr;
  const bool br = qr1 < 0.0;
  const double ql1 = br ? ql + qr1 : ql;
  const bool bl = ql1 < 0.0;
  // reverse; each name_b below is the adjoint of that version of the value
  double lcpk_b = 0.0, icpk_b = 0.0;
  double ql1_b = ql_b;
  if (bl) {  // qv += ql1; tz -= ql1 lcpk; ql = 0
    ql1_b = qv_b - tz_b * lcpk;
    lcpk_b -= tz_b * ql1;
  }
  const double qr1_b = br ? ql1_b : qr_b;  // ql1 = ql + qr1; qr = 0
  double qg1_b = qg_b;
  if (bg) {  // qr1 = qr + qg1; tz -= qg1 icpk; qg = 0
    qg1_b = qr1_b - tz_b * icpk;
    icpk_b -= tz_b * qg1;
  }
  const double qs1_b = bs ? qg1_b : qs_b;  // qg1 = qg + qs1; qs = 0
  const double qi0_b = bi ? qs1_b : qi_b;  // qs1 = qs + qi; qi = 0
  // lcpk = lhl / cvm, icpk = lhi / cvm
  const double cvm_b = -lcpk_b * lcpk / cvm - icpk_b * icpk / cvm;
  tz_b += lcpk_b / cvm * K.d0_vap + icpk_b / cvm * K.DC_ICE;
  qv_b += cvm_b * K.c_vap;
  ql_b = ql1_b + cvm_b * K.C_LIQ;
  qr_b = qr1_b + cvm_b * K.C_LIQ;
  qi_b = qi0_b + cvm_b * K.C_ICE;
  qs_b = qs1_b + cvm_b * K.C_ICE;
  qg_b = qg1_b + cvm_b * K.C_ICE;
}

}  // namespace shield
