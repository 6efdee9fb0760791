// Mixed-precision process rates of the GFDL microphysics, for one level.
//
// Same processes and branch structure as mp_physics.cuh (each function cites
// the pySHiELD/functions/microphysics_funcs.py lines it follows), with this
// split of the arithmetic:
//  * FP32: the process-rate expressions -- rain evaporation/accretion and
//    their saturation humidity, fall speeds, autoconversion, the ice-phase
//    melting/accretion/conversion rates, and the deposition/sublimation rates
//    inside the saturation adjustment;
//  * FP64: every state update (each transfer is computed once and added to
//    one species and subtracted from the other, so total water is conserved
//    to FP64 round-off), the heat capacities and latent-heat temperature
//    updates (the energy budget), the saturation humidities and latent-heat
//    steps of the saturation adjustment, the sedimentation and the surface
//    precipitation (in the kernel).
#pragma once

#include "mp_physics.cuh"

namespace shield {

SHD float sqf(float x) { return x * x; }
SHD float dimf(float x, float y) {
  float d = x - y;
  return d > 0.0f ? d : 0.0f;
}

// ---------------------------------------------------- microphysics_funcs.py:52-72 in FP32
SHD float wqs1_f(const MpConstF& F, float ta, float den) {
  return (F.E00 * expf((F.DC_VAP * logf(ta / F.TICE) + F.LV0 * (ta - F.TICE) / (ta * F.TICE)) / F.RVGAS)) /
         (F.RVGAS * ta * den);
}
SHD float wqs2_f(const MpConstF& F, float ta, float den, float& dqdt) {
  float tmp = wqs1_f(F, ta, den);
  dqdt = tmp * (F.DC_VAP + F.LV0 / ta) / (F.RVGAS * ta);
  return tmp;
}

SHD float acr3d_f(float v1, float v2, float q1, float q2, float c, float cac_ik, float cac_i1k, float cac_i2k,
                  float rho) {
  float t1 = sqrtf(q1 * rho);
  float s1 = sqrtf(q2 * rho);
  float s2 = sqrtf(s1);
  return c * fabsf(v1 - v2) * q1 * s2 * (cac_ik * t1 + cac_i1k * sqrtf(t1) * s2 + cac_i2k * s1);
}

// ---------------------------------------------------- microphysics_funcs.py:182-265
SHD void revap_racc_m(const MpConst& K, const MpConstF& F, double dt, double h_var, double& qg, double& qi,
                      double& ql, double& qr, double& qs, double& qv, double& tz, double den, double denfac) {
  if ((tz > K.t_wfr) && (qr > QRMIN)) {
    const double lhl = K.lv00 + K.d0_vap * tz;
    double q_liq = ql + qr;
    const double q_sol = qi + qs + qg;
    double cvm = cvm_of(K, qv, q_liq, q_sol);
    const double lcpk = lhl / cvm;
    const double tin = tz - lcpk * ql;
    const double qpz = qv + ql;
    float dqsdt_f;
    const double qsat = wqs2_f(F, (float)tin, (float)den, dqsdt_f);
    const double dqsdt = dqsdt_f;
    double dqh = fmax(ql, h_var * fmax(qpz, QCMIN));
    dqh = fmin(dqh, 0.2 * qpz);
    const double dqv = qsat - qv;
    const double q_minus = qpz - dqh;
    const double q_plus = qpz + dqh;
    if ((dqv > QVMIN) && (qsat > q_minus)) {
      float dq;
      if (qsat > q_plus)
        dq = (float)(qsat - qpz);
      else
        dq = 0.25f * sqf((float)(q_minus - qsat)) / (float)dqh;
      const float qden = (float)(qr * den);
      const float t2 = (float)tin * (float)tin;
      const float evap_rate = F.crevp[0] * t2 * dq * (F.crevp[1] * sqrtf(qden) + F.crevp[2] * expf(0.725f * logf(qden))) /
                              (F.crevp[3] * t2 + F.crevp[4] * (float)qsat * (float)den);
      const double evap = fmin(qr, fmin(dt * (double)evap_rate, dqv / (1.0 + lcpk * dqsdt)));
      qr = qr - evap;
      qv = qv + evap;
      q_liq = q_liq - evap;
      cvm = cvm_of(K, qv, q_liq, q_sol);
      tz = tz - evap * lhl / cvm;
    }
    if ((qr > QRMIN) && (ql > 1.0e-6) && (qsat < q_minus)) {
      float sink = (float)dt * (float)denfac * F.cracw * expf(0.95f * logf((float)(qr * den)));
      sink = sink / (1.0f + sink);
      const double s = (double)sink * ql;
      ql = ql - s;
      qr = qr + s;
    }
  }
}

// ---------------------------------------------------- microphysics_funcs.py:268-372
SHD void fall_speed_m(const MpConst& K, const MpConstF& F, double qg, double qi, double qs, double tk, double den,
                      double& vtg, double& vti, double& vts) {
  const float denf = (float)den;
  const float rhof = sqrtf(fminf(10.0f, (float)SFCRHO / denf));
  if (K.const_vi) {
    vti = K.vi_fac;
  } else if (qi < THI) {
    vti = VF_MIN;
  } else {
    const float vi0 = 0.01f * (float)K.vi_fac;
    const float tc = (float)(tk - K.tice);
    float v = (3.0f + logf((float)qi * denf) / F.log_10) * (tc * ((float)AA * tc + (float)BB) + (float)CC) +
              (float)DD_FS * tc + (float)EE;
    v = vi0 * expf(F.log_10 * v) * 0.8f;
    vti = fmin(K.vi_max, fmax(VF_MIN, (double)v));
  }
  if (K.const_vs) {
    vts = K.vs_fac;
  } else if (qs < THS) {
    vts = VF_MIN;
  } else {
    const float v = (float)K.vs_fac * (float)VCONS * rhof * expf(0.0625f * logf((float)qs * denf / (float)NORMS));
    vts = fmin(K.vs_max, fmax(VF_MIN, (double)v));
  }
  if (K.const_vg) {
    vtg = K.vg_fac;
  } else if (qg < THG) {
    vtg = VF_MIN;
  } else {
    const float v = (float)K.vg_fac * (float)VCONG * rhof * sqrtf(sqrtf(sqrtf((float)qg * denf / (float)NORMG)));
    vtg = fmin(K.vg_max, fmax(VF_MIN, (double)v));
  }
}

SHD double rain_fspeed_m(const MpConst& K, double qrz, double den) {
  if (K.const_vr) return K.vr_fac;
  if (qrz < THR) return VR_MIN;
  const float denf = (float)den;
  const float v = (float)K.vr_fac * (float)VCONR * sqrtf(fminf(10.0f, (float)SFCRHO / denf)) *
                  expf(0.2f * logf((float)qrz * denf / (float)NORMR));
  return fmin(K.vr_max, fmax(VR_MIN, (double)v));
}

// ---------------------------------------------------- microphysics_funcs.py:375-428
SHD void autoconv_no_subgrid_var_m(const MpConst& K, const MpConstF& F, double& qlz, double& qrz, double tz,
                                   double den, double ccn, double c_praut) {
  const double qc0 = K.fac_rc * ccn;
  if (tz > K.t_wfr) {
    const double qc = K.use_ccn ? qc0 : qc0 / den;
    const double dq = qlz - qc;
    if (dq > 0.0) {
      const float rate = F.dt_rain * (float)c_praut * (float)den * expf(F.so3 * logf((float)qlz));
      const double sink = fmin(dq, (double)rate);
      qlz = qlz - sink;
      qrz = qrz + sink;
    }
  }
}
SHD void autoconv_subgrid_var_m(const MpConst& K, const MpConstF& F, double& qlz, double& qrz, double tz, double den,
                                double ccn, double c_praut, double dl) {
  const double qc0 = K.fac_rc * ccn;
  if (tz > K.t_wfr + DT_FR) {
    dl = fmin(fmax(1.0e-6, dl), 0.5 * qlz);
    const double qc = K.use_ccn ? qc0 : qc0 / den;
    const double dq = 0.5 * (qlz + dl - qc);
    if (dq > 0.0) {
      const float rate = fminf(1.0f, (float)(dq / dl)) * F.dt_rain * (float)c_praut * (float)den *
                         expf(F.so3 * logf((float)qlz));
      const double sink = (double)rate;
      qlz = qlz - sink;
      qrz = qrz + sink;
    }
  }
}

// ---------------------------------------------------- microphysics_funcs.py:853-1227
SHD void icloud_processes_m(const MpConst& K, const MpConstF& F, double& qgz, double& qiz, double& qlz, double& qrz,
                            double& qsz, double qvz, double& tz, double den, double denfac, double vtgz, double vtrz,
                            double vtsz, double p1, double di, double q_liq, double q_sol, double cvm) {
  const double tice = K.tice, dts = K.dts;
  const float denf = (float)den, denfacf = (float)denfac, dtsf = F.dts;
  const float vtg = (float)vtgz, vtr = (float)vtrz, vts = (float)vtsz;
  double lhi = K.LI00 + K.DC_ICE * tz;
  double rcpk = cvm / lhi;  // 1 / icpk: every use of icpk here divides by it
  if (!(p1 >= P_MIN)) return;
  double tc = tz - tice;
  if (tc >= 0.0) {
    const float dqs0 = (float)(K.ces0 / p1 - qvz);
    if (qsz > QCMIN) {
      float psacw = 0.0f, psacr = 0.0f, pracs = 0.0f;
      const float qsf = (float)qsz, qlf = (float)qlz, qrf = (float)qrz;
      if (qlz > QRMIN) {
        const float factor = denfacf * F.csacw * expf(0.8125f * logf(qsf * denf));
        psacw = factor / (1.0f + dtsf * factor) * qlf;
      }
      if (qrz > QRMIN) {
        psacr = fminf(acr3d_f(vts, vtr, qrf, qsf, F.csacr, F.acco[0][1], F.acco[1][1], F.acco[2][1], denf),
                      qrf * F.rdts);
        pracs = acr3d_f(vtr, vts, qsf, qrf, F.cracs, F.acco[0][0], F.acco[1][0], F.acco[2][0], denf);
      }
      const float tcf = (float)tc;
      const float qsrho = qsf * denf;
      const float smlt_rate = (F.csmlt[0] * tcf / denf - F.csmlt[1] * dqs0) *
                                  (F.csmlt[2] * sqrtf(qsrho) + F.csmlt[3] * powf(qsrho, 0.65625f) * sqrtf(denfacf)) +
                              F.csmlt[4] * tcf * (psacw + psacr);
      const double psmlt = fmax(0.0, (double)smlt_rate);
      const double sink = fmin(qsz, fmin(dts * (psmlt + (double)pracs), tc * rcpk));
      qsz = qsz - sink;
      const double tmp = fmin(sink, dim(K.qs_mlt, qlz));
      qlz = qlz + tmp;
      qrz = qrz + sink - tmp;
      q_liq = q_liq + sink;
      q_sol = q_sol - sink;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz - sink * lhi / cvm;
      tc = tz - tice;
    }
    lhi = K.LI00 + K.DC_ICE * tz;
    rcpk = cvm / lhi;
    if ((qgz > QCMIN) && (tc > 0.0)) {
      float pgacr = 0.0f, pgacw = 0.0f;
      const float qgf = (float)qgz, qrf = (float)qrz, qlf = (float)qlz;
      if (qrz > QRMIN)
        pgacr = fminf(acr3d_f(vtg, vtr, qrf, qgf, F.cgacr, F.acco[0][2], F.acco[1][2], F.acco[2][2], denf),
                      F.rdts * qrf);
      const float qden = qgf * denf;
      if (qlz > QRMIN) {
        const float factor = F.cgacw * qden / sqrtf(denf * sqrtf(sqrtf(qden)));
        pgacw = factor / (1.0f + dtsf * factor) * qlf;
      }
      const float tcf = (float)tc;
      const float gmlt_rate = (F.cgmlt[0] * tcf / denf - F.cgmlt[1] * dqs0) *
                                  (F.cgmlt[2] * sqrtf(qden) + F.cgmlt[3] * powf(qden, 0.6875f) / powf(denf, 0.25f)) +
                              F.cgmlt[4] * tcf * (pgacw + pgacr);
      double pgmlt = dts * (double)gmlt_rate;
      pgmlt = fmin(fmax(0.0, pgmlt), fmin(qgz, tc * rcpk));
      qgz = qgz - pgmlt;
      qrz = qrz + pgmlt;
      q_liq = q_liq + pgmlt;
      q_sol = q_sol - pgmlt;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz - pgmlt * lhi / cvm;
    }
  } else {
    if (qiz > 3.0e-7) {
      const float tcf = (float)tc;
      float psaci = 0.0f;
      if (qsz > 1.0e-7) {
        const float factor = dtsf * denfacf * F.csaci * expf(0.05f * tcf + 0.8125f * logf((float)qsz * denf));
        psaci = factor / (1.0f + factor) * (float)qiz;
      }
      const double qim = K.qi0_crt / den;
      const double tmp = K.const_vi ? K.fac_i2s : K.fac_i2s * (double)expf(0.025f * tcf);
      di = fmax(di, QRMIN);
      const double q_plus = qiz + di;
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
      const double sink = fmin(0.75 * qiz, (double)psaci + psaut);
      qiz = qiz - sink;
      qsz = qsz + sink;
      if (qgz > 1.0e-6) {
        const float factor = dtsf * F.cgaci * sqrtf(denf) * (float)qgz;
        const double pgaci = (double)(factor / (1.0f + factor)) * qiz;
        qiz = qiz - pgaci;
        qgz = qgz + pgaci;
      }
    }
    tc = tz - tice;
    if ((qrz > 1e-7) && (tc < 0.0)) {
      const float qrf = (float)qrz, tcf = (float)tc;
      float psacr = 0.0f;
      if (qsz > 1.0e-7)
        psacr = dtsf * acr3d_f(vts, vtr, qrf, (float)qsz, F.csacr, F.acco[0][1], F.acco[1][1], F.acco[2][1], denf);
      float pgfr = dtsf * F.cgfr[0] / denf * (expf(-F.cgfr[1] * tcf) - 1.0f) * expf(1.75f * logf(qrf * denf));
      const double sink0 = (double)psacr + (double)pgfr;
      const double factor = fmin(sink0, fmin(qrz, -tc * rcpk)) / fmax(sink0, QRMIN);
      const double ps = factor * (double)psacr;
      const double pg = factor * (double)pgfr;
      const double sink = ps + pg;
      qrz = qrz - sink;
      qsz = qsz + ps;
      qgz = qgz + pg;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(K, qvz, q_liq, q_sol);
      tz = tz + sink * lhi / cvm;
    }
    lhi = K.LI00 + K.DC_ICE * tz;
    rcpk = cvm / lhi;
    if (qsz > 1.0e-7) {
      double sink;
      if (qgz > QRMIN)
        sink = dts * (double)acr3d_f(vtg, vts, (float)qsz, (float)qgz, F.cgacs, F.acco[0][3], F.acco[1][3],
                                     F.acco[2][3], denf);
      else
        sink = 0.0;
      const double qsm = K.qs0_crt / den;
      if (qsz > qsm) {
        const float factor = dtsf * 1.0e-3f * expf(0.09f * (float)(tz - tice));
        sink = sink + (double)(factor / (1.0f + factor)) * (qsz - qsm);
      }
      sink = fmin(qsz, sink);
      qsz = qsz - sink;
      qgz = qgz + sink;
    }
    if ((qgz > 1.0e-7) && (tz < K.tice0)) {
      double pgacw, pgacr;
      if (qlz > 1.0e-6) {
        const float qden = (float)qgz * denf;
        const float factor = dtsf * F.cgacw * qden / sqrtf(denf * sqrtf(sqrtf(qden)));
        pgacw = (double)(factor / (1.0f + factor)) * qlz;
      } else {
        pgacw = 0.0;
      }
      if (qrz > 1.0e-6) {
        pgacr = fmin(dts * (double)acr3d_f(vtg, vtr, (float)qrz, (float)qgz, F.cgacr, F.acco[0][2], F.acco[1][2],
                                           F.acco[2][2], denf),
                     qrz);
      } else {
        pgacr = 0.0;
      }
      double sink = pgacr + pgacw;
      const double factor = fmin(sink, dim(tice, tz) * rcpk) / fmax(sink, QRMIN);
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
