// One column of the microphysics step as plain sequential C++, templated on
// the real type (test infrastructure for the adjoint tests).
//
// The pointwise processes are the templates of mp_physics.cuh themselves;
// the vertical operations that the CUDA kernel does with warp scans and
// level exchanges are written here as loops over the levels, in the
// kernel's order of stages (fields_init; per sub-step: geometry, warm_rain,
// sedimentation, warm_rain, icloud; fields_update). Run with dual numbers
// seeded along an input direction dx, it gives J dx of the whole step
// exactly (on the branches the input takes), the reference for the adjoint
// kernel's J^T ybar. Values agree with the kernel to rounding (sums and
// scans run in another order); derivatives agree to rounding wherever no
// branch decision sits within rounding of its threshold.
#pragma once

#include "mp_physics.cuh"

namespace shield {
namespace colref {

constexpr int LMAX = 128;

// input rows (InField order), output rows (OutField order)
enum { X_PT = 0, X_QV, X_QL, X_QR, X_QI, X_QS, X_QG, X_QA, X_UA, X_VA, X_DELP, X_DELZ, X_W, X_QAZ, NX };
enum { Y_PT = 0, Y_QV, Y_QL, Y_QR, Y_QI, Y_QS, Y_QG, Y_QA, Y_U, Y_V, Y_W, Y_QAZ, NY };

template <class T>
T mono_slope_at(const T* q, int k, int L) {
  T v = 0.0;
  if (k >= 1 && k <= L - 2) {
    const T dq = 0.5 * (q[k] - q[k - 1]);
    const T dqn = 0.5 * (q[k + 1] - q[k]);
    v = 0.5 * fmin(fabs(dq + dqn), 0.5 * q[k]);
    if (dq * dqn <= 0.0) {
      if (dq > 0.0)
        v = fmin(v, fmin(dq, -dqn));
      else
        v = 0.0;
    }
  }
  return v;
}

// r_k (dz_k + dd_k) = qmass_k + dd_{k-1} r_{k-1}; returns the flux dd r and
// updates q to r dz / dp1
template <class T>
void implicit_fall(int L, T* q, const T* vt, const T* dz, const T* dp1, double dtf, T* flux) {
  T rprev = 0.0, ddprev = 0.0;
  for (int k = 0; k < L; ++k) {
    const T dd = dtf * vt[k];
    const T D = dz[k] + dd;
    const T a = q[k] * dp1[k] / D;
    const T r = (k == 0) ? a : a + (ddprev / D) * rprev;
    q[k] = r * dz[k] / dp1[k];
    flux[k] = dd * r;
    rprev = r;
    ddprev = dd;
  }
}

template <class T>
T w_update_t(int k, T w, T dm, T flux, T vt, T fp, T vp) {
  if (k == 0) return (dm * w + flux * vt) / (dm - flux);
  return (dm * w - fp * vp + flux * vt) / (dm + fp - flux);
}

// Implicit heating by falling condensate (microphysics.py:516-557 with
// C_LIQ, :1176-1217 with C_ICE), level by level: flux[k] leaves level k,
// fp[k] enters it from above.
template <class T>
struct Col;
template <class T>
void sedi_heat(const MpConst& K, int L, Col<T>& c, const T* flux, const T* fp, double c_cond) {
  T xprev = 0.0;
  for (int k = 0; k < L; ++k) {
    const T dgz = -0.5 * K.GRAV * c.dz1[k];
    const T cvn =
        c.dp1[k] * (K.CV_AIR + c.qv[k] * K.CV_VAP + (c.qr[k] + c.ql[k]) * K.C_LIQ + (c.qi[k] + c.qs[k] + c.qg[k]) * K.C_ICE);
    T x;
    if (k == 0) {
      const T tmp = cvn + flux[k] * c_cond;
      x = c.tz[k] + flux[k] * dgz / tmp;
    } else {
      const T D = cvn + c_cond * flux[k];
      const T a = ((cvn + c_cond * (flux[k] - fp[k])) * c.tz[k] + dgz * (fp[k] + flux[k])) / D;
      const T b = fp[k] * c_cond / D;
      x = a + b * xprev;
    }
    c.tz[k] = x;
    xprev = x;
  }
}

template <class T>
struct Col {
  T qv[LMAX], ql[LMAX], qr[LMAX], qi[LMAX], qs[LMAX], qg[LMAX], tz[LMAX], w[LMAX];
  T dp1[LMAX], p1[LMAX], den[LMAX], denfac[LMAX], dz1[LMAX], dz[LMAX];
  T ccn, c_praut;
  double h_var, rh_adj, rh_rain;
};

template <class T>
void warm_rain(const MpConst& K, int L, Col<T>& c, T* vtr, T* m1r, T& r1) {
  const double dt5 = 0.5 * K.dt_rain;
  bool fall = false;
  for (int k = 0; k < L; ++k) fall = fall || (c.qr[k] > QRMIN);
  for (int k = 0; k < L; ++k) m1r[k] = 0.0;
  r1 = 0.0;
  if (!fall) {
    for (int k = 0; k < L; ++k) vtr[k] = VF_MIN;
  } else {
    T dm[LMAX];
    for (int k = 0; k < L; ++k) {
      vtr[k] = rain_fspeed<T>(K, c.qr[k], c.den[k]);
      revap_racc<T>(K, dt5, c.h_var, c.qg[k], c.qi[k], c.ql[k], c.qr[k], c.qs[k], c.qv[k], c.tz[k], c.den[k],
                    c.denfac[k]);
      dm[k] = c.dp1[k] * (1.0 + c.qv[k] + c.ql[k] + c.qr[k] + c.qi[k] + c.qs[k] + c.qg[k]);
    }
    implicit_fall<T>(L, c.qr, vtr, c.dz, c.dp1, K.dt_rain, m1r);
    r1 = m1r[L - 1];
    if (K.do_sedi_w)
      for (int k = 0; k < L; ++k)
        c.w[k] = w_update_t<T>(k, c.w[k], dm[k], m1r[k], vtr[k], k > 0 ? m1r[k - 1] : T(0.0),
                               k > 0 ? vtr[k - 1] : T(0.0));
    if (K.do_sedi_heat) {
      T fp[LMAX];
      for (int k = 0; k < L; ++k) fp[k] = k > 0 ? m1r[k - 1] : T(0.0);
      sedi_heat<T>(K, L, c, m1r, fp, K.C_LIQ);
    }
    for (int k = 0; k < L; ++k)
      revap_racc<T>(K, dt5, c.h_var, c.qg[k], c.qi[k], c.ql[k], c.qr[k], c.qs[k], c.qv[k], c.tz[k], c.den[k],
                    c.denfac[k]);
  }
  if (K.irain_f != 0) {
    for (int k = 0; k < L; ++k)
      autoconv_no_subgrid_var<T>(K, c.ql[k], c.qr[k], c.tz[k], c.den[k], c.ccn, c.c_praut);
  } else {
    T dl[LMAX];
    for (int k = 0; k < L; ++k) {
      const T inner = fmax(QVMIN, c.h_var * c.ql[k]);
      dl[k] = K.z_slope_liq ? fmax(mono_slope_at<T>(c.ql, k, L), inner) : inner;
    }
    for (int k = 0; k < L; ++k)
      autoconv_subgrid_var<T>(K, c.ql[k], c.qr[k], c.tz[k], c.den[k], c.ccn, c.c_praut, dl[k]);
  }
}

template <class T>
void sedimentation(const MpConst& K, int L, Col<T>& c, T* vtg, T* vts, T* m1s, T* sfc /* ice snow graupel */) {
  T vti[LMAX];
  for (int k = 0; k < L; ++k) fall_speed<T>(K, c.qg[k], c.qi[k], c.qs[k], c.tz[k], c.den[k], vtg[k], vti[k], vts[k]);
  int first = 1 << 30;
  for (int k = L - 1; k >= 0; --k)
    if (c.tz[k] > K.tice) first = k;
  for (int k = 0; k < L; ++k)
    if (k >= first || k == L - 1) sedi_ice_melt<T>(K, c.qv[k], c.ql[k], c.qr[k], c.qi[k], c.qs[k], c.qg[k], c.tz[k]);
  bool fi = false, fs = false, fg = false;
  for (int k = 0; k < L; ++k) {
    fi = fi || (c.qi[k] > QRMIN);
    fs = fs || (c.qs[k] > QRMIN);
    fg = fg || (c.qg[k] > QRMIN);
  }
  fi = fi && (K.vi_fac >= 1.0e-5);
  for (int k = 0; k < L; ++k) m1s[k] = 0.0;
  T mp[LMAX];  // the falling species' flux entering each level from above
  for (int k = 0; k < L; ++k) mp[k] = 0.0;
  if (!(fi || fs || fg)) {
    if (K.do_sedi_heat) sedi_heat<T>(K, L, c, m1s, mp, K.C_ICE);
    return;
  }
  T* vt[3] = {vti, vts, vtg};
  T qq[3][LMAX], flux[3][LMAX];
  for (int k = 0; k < L; ++k) {
    qq[0][k] = c.qi[k];
    qq[1][k] = c.qs[k];
    qq[2][k] = c.qg[k];
  }
  for (int n = 0; n < 3; ++n) implicit_fall<T>(L, qq[n], vt[n], c.dz, c.dp1, K.dts, flux[n]);
  T dmi[LMAX], dms[LMAX], dmg[LMAX];
  for (int k = 0; k < L; ++k) {
    dmi[k] = c.dp1[k] * (1.0 + c.qv[k] + c.ql[k] + c.qr[k] + c.qi[k] + c.qs[k] + c.qg[k]);
    if (fi) c.qi[k] = qq[0][k];
    dms[k] = c.dp1[k] * (1.0 + c.qv[k] + c.ql[k] + c.qr[k] + c.qi[k] + c.qs[k] + c.qg[k]);
    if (fs) c.qs[k] = qq[1][k];
    dmg[k] = c.dp1[k] * (1.0 + c.qv[k] + c.ql[k] + c.qr[k] + c.qi[k] + c.qs[k] + c.qg[k]);
    if (fg) c.qg[k] = qq[2][k];
  }
  for (int k = 0; k < L; ++k) {
    const int p = k > 0 ? k - 1 : 0;
    const T z = 0.0;
    if (fi) mp[k] = k > 0 ? flux[0][p] : z;
    if (fs) mp[k] = mp[k] + (k > 0 ? flux[1][p] : z);
    if (fg) mp[k] = mp[k] + (k > 0 ? flux[2][p] : z);
    if (fi) {
      m1s[k] = flux[0][k];
      if (K.do_sedi_w) c.w[k] = w_update_t<T>(k, c.w[k], dmi[k], flux[0][k], vti[k], flux[0][p], vti[p]);
    }
    if (fs) {
      m1s[k] = m1s[k] + flux[1][k];
      if (K.do_sedi_w) c.w[k] = w_update_t<T>(k, c.w[k], dms[k], flux[1][k], vts[k], flux[1][p], vts[p]);
    }
    if (fg) {
      m1s[k] = m1s[k] + flux[2][k];
      if (K.do_sedi_w) c.w[k] = w_update_t<T>(k, c.w[k], dmg[k], flux[2][k], vtg[k], flux[2][p], vtg[p]);
    }
  }
  if (K.do_sedi_heat) sedi_heat<T>(K, L, c, m1s, mp, K.C_ICE);
  if (fi) sfc[0] = sfc[0] + flux[0][L - 1];
  if (fs) sfc[1] = sfc[1] + flux[1][L - 1];
  if (fg) sfc[2] = sfc[2] + flux[2][L - 1];
}

template <class T>
void icloud(const MpConst& K, int L, Col<T>& c, T* qa, const T* vtg, const T* vtr, const T* vts) {
  T q_liq[LMAX], q_sol[LMAX], cvm[LMAX], di[LMAX];
  for (int k = 0; k < L; ++k)
    icloud_melt_freeze<T>(K, c.qv[k], c.ql[k], c.qr[k], c.qi[k], c.qs[k], c.qg[k], c.tz[k], c.den[k], q_liq[k],
                          q_sol[k], cvm[k]);
  for (int k = 0; k < L; ++k) {
    const T inner = fmax(QVMIN, c.h_var * c.qi[k]);
    di[k] = K.z_slope_ice ? fmax(mono_slope_at<T>(c.qi, k, L), inner) : inner;
  }
  for (int k = 0; k < L; ++k) {
    icloud_processes<T>(K, c.qg[k], c.qi[k], c.ql[k], c.qr[k], c.qs[k], c.qv[k], c.tz[k], c.den[k], c.denfac[k],
                        vtg[k], vtr[k], vts[k], c.p1[k], di[k], q_liq[k], q_sol[k], cvm[k]);
    subgrid_z_proc<T>(K, c.h_var, c.rh_adj, c.rh_rain, qa[k], c.qg[k], c.qi[k], c.ql[k], c.qr[k], c.qs[k], c.qv[k],
                      c.tz[k], c.den[k], c.denfac[k], c.p1[k]);
  }
}

// x: NX rows of L levels (the step's input state and accumulator); y: NY
// rows (the ten increments as the kernel writes them, the output w and
// accumulator); s: the four surface totals (rain, snow, ice, graupel) in
// mm/day
template <class T>
void column_step(const MpConst& K, int L, double land, double area, T (*x)[LMAX], T (*y)[LMAX], T* s) {
  Col<T> c;
  for (int k = 0; k < L; ++k) {
    c.tz[k] = x[X_PT][k];
    c.dp1[k] = x[X_DELP][k];
    c.dp1[k] = c.dp1[k] * (1.0 - x[X_QV][k]);
    const T omq = x[X_DELP][k] / c.dp1[k];
    c.qv[k] = x[X_QV][k] * omq;
    c.ql[k] = x[X_QL][k] * omq;
    c.qr[k] = x[X_QR][k] * omq;
    c.qi[k] = x[X_QI][k] * omq;
    c.qs[k] = x[X_QS][k] * omq;
    c.qg[k] = x[X_QG][k] * omq;
    const T den0 = -c.dp1[k] / (K.GRAV * x[X_DELZ][k]);
    c.p1[k] = den0 * K.RDGAS * x[X_PT][k];
    c.w[k] = x[X_W][k];
  }
  if (K.prog_ccn) {
    c.ccn = 0.0 * 1.0e6;
  } else {
    c.ccn = (K.ccn_l * land + K.ccn_o * (1.0 - land)) * 1.0e6;
    if (K.use_ccn) c.ccn = c.ccn * K.RDGAS * c.tz[L - 1] / c.p1[L - 1];
  }
  c.c_praut = K.cpaut * xpow(c.ccn * RHOR, -1.0 / 3.0);
  const double s_leng = std::sqrt(std::sqrt(area * 1.0e-10));
  const double hv = K.dw_land * s_leng * land + K.dw_ocean * s_leng * (1.0 - land);
  c.h_var = std::fmin(0.2, std::fmax(0.01, hv));
  c.rh_adj = 1.0 - c.h_var - K.rh_inc;
  c.rh_rain = std::fmax(0.35, c.rh_adj - K.rh_inr);
  if (K.fix_negative) {
    for (int k = 0; k < L; ++k)
      fix_negative_point<T>(K, c.qv[k], c.ql[k], c.qr[k], c.qi[k], c.qs[k], c.qg[k], c.tz[k]);
    for (int k = 1; k < L; ++k)
      if (c.qv[k - 1] < 0.0) c.qv[k] = c.qv[k] + c.qv[k - 1] * c.dp1[k - 1] / c.dp1[k];
    for (int k = 0; k < L - 1; ++k)
      if (c.qv[k] < 0.0) c.qv[k] = 0.0;
    const T qb = c.qv[L - 1], qb1 = c.qv[L - 2];
    if ((qb < 0.0) && (qb1 > 0.0)) {
      const T dq = fmin(-qb * c.dp1[L - 1], qb1 * c.dp1[L - 2]);
      c.qv[L - 2] = c.qv[L - 2] - dq / c.dp1[L - 2];
      c.qv[L - 1] = c.qv[L - 1] + dq / c.dp1[L - 1];
    }
  }
  T m1[LMAX], m1r[LMAX], m1s[LMAX], vtr[LMAX], vtg[LMAX], vts[LMAX], qa[LMAX];
  for (int k = 0; k < L; ++k) {
    m1[k] = 0.0;
    qa[k] = x[X_QAZ][k];
    vtr[k] = VF_MIN;
    vtg[k] = VF_MIN;
    vts[k] = VF_MIN;
  }
  T rain = 0.0, sfc[3] = {0.0, 0.0, 0.0};
  for (int it = 0; it < K.ntimes; ++it) {
    for (int k = 0; k < L; ++k) {
      const T dz0 = x[X_DELZ][k];
      const T den0 = -c.dp1[k] / (K.GRAV * dz0);
      c.dz1[k] = dz0 * c.tz[k] / x[X_PT][k];
      c.den[k] = den0 * dz0 / c.dz1[k];
      c.denfac[k] = sqrt(SFCRHO / c.den[k]);
      c.dz[k] = -c.dz1[k];
    }
    T r1;
    warm_rain<T>(K, L, c, vtr, m1r, r1);
    rain = rain + r1;
    for (int k = 0; k < L; ++k) m1[k] = m1[k] + m1r[k];
    sedimentation<T>(K, L, c, vtg, vts, m1s, sfc);
    warm_rain<T>(K, L, c, vtr, m1r, r1);
    rain = rain + r1;
    for (int k = 0; k < L; ++k) m1[k] = m1[k] + m1r[k] + m1s[k];
    icloud<T>(K, L, c, qa, vtg, vtr, vts);
  }
  // fields_update
  const double rdt = K.rdt;
  T u1 = 0.0, v1 = 0.0;
  for (int k = 0; k < L; ++k) {
    const T dp0 = x[X_DELP][k], u0 = x[X_UA][k], v0 = x[X_VA][k];
    if (K.sedi_transport) {
      if (k == 0) {
        u1 = u0;
        v1 = v0;
      } else {
        const T D = dp0 + m1[k - 1];
        u1 = dp0 * u0 / D + (m1[k - 1] / D) * u1;
        v1 = dp0 * v0 / D + (m1[k - 1] / D) * v1;
      }
    }
    const T omq0 = dp0 / c.dp1[k], omq = c.dp1[k] / dp0;
    const T* q[6] = {c.qv, c.ql, c.qr, c.qi, c.qs, c.qg};
    for (int n = 0; n < 6; ++n) y[Y_QV + n][k] = rdt * (q[n][k] - x[X_QV + n][k] * omq0) * omq;
    const T cvm = K.c_air + c.qv[k] * K.c_vap + (c.qr[k] + c.ql[k]) * K.C_LIQ +
                  (c.qi[k] + c.qs[k] + c.qg[k]) * K.C_ICE;
    y[Y_PT][k] = rdt * (c.tz[k] - x[X_PT][k]) * cvm / K.CP_AIR;
    y[Y_QA][k] = K.do_qa ? T(0.0) : rdt * (qa[k] / (double)K.ntimes - x[X_QA][k]);
    y[Y_U][k] = (K.sedi_transport && k >= 1) ? (u1 - u0) * rdt : T(0.0);
    y[Y_V][k] = (K.sedi_transport && k >= 1) ? (v1 - v0) * rdt : T(0.0);
    y[Y_W][k] = c.w[k];
    y[Y_QAZ][k] = qa[k];
  }
  const double convt = 86400.0 * rdt * K.RGRAV;
  s[0] = rain * convt;
  s[1] = sfc[1] * convt;
  s[2] = sfc[0] * convt;
  s[3] = sfc[2] * convt;
}

}  // namespace colref
}  // namespace shield
