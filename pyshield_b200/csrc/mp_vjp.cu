// Adjoint of the microphysics step (FP64): the vector-Jacobian product of
// the step's outputs -- the ten tendencies, wmp, the persistent
// cloud-fraction accumulator and the surface totals -- with respect to its
// inputs (pt, the six water species, qcld, ua, va, delprsi, delz, wmp and
// the accumulator), for pySHiELD's Microphysics.__call__
// (pySHiELD/stencils/microphysics.py:1981-2263).
//
// One thread per level and one group of NW warps per column, as in the
// forward kernel. Each group
//  1. replays the step with the forward's own stage functions, keeping the
//     level's state at the entry of every stage of every sub-step in a
//     small per-thread store (local memory);
//  2. reverses fields_update (including the momentum scan);
//  3. for each sub-step from the last, recomputes the sub-step geometry and
//     reverses icloud, the second warm_rain pass, sedimentation and the
//     first pass, each from its stored entry state (pointwise processes
//     through the hand-written adjoints of mp_adjoint.cuh, vertical
//     recurrences through bottom-up scans, level exchanges through their
//     transposes);
//  4. reverses fields_init.
// Branches follow the forward at the given input (the VJP of the piecewise
// smooth map on the branch it takes).
#include <cuda_runtime.h>

#include "mp_adjoint.cuh"
#include "mp_kernel.cuh"
#include "mp_launch.h"

namespace shield {
namespace {

constexpr int VJP_MAXNT = 4;  // sub-steps whose stage states fit the store

// launch shape: columns per block for 65-96 levels, and the minimum
// resident blocks per SM given to __launch_bounds__
#ifndef SHIELD_VJP_G3
#define SHIELD_VJP_G3 4
#endif
#ifndef SHIELD_VJP_MINB
#define SHIELD_VJP_MINB 1
#endif
constexpr int NT_IN = N_VJP_IN + N_VJP_COT;

// Shared memory: NT_IN input tiles (inputs, then cotangents), N_VJP_GRAD
// gradient tiles, G x 2 x SCR exchange scratch, G x 4 x RP work rows.
template <int NW, int G>
struct VjpSmem {
  static constexpr int RP = Tiles<NW>::RP;
  static constexpr size_t out = (size_t)NT_IN * G * RP;
  static constexpr size_t scratch = out + (size_t)N_VJP_GRAD * G * RP;
  static constexpr size_t work = scratch + (size_t)G * 2 * Tiles<NW>::SCR;
  static constexpr size_t total = work + (size_t)G * 4 * RP;
  static constexpr size_t bytes = total * sizeof(double);
};

// load NF fields into tiles [f * G + g][k] (all loads issued before any
// store); a field with a null pointer reads as zero
template <int NW, int G, int NF>
SHD void load_tiles(const Fld3* F, double* tiles, int64_t ncol, int nx, int L, int64_t c0) {
  constexpr int RP = Tiles<NW>::RP;
  const int tid = threadIdx.x;
  const int g = tid % G, k = tid / G;
  const int64_t col = c0 + g;
  const bool ok = col < ncol && k < L;
  const int64_t i = ok ? col % nx : 0, j = ok ? col / nx : 0;
  const int gk = tid / (32 * NW), kk = tid % (32 * NW);
  const int64_t colk = c0 + gk;
  const bool okk = colk < ncol && kk < L;
  const int64_t ik = okk ? colk % nx : 0, jk = okk ? colk / nx : 0;
  double v[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    v[f] = 0.0;
    if (!F[f].p) {
    } else if (F[f].sk == 1) {
      if (okk) v[f] = F[f].p[ik * F[f].si + jk * F[f].sj + kk];
    } else if (ok) {
      v[f] = F[f].p[i * F[f].si + j * F[f].sj + (int64_t)k * F[f].sk];
    }
  }
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    if (F[f].sk == 1) {
      if (okk) tiles[(f * G + gk) * RP + kk] = v[f];
    } else if (ok) {
      tiles[(f * G + g) * RP + k] = v[f];
    }
  }
}

template <int NW, int G, int NF>
SHD void store_tiles(const Fld3* F, const double* tiles, int64_t ncol, int nx, int L, int64_t c0) {
  constexpr int RP = Tiles<NW>::RP;
  const int tid = threadIdx.x;
  const int g = tid % G, k = tid / G;
  const int64_t col = c0 + g;
  const bool ok = col < ncol && k < L;
  const int64_t i = ok ? col % nx : 0, j = ok ? col / nx : 0;
  const int gk = tid / (32 * NW), kk = tid % (32 * NW);
  const int64_t colk = c0 + gk;
  const bool okk = colk < ncol && kk < L;
  const int64_t ik = okk ? colk % nx : 0, jk = okk ? colk / nx : 0;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    if (!F[f].p) continue;
    if (F[f].sk == 1) {
      if (okk) F[f].p[ik * F[f].si + jk * F[f].sj + kk] = tiles[(f * G + gk) * RP + kk];
    } else if (ok) {
      F[f].p[i * F[f].si + j * F[f].sj + (int64_t)k * F[f].sk] = tiles[(f * G + g) * RP + k];
    }
  }
}

// w_update (microphysics.py:492-515): w_b holds the adjoint of the updated
// value on entry and of the old one on return
SHD void w_update_b(int k, double w, double dm, double flux, double vt, double fp, double vp, double& w_b,
                    double& dm_b, double& flux_b, double& vt_b, double& fp_b, double& vp_b) {
  const double wo_b = w_b;
  if (k == 0) {
    const double Dd = dm - flux;
    const double wo = (dm * w + flux * vt) / Dd;
    const double N_b = wo_b / Dd, Dd_b = -wo_b * wo / Dd;
    w_b = N_b * dm;
    dm_b += N_b * w + Dd_b;
    flux_b += N_b * vt - Dd_b;
    vt_b += N_b * flux;
  } else {
    const double Dd = dm + fp - flux;
    const double wo = (dm * w - fp * vp + flux * vt) / Dd;
    const double N_b = wo_b / Dd, Dd_b = -wo_b * wo / Dd;
    w_b = N_b * dm;
    dm_b += N_b * w + Dd_b;
    fp_b += -N_b * vp + Dd_b;
    vp_b -= N_b * fp;
    flux_b += N_b * vt - Dd_b;
    vt_b += N_b * flux;
  }
}

// mono_slope: v_b is the adjoint of the slope at this level; adds the
// adjoints of q at k - 1, k and k + 1 into the owning levels' q_b
template <int NW>
SHD void mono_slope_b(Column<NW>& C, double q, double v_b, double& q_b, bool valid) {
  double qp, qn;
  C.nbrs(q, qp, qn);
  const int k = C.k;
  double cq = 0.0, cp = 0.0, cn = 0.0;
  if (valid && k >= 1 && k <= C.L - 2) {
    const double dq = 0.5 * (q - qp);
    const double dqn = 0.5 * (qn - q);
    const double s = dq + dqn;
    const double A1 = fabs(s), A2 = 0.5 * q;
    const double v0 = 0.5 * fmin(A1, A2);
    double v0_b = 0.0, dq_b = 0.0, dqn_b = 0.0;
    if (dq * dqn <= 0.0) {
      if (dq > 0.0) {
        const double m2 = fmin(dq, -dqn);
        if (min_first(v0, m2))
          v0_b = v_b;
        else if (min_first(dq, -dqn))
          dq_b += v_b;
        else
          dqn_b -= v_b;
      }
    } else {
      v0_b = v_b;
    }
    if (min_first(A1, A2)) {
      const double s_b = 0.5 * v0_b * (s >= 0.0 ? 1.0 : -1.0);
      dq_b += s_b;
      dqn_b += s_b;
    } else {
      cq += 0.25 * v0_b;
    }
    cq += 0.5 * dq_b - 0.5 * dqn_b;
    cp = -0.5 * dq_b;
    cn = 0.5 * dqn_b;
  }
  double from_prev, from_next;
  C.prev_next(cn, cp, from_prev, from_next);
  if (valid) {
    q_b += cq;
    if (k >= 1) q_b += from_prev;
    if (k <= C.L - 2) q_b += from_next;
  }
}

// implicit_fall replayed with its intermediates kept
struct FallRec {
  double dd, D, a, b, r, q1, flux;
};
template <int NW>
SHD FallRec implicit_fall_rec(Column<NW>& C, double q, double vt, double dz, double dp1, bool valid, double dtf) {
  FallRec R;
  R.dd = dtf * vt;
  const double qmass = valid ? q * dp1 : 0.0;
  const double ddp = C.prev(R.dd);
  R.D = dz + R.dd;
  R.a = qmass / R.D;
  R.b = (C.k == 0) ? 0.0 : ddp / R.D;
  if (!valid) {
    R.a = 0.0;
    R.b = 0.0;
  }
  R.r = C.scan_affine(R.a, R.b);
  R.q1 = valid ? R.r * dz / dp1 : q;
  R.flux = valid ? R.dd * R.r : 0.0;
  return R;
}
// q_b: adjoint of the fallen q on entry, of the entry q on return
template <int NW>
SHD void implicit_fall_b(Column<NW>& C, const FallRec& R, double q, double dz, double dp1, bool valid, double dtf,
                         double& q_b, double flux_b, double& vt_b, double& dz_b, double& dp1_b) {
  const int k = C.k, L = C.L;
  double r_b = 0.0, dd_b = 0.0;
  if (valid) {
    r_b = q_b * dz / dp1 + flux_b * R.dd;
    dz_b += q_b * R.r / dp1;
    dp1_b -= q_b * R.q1 / dp1;
    dd_b = flux_b * R.r;
  }
  double bv[1] = {R.b}, bn[1];
  C.template nextN<1>(bv, bn);
  const double cc = (valid && k < L - 1) ? bn[0] : 0.0;
  const double lam = C.scan_affine_rev(valid ? r_b : 0.0, cc);
  const double rp = C.prev(R.r);
  double ddp_b = 0.0;
  if (valid) {
    const double a_b = lam;
    const double b_b = (k > 0) ? lam * rp : 0.0;
    const double qmass_b = a_b / R.D;
    const double D_b = -a_b * R.a / R.D - b_b * R.b / R.D;
    ddp_b = b_b / R.D;
    dz_b += D_b;
    dd_b += D_b;
    q_b = qmass_b * dp1;
    dp1_b += qmass_b * q;
  } else {
    q_b = 0.0;
  }
  double dv[1] = {ddp_b}, dn[1];
  C.template nextN<1>(dv, dn);
  if (valid && k < L - 1) dd_b += dn[0];
  if (valid) vt_b += dd_b * dtf;
}

// Adjoint accumulators of one sub-step's geometry and of the step constants.
struct StepAdj {
  double den, denfac, dz, dp1, p1, ccn, c_praut;
};

// warm_rain reverse from its entry state S0. m1r_b: adjoint of the rain flux
// at this level; rain_c: cotangent of the surface rain total; vtr_b: adjoint
// of the pass's output fall speed.
template <int NW>
static __device__ __noinline__ void warm_rain_b(Column<NW>& C, const MpConst& K, bool valid, const LevState& S0, const StepGeom& P, double m1r_b,
                     double rain_c, double vtr_b, LevState& Sb, StepAdj& Ab) {
  const int k = C.k, L = C.L;
  const double dt5 = 0.5 * K.dt_rain;
  const bool fall = C.any(valid && (S0.qr > QRMIN));
  LevState S1 = S0, S2 = S0, S3 = S0;
  double vtr = VF_MIN, dm = 0.0, pv[2] = {0.0, 0.0};
  FallRec R{};
  if (fall) {
    vtr = rain_fspeed(K, S0.qr, P.den);
    revap_racc(K, dt5, P.h_var, S1.qg, S1.qi, S1.ql, S1.qr, S1.qs, S1.qv, S1.tz, P.den, P.denfac);
    dm = P.dp1 * (1.0 + S1.qv + S1.ql + S1.qr + S1.qi + S1.qs + S1.qg);
    R = implicit_fall_rec<NW>(C, S1.qr, vtr, P.dz, P.dp1, valid, K.dt_rain);
    S2 = S1;
    S2.qr = R.q1;
    double fv[2] = {R.flux, vtr};
    C.template prevN<2>(fv, pv);
    if (K.do_sedi_w) S2.w = w_update(k, S1.w, dm, R.flux, vtr, pv[0], pv[1]);
    S3 = S2;
    revap_racc(K, dt5, P.h_var, S3.qg, S3.qi, S3.ql, S3.qr, S3.qs, S3.qv, S3.tz, P.den, P.denfac);
  }
  // autoconversion
  if (K.irain_f != 0) {
    if (valid)
      autoconv_no_subgrid_var_b(K, S3.ql, S3.qr, S3.tz, P.den, P.ccn, P.c_praut, Sb.ql, Sb.qr, Ab.den, Ab.ccn,
                                Ab.c_praut);
  } else {
    const double hq = P.h_var * S3.ql;
    const double inner = fmax(QVMIN, hq);
    double sl = 0.0, dl = inner;
    if (K.z_slope_liq) {
      sl = mono_slope(C, S3.ql);
      dl = fmax(sl, inner);
    }
    double dl_b = 0.0;
    if (valid)
      autoconv_subgrid_var_b(K, S3.ql, S3.qr, S3.tz, P.den, P.ccn, P.c_praut, dl, Sb.ql, Sb.qr, Ab.den, Ab.ccn,
                             Ab.c_praut, dl_b);
    double sl_b = 0.0;
    if (K.z_slope_liq && max_first(sl, inner))
      sl_b = dl_b;
    else if (!max_first(QVMIN, hq))
      Sb.ql += dl_b * P.h_var;
    if (K.z_slope_liq) mono_slope_b<NW>(C, S3.ql, sl_b, Sb.ql, valid);
  }
  if (!fall) return;  // vtr = VF_MIN: no adjoint
  // second evaporation / accretion
  if (valid)
    revap_racc_b(K, dt5, P.h_var, S2.qg, S2.qi, S2.ql, S2.qr, S2.qs, S2.qv, S2.tz, P.den, P.denfac, Sb.qg, Sb.qi,
                 Sb.ql, Sb.qr, Sb.qs, Sb.qv, Sb.tz, Ab.den, Ab.denfac);
  double flux_b = m1r_b, vt_b = vtr_b, dm_b = 0.0, pv_b[2] = {0.0, 0.0};
  if (K.do_sedi_w && valid)
    w_update_b(k, S1.w, dm, R.flux, vtr, pv[0], pv[1], Sb.w, dm_b, flux_b, vt_b, pv_b[0], pv_b[1]);
  if (k == L - 1) flux_b += rain_c;  // rain += the surface flux
  double pn[2];
  C.template nextN<2>(pv_b, pn);
  if (valid && k < L - 1) {
    flux_b += pn[0];
    vt_b += pn[1];
  }
  double qr_b = Sb.qr;
  implicit_fall_b<NW>(C, R, S1.qr, P.dz, P.dp1, valid, K.dt_rain, qr_b, flux_b, vt_b, Ab.dz, Ab.dp1);
  Sb.qr = qr_b;
  if (valid) {
    // dm = dp1 (1 + qv + ql + qr + qi + qs + qg)
    Ab.dp1 += dm_b * (1.0 + S1.qv + S1.ql + S1.qr + S1.qi + S1.qs + S1.qg);
    const double t = dm_b * P.dp1;
    Sb.qv += t;
    Sb.ql += t;
    Sb.qr += t;
    Sb.qi += t;
    Sb.qs += t;
    Sb.qg += t;
    revap_racc_b(K, dt5, P.h_var, S0.qg, S0.qi, S0.ql, S0.qr, S0.qs, S0.qv, S0.tz, P.den, P.denfac, Sb.qg, Sb.qi,
                 Sb.ql, Sb.qr, Sb.qs, Sb.qv, Sb.tz, Ab.den, Ab.denfac);
    rain_fspeed_b(K, S0.qr, P.den, vt_b, Sb.qr, Ab.den);
  }
}

// sedimentation reverse from its entry state S0. m1s_b: adjoint of the
// solid flux at this level; ice_c, snow_c, graupel_c: cotangents of the
// surface totals; vtg_b, vts_b: adjoints of the output fall speeds.
template <int NW>
static __device__ __noinline__ void sedimentation_b(Column<NW>& C, const MpConst& K, bool valid, const LevState& S0, const StepGeom& P,
                         double m1s_b, double ice_c, double snow_c, double graupel_c, double vtg_b, double vts_b,
                         LevState& Sb, StepAdj& Ab) {
  const int k = C.k, L = C.L;
  const double dp1 = P.dp1, dz = P.dz;
  double vtg, vti, vts;
  fall_speed(K, S0.qg, S0.qi, S0.qs, S0.tz, P.den, vtg, vti, vts);
  const int first = C.min_int((valid && S0.tz > K.tice) ? k : (1 << 30));
  const bool melt_lev = (k >= first || k == L - 1) && valid;
  LevState S1 = S0;
  if (melt_lev) sedi_ice_melt(K, S1.qv, S1.ql, S1.qr, S1.qi, S1.qs, S1.qg, S1.tz);
  bool fi, fs, fg;
  C.any3(valid && (S1.qi > QRMIN), valid && (S1.qs > QRMIN), valid && (S1.qg > QRMIN), fi, fs, fg);
  fi = fi && (K.vi_fac >= 1.0e-5);
  double vt_b[3] = {0.0, vts_b, vtg_b};  // vti, vts, vtg
  if (fi || fs || fg) {
    const double dd[3] = {K.dts * vti, K.dts * vts, K.dts * vtg};
    double ddp[3];
    C.template prevN<3>(dd, ddp);
    const double qq[3] = {S1.qi, S1.qs, S1.qg};
    double ra[3], rb[3], D[3], r[3];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const double qmass = valid ? qq[n] * dp1 : 0.0;
      D[n] = dz + dd[n];
      ra[n] = qmass / D[n];
      rb[n] = (k == 0) ? 0.0 : ddp[n] / D[n];
      if (!valid) {
        ra[n] = 0.0;
        rb[n] = 0.0;
      }
    }
    C.template scanN<3>(ra, rb, r);
    double flux[3];
#pragma unroll
    for (int n = 0; n < 3; ++n) flux[n] = valid ? dd[n] * r[n] : 0.0;
    const double dm_i = dp1 * (1.0 + S1.qv + S1.ql + S1.qr + S1.qi + S1.qs + S1.qg);
    const double qi2 = (fi && valid) ? r[0] * dz / dp1 : S1.qi;
    const double dm_s = dp1 * (1.0 + S1.qv + S1.ql + S1.qr + qi2 + S1.qs + S1.qg);
    const double qs2 = (fs && valid) ? r[1] * dz / dp1 : S1.qs;
    const double dm_g = dp1 * (1.0 + S1.qv + S1.ql + S1.qr + qi2 + qs2 + S1.qg);
    const double qg2 = (fg && valid) ? r[2] * dz / dp1 : S1.qg;
    const double nv[6] = {flux[0], vti, flux[1], vts, flux[2], vtg};
    double pv[6];
    C.template prevN<6>(nv, pv);
    const double w0 = S1.w;
    const double w1 = (fi && K.do_sedi_w) ? w_update(k, w0, dm_i, flux[0], vti, pv[0], pv[1]) : w0;
    const double w2 = (fs && K.do_sedi_w) ? w_update(k, w1, dm_s, flux[1], vts, pv[2], pv[3]) : w1;
    // reverse: vertical velocity, in the reverse species order
    double flux_b[3] = {0.0, 0.0, 0.0}, dm_b[3] = {0.0, 0.0, 0.0}, pv_b[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double wb = Sb.w;
    if (valid) {
      if (fg) {
        if (K.do_sedi_w)
          w_update_b(k, w2, dm_g, flux[2], vtg, pv[4], pv[5], wb, dm_b[2], flux_b[2], vt_b[2], pv_b[4], pv_b[5]);
        flux_b[2] += m1s_b;
      }
      if (fs) {
        if (K.do_sedi_w)
          w_update_b(k, w1, dm_s, flux[1], vts, pv[2], pv[3], wb, dm_b[1], flux_b[1], vt_b[1], pv_b[2], pv_b[3]);
        flux_b[1] += m1s_b;
      }
      if (fi) {
        if (K.do_sedi_w)
          w_update_b(k, w0, dm_i, flux[0], vti, pv[0], pv[1], wb, dm_b[0], flux_b[0], vt_b[0], pv_b[0], pv_b[1]);
        flux_b[0] += m1s_b;
      }
      if (k == L - 1) {
        if (fi) flux_b[0] += ice_c;
        if (fs) flux_b[1] += snow_c;
        if (fg) flux_b[2] += graupel_c;
      }
    }
    Sb.w = wb;
    double pn[6];
    C.template nextN<6>(pv_b, pn);
    if (valid && k < L - 1) {
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        flux_b[n] += pn[2 * n];
        vt_b[n] += pn[2 * n + 1];
      }
    }
    // the three mixing-ratio updates and their dm's, in reverse
    double r_b[3] = {0.0, 0.0, 0.0};
    if (valid) {
      if (fg) {
        r_b[2] += Sb.qg * dz / dp1;
        Ab.dz += Sb.qg * r[2] / dp1;
        Ab.dp1 -= Sb.qg * qg2 / dp1;
        Sb.qg = 0.0;
      }
      {
        Ab.dp1 += dm_b[2] * (1.0 + S1.qv + S1.ql + S1.qr + qi2 + qs2 + S1.qg);
        const double t = dm_b[2] * dp1;
        Sb.qv += t, Sb.ql += t, Sb.qr += t, Sb.qi += t, Sb.qs += t, Sb.qg += t;
      }
      if (fs) {
        r_b[1] += Sb.qs * dz / dp1;
        Ab.dz += Sb.qs * r[1] / dp1;
        Ab.dp1 -= Sb.qs * qs2 / dp1;
        Sb.qs = 0.0;
      }
      {
        Ab.dp1 += dm_b[1] * (1.0 + S1.qv + S1.ql + S1.qr + qi2 + S1.qs + S1.qg);
        const double t = dm_b[1] * dp1;
        Sb.qv += t, Sb.ql += t, Sb.qr += t, Sb.qi += t, Sb.qs += t, Sb.qg += t;
      }
      if (fi) {
        r_b[0] += Sb.qi * dz / dp1;
        Ab.dz += Sb.qi * r[0] / dp1;
        Ab.dp1 -= Sb.qi * qi2 / dp1;
        Sb.qi = 0.0;
      }
      {
        Ab.dp1 += dm_b[0] * (1.0 + S1.qv + S1.ql + S1.qr + S1.qi + S1.qs + S1.qg);
        const double t = dm_b[0] * dp1;
        Sb.qv += t, Sb.ql += t, Sb.qr += t, Sb.qi += t, Sb.qs += t, Sb.qg += t;
      }
    }
    // flux = dd r, then the implicit recurrences
    double dd_b[3] = {0.0, 0.0, 0.0};
    if (valid) {
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        r_b[n] += flux_b[n] * dd[n];
        dd_b[n] = flux_b[n] * r[n];
      }
    }
    double rbn[3], cc[3], aa[3], lam[3], rp[3];
    C.template nextN<3>(rb, rbn);
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      cc[n] = (valid && k < L - 1) ? rbn[n] : 0.0;
      aa[n] = valid ? r_b[n] : 0.0;
    }
    C.template scanN_rev<3>(aa, cc, lam);
    C.template prevN<3>(r, rp);
    double ddp_b[3] = {0.0, 0.0, 0.0};
    if (valid) {
      double q_b[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        const double a_b = lam[n];
        const double b_b = (k > 0) ? lam[n] * rp[n] : 0.0;
        const double qmass_b = a_b / D[n];
        const double D_b = -a_b * ra[n] / D[n] - b_b * rb[n] / D[n];
        ddp_b[n] = b_b / D[n];
        Ab.dz += D_b;
        dd_b[n] += D_b;
        q_b[n] = qmass_b * dp1;
        Ab.dp1 += qmass_b * qq[n];
      }
      Sb.qi += q_b[0];
      Sb.qs += q_b[1];
      Sb.qg += q_b[2];
    }
    double ddn[3];
    C.template nextN<3>(ddp_b, ddn);
    if (valid) {
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        if (k < L - 1) dd_b[n] += ddn[n];
        vt_b[n] += dd_b[n] * K.dts;
      }
    }
  }
  if (melt_lev)
    sedi_ice_melt_b(K, S0.qv, S0.ql, S0.qr, S0.qi, S0.qs, S0.qg, S0.tz, Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg,
                    Sb.tz);
  if (valid)
    fall_speed_b(K, S0.qg, S0.qi, S0.qs, S0.tz, P.den, vt_b[2], vt_b[0], vt_b[1], Sb.qg, Sb.qi, Sb.qs, Sb.tz, Ab.den);
}

// icloud reverse from its entry state S0 and the state S2 between the ice
// processes and the saturation adjustment; qa_b: adjoint of the level's
// cloud-fraction accumulator
template <int NW>
static __device__ __noinline__ void icloud_b(Column<NW>& C, const MpConst& K, bool valid, const LevState& S0,
                                             const LevState& S2, const StepGeom& P, double vtg, double vtr,
                                             double vts, double qa_b, LevState& Sb, StepAdj& Ab, double& vtg_b,
                                             double& vtr_b, double& vts_b) {
  LevState S1 = S0;
  double q_liq, q_sol, cvm;
  icloud_melt_freeze(K, S1.qv, S1.ql, S1.qr, S1.qi, S1.qs, S1.qg, S1.tz, P.den, q_liq, q_sol, cvm);
  const double hq = P.h_var * S1.qi;
  const double inner = fmax(QVMIN, hq);
  double sl = 0.0, di = inner;
  if (K.z_slope_ice) {
    sl = mono_slope(C, S1.qi);
    di = fmax(sl, inner);
  }
  double di_b = 0.0, qliq_b = 0.0, qsol_b = 0.0, cvm_b = 0.0;
  if (valid) {
    subgrid_z_proc_b(K, P.h_var, P.rh_adj, P.rh_rain, qa_b, S2.qg, S2.qi, S2.ql, S2.qr, S2.qs, S2.qv, S2.tz, P.den,
                     P.denfac, P.p1, Sb.qg, Sb.qi, Sb.ql, Sb.qr, Sb.qs, Sb.qv, Sb.tz, Ab.den, Ab.denfac);
    const IcState Z0{S1.qg, S1.qi, S1.ql, S1.qr, S1.qs, S1.tz, q_liq, q_sol, cvm};
    const IcIn I{S1.qv, P.den, P.denfac, vtg, vtr, vts, P.p1, di};
    IcState Zb{Sb.qg, Sb.qi, Sb.ql, Sb.qr, Sb.qs, Sb.tz, 0.0, 0.0, 0.0};
    IcIn Ib{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    icloud_processes_b(K, Z0, I, Zb, Ib);
    Sb.qg = Zb.qg;
    Sb.qi = Zb.qi;
    Sb.ql = Zb.ql;
    Sb.qr = Zb.qr;
    Sb.qs = Zb.qs;
    Sb.tz = Zb.tz;
    Sb.qv += Ib.qv;
    Ab.den += Ib.den;
    Ab.denfac += Ib.denfac;
    Ab.p1 += Ib.p1;
    vtg_b += Ib.vtg;
    vtr_b += Ib.vtr;
    vts_b += Ib.vts;
    di_b = Ib.di;
    qliq_b = Zb.q_liq;
    qsol_b = Zb.q_sol;
    cvm_b = Zb.cvm;
  }
  double sl_b = 0.0;
  if (K.z_slope_ice && max_first(sl, inner))
    sl_b = di_b;
  else if (valid && !max_first(QVMIN, hq))
    Sb.qi += di_b * P.h_var;
  if (K.z_slope_ice) mono_slope_b<NW>(C, S1.qi, sl_b, Sb.qi, valid);
  if (valid)
    icloud_melt_freeze_b(K, S0.qv, S0.ql, S0.qr, S0.qi, S0.qs, S0.qg, S0.tz, P.den, qliq_b, qsol_b, cvm_b, Sb.qv,
                         Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg, Sb.tz, Ab.den);
}

// forward stages of the replay, out of line (one copy each)
template <int NW>
static __device__ __noinline__ void fwd_warm_rain(Column<NW>& C, const MpConst& K, const MpConstF& KF, bool valid,
                                                  LevState& S, const StepGeom& P, double& vtr, double& m1r,
                                                  double& r1) {
  warm_rain<false>(C, K, KF, valid, S, P, vtr, m1r, r1);
}
template <int NW>
static __device__ __noinline__ void fwd_sedimentation(Column<NW>& C, const MpConst& K, const MpConstF& KF, bool valid,
                                                      LevState& S, const StepGeom& P, double& vtg, double& vts,
                                                      double& m1s, double& ice, double& snow, double& graupel) {
  sedimentation<false>(C, K, KF, valid, S, P, vtg, vts, m1s, ice, snow, graupel);
}
template <int NW>
static __device__ __noinline__ void fwd_icloud(Column<NW>& C, const MpConst& K, const MpConstF& KF, bool valid,
                                               LevState& S, const StepGeom& P, double& qa, double vtg, double vtr,
                                               double vts, LevState& rec) {
  icloud<false>(C, K, KF, valid, S, P, qa, vtg, vtr, vts, &rec);
}

template <int NW, int G, int MINB>
__global__ void __launch_bounds__(32 * NW * G, MINB) mp_vjp_kernel(const __grid_constant__ VjpArgs A) {
  extern __shared__ double sm[];
  using SM = VjpSmem<NW, G>;
  constexpr int RP = Tiles<NW>::RP;
  const MpConst& K = A.K;
  const MpConstF& KF = A.KF;
  const int L = A.nz;
  const int tid = threadIdx.x;
  const int g = tid / (32 * NW);
  const int64_t c0 = (int64_t)blockIdx.x * G;
  load_tiles<NW, G, N_VJP_IN>(A.in, sm, A.ncol, A.nx, L, c0);
  load_tiles<NW, G, N_VJP_COT>(A.cot, sm + (size_t)N_VJP_IN * G * RP, A.ncol, A.nx, L, c0);
  __syncthreads();

  const int64_t col = c0 + g;
  Column<NW> C;
  C.w = (tid >> 5) % NW;
  C.lane = tid & 31;
  C.k = 32 * C.w + C.lane;
  C.L = L;
  C.bar = 1 + g;
  C.scr = sm + SM::scratch + (size_t)g * 2 * Tiles<NW>::SCR;
  C.work = sm + SM::work + (size_t)g * 4 * RP;
  C.par = 0;
  const int k = C.k;
  const bool valid = k < L;
  const double* tile = sm + (size_t)g * RP + k;
  auto TI = [&](int f, double dflt) -> double { return valid ? tile[(size_t)f * G * RP] : dflt; };
  auto TC = [&](int f) -> double { return valid ? tile[(size_t)(N_VJP_IN + f) * G * RP] : 0.0; };
  double* gtile = sm + SM::out + (size_t)g * RP + k;
  auto TG = [&](int f) -> double& { return gtile[(size_t)f * G * RP]; };

  if (col < A.ncol) {
    const int64_t ci = col % A.nx, cj = col / A.nx;
    const double land = A.land.p[ci * A.land.si + cj * A.land.sj];
    const double area = A.area.p[ci * A.area.si + cj * A.area.sj];
    const double pt = TI(IN_PT, 250.0), delp = TI(IN_DELP, 1.0), dz0 = TI(IN_DELZ, -100.0);
    const double qin[6] = {TI(IN_QV, 0.0), TI(IN_QL, 0.0), TI(IN_QR, 0.0), TI(IN_QI, 0.0), TI(IN_QS, 0.0),
                           TI(IN_QG, 0.0)};
    // ------------------------------------------------------ forward replay
    LevState S;
    StepGeom P;
    P.den = 1.0;
    P.denfac = 1.0;
    P.dz1 = -100.0;
    P.dz = 100.0;
    fields_init(C, K, valid, pt, qin[0], qin[1], qin[2], qin[3], qin[4], qin[5], delp, TI(IN_W, 0.0), dz0, land,
                    area, S, P);
    LevState ck[VJP_MAXNT][5];  // entries of the four stages, and the state before the adjustment
    double ckv[VJP_MAXNT][3];
    double m1 = 0.0, m1_sol = 0.0, vtr = VF_MIN, vtg = VF_MIN, vts = VF_MIN, qa = 0.0, ice = 0.0, snow = 0.0,
           graupel = 0.0;
    const int nt = K.ntimes;
#pragma unroll 1
    for (int it = 0; it < nt; ++it) {
      substep_geometry(C, K, valid, pt, dz0, S, P);
#pragma unroll 1
      for (int pass = 0; pass < 2; ++pass) {
        double m1r, r1;
        ck[it][2 * pass] = S;
        fwd_warm_rain<NW>(C, K, KF, valid, S, P, vtr, m1r, r1);
        m1 = (pass == 0) ? m1 + m1r : m1 + m1r + m1_sol;
        ck[it][2 * pass + 1] = S;
        if (pass == 1) break;
        fwd_sedimentation<NW>(C, K, KF, valid, S, P, vtg, vts, m1_sol, ice, snow, graupel);
      }
      ckv[it][0] = vtr;
      ckv[it][1] = vtg;
      ckv[it][2] = vts;
      fwd_icloud<NW>(C, K, KF, valid, S, P, qa, vtg, vtr, vts, ck[it][4]);
    }

    // ------------------------------------------------- fields_update reverse
    const double rdt = K.rdt;
    LevState Sb{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    StepAdj Ab{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double pt_b = 0.0, delp_b = 0.0, dz0_b = 0.0, u0_b = 0.0, v0_b = 0.0, qa0_b = 0.0, qa_b = 0.0;
    double qin_b[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid) {
      const double cq[6] = {TC(OUT_QV_DT), TC(OUT_QL_DT), TC(OUT_QR_DT), TC(OUT_QI_DT), TC(OUT_QS_DT), TC(OUT_QG_DT)};
      const double qf[6] = {S.qv, S.ql, S.qr, S.qi, S.qs, S.qg};
      const double dp1 = P.dp1, dp0 = delp;
      const double omq0 = dp0 / dp1, omq = dp1 / dp0;
      double qfb[6], omq_b = 0.0, omq0_b = 0.0;
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        const double q0 = qin[n] * omq0;
        qfb[n] = cq[n] * rdt * omq;
        const double q0_b = -cq[n] * rdt * omq;
        omq_b += cq[n] * rdt * (qf[n] - q0);
        qin_b[n] += q0_b * omq0;
        omq0_b += q0_b * qin[n];
      }
      const double cvm = K.c_air + S.qv * K.c_vap + (S.qr + S.ql) * K.C_LIQ + (S.qi + S.qs + S.qg) * K.C_ICE;
      const double gpt = TC(OUT_PT_DT) * rdt / K.CP_AIR;
      Sb.tz = gpt * cvm;
      pt_b -= gpt * cvm;
      const double cvm_b = gpt * (S.tz - pt);
      qfb[0] += cvm_b * K.c_vap;
      qfb[1] += cvm_b * K.C_LIQ;
      qfb[2] += cvm_b * K.C_LIQ;
      qfb[3] += cvm_b * K.C_ICE;
      qfb[4] += cvm_b * K.C_ICE;
      qfb[5] += cvm_b * K.C_ICE;
      Sb.qv = qfb[0], Sb.ql = qfb[1], Sb.qr = qfb[2], Sb.qi = qfb[3], Sb.qs = qfb[4], Sb.qg = qfb[5];
      Ab.dp1 += omq_b / dp0 - omq0_b * omq0 / dp1;
      delp_b += -omq_b * omq / dp0 + omq0_b / dp1;
      // the accumulator: qaz_out = qaz_in + the step's increments, and
      // qa_dt = rdt (qaz_out / ntimes - qa0) (without do_qa, which leaves
      // both alone)
      qa_b = TC(OUT_QAZ);
      if (!K.do_qa) {
        qa_b += TC(OUT_QA_DT) * rdt / (double)K.ntimes;
        qa0_b = -TC(OUT_QA_DT) * rdt;
      }
      Sb.w = TC(OUT_W);  // without do_sedi_w, wmp passes through unchanged
    }
    double m1_b = 0.0;
    if (K.sedi_transport) {
      const double u0 = TI(IN_UA, 0.0), v0 = TI(IN_VA, 0.0);
      const double mp = C.prev(m1);
      double au, av, b, D = 1.0;
      if (k == 0 || !valid) {
        au = u0;
        av = v0;
        b = 0.0;
      } else {
        D = delp + mp;
        au = delp * u0 / D;
        av = delp * v0 / D;
        b = mp / D;
      }
      double u1, v1;
      C.scan_affine2(au, b, av, b, u1, v1);
      const bool out_k = valid && k >= 1;  // udt, vdt are written for k >= 1 only
      const double cu = out_k ? TC(OUT_UDT) * rdt : 0.0, cv = out_k ? TC(OUT_VDT) * rdt : 0.0;
      u0_b -= cu;
      v0_b -= cv;
      double bv[1] = {b}, bn[1];
      C.template nextN<1>(bv, bn);
      const double cn = (valid && k < L - 1) ? bn[0] : 0.0;
      const double aa[2] = {cu, cv}, cc[2] = {cn, cn};
      double lam[2];
      C.template scanN_rev<2>(aa, cc, lam);
      const double pu[2] = {u1, v1};
      double pp[2];
      C.template prevN<2>(pu, pp);
      double mp_b = 0.0;
      if (valid) {
        if (k == 0) {
          u0_b += lam[0];
          v0_b += lam[1];
        } else {
          const double b_b = lam[0] * pp[0] + lam[1] * pp[1];
          u0_b += lam[0] * delp / D;
          v0_b += lam[1] * delp / D;
          delp_b += lam[0] * u0 / D + lam[1] * v0 / D;
          const double D_b = -lam[0] * au / D - lam[1] * av / D - b_b * b / D;
          delp_b += D_b;
          mp_b = b_b / D + D_b;
        }
      }
      double mv[1] = {mp_b}, mn[1];
      C.template nextN<1>(mv, mn);
      m1_b = (valid && k < L - 1) ? mn[0] : 0.0;
    }
    // surface totals: out = total * 86400 rdt / g
    const double convt = 86400.0 * K.rdt * K.RGRAV;
    const double rain_c = A.rain_b ? A.rain_b[col] * convt : 0.0;
    const double snow_c = A.snow_b ? A.snow_b[col] * convt : 0.0;
    const double ice_c = A.ice_b ? A.ice_b[col] * convt : 0.0;
    const double graupel_c = A.graupel_b ? A.graupel_b[col] * convt : 0.0;

    // ------------------------------------------------------ sub-steps, reversed
#pragma unroll 1
    for (int it = nt - 1; it >= 0; --it) {
      StepGeom Pg = P;
      substep_geometry(C, K, valid, pt, dz0, ck[it][0], Pg);
      Ab.den = 0.0;
      Ab.denfac = 0.0;
      Ab.dz = 0.0;
      double vtg_b = 0.0, vtr_b = 0.0, vts_b = 0.0;
      icloud_b<NW>(C, K, valid, ck[it][3], ck[it][4], Pg, ckv[it][1], ckv[it][0], ckv[it][2], qa_b, Sb, Ab, vtg_b,
                   vtr_b, vts_b);
#pragma unroll 1
      for (int pass = 1; pass >= 0; --pass) {
        warm_rain_b<NW>(C, K, valid, ck[it][2 * pass], Pg, m1_b, rain_c, pass == 1 ? vtr_b : 0.0, Sb, Ab);
        if (pass == 1)
          sedimentation_b<NW>(C, K, valid, ck[it][1], Pg, m1_b, ice_c, snow_c, graupel_c, vtg_b, vts_b, Sb, Ab);
      }
      // geometry: denfac = sqrt(SFCRHO / den), den = den0 dz0 / dz1,
      // dz1 = dz0 tz / t0, dz = heights(-dz1), den0 = -dp1 / (g dz0)
      if (valid) {
        const double den0 = -Pg.dp1 / (K.GRAV * dz0);
        const double den_b = Ab.den - Ab.denfac * 0.5 * Pg.denfac / Pg.den;
        double dz1_b = -Ab.dz;
        const double den0_b = den_b * dz0 / Pg.dz1;
        dz0_b += den_b * den0 / Pg.dz1;
        dz1_b -= den_b * Pg.den / Pg.dz1;
        dz0_b += dz1_b * ck[it][0].tz / pt;
        Sb.tz += dz1_b * dz0 / pt;
        pt_b -= dz1_b * Pg.dz1 / pt;
        Ab.dp1 -= den0_b / (K.GRAV * dz0);
        dz0_b += den0_b * Pg.dp1 / (K.GRAV * dz0 * dz0);
      }
    }

    // ----------------------------------------------------- fields_init reverse
    // replay to the state before fix_negative, then reverse the fix
    const double omq = delp / P.dp1;
    LevState S0{qin[0] * omq, qin[1] * omq, qin[2] * omq, qin[3] * omq, qin[4] * omq, qin[5] * omq, pt,
                TI(IN_W, 0.0)};
    if (K.fix_negative) {
      LevState S1 = S0;
      fix_negative_point(K, S1.qv, S1.ql, S1.qr, S1.qi, S1.qs, S1.qg, S1.tz);
      double* wq = C.work;
      double* wd = wq + RP;
      double* wqb = wq + 2 * RP;
      double* wdb = wq + 3 * RP;
      const bool sweep = C.any(valid && k < L - 1 && S1.qv < 0.0);
      double qv2 = S1.qv;
      if (sweep) {
        if (valid) {
          wq[k] = S1.qv;
          wd[k] = P.dp1;
        }
        C.sync();
        if (k == 0) {
          for (int kk = 1; kk < L; ++kk) {
            const double pq = wq[kk - 1];
            if (pq < 0.0) wq[kk] = wq[kk] + pq * wd[kk - 1] / wd[kk];
          }
        }
        C.sync();
        if (valid) qv2 = wq[k];
      }
      const bool clamp = k < L - 1 && qv2 < 0.0;
      const double qv3 = clamp ? 0.0 : qv2;
      double qb, db, qb1, db1;
      C.bcast2(qv3, P.dp1, L - 1, qb, db);
      C.bcast2(qv3, P.dp1, L - 2, qb1, db1);
      if ((qb < 0.0) && (qb1 > 0.0)) {
        const double dq = fmin(-qb * db, qb1 * db1);
        double c = 0.0;
        if (k == L - 2) {
          c = -Sb.qv / P.dp1;
          Ab.dp1 += Sb.qv * dq / (P.dp1 * P.dp1);
        }
        if (k == L - 1) {
          c = Sb.qv / P.dp1;
          Ab.dp1 -= Sb.qv * dq / (P.dp1 * P.dp1);
        }
        const double dq_b = C.colsum(c);
        if (min_first(-qb * db, qb1 * db1)) {
          if (k == L - 1) {
            Sb.qv -= dq_b * db;
            Ab.dp1 -= dq_b * qb;
          }
        } else {
          if (k == L - 2) {
            Sb.qv += dq_b * db1;
            Ab.dp1 += dq_b * qb1;
          }
        }
      }
      if (clamp) Sb.qv = 0.0;
      if (sweep) {
        if (valid) {
          wqb[k] = Sb.qv;
          wdb[k] = 0.0;
        }
        C.sync();
        if (k == 0) {
          for (int kk = L - 1; kk >= 1; --kk) {
            const double pq = wq[kk - 1];
            if (pq < 0.0) {
              const double gq = wqb[kk];
              wqb[kk - 1] += gq * wd[kk - 1] / wd[kk];
              wdb[kk - 1] += gq * pq / wd[kk];
              wdb[kk] -= gq * pq * wd[kk - 1] / (wd[kk] * wd[kk]);
            }
          }
        }
        C.sync();
        if (valid) {
          Sb.qv = wqb[k];
          Ab.dp1 += wdb[k];
        }
      }
      if (valid)
        fix_negative_point_b(K, S0.qv, S0.ql, S0.qr, S0.qi, S0.qs, S0.qg, S0.tz, Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs,
                             Sb.qg, Sb.tz);
    }
    // c_praut = cpaut (ccn RHOR)^(-1/3); ccn is one value per column
    double ccn_b = C.colsum(valid ? Ab.ccn : 0.0);
    const double cpr_b = C.colsum(valid ? Ab.c_praut : 0.0);
    if (!K.prog_ccn) {
      ccn_b += cpr_b * P.c_praut * (-1.0 / 3.0) / P.ccn;
      if (K.use_ccn) {
        // ccn = ccn0 RDGAS tz / p1 of the bottom level, tz = pt there
        double tzb, p1b;
        C.bcast2(pt, P.p1, L - 1, tzb, p1b);
        if (k == L - 1) {
          pt_b += ccn_b * P.ccn / tzb;
          Ab.p1 -= ccn_b * P.ccn / p1b;
        }
      }
    }
    if (valid) {
      // p1 = den0 RDGAS pt, den0 = -dp1 / (g dz0)
      const double den0 = -P.dp1 / (K.GRAV * dz0);
      const double den0_b = Ab.p1 * K.RDGAS * pt;
      pt_b += Ab.p1 * den0 * K.RDGAS;
      Ab.dp1 -= den0_b / (K.GRAV * dz0);
      dz0_b += den0_b * P.dp1 / (K.GRAV * dz0 * dz0);
      // q = q_in omq, omq = delp / dp1, dp1 = delp (1 - qv_in)
      const double sq_b[6] = {Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg};
      double omq_b = 0.0;
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        omq_b += sq_b[n] * qin[n];
        qin_b[n] += sq_b[n] * omq;
      }
      delp_b += omq_b / P.dp1;
      Ab.dp1 -= omq_b * omq / P.dp1;
      delp_b += Ab.dp1 * (1.0 - qin[0]);
      qin_b[0] -= Ab.dp1 * delp;
      pt_b += Sb.tz;
      TG(IN_PT) = pt_b;
      TG(IN_QV) = qin_b[0];
      TG(IN_QL) = qin_b[1];
      TG(IN_QR) = qin_b[2];
      TG(IN_QI) = qin_b[3];
      TG(IN_QS) = qin_b[4];
      TG(IN_QG) = qin_b[5];
      TG(IN_QA) = qa0_b;
      TG(IN_UA) = u0_b;
      TG(IN_VA) = v0_b;
      TG(IN_DELP) = delp_b;
      TG(IN_DELZ) = dz0_b;
      TG(IN_W) = Sb.w;
      TG(IN_QAZ) = qa_b;
    }
  }
  __syncthreads();
  store_tiles<NW, G, N_VJP_GRAD>(A.grad, sm + SM::out, A.ncol, A.nx, L, c0);
}

template <int NW, int G, int MINB>
cudaError_t launch_vjp(const VjpArgs& A, cudaStream_t st) {
  auto kern = mp_vjp_kernel<NW, G, MINB>;
  const size_t smem = VjpSmem<NW, G>::bytes;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t nblk = (A.ncol + G - 1) / G;
  kern<<<(unsigned)nblk, 32 * NW * G, smem, st>>>(A);
  return cudaGetLastError();
}

}  // namespace

int mp_vjp_max_substeps() { return VJP_MAXNT; }

cudaError_t mp_launch_vjp(const VjpArgs& A, cudaStream_t st) {
  const int L = A.nz;
  if (L <= 32) return launch_vjp<1, 2, SHIELD_VJP_MINB>(A, st);
  if (L <= 64) return launch_vjp<2, 2, SHIELD_VJP_MINB>(A, st);
  if (L <= 96) return launch_vjp<3, SHIELD_VJP_G3, SHIELD_VJP_MINB>(A, st);
  // 3 columns of 4 warps: 12 warps share each instruction fetch, as at L79
  // (C48 L127: 14.2 ms against 25.9 ms with one column per block)
  if (L <= 128) return launch_vjp<4, 3, 1>(A, st);
  return launch_vjp<8, 1, 1>(A, st);
}

}  // namespace shield
