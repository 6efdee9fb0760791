// Adjoint of the microphysics step (FP64): the vector-Jacobian product of
// the step's outputs -- the ten tendencies, wmp, the persistent
// cloud-fraction accumulator and the surface totals -- with respect to its
// inputs (pt, the six water species, qcld, ua, va, delprsi, delz, wmp and
// the accumulator), for pySHiELD's Microphysics.__call__
// (pySHiELD/stencils/microphysics.py:1981-2263).
//
// A sequence of launches over a workspace in global memory:
//  1. the replay, on the forward step's own thread layout (one thread per
//     level), runs the step with the forward's own stage functions and
//     records, per sub-step and point, the fields each stage changes at the
//     entry of every stage and inside warm_rain and icloud, the sub-step
//     geometry, the fall speeds and slopes, and each column's rain-fall
//     decisions (through shared-memory tiles, in whole-sector stores);
//     fields_update's reverse follows as a point launch and a column launch
//     of the momentum recurrence;
//  2. per sub-step, from the last: the pointwise reverses run one thread per
//     (level, column) point with consecutive columns on consecutive lanes,
//     so that a warp's 32 points take the same physics branches far more
//     often than the levels of one column do, and every warp of the launch
//     runs the same short code. The reverses of the vertical recurrences
//     (the rain fall, sedimentation's falls) run on the column layout
//     between them. The transposes of the slopes' three-point stencils are
//     gathered at the start of the next point launch;
//  3. fields_init's reverse: a column launch for fix_negative's borrows and
//     the CCN sums, then a point launch that writes the gradients.
// Branches follow the forward at the given input (the VJP of the piecewise
// smooth map on the branch it takes).
#include <cuda_runtime.h>

#include "mp_adjoint.cuh"
#include "mp_kernel.cuh"
#include "mp_launch.h"

namespace shield {

// ------------------------------------------------------------- workspace
// Every array holds one double per point p = k * ncol + col (level-major,
// consecutive columns adjacent) or per column.
//
// per sub-step and point: the states at
enum VjpCkSlot {
  CK_E0,   // the first warm_rain pass's entry
  CK_W1A,  // its state after the first evaporation,
  CK_W2A,  // after the fall,
  CK_W3A,  // after the second evaporation
  CK_E1,   // sedimentation's entry
  CK_E2,   // the second warm_rain pass's entry
  CK_W1B, CK_W2B, CK_W3B,
  CK_E3,   // icloud's entry
  CK_E4,   // the state between the ice processes and the adjustment
  N_CK
};
// Of these, only the fields a stage changes are stored (N_CKF per sub-step
// and point): the entry of each warm_rain pass in full (qv ql qr qi qs qg tz
// w), then the pass's block: after the first evaporation qv ql qr tz (+0),
// after the fall qr w tz (+4), after the second evaporation qv ql qr tz
// (+7), after autoconversion ql qr (+11); icloud's adjustment entry in full.
// Evaporation / accretion changes qv ql qr tz, the fall qr w (and tz with
// the heating), autoconversion ql qr.
enum VjpCkField { CKF_E0 = 0, CKF_PASS = 21, CKF_BLOCK = 8, CKF_E4 = 42, N_CKF = 50 };

// per sub-step and point: scalars
enum VjpSubScalar {
  SS_DEN, SS_DENFAC, SS_DZ, SS_DZ1,  // the sub-step geometry
  SS_VTR_A, SS_VTR_B,                // rain fall speed of each pass
  SS_VTG, SS_VTS, SS_VTI,            // graupel, snow and cloud ice fall speeds of sedimentation
  SS_SL_A, SS_SL_B,                  // liquid slope of each pass's autoconversion
  SS_SL_I, SS_S1QI,                  // icloud's ice slope and cloud ice after melting / freezing
  N_SS
};
// per sub-step and column: the rain-fall decisions of the two passes (0 / 1)
enum VjpSubColumn { SCC_FALL_A, SCC_FALL_B, N_SCC };
// per point, once: fields_init's dry mass and pressure
// per point, once: fields_init's dry mass and pressure, the precipitation
// flux summed over the sub-steps, and the final state (8)
enum VjpStepPoint { SP_DP1, SP_P1, SP_M1, SP_FIN, N_SP = SP_FIN + 8 };
// per column, once: fields_init's column values
// (SC_CCNB: the CCN cotangent's column total, set by the fields_init reverse)
enum VjpStepColumn { SC_HVAR, SC_RHADJ, SC_RHRAIN, SC_CCN, SC_CPRAUT, SC_CCNB, N_SC };
// per point: the adjoint state carried between the launches
enum VjpAdjField {
  AS_QV, AS_QL, AS_QR, AS_QI, AS_QS, AS_QG, AS_TZ, AS_W,  // the state's cotangent
  AS_DEN, AS_DENFAC, AS_DZ,                               // of the sub-step geometry
  AS_DP1, AS_P1, AS_CCN, AS_CPRAUT,                       // of fields_init's values
  AS_PT, AS_DELP, AS_DZ0, AS_QIN0,                        // of the inputs (six species from AS_QIN0)
  AS_QA = AS_QIN0 + 6,                                    // of the accumulator (passes through)
  AS_QA0, AS_U0, AS_V0,                                   // final: qcld, ua, va
  AS_M1,                                                  // of the precipitation flux at the level
  AS_VTR, AS_VTG, AS_VTS,                                 // of icloud's fall speeds
  AS_VTT,                                                 // of a pass's rain fall speed (fall to evaporation)
  AS_QLIQ, AS_QSOL, AS_CVM,                               // of icloud's melting / freezing outputs
  AS_SLI, AS_SLL,                                         // of the ice and liquid slopes
  AS_VTI,                                                 // of sedimentation's cloud ice fall speed
  AS_MELT,                                                // 1 where sedimentation melted cloud ice
  N_AS
};

int64_t mp_vjp_workspace_doubles(int nt, int64_t npts, int64_t ncol) {
  return npts * ((int64_t)nt * (N_CKF + N_SS) + N_SP + N_AS) + ncol * ((int64_t)nt * N_SCC + N_SC);
}

namespace {

struct Ws {
  double* base;
  int64_t npts, ncol;
  int nt;
  // stored checkpoint field f of sub-step it (VjpCkField offsets)
  SHD double* ckf(int it, int f) const { return base + ((int64_t)it * N_CKF + f) * npts; }
  SHD double* ss(int it, int s) const { return base + ((int64_t)nt * N_CKF + (int64_t)it * N_SS + s) * npts; }
  SHD double* sp(int s) const { return base + ((int64_t)nt * (N_CKF + N_SS) + s) * npts; }
  SHD double* as(int f) const { return base + ((int64_t)nt * (N_CKF + N_SS) + N_SP + f) * npts; }
  SHD double* cbase() const { return base + ((int64_t)nt * (N_CKF + N_SS) + N_SP + N_AS) * npts; }
  // the 8 field arrays (qv ql qr qi qs qg tz w) of the state at slot s of
  // sub-step it, from the fields stored there and at the slots before it
  SHD void ck(int it, int s, const double* (&f)[8]) const {
    if (s == CK_E4) {
      for (int n = 0; n < 8; ++n) f[n] = ckf(it, CKF_E4 + n);
      return;
    }
    const int pass = s >= CK_E2;
    const int b = pass * CKF_PASS, w = b + CKF_BLOCK;
    const int st = s - (pass ? CK_E2 : CK_E0);  // 0 entry, 1..3 W1..W3, 4 after autoconversion
    for (int n = 0; n < 8; ++n) f[n] = ckf(it, b + n);
    if (st == 1) {
      f[0] = ckf(it, w), f[1] = ckf(it, w + 1), f[2] = ckf(it, w + 2), f[6] = ckf(it, w + 3);
    } else if (st >= 2) {
      f[7] = ckf(it, w + 5);  // w after the fall
      if (st == 2) {
        f[0] = ckf(it, w), f[1] = ckf(it, w + 1), f[2] = ckf(it, w + 4), f[6] = ckf(it, w + 6);
      } else {
        f[0] = ckf(it, w + 7), f[1] = ckf(it, w + 8), f[2] = ckf(it, w + 9), f[6] = ckf(it, w + 10);
        if (st == 4) f[1] = ckf(it, w + 11), f[2] = ckf(it, w + 12);
      }
    }
  }
  SHD LevState ck_state(int it, int s, int64_t p) const {
    const double* f[8];
    ck(it, s, f);
    return LevState{f[0][p], f[1][p], f[2][p], f[3][p], f[4][p], f[5][p], f[6][p], f[7][p]};
  }
  SHD double* scc(int it, int s) const { return cbase() + ((int64_t)it * N_SCC + s) * ncol; }
  SHD double* sc(int s) const { return cbase() + ((int64_t)nt * N_SCC + s) * ncol; }
};

SHD Ws workspace(const VjpArgs& A) { return Ws{A.ws, (int64_t)A.nz * A.ncol, A.ncol, A.K.ntimes}; }

// a state's 8 fields, npts apart from p
SHD LevState load_lev(const double* q, int64_t npts) {
  return LevState{q[0], q[npts], q[2 * npts], q[3 * npts], q[4 * npts], q[5 * npts], q[6 * npts], q[7 * npts]};
}
SHD void store_lev(double* q, int64_t npts, const LevState& S) {
  q[0] = S.qv;
  q[npts] = S.ql;
  q[2 * npts] = S.qr;
  q[3 * npts] = S.qi;
  q[4 * npts] = S.qs;
  q[5 * npts] = S.qg;
  q[6 * npts] = S.tz;
  q[7 * npts] = S.w;
}

// The replay's recorder (NoRec's interface, mp_kernel.cuh): states to
// consecutive checkpoint slots from `st`, values to consecutive sub-step
// scalars from `val`, the column decision to `flg` (written by level 0).
// A warm_rain recorder (full false) stores the fields its stage changed
// into the pass's block at `st`; icloud's (full true) the whole state.
struct VjpRec {
  double *st, *val, *flg;
  int64_t npts;
  bool valid, head, full;
  SHD void state(int s, const LevState& S) const {
    if (!valid) return;
    if (full) {
      store_lev(st, npts, S);
    } else if (s == 1) {
      st[4 * npts] = S.qr;
      st[5 * npts] = S.w;
      st[6 * npts] = S.tz;
    } else {
      double* q = st + (s == 0 ? 0 : 7) * npts;
      q[0] = S.qv;
      q[npts] = S.ql;
      q[2 * npts] = S.qr;
      q[3 * npts] = S.tz;
    }
  }
  SHD void value(int s, double v) const {
    if (valid) val[(int64_t)s * npts] = v;
  }
  SHD void flag(bool f) const {
    if (head && flg) *flg = f ? 1.0 : 0.0;
  }
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

// mono_slope's derivative at a level with neighbours qp (above) and qn
// (below), times the slope's cotangent v_b: the contributions to q there
// (cq), above (cp) and below (cn). Zero outside 1 <= k <= L - 2.
SHD void mono_slope_coeffs(double qp, double q, double qn, int k, int L, double v_b, double& cp, double& cq,
                           double& cn) {
  cp = cq = cn = 0.0;
  if (k < 1 || k > L - 2) return;
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

// The transpose of the slope stencil gathered at level k of point p: q holds
// the slope's input field and vb the slopes' cotangents (level-major, ncol
// apart); the sum over the levels k - 1, k, k + 1 of their contribution to
// q at k.
SHD double slope_gather(const double* q, const double* vb, int64_t p, int64_t ncol, int k, int L) {
  double qq[5];
#pragma unroll
  for (int d = -2; d <= 2; ++d) qq[d + 2] = (k + d >= 0 && k + d < L) ? q[p + d * ncol] : 0.0;
  double cp, cq, cn, r = 0.0;
  mono_slope_coeffs(qq[1], qq[2], qq[3], k, L, vb[p], cp, cq, cn);
  r += cq;
  if (k >= 1) {
    mono_slope_coeffs(qq[0], qq[1], qq[2], k - 1, L, vb[p - ncol], cp, cq, cn);
    r += cn;
  }
  if (k <= L - 2) {
    mono_slope_coeffs(qq[2], qq[3], qq[4], k + 1, L, vb[p + ncol], cp, cq, cn);
    r += cp;
  }
  return r;
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

// sedi_heat reversed (microphysics.py:516-557 with C_LIQ, :1176-1217 with
// C_ICE) from the temperature tz before the heating and the species it saw.
// Sb.tz holds the heated temperature's cotangent on entry and the entry
// temperature's on return; the species' cotangents (through the heat
// capacity), flux_b (the flux leaving this level), dz1_b and dp1_b are added
// to; fp_b is set to the cotangent of fp, the flux entering from above,
// which the caller hands to the level above.
template <int NW>
SHD void sedi_heat_b(Column<NW>& C, const MpConst& K, double tz, double dz1, double dp1, double qv, double ql,
                     double qr, double qi, double qs, double qg, double flux, double fp, bool valid, double c_cond,
                     LevState& Sb, double& flux_b, double& fp_b, double& dz1_b, double& dp1_b) {
  const int k = C.k, L = C.L;
  const double dgz = -0.5 * K.GRAV * dz1;
  const double cs = K.CV_AIR + qv * K.CV_VAP + (qr + ql) * K.C_LIQ + (qi + qs + qg) * K.C_ICE;
  const double cvn = dp1 * cs;
  double a, b, D = 1.0, tmp = 1.0;
  if (k == 0) {
    tmp = cvn + flux * c_cond;
    a = tz + flux * dgz / tmp;
    b = 0.0;
  } else {
    D = cvn + c_cond * flux;
    a = ((cvn + c_cond * (flux - fp)) * tz + dgz * (fp + flux)) / D;
    b = fp * c_cond / D;
  }
  if (!valid) {
    a = tz;
    b = 0.0;
  }
  const double x = C.scan_affine(a, b);
  double bv[1] = {b}, bn[1];
  C.template nextN<1>(bv, bn);
  const double cn = (valid && k < L - 1) ? bn[0] : 0.0;
  const double lam = C.scan_affine_rev(valid ? Sb.tz : 0.0, cn);
  const double xp = C.prev(x);
  fp_b = 0.0;
  if (!valid) return;
  double cvn_b = 0.0, dgz_b = 0.0;
  if (k == 0) {
    const double u = flux * dgz;
    const double u_b = lam / tmp, tmp_b = -lam * u / (tmp * tmp);
    Sb.tz = lam;
    flux_b += u_b * dgz + tmp_b * c_cond;
    dgz_b += u_b * flux;
    cvn_b += tmp_b;
  } else {
    const double b_b = lam * xp;
    const double N_b = lam / D;
    const double D_b = -lam * a / D - b_b * b / D;
    Sb.tz = N_b * (cvn + c_cond * (flux - fp));
    cvn_b += N_b * tz + D_b;
    flux_b += N_b * (c_cond * tz + dgz) + D_b * c_cond;
    fp_b += N_b * (dgz - c_cond * tz) + b_b * c_cond / D;
    dgz_b += N_b * (fp + flux);
  }
  dz1_b += -0.5 * K.GRAV * dgz_b;
  dp1_b += cvn_b * cs;
  const double t = cvn_b * dp1;
  Sb.qv += t * K.CV_VAP;
  Sb.ql += t * K.C_LIQ;
  Sb.qr += t * K.C_LIQ;
  Sb.qi += t * K.C_ICE;
  Sb.qs += t * K.C_ICE;
  Sb.qg += t * K.C_ICE;
}

// sedimentation's falls reversed from its entry state S0 and the fall speeds
// the forward computed there: the ice, snow and graupel falls with their
// vertical-velocity transport and heating. m1s_b: cotangent of the solid
// flux at this level; ice_c, snow_c, graupel_c: of the surface totals; vt_b:
// the fall speeds' (vti, vts, vtg) cotangents, added to. Leaves Sb with
// respect to the state after cloud ice melting, which happened where
// melt_lev is set (the reverses of the melting and of the fall speeds are
// pointwise and run in their own launch).
template <int NW>
SHD void sedimentation_b(Column<NW>& C, const MpConst& K, bool valid, const LevState& S0, const StepGeom& P,
                         double vtg, double vti, double vts, double m1s_b, double ice_c, double snow_c,
                         double graupel_c, double (&vt_b)[3], LevState& Sb, StepAdj& Ab, bool& melt_lev) {
  const int k = C.k, L = C.L;
  const double dp1 = P.dp1, dz = P.dz;
  const int first = C.min_int((valid && S0.tz > K.tice) ? k : (1 << 30));
  melt_lev = (k >= first || k == L - 1) && valid;
  LevState S1 = S0;
  if (melt_lev) sedi_ice_melt(K, S1.qv, S1.ql, S1.qr, S1.qi, S1.qs, S1.qg, S1.tz);
  bool fi, fs, fg;
  C.any3(valid && (S1.qi > QRMIN), valid && (S1.qs > QRMIN), valid && (S1.qg > QRMIN), fi, fs, fg);
  fi = fi && (K.vi_fac >= 1.0e-5);
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
    // reverse: the heating by the falling species, which saw the fallen
    // state and their summed fluxes (do_sedi_heat) ...
    double flux_b[3] = {0.0, 0.0, 0.0}, dm_b[3] = {0.0, 0.0, 0.0}, pv_b[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (K.do_sedi_heat) {
      double m1s = 0.0, mp = 0.0;
      if (fi) {
        m1s = flux[0];
        mp = pv[0];
      }
      if (fs) {
        m1s = m1s + flux[1];
        mp = mp + pv[2];
      }
      if (fg) {
        m1s = m1s + flux[2];
        mp = mp + pv[4];
      }
      double hflux_b = 0.0, hmp_b = 0.0, dz1_b = 0.0;
      sedi_heat_b<NW>(C, K, S1.tz, P.dz1, dp1, S1.qv, S1.ql, S1.qr, qi2, qs2, qg2, m1s, mp, valid, K.C_ICE, Sb,
                      hflux_b, hmp_b, dz1_b, Ab.dp1);
      Ab.dz -= dz1_b;  // dz = -dz1 in exact arithmetic: the geometry's reverse takes -dz_b as dz1's cotangent
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        if ((n == 0 && fi) || (n == 1 && fs) || (n == 2 && fg)) {
          flux_b[n] += hflux_b;
          pv_b[2 * n] += hmp_b;
        }
      }
    }
    // ... then the vertical velocity, in the reverse species order
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
  } else if (K.do_sedi_heat) {
    // no species falls: the heating with zero fluxes
    double hflux_b = 0.0, hmp_b = 0.0, dz1_b = 0.0;
    sedi_heat_b<NW>(C, K, S1.tz, P.dz1, dp1, S1.qv, S1.ql, S1.qr, S1.qi, S1.qs, S1.qg, 0.0, 0.0, valid, K.C_ICE, Sb,
                    hflux_b, hmp_b, dz1_b, Ab.dp1);
    Ab.dz -= dz1_b;
  }
}
// The rain fall of a warm_rain pass reversed (microphysics.py:459-515), from
// W1, the state after the first evaporation: the vertical-velocity update,
// the implicit fall and the fall's dm. m1r_b: cotangent of the rain flux at
// this level; rain_c: of the surface rain total; vt_b: of the pass's fall
// speed on entry, with the fall's own part added on return.
template <int NW>
SHD void rain_fall_b(Column<NW>& C, const MpConst& K, bool valid, const LevState& W1, const StepGeom& P,
                     double vtr, double m1r_b, double rain_c, LevState& Sb, StepAdj& Ab, double& vt_b) {
  const int k = C.k, L = C.L;
  const double dm = P.dp1 * (1.0 + W1.qv + W1.ql + W1.qr + W1.qi + W1.qs + W1.qg);
  const FallRec R = implicit_fall_rec<NW>(C, W1.qr, vtr, P.dz, P.dp1, valid, K.dt_rain);
  double fv[2] = {R.flux, vtr}, pv[2];
  C.template prevN<2>(fv, pv);
  double flux_b = m1r_b, dm_b = 0.0, pv_b[2] = {0.0, 0.0};
  if (K.do_sedi_heat) {
    // the heating by the falling rain, which saw the fallen state
    double fp_b = 0.0, dz1_b = 0.0;
    sedi_heat_b<NW>(C, K, W1.tz, P.dz1, P.dp1, W1.qv, W1.ql, R.q1, W1.qi, W1.qs, W1.qg, R.flux, pv[0], valid,
                    K.C_LIQ, Sb, flux_b, fp_b, dz1_b, Ab.dp1);
    Ab.dz -= dz1_b;  // dz = -dz1 in exact arithmetic: the geometry's reverse takes -dz_b as dz1's cotangent
    pv_b[0] += fp_b;
  }
  if (K.do_sedi_w && valid)
    w_update_b(k, W1.w, dm, R.flux, vtr, pv[0], pv[1], Sb.w, dm_b, flux_b, vt_b, pv_b[0], pv_b[1]);
  if (k == L - 1) flux_b += rain_c;  // rain += the surface flux
  double pn[2];
  C.template nextN<2>(pv_b, pn);
  if (valid && k < L - 1) {
    flux_b += pn[0];
    vt_b += pn[1];
  }
  double qr_b = Sb.qr;
  implicit_fall_b<NW>(C, R, W1.qr, P.dz, P.dp1, valid, K.dt_rain, qr_b, flux_b, vt_b, Ab.dz, Ab.dp1);
  Sb.qr = qr_b;
  if (valid) {
    // dm = dp1 (1 + qv + ql + qr + qi + qs + qg)
    Ab.dp1 += dm_b * (1.0 + W1.qv + W1.ql + W1.qr + W1.qi + W1.qs + W1.qg);
    const double t = dm_b * P.dp1;
    Sb.qv += t;
    Sb.ql += t;
    Sb.qr += t;
    Sb.qi += t;
    Sb.qs += t;
    Sb.qg += t;
  }
}

// ------------------------------------------------------- column launches
// Shared memory of the column launches: NTILE field tiles (G rows of RP
// each), then G x 2 x SCR exchange scratch and G x NWORK work rows.
template <int NW, int G, int NTILE, int NWORK>
struct ColSmem {
  static constexpr int RP = Tiles<NW>::RP;
  static constexpr size_t scratch = (size_t)NTILE * G * RP;
  static constexpr size_t work = scratch + (size_t)G * 2 * Tiles<NW>::SCR;
  static constexpr size_t total = work + (size_t)G * NWORK * RP;
  static constexpr size_t bytes = total * sizeof(double);
};

// this thread's column group g and its level operations
template <int NW, int G, int NTILE, int NWORK>
SHD Column<NW> column_of(double* sm, int L, int& g) {
  using SM = ColSmem<NW, G, NTILE, NWORK>;
  const int tid = threadIdx.x;
  g = tid / (32 * NW);
  Column<NW> C;
  C.w = (tid >> 5) % NW;
  C.lane = tid & 31;
  C.k = 32 * C.w + C.lane;
  C.L = L;
  C.bar = 1 + g;
  C.scr = sm + SM::scratch + (size_t)g * 2 * Tiles<NW>::SCR;
  C.work = sm + SM::work + (size_t)g * NWORK * Tiles<NW>::RP;
  C.par = 0;
  return C;
}

// The column launches move their workspace fields through shared-memory
// tiles (field f, block column g, level k at (f * G + g) * RP + k):
// consecutive threads take consecutive columns of one level, so that a warp
// reads or writes whole sectors, and every load of a launch is issued before
// any of its arithmetic. 32 NW G >= G L threads: one element per thread and
// field. A null source reads as zero; a null destination is not written.
template <int NW, int G, int NF>
SHD void ws_gather(const double* const (&src)[NF], double* tiles, int64_t ncol, int L, int64_t c0) {
  constexpr int RP = Tiles<NW>::RP;
  const int tid = threadIdx.x, g = tid % G, k = tid / G;
  const bool ok = k < L && c0 + g < ncol;
  const int64_t o = (int64_t)k * ncol + c0 + g;
  double v[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) v[f] = (ok && src[f]) ? src[f][o] : 0.0;
  if (ok) {
#pragma unroll
    for (int f = 0; f < NF; ++f) tiles[(f * G + g) * RP + k] = v[f];
  }
}
template <int NW, int G, int NF>
SHD void ws_scatter(double* const (&dst)[NF], const double* tiles, int64_t ncol, int L, int64_t c0) {
  constexpr int RP = Tiles<NW>::RP;
  const int tid = threadIdx.x, g = tid % G, k = tid / G;
  if (!(k < L && c0 + g < ncol)) return;
  const int64_t o = (int64_t)k * ncol + c0 + g;
#pragma unroll
  for (int f = 0; f < NF; ++f)
    if (dst[f]) dst[f][o] = tiles[(f * G + g) * RP + k];
}

// de_ice (microphysics.py:110-120; the forward's de_ice_kernel) at one
// point, with the incoming qi_dt: qi and qs become the step's input state.
// Returns 0 when it leaves them, 1 when qi becomes qi - timestep qi_dt, 2
// when qi becomes qi0_max.
SHD int de_ice_point(const MpConst& K, double& qi, double& qs, double qi_dt) {
  const double qio = qi - K.timestep * qi_dt;
  const double qin = fmax(qio, K.qi0_max);
  if (!(qi > qin)) return 0;
  qs = qs + qi - qin;
  qi = qin;
  return max_first(qio, K.qi0_max) ? 1 : 2;
}
SHD double de_ice_qi_dt(const VjpArgs& A, int64_t col, int k) {
  const Fld3& f = A.de_ice_qi_dt;
  if (!f.p) return 0.0;
  return f.p[(col % A.nx) * f.si + (col / A.nx) * f.sj + (int64_t)k * f.sk];
}

// With de_ice, the block's staged qi and qs tiles (tiles[(f * G + g) * RP +
// k]) become the step's input state; then a block barrier.
template <int G, int RP>
SHD void de_ice_tiles(const VjpArgs& A, double* tiles, int64_t c0) {
  if (!A.K.de_ice) return;  // uniform over the block
  for (int e = threadIdx.x; e < G * A.nz; e += blockDim.x) {
    const int g = e % G, k = e / G;
    const int64_t col = c0 + g;
    if (col >= A.ncol) continue;
    de_ice_point(A.K, tiles[(IN_QI * G + g) * RP + k], tiles[(IN_QS * G + g) * RP + k], de_ice_qi_dt(A, col, k));
  }
  __syncthreads();
}

// 1a. The replay with its records, on the forward step's own thread layout
// LY (so that its vertical sums round as the forward's do): one block's G
// columns staged into shared memory as the forward kernel stages them.
template <class LY>
struct ReplaySmem {
  static constexpr size_t scratch = (size_t)N_VJP_IN * LY::G * LY::RP;
  static constexpr size_t work = scratch + (size_t)LY::NGRP * 2 * LY::SCR;
  static constexpr size_t rec = work + (size_t)LY::NGRP * LY::WORK;
  static constexpr int NREC = 15;  // record tiles: the largest group stored at once
  static constexpr size_t bytes = (rec + (size_t)NREC * LY::G * LY::RP) * sizeof(double);
};

// The replay's records collect in shared-memory tiles (field f of block
// column g at level k at (f * G + g) * RP + k) and go to their workspace
// rows dst[f] at block-uniform points: consecutive threads take consecutive
// columns of one level, so each warp stores whole sectors (stored where they
// arise, each warp store touched about 30 sectors: a warp holds the levels
// of one column). Block barriers on both sides.
template <int G, int RP, int NMAX>
SHD void flush_records(const double* rec, double* const (&dst)[NMAX], int n, int64_t ncol, int L, int64_t c0) {
  __syncthreads();
  for (int e = threadIdx.x; e < G * L; e += blockDim.x) {
    const int g = e % G, k = e / G;
    if (c0 + g >= ncol) continue;
    const int64_t o = (int64_t)k * ncol + c0 + g;
    for (int f = 0; f < n; ++f) dst[f][o] = rec[(f * G + g) * RP + k];
  }
  __syncthreads();
}

template <class LY, int MINB>
__global__ void __launch_bounds__(LY::THREADS, MINB) vjp_replay_kernel(const __grid_constant__ VjpArgs A) {
  extern __shared__ double sm[];
  using SM = ReplaySmem<LY>;
  constexpr int RP = LY::RP, G = LY::G;
  const MpConst& K = A.K;
  const MpConstF& KF = A.KF;
  const int L = A.nz;
  const int64_t c0 = (int64_t)blockIdx.x * G;
  {
    // element e < G L of each input tile (i-fastest storages: consecutive
    // columns on consecutive threads; k-fastest: consecutive levels)
    const int tid = threadIdx.x;
    const int g = tid % G, k = tid / G, gk = tid / L, kk = tid % L;
    const bool ok = c0 + g < A.ncol && k < L, okk = gk < G && c0 + gk < A.ncol;
    const int64_t i = ok ? (c0 + g) % A.nx : 0, j = ok ? (c0 + g) / A.nx : 0;
    const int64_t ik = okk ? (c0 + gk) % A.nx : 0, jk = okk ? (c0 + gk) / A.nx : 0;
    double v[N_VJP_IN];
#pragma unroll
    for (int f = 0; f < N_VJP_IN; ++f) {
      const Fld3 F = A.in[f];
      v[f] = 0.0;
      if (F.sk == 1) {
        if (okk) v[f] = F.p[ik * F.si + jk * F.sj + kk];
      } else if (ok) {
        v[f] = F.p[i * F.si + j * F.sj + (int64_t)k * F.sk];
      }
    }
#pragma unroll
    for (int f = 0; f < N_VJP_IN; ++f) {
      if (A.in[f].sk == 1) {
        if (okk) sm[(f * G + gk) * RP + kk] = v[f];
      } else if (ok) {
        sm[(f * G + g) * RP + k] = v[f];
      }
    }
  }
  __syncthreads();
  de_ice_tiles<G, RP>(A, sm, c0);
  typename LY::Col C;
  const int g = LY::setup(C, threadIdx.x, L, sm + SM::scratch, sm + SM::work);
  const bool slot_ok = g < G;
  const int64_t col = c0 + (slot_ok ? g : 0);
  const bool col_ok = slot_ok && col < A.ncol;
  const int k = C.k;
  const bool valid = col_ok && k < L;
  const double* tile = sm + (size_t)(slot_ok ? g : 0) * RP + (valid ? k : 0);
  auto TI = [&](int f, double dflt) -> double { return valid ? tile[(size_t)f * G * RP] : dflt; };
  const Ws W = workspace(A);
  const int64_t cc = col_ok ? col : 0;
  const int64_t p = (int64_t)(valid ? k : 0) * A.ncol + cc;
  const bool head = col_ok && k == 0;
  const int64_t ci = cc % A.nx, cj = cc / A.nx;
  const double land = A.land.p[ci * A.land.si + cj * A.land.sj];
  const double area = A.area.p[ci * A.area.si + cj * A.area.sj];
  const double pt = TI(IN_PT, 250.0), dz0 = TI(IN_DELZ, -100.0);
  LevState S;
  StepGeom P;
  P.den = 1.0;
  P.denfac = 1.0;
  P.dz1 = -100.0;
  P.dz = 100.0;
  fields_init(C, K, valid, pt, TI(IN_QV, 0.0), TI(IN_QL, 0.0), TI(IN_QR, 0.0), TI(IN_QI, 0.0), TI(IN_QS, 0.0),
              TI(IN_QG, 0.0), TI(IN_DELP, 1.0), TI(IN_W, 0.0), dz0, land, area, S, P);
  if (valid) {
    W.sp(SP_DP1)[p] = P.dp1;
    W.sp(SP_P1)[p] = P.p1;
  }
  if (head) {
    W.sc(SC_HVAR)[cc] = P.h_var;
    W.sc(SC_RHADJ)[cc] = P.rh_adj;
    W.sc(SC_RHRAIN)[cc] = P.rh_rain;
    W.sc(SC_CCN)[cc] = P.ccn;
    W.sc(SC_CPRAUT)[cc] = P.c_praut;
  }
  double m1 = 0.0, m1_sol = 0.0, vtr = VF_MIN, vtg = VF_MIN, vts = VF_MIN, qa = 0.0, ice = 0.0, snow = 0.0,
         graupel = 0.0;
  constexpr int NREC = SM::NREC;
  constexpr int64_t RS = (int64_t)G * RP;  // stride between record tiles
  const double* rec = sm + SM::rec;
  double* rt = sm + SM::rec + (size_t)(slot_ok ? g : 0) * RP + (valid ? k : 0);  // this thread's record slot
  auto put = [&](int f, double v) {
    if (valid) rt[f * RS] = v;
  };
  auto put_lev = [&](int f, const LevState& X) {
    if (valid) store_lev(rt + f * RS, RS, X);
  };
  const int nt = K.ntimes;
#pragma unroll 1
  for (int it = 0; it < nt; ++it) {
    substep_geometry(C, K, valid, pt, dz0, S, P);
    put_lev(0, S);
    put(8, P.den);
    put(9, P.denfac);
    put(10, P.dz);
    put(11, P.dz1);
    {
      double* d[NREC] = {};
      for (int f = 0; f < 8; ++f) d[f] = W.ckf(it, CKF_E0 + f);
      d[8] = W.ss(it, SS_DEN), d[9] = W.ss(it, SS_DENFAC), d[10] = W.ss(it, SS_DZ), d[11] = W.ss(it, SS_DZ1);
      flush_records<G, RP, NREC>(rec, d, 12, A.ncol, L, c0);
    }
    // the first warm_rain pass, sedimentation, the second pass (one copy of
    // the warm_rain code, run twice, as in the forward kernel)
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      double m1r, r1;
      // tiles 0 .. 12: the pass's block; 13: the fall speed; 14: the slope
      warm_rain<false>(C, K, KF, valid, S, P, vtr, m1r, r1, nullptr,
                       VjpRec{rt, rt + 14 * RS, W.scc(it, pass ? SCC_FALL_B : SCC_FALL_A) + cc, RS, valid, head,
                              false});
      m1 = (pass == 0) ? m1 + m1r : m1 + m1r + m1_sol;
      put(13, vtr);
      put(11, S.ql);  // autoconversion changed ql and qr
      put(12, S.qr);
      {
        double* d[NREC] = {};
        for (int f = 0; f < 13; ++f) d[f] = W.ckf(it, pass * CKF_PASS + CKF_BLOCK + f);
        d[13] = W.ss(it, pass ? SS_VTR_B : SS_VTR_A);
        d[14] = W.ss(it, pass ? SS_SL_B : SS_SL_A);
        flush_records<G, RP, NREC>(rec, d, 15, A.ncol, L, c0);
      }
      if (pass == 1) break;
      // tiles 0 .. 7: the state after sedimentation; 8, 9, 10: vtg, vts, vti
      sedimentation<false>(C, K, KF, valid, S, P, vtg, vts, m1_sol, ice, snow, graupel, nullptr,
                           VjpRec{nullptr, rt + 10 * RS, nullptr, RS, valid, false, false});
      put_lev(0, S);
      put(8, vtg);
      put(9, vts);
      {
        double* d[NREC] = {};
        for (int f = 0; f < 8; ++f) d[f] = W.ckf(it, CKF_PASS + f);
        d[8] = W.ss(it, SS_VTG), d[9] = W.ss(it, SS_VTS), d[10] = W.ss(it, SS_VTI);
        flush_records<G, RP, NREC>(rec, d, 11, A.ncol, L, c0);
      }
    }
    // tiles 0 .. 7: the state before the adjustment; 8, 9: the ice slope and
    // the melted / frozen cloud ice
    icloud<false>(C, K, KF, valid, S, P, qa, vtg, vtr, vts, VjpRec{rt, rt + 8 * RS, nullptr, RS, valid, false, true});
    {
      double* d[NREC] = {};
      for (int f = 0; f < 8; ++f) d[f] = W.ckf(it, CKF_E4 + f);
      d[8] = W.ss(it, SS_SL_I), d[9] = W.ss(it, SS_S1QI);
      flush_records<G, RP, NREC>(rec, d, 10, A.ncol, L, c0);
    }
  }
  put(0, m1);
  put_lev(1, S);
  {
    double* d[NREC] = {};
    d[0] = W.sp(SP_M1);
    for (int f = 0; f < 8; ++f) d[1 + f] = W.sp(SP_FIN + f);
    flush_records<G, RP, NREC>(rec, d, 9, A.ncol, L, c0);
  }
}

// ------------------------------------------------------- point launches
// One thread per point p = k * ncol + col: consecutive columns of one level
// on consecutive lanes.
#ifndef SHIELD_VJP_PT_THREADS
#define SHIELD_VJP_PT_THREADS 128
#endif
#ifndef SHIELD_VJP_PT_MINB
#define SHIELD_VJP_PT_MINB 4
#endif
constexpr int PT_THREADS = SHIELD_VJP_PT_THREADS;

struct PointIdx {
  int64_t p, col;
  int k;
};
SHD bool point_of(const Ws& W, PointIdx& q) {
  q.p = (int64_t)blockIdx.x * PT_THREADS + threadIdx.x;
  if (q.p >= W.npts) return false;
  q.k = (int)(q.p / W.ncol);
  q.col = q.p - (int64_t)q.k * W.ncol;
  return true;
}

// 1b. fields_update reversed (:1452-1553), pointwise part: the tendencies
// and wmp from the replay's final state, the accumulator; starts the adjoint
// state. One thread per point, consecutive columns on consecutive lanes.
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_update_pt(const __grid_constant__ VjpArgs A) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const int k = q.k;
  const MpConst& K = A.K;
  const int64_t i = col % A.nx, j = col / A.nx;
  auto in = [&](int f) -> double { return A.in[f].p[i * A.in[f].si + j * A.in[f].sj + (int64_t)k * A.in[f].sk]; };
  auto cot = [&](int f) -> double {
    const Fld3& F = A.cot[f];
    return F.p ? F.p[i * F.si + j * F.sj + (int64_t)k * F.sk] : 0.0;
  };
  const double rdt = K.rdt;
  const double pt = in(IN_PT), delp = in(IN_DELP);
  double qin[6] = {in(IN_QV), in(IN_QL), in(IN_QR), in(IN_QI), in(IN_QS), in(IN_QG)};
  if (K.de_ice) de_ice_point(K, qin[3], qin[4], de_ice_qi_dt(A, col, k));
  const LevState S = load_lev(W.sp(SP_FIN) + p, np);
  const double dp1 = W.sp(SP_DP1)[p];
  // q_dt = rdt (q - q0 omq0) omq, pt_dt = rdt (tz - t0) cvm / cp_air
  const double cq[6] = {cot(OUT_QV_DT), cot(OUT_QL_DT), cot(OUT_QR_DT), cot(OUT_QI_DT), cot(OUT_QS_DT), cot(OUT_QG_DT)};
  const double qf[6] = {S.qv, S.ql, S.qr, S.qi, S.qs, S.qg};
  const double dp0 = delp;
  const double omq0 = dp0 / dp1, omq = dp1 / dp0;
  double qfb[6], qin_b[6], omq_b = 0.0, omq0_b = 0.0;
#pragma unroll
  for (int n = 0; n < 6; ++n) {
    const double q0 = qin[n] * omq0;
    qfb[n] = cq[n] * rdt * omq;
    const double q0_b = -cq[n] * rdt * omq;
    omq_b += cq[n] * rdt * (qf[n] - q0);
    qin_b[n] = q0_b * omq0;
    omq0_b += q0_b * qin[n];
  }
  const double cvm = K.c_air + S.qv * K.c_vap + (S.qr + S.ql) * K.C_LIQ + (S.qi + S.qs + S.qg) * K.C_ICE;
  const double gpt = cot(OUT_PT_DT) * rdt / K.CP_AIR;
  LevState Sb;
  Sb.tz = gpt * cvm;
  const double pt_b = -gpt * cvm;
  const double cvm_b = gpt * (S.tz - pt);
  qfb[0] += cvm_b * K.c_vap;
  qfb[1] += cvm_b * K.C_LIQ;
  qfb[2] += cvm_b * K.C_LIQ;
  qfb[3] += cvm_b * K.C_ICE;
  qfb[4] += cvm_b * K.C_ICE;
  qfb[5] += cvm_b * K.C_ICE;
  Sb.qv = qfb[0], Sb.ql = qfb[1], Sb.qr = qfb[2], Sb.qi = qfb[3], Sb.qs = qfb[4], Sb.qg = qfb[5];
  Sb.w = cot(OUT_W);  // without do_sedi_w, wmp passes through unchanged
  // the accumulator: qaz_out = qaz_in + the step's increments, and
  // qa_dt = rdt (qaz_out / ntimes - qa0) (without do_qa, which leaves both)
  double qa_b = cot(OUT_QAZ), qa0_b = 0.0;
  if (!K.do_qa) {
    qa_b += cot(OUT_QA_DT) * rdt / (double)K.ntimes;
    qa0_b = -cot(OUT_QA_DT) * rdt;
  }
  store_lev(W.as(AS_QV) + p, np, Sb);
  W.as(AS_DP1)[p] = omq_b / dp0 - omq0_b * omq0 / dp1;
  W.as(AS_P1)[p] = 0.0;
  W.as(AS_CCN)[p] = 0.0;
  W.as(AS_CPRAUT)[p] = 0.0;
  W.as(AS_PT)[p] = pt_b;
  W.as(AS_DELP)[p] = -omq_b * omq / dp0 + omq0_b / dp1;
  W.as(AS_DZ0)[p] = 0.0;
#pragma unroll
  for (int n = 0; n < 6; ++n) W.as(AS_QIN0 + n)[p] = qin_b[n];
  W.as(AS_QA)[p] = qa_b;
  W.as(AS_QA0)[p] = qa0_b;
  if (!K.sedi_transport) {
    W.as(AS_U0)[p] = 0.0;
    W.as(AS_V0)[p] = 0.0;
    W.as(AS_M1)[p] = 0.0;
  }
}

// 1c. (sedi_transport) the momentum transport reversed (:1466-1532): the
// implicit recurrence of u and v by the precipitation flux, on the column
// layout. Tiles: u0, v0, delp, the summed flux m1, the udt / vdt
// cotangents; then the delp cotangent (read and written), the winds' and
// m1's cotangents (written).
enum MomTile { MT_U0 = 0, MT_V0, MT_DELP, MT_M1, MT_CU, MT_CV, MT_OUT, MT_ADELP = MT_OUT, MT_U0B, MT_V0B, MT_M1B, N_MT };
template <int NW, int G, int MINB>
__global__ void __launch_bounds__(32 * NW * G, MINB) vjp_momentum_kernel(const __grid_constant__ VjpArgs A) {
  extern __shared__ double sm[];
  constexpr int RP = Tiles<NW>::RP;
  const int L = A.nz;
  const int64_t c0 = (int64_t)blockIdx.x * G;
  const Ws W = workspace(A);
  {
    const Fld3 F[6] = {A.in[IN_UA], A.in[IN_VA], A.in[IN_DELP], Fld3{nullptr, 0, 0, 0}, A.cot[OUT_UDT], A.cot[OUT_VDT]};
    load_tiles<NW, G, 6>(F, sm, A.ncol, A.nx, L, c0);
    // the null fourth field's zero tile is overwritten by m1 (same thread, same element)
    const double* sm1[1] = {W.sp(SP_M1)};
    const double* sdp[1] = {W.as(AS_DELP)};
    ws_gather<NW, G, 1>(sm1, sm + (size_t)MT_M1 * G * RP, A.ncol, L, c0);
    ws_gather<NW, G, 1>(sdp, sm + (size_t)MT_ADELP * G * RP, A.ncol, L, c0);
  }
  __syncthreads();
  int g;
  Column<NW> C = column_of<NW, G, N_MT, 0>(sm, L, g);
  const int64_t col = c0 + g;
  if (col < A.ncol) {  // uniform over the column group
    const double rdt = A.K.rdt;
    const int k = C.k;
    const bool valid = k < L;
    double* tile = sm + (size_t)g * RP + (valid ? k : 0);
    auto T = [&](int f) -> double& { return tile[(size_t)f * G * RP]; };
    const double u0 = valid ? T(MT_U0) : 0.0, v0 = valid ? T(MT_V0) : 0.0, delp = valid ? T(MT_DELP) : 1.0;
    const double m1 = valid ? T(MT_M1) : 0.0;
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
    const double cu = out_k ? T(MT_CU) * rdt : 0.0, cv = out_k ? T(MT_CV) * rdt : 0.0;
    double u0_b = -cu, v0_b = -cv, delp_b = 0.0;
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
    if (valid) {
      T(MT_ADELP) += delp_b;
      T(MT_U0B) = u0_b;
      T(MT_V0B) = v0_b;
      T(MT_M1B) = k < L - 1 ? mn[0] : 0.0;
    }
  }
  __syncthreads();
  double* dst[N_MT - MT_OUT] = {W.as(AS_DELP), W.as(AS_U0), W.as(AS_V0), W.as(AS_M1)};
  ws_scatter<NW, G, N_MT - MT_OUT>(dst, sm + (size_t)MT_OUT * G * RP, A.ncol, L, c0);
}

// 2a. icloud's saturation adjustment reversed (subgrid_z_proc,
// microphysics_funcs.py:431-850) from the recorded state before it. Its own
// launch, ahead of the ice processes': each launch's code is half as long
// (C48 L79: 0.81 + 0.33 ms, against 1.46 ms for the two in one launch).
// Starts the sub-step's geometry cotangents.
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_subgrid_pt(const __grid_constant__ VjpArgs A,
                                                                                 int it) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const MpConst& K = A.K;
  const LevState E4 = W.ck_state(it, CK_E4, p);
  const double den = W.ss(it, SS_DEN)[p], denfac = W.ss(it, SS_DENFAC)[p], p1 = W.sp(SP_P1)[p];
  const double h_var = W.sc(SC_HVAR)[col], rh_adj = W.sc(SC_RHADJ)[col], rh_rain = W.sc(SC_RHRAIN)[col];
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  const double qa_b = W.as(AS_QA)[p];
  double den_b = 0.0, denfac_b = 0.0;
  subgrid_z_proc_b(K, h_var, rh_adj, rh_rain, qa_b, E4.qg, E4.qi, E4.ql, E4.qr, E4.qs, E4.qv, E4.tz, den, denfac, p1,
                   Sb.qg, Sb.qi, Sb.ql, Sb.qr, Sb.qs, Sb.qv, Sb.tz, den_b, denfac_b);
  store_lev(W.as(AS_QV) + p, np, Sb);
  W.as(AS_DEN)[p] = den_b;
  W.as(AS_DENFAC)[p] = denfac_b;
}

// 2b. icloud's melting / freezing and ice processes reversed
// (microphysics.py:1220-1449, icloud_main: microphysics_funcs.py:853-1260).
// Leaves the state's cotangent with respect to the melted / frozen state
// without the ice slope's part, the cotangents of melting / freezing's
// other outputs, of the slope and of the fall speeds.
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_icloud_pt(const __grid_constant__ VjpArgs A,
                                                                                int it) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const MpConst& K = A.K;
  const LevState E3 = W.ck_state(it, CK_E3, p);
  const double den = W.ss(it, SS_DEN)[p], denfac = W.ss(it, SS_DENFAC)[p], p1 = W.sp(SP_P1)[p];
  const double h_var = W.sc(SC_HVAR)[col];
  const double vtg = W.ss(it, SS_VTG)[p], vtr = W.ss(it, SS_VTR_B)[p], vts = W.ss(it, SS_VTS)[p];
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  const double den_b = W.as(AS_DEN)[p], denfac_b = W.as(AS_DENFAC)[p];
  LevState S1 = E3;
  double q_liq, q_sol, cvm;
  icloud_melt_freeze(K, S1.qv, S1.ql, S1.qr, S1.qi, S1.qs, S1.qg, S1.tz, den, q_liq, q_sol, cvm);
  const double hq = h_var * S1.qi;
  const double inner = fmax(QVMIN, hq);
  double sl = 0.0, di = inner;
  if (K.z_slope_ice) {
    sl = W.ss(it, SS_SL_I)[p];
    di = fmax(sl, inner);
  }
  const IcState Z0{S1.qg, S1.qi, S1.ql, S1.qr, S1.qs, S1.tz, q_liq, q_sol, cvm};
  const IcIn I{S1.qv, den, denfac, vtg, vtr, vts, p1, di};
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
  double sl_b = 0.0;
  if (K.z_slope_ice && max_first(sl, inner))
    sl_b = Ib.di;
  else if (!max_first(QVMIN, hq))
    Sb.qi += Ib.di * h_var;
  store_lev(W.as(AS_QV) + p, np, Sb);
  W.as(AS_DEN)[p] = den_b + Ib.den;
  W.as(AS_DENFAC)[p] = denfac_b + Ib.denfac;
  W.as(AS_DZ)[p] = 0.0;
  W.as(AS_P1)[p] += Ib.p1;
  W.as(AS_VTR)[p] = Ib.vtr;
  W.as(AS_VTG)[p] = Ib.vtg;
  W.as(AS_VTS)[p] = Ib.vts;
  W.as(AS_QLIQ)[p] = Zb.q_liq;
  W.as(AS_QSOL)[p] = Zb.q_sol;
  W.as(AS_CVM)[p] = Zb.cvm;
  W.as(AS_SLI)[p] = sl_b;
}

// 2c. Autoconversion of a warm_rain pass reversed (microphysics.py:559-653),
// without the liquid slope's transpose; for the second pass, first the end
// of icloud's reverse: the ice slope's transpose and melting / freezing.
template <int PASS>
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_autoconv_pt(const __grid_constant__ VjpArgs A,
                                                                                  int it) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const MpConst& K = A.K;
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  const double den = W.ss(it, SS_DEN)[p];
  double den_b = 0.0;
  if (PASS == 1) {
    if (K.z_slope_ice) Sb.qi += slope_gather(W.ss(it, SS_S1QI), W.as(AS_SLI), p, W.ncol, q.k, A.nz);
    const LevState E3 = W.ck_state(it, CK_E3, p);
    icloud_melt_freeze_b(K, E3.qv, E3.ql, E3.qr, E3.qi, E3.qs, E3.qg, E3.tz, den, W.as(AS_QLIQ)[p],
                         W.as(AS_QSOL)[p], W.as(AS_CVM)[p], Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg, Sb.tz, den_b);
  }
  const LevState W3 = W.ck_state(it, PASS ? CK_W3B : CK_W3A, p);
  const double h_var = W.sc(SC_HVAR)[col], ccn = W.sc(SC_CCN)[col], c_praut = W.sc(SC_CPRAUT)[col];
  double ccn_b = 0.0, cpr_b = 0.0, sl_b = 0.0;
  if (K.irain_f != 0) {
    autoconv_no_subgrid_var_b(K, W3.ql, W3.qr, W3.tz, den, ccn, c_praut, Sb.ql, Sb.qr, den_b, ccn_b, cpr_b);
  } else {
    const double hq = h_var * W3.ql;
    const double inner = fmax(QVMIN, hq);
    double sl = 0.0, dl = inner;
    if (K.z_slope_liq) {
      sl = W.ss(it, PASS ? SS_SL_B : SS_SL_A)[p];
      dl = fmax(sl, inner);
    }
    double dl_b = 0.0;
    autoconv_subgrid_var_b(K, W3.ql, W3.qr, W3.tz, den, ccn, c_praut, dl, Sb.ql, Sb.qr, den_b, ccn_b, cpr_b, dl_b);
    if (K.z_slope_liq && max_first(sl, inner))
      sl_b = dl_b;
    else if (!max_first(QVMIN, hq))
      Sb.ql += dl_b * h_var;
  }
  store_lev(W.as(AS_QV) + p, np, Sb);
  W.as(AS_DEN)[p] += den_b;
  W.as(AS_CCN)[p] += ccn_b;
  W.as(AS_CPRAUT)[p] += cpr_b;
  W.as(AS_SLL)[p] = sl_b;
}

// 2d. The liquid slope's transpose, then the second evaporation / accretion
// of a warm_rain pass reversed (columns with falling rain).
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_revap2_pt(const __grid_constant__ VjpArgs A,
                                                                                int it, int pass) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const MpConst& K = A.K;
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  if (K.irain_f == 0 && K.z_slope_liq)
    Sb.ql += slope_gather(W.ckf(it, pass * CKF_PASS + CKF_BLOCK + 8), W.as(AS_SLL), p, W.ncol, q.k, A.nz);
  if (W.scc(it, pass ? SCC_FALL_B : SCC_FALL_A)[col] != 0.0) {
    const LevState W2 = W.ck_state(it, pass ? CK_W2B : CK_W2A, p);
    const double den = W.ss(it, SS_DEN)[p], denfac = W.ss(it, SS_DENFAC)[p], h_var = W.sc(SC_HVAR)[col];
    double den_b = 0.0, denfac_b = 0.0;
    revap_racc_b(K, 0.5 * K.dt_rain, h_var, W2.qg, W2.qi, W2.ql, W2.qr, W2.qs, W2.qv, W2.tz, den, denfac, Sb.qg,
                 Sb.qi, Sb.ql, Sb.qr, Sb.qs, Sb.qv, Sb.tz, den_b, denfac_b);
    W.as(AS_DEN)[p] += den_b;
    W.as(AS_DENFAC)[p] += denfac_b;
  }
  store_lev(W.as(AS_QV) + p, np, Sb);
}

// 2f. The first evaporation / accretion and the fall speed of a warm_rain
// pass reversed (columns with falling rain); after the first pass, the
// reverse of the sub-step geometry (density, fall factor, layer thickness
// from the entry temperature: warm_rain with is_first, :349-380).
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_revap1_pt(const __grid_constant__ VjpArgs A,
                                                                                int it, int pass) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const MpConst& K = A.K;
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  const double den = W.ss(it, SS_DEN)[p], denfac = W.ss(it, SS_DENFAC)[p];
  double den_b = 0.0, denfac_b = 0.0;
  if (W.scc(it, pass ? SCC_FALL_B : SCC_FALL_A)[col] != 0.0) {
    const LevState W0 = W.ck_state(it, pass ? CK_E2 : CK_E0, p);
    const double h_var = W.sc(SC_HVAR)[col];
    revap_racc_b(K, 0.5 * K.dt_rain, h_var, W0.qg, W0.qi, W0.ql, W0.qr, W0.qs, W0.qv, W0.tz, den, denfac, Sb.qg,
                 Sb.qi, Sb.ql, Sb.qr, Sb.qs, Sb.qv, Sb.tz, den_b, denfac_b);
    rain_fspeed_b(K, W0.qr, den, W.as(AS_VTT)[p], Sb.qr, den_b);
  }
  if (pass == 0) {
    // den = den0 dz0 / dz1, den0 = -dp1 / (g dz0), denfac = sqrt(SFCRHO / den),
    // dz1 = dz0 tz / t0, dz = heights(-dz1) (= -dz1 in exact arithmetic)
    const int64_t i = col % A.nx, j = col / A.nx;
    const Fld3& fp = A.in[IN_PT];
    const Fld3& fz = A.in[IN_DELZ];
    const double pt = fp.p[i * fp.si + j * fp.sj + (int64_t)q.k * fp.sk];
    const double dz0 = fz.p[i * fz.si + j * fz.sj + (int64_t)q.k * fz.sk];
    const double dp1 = W.sp(SP_DP1)[p], dz1 = W.ss(it, SS_DZ1)[p], tz0 = W.ckf(it, CKF_E0 + 6)[p];
    const double aden = W.as(AS_DEN)[p] + den_b, adenfac = W.as(AS_DENFAC)[p] + denfac_b;
    const double den0 = -dp1 / (K.GRAV * dz0);
    const double dn_b = aden - adenfac * 0.5 * denfac / den;
    double dz1_b = -W.as(AS_DZ)[p];
    const double den0_b = dn_b * dz0 / dz1;
    double dz0_b = dn_b * den0 / dz1;
    dz1_b -= dn_b * den / dz1;
    dz0_b += dz1_b * tz0 / pt;
    Sb.tz += dz1_b * dz0 / pt;
    const double pt_b = -dz1_b * dz1 / pt;
    const double dp1_b = -den0_b / (K.GRAV * dz0);
    dz0_b += den0_b * dp1 / (K.GRAV * dz0 * dz0);
    W.as(AS_DZ0)[p] += dz0_b;
    W.as(AS_PT)[p] += pt_b;
    W.as(AS_DP1)[p] += dp1_b;
  } else {
    W.as(AS_DEN)[p] += den_b;
    W.as(AS_DENFAC)[p] += denfac_b;
  }
  store_lev(W.as(AS_QV) + p, np, Sb);
}

// ------------------------------------------------------- column launches
// The values the column reverses take on a padding level k >= L (finite, so
// that a zero cotangent stays zero through the scans).
SHD LevState pad_state() { return LevState{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 250.0, 0.0}; }

// 2e. The rain fall of a warm_rain pass reversed (columns with falling rain).
// Tiles, read-only first: W1 (8), dp1, dz, the fall speed, the flux's
// cotangent, icloud's fall-speed cotangent; then read and written: the
// state's cotangent (8), the geometry's dz and dp1 cotangents, the fall
// speed's cotangent (written only).
enum FallTile { FT_W1 = 0, FT_DP1 = 8, FT_DZ, FT_DZ1, FT_VTR, FT_M1, FT_VTRB, FT_OUT, FT_SB = FT_OUT, FT_ADZ = FT_SB + 8,
                FT_ADP1, FT_VTT, N_FT };
template <int NW, int G, int MINB>
__global__ void __launch_bounds__(32 * NW * G, MINB) vjp_fall_kernel(const __grid_constant__ VjpArgs A, int it,
                                                                     int pass) {
  extern __shared__ double sm[];
  constexpr int RP = Tiles<NW>::RP;
  const int L = A.nz;
  const int64_t c0 = (int64_t)blockIdx.x * G;
  const Ws W = workspace(A);
  const int64_t np = W.npts;
  const double* w1[8];
  W.ck(it, pass ? CK_W1B : CK_W1A, w1);
  double* sb = W.as(AS_QV);
  {
    const double* src[N_FT] = {w1[0], w1[1], w1[2], w1[3], w1[4], w1[5], w1[6], w1[7], W.sp(SP_DP1), W.ss(it, SS_DZ), A.K.do_sedi_heat ? W.ss(it, SS_DZ1) : nullptr,
                               W.ss(it, pass ? SS_VTR_B : SS_VTR_A),
                               W.as(AS_M1), pass ? W.as(AS_VTR) : nullptr, sb, sb + np, sb + 2 * np, sb + 3 * np,
                               sb + 4 * np, sb + 5 * np, sb + 6 * np, sb + 7 * np, W.as(AS_DZ), W.as(AS_DP1),
                               nullptr};
    ws_gather<NW, G, N_FT>(src, sm, A.ncol, L, c0);
  }
  __syncthreads();
  int g;
  Column<NW> C = column_of<NW, G, N_FT, 0>(sm, L, g);
  const int64_t col = c0 + g;
  // uniform over the column group
  if (col < A.ncol && W.scc(it, pass ? SCC_FALL_B : SCC_FALL_A)[col] != 0.0) {
    const MpConst& K = A.K;
    const int k = C.k;
    const bool valid = k < L;
    double* tile = sm + (size_t)g * RP + (valid ? k : 0);
    auto T = [&](int f) -> double& { return tile[(size_t)f * G * RP]; };
    const LevState W1 = valid ? LevState{T(FT_W1), T(FT_W1 + 1), T(FT_W1 + 2), T(FT_W1 + 3), T(FT_W1 + 4),
                                         T(FT_W1 + 5), T(FT_W1 + 6), T(FT_W1 + 7)}
                              : pad_state();
    StepGeom P;
    P.dp1 = valid ? T(FT_DP1) : 1.0;
    P.dz = valid ? T(FT_DZ) : 100.0;
    P.dz1 = valid ? T(FT_DZ1) : -100.0;
    const double vtr = valid ? T(FT_VTR) : VF_MIN;
    LevState Sb{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid)
      Sb = LevState{T(FT_SB), T(FT_SB + 1), T(FT_SB + 2), T(FT_SB + 3), T(FT_SB + 4), T(FT_SB + 5), T(FT_SB + 6),
                    T(FT_SB + 7)};
    StepAdj Ab{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double m1_b = valid ? T(FT_M1) : 0.0;
    const double rain_c = A.rain_b ? A.rain_b[col] * (86400.0 * K.rdt * K.RGRAV) : 0.0;
    double vt_b = valid ? T(FT_VTRB) : 0.0;
    rain_fall_b<NW>(C, K, valid, W1, P, vtr, m1_b, rain_c, Sb, Ab, vt_b);
    if (valid) {
      T(FT_SB) = Sb.qv;
      T(FT_SB + 1) = Sb.ql;
      T(FT_SB + 2) = Sb.qr;
      T(FT_SB + 3) = Sb.qi;
      T(FT_SB + 4) = Sb.qs;
      T(FT_SB + 5) = Sb.qg;
      T(FT_SB + 6) = Sb.tz;
      T(FT_SB + 7) = Sb.w;
      T(FT_ADZ) += Ab.dz;
      T(FT_ADP1) += Ab.dp1;
      T(FT_VTT) = vt_b;
    }
  }
  __syncthreads();
  // a column without falling rain writes back what it read (its fall-speed
  // cotangent is not read)
  double* dst[N_FT - FT_OUT] = {sb, sb + np, sb + 2 * np, sb + 3 * np, sb + 4 * np, sb + 5 * np, sb + 6 * np,
                                sb + 7 * np, W.as(AS_DZ), W.as(AS_DP1), W.as(AS_VTT)};
  ws_scatter<NW, G, N_FT - FT_OUT>(dst, sm + (size_t)FT_OUT * G * RP, A.ncol, L, c0);
}

// 2g. sedimentation's falls reversed (the ice, snow and graupel falls with
// their vertical-velocity transport and heating). Tiles, read-only first:
// E1 (8), dp1, dz, dz1, the flux's cotangent; then read and written: the
// state's cotangent (8), the geometry's dz and dp1 cotangents, the fall
// speeds (replaced by their cotangents: icloud's in, the totals out), the
// melting flag (written only).
enum SedTile { ST_E1 = 0, ST_DP1 = 8, ST_DZ, ST_DZ1, ST_M1, ST_OUT, ST_SB = ST_OUT, ST_ADZ = ST_SB + 8, ST_ADP1,
               ST_VTI, ST_VTS, ST_VTG, ST_MELT, N_ST };
template <int NW, int G, int MINB>
__global__ void __launch_bounds__(32 * NW * G, MINB) vjp_sed_kernel(const __grid_constant__ VjpArgs A, int it) {
  extern __shared__ double sm[];
  constexpr int RP = Tiles<NW>::RP;
  const int L = A.nz;
  const int64_t c0 = (int64_t)blockIdx.x * G;
  const Ws W = workspace(A);
  const int64_t np = W.npts;
  const double* e1[8];
  W.ck(it, CK_E1, e1);
  double* sb = W.as(AS_QV);
  {
    const double* src[N_ST] = {e1[0], e1[1], e1[2], e1[3], e1[4], e1[5], e1[6], e1[7], W.sp(SP_DP1), W.ss(it, SS_DZ),
                               A.K.do_sedi_heat ? W.ss(it, SS_DZ1) : nullptr, W.as(AS_M1), sb, sb + np, sb + 2 * np,
                               sb + 3 * np, sb + 4 * np, sb + 5 * np, sb + 6 * np, sb + 7 * np, W.as(AS_DZ),
                               W.as(AS_DP1), nullptr, W.as(AS_VTS), W.as(AS_VTG), nullptr};
    ws_gather<NW, G, N_ST>(src, sm, A.ncol, L, c0);
  }
  __syncthreads();
  int g;
  Column<NW> C = column_of<NW, G, N_ST, 0>(sm, L, g);
  const int64_t col = c0 + g;
  if (col < A.ncol) {
    const MpConst& K = A.K;
    const int k = C.k;
    const bool valid = k < L;
    double* tile = sm + (size_t)g * RP + (valid ? k : 0);
    auto T = [&](int f) -> double& { return tile[(size_t)f * G * RP]; };
    const int64_t p = (int64_t)(valid ? k : 0) * A.ncol + col;
    const LevState E1 = valid ? LevState{T(ST_E1), T(ST_E1 + 1), T(ST_E1 + 2), T(ST_E1 + 3), T(ST_E1 + 4),
                                         T(ST_E1 + 5), T(ST_E1 + 6), T(ST_E1 + 7)}
                              : pad_state();
    StepGeom P;
    P.dp1 = valid ? T(ST_DP1) : 1.0;
    P.dz = valid ? T(ST_DZ) : 100.0;
    P.dz1 = valid ? T(ST_DZ1) : -100.0;
    // the forward's fall speeds at sedimentation's entry
    const double vtg = valid ? W.ss(it, SS_VTG)[p] : VF_MIN, vts = valid ? W.ss(it, SS_VTS)[p] : VF_MIN,
                 vti = valid ? W.ss(it, SS_VTI)[p] : VF_MIN;
    LevState Sb{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid)
      Sb = LevState{T(ST_SB), T(ST_SB + 1), T(ST_SB + 2), T(ST_SB + 3), T(ST_SB + 4), T(ST_SB + 5), T(ST_SB + 6),
                    T(ST_SB + 7)};
    StepAdj Ab{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double convt = 86400.0 * K.rdt * K.RGRAV;
    const double snow_c = A.snow_b ? A.snow_b[col] * convt : 0.0;
    const double ice_c = A.ice_b ? A.ice_b[col] * convt : 0.0;
    const double graupel_c = A.graupel_b ? A.graupel_b[col] * convt : 0.0;
    const double m1_b = valid ? T(ST_M1) : 0.0;
    double vt_b[3] = {0.0, valid ? T(ST_VTS) : 0.0, valid ? T(ST_VTG) : 0.0};
    bool melt_lev;
    sedimentation_b<NW>(C, K, valid, E1, P, vtg, vti, vts, m1_b, ice_c, snow_c, graupel_c, vt_b, Sb, Ab, melt_lev);
    if (valid) {
      T(ST_SB) = Sb.qv;
      T(ST_SB + 1) = Sb.ql;
      T(ST_SB + 2) = Sb.qr;
      T(ST_SB + 3) = Sb.qi;
      T(ST_SB + 4) = Sb.qs;
      T(ST_SB + 5) = Sb.qg;
      T(ST_SB + 6) = Sb.tz;
      T(ST_SB + 7) = Sb.w;
      T(ST_ADZ) += Ab.dz;
      T(ST_ADP1) += Ab.dp1;
      T(ST_VTI) = vt_b[0];
      T(ST_VTS) = vt_b[1];
      T(ST_VTG) = vt_b[2];
      T(ST_MELT) = melt_lev ? 1.0 : 0.0;
    }
  }
  __syncthreads();
  double* dst[N_ST - ST_OUT] = {sb,          sb + np,     sb + 2 * np, sb + 3 * np,  sb + 4 * np,  sb + 5 * np,
                                sb + 6 * np, sb + 7 * np, W.as(AS_DZ), W.as(AS_DP1), W.as(AS_VTI), W.as(AS_VTS),
                                W.as(AS_VTG), W.as(AS_MELT)};
  ws_scatter<NW, G, N_ST - ST_OUT>(dst, sm + (size_t)ST_OUT * G * RP, A.ncol, L, c0);
}

// 2h. The pointwise end of sedimentation's reverse: cloud ice melting
// (:702-746) where it happened, then the fall speeds (microphysics_funcs.py:
// 269-341) at the entry state.
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_sed_tail_pt(const __grid_constant__ VjpArgs A,
                                                                                  int it) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts;
  const MpConst& K = A.K;
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  const LevState E1 = W.ck_state(it, CK_E1, p);
  if (W.as(AS_MELT)[p] != 0.0)
    sedi_ice_melt_b(K, E1.qv, E1.ql, E1.qr, E1.qi, E1.qs, E1.qg, E1.tz, Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg,
                    Sb.tz);
  double den_b = 0.0;
  fall_speed_b(K, E1.qg, E1.qi, E1.qs, E1.tz, W.ss(it, SS_DEN)[p], W.as(AS_VTG)[p], W.as(AS_VTI)[p],
               W.as(AS_VTS)[p], Sb.qg, Sb.qi, Sb.qs, Sb.tz, den_b);
  store_lev(W.as(AS_QV) + p, np, Sb);
  W.as(AS_DEN)[p] += den_b;
}

// 3a. fields_init reversed (:27-276), column part: fix_negative's borrows
// of vapour from the level above and by the bottom level (:229-276), and
// the column sums of the CCN cotangents (their total per column goes to
// SC_CCNB). Tiles: the inputs (those fields_init reads), dp1 and the CCN
// cotangents; then the vapour's and dp1's cotangents (read and written).
enum FixTile { XT_DP1 = N_VJP_IN, XT_CCN, XT_CPR, XT_OUT, XT_QVB = XT_OUT, XT_DP1B, N_XT };
template <int NW, int G, int MINB>
__global__ void __launch_bounds__(32 * NW * G, MINB) vjp_fixneg_kernel(const __grid_constant__ VjpArgs A) {
  extern __shared__ double sm[];
  constexpr int RP = Tiles<NW>::RP;
  const MpConst& K = A.K;
  const int L = A.nz;
  const int64_t c0 = (int64_t)blockIdx.x * G;
  const Ws W = workspace(A);
  {
    Fld3 F[N_VJP_IN];
    const Fld3 none{nullptr, 0, 0, 0};
    for (int f = 0; f < N_VJP_IN; ++f) F[f] = (f <= IN_QG || f == IN_DELP) ? A.in[f] : none;
    load_tiles<NW, G, N_VJP_IN>(F, sm, A.ncol, A.nx, L, c0);
    const double* src[N_XT - N_VJP_IN] = {W.sp(SP_DP1), W.as(AS_CCN), W.as(AS_CPRAUT), W.as(AS_QV), W.as(AS_DP1)};
    ws_gather<NW, G, N_XT - N_VJP_IN>(src, sm + (size_t)N_VJP_IN * G * RP, A.ncol, L, c0);
  }
  __syncthreads();
  de_ice_tiles<G, RP>(A, sm, c0);
  int g;
  Column<NW> C = column_of<NW, G, N_XT, 4>(sm, L, g);
  const int64_t col = c0 + g;
  if (col < A.ncol) {  // uniform over the column group
    const int k = C.k;
    const bool valid = k < L;
    double* tile = sm + (size_t)g * RP + (valid ? k : 0);
    auto T = [&](int f) -> double& { return tile[(size_t)f * G * RP]; };
    auto TI = [&](int f, double dflt) -> double { return valid ? T(f) : dflt; };
    const double pt = TI(IN_PT, 250.0), delp = TI(IN_DELP, 1.0);
    const double qin[6] = {TI(IN_QV, 0.0), TI(IN_QL, 0.0), TI(IN_QR, 0.0), TI(IN_QI, 0.0), TI(IN_QS, 0.0),
                           TI(IN_QG, 0.0)};
    StepGeom P;
    P.dp1 = valid ? T(XT_DP1) : 1.0;
    LevState Sb{valid ? T(XT_QVB) : 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    StepAdj Ab{0.0, 0.0, 0.0, valid ? T(XT_DP1B) : 0.0, 0.0, 0.0, 0.0};
    // c_praut = cpaut (ccn RHOR)^(-1/3); ccn is one value per column
    double ccn_b = C.colsum(valid ? T(XT_CCN) : 0.0);
    const double cpr_b = C.colsum(valid ? T(XT_CPR) : 0.0);
    if (!K.prog_ccn) ccn_b += cpr_b * W.sc(SC_CPRAUT)[col] * (-1.0 / 3.0) / W.sc(SC_CCN)[col];
    if (k == 0) W.sc(SC_CCNB)[col] = ccn_b;
    const double omq = delp / P.dp1;
    const LevState S0{qin[0] * omq, qin[1] * omq, qin[2] * omq, qin[3] * omq, qin[4] * omq, qin[5] * omq, pt, 0.0};
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
    }
    if (valid) {
      T(XT_QVB) = Sb.qv;
      T(XT_DP1B) = Ab.dp1;
    }
  }
  __syncthreads();
  double* dst[N_XT - XT_OUT] = {W.as(AS_QV), W.as(AS_DP1)};
  ws_scatter<NW, G, N_XT - XT_OUT>(dst, sm + (size_t)XT_OUT * G * RP, A.ncol, L, c0);
}

// 3b. fields_init reversed, pointwise part: fix_negative's point step, the
// bottom level's CCN (use_ccn), the pressure, the mixing-ratio conversion,
// de_ice; writes the gradients.
__global__ void __launch_bounds__(PT_THREADS, SHIELD_VJP_PT_MINB) vjp_init_pt(const __grid_constant__ VjpArgs A) {
  const Ws W = workspace(A);
  PointIdx q;
  if (!point_of(W, q)) return;
  const int64_t p = q.p, np = W.npts, col = q.col;
  const int k = q.k, L = A.nz;
  const MpConst& K = A.K;
  const int64_t i = col % A.nx, j = col / A.nx;
  auto at = [&](const Fld3& F) -> double { return F.p[i * F.si + j * F.sj + (int64_t)k * F.sk]; };
  auto put = [&](const Fld3& F, double v) {
    if (F.p) F.p[i * F.si + j * F.sj + (int64_t)k * F.sk] = v;
  };
  const double pt = at(A.in[IN_PT]), delp = at(A.in[IN_DELP]), dz0 = at(A.in[IN_DELZ]);
  double qin[6] = {at(A.in[IN_QV]), at(A.in[IN_QL]), at(A.in[IN_QR]), at(A.in[IN_QI]), at(A.in[IN_QS]),
                   at(A.in[IN_QG])};
  int de_ice_branch = 0;
  if (K.de_ice) de_ice_branch = de_ice_point(K, qin[3], qin[4], de_ice_qi_dt(A, col, k));
  const double dp1 = W.sp(SP_DP1)[p];
  LevState Sb = load_lev(W.as(AS_QV) + p, np);
  double Ab_dp1 = W.as(AS_DP1)[p], Ab_p1 = W.as(AS_P1)[p];
  double pt_b = W.as(AS_PT)[p], delp_b = W.as(AS_DELP)[p], dz0_b = W.as(AS_DZ0)[p];
  double qin_b[6];
#pragma unroll
  for (int n = 0; n < 6; ++n) qin_b[n] = W.as(AS_QIN0 + n)[p];
  const double omq = delp / dp1;
  if (K.fix_negative)
    fix_negative_point_b(K, qin[0] * omq, qin[1] * omq, qin[2] * omq, qin[3] * omq, qin[4] * omq, qin[5] * omq, pt,
                         Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg, Sb.tz);
  if (!K.prog_ccn && K.use_ccn && k == L - 1) {
    // ccn = ccn0 RDGAS tz / p1 of the bottom level, tz = pt there
    const double ccn_b = W.sc(SC_CCNB)[col], ccn = W.sc(SC_CCN)[col];
    pt_b += ccn_b * ccn / pt;
    Ab_p1 -= ccn_b * ccn / W.sp(SP_P1)[p];
  }
  // p1 = den0 RDGAS pt, den0 = -dp1 / (g dz0)
  const double den0 = -dp1 / (K.GRAV * dz0);
  const double den0_b = Ab_p1 * K.RDGAS * pt;
  pt_b += Ab_p1 * den0 * K.RDGAS;
  Ab_dp1 -= den0_b / (K.GRAV * dz0);
  dz0_b += den0_b * dp1 / (K.GRAV * dz0 * dz0);
  // q = q_in omq, omq = delp / dp1, dp1 = delp (1 - qv_in)
  const double sq_b[6] = {Sb.qv, Sb.ql, Sb.qr, Sb.qi, Sb.qs, Sb.qg};
  double omq_b = 0.0;
#pragma unroll
  for (int n = 0; n < 6; ++n) {
    omq_b += sq_b[n] * qin[n];
    qin_b[n] += sq_b[n] * omq;
  }
  delp_b += omq_b / dp1;
  Ab_dp1 -= omq_b * omq / dp1;
  delp_b += Ab_dp1 * (1.0 - qin[0]);
  qin_b[0] -= Ab_dp1 * delp;
  pt_b += Sb.tz;
  if (de_ice_branch == 2) {
    // de_ice reversed: where qi became qi0_max, the input qi moves qs
    // (qs + qi - qi0_max) and the tendencies it sets (qi_dt = dqi,
    // qs_dt += qi_dt - dqi, dqi = (qi0_max - qi + timestep qi_dt) rdt);
    // elsewhere qi and qs pass through
    auto cot = [&](int o) -> double { return A.cot[o].p ? at(A.cot[o]) : 0.0; };
    qin_b[3] = qin_b[4] + (cot(OUT_QS_DT) - cot(OUT_QI_DT)) * K.rdt;
  }
  put(A.grad[IN_PT], pt_b);
  put(A.grad[IN_QV], qin_b[0]);
  put(A.grad[IN_QL], qin_b[1]);
  put(A.grad[IN_QR], qin_b[2]);
  put(A.grad[IN_QI], qin_b[3]);
  put(A.grad[IN_QS], qin_b[4]);
  put(A.grad[IN_QG], qin_b[5]);
  put(A.grad[IN_QA], W.as(AS_QA0)[p]);
  put(A.grad[IN_UA], W.as(AS_U0)[p]);
  put(A.grad[IN_VA], W.as(AS_V0)[p]);
  put(A.grad[IN_DELP], delp_b);
  put(A.grad[IN_DELZ], dz0_b);
  put(A.grad[IN_W], Sb.w);
  put(A.grad[IN_QAZ], W.as(AS_QA)[p]);
}

// ---------------------------------------------------------------- launch
// The replay on layout RL (the forward step's), the column reverses on NW
// warps per column, G columns per block.
// Resident blocks per SM of the column reverses (__launch_bounds__): the
// rain fall's short code gains from two (C48 L79: 0.22 -> 0.16 ms per
// launch, 80 registers); sedimentation's and the update's did not, and the
// init launch's shared memory holds one.
#ifndef SHIELD_VJP_COL_MINB
#define SHIELD_VJP_COL_MINB 1
#endif
#ifndef SHIELD_VJP_FALL_MINB
#define SHIELD_VJP_FALL_MINB 2
#endif
#ifndef SHIELD_VJP_SED_MINB
#define SHIELD_VJP_SED_MINB 1
#endif
template <class RL, int RMINB, int NW, int G, int CMINB = SHIELD_VJP_COL_MINB, int FMINB = SHIELD_VJP_FALL_MINB,
          int SMINB = SHIELD_VJP_SED_MINB>
cudaError_t launch_vjp(const VjpArgs& A, cudaStream_t st) {
  using SU = ColSmem<NW, G, N_MT, 0>;
  using SF = ColSmem<NW, G, N_FT, 0>;
  using SS = ColSmem<NW, G, N_ST, 0>;
  using SI = ColSmem<NW, G, N_XT, 4>;
  cudaError_t e = cudaFuncSetAttribute(vjp_replay_kernel<RL, RMINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ReplaySmem<RL>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vjp_momentum_kernel<NW, G, CMINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SU::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vjp_fixneg_kernel<NW, G, CMINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SI::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vjp_fall_kernel<NW, G, FMINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SF::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vjp_sed_kernel<NW, G, SMINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SS::bytes);
  if (e != cudaSuccess) return e;
  const unsigned rblk = (unsigned)((A.ncol + RL::G - 1) / RL::G);
  const unsigned nblk = (unsigned)((A.ncol + G - 1) / G);
  const int64_t npts = (int64_t)A.nz * A.ncol;
  const unsigned pblk = (unsigned)((npts + PT_THREADS - 1) / PT_THREADS);
  constexpr int T = 32 * NW * G;
  vjp_replay_kernel<RL, RMINB><<<rblk, RL::THREADS, ReplaySmem<RL>::bytes, st>>>(A);
  vjp_update_pt<<<pblk, PT_THREADS, 0, st>>>(A);
  if (A.K.sedi_transport) vjp_momentum_kernel<NW, G, CMINB><<<nblk, T, SU::bytes, st>>>(A);
  for (int it = A.K.ntimes - 1; it >= 0; --it) {
    vjp_subgrid_pt<<<pblk, PT_THREADS, 0, st>>>(A, it);
    vjp_icloud_pt<<<pblk, PT_THREADS, 0, st>>>(A, it);
    vjp_autoconv_pt<1><<<pblk, PT_THREADS, 0, st>>>(A, it);
    vjp_revap2_pt<<<pblk, PT_THREADS, 0, st>>>(A, it, 1);
    vjp_fall_kernel<NW, G, FMINB><<<nblk, T, SF::bytes, st>>>(A, it, 1);
    vjp_revap1_pt<<<pblk, PT_THREADS, 0, st>>>(A, it, 1);
    vjp_sed_kernel<NW, G, SMINB><<<nblk, T, SS::bytes, st>>>(A, it);
    vjp_sed_tail_pt<<<pblk, PT_THREADS, 0, st>>>(A, it);
    vjp_autoconv_pt<0><<<pblk, PT_THREADS, 0, st>>>(A, it);
    vjp_revap2_pt<<<pblk, PT_THREADS, 0, st>>>(A, it, 0);
    vjp_fall_kernel<NW, G, FMINB><<<nblk, T, SF::bytes, st>>>(A, it, 0);
    vjp_revap1_pt<<<pblk, PT_THREADS, 0, st>>>(A, it, 0);
  }
  vjp_fixneg_kernel<NW, G, CMINB><<<nblk, T, SI::bytes, st>>>(A);
  vjp_init_pt<<<pblk, PT_THREADS, 0, st>>>(A);
  return cudaGetLastError();
}

}  // namespace

// The replay takes the plain step's launch shape for each level range
// (mp_plain.cu), so that it repeats the step's arithmetic exactly.
cudaError_t mp_launch_vjp(const VjpArgs& A, cudaStream_t st) {
  const int L = A.nz;
  if (L <= 32) return launch_vjp<ColumnLayout<1, 4>, 2, 1, 2>(A, st);
  if (L <= 64) return launch_vjp<ColumnLayout<2, 2>, 2, 2, 2>(A, st);
  if (L <= PACK80_LMAX) return launch_vjp<Packed80, PACK80_MINB, 3, 4>(A, st);
  if (L <= 96) return launch_vjp<ColumnLayout<3, 4>, 1, 3, 4>(A, st);
  if (L <= 128) return launch_vjp<ColumnLayout<4, 5>, 1, 4, 3>(A, st);
  return launch_vjp<ColumnLayout<8, 1>, 2, 8, 1>(A, st);
}

}  // namespace shield
