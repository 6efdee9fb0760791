// CPU harness for the adjoint tests (test infrastructure, built with g++ by
// tests/test_adjoint_pointwise.py).
//
// For each pointwise routine it evaluates, at n points, the hand-written
// adjoint (mp_adjoint.cuh) and the exact Jacobian-transpose product obtained
// by running the routine's own template with dual numbers, so the two can be
// compared to rounding. Inputs per point: NIN doubles, the first ND of which
// are differentiated (the rest are parameters); NOUT outputs.
#include <cstring>
#include <string>

#include "dual.h"  // before the physics, so its overloads are found
#include "mp_adjoint.cuh"
#include "mp_setup.h"
#include "column.h"

using namespace shield;

namespace {

MpConst make_K(const ShieldMpConfig* cfg, double ts) {
  MpConst K;
  std::memset(&K, 0, sizeof(K));
  setupm(*cfg, K);
  std::string why;
  set_timestep(*cfg, K, ts, why);
  return K;
}

template <class R>
int run(const ShieldMpConfig* cfg, double ts, int n, const double* X, const double* YB, double* XBH, double* XBD,
        double* Y, double* XBS) {
  static_assert(R::ND <= NDIR, "too many directions");
  const MpConst K = make_K(cfg, ts);
  for (int p = 0; p < n; ++p) {
    const double* x = X + (size_t)p * R::NIN;
    const double* yb = YB + (size_t)p * R::NOUT;
    Dual xd[R::NIN];
    for (int i = 0; i < R::NIN; ++i) xd[i] = (i < R::ND) ? Dual::seed(x[i], i) : Dual(x[i]);
    Dual yd[R::NOUT];
    R::template fwd<Dual>(K, xd, yd);
    // the same with magnitude duals: the size of the terms of each derivative
    ADual xa[R::NIN];
    for (int i = 0; i < R::NIN; ++i) xa[i] = (i < R::ND) ? ADual::seed(x[i], i) : ADual(x[i]);
    ADual ya[R::NOUT];
    R::template fwd<ADual>(K, xa, ya);
    for (int j = 0; j < R::ND; ++j) {
      double s = 0.0, a = 0.0;
      for (int i = 0; i < R::NOUT; ++i) {
        s += yb[i] * yd[i].d[j];
        a += std::fabs(yb[i]) * ya[i].d[j];
      }
      XBD[(size_t)p * R::ND + j] = s;
      XBS[(size_t)p * R::ND + j] = a;
    }
    double xv[R::NIN], yv[R::NOUT];
    for (int i = 0; i < R::NIN; ++i) xv[i] = x[i];
    R::template fwd<double>(K, xv, yv);
    for (int i = 0; i < R::NOUT; ++i) Y[(size_t)p * R::NOUT + i] = yv[i];
    double xb[R::ND];
    for (int j = 0; j < R::ND; ++j) xb[j] = 0.0;
    R::bwd(K, x, yb, xb);
    for (int j = 0; j < R::ND; ++j) XBH[(size_t)p * R::ND + j] = xb[j];
  }
  return 0;
}

// x = qg qi ql qr qs qv tz den denfac | dt h_var ; y = qg qi ql qr qs qv tz
struct Revap {
  static constexpr int NIN = 11, ND = 9, NOUT = 7;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    T qg = x[0], qi = x[1], ql = x[2], qr = x[3], qs = x[4], qv = x[5], tz = x[6];
    revap_racc<T>(K, val(x[9]), val(x[10]), qg, qi, ql, qr, qs, qv, tz, x[7], x[8]);
    y[0] = qg, y[1] = qi, y[2] = ql, y[3] = qr, y[4] = qs, y[5] = qv, y[6] = tz;
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    for (int i = 0; i < 7; ++i) xb[i] = yb[i];
    revap_racc_b(K, x[9], x[10], x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], x[8], xb[0], xb[1], xb[2], xb[3],
                 xb[4], xb[5], xb[6], xb[7], xb[8]);
  }
  template <bool A>
  static double val(const DualT<A>& d) {
    return d.v;
  }
  static double val(double d) { return d; }
};

// x = qr den ; y = vtr
struct RainFspeed {
  static constexpr int NIN = 2, ND = 2, NOUT = 1;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    y[0] = rain_fspeed<T>(K, x[0], x[1]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    rain_fspeed_b(K, x[0], x[1], yb[0], xb[0], xb[1]);
  }
};

// x = qg qi qs tk den ; y = vtg vti vts
struct FallSpeed {
  static constexpr int NIN = 5, ND = 5, NOUT = 3;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    fall_speed<T>(K, x[0], x[1], x[2], x[3], x[4], y[0], y[1], y[2]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    fall_speed_b(K, x[0], x[1], x[2], x[3], x[4], yb[0], yb[1], yb[2], xb[0], xb[1], xb[2], xb[3], xb[4]);
  }
};

// x = ql qr tz den ccn c_praut dl ; y = ql qr
struct AutoconvSub {
  static constexpr int NIN = 7, ND = 7, NOUT = 2;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    T ql = x[0], qr = x[1];
    autoconv_subgrid_var<T>(K, ql, qr, x[2], x[3], x[4], x[5], x[6]);
    y[0] = ql, y[1] = qr;
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    xb[0] = yb[0], xb[1] = yb[1];
    autoconv_subgrid_var_b(K, x[0], x[1], x[2], x[3], x[4], x[5], x[6], xb[0], xb[1], xb[3], xb[4], xb[5], xb[6]);
  }
};

// x = ql qr tz den ccn c_praut ; y = ql qr
struct AutoconvNoSub {
  static constexpr int NIN = 6, ND = 6, NOUT = 2;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    T ql = x[0], qr = x[1];
    autoconv_no_subgrid_var<T>(K, ql, qr, x[2], x[3], x[4], x[5]);
    y[0] = ql, y[1] = qr;
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    xb[0] = yb[0], xb[1] = yb[1];
    autoconv_no_subgrid_var_b(K, x[0], x[1], x[2], x[3], x[4], x[5], xb[0], xb[1], xb[3], xb[4], xb[5]);
  }
};

// x = v1 v2 q1 q2 rho | c a0 a1 a2 ; y
struct Acr3d {
  static constexpr int NIN = 9, ND = 5, NOUT = 1;
  template <class T>
  static void fwd(const MpConst&, const T* x, T* y) {
    y[0] = acr3d<T>(x[0], x[1], x[2], x[3], x[5], x[6], x[7], x[8], x[4]);
  }
  static void bwd(const MpConst&, const double* x, const double* yb, double* xb) {
    acr3d_b(x[0], x[1], x[2], x[3], x[5], x[6], x[7], x[8], x[4], yb[0], xb[0], xb[1], xb[2], xb[3], xb[4]);
  }
};

// x = ta den ; y = q dqdt
struct Wqs2 {
  static constexpr int NIN = 2, ND = 2, NOUT = 2;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    y[0] = wqs2<T>(K, x[0], x[1], y[1]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    double d;
    const double q = wqs2<double>(K, x[0], x[1], d);
    wqs2_b(K, x[0], x[1], q, d, yb[0], yb[1], xb[0], xb[1]);
  }
};
struct Iqs2 {
  static constexpr int NIN = 2, ND = 2, NOUT = 2;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    y[0] = iqs2<T>(K, x[0], x[1], y[1]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    double d;
    const double q = iqs2<double>(K, x[0], x[1], d);
    iqs2_b(K, x[0], x[1], q, d, yb[0], yb[1], xb[0], xb[1]);
  }
};

// x = tc dqs qsrho psacw psacr rho rhofac | c0..c4 ; y
struct Smlt {
  static constexpr int NIN = 12, ND = 7, NOUT = 1;
  template <class T>
  static void fwd(const MpConst&, const T* x, T* y) {
    y[0] = smlt<T>(x[0], x[1], x[2], x[3], x[4], x[7], x[8], x[9], x[10], x[11], x[5], x[6]);
  }
  static void bwd(const MpConst&, const double* x, const double* yb, double* xb) {
    smlt_b(x[0], x[1], x[2], x[3], x[4], x[7], x[8], x[9], x[10], x[11], x[5], x[6], yb[0], xb[0], xb[1], xb[2],
           xb[3], xb[4], xb[5], xb[6]);
  }
};

// x = tc dqs qgrho pgacw pgacr rho | c0..c4 ; y
struct Gmlt {
  static constexpr int NIN = 11, ND = 6, NOUT = 1;
  template <class T>
  static void fwd(const MpConst&, const T* x, T* y) {
    y[0] = gmlt<T>(x[0], x[1], x[2], x[3], x[4], x[6], x[7], x[8], x[9], x[10], x[5]);
  }
  static void bwd(const MpConst&, const double* x, const double* yb, double* xb) {
    gmlt_b(x[0], x[1], x[2], x[3], x[4], x[6], x[7], x[8], x[9], x[10], x[5], yb[0], xb[0], xb[1], xb[2], xb[3],
           xb[4], xb[5]);
  }
};

// x = qg qi ql qr qs qv tz den denfac vtg vtr vts p1 di q_liq q_sol cvm ; y = qg qi ql qr qs tz
struct Icloud {
  static constexpr int NIN = 17, ND = 17, NOUT = 6;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    T qg = x[0], qi = x[1], ql = x[2], qr = x[3], qs = x[4], tz = x[6];
    icloud_processes<T>(K, qg, qi, ql, qr, qs, x[5], tz, x[7], x[8], x[9], x[10], x[11], x[12], x[13], x[14], x[15],
                        x[16]);
    y[0] = qg, y[1] = qi, y[2] = ql, y[3] = qr, y[4] = qs, y[5] = tz;
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    const IcState Z0{x[0], x[1], x[2], x[3], x[4], x[6], x[14], x[15], x[16]};
    const IcIn I{x[5], x[7], x[8], x[9], x[10], x[11], x[12], x[13]};
    IcState Zb{yb[0], yb[1], yb[2], yb[3], yb[4], yb[5], 0.0, 0.0, 0.0};
    IcIn Ib{0, 0, 0, 0, 0, 0, 0, 0};
    icloud_processes_b(K, Z0, I, Zb, Ib);
    const double v[17] = {Zb.qg, Zb.qi, Zb.ql, Zb.qr, Zb.qs, Ib.qv, Zb.tz, Ib.den, Ib.denfac, Ib.vtg, Ib.vtr, Ib.vts,
                          Ib.p1, Ib.di, Zb.q_liq, Zb.q_sol, Zb.cvm};
    for (int i = 0; i < 17; ++i) xb[i] = v[i];
  }
};

// x = qg qi ql qr qs qv tz den denfac p1 | qa h_var rh_adj rh_rain ; y = qa qg qi ql qr qs qv tz
struct Subgrid {
  static constexpr int NIN = 14, ND = 10, NOUT = 8;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    T qa = x[10], qg = x[0], qi = x[1], ql = x[2], qr = x[3], qs = x[4], qv = x[5], tz = x[6];
    subgrid_z_proc<T>(K, Revap::val(x[11]), Revap::val(x[12]), Revap::val(x[13]), qa, qg, qi, ql, qr, qs, qv, tz, x[7],
                      x[8], x[9]);
    y[0] = qa, y[1] = qg, y[2] = qi, y[3] = ql, y[4] = qr, y[5] = qs, y[6] = qv, y[7] = tz;
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    for (int i = 0; i < 7; ++i) xb[i] = yb[i + 1];
    xb[7] = xb[8] = xb[9] = 0.0;
    subgrid_z_proc_b(K, x[11], x[12], x[13], yb[0], x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], x[8], x[9], xb[0],
                     xb[1], xb[2], xb[3], xb[4], xb[5], xb[6], xb[7], xb[8]);
  }
};

// x = qv ql qr qi qs qg tz ; y = the same after the block
struct SediMelt {
  static constexpr int NIN = 7, ND = 7, NOUT = 7;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    for (int i = 0; i < 7; ++i) y[i] = x[i];
    sedi_ice_melt<T>(K, y[0], y[1], y[2], y[3], y[4], y[5], y[6]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    for (int i = 0; i < 7; ++i) xb[i] = yb[i];
    sedi_ice_melt_b(K, x[0], x[1], x[2], x[3], x[4], x[5], x[6], xb[0], xb[1], xb[2], xb[3], xb[4], xb[5], xb[6]);
  }
};
// x = qv ql qr qi qs qg tz den ; y = qv ql qr qi qs qg tz q_liq q_sol cvm
struct MeltFreeze {
  static constexpr int NIN = 8, ND = 8, NOUT = 10;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    for (int i = 0; i < 7; ++i) y[i] = x[i];
    icloud_melt_freeze<T>(K, y[0], y[1], y[2], y[3], y[4], y[5], y[6], x[7], y[7], y[8], y[9]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    for (int i = 0; i < 7; ++i) xb[i] = yb[i];
    xb[7] = 0.0;
    icloud_melt_freeze_b(K, x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], yb[7], yb[8], yb[9], xb[0], xb[1], xb[2],
                         xb[3], xb[4], xb[5], xb[6], xb[7]);
  }
};
// x = qv ql qr qi qs qg tz ; y = the same after the block
struct FixNeg {
  static constexpr int NIN = 7, ND = 7, NOUT = 7;
  template <class T>
  static void fwd(const MpConst& K, const T* x, T* y) {
    for (int i = 0; i < 7; ++i) y[i] = x[i];
    fix_negative_point<T>(K, y[0], y[1], y[2], y[3], y[4], y[5], y[6]);
  }
  static void bwd(const MpConst& K, const double* x, const double* yb, double* xb) {
    for (int i = 0; i < 7; ++i) xb[i] = yb[i];
    fix_negative_point_b(K, x[0], x[1], x[2], x[3], x[4], x[5], x[6], xb[0], xb[1], xb[2], xb[3], xb[4], xb[5], xb[6]);
  }
};

}  // namespace

#define SHIELD_ADJ_ENTRY(NAME, R)                                                                               \
  extern "C" int adj_##NAME(const ShieldMpConfig* cfg, double ts, int n, const double* X, const double* YB,     \
                            double* XBH, double* XBD, double* Y, double* XBS) {                                \
    return run<R>(cfg, ts, n, X, YB, XBH, XBD, Y, XBS);                                                         \
  }                                                                                                            \
  extern "C" void adj_##NAME##_dims(int* d) {                                                                   \
    d[0] = R::NIN;                                                                                             \
    d[1] = R::ND;                                                                                              \
    d[2] = R::NOUT;                                                                                            \
  }

SHIELD_ADJ_ENTRY(revap_racc, Revap)
SHIELD_ADJ_ENTRY(rain_fspeed, RainFspeed)
SHIELD_ADJ_ENTRY(fall_speed, FallSpeed)
SHIELD_ADJ_ENTRY(autoconv_subgrid_var, AutoconvSub)
SHIELD_ADJ_ENTRY(autoconv_no_subgrid_var, AutoconvNoSub)
SHIELD_ADJ_ENTRY(acr3d, Acr3d)
SHIELD_ADJ_ENTRY(wqs2, Wqs2)
SHIELD_ADJ_ENTRY(iqs2, Iqs2)
SHIELD_ADJ_ENTRY(smlt, Smlt)
SHIELD_ADJ_ENTRY(gmlt, Gmlt)
SHIELD_ADJ_ENTRY(icloud_processes, Icloud)
SHIELD_ADJ_ENTRY(subgrid_z_proc, Subgrid)
SHIELD_ADJ_ENTRY(sedi_ice_melt, SediMelt)
SHIELD_ADJ_ENTRY(icloud_melt_freeze, MeltFreeze)
SHIELD_ADJ_ENTRY(fix_negative_point, FixNeg)

// One column of the whole step with dual numbers: input field f is seeded
// along DX[f] (direction f), so for every output row o and field f
//   JD[o][f] = sum over the output's levels of ybar_o (J dx_f)_o
// and JS[o][f] the same with magnitude duals and |ybar| (the size of the
// terms). X: NX rows of L levels; DX likewise; YB: NY rows of L levels then
// the 4 surface totals; Y: the output values (same layout as YB).
extern "C" int adj_column(const ShieldMpConfig* cfg, double ts, int L, double land, double area, const double* X,
                          const double* DX, const double* YB, double* JD, double* JS, double* Y) {
  using namespace colref;
  if (L < 3 || L > LMAX) return -1;
  const MpConst K = make_K(cfg, ts);
  constexpr int NO = NY + 4;
  auto* xd = new Dual[NX][LMAX];
  auto* yd = new Dual[NY][LMAX];
  auto* xa = new ADual[NX][LMAX];
  auto* ya = new ADual[NY][LMAX];
  Dual sd[4];
  ADual sa[4];
  for (int f = 0; f < NX; ++f)
    for (int k = 0; k < L; ++k) {
      xd[f][k] = Dual(X[f * L + k]);
      xd[f][k].d[f] = DX[f * L + k];
      xa[f][k] = ADual(X[f * L + k]);
      xa[f][k].d[f] = std::fabs(DX[f * L + k]);
    }
  column_step<Dual>(K, L, land, area, xd, yd, sd);
  column_step<ADual>(K, L, land, area, xa, ya, sa);
  for (int o = 0; o < NO; ++o)
    for (int f = 0; f < NX; ++f) {
      double s = 0.0, a = 0.0;
      if (o < NY) {
        for (int k = 0; k < L; ++k) {
          s += YB[o * L + k] * yd[o][k].d[f];
          a += std::fabs(YB[o * L + k]) * ya[o][k].d[f];
        }
      } else {
        s = YB[NY * L + (o - NY)] * sd[o - NY].d[f];
        a = std::fabs(YB[NY * L + (o - NY)]) * sa[o - NY].d[f];
      }
      JD[o * NX + f] = s;
      JS[o * NX + f] = a;
    }
  for (int o = 0; o < NY; ++o)
    for (int k = 0; k < L; ++k) Y[o * L + k] = yd[o][k].v;
  for (int i = 0; i < 4; ++i) Y[NY * L + i] = sd[i].v;
  delete[] xd;
  delete[] yd;
  delete[] xa;
  delete[] ya;
  return 0;
}

// A window of nsteps steps on one column, each followed by the state update
// of update_physics_state_with_tendencies (X += dt X_dt for the six species,
// qcld, pt, ua, va; wmp and the accumulator carried; delprsi, delz kept).
// XB: cotangents of the final state (NX rows of L). For every input row f:
// JD[f] = <XB, J_window dx_f>, JS[f] the size of its terms; XF: the final
// state values.
extern "C" int adj_column_window(const ShieldMpConfig* cfg, double ts, int L, double land, double area, int nsteps,
                                 const double* X, const double* DX, const double* XB, double* JD, double* JS,
                                 double* XF) {
  using namespace colref;
  if (L < 3 || L > LMAX || nsteps < 1) return -1;
  const MpConst K = make_K(cfg, ts);
  auto* xd = new Dual[NX][LMAX];
  auto* yd = new Dual[NY][LMAX];
  auto* xa = new ADual[NX][LMAX];
  auto* ya = new ADual[NY][LMAX];
  Dual sd[4];
  ADual sa[4];
  for (int f = 0; f < NX; ++f)
    for (int k = 0; k < L; ++k) {
      xd[f][k] = Dual(X[f * L + k]);
      xd[f][k].d[f] = DX[f * L + k];
      xa[f][k] = ADual(X[f * L + k]);
      xa[f][k].d[f] = std::fabs(DX[f * L + k]);
    }
  const int adv[10][2] = {{X_QV, Y_QV}, {X_QL, Y_QL}, {X_QR, Y_QR}, {X_QI, Y_QI}, {X_QS, Y_QS},
                          {X_QG, Y_QG}, {X_QA, Y_QA}, {X_PT, Y_PT}, {X_UA, Y_U}, {X_VA, Y_V}};
  for (int n = 0; n < nsteps; ++n) {
    column_step<Dual>(K, L, land, area, xd, yd, sd);
    column_step<ADual>(K, L, land, area, xa, ya, sa);
    for (int k = 0; k < L; ++k) {
      for (auto& a : adv) {
        xd[a[0]][k] = xd[a[0]][k] + yd[a[1]][k] * ts;
        xa[a[0]][k] = xa[a[0]][k] + ya[a[1]][k] * ts;
      }
      xd[X_W][k] = yd[Y_W][k];
      xa[X_W][k] = ya[Y_W][k];
      xd[X_QAZ][k] = yd[Y_QAZ][k];
      xa[X_QAZ][k] = ya[Y_QAZ][k];
    }
  }
  for (int f = 0; f < NX; ++f) {
    double s = 0.0, a = 0.0;
    for (int r = 0; r < NX; ++r)
      for (int k = 0; k < L; ++k) {
        s += XB[r * L + k] * xd[r][k].d[f];
        a += std::fabs(XB[r * L + k]) * xa[r][k].d[f];
      }
    JD[f] = s;
    JS[f] = a;
  }
  for (int r = 0; r < NX; ++r)
    for (int k = 0; k < L; ++k) XF[r * L + k] = xd[r][k].v;
  delete[] xd;
  delete[] yd;
  delete[] xa;
  delete[] ya;
  return 0;
}
