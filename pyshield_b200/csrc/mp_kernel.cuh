// The fused GFDL microphysics step: one warp per column, levels across lanes.
//
// Restates Microphysics.__call__ (pySHiELD/stencils/microphysics.py:1981-2263):
// fields_init, ntimes x [warm_rain(first), sedimentation, warm_rain, icloud],
// fields_update, all inside one launch.
//
// Layout of the work:
//  * a block owns CPB consecutive columns (warp w <-> column c0 + w);
//  * lane l of a warp holds levels k = l*P .. l*P+P-1 (k = 0 is the model
//    top), so the whole column state stays in registers for the whole step;
//  * the 14 input fields (13 state fields + the persistent cloud-fraction
//    accumulator) are staged once through shared memory with coalesced
//    loads (consecutive threads read consecutive columns of an i-fastest
//    field, or consecutive levels of a k-fastest one); the same tiles carry
//    the outputs back, so HBM traffic is the algorithmic bytes;
//  * column reductions (the ``no_fall`` flags) are __any_sync; the implicit
//    sedimentation, heating and momentum recurrences (first-order linear in
//    the level above) are warp scans of affine maps; heights are a warp
//    suffix sum.
#pragma once

#include "mp_physics.cuh"

namespace shield {

#define FULLMASK 0xffffffffu

template <int P>
struct Lev {
  static constexpr int PP = (P & 1) ? P : P + 1;  // odd lane pitch: conflict-free smem reads
  static constexpr int ROW = 32 * PP + 1;          // doubles per (field, column) tile row
  static __host__ __device__ constexpr int pos(int k) { return (k / P) * PP + (k % P); }
};

template <int P>
SHD void prev_vals(const double (&x)[P], double (&o)[P]) {
  double u = __shfl_up_sync(FULLMASK, x[P - 1], 1);
  o[0] = u;
#pragma unroll
  for (int s = 1; s < P; ++s) o[s] = x[s - 1];
}
template <int P>
SHD void next_vals(const double (&x)[P], double (&o)[P]) {
  double d = __shfl_down_sync(FULLMASK, x[0], 1);
#pragma unroll
  for (int s = 0; s < P - 1; ++s) o[s] = x[s + 1];
  o[P - 1] = d;
}
template <int P>
SHD double at_level(const double (&x)[P], int k) {
  const int owner = k / P, so = k - owner * P;
  double v = x[0];
#pragma unroll
  for (int s = 1; s < P; ++s)
    if (so == s) v = x[s];
  return __shfl_sync(FULLMASK, v, owner);
}
template <int P>
SHD bool col_any(const bool (&p)[P]) {
  bool a = false;
#pragma unroll
  for (int s = 0; s < P; ++s) a = a || p[s];
  return __any_sync(FULLMASK, a);
}

// X_k = a_k + b_k * X_{k-1} from the top down (b_0 must be 0). On return
// a[] holds X for this lane's levels.
template <int P>
SHD void scan_affine(double (&a)[P], const double (&b)[P], int lane) {
  double A = a[0], B = b[0];
#pragma unroll
  for (int s = 1; s < P; ++s) {
    A = a[s] + b[s] * A;
    B = b[s] * B;
  }
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    double pA = __shfl_up_sync(FULLMASK, A, d);
    double pB = __shfl_up_sync(FULLMASK, B, d);
    if (lane >= d) {
      A = A + B * pA;
      B = B * pB;
    }
  }
  double X = __shfl_up_sync(FULLMASK, A, 1);
  if (lane == 0) X = 0.0;
#pragma unroll
  for (int s = 0; s < P; ++s) {
    X = a[s] + b[s] * X;
    a[s] = X;
  }
}

// Layer-thickness from the BACKWARD height sweep ze_k = ze_{k+1} - dz1_k,
// ze_{L-1} = zs - dz1_{L-1}; dz_k = ze_k - ze_{k+1}, dz_{L-1} = ze_{L-1} - zs
// (microphysics.py:373-380, 445-452, 756-765, 830-837).
template <int P>
SHD void layer_dz(const double (&dz1)[P], const bool (&valid)[P], double zs, double (&dz)[P], int lane, int L) {
  double T = 0.0;
#pragma unroll
  for (int s = P - 1; s >= 0; --s)
    if (valid[s]) T = T - dz1[s];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    double v = __shfl_down_sync(FULLMASK, T, d);
    if (lane + d < 32) T = T + v;
  }
  double excl = __shfl_down_sync(FULLMASK, T, 1);
  if (lane == 31) excl = 0.0;
  double ze[P];
  double Y = zs + excl;
#pragma unroll
  for (int s = P - 1; s >= 0; --s) {
    if (valid[s]) Y = Y - dz1[s];
    ze[s] = Y;
  }
  double zn[P];
  next_vals<P>(ze, zn);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = lane * P + s;
    dz[s] = (k == L - 1) ? ze[s] - zs : ze[s] - zn[s];
  }
}

// Implicit upwind fall of one species (use_ppm = False): q is the dry mixing
// ratio (updated), dtf the fall time step; flux[] receives the cumulative
// mass flux m1; returns the surface flux (microphysics.py:454-507 and the
// ice/snow/graupel repeats).
//
// The reference accumulates m1_k = (m1_{k-1} + q_k) - qm_k level by level.
// With r_k the density from the implicit recurrence, r_k (dz_k + dd_k) =
// q_k + dd_{k-1} r_{k-1}, that running sum telescopes to m1_k = dd_k r_k:
// the mass leaving the bottom of level k. The telescoped form is used here.
// It equals the running sum in exact arithmetic, but it does not cancel: the
// running sum loses all its digits when little mass reaches the ground.
template <int P>
SHD double implicit_fall(double (&q)[P], const double (&vt)[P], const double (&dz)[P], const double (&dp1)[P],
                         const bool (&valid)[P], double dtf, double (&flux)[P], int lane, int L) {
  double dd[P], ddp[P], a[P], b[P], qmass[P];
#pragma unroll
  for (int s = 0; s < P; ++s) {
    dd[s] = dtf * vt[s];
    qmass[s] = valid[s] ? q[s] * dp1[s] : 0.0;
  }
  prev_vals<P>(dd, ddp);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = lane * P + s;
    const double D = dz[s] + dd[s];
    a[s] = qmass[s] / D;
    b[s] = (k == 0) ? 0.0 : ddp[s] / D;
    if (!valid[s]) {
      a[s] = 0.0;
      b[s] = 0.0;
    }
  }
  scan_affine<P>(a, b, lane);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    flux[s] = valid[s] ? dd[s] * a[s] : 0.0;
    if (valid[s]) q[s] = a[s] * dz[s] / dp1[s];
  }
  return at_level<P>(flux, L - 1);
}

// Vertical-velocity transport by the falling species (microphysics.py:492-515).
template <int P>
SHD void w_transport(double (&w)[P], const double (&dm)[P], const double (&flux)[P], const double (&vt)[P],
                     int lane) {
  double fp[P], vp[P];
  prev_vals<P>(flux, fp);
  prev_vals<P>(vt, vp);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = lane * P + s;
    if (k == 0)
      w[s] = (dm[s] * w[s] + flux[s] * vt[s]) / (dm[s] - flux[s]);
    else
      w[s] = (dm[s] * w[s] - fp[s] * vp[s] + flux[s] * vt[s]) / (dm[s] + fp[s] - flux[s]);
  }
}

// Implicit heating by falling condensate (microphysics.py:516-557 with
// C_LIQ, :1176-1217 with C_ICE).
template <int P>
SHD void sedi_heat(const MpConst& K, double (&tz)[P], const double (&dz1)[P], const double (&dp1)[P],
                   const double (&qv)[P], const double (&ql)[P], const double (&qr)[P], const double (&qi)[P],
                   const double (&qs)[P], const double (&qg)[P], const double (&flux)[P], const bool (&valid)[P],
                   double c_cond, int lane) {
  double fp[P], a[P], b[P];
  prev_vals<P>(flux, fp);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = lane * P + s;
    const double dgz = -0.5 * K.GRAV * dz1[s];
    const double cvn = dp1[s] * (K.CV_AIR + qv[s] * K.CV_VAP + (qr[s] + ql[s]) * K.C_LIQ + (qi[s] + qs[s] + qg[s]) * K.C_ICE);
    if (k == 0) {
      const double tmp = cvn + flux[s] * c_cond;
      a[s] = tz[s] + flux[s] * dgz / tmp;
      b[s] = 0.0;
    } else {
      const double D = cvn + c_cond * flux[s];
      a[s] = ((cvn + c_cond * (flux[s] - fp[s])) * tz[s] + dgz * (fp[s] + flux[s])) / D;
      b[s] = fp[s] * c_cond / D;
    }
    if (!valid[s]) {
      a[s] = tz[s];
      b[s] = 0.0;
    }
  }
  scan_affine<P>(a, b, lane);
#pragma unroll
  for (int s = 0; s < P; ++s) tz[s] = a[s];
}

// Monotone vertical slope for autoconversion (microphysics.py:595-620,
// 1341-1367), before the h_var floor.
template <int P>
SHD void mono_slope(const double (&q)[P], double (&d)[P], int lane, int L) {
  double qp[P], dq[P], dqn[P];
  prev_vals<P>(q, qp);
#pragma unroll
  for (int s = 0; s < P; ++s) dq[s] = 0.5 * (q[s] - qp[s]);
  next_vals<P>(dq, dqn);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = lane * P + s;
    double v = 0.0;
    if (k >= 1 && k <= L - 2) {
      v = 0.5 * fmin(fabs(dq[s] + dqn[s]), 0.5 * q[s]);
      if (dq[s] * dqn[s] <= 0.0) {
        if (dq[s] > 0.0)
          v = fmin(v, fmin(dq[s], -dqn[s]));
        else
          v = 0.0;
      }
    }
    d[s] = v;
  }
}

// ----------------------------------------------------------------- staging
template <int P, int CPB>
SHD void stage_in(const MpArgs& A, double* sm, int64_t c0) {
  using LV = Lev<P>;
  const int L = A.nz;
  const int tid = threadIdx.x;
  const int w = tid % CPB;
  const int kk0 = tid / CPB;
  constexpr int KSTEP = 32;  // (CPB * 32) / CPB
  const int64_t col = c0 + w;
  const bool ok = col < A.ncol;
  const int64_t i = ok ? col % A.nx : 0, j = ok ? col / A.nx : 0;
  const int ww = tid >> 5, ln = tid & 31;
  const int64_t colw = c0 + ww;
  const bool okw = colw < A.ncol;
  const int64_t iw = okw ? colw % A.nx : 0, jw = okw ? colw / A.nx : 0;
#pragma unroll 1
  for (int f = 0; f < N_IN; ++f) {
    const Fld3 F = A.in[f];
    if (F.sk == 1) {
      if (okw) {
        const double* src = F.p + iw * F.si + jw * F.sj;
        double* dst = sm + (f * CPB + ww) * LV::ROW;
#pragma unroll 4
        for (int k = ln; k < L; k += 32) dst[LV::pos(k)] = src[k];
      }
    } else if (ok) {
      const double* src = F.p + i * F.si + j * F.sj;
      double* dst = sm + (f * CPB + w) * LV::ROW;
#pragma unroll 4
      for (int k = kk0; k < L; k += KSTEP) dst[LV::pos(k)] = src[(int64_t)k * F.sk];
    }
  }
}

enum OutMode { OM_SKIP = 0, OM_ADD = 1, OM_ADD_K1 = 2, OM_SET = 3 };

template <int P, int CPB>
SHD void stage_out(const MpArgs& A, const double* sm, int64_t c0) {
  using LV = Lev<P>;
  const MpConst& K = A.K;
  const int L = A.nz;
  const int tid = threadIdx.x;
  const int w = tid % CPB;
  const int kk0 = tid / CPB;
  const int64_t col = c0 + w;
  const bool ok = col < A.ncol;
  const int64_t i = ok ? col % A.nx : 0, j = ok ? col / A.nx : 0;
  const int ww = tid >> 5, ln = tid & 31;
  const int64_t colw = c0 + ww;
  const bool okw = colw < A.ncol;
  const int64_t iw = okw ? colw % A.nx : 0, jw = okw ? colw / A.nx : 0;
#pragma unroll 1
  for (int o = 0; o < N_OUT; ++o) {
    int mode = OM_ADD;
    if (o == OUT_UDT || o == OUT_VDT) mode = K.sedi_transport ? OM_ADD_K1 : OM_SKIP;
    if (o == OUT_QA_DT && K.do_qa) mode = OM_SET;
    if (o == OUT_W) mode = K.do_sedi_w ? OM_SET : OM_SKIP;
    if (o == OUT_QAZ) mode = OM_SET;
    if (mode == OM_SKIP) continue;
    const Fld3 F = A.out[o];
    const int kmin = (mode == OM_ADD_K1) ? 1 : 0;
    if (F.sk == 1) {
      if (okw) {
        double* dst = F.p + iw * F.si + jw * F.sj;
        const double* src = sm + (o * CPB + ww) * LV::ROW;
        for (int k = ln; k < L; k += 32) {
          if (k < kmin) continue;
          const double v = src[LV::pos(k)];
          dst[k] = (mode == OM_SET) ? v : dst[k] + v;
        }
      }
    } else if (ok) {
      double* dst = F.p + i * F.si + j * F.sj;
      const double* src = sm + (o * CPB + w) * LV::ROW;
#pragma unroll 4
      for (int k = kk0; k < L; k += 32) {
        if (k < kmin) continue;
        const double v = src[LV::pos(k)];
        double* d = dst + (int64_t)k * F.sk;
        *d = (mode == OM_SET) ? v : *d + v;
      }
    }
  }
}

// ------------------------------------------------------------------ kernel
template <int P, int CPB>
__global__ void __launch_bounds__(CPB * 32, (CPB <= 4) ? 2 : 1) mp_step_kernel(const __grid_constant__ MpArgs A) {
  using LV = Lev<P>;
  extern __shared__ double sm[];
  const MpConst& K = A.K;
  const int L = A.nz;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t c0 = (int64_t)blockIdx.x * CPB;

  stage_in<P, CPB>(A, sm, c0);
  __syncthreads();

  const int64_t col = c0 + warp;
  double* tile = sm + warp * LV::ROW + lane * LV::PP;  // + f * CPB * ROW + s
  auto TL = [&](int f, int s) -> double& { return tile[f * CPB * LV::ROW + s]; };

  if (col < A.ncol) {
    const int64_t ci = col % A.nx, cj = col / A.nx;
    bool valid[P];
    double qv[P], ql[P], qr[P], qi[P], qs[P], qg[P], tz[P], qa[P], m1[P], w[P], dp1[P], p1[P];
    double den[P], denfac[P], dz1[P], dz[P], m1_sol[P], vtr[P], vtg[P], vts[P];

    // ------------------------------------------------ fields_init (:27-276)
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int k = lane * P + s;
      valid[s] = k < L;
      double pt = 250.0, qvi = 0.0, qli = 0.0, qri = 0.0, qii = 0.0, qsi = 0.0, qgi = 0.0, delp = 1.0,
             wz = 0.0, qaz = 0.0;
      if (valid[s]) {
        pt = TL(IN_PT, s);
        qvi = TL(IN_QV, s);
        qli = TL(IN_QL, s);
        qri = TL(IN_QR, s);
        qii = TL(IN_QI, s);
        qsi = TL(IN_QS, s);
        qgi = TL(IN_QG, s);
        delp = TL(IN_DELP, s);
        wz = TL(IN_W, s);
        qaz = TL(IN_QAZ, s);
      }
      tz[s] = pt;
      dp1[s] = delp;
      dp1[s] = dp1[s] * (1.0 - qvi);
      const double omq = delp / dp1[s];
      qv[s] = qvi * omq;
      ql[s] = qli * omq;
      qr[s] = qri * omq;
      qi[s] = qii * omq;
      qs[s] = qsi * omq;
      qg[s] = qgi * omq;
      const double dz0 = valid[s] ? TL(IN_DELZ, s) : -100.0;
      const double den0 = -dp1[s] / (K.GRAV * dz0);
      p1[s] = den0 * K.RDGAS * pt;
      m1[s] = 0.0;
      w[s] = wz;
      qa[s] = qaz;
      m1_sol[s] = 0.0;
    }
    const double land = A.land.p[ci * A.land.si + cj * A.land.sj];
    const double area = A.area.p[ci * A.area.si + cj * A.area.sj];
    double ccn;
    if (K.prog_ccn) {
      ccn = 0.0 * 1.0e6;
    } else {
      ccn = (K.ccn_l * land + K.ccn_o * (1.0 - land)) * 1.0e6;
      if (K.use_ccn) {
        const double tzb = at_level<P>(tz, L - 1);
        const double p1b = at_level<P>(p1, L - 1);
        ccn = ccn * K.RDGAS * tzb / p1b;
      }
    }
    const double c_praut = K.cpaut * pow(ccn * RHOR, -1.0 / 3.0);
    const double s_leng = sqrt(sqrt(area * 1.0e-10));
    const double t_land = K.dw_land * s_leng;
    const double t_ocean = K.dw_ocean * s_leng;
    double h_var = t_land * land + t_ocean * (1.0 - land);
    h_var = fmin(0.2, fmax(0.01, h_var));
    const double rh_adj = 1.0 - h_var - K.rh_inc;
    const double rh_rain = fmax(0.35, rh_adj - K.rh_inr);

    if (K.fix_negative) {
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const double cvm = K.c_air + qv[s] * K.c_vap + (qr[s] + ql[s]) * K.C_LIQ + (qi[s] + qs[s] + qg[s]) * K.C_ICE;
        const double lcpk = (K.lv00 + K.d0_vap * tz[s]) / cvm;
        const double icpk = (K.LI00 + K.DC_ICE * tz[s]) / cvm;
        if (qi[s] < 0.0) {
          qs[s] = qs[s] + qi[s];
          qi[s] = 0.0;
        }
        if (qs[s] < 0.0) {
          qg[s] = qg[s] + qs[s];
          qs[s] = 0.0;
        }
        if (qg[s] < 0.0) {
          qr[s] = qr[s] + qg[s];
          tz[s] = tz[s] - qg[s] * icpk;
          qg[s] = 0.0;
        }
        if (qr[s] < 0.0) {
          ql[s] = ql[s] + qr[s];
          qr[s] = 0.0;
        }
        if (ql[s] < 0.0) {
          qv[s] = qv[s] + ql[s];
          tz[s] = tz[s] - ql[s] * lcpk;
          ql[s] = 0.0;
        }
      }
      // FORWARD borrow of negative vapour from the level above (:244-247):
      // a sequential sweep, taken only when some level above the bottom is negative
      bool neg[P];
#pragma unroll
      for (int s = 0; s < P; ++s) neg[s] = valid[s] && (lane * P + s < L - 1) && (qv[s] < 0.0);
      if (col_any<P>(neg)) {
        double cq = __shfl_sync(FULLMASK, 0.0, 0), cdp = 1.0;
        const int nl = (L + P - 1) / P;
        for (int l = 0; l < nl; ++l) {
          if (lane == l) {
#pragma unroll
            for (int s = 0; s < P; ++s) {
              const int k = l * P + s;
              if (k >= 1 && k < L) {
                const double pq = (s == 0) ? cq : qv[s > 0 ? s - 1 : 0];
                const double pdp = (s == 0) ? cdp : dp1[s > 0 ? s - 1 : 0];
                if (pq < 0.0) qv[s] = qv[s] + pq * pdp / dp1[s];
              }
            }
          }
          cq = __shfl_sync(FULLMASK, qv[P - 1], l);
          cdp = __shfl_sync(FULLMASK, dp1[P - 1], l);
        }
      }
#pragma unroll
      for (int s = 0; s < P; ++s)
        if (lane * P + s < L - 1 && qv[s] < 0.0) qv[s] = 0.0;
      // bottom layer borrows from the layer above (:253-276)
      const double qb = at_level<P>(qv, L - 1), qb1 = at_level<P>(qv, L - 2);
      const double db = at_level<P>(dp1, L - 1), db1 = at_level<P>(dp1, L - 2);
      if ((qb < 0.0) && (qb1 > 0.0)) {
        const double dq = fmin(-qb * db, qb1 * db1);
#pragma unroll
        for (int s = 0; s < P; ++s) {
          const int k = lane * P + s;
          if (k == L - 2) qv[s] = qv[s] - dq / dp1[s];
          if (k == L - 1) qv[s] = qv[s] + dq / dp1[s];
        }
      }
    }

    double rain = 0.0, snow = 0.0, ice = 0.0, graupel = 0.0;

    for (int it = 0; it < K.ntimes; ++it) {
      // -------------------------------- warm_rain, is_first (:280-653)
      for (int pass = 0; pass < 2; ++pass) {
        const bool is_first = pass == 0;
        if (is_first) {
#pragma unroll
          for (int s = 0; s < P; ++s) {
            const double t0 = valid[s] ? TL(IN_PT, s) : 250.0;
            const double dz0 = valid[s] ? TL(IN_DELZ, s) : -100.0;
            const double den0 = -dp1[s] / (K.GRAV * dz0);
            dz1[s] = dz0 * tz[s] / t0;
            den[s] = den0 * dz0 / dz1[s];
            denfac[s] = sqrt(SFCRHO / den[s]);
          }
          layer_dz<P>(dz1, valid, K.zs, dz, lane, L);
        }
        const double dt5 = 0.5 * K.dt_rain;
        double m1_rain[P];
#pragma unroll
        for (int s = 0; s < P; ++s) m1_rain[s] = 0.0;
        bool pr[P];
#pragma unroll
        for (int s = 0; s < P; ++s) pr[s] = valid[s] && (qr[s] > QRMIN);
        const bool fall = col_any<P>(pr);
        double r1 = 0.0;
        if (!fall) {
#pragma unroll
          for (int s = 0; s < P; ++s) vtr[s] = VF_MIN;
        } else {
#pragma unroll
          for (int s = 0; s < P; ++s) vtr[s] = rain_fspeed(K, qr[s], den[s]);
#pragma unroll
          for (int s = 0; s < P; ++s)
            revap_racc(K, dt5, h_var, qg[s], qi[s], ql[s], qr[s], qs[s], qv[s], tz[s], den[s], denfac[s]);
          double dm[P];
          if (K.do_sedi_w) {
#pragma unroll
            for (int s = 0; s < P; ++s) dm[s] = dp1[s] * (1.0 + qv[s] + ql[s] + qr[s] + qi[s] + qs[s] + qg[s]);
          }
          r1 = implicit_fall<P>(qr, vtr, dz, dp1, valid, K.dt_rain, m1_rain, lane, L);
          if (K.do_sedi_w) w_transport<P>(w, dm, m1_rain, vtr, lane);
          if (K.do_sedi_heat) sedi_heat<P>(K, tz, dz1, dp1, qv, ql, qr, qi, qs, qg, m1_rain, valid, K.C_LIQ, lane);
#pragma unroll
          for (int s = 0; s < P; ++s)
            revap_racc(K, dt5, h_var, qg[s], qi[s], ql[s], qr[s], qs[s], qv[s], tz[s], den[s], denfac[s]);
        }
        if (K.irain_f != 0) {
#pragma unroll
          for (int s = 0; s < P; ++s) autoconv_no_subgrid_var(K, ql[s], qr[s], tz[s], den[s], ccn, c_praut);
        } else {
          double dl[P];
          if (K.z_slope_liq) {
            mono_slope<P>(ql, dl, lane, L);
#pragma unroll
            for (int s = 0; s < P; ++s) dl[s] = fmax(dl[s], fmax(QVMIN, h_var * ql[s]));
          } else {
#pragma unroll
            for (int s = 0; s < P; ++s) dl[s] = fmax(QVMIN, h_var * ql[s]);
          }
#pragma unroll
          for (int s = 0; s < P; ++s) autoconv_subgrid_var(K, ql[s], qr[s], tz[s], den[s], ccn, c_praut, dl[s]);
        }
        rain = rain + r1;
#pragma unroll
        for (int s = 0; s < P; ++s) m1[s] = is_first ? m1[s] + m1_rain[s] : m1[s] + m1_rain[s] + m1_sol[s];

        if (!is_first) break;

        // ------------------------------------ sedimentation (:657-1217)
        double vti[P];
#pragma unroll
        for (int s = 0; s < P; ++s) {
          fall_speed(K, qg[s], qi[s], qs[s], tz[s], den[s], vtg[s], vti[s], vts[s]);
          m1_sol[s] = 0.0;
        }
        // cloud ice melting at and below the first level warmer than tice (:702-746)
        int first = 1 << 30;
#pragma unroll
        for (int s = P - 1; s >= 0; --s)
          if (valid[s] && tz[s] > K.tice) first = lane * P + s;
        first = __reduce_min_sync(FULLMASK, first);
#pragma unroll
        for (int s = 0; s < P; ++s) {
          const int k = lane * P + s;
          if (!(k >= first || k == L - 1) || !valid[s]) continue;
          const double lhi = K.LI00 + K.DC_ICE * tz[s];
          double q_liq = ql[s] + qr[s];
          double q_sol = qi[s] + qs[s] + qg[s];
          double cvm = K.c_air + qv[s] * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
          const double icpk = lhi / cvm;
          const double tc = tz[s] - K.tice;
          if ((qi[s] > QCMIN) && (tc > 0.0)) {
            const double sink = fmin(qi[s], K.fac_imlt * tc / icpk);
            const double tmp = fmin(sink, dim(K.ql_mlt, ql[s]));
            ql[s] = ql[s] + tmp;
            qr[s] = qr[s] + sink - tmp;
            qi[s] = qi[s] - sink;
            q_liq = q_liq + sink;
            q_sol = q_sol - sink;
            cvm = K.c_air + qv[s] * K.c_vap + q_liq * K.C_LIQ + q_sol * K.C_ICE;
            tz[s] = tz[s] - sink * lhi / cvm;
          }
        }
        double flux[P], dm[P];
        // ice (:773-900)
        bool pi_[P];
#pragma unroll
        for (int s = 0; s < P; ++s) pi_[s] = valid[s] && (qi[s] > QRMIN);
        if ((K.vi_fac >= 1.0e-5) && col_any<P>(pi_)) {
          if (K.do_sedi_w) {
#pragma unroll
            for (int s = 0; s < P; ++s) dm[s] = dp1[s] * (1.0 + qv[s] + ql[s] + qr[s] + qi[s] + qs[s] + qg[s]);
          }
          const double i1 = implicit_fall<P>(qi, vti, dz, dp1, valid, K.dts, flux, lane, L);
#pragma unroll
          for (int s = 0; s < P; ++s) m1_sol[s] = flux[s];
          if (K.do_sedi_w) w_transport<P>(w, dm, flux, vti, lane);
          ice = ice + i1;
        }
        // snow (:902-1035)
        bool ps_[P];
#pragma unroll
        for (int s = 0; s < P; ++s) ps_[s] = valid[s] && (qs[s] > QRMIN);
        if (col_any<P>(ps_)) {
          if (K.do_sedi_w) {
#pragma unroll
            for (int s = 0; s < P; ++s) dm[s] = dp1[s] * (1.0 + qv[s] + ql[s] + qr[s] + qi[s] + qs[s] + qg[s]);
          }
          const double s1 = implicit_fall<P>(qs, vts, dz, dp1, valid, K.dts, flux, lane, L);
#pragma unroll
          for (int s = 0; s < P; ++s) m1_sol[s] = m1_sol[s] + flux[s];
          if (K.do_sedi_w) w_transport<P>(w, dm, flux, vts, lane);
          snow = snow + s1;
        }
        // graupel (:1037-1168)
        bool pg_[P];
#pragma unroll
        for (int s = 0; s < P; ++s) pg_[s] = valid[s] && (qg[s] > QRMIN);
        if (col_any<P>(pg_)) {
          if (K.do_sedi_w) {
#pragma unroll
            for (int s = 0; s < P; ++s) dm[s] = dp1[s] * (1.0 + qv[s] + ql[s] + qr[s] + qi[s] + qs[s] + qg[s]);
          }
          const double g1 = implicit_fall<P>(qg, vtg, dz, dp1, valid, K.dts, flux, lane, L);
#pragma unroll
          for (int s = 0; s < P; ++s) m1_sol[s] = m1_sol[s] + flux[s];
          if (K.do_sedi_w) w_transport<P>(w, dm, flux, vtg, lane);
          graupel = graupel + g1;
        }
        rain = rain + 0.0;
        if (K.do_sedi_heat) sedi_heat<P>(K, tz, dz1, dp1, qv, ql, qr, qi, qs, qg, m1_sol, valid, K.C_ICE, lane);
      }

      // ------------------------------------------------ icloud (:1220-1449)
      double q_liq[P], q_sol[P], cvm[P];
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const double lhi = K.LI00 + K.DC_ICE * tz[s];
        q_liq[s] = ql[s] + qr[s];
        q_sol[s] = qi[s] + qs[s] + qg[s];
        cvm[s] = K.c_air + qv[s] * K.c_vap + q_liq[s] * K.C_LIQ + q_sol[s] * K.C_ICE;
        const double icpk = lhi / cvm[s];
        if ((tz[s] > K.tice) && (qi[s] > QCMIN)) {
          const double melt = fmin(qi[s], K.fac_imlt * (tz[s] - K.tice) / icpk);
          const double tmp = fmin(melt, dim(K.ql_mlt, ql[s]));
          ql[s] = ql[s] + tmp;
          qr[s] = qr[s] + melt - tmp;
          qi[s] = qi[s] - melt;
          q_liq[s] = q_liq[s] + melt;
          q_sol[s] = q_sol[s] - melt;
          cvm[s] = K.c_air + qv[s] * K.c_vap + q_liq[s] * K.C_LIQ + q_sol[s] * K.C_ICE;
          tz[s] = tz[s] - melt * lhi / cvm[s];
        } else if ((tz[s] < K.t_wfr) && (ql[s] > QCMIN)) {
          const double dtmp = K.t_wfr - tz[s];
          const double factor = fmin(1.0, dtmp / DT_FR);
          const double sink = fmin(ql[s] * factor, dtmp / icpk);
          const double qi_crt = K.qi_gen * fmin(K.qi_lim, 0.1 * (K.tice - tz[s])) / den[s];
          const double tmp = fmin(sink, dim(qi_crt, qi[s]));
          ql[s] = ql[s] - sink;
          qs[s] = qs[s] + sink - tmp;
          qi[s] = qi[s] + tmp;
          q_liq[s] = q_liq[s] - sink;
          q_sol[s] = q_sol[s] + sink;
          cvm[s] = K.c_air + qv[s] * K.c_vap + q_liq[s] * K.C_LIQ + q_sol[s] * K.C_ICE;
          tz[s] = tz[s] + sink * lhi / cvm[s];
        }
      }
      double di[P];
      if (K.z_slope_ice) {
        mono_slope<P>(qi, di, lane, L);
#pragma unroll
        for (int s = 0; s < P; ++s) di[s] = fmax(di[s], fmax(QVMIN, h_var * qi[s]));
      } else {
#pragma unroll
        for (int s = 0; s < P; ++s) di[s] = fmax(QVMIN, h_var * qi[s]);
      }
#pragma unroll
      for (int s = 0; s < P; ++s) {
        if (!valid[s]) continue;
        icloud_processes(K, qg[s], qi[s], ql[s], qr[s], qs[s], qv[s], tz[s], den[s], denfac[s], vtg[s], vtr[s],
                         vts[s], p1[s], di[s], q_liq[s], q_sol[s], cvm[s]);
        subgrid_z_proc(K, h_var, rh_adj, rh_rain, qa[s], qg[s], qi[s], ql[s], qr[s], qs[s], qv[s], tz[s], den[s],
                       denfac[s], p1[s]);
      }
    }

    // ------------------------------------------------ fields_update (:1452-1553)
    double u1[P], v1[P];
    if (K.sedi_transport) {
      double mp[P], au[P], av[P], b[P];
      prev_vals<P>(m1, mp);
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const int k = lane * P + s;
        const double dp0 = valid[s] ? TL(IN_DELP, s) : 1.0;
        const double u0 = valid[s] ? TL(IN_UA, s) : 0.0;
        const double v0 = valid[s] ? TL(IN_VA, s) : 0.0;
        if (k == 0) {
          au[s] = u0;
          av[s] = v0;
          b[s] = 0.0;
        } else {
          const double D = dp0 + mp[s];
          au[s] = dp0 * u0 / D;
          av[s] = dp0 * v0 / D;
          b[s] = mp[s] / D;
        }
        if (!valid[s]) {
          au[s] = 0.0;
          av[s] = 0.0;
          b[s] = 0.0;
        }
      }
      scan_affine<P>(au, b, lane);
      scan_affine<P>(av, b, lane);
#pragma unroll
      for (int s = 0; s < P; ++s) {
        u1[s] = au[s];
        v1[s] = av[s];
      }
    }
    double inc[N_OUT][P];
    const double rdt = K.rdt;
#pragma unroll
    for (int s = 0; s < P; ++s) {
      if (!valid[s]) {
#pragma unroll
        for (int o = 0; o < N_OUT; ++o) inc[o][s] = 0.0;
        continue;
      }
      const double delp = TL(IN_DELP, s);
      const double omq0 = delp / dp1[s];
      const double qv0 = TL(IN_QV, s) * omq0, ql0 = TL(IN_QL, s) * omq0, qr0 = TL(IN_QR, s) * omq0;
      const double qi0 = TL(IN_QI, s) * omq0, qs0 = TL(IN_QS, s) * omq0, qg0 = TL(IN_QG, s) * omq0;
      const double t0 = TL(IN_PT, s), qa0 = TL(IN_QA, s);
      const double u0 = TL(IN_UA, s), v0 = TL(IN_VA, s);
      const double omq = dp1[s] / delp;
      inc[OUT_QV_DT][s] = rdt * (qv[s] - qv0) * omq;
      inc[OUT_QL_DT][s] = rdt * (ql[s] - ql0) * omq;
      inc[OUT_QR_DT][s] = rdt * (qr[s] - qr0) * omq;
      inc[OUT_QI_DT][s] = rdt * (qi[s] - qi0) * omq;
      inc[OUT_QS_DT][s] = rdt * (qs[s] - qs0) * omq;
      inc[OUT_QG_DT][s] = rdt * (qg[s] - qg0) * omq;
      const double cvm = K.c_air + qv[s] * K.c_vap + (qr[s] + ql[s]) * K.C_LIQ + (qi[s] + qs[s] + qg[s]) * K.C_ICE;
      inc[OUT_PT_DT][s] = rdt * (tz[s] - t0) * cvm / K.CP_AIR;
      inc[OUT_QA_DT][s] = K.do_qa ? 0.0 : rdt * (qa[s] / (double)K.ntimes - qa0);
      inc[OUT_UDT][s] = K.sedi_transport ? (u1[s] - u0) * rdt : 0.0;
      inc[OUT_VDT][s] = K.sedi_transport ? (v1[s] - v0) * rdt : 0.0;
      inc[OUT_W][s] = w[s];
      inc[OUT_QAZ][s] = qa[s];
    }
#pragma unroll
    for (int s = 0; s < P; ++s)
#pragma unroll
      for (int o = 0; o < N_OUT; ++o) TL(o, s) = inc[o][s];

    if (lane == 0) {
      const double convt = 86400.0 * rdt * K.RGRAV;
      if (A.rain) A.rain[col] = rain * convt;
      if (A.snow) A.snow[col] = snow * convt;
      if (A.ice) A.ice[col] = ice * convt;
      if (A.graupel) A.graupel[col] = graupel * convt;
    }
  }
  __syncthreads();
  stage_out<P, CPB>(A, sm, c0);
}

// de_ice (microphysics.py:110-120): applied in place before the step.
__global__ void de_ice_kernel(const __grid_constant__ MpArgs A, Fld3 qi_dt, Fld3 qs_dt) {
  const MpConst& K = A.K;
  const int64_t n = A.ncol * (int64_t)A.nz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e % A.ncol, k = e / A.ncol;
    const int64_t i = c % A.nx, j = c / A.nx;
    double* qi = A.in[IN_QI].p + i * A.in[IN_QI].si + j * A.in[IN_QI].sj + k * A.in[IN_QI].sk;
    double* qs = A.in[IN_QS].p + i * A.in[IN_QS].si + j * A.in[IN_QS].sj + k * A.in[IN_QS].sk;
    double* pqi = qi_dt.p + i * qi_dt.si + j * qi_dt.sj + k * qi_dt.sk;
    double* pqs = qs_dt.p + i * qs_dt.si + j * qs_dt.sj + k * qs_dt.sk;
    const double qio = *qi - K.timestep * *pqi;
    const double qin = fmax(qio, K.qi0_max);
    if (*qi > qin) {
      *qs = *qs + *qi - qin;
      *qi = qin;
      const double dqi = (qin - qio) * K.rdt;
      *pqs = *pqs + *pqi - dqi;
      *pqi = dqi;
    }
  }
}

}  // namespace shield
