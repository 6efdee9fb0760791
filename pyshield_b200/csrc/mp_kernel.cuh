// The fused GFDL microphysics step: one thread per model level, one group of
// NW warps per column.
//
// Restates Microphysics.__call__ (pySHiELD/stencils/microphysics.py:1981-2263):
// fields_init, ntimes x [warm_rain(first), sedimentation, warm_rain, icloud],
// fields_update, all inside one launch.
//
// Layout of the work:
//  * a block owns G consecutive columns; column g of the block is served by
//    NW = ceil(L / 32) warps, and thread (warp w, lane l) of that group holds
//    level k = 32 w + l (k = 0 is the model top). A warp therefore covers 32
//    adjacent levels, whose physics takes similar branches, and each thread
//    keeps one level's state in registers for the whole step;
//  * the 14 input fields (13 state fields + the persistent cloud-fraction
//    accumulator) are staged once through shared memory with coalesced loads
//    (consecutive threads read consecutive columns of an i-fastest field, or
//    consecutive levels of a k-fastest one); the same tiles carry the outputs
//    back, so HBM traffic is the algorithmic bytes;
//  * vertical operations are warp shuffles plus a carry between the group's
//    warps through shared memory, synchronised by the group's own named
//    barrier: the column any() flags (bar.red.or), the implicit
//    sedimentation, heating and momentum recurrences (first-order linear in
//    the level above, as warp scans of affine maps), the height sweep (a
//    suffix sum) and neighbour reads.
#pragma once

#include "mp_physics.cuh"
#include "mp_physics_mixed.cuh"

namespace shield {

#define FULLMASK 0xffffffffu

template <int NW>
struct Tiles {
  static constexpr int RP = 32 * NW + 1;  // doubles per (field, column) row; odd pitch
  static constexpr int SCR = 8 * NW + 8;  // per-column scratch doubles per parity
};

// Vertical operations of one column group. Every thread of the group calls
// the same sequence of operations (group-uniform control flow); each
// operation uses the next of two alternating scratch slots, so one named
// barrier per operation suffices.
template <int NW>
struct Column {
  static constexpr int WP = Tiles<NW>::RP;  // pitch of the work rows
  int w, lane, k, L, bar;
  double* scr;   // 2 * SCR doubles
  double* work;  // 2 * RP doubles, for the sequential vapour borrow
  int par;

  SHD void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(32 * NW) : "memory"); }
  SHD double* slot() {
    double* s = scr + par * Tiles<NW>::SCR;
    par ^= 1;
    return s;
  }
  // value at level k - 1 (undefined at k = 0)
  SHD double prev(double x) {
    double u = __shfl_up_sync(FULLMASK, x, 1);
    if (NW == 1) return u;
    double* s = slot();
    if (lane == 31) s[w] = x;
    sync();
    if (lane == 0 && w > 0) u = s[w - 1];
    return u;
  }
  SHD void prev2(double x, double y, double& px, double& py) {
    px = __shfl_up_sync(FULLMASK, x, 1);
    py = __shfl_up_sync(FULLMASK, y, 1);
    if (NW == 1) return;
    double* s = slot();
    if (lane == 31) {
      s[2 * w] = x;
      s[2 * w + 1] = y;
    }
    sync();
    if (lane == 0 && w > 0) {
      px = s[2 * w - 2];
      py = s[2 * w - 1];
    }
  }
  // value at level k + 1 (undefined at k = 32 NW - 1)
  SHD double next(double x) {
    double d = __shfl_down_sync(FULLMASK, x, 1);
    if (NW == 1) return d;
    double* s = slot();
    if (lane == 0) s[w] = x;
    sync();
    if (lane == 31 && w < NW - 1) d = s[w + 1];
    return d;
  }
  SHD bool any(bool p) {
    if (NW == 1) return __any_sync(FULLMASK, p);
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred q, %2, %3, q;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((unsigned)p), "r"(bar), "r"(32 * NW)
        : "memory");
    return r != 0;
  }
  // any() over every thread that shares this object's barrier: the whole
  // column here (control flow around vertical operations must be uniform
  // over the barrier's threads)
  SHD bool group_any(bool p) { return any(p); }
  // any() with the group's any() from the same exchange (one column here)
  SHD bool any_group(bool p, bool& g) {
    g = any(p);
    return g;
  }
  SHD void any3_group(bool a, bool b, bool c, bool& ra, bool& rb, bool& rc, bool& ga, bool& gb, bool& gc) {
    any3(a, b, c, ra, rb, rc);
    ga = ra;
    gb = rb;
    gc = rc;
  }
  SHD int min_int(int v) {
    v = __reduce_min_sync(FULLMASK, v);
    if (NW == 1) return v;
    double* s = slot();
    int* si = reinterpret_cast<int*>(s);
    if (lane == 0) si[w] = v;
    sync();
    int m = si[0];
#pragma unroll
    for (int u = 1; u < NW; ++u) m = min(m, si[u]);
    return m;
  }
  // values of x and y at level k0 (every level receives them)
  SHD void bcast2(double x, double y, int k0, double& x0, double& y0) {
    const int w0 = k0 >> 5, l0 = k0 & 31;
    x0 = __shfl_sync(FULLMASK, x, l0);
    y0 = __shfl_sync(FULLMASK, y, l0);
    if (NW == 1) return;
    double* s = slot();
    if (w == w0 && lane == 0) {
      s[0] = x0;
      s[1] = y0;
    }
    sync();
    x0 = s[0];
    y0 = s[1];
  }
  SHD double bcast(double x, int k0) {
    double x0, y0;
    bcast2(x, x, k0, x0, y0);
    return x0;
  }
  // X_k = a_k + b_k X_{k-1} from the top down (b must vanish at k = 0)
  SHD double scan_affine(double a, double b) {
    double A = a, B = b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      double pA = __shfl_up_sync(FULLMASK, A, d);
      double pB = __shfl_up_sync(FULLMASK, B, d);
      if (lane >= d) {
        A = A + B * pA;
        B = B * pB;
      }
    }
    if (NW == 1) return A;
    double* s = slot();
    if (lane == 31) {
      s[2 * w] = A;
      s[2 * w + 1] = B;
    }
    sync();
    double X = 0.0;
    for (int u = 0; u < w; ++u) X = s[2 * u] + s[2 * u + 1] * X;
    return A + B * X;
  }
  // two independent scans sharing one barrier
  SHD void scan_affine2(double a1, double b1, double a2, double b2, double& x1, double& x2) {
    double A1 = a1, B1 = b1, A2 = a2, B2 = b2;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      double pA1 = __shfl_up_sync(FULLMASK, A1, d), pB1 = __shfl_up_sync(FULLMASK, B1, d);
      double pA2 = __shfl_up_sync(FULLMASK, A2, d), pB2 = __shfl_up_sync(FULLMASK, B2, d);
      if (lane >= d) {
        A1 = A1 + B1 * pA1;
        B1 = B1 * pB1;
        A2 = A2 + B2 * pA2;
        B2 = B2 * pB2;
      }
    }
    if (NW == 1) {
      x1 = A1;
      x2 = A2;
      return;
    }
    double* s = slot();
    if (lane == 31) {
      s[4 * w] = A1;
      s[4 * w + 1] = B1;
      s[4 * w + 2] = A2;
      s[4 * w + 3] = B2;
    }
    sync();
    double X1 = 0.0, X2 = 0.0;
    for (int u = 0; u < w; ++u) {
      X1 = s[4 * u] + s[4 * u + 1] * X1;
      X2 = s[4 * u + 2] + s[4 * u + 3] * X2;
    }
    x1 = A1 + B1 * X1;
    x2 = A2 + B2 * X2;
  }
  // values at levels k - 1 of N fields with one barrier (undefined at k = 0)
  template <int N>
  SHD void prevN(const double (&x)[N], double (&px)[N]) {
#pragma unroll
    for (int n = 0; n < N; ++n) px[n] = __shfl_up_sync(FULLMASK, x[n], 1);
    if (NW == 1) return;
    double* s = slot();
    if (lane == 31) {
#pragma unroll
      for (int n = 0; n < N; ++n) s[N * w + n] = x[n];
    }
    sync();
    if (lane == 0 && w > 0) {
#pragma unroll
      for (int n = 0; n < N; ++n) px[n] = s[N * (w - 1) + n];
    }
  }
  // values at levels k - 1 and k + 1 with one barrier
  SHD void nbrs(double x, double& xp, double& xn) {
    xp = __shfl_up_sync(FULLMASK, x, 1);
    xn = __shfl_down_sync(FULLMASK, x, 1);
    if (NW == 1) return;
    double* s = slot();
    if (lane == 0) s[2 * w] = x;
    if (lane == 31) s[2 * w + 1] = x;
    sync();
    if (lane == 0 && w > 0) xp = s[2 * w - 1];
    if (lane == 31 && w < NW - 1) xn = s[2 * w + 2];
  }
  // three column any() flags with one barrier
  SHD void any3(bool a, bool b, bool c, bool& ra, bool& rb, bool& rc) {
    const unsigned m = (__any_sync(FULLMASK, a) ? 1u : 0u) | (__any_sync(FULLMASK, b) ? 2u : 0u) |
                       (__any_sync(FULLMASK, c) ? 4u : 0u);
    unsigned r = m;
    if (NW > 1) {
      double* s = slot();
      unsigned* su = reinterpret_cast<unsigned*>(s);
      if (lane == 0) su[w] = m;
      sync();
      r = 0;
#pragma unroll
      for (int u = 0; u < NW; ++u) r |= su[u];
    }
    ra = (r & 1u) != 0;
    rb = (r & 2u) != 0;
    rc = (r & 4u) != 0;
  }
  // N independent top-down affine scans with one barrier
  template <int N>
  SHD void scanN(const double (&a)[N], const double (&b)[N], double (&x)[N]) {
    double A[N], B[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
      A[n] = a[n];
      B[n] = b[n];
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
      for (int n = 0; n < N; ++n) {
        const double pA = __shfl_up_sync(FULLMASK, A[n], d);
        const double pB = __shfl_up_sync(FULLMASK, B[n], d);
        if (lane >= d) {
          A[n] = A[n] + B[n] * pA;
          B[n] = B[n] * pB;
        }
      }
    }
    if (NW == 1) {
#pragma unroll
      for (int n = 0; n < N; ++n) x[n] = A[n];
      return;
    }
    double* s = slot();
    if (lane == 31) {
#pragma unroll
      for (int n = 0; n < N; ++n) {
        s[2 * N * w + 2 * n] = A[n];
        s[2 * N * w + 2 * n + 1] = B[n];
      }
    }
    sync();
#pragma unroll
    for (int n = 0; n < N; ++n) {
      double X = 0.0;
      for (int u = 0; u < w; ++u) X = s[2 * N * u + 2 * n] + s[2 * N * u + 2 * n + 1] * X;
      x[n] = A[n] + B[n] * X;
    }
  }
  // values of N fields at level k0 with one barrier
  template <int N>
  SHD void bcastN(const double (&x)[N], int k0, double (&x0)[N]) {
    const int w0 = k0 >> 5, l0 = k0 & 31;
#pragma unroll
    for (int n = 0; n < N; ++n) x0[n] = __shfl_sync(FULLMASK, x[n], l0);
    if (NW == 1) return;
    double* s = slot();
    if (w == w0 && lane == 0) {
#pragma unroll
      for (int n = 0; n < N; ++n) s[n] = x0[n];
    }
    sync();
#pragma unroll
    for (int n = 0; n < N; ++n) x0[n] = s[n];
  }
  // layer thickness from the BACKWARD height sweep with one barrier:
  // ze_k = zs + sum_{j >= k} (-dz1_j); dz_k = ze_k - ze_{k+1}, dz_{L-1} = ze_{L-1} - zs
  SHD double heights(double t, double zs) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      double v = __shfl_down_sync(FULLMASK, t, d);
      if (lane + d < 32) t = t + v;
    }
    double zn_in_warp = __shfl_down_sync(FULLMASK, t, 1);  // suffix at k + 1 within the warp
    double c = 0.0, cn = 0.0;
    if (NW > 1) {
      double* s = slot();
      if (lane == 0) s[w] = t;
      sync();
      for (int u = NW - 1; u > w; --u) c = c + s[u];
      // for lane 31 the level below is lane 0 of warp w + 1: its suffix is
      // s[w + 1] plus the carry from the warps below it
      if (lane == 31 && w < NW - 1) {
        for (int u = NW - 1; u > w + 1; --u) cn = cn + s[u];
        zn_in_warp = s[w + 1];
      }
    }
    const double ze = zs + (t + c);
    double zn;
    if (lane == 31)
      zn = zs + (zn_in_warp + cn);
    else
      zn = zs + (zn_in_warp + c);
    return (k == L - 1) ? ze - zs : ze - zn;
  }
  // ---------------------------------------------- exchanges of the adjoint
  // values at level k + 1 of N fields with one barrier (undefined at the
  // last level of the group)
  template <int N>
  SHD void nextN(const double (&x)[N], double (&xn)[N]) {
#pragma unroll
    for (int n = 0; n < N; ++n) xn[n] = __shfl_down_sync(FULLMASK, x[n], 1);
    if (NW == 1) return;
    double* s = slot();
    if (lane == 0) {
#pragma unroll
      for (int n = 0; n < N; ++n) s[N * w + n] = x[n];
    }
    sync();
    if (lane == 31 && w < NW - 1) {
#pragma unroll
      for (int n = 0; n < N; ++n) xn[n] = s[N * (w + 1) + n];
    }
  }
  // x at level k - 1 and y at level k + 1 with one barrier
  SHD void prev_next(double x, double y, double& xp, double& yn) {
    xp = __shfl_up_sync(FULLMASK, x, 1);
    yn = __shfl_down_sync(FULLMASK, y, 1);
    if (NW == 1) return;
    double* s = slot();
    if (lane == 31) s[2 * w] = x;
    if (lane == 0) s[2 * w + 1] = y;
    sync();
    if (lane == 0 && w > 0) xp = s[2 * (w - 1)];
    if (lane == 31 && w < NW - 1) yn = s[2 * (w + 1) + 1];
  }
  // N independent bottom-up affine scans X_k = a_k + c_k X_{k+1} with one
  // barrier (c must vanish at the last level); the adjoints of the
  // top-down recurrences
  template <int N>
  SHD void scanN_rev(const double (&a)[N], const double (&c)[N], double (&x)[N]) {
    double A[N], B[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
      A[n] = a[n];
      B[n] = c[n];
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
      for (int n = 0; n < N; ++n) {
        const double pA = __shfl_down_sync(FULLMASK, A[n], d);
        const double pB = __shfl_down_sync(FULLMASK, B[n], d);
        if (lane + d < 32) {
          A[n] = A[n] + B[n] * pA;
          B[n] = B[n] * pB;
        }
      }
    }
    if (NW == 1) {
#pragma unroll
      for (int n = 0; n < N; ++n) x[n] = A[n];
      return;
    }
    double* s = slot();
    if (lane == 0) {
#pragma unroll
      for (int n = 0; n < N; ++n) {
        s[2 * N * w + 2 * n] = A[n];
        s[2 * N * w + 2 * n + 1] = B[n];
      }
    }
    sync();
#pragma unroll
    for (int n = 0; n < N; ++n) {
      double X = 0.0;
      for (int u = NW - 1; u > w; --u) X = s[2 * N * u + 2 * n] + s[2 * N * u + 2 * n + 1] * X;
      x[n] = A[n] + B[n] * X;
    }
  }
  SHD double scan_affine_rev(double a, double c) {
    const double aa[1] = {a}, cc[1] = {c};
    double xx[1];
    scanN_rev<1>(aa, cc, xx);
    return xx[0];
  }
  // sum over the column's levels (every level receives it), in a fixed order
  SHD double colsum(double x) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) x = x + __shfl_xor_sync(FULLMASK, x, d);
    if (NW == 1) return x;
    double* s = slot();
    if (lane == 0) s[w] = x;
    sync();
    double t = s[0];
    for (int u = 1; u < NW; ++u) t = t + s[u];
    return t;
  }
  // inclusive sum from the bottom: sum over levels j >= k
  SHD double suffix_sum(double t) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      double v = __shfl_down_sync(FULLMASK, t, d);
      if (lane + d < 32) t = t + v;
    }
    if (NW == 1) return t;
    double* s = slot();
    if (lane == 0) s[w] = t;
    sync();
    double c = 0.0;
    for (int u = NW - 1; u > w; --u) c = c + s[u];
    return t + c;
  }
};

// P columns of L levels packed one after another on the 32 NWG threads of
// a group, which share one named barrier: thread t of the group holds level
// k = t - c L of column c = t / L; the threads from P L on form an idle tail
// (column slot P). With L = 79, two columns fill 5 warps (158 of 160
// threads) where one column per 3 warps leaves 17 of 96 threads idle.
//
// Every vertical operation is segmented by column: a value never enters
// arithmetic with another column's (the warp scans combine lanes of one
// column only, the carries between warps come from that column's warps, the
// any/min reductions and broadcasts keep a slot per column). A column spans
// whole warps except at its ends, so a warp holds parts of at most two
// segments (L > 32): the one holding its lane 0 (head) and the one holding
// its lane 31 (tail). Control flow around a vertical operation must be
// uniform over the whole group (group_any), not only over a column.
template <int NWG, int P>
struct PackedColumn {
  static constexpr int T = 32 * NWG;   // threads of the group
  static constexpr int LMAX = T / P;   // longest column that fits
  static constexpr int WP = LMAX + 1;  // pitch of the work rows
  static constexpr int SCR = 8 * NWG + 8 + 4 * (P + 1);  // scratch doubles per parity
  // t: thread of the group; c: its column slot (P for the idle tail); k:
  // its level. The segment's extent is derived from these when needed,
  // which keeps the per-thread state small.
  int t, c, k, L, bar;
  double* scr;   // 2 * SCR doubles
  double* work;  // this column's two work rows (WP doubles each)
  int par;

  // scr_grp / work_grp: the group's scratch and its (P + 1) x 2 work rows
  SHD void init(int t_, int L_, int bar_, double* scr_grp, double* work_grp) {
    t = t_;
    L = L_;
    bar = bar_;
    c = t / L;
    if (c > P) c = P;
    k = t - c * L;
    scr = scr_grp;
    work = work_grp + (size_t)c * 2 * WP;
    par = 0;
  }
  SHD int w() const { return t >> 5; }
  SHD int lane() const { return t & 31; }
  SHD int seg0() const { return t - k; }
  SHD int seglen() const { return (c < P) ? L : T - P * L; }
  SHD int wfirst() const { return seg0() >> 5; }
  SHD int wlast() const { return (seg0() + seglen() - 1) >> 5; }
  // the slot, in a per-warp pair of partials, that holds this segment's
  // part of warp u (the head partial unless the segment starts inside u)
  SHD int part(int u) const { return 2 * u + ((u == wfirst() && (seg0() & 31) != 0) ? 1 : 0); }
  // lanes of this warp in this segment
  SHD unsigned segmask() const {
    const int w_ = w();
    const int lo = max(seg0() - 32 * w_, 0), hi = min(seg0() + seglen() - 32 * w_, 32);
    const unsigned up = (hi >= 32) ? FULLMASK : ((1u << hi) - 1u);
    return up & ~((1u << lo) - 1u);
  }
  // this lane is the last of its segment within its warp
  SHD bool seg_last_in_warp() const { return lane() == 31 || k == seglen() - 1; }
  // this lane's segment is the one holding lane 0 of the warp
  SHD bool in_head() const { return seg0() <= 32 * w(); }

  SHD void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(T) : "memory"); }
  SHD double* slot() {
    double* s = scr + par * SCR;
    par ^= 1;
    return s;
  }
  SHD bool group_any(bool p) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred q, %2, %3, q;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((unsigned)p), "r"(bar), "r"(T)
        : "memory");
    return r != 0;
  }
  // ------------------------------------------------ neighbour exchanges
  // (values of another column, read at a column's ends, are not used by
  // the callers, which select the boundary value at k = 0 / k = L - 1)
  SHD double prev(double x) {
    double u = __shfl_up_sync(FULLMASK, x, 1);
    double* s = slot();
    if (lane() == 31) s[w()] = x;
    sync();
    if (lane() == 0 && w() > 0) u = s[w() - 1];
    return u;
  }
  template <int N>
  SHD void prevN(const double (&x)[N], double (&px)[N]) {
#pragma unroll
    for (int n = 0; n < N; ++n) px[n] = __shfl_up_sync(FULLMASK, x[n], 1);
    double* s = slot();
    if (lane() == 31) {
#pragma unroll
      for (int n = 0; n < N; ++n) s[N * w() + n] = x[n];
    }
    sync();
    if (lane() == 0 && w() > 0) {
#pragma unroll
      for (int n = 0; n < N; ++n) px[n] = s[N * (w() - 1) + n];
    }
  }
  SHD void nbrs(double x, double& xp, double& xn) {
    xp = __shfl_up_sync(FULLMASK, x, 1);
    xn = __shfl_down_sync(FULLMASK, x, 1);
    double* s = slot();
    if (lane() == 0) s[2 * w()] = x;
    if (lane() == 31) s[2 * w() + 1] = x;
    sync();
    if (lane() == 0 && w() > 0) xp = s[2 * w() - 1];
    if (lane() == 31 && w() < NWG - 1) xn = s[2 * w() + 2];
  }
  // ------------------------------------------------ column reductions
  SHD bool any(bool p) {
    unsigned m[1] = {p ? 1u : 0u};
    anyN<1>(m);
    return m[0] != 0;
  }
  SHD void any3(bool a, bool b, bool c3, bool& ra, bool& rb, bool& rc) {
    unsigned m[3] = {a ? 1u : 0u, b ? 1u : 0u, c3 ? 1u : 0u};
    anyN<3>(m);
    ra = m[0] != 0;
    rb = m[1] != 0;
    rc = m[2] != 0;
  }
  // the column's any() and, from the same exchange, the group's (every
  // warp's parts ORed)
  SHD bool any_group(bool p, bool& g) {
    unsigned m[1] = {p ? 1u : 0u}, gm = 0;
    anyN<1>(m, &gm);
    g = gm != 0;
    return m[0] != 0;
  }
  SHD void any3_group(bool a, bool b, bool c3, bool& ra, bool& rb, bool& rc, bool& ga, bool& gb, bool& gc) {
    unsigned m[3] = {a ? 1u : 0u, b ? 1u : 0u, c3 ? 1u : 0u}, gm = 0;
    anyN<3>(m, &gm);
    ra = m[0] != 0;
    rb = m[1] != 0;
    rc = m[2] != 0;
    ga = (gm & 1u) != 0;
    gb = (gm & 2u) != 0;
    gc = (gm & 4u) != 0;
  }
  template <int N>
  SHD void anyN(unsigned (&m)[N], unsigned* group = nullptr) {
    const unsigned sm_ = segmask();
    unsigned bits = 0;
#pragma unroll
    for (int n = 0; n < N; ++n) bits |= ((__ballot_sync(FULLMASK, m[n] != 0) & sm_) != 0u ? 1u : 0u) << n;
    unsigned* s = reinterpret_cast<unsigned*>(slot());
    if (lane() == 0) s[2 * w()] = bits;
    if (lane() == 31) s[2 * w() + 1] = bits;
    sync();
    unsigned r = 0;
    for (int u = wfirst(); u <= wlast(); ++u) r |= s[part(u)];
    if (group) {
      unsigned gr = 0;
#pragma unroll
      for (int u = 0; u < NWG; ++u) gr |= s[2 * u] | s[2 * u + 1];
      *group = gr;
    }
#pragma unroll
    for (int n = 0; n < N; ++n) m[n] = (r >> n) & 1u;
  }
  SHD int min_int(int v) {
    // segmented inclusive min-scan down the warp, then the per-warp parts
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(FULLMASK, v, d);
      if (lane() >= d && k >= d) v = min(v, o);
    }
    int* s = reinterpret_cast<int*>(slot());
    if (lane() == 31) s[2 * w() + 1] = v;
    if (in_head() && seg_last_in_warp()) s[2 * w()] = v;
    sync();
    int m = s[part(wfirst())];
    for (int u = wfirst() + 1; u <= wlast(); ++u) m = min(m, s[part(u)]);
    return m;
  }
  // values of N fields at level k0 of this column (the idle tail reads the
  // last column's)
  template <int N>
  SHD void bcastN(const double (&x)[N], int k0, double (&x0)[N]) {
    double* s = slot();
    if (k == k0 && c < P) {
#pragma unroll
      for (int n = 0; n < N; ++n) s[N * c + n] = x[n];
    }
    sync();
    const int cc = c < P ? c : P - 1;
#pragma unroll
    for (int n = 0; n < N; ++n) x0[n] = s[N * cc + n];
  }
  SHD void bcast2(double x, double y, int k0, double& x0, double& y0) {
    const double v[2] = {x, y};
    double r[2];
    bcastN<2>(v, k0, r);
    x0 = r[0];
    y0 = r[1];
  }
  SHD double bcast(double x, int k0) {
    const double v[1] = {x};
    double r[1];
    bcastN<1>(v, k0, r);
    return r[0];
  }
  // ------------------------------------------------ recurrences
  // N independent top-down affine scans X_k = a_k + b_k X_{k-1} (b must
  // vanish at k = 0)
  template <int N>
  SHD void scanN(const double (&a)[N], const double (&b)[N], double (&x)[N]) {
    double A[N], B[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
      A[n] = a[n];
      B[n] = b[n];
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
      for (int n = 0; n < N; ++n) {
        const double pA = __shfl_up_sync(FULLMASK, A[n], d);
        const double pB = __shfl_up_sync(FULLMASK, B[n], d);
        if (lane() >= d && k >= d) {
          A[n] = A[n] + B[n] * pA;
          B[n] = B[n] * pB;
        }
      }
    }
    double* s = slot();
    if (lane() == 31) {
#pragma unroll
      for (int n = 0; n < N; ++n) {
        s[2 * N * w() + 2 * n] = A[n];
        s[2 * N * w() + 2 * n + 1] = B[n];
      }
    }
    sync();
    // the carry from this column's earlier warps (lane 31 of each is in it)
#pragma unroll
    for (int n = 0; n < N; ++n) {
      double X = 0.0;
      for (int u = wfirst(); u < w(); ++u) X = s[2 * N * u + 2 * n] + s[2 * N * u + 2 * n + 1] * X;
      x[n] = (w() > wfirst()) ? A[n] + B[n] * X : A[n];
    }
  }
  SHD double scan_affine(double a, double b) {
    const double aa[1] = {a}, bb[1] = {b};
    double xx[1];
    scanN<1>(aa, bb, xx);
    return xx[0];
  }
  SHD void scan_affine2(double a1, double b1, double a2, double b2, double& x1, double& x2) {
    const double aa[2] = {a1, a2}, bb[2] = {b1, b2};
    double xx[2];
    scanN<2>(aa, bb, xx);
    x1 = xx[0];
    x2 = xx[1];
  }
  // layer thickness from the BACKWARD height sweep:
  // ze_k = zs + sum_{j >= k} (-dz1_j); dz_k = ze_k - ze_{k+1}, dz_{L-1} = ze_{L-1} - zs
  SHD double heights(double x, double zs) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const double v = __shfl_down_sync(FULLMASK, x, d);
      if (lane() + d < 32 && k + d < seglen()) x = x + v;
    }
    double zn_in_warp = __shfl_down_sync(FULLMASK, x, 1);  // suffix at k + 1 within the warp
    double* s = slot();
    // lane 0 of each of this column's later warps holds that warp's part
    if (lane() == 0) s[w()] = x;
    sync();
    double cc = 0.0, cn = 0.0;
    for (int u = wlast(); u > w(); --u) cc = cc + s[u];
    if (lane() == 31 && w() < wlast()) {
      for (int u = wlast(); u > w() + 1; --u) cn = cn + s[u];
      zn_in_warp = s[w() + 1];
    }
    const double ze = zs + (x + cc);
    const double zn = (lane() == 31) ? zs + (zn_in_warp + cn) : zs + (zn_in_warp + cc);
    return (k == L - 1) ? ze - zs : ze - zn;
  }
};

// Implicit upwind fall of one species (use_ppm = False): q is the dry mixing
// ratio (updated), dtf the fall time step; returns the cumulative mass flux
// m1 at this level (microphysics.py:454-507 and the ice/snow/graupel repeats).
//
// The reference accumulates m1_k = (m1_{k-1} + q_k) - qm_k level by level.
// With r_k the density from the implicit recurrence, r_k (dz_k + dd_k) =
// q_k + dd_{k-1} r_{k-1}, that running sum telescopes to m1_k = dd_k r_k:
// the mass leaving the bottom of level k. The telescoped form is used here.
// It equals the running sum in exact arithmetic, but it does not cancel: the
// running sum loses all its digits when little mass reaches the ground.
template <class Col>
SHD double implicit_fall(Col& C, double& q, double vt, double dz, double dp1, bool valid, double dtf) {
  const double dd = dtf * vt;
  const double qmass = valid ? q * dp1 : 0.0;
  const double ddp = C.prev(dd);
  const double D = dz + dd;
  double a = qmass / D;
  double b = (C.k == 0) ? 0.0 : ddp / D;
  if (!valid) {
    a = 0.0;
    b = 0.0;
  }
  const double r = C.scan_affine(a, b);
  if (valid) q = r * dz / dp1;
  return valid ? dd * r : 0.0;
}

// Implicit heating by falling condensate (microphysics.py:516-557 with
// C_LIQ, :1176-1217 with C_ICE); fp is the flux at the level above.
template <class Col>
SHD void sedi_heat(Col& C, const MpConst& K, double& tz, double dz1, double dp1, double qv, double ql,
                   double qr, double qi, double qs, double qg, double flux, double fp, bool valid, double c_cond) {
  const double dgz = -0.5 * K.GRAV * dz1;
  const double cvn = dp1 * (K.CV_AIR + qv * K.CV_VAP + (qr + ql) * K.C_LIQ + (qi + qs + qg) * K.C_ICE);
  double a, b;
  if (C.k == 0) {
    const double tmp = cvn + flux * c_cond;
    a = tz + flux * dgz / tmp;
    b = 0.0;
  } else {
    const double D = cvn + c_cond * flux;
    a = ((cvn + c_cond * (flux - fp)) * tz + dgz * (fp + flux)) / D;
    b = fp * c_cond / D;
  }
  if (!valid) {
    a = tz;
    b = 0.0;
  }
  tz = C.scan_affine(a, b);
}

// Vertical-velocity update by one falling species given the flux and fall
// speed at this level and the level above (microphysics.py:492-515).
SHD double w_update(int k, double w, double dm, double flux, double vt, double fp, double vp) {
  if (k == 0) return (dm * w + flux * vt) / (dm - flux);
  return (dm * w - fp * vp + flux * vt) / (dm + fp - flux);
}

// Monotone vertical slope for autoconversion (microphysics.py:595-620,
// 1341-1367), before the h_var floor: dq_k = 0.5 (q_k - q_{k-1}).
template <class Col>
SHD double mono_slope(Col& C, double q) {
  double qp, qn;
  C.nbrs(q, qp, qn);
  const double dq = 0.5 * (q - qp);
  const double dqn = 0.5 * (qn - q);
  double v = 0.0;
  if (C.k >= 1 && C.k <= C.L - 2) {
    v = 0.5 * fmin(fabs(dq + dqn), 0.5 * q);
    if (dq * dqn <= 0.0) {
      if (dq > 0.0)
        v = fmin(v, fmin(dq, -dqn));
      else
        v = 0.0;
    }
  }
  return v;
}

// ----------------------------------------------------------------- layouts
// How a block's threads map onto its G columns. A layout gives the column
// type the stages run on, the block's thread count, the pitch RP (>= L) of
// the staging tiles, and the scratch and work doubles of each of its NGRP
// barrier groups.
//
// ColumnLayout<NW, G>: each of the G columns on NW whole warps of its own
// (level k = 32 w + lane); one barrier group per column.
template <int NW, int G_>
struct ColumnLayout {
  using Col = Column<NW>;
  static constexpr int G = G_;
  static constexpr int NGRP = G_;
  static constexpr int THREADS = 32 * NW * G_;
  static constexpr int RP = Tiles<NW>::RP;
  static constexpr int SCR = Tiles<NW>::SCR;
  static constexpr int WORK = 2 * RP;
  // set up thread tid's column object; returns its block column (G: none)
  static SHD int setup(Col& C, int tid, int L, double* scr, double* work) {
    const int g = tid / (32 * NW);
    C.w = (tid >> 5) % NW;
    C.lane = tid & 31;
    C.k = 32 * C.w + C.lane;
    C.L = L;
    C.bar = 1 + g;
    C.scr = scr + (size_t)g * 2 * SCR;
    C.work = work + (size_t)g * WORK;
    C.par = 0;
    return g;
  }
};

// PackedLayout<NWG, P, NGRP>: NGRP groups of NWG warps, each holding P
// columns back to back (PackedColumn); G = P NGRP columns per block.
template <int NWG, int P, int NGRP_>
struct PackedLayout {
  using Col = PackedColumn<NWG, P>;
  static constexpr int G = P * NGRP_;
  static constexpr int NGRP = NGRP_;
  static constexpr int THREADS = 32 * NWG * NGRP_;
  static constexpr int RP = Col::WP;
  static constexpr int SCR = Col::SCR;
  static constexpr int WORK = (P + 1) * 2 * Col::WP;
  static SHD int setup(Col& C, int tid, int L, double* scr, double* work) {
    const int gi = tid / (32 * NWG);
    C.init(tid % (32 * NWG), L, 1 + gi, scr + (size_t)gi * 2 * SCR, work + (size_t)gi * WORK);
    return C.c < P ? gi * P + C.c : G;
  }
};

// ----------------------------------------------------------------- staging
// Shared memory: N_IN tiles of G rows of RP doubles (field f, block column g,
// level k at (f * G + g) * RP + k), then the groups' scratch (NGRP x 2 x SCR
// doubles), then their work rows for the rare sequential vapour borrow.
template <class LY>
struct Smem {
  static constexpr size_t tiles = (size_t)N_IN * LY::G * LY::RP;
  static constexpr size_t scratch = tiles;
  static constexpr size_t work = scratch + (size_t)LY::NGRP * 2 * LY::SCR;
  static constexpr size_t total = work + (size_t)LY::NGRP * LY::WORK;
  static constexpr size_t bytes = total * sizeof(double);
};

// Element e < G L of a field's block tile for thread e, in the two memory
// orders: i-fastest storages take consecutive columns on consecutive
// threads (g = e % G, k = e / G), k-fastest ones consecutive levels
// (g = e / L, k = e % L). Every layout has at least G L threads, so each
// thread moves at most one element of each field, and all loads of a stage
// are issued before any store: one memory round trip per stage.
struct StageMap {
  int g, k, gk, kk;
  bool ok, okk;
  int64_t i, j, ik, jk;
  template <int G>
  SHD void set(const MpArgs& A, int tid, int64_t c0) {
    const int L = A.nz;
    g = tid % G;
    k = tid / G;
    const int64_t col = c0 + g;
    ok = col < A.ncol && k < L;
    i = ok ? col % A.nx : 0;
    j = ok ? col / A.nx : 0;
    gk = tid / L;
    kk = tid % L;
    const int64_t colk = c0 + gk;
    okk = gk < G && colk < A.ncol;
    ik = okk ? colk % A.nx : 0;
    jk = okk ? colk / A.nx : 0;
  }
};

template <class LY>
SHD void stage_in(const MpArgs& A, double* sm, int64_t c0) {
  constexpr int RP = LY::RP, G = LY::G;
  StageMap M;
  M.template set<G>(A, threadIdx.x, c0);
  double v[N_IN];
#pragma unroll
  for (int f = 0; f < N_IN; ++f) {
    const Fld3 F = A.in[f];
    v[f] = 0.0;
    if (F.sk == 1) {
      if (M.okk) v[f] = F.p[M.ik * F.si + M.jk * F.sj + M.kk];
    } else if (M.ok) {
      v[f] = F.p[M.i * F.si + M.j * F.sj + (int64_t)M.k * F.sk];
    }
  }
#pragma unroll
  for (int f = 0; f < N_IN; ++f) {
    const Fld3 F = A.in[f];
    if (F.sk == 1) {
      if (M.okk) sm[(f * G + M.gk) * RP + M.kk] = v[f];
    } else if (M.ok) {
      sm[(f * G + M.g) * RP + M.k] = v[f];
    }
  }
}

enum OutMode { OM_SKIP = 0, OM_ADD = 1, OM_ADD_K1 = 2, OM_SET = 3 };

SHD int out_mode(const MpConst& K, int o) {
  int m = OM_ADD;
  if (o == OUT_UDT || o == OUT_VDT) m = K.sedi_transport ? OM_ADD_K1 : OM_SKIP;
  if (o == OUT_QA_DT && K.do_qa) m = OM_SET;
  if (o == OUT_W) m = K.do_sedi_w ? OM_SET : OM_SKIP;
  if (o == OUT_QAZ) m = OM_SET;
  return m;
}

template <class LY>
SHD void stage_out(const MpArgs& A, const double* sm, int64_t c0) {
  constexpr int RP = LY::RP, G = LY::G;
  const MpConst& K = A.K;
  StageMap M;
  M.template set<G>(A, threadIdx.x, c0);
  int mode[N_OUT];
  double* dst[N_OUT];
  double old[N_OUT];
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) {
    int m = out_mode(K, o);
    const Fld3 F = A.out[o];
    const bool kf = F.sk == 1;
    const int lev = kf ? M.kk : M.k;
    if (!(kf ? M.okk : M.ok) || (m == OM_ADD_K1 && lev < 1)) m = OM_SKIP;
    mode[o] = m;
    dst[o] = kf ? F.p + M.ik * F.si + M.jk * F.sj + M.kk : F.p + M.i * F.si + M.j * F.sj + (int64_t)M.k * F.sk;
    old[o] = (m == OM_ADD || m == OM_ADD_K1) ? *dst[o] : 0.0;
  }
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) {
    if (mode[o] == OM_SKIP) continue;
    const bool kf = A.out[o].sk == 1;
    const double v = kf ? sm[(o * G + M.gk) * RP + M.kk] : sm[(o * G + M.g) * RP + M.k];
    *dst[o] = (mode[o] == OM_SET) ? v : old[o] + v;
  }
}

// ------------------------------------------------------------ step stages
// The step body as stages, shared by the forward kernels and the adjoint
// (which replays them). Per level: the prognostic state, and the values set
// by fields_init or at the start of each sub-step that later stages read.
struct LevState {
  double qv, ql, qr, qi, qs, qg, tz, w;
};
struct StepGeom {
  double dp1, p1, h_var, rh_adj, rh_rain, ccn, c_praut;  // fields_init
  double den, denfac, dz1, dz;                           // start of each sub-step
};

// fields_init (:27-276) for one level from its input values (defaults on
// the padding levels k >= L, whose values never reach a real level).
template <class Col>
SHD void fields_init(Col& C, const MpConst& K, bool valid, double pt, double qvi, double qli, double qri,
                     double qii, double qsi, double qgi, double delp, double wz, double dz0, double land, double area,
                     LevState& S, StepGeom& P) {
  const int k = C.k, L = C.L;
  S.tz = pt;
  P.dp1 = delp;
  P.dp1 = P.dp1 * (1.0 - qvi);
  const double omq = delp / P.dp1;
  S.qv = qvi * omq;
  S.ql = qli * omq;
  S.qr = qri * omq;
  S.qi = qii * omq;
  S.qs = qsi * omq;
  S.qg = qgi * omq;
  const double den0 = -P.dp1 / (K.GRAV * dz0);
  P.p1 = den0 * K.RDGAS * pt;
  S.w = wz;
  double ccn;
  if (K.prog_ccn) {
    ccn = 0.0 * 1.0e6;
  } else {
    ccn = (K.ccn_l * land + K.ccn_o * (1.0 - land)) * 1.0e6;
    if (K.use_ccn) {
      double tzb, p1b;
      C.bcast2(S.tz, P.p1, L - 1, tzb, p1b);
      ccn = ccn * K.RDGAS * tzb / p1b;
    }
  }
  P.ccn = ccn;
  P.c_praut = K.cpaut * xpow(ccn * RHOR, -1.0 / 3.0);
  const double s_leng = sqrt(sqrt(area * 1.0e-10));
  const double t_land = K.dw_land * s_leng;
  const double t_ocean = K.dw_ocean * s_leng;
  double h_var = t_land * land + t_ocean * (1.0 - land);
  P.h_var = fmin(0.2, fmax(0.01, h_var));
  P.rh_adj = 1.0 - P.h_var - K.rh_inc;
  P.rh_rain = fmax(0.35, P.rh_adj - K.rh_inr);

  if (K.fix_negative) {
    fix_negative_point(K, S.qv, S.ql, S.qr, S.qi, S.qs, S.qg, S.tz);
    // FORWARD borrow of negative vapour from the level above (:244-247):
    // a sequential sweep by one thread over the column, taken only when
    // some level above the bottom is negative (in any column sharing the
    // barrier: the sweep leaves a column without such a level unchanged)
    if (C.group_any(valid && k < L - 1 && S.qv < 0.0)) {
      double* wq = C.work;
      double* wd = wq + Col::WP;
      if (valid) {
        wq[k] = S.qv;
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
      if (valid) S.qv = wq[k];
    }
    if (k < L - 1 && S.qv < 0.0) S.qv = 0.0;
    // bottom layer borrows from the layer above (:253-276)
    double qb, db, qb1, db1;
    C.bcast2(S.qv, P.dp1, L - 1, qb, db);
    C.bcast2(S.qv, P.dp1, L - 2, qb1, db1);
    if ((qb < 0.0) && (qb1 > 0.0)) {
      const double dq = fmin(-qb * db, qb1 * db1);
      if (k == L - 2) S.qv = S.qv - dq / P.dp1;
      if (k == L - 1) S.qv = S.qv + dq / P.dp1;
    }
  }
}

// density, fall factor and layer thickness at the start of a sub-step
// (warm_rain with is_first, :349-380)
template <class Col>
SHD void substep_geometry(Col& C, const MpConst& K, bool valid, double t0, double dz0, const LevState& S,
                          StepGeom& P) {
  const double den0 = -P.dp1 / (K.GRAV * dz0);
  P.dz1 = dz0 * S.tz / t0;
  P.den = den0 * dz0 / P.dz1;
  P.denfac = sqrt(SFCRHO / P.den);
  P.dz = C.heights(valid ? -P.dz1 : 0.0, K.zs);
}

// Recorder of a stage's intermediate states. The forward kernels pass
// NoRec (every call compiles away); the adjoint's replay passes one that
// stores the states the reverse sweeps start from.
struct NoRec {
  SHD void state(int, const LevState&) const {}
  SHD void value(int, double) const {}
  SHD void flag(bool) const {}
};

// warm_rain (:280-653) after the geometry: rain evaporation and accretion,
// implicit rain fall with the vertical-velocity transport and heating, then
// autoconversion. Returns the rain flux m1_rain at this level and the
// surface flux r1.
// A recorder gets the states after the first evaporation (slot 0), after the
// fall (1) and after the second evaporation (2), the liquid slope (value 0)
// and the column's rain-fall decision.
template <bool MIXED, class Col, class Rec = NoRec>
SHD void warm_rain(Col& C, const MpConst& K, const MpConstF& KF, bool valid, LevState& S, const StepGeom& P,
                   double& vtr, double& m1_rain, double& r1, bool* falls = nullptr, const Rec& rec = Rec()) {
  const int k = C.k, L = C.L;
  double &qv = S.qv, &ql = S.ql, &qr = S.qr, &qi = S.qi, &qs = S.qs, &qg = S.qg, &tz = S.tz, &w = S.w;
  const double dt5 = 0.5 * K.dt_rain;
  m1_rain = 0.0;
  bool gfall;
  const bool fall = C.any_group(valid && (qr > QRMIN), gfall);
  if (falls) *falls = fall;
  rec.flag(fall);
  r1 = 0.0;
  if (!fall) vtr = VF_MIN;
  // The fall's vertical operations run whenever a column sharing the
  // barrier has falling rain; a column without it takes part with no mass
  // (valid false), which leaves its state unchanged and its flux zero.
  if (gfall) {
    const bool vf = valid && fall;
    if (fall) {
      if constexpr (MIXED) {
        vtr = rain_fspeed_m(K, qr, P.den);
        revap_racc_m(K, KF, dt5, P.h_var, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac);
      } else {
        vtr = rain_fspeed(K, qr, P.den);
        revap_racc(K, dt5, P.h_var, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac);
      }
    }
    rec.state(0, S);
    const double dm = P.dp1 * (1.0 + qv + ql + qr + qi + qs + qg);
    m1_rain = implicit_fall(C, qr, vtr, P.dz, P.dp1, vf, K.dt_rain);
    double fv[2] = {m1_rain, vtr}, pv[2];
    C.template prevN<2>(fv, pv);
    r1 = C.bcast(m1_rain, L - 1);
    if (fall && K.do_sedi_w) w = w_update(k, w, dm, m1_rain, vtr, pv[0], pv[1]);
    if (K.do_sedi_heat) sedi_heat(C, K, tz, P.dz1, P.dp1, qv, ql, qr, qi, qs, qg, m1_rain, pv[0], vf, K.C_LIQ);
    rec.state(1, S);
    if (fall) {
      if constexpr (MIXED)
        revap_racc_m(K, KF, dt5, P.h_var, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac);
      else
        revap_racc(K, dt5, P.h_var, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac);
    }
    rec.state(2, S);
  } else {
    rec.state(0, S);
    rec.state(1, S);
    rec.state(2, S);
  }
  if (K.irain_f != 0) {
    if constexpr (MIXED)
      autoconv_no_subgrid_var_m(K, KF, ql, qr, tz, P.den, P.ccn, P.c_praut);
    else
      autoconv_no_subgrid_var(K, ql, qr, tz, P.den, P.ccn, P.c_praut);
  } else {
    double dl;
    if (K.z_slope_liq) {
      dl = mono_slope(C, ql);
      rec.value(0, dl);
      dl = fmax(dl, fmax(QVMIN, P.h_var * ql));
    } else {
      dl = fmax(QVMIN, P.h_var * ql);
    }
    if constexpr (MIXED)
      autoconv_subgrid_var_m(K, KF, ql, qr, tz, P.den, P.ccn, P.c_praut, dl);
    else
      autoconv_subgrid_var(K, ql, qr, tz, P.den, P.ccn, P.c_praut, dl);
  }
}

// sedimentation (:657-1217): fall speeds, cloud ice melting, and the
// implicit falls of ice, snow and graupel with their vertical-velocity
// transport and heating. Returns the solid flux m1_sol at this level and
// adds the surface fluxes to ice, snow and graupel.
// A recorder gets the cloud ice fall speed (value 0).
template <bool MIXED, class Col, class Rec = NoRec>
SHD void sedimentation(Col& C, const MpConst& K, const MpConstF& KF, bool valid, LevState& S,
                       const StepGeom& P, double& vtg, double& vts, double& m1_sol, double& ice, double& snow,
                       double& graupel, unsigned* flags = nullptr, const Rec& rec = Rec()) {
  const int k = C.k, L = C.L;
  double &qv = S.qv, &ql = S.ql, &qr = S.qr, &qi = S.qi, &qs = S.qs, &qg = S.qg, &tz = S.tz, &w = S.w;
  const double dp1 = P.dp1, dz = P.dz;
  double vti;
  if constexpr (MIXED)
    fall_speed_m(K, KF, qg, qi, qs, tz, P.den, vtg, vti, vts);
  else
    fall_speed(K, qg, qi, qs, tz, P.den, vtg, vti, vts);
  rec.value(0, vti);
  m1_sol = 0.0;
  // cloud ice melting at and below the first level warmer than tice (:702-746)
  const int first = C.min_int((valid && tz > K.tice) ? k : (1 << 30));
  if ((k >= first || k == L - 1) && valid) sedi_ice_melt(K, qv, ql, qr, qi, qs, qg, tz);
  // ice (:773-900), snow (:902-1035) and graupel (:1037-1168): their
  // implicit falls are independent of one another, so the three share
  // each column exchange; the vertical-velocity updates, which the
  // reference applies species after species, stay in that order.
  bool fi, fs, fg, gi, gs, gg;
  C.any3_group(valid && (qi > QRMIN), valid && (qs > QRMIN), valid && (qg > QRMIN), fi, fs, fg, gi, gs, gg);
  fi = fi && (K.vi_fac >= 1.0e-5);
  gi = gi && (K.vi_fac >= 1.0e-5);
  if (flags)
    *flags |= (fi ? FLAG_ICE_FALLS : 0u) | (fs ? FLAG_SNOW_FALLS : 0u) | (fg ? FLAG_GRAUPEL_FALLS : 0u) |
              ((unsigned)min(first, L - 1) << FLAG_MELT_SHIFT);
  double mp = 0.0;  // m1_sol at the level above, for the heating
  // taken by every column sharing the barrier when one of them has a
  // falling species; each species' results apply only where it falls
  if (gi || gs || gg) {
    const double dd[3] = {K.dts * vti, K.dts * vts, K.dts * vtg};
    double ddp[3];
    C.template prevN<3>(dd, ddp);
    const double qq[3] = {qi, qs, qg};
    double ra[3], rb[3], r[3];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const double qmass = valid ? qq[n] * dp1 : 0.0;
      const double D = dz + dd[n];
      ra[n] = qmass / D;
      rb[n] = (k == 0) ? 0.0 : ddp[n] / D;
      if (!valid) {
        ra[n] = 0.0;
        rb[n] = 0.0;
      }
    }
    C.template scanN<3>(ra, rb, r);
    double flux[3];
#pragma unroll
    for (int n = 0; n < 3; ++n) flux[n] = valid ? dd[n] * r[n] : 0.0;
    const double dm_i = dp1 * (1.0 + qv + ql + qr + qi + qs + qg);
    if (fi && valid) qi = r[0] * dz / dp1;
    const double dm_s = dp1 * (1.0 + qv + ql + qr + qi + qs + qg);
    if (fs && valid) qs = r[1] * dz / dp1;
    const double dm_g = dp1 * (1.0 + qv + ql + qr + qi + qs + qg);
    if (fg && valid) qg = r[2] * dz / dp1;
    double sfc[3];
    C.template bcastN<3>(flux, L - 1, sfc);
    const double nv[6] = {flux[0], vti, flux[1], vts, flux[2], vtg};
    double pv[6];
    C.template prevN<6>(nv, pv);
    if (fi) {
      m1_sol = flux[0];
      mp = pv[0];
      if (K.do_sedi_w) w = w_update(k, w, dm_i, flux[0], vti, pv[0], pv[1]);
      ice = ice + sfc[0];
    }
    if (fs) {
      m1_sol = m1_sol + flux[1];
      mp = mp + pv[2];
      if (K.do_sedi_w) w = w_update(k, w, dm_s, flux[1], vts, pv[2], pv[3]);
      snow = snow + sfc[1];
    }
    if (fg) {
      m1_sol = m1_sol + flux[2];
      mp = mp + pv[4];
      if (K.do_sedi_w) w = w_update(k, w, dm_g, flux[2], vtg, pv[4], pv[5]);
      graupel = graupel + sfc[2];
    }
  }
  if (K.do_sedi_heat) sedi_heat(C, K, tz, P.dz1, dp1, qv, ql, qr, qi, qs, qg, m1_sol, mp, valid, K.C_ICE);
}

// icloud (:1220-1449): instant melting or freezing, the ice slope, the ice
// processes and the saturation adjustment. A recorder gets the state between
// the ice processes and the adjustment (slot 0), the ice slope (value 0) and
// the cloud ice after melting and freezing (value 1).
template <bool MIXED, class Col, class Rec = NoRec>
SHD void icloud(Col& C, const MpConst& K, const MpConstF& KF, bool valid, LevState& S, const StepGeom& P,
                double& qa, double vtg, double vtr, double vts, const Rec& rec = Rec()) {
  double &qv = S.qv, &ql = S.ql, &qr = S.qr, &qi = S.qi, &qs = S.qs, &qg = S.qg, &tz = S.tz;
  double q_liq, q_sol, cvm;
  icloud_melt_freeze(K, qv, ql, qr, qi, qs, qg, tz, P.den, q_liq, q_sol, cvm);
  rec.value(1, qi);
  double di;
  if (K.z_slope_ice) {
    di = mono_slope(C, qi);
    rec.value(0, di);
    di = fmax(di, fmax(QVMIN, P.h_var * qi));
  } else {
    di = fmax(QVMIN, P.h_var * qi);
  }
  if (valid) {
    if constexpr (MIXED)
      icloud_processes_m(K, KF, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac, vtg, vtr, vts, P.p1, di, q_liq, q_sol,
                         cvm);
    else
      icloud_processes(K, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac, vtg, vtr, vts, P.p1, di, q_liq, q_sol, cvm);
    rec.state(0, S);
    if constexpr (MIXED)
      subgrid_z_proc<double, float>(K, P.h_var, P.rh_adj, P.rh_rain, qa, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac,
                                    P.p1, &KF);
    else
      subgrid_z_proc(K, P.h_var, P.rh_adj, P.rh_rain, qa, qg, qi, ql, qr, qs, qv, tz, P.den, P.denfac, P.p1);
  }
}

// ------------------------------------------------------------------ kernel
// The step of columns c0 .. c0 + G - 1 between staging in and staging out,
// on layout LY: inputs are read from, and outputs written to, the tiles at
// `sm` (field f of block column g at level k at (f * G + g) * RP + k);
// `scr` and `work` are the barrier groups' scratch and work rows. Every
// thread of a barrier group runs the whole step, idle ones (levels beyond L,
// columns beyond the domain, a packed group's idle tail) with valid false,
// so that the groups' vertical operations see all their threads.
// MIXED selects the mixed-precision process rates (mp_physics_mixed.cuh).
template <class LY, bool MIXED, bool FLAGS = false>
SHD void mp_body(const MpArgs& A, double* sm, double* scr, double* work, const int64_t c0) {
  constexpr int RP = LY::RP;
  constexpr int G = LY::G;
  const MpConst& K = A.K;
  const MpConstF& KF = A.KF;
  const int L = A.nz;
  typename LY::Col C;
  const int g = LY::setup(C, threadIdx.x, L, scr, work);
  const bool slot_ok = g < G;
  const int64_t col = c0 + (slot_ok ? g : 0);
  const bool col_ok = slot_ok && col < A.ncol;
  const int k = C.k;
  const bool valid = col_ok && k < L;
  double* tile = sm + (size_t)(slot_ok ? g : 0) * RP + (valid ? k : 0);  // field f of this level at tile[f * G * RP]
  auto TL = [&](int f) -> double& { return tile[(size_t)f * G * RP]; };

  const int64_t cc = col < A.ncol ? col : A.ncol - 1;
  const int64_t ci = cc % A.nx, cj = cc / A.nx;
  LevState S;
  StepGeom P;
  double qa = valid ? TL(IN_QAZ) : 0.0;
  double m1 = 0.0, m1_sol = 0.0, vtr = VF_MIN, vtg = VF_MIN, vts = VF_MIN;
  P.den = 1.0;
  P.denfac = 1.0;
  P.dz1 = -100.0;
  P.dz = 100.0;
  // ------------------------------------------------ fields_init (:27-276)
  fields_init(C, K, valid, valid ? TL(IN_PT) : 250.0, valid ? TL(IN_QV) : 0.0, valid ? TL(IN_QL) : 0.0,
              valid ? TL(IN_QR) : 0.0, valid ? TL(IN_QI) : 0.0, valid ? TL(IN_QS) : 0.0, valid ? TL(IN_QG) : 0.0,
              valid ? TL(IN_DELP) : 1.0, valid ? TL(IN_W) : 0.0, valid ? TL(IN_DELZ) : -100.0,
              A.land.p[ci * A.land.si + cj * A.land.sj], A.area.p[ci * A.area.si + cj * A.area.sj], S, P);

  double rain = 0.0, snow = 0.0, ice = 0.0, graupel = 0.0;
#pragma unroll 1
  for (int it = 0; it < K.ntimes; ++it) {
    unsigned fl = 0u;  // this sub-step's column flags (FLAGS only)
    // warm_rain with is_first, sedimentation, warm_rain again (one copy
    // of the warm_rain code, run twice)
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      const bool is_first = pass == 0;
      if (is_first) substep_geometry(C, K, valid, valid ? TL(IN_PT) : 250.0, valid ? TL(IN_DELZ) : -100.0, S, P);
      double m1_rain, r1;
      bool falls = false;
      warm_rain<MIXED>(C, K, KF, valid, S, P, vtr, m1_rain, r1, FLAGS ? &falls : nullptr);
      if constexpr (FLAGS) fl |= falls ? (is_first ? FLAG_RAIN_FALLS_1 : FLAG_RAIN_FALLS_2) : 0u;
      rain = rain + r1;
      m1 = is_first ? m1 + m1_rain : m1 + m1_rain + m1_sol;
      if (!is_first) break;
      sedimentation<MIXED>(C, K, KF, valid, S, P, vtg, vts, m1_sol, ice, snow, graupel, FLAGS ? &fl : nullptr);
      rain = rain + 0.0;
    }
    icloud<MIXED>(C, K, KF, valid, S, P, qa, vtg, vtr, vts);
    if constexpr (FLAGS) {
      if (k == 0 && col_ok) A.flags[(int64_t)it * A.ncol + col] = (int)fl;
    }
  }
  const double qv = S.qv, ql = S.ql, qr = S.qr, qi = S.qi, qs = S.qs, qg = S.qg, tz = S.tz, w = S.w;
  const double dp1 = P.dp1;
  // ------------------------------------------------ fields_update (:1452-1553)
  const double dp0 = valid ? TL(IN_DELP) : 1.0;
  const double u0 = valid ? TL(IN_UA) : 0.0;
  const double v0 = valid ? TL(IN_VA) : 0.0;
  double u1 = u0, v1 = v0;
  if (K.sedi_transport) {
    const double mp = C.prev(m1);
    double au, av, b;
    if (k == 0 || !valid) {
      au = u0;
      av = v0;
      b = 0.0;
    } else {
      const double D = dp0 + mp;
      au = dp0 * u0 / D;
      av = dp0 * v0 / D;
      b = mp / D;
    }
    C.scan_affine2(au, b, av, b, u1, v1);
  }
  if (valid) {
    const double rdt = K.rdt;
    const double omq0 = dp0 / dp1;
    const double qv0 = TL(IN_QV) * omq0, ql0 = TL(IN_QL) * omq0, qr0 = TL(IN_QR) * omq0;
    const double qi0 = TL(IN_QI) * omq0, qs0 = TL(IN_QS) * omq0, qg0 = TL(IN_QG) * omq0;
    const double t0 = TL(IN_PT), qa0 = TL(IN_QA);
    const double omq = dp1 / dp0;
    const double inc_qv = rdt * (qv - qv0) * omq;
    const double inc_ql = rdt * (ql - ql0) * omq;
    const double inc_qr = rdt * (qr - qr0) * omq;
    const double inc_qi = rdt * (qi - qi0) * omq;
    const double inc_qs = rdt * (qs - qs0) * omq;
    const double inc_qg = rdt * (qg - qg0) * omq;
    const double cvm = K.c_air + qv * K.c_vap + (qr + ql) * K.C_LIQ + (qi + qs + qg) * K.C_ICE;
    const double inc_pt = rdt * (tz - t0) * cvm / K.CP_AIR;
    const double inc_qa = K.do_qa ? 0.0 : rdt * (qa / (double)K.ntimes - qa0);
    const double inc_u = K.sedi_transport ? (u1 - u0) * rdt : 0.0;
    const double inc_v = K.sedi_transport ? (v1 - v0) * rdt : 0.0;
    TL(OUT_PT_DT) = inc_pt;
    TL(OUT_QV_DT) = inc_qv;
    TL(OUT_QL_DT) = inc_ql;
    TL(OUT_QR_DT) = inc_qr;
    TL(OUT_QI_DT) = inc_qi;
    TL(OUT_QS_DT) = inc_qs;
    TL(OUT_QG_DT) = inc_qg;
    TL(OUT_QA_DT) = inc_qa;
    TL(OUT_UDT) = inc_u;
    TL(OUT_VDT) = inc_v;
    TL(OUT_W) = w;
    TL(OUT_QAZ) = qa;
    // the device error word: the first column (+ 1) that produced a NaN or
    // an infinity, for the host to read after the step (never traps)
    if (A.err && !(isfinite(inc_pt) && isfinite(inc_qv) && isfinite(inc_ql) && isfinite(inc_qr) &&
                   isfinite(inc_qi) && isfinite(inc_qs) && isfinite(inc_qg) && isfinite(inc_qa) &&
                   isfinite(inc_u) && isfinite(inc_v) && isfinite(w) && isfinite(qa)))
      atomicCAS(A.err, 0, (int)(col + 1));
  }
  if (k == 0 && col_ok) {
    const double convt = 86400.0 * K.rdt * K.RGRAV;
    if (A.rain) A.rain[col] = rain * convt;
    if (A.snow) A.snow[col] = snow * convt;
    if (A.ice) A.ice[col] = ice * convt;
    if (A.graupel) A.graupel[col] = graupel * convt;
    if (A.err && !(isfinite(rain) && isfinite(snow) && isfinite(ice) && isfinite(graupel)))
      atomicCAS(A.err, 0, (int)(col + 1));
  }
}

// One block's work: columns c0 .. c0 + G - 1 of the domain described by A.
template <class LY, bool MIXED, bool FLAGS = false>
SHD void mp_block(const MpArgs& A, double* sm, const int64_t c0) {
  using SM = Smem<LY>;
  stage_in<LY>(A, sm, c0);
  __syncthreads();
  mp_body<LY, MIXED, FLAGS>(A, sm, sm + SM::scratch, sm + SM::work, c0);
  __syncthreads();
  stage_out<LY>(A, sm, c0);
}

// ------------------------------------------------- persistent, double-buffered
// The same step with the staging taken off the critical path: a persistent
// block walks its share of the column blocks and, while it computes one,
// copies the next one's inputs into the other buffer with cp.async: the 14
// input fields and, where the two buffers have room for them (NT = N_TILE),
// the 10 old tendencies the step adds to. With NT = N_IN the stage-out reads
// the old tendencies itself, as the one-block-per-column-block kernel does.
//
// Shared memory: two buffers of NT rows per block column, then the scratch
// and work rows.
constexpr int N_TILE = N_IN + 10;  // the inputs, then the tendencies read before the update

template <class LY, int NT = N_TILE>
struct SmemP {
  static constexpr size_t buf = (size_t)NT * LY::G * LY::RP;
  static constexpr size_t scratch = 2 * buf;
  static constexpr size_t work = scratch + (size_t)LY::NGRP * 2 * LY::SCR;
  static constexpr size_t total = work + (size_t)LY::NGRP * LY::WORK;
  static constexpr size_t bytes = total * sizeof(double);
};

SHD void cp_async8(double* dst_smem, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
SHD void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
SHD void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Tile row of the old value of tendency o (o < 10), after the inputs.
SHD int tend_row(int o) { return N_IN + o; }

SHD const Fld3& tile_src(const MpArgs& A, int r) { return r < N_IN ? A.in[r] : A.out[r - N_IN]; }

// stage_in's mapping, each element copied asynchronously (no register pass):
// the first NT tile rows (the inputs, then the old tendencies).
template <class LY, int NT = N_TILE>
SHD void stage_in_async(const MpArgs& A, double* sm, int64_t c0) {
  constexpr int RP = LY::RP, G = LY::G;
  const MpConst& K = A.K;
  StageMap M;
  M.template set<G>(A, threadIdx.x, c0);
#pragma unroll
  for (int r = 0; r < NT; ++r) {
    if (r >= N_IN) {
      // a tendency the update adds to (stage_out's OM_ADD / OM_ADD_K1 fields)
      const int o = r - N_IN;
      if ((o == OUT_UDT || o == OUT_VDT) && !K.sedi_transport) continue;
      if (o == OUT_QA_DT && K.do_qa) continue;
    }
    const Fld3& F = tile_src(A, r);
    if (F.sk == 1) {
      if (M.okk) cp_async8(&sm[(r * G + M.gk) * RP + M.kk], F.p + M.ik * F.si + M.jk * F.sj + M.kk);
    } else if (M.ok) {
      cp_async8(&sm[(r * G + M.g) * RP + M.k], F.p + M.i * F.si + M.j * F.sj + (int64_t)M.k * F.sk);
    }
  }
}

// stage_out with the old tendencies taken from the tile.
template <class LY>
SHD void stage_out_tiled(const MpArgs& A, const double* sm, int64_t c0) {
  constexpr int RP = LY::RP, G = LY::G;
  const MpConst& K = A.K;
  StageMap M;
  M.template set<G>(A, threadIdx.x, c0);
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) {
    int m = out_mode(K, o);
    const Fld3 F = A.out[o];
    const bool kf = F.sk == 1;
    const int lev = kf ? M.kk : M.k;
    if (!(kf ? M.okk : M.ok) || (m == OM_ADD_K1 && lev < 1)) m = OM_SKIP;
    if (m == OM_SKIP) continue;
    const int gg = kf ? M.gk : M.g;
    const double v = sm[(o * G + gg) * RP + lev];
    double* dst = kf ? F.p + M.ik * F.si + M.jk * F.sj + M.kk : F.p + M.i * F.si + M.j * F.sj + (int64_t)M.k * F.sk;
    *dst = (m == OM_SET) ? v : sm[(tend_row(o) * G + gg) * RP + lev] + v;
  }
}

template <class LY, int MINB, bool MIXED, int NT>
__global__ void __launch_bounds__(LY::THREADS, MINB)
    mp_step_persistent_kernel(const __grid_constant__ MpArgs A, const int64_t nblk) {
  extern __shared__ double sm[];
  using SP = SmemP<LY, NT>;
  constexpr int G = LY::G;
  double* const scr = sm + SP::scratch;
  double* const work = sm + SP::work;
  int64_t b = blockIdx.x;
  if (b < nblk) stage_in_async<LY, NT>(A, sm, b * G);
  cp_async_commit();
  for (int it = 0; b < nblk; b += gridDim.x, ++it) {
    double* const cur = sm + (it & 1) * SP::buf;
    double* const nxt = sm + ((it + 1) & 1) * SP::buf;
    cp_async_wait_all();
    __syncthreads();  // this block's inputs have landed; the previous one's stage-out is done with nxt
    if (b + gridDim.x < nblk) stage_in_async<LY, NT>(A, nxt, (b + gridDim.x) * G);
    cp_async_commit();
    mp_body<LY, MIXED>(A, cur, scr, work, b * G);
    __syncthreads();
    if constexpr (NT == N_TILE)
      stage_out_tiled<LY>(A, cur, b * G);
    else
      stage_out<LY>(A, cur, b * G);
  }
  cp_async_wait_all();
}

template <class LY, int MINB, bool MIXED, bool FLAGS = false>
__global__ void __launch_bounds__(LY::THREADS, MINB) mp_step_kernel(const __grid_constant__ MpArgs A) {
  extern __shared__ double sm[];
  mp_block<LY, MIXED, FLAGS>(A, sm, (int64_t)blockIdx.x * LY::G);
}

// Many domains (ensemble members) in one persistent launch. Work item wi
// of the flattened index space is block (wi - offs[m]) of member m, where
// offs[m] <= wi < offs[m + 1] (offs holds nm + 1 prefix sums of each member's
// ceil(ncol / G)). The persistent blocks take items from a device counter
// (zero at launch), so a block that drew cheap columns takes more of them:
// the items' cost varies with the physics their columns run. A block copies
// its member's parameter block into shared memory when the member changes;
// the step body reads its constants from there. Measured with 64 members
// (C24/C48/C96, L79): a fixed stride of items per block and a prefetch of
// the next item's inputs were both slower.
SHD int find_member(const int64_t* __restrict__ offs, int nm, int64_t wi) {
  int lo = 0, hi = nm - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (offs[mid] <= wi)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <class LY, int MINB, bool MIXED>
__global__ void __launch_bounds__(LY::THREADS, MINB)
    mp_ensemble_kernel(const MpArgs* __restrict__ members, const int64_t* __restrict__ offs, int nm,
                       unsigned long long* __restrict__ counter) {
  extern __shared__ double sm[];
  __shared__ MpArgs sargs;
  __shared__ long long sitem;
  __shared__ int smember;
  const int64_t total = offs[nm];
  int loaded = -1;
  for (;;) {
    if (threadIdx.x == 0) {
      sitem = (long long)atomicAdd(counter, 1ull);
      smember = sitem < total ? find_member(offs, nm, sitem) : 0;
    }
    __syncthreads();
    const int64_t wi = sitem;
    const int m = smember;
    if (wi >= total) break;
    if (m != loaded) {
      const int* src = reinterpret_cast<const int*>(members + m);
      int* dst = reinterpret_cast<int*>(&sargs);
      constexpr int nwords = (int)(sizeof(MpArgs) / sizeof(int));
      for (int e = threadIdx.x; e < nwords; e += blockDim.x) dst[e] = src[e];
      loaded = m;
      __syncthreads();
    }
    mp_block<LY, MIXED>(sargs, sm, (wi - offs[m]) * LY::G);
    __syncthreads();  // the item is done with sargs, sitem and the tiles
  }
}

#ifndef SHIELD_PREFETCH_INPUTS_ONLY
#define SHIELD_PREFETCH_INPUTS_ONLY 0
#endif

// Launch the step over ceil(ncol / G) column blocks. PERSIST: as many
// persistent, double-buffered blocks as fit on the device at once, each
// walking every gridDim.x-th column block; else one block per column block,
// scheduled by the hardware.
template <class LY, int MINB, bool MIXED, bool PERSIST, bool FLAGS = false>
cudaError_t launch_step(const MpArgs& A, cudaStream_t st) {
  constexpr int G = LY::G;
  const int64_t nblk = (A.ncol + G - 1) / G;
  const int threads = LY::THREADS;
  if (PERSIST) {
    // the old tendencies join the prefetch where both buffers have room
    constexpr bool kTend = SmemP<LY, N_TILE>::bytes <= 220 * 1024 && !SHIELD_PREFETCH_INPUTS_ONLY;
    constexpr int NT = kTend ? N_TILE : N_IN;
    auto kern = mp_step_persistent_kernel<LY, MINB, MIXED, NT>;
    const size_t smem = SmemP<LY, NT>::bytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int64_t resident = (int64_t)nsm * per_sm;
    const int64_t grid = nblk < resident ? nblk : resident;
    kern<<<(unsigned)grid, threads, smem, st>>>(A, nblk);
    return cudaGetLastError();
  }
  auto kern = mp_step_kernel<LY, MINB, MIXED, FLAGS>;
  const size_t smem = Smem<LY>::bytes;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)nblk, threads, smem, st>>>(A);
  return cudaGetLastError();
}

// Launch shape of 65..80 levels (L79): two columns on each group of 5 warps
// (PackedLayout), SHIELD_PACK_NGRP groups per block, __launch_bounds__
// minimum SHIELD_PACK_MINB blocks per SM. Every launch of this level range
// (plain, mixed, flag-recording, ensemble) packs two columns per 5 warps,
// so a column's arithmetic, and with it its rounding, is the same in all.
// Measured at C96 L79 (ms per step, plain / mixed; the register cap is
// 65,536 / threads): 2 groups (320 threads, 168 registers) 5.70 / 4.23,
// 3 groups (480, 128 with spills) 4.16 / 3.17, 4 groups (640, 96 with spills)
// 3.65 / 2.50, 5 groups 4.09 / 2.61, 6 groups 3.81 / 2.65; one column per 3
// warps, 4 columns per block (12 warps, 160 registers) was 5.66 / 3.65. The
// step is bound by the latency of dependent FP64 work, so resident warps
// count for more than spilled registers.
#ifndef SHIELD_PACK_NGRP
#define SHIELD_PACK_NGRP 4
#endif
#ifndef SHIELD_PACK_MINB
#define SHIELD_PACK_MINB 1
#endif
#ifndef SHIELD_PACK_NWG
#define SHIELD_PACK_NWG 5
#endif
#ifndef SHIELD_PACK_P
#define SHIELD_PACK_P 2
#endif
using Packed80 = PackedLayout<SHIELD_PACK_NWG, SHIELD_PACK_P, SHIELD_PACK_NGRP>;
constexpr int PACK80_MINB = SHIELD_PACK_MINB;
constexpr int PACK80_LMIN = 65, PACK80_LMAX = 80;

// Launch of the ensemble kernel with `grid` persistent blocks; `counter`
// (one word) is zeroed on `st` first.
template <class LY, int MINB, bool MIXED>
cudaError_t launch_ensemble(const MpArgs* members, const int64_t* offs, int nm, unsigned long long* counter, int grid,
                            cudaStream_t st) {
  const size_t smem = Smem<LY>::bytes;
  auto kern = mp_ensemble_kernel<LY, MINB, MIXED>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  kern<<<grid, LY::THREADS, smem, st>>>(members, offs, nm, counter);
  return cudaGetLastError();
}

}  // namespace shield
