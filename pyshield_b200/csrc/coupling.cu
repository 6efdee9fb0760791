// Physics-to-dynamics column coupling kernels (compiled with -fmad=false).
//
//  * update_physics_state_with_tendencies  pySHiELD/stencils/physics.py:146-194
//  * fill_gfs_delp                         pySHiELD/update/update_atmos_state.py:21-37
//  * prepare_tendencies_and_update_tracers pySHiELD/update/update_atmos_state.py:40-92
//  * moist_cv                              pySHiELD/update/fv_update_phys.py:20-51
//  * update_pressure_and_surface_winds     pySHiELD/update/fv_update_phys.py:54-75
//  * copy_dycore_to_physics                pySHiELD/update/update_atmos_state.py:95-142
//
// All are HBM-streaming work. The first is elementwise (one thread per point,
// the fastest-varying storage dimension mapped to consecutive threads), as
// is the dycore-to-physics copy. The other four are fused into one kernel
// over tiles of columns that runs them in the reference's order, so that the
// updated vapour, delp, pt and tendencies pass from one stencil to the next
// in registers and shared memory instead of HBM.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/shield_mp.h"

namespace shield {
void set_last_error(const std::string& msg);
}

namespace {

struct F3 {
  double* p;
  int64_t si, sj, sk;
  __device__ __forceinline__ double& at(int64_t i, int64_t j, int64_t k) const { return p[i * si + j * sj + k * sk]; }
};

F3 mk(const ShieldField3D& f) { return F3{f.ptr, f.si, f.sj, f.sk}; }

struct UpdArgs {
  F3 x[10], t[10], o[10];
  int nx, ny, nz;
  int kfast;
  double dt;
};

// The two field kernels below work per field and per stretch of lines: a
// block handles one field (blockIdx.z) over LINES consecutive lines of the
// domain, a line being a (j, k) row (or, with k fastest in memory, an (i, j)
// column) whose points lie on consecutive threads. Its reads, then its
// writes, are contiguous stretches of a few storages instead of short lines
// of many, which keeps DRAM pages open. All of a block's loads are issued
// before its stores; index arithmetic is 32-bit (the entry points check the
// box).
constexpr int LINES = 8;
__device__ __forceinline__ void line_ijk(int kfast, int nx, int ny, int row, int t, int& i, int& j, int& k) {
  if (kfast) {
    k = t;
    i = row % nx;
    j = row / nx;
  } else {
    i = t;
    j = row % ny;
    k = row / ny;
  }
}

__global__ void update_physics_state_kernel(const __grid_constant__ UpdArgs A) {
  const int rows = A.kfast ? A.nx * A.ny : A.ny * A.nz;
  const int len = A.kfast ? A.nz : A.nx;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= len) return;
  const F3& X = A.x[blockIdx.z];
  const F3& T = A.t[blockIdx.z];
  const F3& O = A.o[blockIdx.z];
  for (int r0 = blockIdx.y * LINES; r0 < rows; r0 += gridDim.y * LINES) {
    double x[LINES], d[LINES];
    int64_t oo[LINES];
#pragma unroll
    for (int b = 0; b < LINES; ++b) {
      int i, j, k;
      line_ijk(A.kfast, A.nx, A.ny, r0 + b < rows ? r0 + b : rows - 1, t, i, j, k);
      x[b] = X.at(i, j, k);
      d[b] = T.at(i, j, k);
      oo[b] = i * O.si + j * O.sj + k * O.sk;
    }
#pragma unroll
    for (int b = 0; b < LINES; ++b)
      if (r0 + b < rows) O.p[oo[b]] = x[b] + d[b] * A.dt;
  }
}

enum {
  U_DT = 0, V_DT, PT_DT, U_T1, V_T1, PU_PT, PU_QV, PU_QL, PU_QR, PU_QS, PU_QI, PU_QG, U_T0, V_T0, PT_T0,
  D_QV, D_QL, D_QR, D_QS, D_QI, D_QG, PRSI, D_DELP, D_PT, PE, PELN, PK, D_UA, D_VA, N_ATM
};

struct AtmArgs {
  F3 f[N_ATM];
  F3 ps, us, vs;
  int nx, ny, nz, hx, mode;
  double rdt, dt, kappa, cp_air;
  double CV_AIR, CV_VAP, C_LIQ, C_ICE;
};

// The column stencils of UpdateAtmosphereState in one kernel. A block owns
// a tile of AT_TC = 32 consecutive columns of the full domain (lane =
// column: every level's accesses are coalesced in the i-fastest layout) and
// AT_NW warps that share its levels. The pointwise work runs
// level-parallel; the level-by-level recurrences run in one warp over
// shared-memory columns, in the reference's order:
//   1 (all warps)  the vapour and delp of every level into shared memory;
//   2 (one warp)   fill_gfs_delp's three sweeps;
//   3 (all warps)  the filled vapour back (full domain); on the compute
//                  domain prepare_tendencies_and_update_tracers and moist_cv
//                  level by level (moist_cv reads what prepare wrote at the
//                  same level); the new delp into shared memory;
//   4 (one warp)   update_pressure_and_surface_winds' pe sum;
//   5 (all warps)  pe, peln, pk.
// Four warps per block and 49 KB of shared memory let three or four blocks
// share an SM, so one block's loads overlap another's one-warp recurrences.
constexpr int AT_TC = 32;
constexpr int AT_NW = 4;

template <int NKMAX>
struct AtmSmem {
  double q[NKMAX][AT_TC];   // the vapour fill_gfs_delp works on
  double dp[NKMAX][AT_TC];  // the dycore delp it reads; then prepare's new
                            // delp (each level's thread replaces its own);
                            // then the interface pressure
};

template <int NKMAX>
__global__ void __launch_bounds__(AT_TC * AT_NW) update_atmos_state_kernel(const __grid_constant__ AtmArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  AtmSmem<NKMAX>& S = *reinterpret_cast<AtmSmem<NKMAX>*>(smem_raw);
  const int nxf = A.nx + 2 * A.hx, nyf = A.ny + 2 * A.hx;
  const int64_t ncf = (int64_t)nxf * nyf;
  const int nk = A.nz + 1;  // the reference builds these stencils on nz + 1 levels
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * AT_TC + lane;
  const bool live = c < ncf;
  const int64_t i = live ? c % nxf - A.hx : 0, j = live ? c / nxf - A.hx : 0;
  const bool compute = live && i >= 0 && j >= 0 && i < A.nx && j < A.ny;
  const bool dycore_only = (A.mode & SHIELD_UAS_DYCORE_ONLY) != 0;
  const bool apply = (A.mode & SHIELD_UAS_APPLY) != 0;
  const F3* f = A.f;
  const F3& Q = dycore_only ? f[D_QV] : f[PU_QV];
  const F3& DP = f[D_DELP];

  // ---- 1: fill_gfs_delp's inputs, levels 0 .. nk - 2
  for (int k = w; k < nk - 1; k += AT_NW) {
    if (live) {
      S.q[k][lane] = Q.at(i, j, k);
      S.dp[k][lane] = DP.at(i, j, k);
    }
  }
  __syncthreads();
  // ---- 2: fill_gfs_delp(delp, q, 1e-9) (update_atmos_state.py:21-37)
  if (w == 0 && live) {
    const double q_min = 1.0e-9;
    // BACKWARD interval(0, -2): borrow from the (updated) level below
    double qn = S.q[nk - 2][lane];
    double dpn = S.dp[nk - 2][lane];
    for (int k = nk - 3; k >= 0; --k) {
      double qk = S.q[k][lane];
      const double dpk = S.dp[k][lane];
      if (qn < q_min) qk = qk + (qn - q_min) * dpn / dpk;
      S.q[k][lane] = qk;
      qn = qk;
      dpn = dpk;
    }
    // PARALLEL interval(1, -1) clamp, FORWARD interval(1, -1) borrow, FORWARD
    // interval(0, -1) zero: the borrow chain runs on the unzeroed values
    double qprev = S.q[0][lane];
    double dprev = S.dp[0][lane];
    if (qprev < 0.0) S.q[0][lane] = 0.0;
    for (int k = 1; k < nk - 1; ++k) {
      double qk = S.q[k][lane];
      const double dpk = S.dp[k][lane];
      if (qk < q_min) qk = q_min;
      if (qprev < 0.0) qk = qk + qprev * (dprev) / (dpk);
      qprev = qk;
      dprev = dpk;
      S.q[k][lane] = (qk < 0.0) ? 0.0 : qk;
    }
  }
  __syncthreads();
  // ---- 3: the filled vapour; prepare_tendencies_and_update_tracers and moist_cv.
  // Every load of a level comes before its first store: the fields are
  // separate storages, but the compiler cannot know that, and a store
  // between two loads would make each group of loads wait for the last.
  for (int k = w; k < nk; k += AT_NW) {
    const bool filled = live && k < nk - 1;
    if (dycore_only || !compute) {
      if (filled) Q.at(i, j, k) = S.q[k][lane];
      continue;
    }
    const bool prep = k < nk - 1;
    // loads
    double dq[6];
    dq[0] = f[D_QV].at(i, j, k);
    dq[1] = f[D_QL].at(i, j, k);
    dq[2] = f[D_QR].at(i, j, k);
    dq[3] = f[D_QS].at(i, j, k);
    dq[4] = f[D_QI].at(i, j, k);
    dq[5] = f[D_QG].at(i, j, k);
    double pt_dt = f[PT_DT].at(i, j, k);
    const double pt = apply ? f[D_PT].at(i, j, k) : 0.0;
    double u_dt = 0.0, v_dt = 0.0, pq[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, dp = 0.0;
    if (prep) {
      u_dt = f[U_DT].at(i, j, k) + (f[U_T1].at(i, j, k) - f[U_T0].at(i, j, k)) * A.rdt;
      v_dt = f[V_DT].at(i, j, k) + (f[V_T1].at(i, j, k) - f[V_T0].at(i, j, k)) * A.rdt;
      pt_dt = pt_dt + (f[PU_PT].at(i, j, k) - f[PT_T0].at(i, j, k)) * A.rdt;
      dp = f[PRSI].at(i, j, k + 1) - f[PRSI].at(i, j, k);
      pq[0] = S.q[k][lane];
      pq[1] = f[PU_QL].at(i, j, k);
      pq[2] = f[PU_QR].at(i, j, k);
      pq[3] = f[PU_QS].at(i, j, k);
      pq[4] = f[PU_QI].at(i, j, k);
      pq[5] = f[PU_QG].at(i, j, k);
    }
    // prepare_tendencies_and_update_tracers, interval(0, -1)
    double q0 = 0.0;
    if (prep) {
      double qw[6];
      for (int t = 0; t < 6; ++t) qw[t] = dp * pq[t];
      const double qt = qw[0] + qw[1] + qw[2] + qw[3] + qw[4] + qw[5];
      const double q_sum = dq[0] + dq[1] + dq[2] + dq[3] + dq[4] + dq[5];
      q0 = S.dp[k][lane] * (1.0 - q_sum) + qt;  // the old delp, read before the store below
      for (int t = 0; t < 6; ++t) dq[t] = qw[t] / q0;
    }
    // moist_cv(dycore q..., dycore pt, t_dt = pt_dt, CP_AIR, dt), nz + 1 levels
    double pt_new = 0.0;
    if (apply) {
      const double ql = dq[1] + dq[2];
      const double qs = dq[4] + dq[3] + dq[5];
      const double gz = ql + qs;
      const double qv = dq[0];
      const double cvm = (1.0 - (qv + gz)) * A.CV_AIR + qv * A.CV_VAP + ql * A.C_LIQ + qs * A.C_ICE;
      pt_new = pt + pt_dt * A.dt * A.cp_air / cvm;
    }
    // stores
    if (filled) Q.at(i, j, k) = S.q[k][lane];
    if (prep) {
      f[U_DT].at(i, j, k) = u_dt;
      f[V_DT].at(i, j, k) = v_dt;
      f[D_DELP].at(i, j, k) = q0;
      S.dp[k][lane] = q0;
      f[D_QV].at(i, j, k) = dq[0];
      f[D_QL].at(i, j, k) = dq[1];
      f[D_QR].at(i, j, k) = dq[2];
      f[D_QS].at(i, j, k) = dq[3];
      f[D_QI].at(i, j, k) = dq[4];
      f[D_QG].at(i, j, k) = dq[5];
    }
    if (apply) {
      f[D_PT].at(i, j, k) = pt_new;
      f[PT_DT].at(i, j, k) = 0.0;
    } else if (prep) {
      f[PT_DT].at(i, j, k) = pt_dt;
    }
  }
  if (dycore_only || !apply) return;  // block-uniform: the mode is the launch's
  __syncthreads();
  // ---- 4: update_pressure_and_surface_winds' sum, pe[k] = pe[k - 1] + delp[k - 1]
  if (w == 0 && compute) {
    double pe = f[PE].at(i, j, 0);
    double dprev = S.dp[0][lane];
    for (int k = 1; k < nk; ++k) {
      pe = pe + dprev;
      dprev = k < nk - 1 ? S.dp[k][lane] : 0.0;
      S.dp[k][lane] = pe;
    }
  }
  __syncthreads();
  // ---- 5: pe, peln, pk on levels 1 .. nk - 1; ps and the surface winds
  for (int k = 1 + w; k < nk; k += AT_NW) {
    if (!compute) continue;
    const double pe = S.dp[k][lane];
    f[PE].at(i, j, k) = pe;
    const double peln = log(pe);
    f[PELN].at(i, j, k) = peln;
    f[PK].at(i, j, k) = exp(A.kappa * peln);
  }
  if (w == 0 && compute) {
    A.ps.at(i, j, 0) = S.dp[nk - 1][lane];
    A.us.at(i, j, 0) = f[D_UA].at(i, j, nk - 2);
    A.vs.at(i, j, 0) = f[D_VA].at(i, j, nk - 2);
  }
}

template <int NKMAX>
cudaError_t launch_atmos(const AtmArgs& A, int64_t ncf, cudaStream_t st) {
  const size_t smem = sizeof(AtmSmem<NKMAX>);
  auto kern = update_atmos_state_kernel<NKMAX>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)((ncf + AT_TC - 1) / AT_TC), AT_TC * AT_NW, smem, st>>>(A);
  return cudaGetLastError();
}

// DycoreToPhysics' copy of 16 fields (update_atmos_state.py:95-142, built at
// :160-167 on the compute domain plus one interface point in x and y,
// PARALLEL interval(0, -1) of nz + 1 levels), the fastest-varying storage
// dimension on consecutive threads.
constexpr int N_D2P = 16;
struct D2PArgs {
  F3 in[N_D2P], out[N_D2P];
  int nx1, ny1, nz;  // the box: nx + 1, ny + 1, nz
  int kfast;
};

// The copy, per field and stretch of lines as update_physics_state_kernel.
__global__ void copy_dycore_to_physics_kernel(const __grid_constant__ D2PArgs A) {
  const int rows = A.kfast ? A.nx1 * A.ny1 : A.ny1 * A.nz;
  const int len = A.kfast ? A.nz : A.nx1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= len) return;
  const F3& src = A.in[blockIdx.z];
  const F3& dst = A.out[blockIdx.z];
  for (int r0 = blockIdx.y * LINES; r0 < rows; r0 += gridDim.y * LINES) {
    double v[LINES];
    int64_t od[LINES];
#pragma unroll
    for (int b = 0; b < LINES; ++b) {
      int i, j, k;
      line_ijk(A.kfast, A.nx1, A.ny1, r0 + b < rows ? r0 + b : rows - 1, t, i, j, k);
      v[b] = src.at(i, j, k);
      od[b] = i * dst.si + j * dst.sj + k * dst.sk;
    }
#pragma unroll
    for (int b = 0; b < LINES; ++b)
      if (r0 + b < rows) dst.p[od[b]] = v[b];
  }
}

// 2-D launch over (line length, rows): 128 threads along a line, at most
// 65,535 block rows (a grid-stride loop covers the rest)
dim3 line_grid(int64_t len, int64_t rows) {
  const int64_t bx = (len + 127) / 128;
  return dim3((unsigned)bx, (unsigned)(rows < 65535 ? (rows > 0 ? rows : 1) : 65535));
}

}  // namespace

extern "C" int shield_update_physics_state(int nx, int ny, int nz, const ShieldField3D* state10,
                                           const ShieldField3D* tend10, const ShieldField3D* out10, double dt,
                                           void* stream) {
  if (!state10 || !tend10 || !out10 || nx < 1 || ny < 1 || nz < 1) {
    shield::set_last_error("shield_update_physics_state: bad arguments");
    return SHIELD_EINVAL;
  }
  UpdArgs A;
  for (int p = 0; p < 10; ++p) {
    if (!state10[p].ptr || !tend10[p].ptr || !out10[p].ptr) {
      shield::set_last_error("shield_update_physics_state: null field");
      return SHIELD_EINVAL;
    }
    A.x[p] = mk(state10[p]);
    A.t[p] = mk(tend10[p]);
    A.o[p] = mk(out10[p]);
  }
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.kfast = (state10[0].sk == 1) ? 1 : 0;
  A.dt = dt;
  const int64_t len = A.kfast ? nz : nx, rows = A.kfast ? (int64_t)nx * ny : (int64_t)ny * nz;
  if (rows * len > INT32_MAX) {
    shield::set_last_error("shield_update_physics_state: box too large for 32-bit indices");
    return SHIELD_ELAYOUT;
  }
  dim3 grid = line_grid(len, (rows + LINES - 1) / LINES);
  grid.z = 10;
  update_physics_state_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_update_physics_state: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}

extern "C" int shield_update_atmos_state(int nx, int ny, int nz, int hx, int mode, const ShieldField3D* f, ShieldField3D ps,
                                         ShieldField3D u_srf, ShieldField3D v_srf, double rdt, double dt, double kappa,
                                         double cp_air, void* stream) {
  if (!f || nx < 1 || ny < 1 || nz < 2 || hx < 0 || !ps.ptr || !u_srf.ptr || !v_srf.ptr) {
    shield::set_last_error("shield_update_atmos_state: bad arguments");
    return SHIELD_EINVAL;
  }
  if (nz > 128) {
    shield::set_last_error("shield_update_atmos_state: nz > 128 is not supported");
    return SHIELD_ELAYOUT;
  }
  AtmArgs A;
  for (int p = 0; p < N_ATM; ++p) {
    if (!f[p].ptr) {
      shield::set_last_error("shield_update_atmos_state: null field " + std::to_string(p));
      return SHIELD_EINVAL;
    }
    A.f[p] = mk(f[p]);
  }
  A.ps = mk(ps);
  A.us = mk(u_srf);
  A.vs = mk(v_srf);
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.hx = hx;
  A.mode = mode;
  A.rdt = rdt;
  A.dt = dt;
  A.kappa = kappa;
  A.cp_air = cp_air;
  // the constants of pyshield_b200/constants.py
  const double RVGAS = 461.50, RDGAS = 287.05, CP_AIR = 1004.6;
  A.CV_AIR = CP_AIR - RDGAS;
  A.CV_VAP = 3.0 * RVGAS;
  A.C_LIQ = 4.1855e3;
  A.C_ICE = 1972.0;
  const int64_t ncf = (int64_t)(nx + 2 * hx) * (ny + 2 * hx);
  const int nk = nz + 1;
  cudaError_t e = nk <= 96 ? launch_atmos<96>(A, ncf, static_cast<cudaStream_t>(stream))
                           : launch_atmos<129>(A, ncf, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_update_atmos_state: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}

extern "C" int shield_copy_dycore_to_physics(int nx, int ny, int nz, const ShieldField3D* dycore16,
                                             const ShieldField3D* physics16, void* stream) {
  if (!dycore16 || !physics16 || nx < 1 || ny < 1 || nz < 1) {
    shield::set_last_error("shield_copy_dycore_to_physics: bad arguments");
    return SHIELD_EINVAL;
  }
  D2PArgs A;
  for (int p = 0; p < N_D2P; ++p) {
    if (!dycore16[p].ptr || !physics16[p].ptr) {
      shield::set_last_error("shield_copy_dycore_to_physics: null field " + std::to_string(p));
      return SHIELD_EINVAL;
    }
    A.in[p] = mk(dycore16[p]);
    A.out[p] = mk(physics16[p]);
  }
  A.nx1 = nx + 1;
  A.ny1 = ny + 1;
  A.nz = nz;
  A.kfast = (physics16[0].sk == 1) ? 1 : 0;
  const int64_t len = A.kfast ? nz : A.nx1, rows = A.kfast ? (int64_t)A.nx1 * A.ny1 : (int64_t)A.ny1 * nz;
  if (rows * len > INT32_MAX) {
    shield::set_last_error("shield_copy_dycore_to_physics: box too large for 32-bit indices");
    return SHIELD_ELAYOUT;
  }
  dim3 grid = line_grid(len, (rows + LINES - 1) / LINES);
  grid.z = N_D2P;
  copy_dycore_to_physics_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_copy_dycore_to_physics: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}
