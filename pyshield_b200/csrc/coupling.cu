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
// is the dycore-to-physics copy. The
// other four are fused into one column-per-thread kernel that runs them in
// the reference's order, so that the updated vapour, delp, pt and tendencies
// pass from one stencil to the next in registers and L1 instead of HBM.
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

// One block row per (j, k) (or, with k fastest in memory, per (i, j)) line
// of the domain and the threads along the line's contiguous dimension: the
// index arithmetic is one 32-bit divide per row, and each point's loads are
// all issued before its stores.
struct Line {
  int64_t i, j, k;
};
__device__ __forceinline__ bool line_point(int kfast, int nx, int ny, int nz, int64_t row, int64_t t, Line& p) {
  if (kfast) {
    if (t >= nz) return false;
    p.k = t;
    p.i = row % nx;
    p.j = row / nx;
  } else {
    if (t >= nx) return false;
    p.i = t;
    p.j = row % ny;
    p.k = row / ny;
  }
  return true;
}

__global__ void update_physics_state_kernel(const __grid_constant__ UpdArgs A) {
  const int64_t rows = A.kfast ? (int64_t)A.nx * A.ny : (int64_t)A.ny * A.nz;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t row = blockIdx.y; row < rows; row += gridDim.y) {
    Line q;
    if (!line_point(A.kfast, A.nx, A.ny, A.nz, row, t, q)) continue;
    double x[10], d[10];
#pragma unroll
    for (int p = 0; p < 10; ++p) {
      x[p] = A.x[p].at(q.i, q.j, q.k);
      d[p] = A.t[p].at(q.i, q.j, q.k);
    }
#pragma unroll
    for (int p = 0; p < 10; ++p) A.o[p].at(q.i, q.j, q.k) = x[p] + d[p] * A.dt;
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

__global__ void update_atmos_state_kernel(const __grid_constant__ AtmArgs A) {
  const int nxf = A.nx + 2 * A.hx, nyf = A.ny + 2 * A.hx;
  const int64_t ncf = (int64_t)nxf * nyf;
  const int nk = A.nz + 1;  // the reference builds these stencils on nz + 1 levels
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncf; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c % nxf - A.hx, j = c / nxf - A.hx;
    // ---- fill_gfs_delp(delp, physics_updated_specific_humidity, 1e-9) on the full domain
    const bool dycore_only = (A.mode & SHIELD_UAS_DYCORE_ONLY) != 0;
    {
      const F3& q = dycore_only ? A.f[D_QV] : A.f[PU_QV];
      const F3& dp = A.f[D_DELP];
      const double q_min = 1.0e-9;
      double qn = q.at(i, j, nk - 2);  // BACKWARD interval(0, -2): reads the updated level below
      double dpn = dp.at(i, j, nk - 2);
      for (int k = nk - 3; k >= 0; --k) {
        double qk = q.at(i, j, k);
        const double dpk = dp.at(i, j, k);
        if (qn < q_min) qk = qk + (qn - q_min) * dpn / dpk;
        q.at(i, j, k) = qk;
        qn = qk;
        dpn = dpk;
      }
      // PARALLEL interval(1, -1) clamp, FORWARD interval(1, -1) borrow, FORWARD interval(0, -1) zero
      double qprev = q.at(i, j, 0);  // level 0 is neither clamped nor borrowed into
      double dprev = dp.at(i, j, 0);
      if (qprev < 0.0) q.at(i, j, 0) = 0.0;
      for (int k = 1; k < nk - 1; ++k) {
        double qk = q.at(i, j, k);
        const double dpk = dp.at(i, j, k);
        if (qk < q_min) qk = q_min;
        if (qprev < 0.0) qk = qk + qprev * (dprev) / (dpk);
        qprev = qk;
        dprev = dpk;
        q.at(i, j, k) = (qk < 0.0) ? 0.0 : qk;
      }
    }
    if (dycore_only || i < 0 || j < 0 || i >= A.nx || j >= A.ny) continue;
    // ---- prepare_tendencies_and_update_tracers, interval(0, -1) of nz + 1 levels
    const F3* f = A.f;
    double p_lo = f[PRSI].at(i, j, 0);
    for (int k = 0; k < nk - 1; ++k) {
      f[U_DT].at(i, j, k) = f[U_DT].at(i, j, k) + (f[U_T1].at(i, j, k) - f[U_T0].at(i, j, k)) * A.rdt;
      f[V_DT].at(i, j, k) = f[V_DT].at(i, j, k) + (f[V_T1].at(i, j, k) - f[V_T0].at(i, j, k)) * A.rdt;
      f[PT_DT].at(i, j, k) = f[PT_DT].at(i, j, k) + (f[PU_PT].at(i, j, k) - f[PT_T0].at(i, j, k)) * A.rdt;
      const double p_hi = f[PRSI].at(i, j, k + 1);
      const double dp = p_hi - p_lo;
      p_lo = p_hi;
      const double qwat_qv = dp * f[PU_QV].at(i, j, k);
      const double qwat_ql = dp * f[PU_QL].at(i, j, k);
      const double qwat_qr = dp * f[PU_QR].at(i, j, k);
      const double qwat_qs = dp * f[PU_QS].at(i, j, k);
      const double qwat_qi = dp * f[PU_QI].at(i, j, k);
      const double qwat_qg = dp * f[PU_QG].at(i, j, k);
      const double qt = qwat_qv + qwat_ql + qwat_qr + qwat_qs + qwat_qi + qwat_qg;
      const double q_sum = f[D_QV].at(i, j, k) + f[D_QL].at(i, j, k) + f[D_QR].at(i, j, k) + f[D_QS].at(i, j, k) +
                           f[D_QI].at(i, j, k) + f[D_QG].at(i, j, k);
      const double q0 = f[D_DELP].at(i, j, k) * (1.0 - q_sum) + qt;
      f[D_DELP].at(i, j, k) = q0;
      f[D_QV].at(i, j, k) = qwat_qv / q0;
      f[D_QL].at(i, j, k) = qwat_ql / q0;
      f[D_QR].at(i, j, k) = qwat_qr / q0;
      f[D_QS].at(i, j, k) = qwat_qs / q0;
      f[D_QI].at(i, j, k) = qwat_qi / q0;
      f[D_QG].at(i, j, k) = qwat_qg / q0;
    }
    if (!(A.mode & SHIELD_UAS_APPLY)) continue;
    // ---- moist_cv(dycore q..., dycore pt, t_dt = pt_dt, CP_AIR, dt) on nz + 1 levels
    for (int k = 0; k < nk; ++k) {
      const double ql = f[D_QL].at(i, j, k) + f[D_QR].at(i, j, k);
      const double qs = f[D_QI].at(i, j, k) + f[D_QS].at(i, j, k) + f[D_QG].at(i, j, k);
      const double gz = ql + qs;
      const double qv = f[D_QV].at(i, j, k);
      const double cvm = (1.0 - (qv + gz)) * A.CV_AIR + qv * A.CV_VAP + ql * A.C_LIQ + qs * A.C_ICE;
      f[D_PT].at(i, j, k) = f[D_PT].at(i, j, k) + f[PT_DT].at(i, j, k) * A.dt * A.cp_air / cvm;
      f[PT_DT].at(i, j, k) = 0.0;
    }
    // ---- update_pressure_and_surface_winds on nz + 1 levels
    double pe = f[PE].at(i, j, 0);
    for (int k = 1; k < nk; ++k) {
      pe = pe + f[D_DELP].at(i, j, k - 1);
      f[PE].at(i, j, k) = pe;
      const double peln = log(pe);
      f[PELN].at(i, j, k) = peln;
      f[PK].at(i, j, k) = exp(A.kappa * peln);
    }
    A.ps.at(i, j, 0) = pe;
    A.us.at(i, j, 0) = f[D_UA].at(i, j, nk - 2);
    A.vs.at(i, j, 0) = f[D_VA].at(i, j, nk - 2);
  }
}

// DycoreToPhysics' copy of 16 fields (update_atmos_state.py:95-142, built at
// :160-167 on the compute domain plus one interface point in x and y,
// PARALLEL interval(0, -1) of nz + 1 levels): one thread per point, the
// fastest-varying storage dimension on consecutive threads.
constexpr int N_D2P = 16;
struct D2PArgs {
  F3 in[N_D2P], out[N_D2P];
  int nx1, ny1, nz;  // the box: nx + 1, ny + 1, nz
  int kfast;
};

__global__ void copy_dycore_to_physics_kernel(const __grid_constant__ D2PArgs A) {
  const int64_t rows = A.kfast ? (int64_t)A.nx1 * A.ny1 : (int64_t)A.ny1 * A.nz;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t row = blockIdx.y; row < rows; row += gridDim.y) {
    Line q;
    if (!line_point(A.kfast, A.nx1, A.ny1, A.nz, row, t, q)) continue;
    double v[N_D2P];
#pragma unroll
    for (int p = 0; p < N_D2P; ++p) v[p] = A.in[p].at(q.i, q.j, q.k);
#pragma unroll
    for (int p = 0; p < N_D2P; ++p) A.out[p].at(q.i, q.j, q.k) = v[p];
  }
}

// 2-D launch over (line length, rows): 128 threads along a line, at most
// 65,535 block rows (a grid-stride loop covers the rest)
dim3 line_grid(int64_t len, int64_t rows) {
  const int64_t bx = (len + 127) / 128;
  return dim3((unsigned)bx, (unsigned)(rows < 65535 ? (rows > 0 ? rows : 1) : 65535));
}

int grid_for(int64_t n, int bs) {
  int64_t nb = (n + bs - 1) / bs;
  return (int)(nb < 148 * 32 ? (nb > 0 ? nb : 1) : 148 * 32);
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
  update_physics_state_kernel<<<line_grid(len, rows), 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
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
  update_atmos_state_kernel<<<grid_for(ncf, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
  cudaError_t e = cudaGetLastError();
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
  copy_dycore_to_physics_kernel<<<line_grid(len, rows), 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_copy_dycore_to_physics: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}
