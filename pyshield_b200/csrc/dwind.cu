// A-grid to D-grid update of the physics wind tendencies (compiled with
// -fmad=false): pySHiELD's AGrid2DGridPhysics, update_dwind_phys.py:12-161
// (stencils) and :171-701 (their domains and order).
//
// The reference runs a prep stencil that turns the A-grid tendencies into
// three Cartesian components averaged onto the D-grid edges (ue, ve), zeroes
// the tendencies, applies up to eight cube-edge corrections to ue and ve, and
// adds dt/2 (ue . es1) to u and dt/2 (ve . ew2) to v. Here one thread per
// (i, j, k) of the D-grid points computes its own ue or ve from the
// tendencies (the corrections read the original ue / ve of a neighbour,
// which the thread recomputes), so no ue / ve / ut / vt field is stored;
// a second launch then zeroes the tendencies on the prep domain, after every
// read of them. Each expression keeps the reference's operand order.
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
struct F2 {
  const double* p;
  int64_t si, sj;
  __device__ __forceinline__ double at(int64_t i, int64_t j) const { return p[i * si + j * sj]; }
};

enum { SOUTH = 0, NORTH, WEST, EAST };

struct DwindArgs {
  F3 u, v, udt, vdt;
  F2 vlon[3], vlat[3], es1[3], ew2[3], ev_w, ev_e;
  const double* ev_s;
  const double* ev_n;
  int64_t ev_stride;
  ShieldEdgePlan plan;
  int nx, ny, nz;
  double dt5;
};

struct Pt {
  const DwindArgs& A;
  int64_t k;
  __device__ __forceinline__ double v3(int m, int64_t i, int64_t j) const {
    return A.udt.at(i, j, k) * A.vlon[m].at(i, j) + A.vdt.at(i, j, k) * A.vlat[m].at(i, j);
  }
  // update_dwind_prep_stencil: ue = v3[0, -1, 0] + v3, ve = v3[-1, 0, 0] + v3
  __device__ __forceinline__ double ue(int m, int64_t i, int64_t j) const { return v3(m, i, j - 1) + v3(m, i, j); }
  __device__ __forceinline__ double ve(int m, int64_t i, int64_t j) const { return v3(m, i - 1, j) + v3(m, i, j); }
};

__global__ void dwind_update_kernel(const __grid_constant__ DwindArgs A) {
  const int64_t nb = (int64_t)(A.nx + 1) * (A.ny + 1) * A.nz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nb; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % (A.nx + 1);
    const int64_t r = e / (A.nx + 1);
    const int64_t j = r % (A.ny + 1), k = r / (A.ny + 1);
    const Pt P{A, k};
    if (i < A.nx) {
      // u point (update_uwind_stencil, j in [0, ny])
      double w[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) w[m] = P.ue(m, i, j);
      // update_dwind_x_edge_{west,east}_stencil on the south and north lines
#pragma unroll
      for (int s = SOUTH; s <= NORTH; ++s) {
        const double* ev = s == SOUTH ? A.ev_s : A.ev_n;
        for (int q = 0; q < A.plan.n[s]; ++q) {
          const ShieldEdgeRegion& R = A.plan.r[s][q];
          if (j != R.line || i < R.lo || i >= R.hi) continue;
          const double c = ev[i * A.ev_stride];
#pragma unroll
          for (int m = 0; m < 3; ++m) w[m] = c * P.ue(m, i + R.dir, j) + (1.0 - c) * w[m];
        }
      }
      A.u.at(i, j, k) = A.u.at(i, j, k) + A.dt5 * (w[0] * A.es1[0].at(i, j) + w[1] * A.es1[1].at(i, j) +
                                                   w[2] * A.es1[2].at(i, j));
    }
    if (j < A.ny) {
      // v point (update_vwind_stencil, i in [0, nx])
      double w[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) w[m] = P.ve(m, i, j);
      // update_dwind_y_edge_{south,north}_stencil on the west and east lines
#pragma unroll
      for (int s = WEST; s <= EAST; ++s) {
        const F2& ev = s == WEST ? A.ev_w : A.ev_e;
        for (int q = 0; q < A.plan.n[s]; ++q) {
          const ShieldEdgeRegion& R = A.plan.r[s][q];
          if (i != R.line || j < R.lo || j >= R.hi) continue;
          const double c = ev.at(i, j);
#pragma unroll
          for (int m = 0; m < 3; ++m) w[m] = c * P.ve(m, i, j + R.dir) + (1.0 - c) * w[m];
        }
      }
      A.v.at(i, j, k) = A.v.at(i, j, k) + A.dt5 * (w[0] * A.ew2[0].at(i, j) + w[1] * A.ew2[1].at(i, j) +
                                                   w[2] * A.ew2[2].at(i, j));
    }
  }
}

// set_winds_zero on the prep domain: i, j in [-1, n + 1)
__global__ void dwind_zero_kernel(const __grid_constant__ DwindArgs A) {
  const int64_t ni = A.nx + 2, nj = A.ny + 2;
  const int64_t nb = ni * nj * A.nz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nb; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % ni - 1;
    const int64_t r = e / ni;
    const int64_t j = r % nj - 1, k = r / nj;
    A.udt.at(i, j, k) = 0.0;
    A.vdt.at(i, j, k) = 0.0;
  }
}

// doubly_periodic_wind_update (update_dwind_phys.py:153-161) on the compute domain
__global__ void dwind_periodic_kernel(const __grid_constant__ DwindArgs A) {
  const int64_t nb = (int64_t)A.nx * A.ny * A.nz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nb; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % A.nx;
    const int64_t r = e / A.nx;
    const int64_t j = r % A.ny, k = r / A.ny;
    A.u.at(i, j, k) = A.u.at(i, j, k) + A.dt5 * (A.udt.at(i, j - 1, k) + A.udt.at(i, j, k));
    A.v.at(i, j, k) = A.v.at(i, j, k) + A.dt5 * (A.vdt.at(i - 1, j, k) + A.vdt.at(i, j, k));
  }
}

int grid_for(int64_t n, int bs) {
  int64_t nb = (n + bs - 1) / bs;
  return (int)(nb < 148 * 32 ? (nb > 0 ? nb : 1) : 148 * 32);
}

F3 mk3(const ShieldField3D& f) { return F3{f.ptr, f.si, f.sj, f.sk}; }
F2 mk2(const ShieldField2D& f) { return F2{f.ptr, f.si, f.sj}; }

}  // namespace

extern "C" int shield_agrid_to_dgrid(int nx, int ny, int nz, int grid_type, double dt5, const ShieldEdgePlan* plan,
                                     const ShieldDwindGeometry* g, ShieldField3D u, ShieldField3D v,
                                     ShieldField3D u_dt, ShieldField3D v_dt, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !u.ptr || !v.ptr || !u_dt.ptr || !v_dt.ptr) {
    shield::set_last_error("shield_agrid_to_dgrid: bad arguments");
    return SHIELD_EINVAL;
  }
  DwindArgs A{};
  A.u = mk3(u);
  A.v = mk3(v);
  A.udt = mk3(u_dt);
  A.vdt = mk3(v_dt);
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.dt5 = dt5;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (grid_type > 3) {
    dwind_periodic_kernel<<<grid_for((int64_t)nx * ny * nz, 256), 256, 0, st>>>(A);
    e = cudaGetLastError();
  } else {
    if (!plan || !g) {
      shield::set_last_error("shield_agrid_to_dgrid: the cube-sphere update needs the edge plan and the geometry");
      return SHIELD_EINVAL;
    }
    for (int s = 0; s < 4; ++s) {
      if (plan->n[s] < 0 || plan->n[s] > 2) {
        shield::set_last_error("shield_agrid_to_dgrid: at most two regions per edge");
        return SHIELD_EINVAL;
      }
    }
    const ShieldField2D* geo[14] = {&g->vlon1, &g->vlon2, &g->vlon3, &g->vlat1, &g->vlat2, &g->vlat3, &g->es1_1,
                                    &g->es1_2, &g->es1_3, &g->ew2_1, &g->ew2_2, &g->ew2_3, &g->edge_vect_w,
                                    &g->edge_vect_e};
    for (int q = 0; q < 14; ++q) {
      if (!geo[q]->ptr) {
        shield::set_last_error("shield_agrid_to_dgrid: null geometry field " + std::to_string(q));
        return SHIELD_EINVAL;
      }
    }
    if (!g->edge_vect_s || !g->edge_vect_n) {
      shield::set_last_error("shield_agrid_to_dgrid: null edge_vect_s / edge_vect_n");
      return SHIELD_EINVAL;
    }
    for (int m = 0; m < 3; ++m) {
      A.vlon[m] = mk2(*geo[m]);
      A.vlat[m] = mk2(*geo[3 + m]);
      A.es1[m] = mk2(*geo[6 + m]);
      A.ew2[m] = mk2(*geo[9 + m]);
    }
    A.ev_w = mk2(g->edge_vect_w);
    A.ev_e = mk2(g->edge_vect_e);
    A.ev_s = g->edge_vect_s;
    A.ev_n = g->edge_vect_n;
    A.ev_stride = g->edge_stride;
    A.plan = *plan;
    dwind_update_kernel<<<grid_for((int64_t)(nx + 1) * (ny + 1) * nz, 256), 256, 0, st>>>(A);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      dwind_zero_kernel<<<grid_for((int64_t)(nx + 2) * (ny + 2) * nz, 256), 256, 0, st>>>(A);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_agrid_to_dgrid: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}
