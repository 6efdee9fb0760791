// Physics driver pre-steps of pySHiELD's Physics.__call__ (compiled with
// -fmad=false), fused into one column-per-thread kernel:
//
//  * atmos_phys_driver_statein  pySHiELD/stencils/physics.py:26-102
//                               (compute domain, nz + 1 levels)
//  * get_prs_fv3                pySHiELD/stencils/get_prs_fv3.py:7-20
//                               (full domain, nz + 1 levels)
//  * get_phi_fv3                pySHiELD/stencils/get_phi_fv3.py:7-25
//                               (full domain, nz + 1 levels)
//  * prepare_microphysics       pySHiELD/stencils/physics.py:105-143
//                               (compute domain, nz levels)
//
// The reference runs them as four stencils over HBM in this order
// (physics.py:276-330). Here one thread owns one column of the full domain
// and runs the column's part of each in three sweeps: a bottom-up sweep
// for statein's interface geopotential, a top-down sweep for the
// tracer/pressure conversion, statein's thickness and get_prs_fv3 (every
// level of these needs only the running interface pressure and the two
// geopotentials around it), and a bottom-up sweep for get_phi_fv3 and
// prepare_microphysics. Halo columns run the get_prs_fv3 / get_phi_fv3
// part only, as the reference's full-domain stencils do. Consecutive
// threads own consecutive i, so every level's loads and stores are
// coalesced in the i-fastest GT4Py layout.
//
// Each statement keeps the reference's operand order; the running sums
// (interface geopotential and pressure) are summed level by level in the
// reference's direction, so the results match the numpy backend to the
// last place except for log/exp.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
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

enum {
  PHII = 0, PRSI, PRSIK, DELZ, DELP, QV, QL, QR, QI, QS, QG, QO3, TKE, PT, DM, DELPRSI, DELGZ, PHIL, OMGA, DZ, WMP,
  TEND0, N_PHYS = TEND0 + 10
};
constexpr int N_TRACER = 7;  // qvapor .. qgraupel, qo3mr: statein's mass-weighted tracers

static_assert(sizeof(ShieldPhysicsFields) == N_PHYS * sizeof(ShieldField3D), "ShieldPhysicsFields layout");
static_assert(offsetof(ShieldPhysicsFields, qvapor) == QV * sizeof(ShieldField3D), "qvapor");
static_assert(offsetof(ShieldPhysicsFields, qo3mr) == QO3 * sizeof(ShieldField3D), "qo3mr");
static_assert(offsetof(ShieldPhysicsFields, del_gz) == DELGZ * sizeof(ShieldField3D), "del_gz");
static_assert(offsetof(ShieldPhysicsFields, wmp) == WMP * sizeof(ShieldField3D), "wmp");
static_assert(offsetof(ShieldPhysicsFields, pt_dt) == TEND0 * sizeof(ShieldField3D), "pt_dt");

struct PhysArgs {
  F3 f[N_PHYS];
  int nx, ny, nz, hx;
  int nwat, prepare;
  double ptop, pk0inv, pktop;
  double GRAV, RGRAV, RDGAS, ZVIR, KAPPA, RDGAS_RGRAV;
};

// numpy's maximum/minimum for finite operands
__device__ __forceinline__ double np_max(double a, double b) { return a >= b ? a : b; }
__device__ __forceinline__ double np_min(double a, double b) { return a <= b ? a : b; }

// Levels handled per batch of the sweeps: their loads are all issued before
// any of their results is stored, so they are in flight together (the
// stores could alias the loads as far as the compiler knows, which would
// otherwise serialise a level's loads behind the previous level's stores).
constexpr int U1 = 8;  // bottom-up geopotential sweep (one load per level)
constexpr int U2 = 2;  // top-down sweep (eleven loads per level)
constexpr int U3 = 8;  // bottom-up get_phi_fv3 sweep (one load per level)

__global__ void __launch_bounds__(64) physics_prestep_kernel(const __grid_constant__ PhysArgs A) {
  const int nxf = A.nx + 2 * A.hx, nyf = A.ny + 2 * A.hx;
  const int64_t ncf = (int64_t)nxf * nyf;
  const int nk = A.nz + 1;
  const F3* f = A.f;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncf; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c % nxf - A.hx, j = c / nxf - A.hx;
    const bool compute = i >= 0 && j >= 0 && i < A.nx && j < A.ny;
    if (compute) {
      // ---- statein, BACKWARD: phii = 0, then phii[k] = phii[k + 1] - delz * GRAV
      double ph = 0.0;
      f[PHII].at(i, j, nk - 1) = ph;
      for (int k0 = nk - 2; k0 >= 0; k0 -= U1) {
        double dz[U1];
#pragma unroll
        for (int u = 0; u < U1; ++u) dz[u] = k0 - u >= 0 ? f[DELZ].at(i, j, k0 - u) : 0.0;
#pragma unroll
        for (int u = 0; u < U1; ++u) {
          if (k0 - u < 0) break;
          ph = ph - dz[u] * A.GRAV;
          f[PHII].at(i, j, k0 - u) = ph;
        }
      }
      // ---- statein (tracers, pressure, thickness), get_prs_fv3, the first
      // statement of get_phi_fv3 and prepare_microphysics' pointwise part,
      // top down; levels 0 .. nk - 2 here, the extra level nk - 1 after
      double p = A.ptop;  // prsi[k]
      f[PRSI].at(i, j, 0) = p;
      double ph_k = f[PHII].at(i, j, 0);
      for (int k0 = 0; k0 < nk - 1; k0 += U2) {
        double dp0[U2], q[U2][N_TRACER], tke[U2], pt[U2], ph1[U2], om[U2];
#pragma unroll
        for (int u = 0; u < U2; ++u) {
          const int k = k0 + u < nk - 1 ? k0 + u : nk - 2;  // a repeated level is loaded but not used
          dp0[u] = f[DELP].at(i, j, k);
#pragma unroll
          for (int t = 0; t < N_TRACER; ++t) q[u][t] = f[QV + t].at(i, j, k);
          tke[u] = f[TKE].at(i, j, k);
          pt[u] = f[PT].at(i, j, k);
          ph1[u] = f[PHII].at(i, j, k + 1);
          om[u] = A.prepare ? f[OMGA].at(i, j, k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U2; ++u) {
          const int k = k0 + u;
          if (k >= nk - 1) break;
#pragma unroll
          for (int t = 0; t < N_TRACER; ++t) q[u][t] = q[u][t] * dp0[u];
          // q[u][1..5]: ql qr qi qs qg (the argument order qliquid, qrain, qice, qsnow, qgraupel)
          const double dpn =
              A.nwat == 6 ? dp0[u] - q[u][1] - q[u][2] - q[u][3] - q[u][4] - q[u][5] : dp0[u];
          const double pn = p + dpn;  // prsi[k + 1]
          f[PRSI].at(i, j, k + 1) = pn;
          f[PRSIK].at(i, j, k) = k == 0 ? A.pktop : log(p);
#pragma unroll
          for (int t = 0; t < N_TRACER; ++t) q[u][t] = q[u][t] / dpn;
#pragma unroll
          for (int t = 0; t < N_TRACER; ++t) f[QV + t].at(i, j, k) = q[u][t];
          f[TKE].at(i, j, k) = tke[u] / dpn;
          const double qgrs_rad = np_max(1.0e-10, q[u][0]);
          const double rTv = A.RDGAS * pt[u] * (1.0 + A.ZVIR * qgrs_rad);
          const double dm = dpn;
          f[DM].at(i, j, k) = dm;
          double d = dm * rTv / (ph_k - ph1[u]);
          d = np_min(d, pn - 0.01 * dm);
          d = np_max(d, p + 0.01 * dm);
          f[DELP].at(i, j, k) = d;
          // get_prs_fv3, then get_phi_fv3's first statement (PARALLEL interval(0, -1))
          f[DELPRSI].at(i, j, k) = pn - p;
          const double tv = 1.0 + A.ZVIR * np_max(0.0, q[u][0]);
          const double gz = (ph_k - ph1[u]) / (pt[u] * tv);
          f[DELGZ].at(i, j, k) = gz * pt[u] * tv;
          if (A.prepare) {
            // prepare_microphysics: wmp and the zeroed tendencies (pointwise;
            // dz needs get_phi_fv3's geopotential and follows below)
            f[WMP].at(i, j, k) = -om[u] * (1.0 + A.ZVIR * q[u][0]) * pt[u] / d * A.RDGAS_RGRAV;
#pragma unroll
            for (int t = 0; t < 10; ++t)
              if (f[TEND0 + t].p) f[TEND0 + t].at(i, j, k) = 0.0;
          }
          p = pn;
          ph_k = ph1[u];
        }
      }
      {
        // the extra level: mass-weighted tracers and thickness, no division
        const int k = nk - 1;
        const double dp0 = f[DELP].at(i, j, k);
        double q[N_TRACER];
#pragma unroll
        for (int t = 0; t < N_TRACER; ++t) q[t] = f[QV + t].at(i, j, k) * dp0;
        const double dpn = A.nwat == 6 ? dp0 - q[1] - q[2] - q[3] - q[4] - q[5] : dp0;
#pragma unroll
        for (int t = 0; t < N_TRACER; ++t) f[QV + t].at(i, j, k) = q[t];
        f[DELP].at(i, j, k) = dpn;
        f[PRSIK].at(i, j, k) = exp(A.KAPPA * log(p)) * A.pk0inv;
      }
    } else {
      // ---- halo column: get_prs_fv3 and get_phi_fv3's first statement
      double p = f[PRSI].at(i, j, 0);
      double ph_k = f[PHII].at(i, j, 0);
      for (int k0 = 0; k0 < nk - 1; k0 += U2) {
        double pn[U2], ph1[U2], pt[U2], qv[U2];
#pragma unroll
        for (int u = 0; u < U2; ++u) {
          const int k = k0 + u < nk - 1 ? k0 + u : nk - 2;
          pn[u] = f[PRSI].at(i, j, k + 1);
          ph1[u] = f[PHII].at(i, j, k + 1);
          pt[u] = f[PT].at(i, j, k);
          qv[u] = f[QV].at(i, j, k);
        }
#pragma unroll
        for (int u = 0; u < U2; ++u) {
          const int k = k0 + u;
          if (k >= nk - 1) break;
          const double tv = 1.0 + A.ZVIR * np_max(0.0, qv[u]);
          f[DELPRSI].at(i, j, k) = pn[u] - p;
          const double gz = (ph_k - ph1[u]) / (pt[u] * tv);
          f[DELGZ].at(i, j, k) = gz * pt[u] * tv;
          p = pn[u];
          ph_k = ph1[u];
        }
      }
    }
    // ---- get_phi_fv3, BACKWARD, and prepare_microphysics' dz on the compute domain
    double ph = 0.0;
    f[PHII].at(i, j, nk - 1) = ph;
    const bool prep = compute && A.prepare;
    for (int k0 = nk - 2; k0 >= 0; k0 -= U3) {
      double g[U3];
#pragma unroll
      for (int u = 0; u < U3; ++u) g[u] = k0 - u >= 0 ? f[DELGZ].at(i, j, k0 - u) : 0.0;
#pragma unroll
      for (int u = 0; u < U3; ++u) {
        const int k = k0 - u;
        if (k < 0) break;
        f[PHIL].at(i, j, k) = 0.5 * (ph + ph + g[u]);
        const double phn = ph + g[u];
        f[PHII].at(i, j, k) = phn;
        if (prep) f[DZ].at(i, j, k) = (ph - phn) * A.RGRAV;
        ph = phn;
      }
    }
  }
}

int grid_for(int64_t n, int bs) {
  int64_t nb = (n + bs - 1) / bs;
  return (int)(nb < 148 * 32 ? (nb > 0 ? nb : 1) : 148 * 32);
}

}  // namespace

extern "C" int shield_physics_prestep(int nx, int ny, int nz, int hx, int nwat, double ptop, int flags,
                                      const ShieldPhysicsFields* fields, void* stream) {
  if (!fields || nx < 1 || ny < 1 || nz < 2 || hx < 0 || !(ptop > 0.0)) {
    shield::set_last_error("shield_physics_prestep: bad arguments");
    return SHIELD_EINVAL;
  }
  const bool prepare = (flags & SHIELD_PHYS_PREPARE_MICROPHYSICS) != 0;
  const ShieldField3D* in = reinterpret_cast<const ShieldField3D*>(fields);
  PhysArgs A;
  for (int p = 0; p < N_PHYS; ++p) {
    const bool optional = p >= TEND0 || (!prepare && (p == OMGA || p == DZ || p == WMP));
    if (!in[p].ptr && !optional) {
      shield::set_last_error("shield_physics_prestep: null field " + std::to_string(p));
      return SHIELD_EINVAL;
    }
    A.f[p] = mk(in[p]);
  }
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.hx = hx;
  A.nwat = nwat;
  A.prepare = prepare ? 1 : 0;
  // Physics.__init__ / _setup_statein (physics.py:219-221, 270-274): p00 = 1e5
  const double p00 = 1.0e5;
  // the constants of pyshield_b200/constants.py
  A.GRAV = 9.80665;
  A.RGRAV = 1.0 / A.GRAV;
  A.RDGAS = 287.05;
  const double RVGAS = 461.50, CP_AIR = 1004.6;
  A.ZVIR = RVGAS / A.RDGAS - 1.0;
  A.KAPPA = A.RDGAS / CP_AIR;
  A.RDGAS_RGRAV = A.RDGAS * A.RGRAV;
  A.ptop = ptop;
  A.pktop = std::pow(ptop / p00, A.KAPPA);
  A.pk0inv = std::pow(1.0 / p00, A.KAPPA);
  const int64_t ncf = (int64_t)(nx + 2 * hx) * (ny + 2 * hx);
  physics_prestep_kernel<<<grid_for(ncf, 64), 64, 0, static_cast<cudaStream_t>(stream)>>>(A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_physics_prestep: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}
