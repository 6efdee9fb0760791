// Physics driver pre-steps of pySHiELD's Physics.__call__ (compiled with
// -fmad=false), fused into one kernel:
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
// (physics.py:276-330). Here one block owns a tile of columns of the full
// domain and runs each column's part of all four (the layout of the work is
// described at the kernel). Halo columns run the get_prs_fv3 / get_phi_fv3
// part only, as the reference's full-domain stencils do.
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

// DycoreToPhysics' 16 fields, in its order (update_atmos_state.py:196-232)
enum {
  D_QV = 0, D_QL, D_QR, D_QS, D_QI, D_QG, D_QO3, D_TKE, D_QCLD, D_PT, D_DELP, D_DELZ, D_UA, D_VA, D_W, D_OMGA, N_D2P
};
// the D2P index of statein's tracer t (qvapor, qliquid, qrain, qice, qsnow,
// qgraupel, qo3mr); t is a compile-time index in the unrolled loops
__host__ __device__ constexpr int tracer_d2p(int t) {
  return t == 0 ? D_QV : t == 1 ? D_QL : t == 2 ? D_QR : t == 3 ? D_QI : t == 4 ? D_QS : t == 5 ? D_QG : D_QO3;
}

struct PhysArgs {
  F3 f[N_PHYS];
  // fused DycoreToPhysics copy (fused != 0): the dycore fields and their
  // physics-state destinations, in the D2P order
  F3 dsrc[N_D2P], ddst[N_D2P];
  int fused;
  int nx, ny, nz, hx;
  int nwat, prepare;
  double ptop, pk0inv, pktop;
  double GRAV, RGRAV, RDGAS, ZVIR, KAPPA, RDGAS_RGRAV;
};

// numpy's maximum/minimum for finite operands
__device__ __forceinline__ double np_max(double a, double b) { return a >= b ? a : b; }
__device__ __forceinline__ double np_min(double a, double b) { return a <= b ? a : b; }

// One block owns a tile of TC = 32 consecutive columns of the full domain
// (lane = column, so every level's loads and stores are coalesced in the
// i-fastest layout) and NWB warps that share its levels. The pointwise work
// runs level-parallel; the two running sums of each stencil pass (statein's
// interface geopotential and pressure, get_phi_fv3's geopotential) run in
// one warp, level by level in the reference's order, over shared-memory
// columns:
//   A  (all warps)  statein's pointwise prelude: delz * GRAV and the
//                   condensate-free thickness dpn of every level into shared
//                   memory (halo columns: their prsi and phii);
//   B  (two warps)  the sums: phii bottom up, prsi top down;
//   C  (all warps)  the rest of statein, get_prs_fv3, the first statement of
//                   get_phi_fv3 and the pointwise part of
//                   prepare_microphysics; del_gz into shared memory;
//   D  (one warp)   get_phi_fv3's bottom-up sum into shared memory; then
//      (all warps)  phii, del_gz, phil and prepare_microphysics' dz.
constexpr int TC = 32;
constexpr int NWB = 8;

template <int NKMAX>
struct PreSmem {
  double ph[NKMAX][TC];  // phase A: delz * GRAV; B: statein's phii
  double p[NKMAX][TC];   // phase A: dpn of the level above; B: prsi
  double gz[NKMAX][TC];  // phase C: get_phi_fv3's del_gz
};

// Two blocks (16 warps) per SM: the kernel waits on memory, so it needs the
// resident warps; the fused copy's extra loads would otherwise take the
// registers of the second block.
template <int NKMAX, bool FUSED>
__global__ void __launch_bounds__(TC * NWB, 2) physics_prestep_kernel(const __grid_constant__ PhysArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PreSmem<NKMAX>& S = *reinterpret_cast<PreSmem<NKMAX>*>(smem_raw);
  const int nxf = A.nx + 2 * A.hx, nyf = A.ny + 2 * A.hx;
  const int64_t ncf = (int64_t)nxf * nyf;
  const int nk = A.nz + 1;
  const F3* f = A.f;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * TC + lane;
  const bool live = c < ncf;
  const int64_t i = live ? c % nxf - A.hx : 0, j = live ? c / nxf - A.hx : 0;
  const bool compute = live && i >= 0 && j >= 0 && i < A.nx && j < A.ny;
  const bool halo = live && !compute;
  // With the fused copy, DycoreToPhysics' domain -- the compute domain plus
  // the interface points i = nx and j = ny, levels 0 .. nz - 1 -- is read
  // from the dycore storages (the values the copy would have left in the
  // physics ones) and copied into the physics storages; the halo columns of
  // that domain (the strip i = nx or j = ny) copy all 16 fields.
  const bool strip = FUSED && halo && i >= 0 && j >= 0 && i <= A.nx && j <= A.ny;
  auto rd = [&](int pf, int df, int k) -> double {
    if constexpr (FUSED) {
      if (k < A.nz && (compute || strip)) return A.dsrc[df].at(i, j, k);
    }
    return f[pf].at(i, j, k);
  };

  // ---- A: statein's prelude (PARALLEL interval(...)): tracers * delp, dpn
  for (int k = w; k < nk; k += NWB) {
    if (compute) {
      if constexpr (FUSED) {
        // the copied fields statein leaves alone, moved here where the
        // level loop has few loads of its own
        if (k < nk - 1) {
          const double cz = A.dsrc[D_DELZ].at(i, j, k), ca = A.dsrc[D_QCLD].at(i, j, k);
          const double cu = A.dsrc[D_UA].at(i, j, k), cv = A.dsrc[D_VA].at(i, j, k), cw = A.dsrc[D_W].at(i, j, k);
          A.ddst[D_DELZ].at(i, j, k) = cz;
          A.ddst[D_QCLD].at(i, j, k) = ca;
          A.ddst[D_UA].at(i, j, k) = cu;
          A.ddst[D_VA].at(i, j, k) = cv;
          A.ddst[D_W].at(i, j, k) = cw;
        }
      }
      if (k < nk - 1) S.ph[k][lane] = rd(DELZ, D_DELZ, k) * A.GRAV;
      const double dp0 = rd(DELP, D_DELP, k);
      double q[N_TRACER];
#pragma unroll
      for (int t = 0; t < N_TRACER; ++t) q[t] = rd(QV + t, tracer_d2p(t), k) * dp0;
      // q[1..5]: ql qr qi qs qg (the argument order qliquid, qrain, qice, qsnow, qgraupel)
      const double dpn = A.nwat == 6 ? dp0 - q[1] - q[2] - q[3] - q[4] - q[5] : dp0;
      if (k < nk - 1) {
        S.p[k + 1][lane] = dpn;
      } else {
        // the extra level: mass-weighted tracers and thickness, no division
#pragma unroll
        for (int t = 0; t < N_TRACER; ++t) f[QV + t].at(i, j, k) = q[t];
        f[DELP].at(i, j, k) = dpn;
      }
    } else if (halo) {
      S.p[k][lane] = f[PRSI].at(i, j, k);
      S.ph[k][lane] = f[PHII].at(i, j, k);
    }
  }
  __syncthreads();
  // ---- B: statein's running sums, in the reference's order (two warps)
  if (w == 0 && compute) {
    double ph = 0.0;
    S.ph[nk - 1][lane] = ph;
    for (int k = nk - 2; k >= 0; --k) {  // BACKWARD: phii[k] = phii[k + 1] - delz * GRAV
      ph = ph - S.ph[k][lane];
      S.ph[k][lane] = ph;
    }
  } else if (w == 1 && compute) {
    double p = A.ptop;  // FORWARD: prsi[k] = prsi[k - 1] + delp[k - 1]
    S.p[0][lane] = p;
    for (int k = 1; k < nk; ++k) {
      p = p + S.p[k][lane];
      S.p[k][lane] = p;
    }
  }
  __syncthreads();
  // ---- C: statein, get_prs_fv3, get_phi_fv3's first statement, prepare_microphysics' pointwise part.
  // Every load of a level comes before its first store: the fields are
  // separate storages, but the compiler cannot know that, and a store
  // between two loads would make each group of loads wait for the last.
  for (int k = w; k < nk; k += NWB) {
    if (compute) {
      const double p = S.p[k][lane];
      if (k == nk - 1) {
        f[PRSI].at(i, j, k) = p;
        f[PRSIK].at(i, j, k) = exp(A.KAPPA * log(p)) * A.pk0inv;
        continue;
      }
      // loads
      const double dp0 = rd(DELP, D_DELP, k);
      double q[N_TRACER];
#pragma unroll
      for (int t = 0; t < N_TRACER; ++t) q[t] = rd(QV + t, tracer_d2p(t), k);
      const double tke = rd(TKE, D_TKE, k);
      const double pt = rd(PT, D_PT, k);
      const double om = (A.prepare || FUSED) ? rd(OMGA, D_OMGA, k) : 0.0;
      // statein
      const double pn = S.p[k + 1][lane];
      const double ph_k = S.ph[k][lane], ph1 = S.ph[k + 1][lane];
#pragma unroll
      for (int t = 0; t < N_TRACER; ++t) q[t] = q[t] * dp0;
      const double dpn = A.nwat == 6 ? dp0 - q[1] - q[2] - q[3] - q[4] - q[5] : dp0;
#pragma unroll
      for (int t = 0; t < N_TRACER; ++t) q[t] = q[t] / dpn;
      const double qv = q[0];
      const double qgrs_rad = np_max(1.0e-10, qv);
      const double rTv = A.RDGAS * pt * (1.0 + A.ZVIR * qgrs_rad);
      const double dm = dpn;
      double d = dm * rTv / (ph_k - ph1);
      d = np_min(d, pn - 0.01 * dm);
      d = np_max(d, p + 0.01 * dm);
      const double tv = 1.0 + A.ZVIR * np_max(0.0, qv);
      const double gz = (ph_k - ph1) / (pt * tv);
      S.gz[k][lane] = gz * pt * tv;
      // stores
      f[PRSI].at(i, j, k) = p;
      f[PRSIK].at(i, j, k) = k == 0 ? A.pktop : log(p);
#pragma unroll
      for (int t = 0; t < N_TRACER; ++t) f[QV + t].at(i, j, k) = q[t];
      f[TKE].at(i, j, k) = tke / dpn;
      f[DM].at(i, j, k) = dm;
      f[DELP].at(i, j, k) = d;
      f[DELPRSI].at(i, j, k) = pn - p;
      if constexpr (FUSED) {
        A.ddst[D_PT].at(i, j, k) = pt;
        A.ddst[D_OMGA].at(i, j, k) = om;
      }
      if (A.prepare) {
        f[WMP].at(i, j, k) = -om * (1.0 + A.ZVIR * qv) * pt / d * A.RDGAS_RGRAV;
#pragma unroll
        for (int t = 0; t < 10; ++t)
          if (f[TEND0 + t].p) f[TEND0 + t].at(i, j, k) = 0.0;
      }
    } else if (halo && k < nk - 1) {
      const double pt = rd(PT, D_PT, k);
      const double qv = rd(QV, D_QV, k);
      if (FUSED && strip) {
        // DycoreToPhysics' copy of this interface column (a few columns:
        // one field at a time, to keep the registers for the compute path)
#pragma unroll 1
        for (int d = 0; d < N_D2P; ++d) A.ddst[d].at(i, j, k) = A.dsrc[d].at(i, j, k);
      }
      const double p = S.p[k][lane], pn = S.p[k + 1][lane];
      const double ph_k = S.ph[k][lane], ph1 = S.ph[k + 1][lane];
      const double tv = 1.0 + A.ZVIR * np_max(0.0, qv);
      f[DELPRSI].at(i, j, k) = pn - p;
      const double gz = (ph_k - ph1) / (pt * tv);
      S.gz[k][lane] = gz * pt * tv;
    }
  }
  __syncthreads();
  // ---- D: get_phi_fv3, BACKWARD: the sum phii[k] = phii[k + 1] + del_gz[k]
  // in one warp into shared memory (statein's phii there is no longer read),
  // then phii, del_gz, phil and prepare_microphysics' dz from all warps
  if (w == 0 && live) {
    double ph = 0.0;
    S.ph[nk - 1][lane] = ph;
    for (int k = nk - 2; k >= 0; --k) {
      const double phn = ph + S.gz[k][lane];
      S.ph[k][lane] = phn;
      ph = phn;
    }
  }
  __syncthreads();
  if (live) {
    const bool prep = compute && A.prepare;
    for (int k = w; k < nk; k += NWB) {
      if (k == nk - 1) {
        f[PHII].at(i, j, k) = 0.0;
        continue;
      }
      const double g = S.gz[k][lane];
      const double ph = S.ph[k + 1][lane], phn = S.ph[k][lane];
      f[DELGZ].at(i, j, k) = g;
      f[PHIL].at(i, j, k) = 0.5 * (ph + ph + g);
      f[PHII].at(i, j, k) = phn;
      if (prep) f[DZ].at(i, j, k) = (ph - phn) * A.RGRAV;
    }
  }
}

template <int NKMAX>
cudaError_t launch_prestep(const PhysArgs& A, int64_t ncf, cudaStream_t st) {
  const size_t smem = sizeof(PreSmem<NKMAX>);
  auto kern = A.fused ? physics_prestep_kernel<NKMAX, true> : physics_prestep_kernel<NKMAX, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t nblk = (ncf + TC - 1) / TC;
  kern<<<(unsigned)nblk, TC * NWB, smem, st>>>(A);
  return cudaGetLastError();
}

}  // namespace

namespace {

int prestep_impl(int nx, int ny, int nz, int hx, int nwat, double ptop, int flags, const ShieldPhysicsFields* fields,
                 const ShieldField3D* dycore16, const ShieldField3D* physics16, void* stream) {
  if (!fields || nx < 1 || ny < 1 || nz < 2 || hx < 0 || !(ptop > 0.0)) {
    shield::set_last_error("shield_physics_prestep: bad arguments");
    return SHIELD_EINVAL;
  }
  if (nz > 128) {
    shield::set_last_error("shield_physics_prestep: nz > 128 is not supported");
    return SHIELD_ELAYOUT;
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
  A.fused = 0;
  if (dycore16 || physics16) {
    if (!dycore16 || !physics16 || hx < 1) {
      shield::set_last_error(
          "shield_physics_prestep_from_dycore: needs the 16 dycore and physics fields and a halo of at least 1");
      return SHIELD_EINVAL;
    }
    for (int d = 0; d < N_D2P; ++d) {
      if (!dycore16[d].ptr || !physics16[d].ptr) {
        shield::set_last_error("shield_physics_prestep_from_dycore: null copy field " + std::to_string(d));
        return SHIELD_EINVAL;
      }
      A.dsrc[d] = mk(dycore16[d]);
      A.ddst[d] = mk(physics16[d]);
    }
    A.fused = 1;
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
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nk = nz + 1;
  cudaError_t e = nk <= 96 ? launch_prestep<96>(A, ncf, st) : launch_prestep<129>(A, ncf, st);
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_physics_prestep: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}

}  // namespace

extern "C" int shield_physics_prestep(int nx, int ny, int nz, int hx, int nwat, double ptop, int flags,
                                      const ShieldPhysicsFields* fields, void* stream) {
  return prestep_impl(nx, ny, nz, hx, nwat, ptop, flags, fields, nullptr, nullptr, stream);
}

extern "C" int shield_physics_prestep_from_dycore(int nx, int ny, int nz, int hx, int nwat, double ptop, int flags,
                                                  const ShieldPhysicsFields* fields, const ShieldField3D* dycore16,
                                                  const ShieldField3D* physics16, void* stream) {
  if (!dycore16 || !physics16) {
    shield::set_last_error("shield_physics_prestep_from_dycore: null dycore or physics fields");
    return SHIELD_EINVAL;
  }
  return prestep_impl(nx, ny, nz, hx, nwat, ptop, flags, fields, dycore16, physics16, stream);
}
