// A-grid to D-grid update of the physics wind tendencies (compiled with
// -fmad=false): pySHiELD's AGrid2DGridPhysics, update_dwind_phys.py:12-161
// (stencils) and :171-701 (their domains and order).
//
// The reference runs a prep stencil that turns the A-grid tendencies into
// three Cartesian components averaged onto the D-grid edges (ue, ve), zeroes
// the tendencies, applies up to eight cube-edge corrections to ue and ve, and
// adds dt/2 (ue . es1) to u and dt/2 (ve . ew2) to v. Here a block computes
// the A-grid vectors of a tile once into shared memory, and each D-grid
// point of the tile forms its own ue or ve from them (the corrections read
// the original ue / ve of a neighbour, which the point forms too), so no
// ue / ve / ut / vt field is stored; a second launch then zeroes the
// tendencies on the prep domain, after every read of them. Each expression
// keeps the reference's operand order.
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

// The zeroing and doubly periodic kernels run over rows: blockIdx.x * DW_BX
// + threadIdx.x is i along a storage line and blockIdx.y walks the (j, k)
// lines, so the index arithmetic is 32-bit and a line's accesses are
// coalesced in the i-fastest layout. At most 65,535 block rows; a loop over
// rows covers the rest.
constexpr int DW_BX = 128;

dim3 row_grid(int len, int64_t rows) {
  return dim3((unsigned)((len + DW_BX - 1) / DW_BX), (unsigned)(rows < 65535 ? (rows > 0 ? rows : 1) : 65535));
}

// The update kernel works on tiles: a block owns DT_X x DT_Y D-grid points
// (i, j) over DT_K consecutive levels. The A-grid vectors v3 = udt vlon +
// vdt vlat (update_dwind_prep_stencil) that its points average lie in
// i0 - 1 .. i0 + DT_X, j0 - 1 .. j0 + DT_Y (the corrections read one more
// point in i or j); the block loads their geometry once and, level by level,
// computes each v3 once into shared memory, where the u and v points of the
// level read it. Only A points in the prep domain [-1, nx] x [-1, ny] are
// touched: every read of a D point lies there.
// 16 levels per block measured the same as 8 (0.111 ms); 4 slower (0.128).
constexpr int DT_X = 32, DT_Y = 8, DT_K = 8;
constexpr int DW_MINB = 3;  // blocks per SM of the update kernels
constexpr int AT_X = DT_X + 2, AT_Y = DT_Y + 2;
// Levels per thread of the zeroing kernel.
constexpr int DW_KB = 4;

// update_uwind_stencil (j in [0, ny]) and update_vwind_stencil (i in [0, nx])
// with the cube-edge corrections of the x-edge (south, north) and y-edge
// (west, east) stencils, on one tile. Each expression keeps the reference's
// operand order; the loads of a level's u and v come before its stores.
// The edge-plan tests and the points' addresses are worked out once, before
// the level loop. The level loop is software-pipelined: the next level's
// udt, vdt, u and v loads are issued before this level's barrier, and v3
// alternates between two shared buffers, so one barrier per level orders
// the writes of a buffer after every read of it two levels before. Six C96
// tiles at L79 in one launch: 0.112 ms at three blocks per SM (80
// registers), 0.127 ms at four (64 registers, more spilled), 0.133 ms at
// two; 0.139 ms for the loop without the pipelining (load, barrier,
// compute, barrier per level) at four.
__device__ __forceinline__ void dwind_update_tile(const DwindArgs& A, int bx, int by, int bz) {
  __shared__ double g_lon[3][AT_Y][AT_X], g_lat[3][AT_Y][AT_X], v3b[2][3][AT_Y][AT_X];
  constexpr int NT = DT_X * DT_Y;
  constexpr int NA = (AT_X * AT_Y + NT - 1) / NT;  // A points per thread
  const int tx = threadIdx.x % DT_X, ty = threadIdx.x / DT_X;
  const int i0 = bx * DT_X, j0 = by * DT_Y, k0 = bz * DT_K;
  const int i = i0 + tx, j = j0 + ty;
  const int k1 = k0 + DT_K < A.nz ? k0 + DT_K : A.nz;
  // this thread's A points: their place in the tile, their geometry, and
  // their offsets in udt and vdt (level 0)
  int ax[NA], ay[NA];
  bool ain[NA];
  int64_t ou[NA], ov[NA];
#pragma unroll
  for (int n = 0; n < NA; ++n) {
    const int e = threadIdx.x + n * NT;
    ax[n] = e % AT_X;
    ay[n] = e / AT_X;
    const int ai = i0 - 1 + ax[n], aj = j0 - 1 + ay[n];
    ain[n] = e < AT_X * AT_Y && ai <= A.nx && aj <= A.ny;  // ai, aj >= -1 by construction
    ou[n] = ain[n] ? ai * A.udt.si + aj * A.udt.sj : 0;
    ov[n] = ain[n] ? ai * A.vdt.si + aj * A.vdt.sj : 0;
    if (ain[n]) {
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        g_lon[m][ay[n]][ax[n]] = A.vlon[m].at(ai, aj);
        g_lat[m][ay[n]][ax[n]] = A.vlat[m].at(ai, aj);
      }
    }
  }
  const bool up = i < A.nx && j <= A.ny, vp = i <= A.nx && j < A.ny;
  double e1[3], e2[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    e1[m] = up ? A.es1[m].at(i, j) : 0.0;
    e2[m] = vp ? A.ew2[m].at(i, j) : 0.0;
  }
  // the cube-edge corrections that apply to this point, in the reference's
  // order: regions q of the south then north lines (u), of the west then
  // east lines (v); at most two regions per line
  bool fu[4], fv[4];
  double cu[4], cv[4];
  int du[4], dv[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int su = t < 2 ? SOUTH : NORTH, sv = t < 2 ? WEST : EAST, q = t & 1;
    fu[t] = fv[t] = false;
    cu[t] = cv[t] = 0.0;
    du[t] = dv[t] = 0;
    if (up && q < A.plan.n[su]) {
      const ShieldEdgeRegion& R = A.plan.r[su][q];
      if (j == R.line && i >= R.lo && i < R.hi) {
        const double* ev = su == SOUTH ? A.ev_s : A.ev_n;
        fu[t] = true;
        cu[t] = ev[i * A.ev_stride];
        du[t] = R.dir;
      }
    }
    if (vp && q < A.plan.n[sv]) {
      const ShieldEdgeRegion& R = A.plan.r[sv][q];
      if (i == R.line && j >= R.lo && j < R.hi) {
        fv[t] = true;
        cv[t] = (sv == WEST ? A.ev_w : A.ev_e).at(i, j);
        dv[t] = R.dir;
      }
    }
  }
  const bool any_u = fu[0] || fu[1] || fu[2] || fu[3], any_v = fv[0] || fv[1] || fv[2] || fv[3];
  double* pu = A.u.p + (up ? i * A.u.si + j * A.u.sj : 0);
  double* pv = A.v.p + (vp ? i * A.v.si + j * A.v.sj : 0);
  // level k0's loads
  double ut[NA], vt[NA];
#pragma unroll
  for (int n = 0; n < NA; ++n) {
    ut[n] = ain[n] ? A.udt.p[ou[n] + k0 * A.udt.sk] : 0.0;
    vt[n] = ain[n] ? A.vdt.p[ov[n] + k0 * A.vdt.sk] : 0.0;
  }
  double un = up && k0 < k1 ? pu[k0 * A.u.sk] : 0.0, vn = vp && k0 < k1 ? pv[k0 * A.v.sk] : 0.0;
  __syncthreads();
  for (int k = k0; k < k1; ++k) {
    double(*v3s)[AT_Y][AT_X] = v3b[(k - k0) & 1];
#pragma unroll
    for (int n = 0; n < NA; ++n) {
      if (!ain[n]) continue;
#pragma unroll
      for (int m = 0; m < 3; ++m)
        v3s[m][ay[n]][ax[n]] = ut[n] * g_lon[m][ay[n]][ax[n]] + vt[n] * g_lat[m][ay[n]][ax[n]];
    }
    const double uk = un, vk = vn;
    if (k + 1 < k1) {
#pragma unroll
      for (int n = 0; n < NA; ++n) {
        if (!ain[n]) continue;
        ut[n] = A.udt.p[ou[n] + (k + 1) * A.udt.sk];
        vt[n] = A.vdt.p[ov[n] + (k + 1) * A.vdt.sk];
      }
      if (up) un = pu[(k + 1) * A.u.sk];
      if (vp) vn = pv[(k + 1) * A.v.sk];
    }
    __syncthreads();
    // A point (ai, aj) sits at v3s[.][aj - j0 + 1][ai - i0 + 1]
    if (up) {
      // ue = v3(i, j - 1) + v3(i, j); a correction's neighbour is at i + dir
      double w[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) w[m] = v3s[m][ty][tx + 1] + v3s[m][ty + 1][tx + 1];
      if (any_u) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          if (!fu[t]) continue;
          const int x = tx + 1 + du[t];
#pragma unroll
          for (int m = 0; m < 3; ++m) w[m] = cu[t] * (v3s[m][ty][x] + v3s[m][ty + 1][x]) + (1.0 - cu[t]) * w[m];
        }
      }
      pu[k * A.u.sk] = uk + A.dt5 * (w[0] * e1[0] + w[1] * e1[1] + w[2] * e1[2]);
    }
    if (vp) {
      // ve = v3(i - 1, j) + v3(i, j); a correction's neighbour is at j + dir
      double w[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) w[m] = v3s[m][ty + 1][tx] + v3s[m][ty + 1][tx + 1];
      if (any_v) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          if (!fv[t]) continue;
          const int y = ty + 1 + dv[t];
#pragma unroll
          for (int m = 0; m < 3; ++m) w[m] = cv[t] * (v3s[m][y][tx] + v3s[m][y][tx + 1]) + (1.0 - cv[t]) * w[m];
        }
      }
      pv[k * A.v.sk] = vk + A.dt5 * (w[0] * e2[0] + w[1] * e2[1] + w[2] * e2[2]);
    }
  }
}

__global__ void __launch_bounds__(DT_X * DT_Y, DW_MINB) dwind_update_kernel(const __grid_constant__ DwindArgs A) {
  dwind_update_tile(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Several tiles (the ranks' subtiles a GPU holds, at most DW_MAXT) in one
// launch: blockIdx.z is (tile, level block); a tile smaller than the grid's
// largest leaves the blocks beyond its points idle.
constexpr int DW_MAXT = 6;  // the batch kernels' switches name tiles 0 .. 5
struct DwindBatch {
  DwindArgs t[DW_MAXT];
  int n, nkz;
};

// One tile of the batch; T is a compile-time index, so that every read of
// the tile's arguments is a fixed offset into the kernel parameters.
template <int T>
__device__ __forceinline__ void dwind_update_batch_tile(const DwindBatch& B) {
  const DwindArgs& A = B.t[T];
  const int bz = blockIdx.z % B.nkz;
  if ((int)blockIdx.x * DT_X > A.nx || (int)blockIdx.y * DT_Y > A.ny || bz * DT_K >= A.nz) return;
  dwind_update_tile(A, blockIdx.x, blockIdx.y, bz);
}

__global__ void __launch_bounds__(DT_X * DT_Y, DW_MINB) dwind_update_batch_kernel(const __grid_constant__ DwindBatch B) {
  switch (blockIdx.z / B.nkz) {
    case 0: dwind_update_batch_tile<0>(B); break;
    case 1: dwind_update_batch_tile<1>(B); break;
    case 2: dwind_update_batch_tile<2>(B); break;
    case 3: dwind_update_batch_tile<3>(B); break;
    case 4: dwind_update_batch_tile<4>(B); break;
    case 5: dwind_update_batch_tile<5>(B); break;
    default: break;
  }
}

// set_winds_zero on the prep domain: i, j in [-1, n + 1), DW_KB levels per thread
__device__ __forceinline__ void dwind_zero_tile(const DwindArgs& A) {
  const int i = blockIdx.x * DW_BX + threadIdx.x - 1;
  if (i > A.nx) return;
  const int nkb = (A.nz + DW_KB - 1) / DW_KB;
  const int nrow = (A.ny + 2) * nkb;
  for (int r = blockIdx.y; r < nrow; r += gridDim.y) {
    const int j = r % (A.ny + 2) - 1, k0 = (r / (A.ny + 2)) * DW_KB;
#pragma unroll
    for (int b = 0; b < DW_KB; ++b) {
      if (k0 + b >= A.nz) continue;
      A.udt.at(i, j, k0 + b) = 0.0;
      A.vdt.at(i, j, k0 + b) = 0.0;
    }
  }
}

__global__ void dwind_zero_kernel(const __grid_constant__ DwindArgs A) { dwind_zero_tile(A); }

// every tile of a batch: blockIdx.z is the tile
__global__ void dwind_zero_batch_kernel(const __grid_constant__ DwindBatch B) {
  switch (blockIdx.z) {
    case 0: dwind_zero_tile(B.t[0]); break;
    case 1: dwind_zero_tile(B.t[1]); break;
    case 2: dwind_zero_tile(B.t[2]); break;
    case 3: dwind_zero_tile(B.t[3]); break;
    case 4: dwind_zero_tile(B.t[4]); break;
    case 5: dwind_zero_tile(B.t[5]); break;
    default: break;
  }
}

// doubly_periodic_wind_update (update_dwind_phys.py:153-161) on the compute domain
__global__ void dwind_periodic_kernel(const __grid_constant__ DwindArgs A) {
  const int i = blockIdx.x * DW_BX + threadIdx.x;
  if (i >= A.nx) return;
  const int nrow = A.ny * A.nz;
  for (int r = blockIdx.y; r < nrow; r += gridDim.y) {
    const int j = r % A.ny, k = r / A.ny;
    const double u0 = A.u.at(i, j, k), ua = A.udt.at(i, j - 1, k), ub = A.udt.at(i, j, k);
    const double v0 = A.v.at(i, j, k), va = A.vdt.at(i - 1, j, k), vb = A.vdt.at(i, j, k);
    A.u.at(i, j, k) = u0 + A.dt5 * (ua + ub);
    A.v.at(i, j, k) = v0 + A.dt5 * (va + vb);
  }
}

F3 mk3(const ShieldField3D& f) { return F3{f.ptr, f.si, f.sj, f.sk}; }
F2 mk2(const ShieldField2D& f) { return F2{f.ptr, f.si, f.sj}; }


// Checked kernel arguments of one tile; the message names the entry point.
int make_args(const char* who, int nx, int ny, int nz, int grid_type, double dt5, const ShieldEdgePlan* plan,
              const ShieldDwindGeometry* g, ShieldField3D u, ShieldField3D v, ShieldField3D u_dt, ShieldField3D v_dt,
              DwindArgs& A) {
  const std::string w(who);
  if (nx < 1 || ny < 1 || nz < 1 || !u.ptr || !v.ptr || !u_dt.ptr || !v_dt.ptr) {
    shield::set_last_error(w + ": bad arguments");
    return SHIELD_EINVAL;
  }
  if ((int64_t)(ny + 2) * nz > INT32_MAX || nx > INT32_MAX - 2 * DW_BX) {
    shield::set_last_error(w + ": domain too large for 32-bit row indices");
    return SHIELD_ELAYOUT;
  }
  A = DwindArgs{};
  A.u = mk3(u);
  A.v = mk3(v);
  A.udt = mk3(u_dt);
  A.vdt = mk3(v_dt);
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.dt5 = dt5;
  if (grid_type > 3) return SHIELD_OK;
  if (!plan || !g) {
    shield::set_last_error(w + ": the cube-sphere update needs the edge plan and the geometry");
    return SHIELD_EINVAL;
  }
  for (int s = 0; s < 4; ++s) {
    if (plan->n[s] < 0 || plan->n[s] > 2) {
      shield::set_last_error(w + ": at most two regions per edge");
      return SHIELD_EINVAL;
    }
  }
  const ShieldField2D* geo[14] = {&g->vlon1, &g->vlon2, &g->vlon3, &g->vlat1, &g->vlat2, &g->vlat3, &g->es1_1,
                                  &g->es1_2, &g->es1_3, &g->ew2_1, &g->ew2_2, &g->ew2_3, &g->edge_vect_w,
                                  &g->edge_vect_e};
  for (int q = 0; q < 14; ++q) {
    if (!geo[q]->ptr) {
      shield::set_last_error(w + ": null geometry field " + std::to_string(q));
      return SHIELD_EINVAL;
    }
  }
  if (!g->edge_vect_s || !g->edge_vect_n) {
    shield::set_last_error(w + ": null edge_vect_s / edge_vect_n");
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
  return SHIELD_OK;
}

}  // namespace

extern "C" int shield_agrid_to_dgrid(int nx, int ny, int nz, int grid_type, double dt5, const ShieldEdgePlan* plan,
                                     const ShieldDwindGeometry* g, ShieldField3D u, ShieldField3D v,
                                     ShieldField3D u_dt, ShieldField3D v_dt, void* stream) {
  DwindArgs A;
  int rc = make_args("shield_agrid_to_dgrid", nx, ny, nz, grid_type, dt5, plan, g, u, v, u_dt, v_dt, A);
  if (rc != SHIELD_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (grid_type > 3) {
    dwind_periodic_kernel<<<row_grid(nx, (int64_t)ny * nz), DW_BX, 0, st>>>(A);
    e = cudaGetLastError();
  } else {
    const dim3 tiles((unsigned)((nx + DT_X) / DT_X), (unsigned)((ny + DT_Y) / DT_Y), (unsigned)((nz + DT_K - 1) / DT_K));
    dwind_update_kernel<<<tiles, DT_X * DT_Y, 0, st>>>(A);
    const int64_t nkb = (nz + DW_KB - 1) / DW_KB;
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      dwind_zero_kernel<<<row_grid(nx + 2, (int64_t)(ny + 2) * nkb), DW_BX, 0, st>>>(A);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_agrid_to_dgrid: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}

extern "C" int shield_agrid_to_dgrid_tiles(int ntiles, const ShieldDwindTile* tiles, void* stream) {
  if (ntiles < 1 || ntiles > DW_MAXT || !tiles) {
    shield::set_last_error("shield_agrid_to_dgrid_tiles: 1 to 6 tiles");
    return SHIELD_EINVAL;
  }
  DwindBatch B{};
  B.n = ntiles;
  int mx = 0, my = 0, mz = 0;
  for (int t = 0; t < ntiles; ++t) {
    const ShieldDwindTile& T = tiles[t];
    if (T.grid_type > 3) {
      shield::set_last_error("shield_agrid_to_dgrid_tiles: cube-sphere tiles only (grid_type <= 3)");
      return SHIELD_EINVAL;
    }
    int rc = make_args("shield_agrid_to_dgrid_tiles", T.nx, T.ny, T.nz, T.grid_type, T.dt5, &T.plan, &T.geometry,
                       T.u, T.v, T.u_dt, T.v_dt, B.t[t]);
    if (rc != SHIELD_OK) return rc;
    mx = T.nx > mx ? T.nx : mx;
    my = T.ny > my ? T.ny : my;
    mz = T.nz > mz ? T.nz : mz;
  }
  B.nkz = (mz + DT_K - 1) / DT_K;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid((unsigned)((mx + DT_X) / DT_X), (unsigned)((my + DT_Y) / DT_Y), (unsigned)(B.nkz * ntiles));
  dwind_update_batch_kernel<<<grid, DT_X * DT_Y, 0, st>>>(B);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    const int64_t nkb = (mz + DW_KB - 1) / DW_KB;
    const dim3 zg = row_grid(mx + 2, (int64_t)(my + 2) * nkb);
    dwind_zero_batch_kernel<<<dim3(zg.x, zg.y, (unsigned)ntiles), DW_BX, 0, st>>>(B);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    shield::set_last_error(std::string("shield_agrid_to_dgrid_tiles: ") + cudaGetErrorString(e));
    return SHIELD_ECUDA;
  }
  return SHIELD_OK;
}
