// Plain FP64 form of the microphysics step. Compiled with -fmad=false so
// that every multiply and add rounds as the reference's numpy expressions do.
#include "mp_kernel.cuh"
#include "mp_launch.h"

namespace shield {

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


namespace {

template <int NW, int G, int MINB, bool FLAGS = false>
cudaError_t launch_nw(const MpArgs& A, cudaStream_t st) {
  return launch_step<ColumnLayout<NW, G>, MINB, false, false, FLAGS>(A, st);
}

__global__ void gather2d(const double* p, int64_t si, int64_t sj, int nx, int64_t n, double* out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    out[c] = p[(c % nx) * si + (c / nx) * sj];
}

}  // namespace

int mp_max_levels() { return 256; }

// Launch shape for 81-96 levels: columns per block and the minimum resident
// blocks per SM given to __launch_bounds__ (which caps the registers per
// thread). Four columns per block (one 384-thread block per SM) measured
// fastest: the staging then reads whole 32-byte sectors. 65-80 levels (L79)
// pack two columns per 5 warps (Packed80).
#ifndef SHIELD_NW3_G
#define SHIELD_NW3_G 4
#endif
#ifndef SHIELD_NW3_MINB
#define SHIELD_NW3_MINB 1
#endif
// 65..80 levels, plain form: the persistent, input-prefetching kernel (1) or
// one block per column block (0).
#ifndef SHIELD_PACK_PERSIST_PLAIN
#define SHIELD_PACK_PERSIST_PLAIN 0
#endif
// 97..128 levels (L127): columns per block of 4 warps each. C96 L127 (ms):
// 4 columns (512 threads, 128 registers) 6.29, 5 columns (640, 96) 5.94,
// 6 columns (768, 80) 5.99.
#ifndef SHIELD_NW4_G
#define SHIELD_NW4_G 5
#endif

cudaError_t mp_launch_plain(const MpArgs& A, cudaStream_t st) {
  const int L = A.nz;
  if (L <= 32) return launch_nw<1, 4, 2>(A, st);
  if (L <= 64) return launch_nw<2, 2, 2>(A, st);
  if (L <= PACK80_LMAX) return launch_step<Packed80, PACK80_MINB, false, SHIELD_PACK_PERSIST_PLAIN>(A, st);
  if (L <= 96) return launch_nw<3, SHIELD_NW3_G, SHIELD_NW3_MINB>(A, st);
  if (L <= 128) return launch_nw<4, SHIELD_NW4_G, 1>(A, st);
  return launch_nw<8, 1, 2>(A, st);
}

// The same launches with the column flags recorded (A.flags non-null).
cudaError_t mp_launch_plain_flags(const MpArgs& A, cudaStream_t st) {
  const int L = A.nz;
  if (L <= 32) return launch_nw<1, 4, 2, true>(A, st);
  if (L <= 64) return launch_nw<2, 2, 2, true>(A, st);
  if (L <= PACK80_LMAX) return launch_step<Packed80, PACK80_MINB, false, false, true>(A, st);
  if (L <= 96) return launch_nw<3, SHIELD_NW3_G, SHIELD_NW3_MINB, true>(A, st);
  if (L <= 128) return launch_nw<4, SHIELD_NW4_G, 1, true>(A, st);
  return launch_nw<8, 1, 2, true>(A, st);
}

cudaError_t mp_launch_mixed(const MpArgs& A, cudaStream_t st);

cudaError_t mp_launch_step(const MpArgs& A, int precision, cudaStream_t st) {
  if (precision == 1) return mp_launch_mixed(A, st);
  return mp_launch_plain(A, st);
}

cudaError_t mp_launch_de_ice(const MpArgs& A, Fld3 qi_dt, Fld3 qs_dt, cudaStream_t st) {
  const int64_t n = A.ncol * (int64_t)A.nz;
  const int64_t nb = (n + 255) / 256;
  de_ice_kernel<<<(unsigned)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, st>>>(A, qi_dt, qs_dt);
  return cudaGetLastError();
}

cudaError_t mp_gather_area(const double* p, int64_t si, int64_t sj, int nx, int ny, double* out) {
  const int64_t n = (int64_t)nx * ny;
  const int64_t nb = (n + 255) / 256;
  gather2d<<<(unsigned)(nb < 4096 ? nb : 4096), 256>>>(p, si, sj, nx, n, out);
  return cudaGetLastError();
}


// Ensemble launch over nz in (64, 128]: G columns per block, a persistent
// grid of `grid` blocks. 65..80 levels: G = 2, 4, 6 or 8 (1 to 4 groups of
// two packed columns; 640 threads per SM where the block size allows);
// 81..128 levels: G = 1, 2 or 4.
cudaError_t mp_launch_ensemble_plain(const MpArgs* members, const int64_t* offs, int nm, int nz, int G, int grid,
                                     unsigned long long* counter, cudaStream_t st) {
  if (nz <= PACK80_LMAX) {
    if (G == 2) return launch_ensemble<PackedLayout<5, 2, 1>, 4, false>(members, offs, nm, counter, grid, st);
    if (G == 4) return launch_ensemble<PackedLayout<5, 2, 2>, 2, false>(members, offs, nm, counter, grid, st);
    if (G == 6) return launch_ensemble<PackedLayout<5, 2, 3>, 1, false>(members, offs, nm, counter, grid, st);
    if (G == 8) return launch_ensemble<PackedLayout<5, 2, 4>, 1, false>(members, offs, nm, counter, grid, st);
  } else if (nz <= 96) {
    if (G == 1) return launch_ensemble<ColumnLayout<3, 1>, 4, false>(members, offs, nm, counter, grid, st);
    if (G == 2) return launch_ensemble<ColumnLayout<3, 2>, 2, false>(members, offs, nm, counter, grid, st);
    if (G == 4) return launch_ensemble<ColumnLayout<3, 4>, 1, false>(members, offs, nm, counter, grid, st);
  } else if (nz <= 128) {
    if (G == 1) return launch_ensemble<ColumnLayout<4, 1>, 4, false>(members, offs, nm, counter, grid, st);
    if (G == 2) return launch_ensemble<ColumnLayout<4, 2>, 2, false>(members, offs, nm, counter, grid, st);
    if (G == 4) return launch_ensemble<ColumnLayout<4, 4>, 1, false>(members, offs, nm, counter, grid, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace shield
