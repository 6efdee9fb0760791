// Mixed-precision form of the microphysics step: process rates in FP32,
// saturation adjustment, sedimentation, precipitation and every state
// update in FP64 (see mp_physics_mixed.cuh). FMA contraction is allowed here.
#include "mp_kernel.cuh"
#include "mp_launch.h"

namespace shield {

namespace {

template <int NW, int G, int MINB>
cudaError_t launch_nw(const MpArgs& A, cudaStream_t st) {
  return launch_step<NW, G, MINB, true, true>(A, st);
}

}  // namespace

cudaError_t mp_launch_mixed(const MpArgs& A, cudaStream_t st) {
  const int L = A.nz;
  if (L <= 32) return launch_nw<1, 4, 2>(A, st);
  if (L <= 64) return launch_nw<2, 2, 2>(A, st);
  if (L <= 96) return launch_nw<3, 4, 1>(A, st);
  // 512 threads, whole-sector staging. At this size the double-buffered
  // persistent form (209 KB of shared memory) measured slower than one block
  // per column block (C96 L127: 4.59 against 4.18 ms).
  if (L <= 128) return launch_step<4, 4, 1, true, false>(A, st);
  return launch_nw<8, 1, 2>(A, st);
}


namespace {

template <int NW, int G, int MINB>
cudaError_t launch_ens(const MpArgs* members, const int64_t* offs, int nm, int grid, cudaStream_t st) {
  const size_t smem = Smem<NW, G>::bytes;
  auto kern = mp_ensemble_kernel<NW, G, MINB, true>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, 32 * NW * G, smem, st>>>(members, offs, nm);
  return cudaGetLastError();
}

}  // namespace

// Ensemble launch over nz in (64, 128]: G columns per block (1, 2 or 4), a
// persistent grid of `grid` blocks.
cudaError_t mp_launch_ensemble_mixed(const MpArgs* members, const int64_t* offs, int nm, int nz, int G, int grid,
                                     cudaStream_t st) {
  if (nz <= 96) {
    if (G == 1) return launch_ens<3, 1, 4>(members, offs, nm, grid, st);
    if (G == 2) return launch_ens<3, 2, 2>(members, offs, nm, grid, st);
    if (G == 4) return launch_ens<3, 4, 1>(members, offs, nm, grid, st);
  } else if (nz <= 128) {
    if (G == 1) return launch_ens<4, 1, 4>(members, offs, nm, grid, st);
    if (G == 2) return launch_ens<4, 2, 2>(members, offs, nm, grid, st);
    if (G == 4) return launch_ens<4, 4, 1>(members, offs, nm, grid, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace shield
