// Mixed-precision form of the microphysics step: process rates in FP32,
// saturation adjustment, sedimentation, precipitation and every state
// update in FP64 (see mp_physics_mixed.cuh). FMA contraction is allowed here.
#include "mp_kernel.cuh"
#include "mp_launch.h"

namespace shield {

namespace {

template <int NW, int G, int MINB>
cudaError_t launch_nw(const MpArgs& A, cudaStream_t st) {
  return launch_step<ColumnLayout<NW, G>, MINB, true, true>(A, st);
}

// 65..80 levels, mixed form: groups of two packed columns per block and the
// __launch_bounds__ minimum blocks per SM (the packing, two columns per 5
// warps, is every L79 launch's); the double-buffered persistent form where
// its two buffers fit in shared memory beside the scratch.
#ifndef SHIELD_PACK_NGRP_MIXED
#define SHIELD_PACK_NGRP_MIXED SHIELD_PACK_NGRP
#endif
#ifndef SHIELD_PACK_MINB_MIXED
#define SHIELD_PACK_MINB_MIXED SHIELD_PACK_MINB
#endif
// (measured at C96 L79: 2.52 ms persistent, prefetching the inputs, against
// 2.51 ms with one block per column block)
#ifndef SHIELD_PACK_PERSIST
#define SHIELD_PACK_PERSIST 0
#endif
using Packed80Mixed = PackedLayout<SHIELD_PACK_NWG, SHIELD_PACK_P, SHIELD_PACK_NGRP_MIXED>;
constexpr bool kPersist80 = SHIELD_PACK_PERSIST && SmemP<Packed80Mixed, N_IN>::bytes <= 220 * 1024;
// 97..128 levels, mixed form: columns per block. C96 L127 (ms): 4 columns
// 4.17, 5 columns 3.70, 6 columns (768 threads, 80 registers) 3.57.
#ifndef SHIELD_NW4_G_MIXED
#define SHIELD_NW4_G_MIXED 6
#endif

}  // namespace

cudaError_t mp_launch_mixed(const MpArgs& A, cudaStream_t st) {
  const int L = A.nz;
  if (L <= 32) return launch_nw<1, 4, 2>(A, st);
  if (L <= 64) return launch_nw<2, 2, 2>(A, st);
  if (L <= PACK80_LMAX) return launch_step<Packed80Mixed, SHIELD_PACK_MINB_MIXED, true, kPersist80>(A, st);
  if (L <= 96) return launch_nw<3, 4, 1>(A, st);
  // At this size the double-buffered persistent form (209 KB of shared
  // memory for 4 columns) measured slower than one block per column block
  // (C96 L127: 4.59 against 4.18 ms).
  if (L <= 128) return launch_step<ColumnLayout<4, SHIELD_NW4_G_MIXED>, 1, true, false>(A, st);
  return launch_nw<8, 1, 2>(A, st);
}

// Ensemble launch over nz in (64, 128]; the shapes of
// mp_launch_ensemble_plain.
cudaError_t mp_launch_ensemble_mixed(const MpArgs* members, const int64_t* offs, int nm, int nz, int G, int grid,
                                     unsigned long long* counter, cudaStream_t st) {
  if (nz <= PACK80_LMAX) {
    if (G == 2) return launch_ensemble<PackedLayout<5, 2, 1>, 4, true>(members, offs, nm, counter, grid, st);
    if (G == 4) return launch_ensemble<PackedLayout<5, 2, 2>, 2, true>(members, offs, nm, counter, grid, st);
    if (G == 6) return launch_ensemble<PackedLayout<5, 2, 3>, 1, true>(members, offs, nm, counter, grid, st);
    if (G == 8) return launch_ensemble<PackedLayout<5, 2, 4>, 1, true>(members, offs, nm, counter, grid, st);
  } else if (nz <= 96) {
    if (G == 1) return launch_ensemble<ColumnLayout<3, 1>, 4, true>(members, offs, nm, counter, grid, st);
    if (G == 2) return launch_ensemble<ColumnLayout<3, 2>, 2, true>(members, offs, nm, counter, grid, st);
    if (G == 4) return launch_ensemble<ColumnLayout<3, 4>, 1, true>(members, offs, nm, counter, grid, st);
  } else if (nz <= 128) {
    if (G == 1) return launch_ensemble<ColumnLayout<4, 1>, 4, true>(members, offs, nm, counter, grid, st);
    if (G == 2) return launch_ensemble<ColumnLayout<4, 2>, 2, true>(members, offs, nm, counter, grid, st);
    if (G == 4) return launch_ensemble<ColumnLayout<4, 4>, 1, true>(members, offs, nm, counter, grid, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace shield
