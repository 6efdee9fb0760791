// Launch entry points of the microphysics kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include "mp_params.h"

namespace shield {

int mp_max_levels();
cudaError_t mp_launch_step(const MpArgs& A, int precision, cudaStream_t st);
cudaError_t mp_launch_plain_flags(const MpArgs& A, cudaStream_t st);
cudaError_t mp_launch_de_ice(const MpArgs& A, Fld3 qi_dt, Fld3 qs_dt, cudaStream_t st);
cudaError_t mp_gather_area(const double* p, int64_t si, int64_t sj, int nx, int ny, double* out);
cudaError_t mp_launch_ensemble_plain(const MpArgs* members, const int64_t* offs, int nm, int nz, int G, int grid,
                                     unsigned long long* counter, cudaStream_t st);
cudaError_t mp_launch_vjp(const VjpArgs& A, cudaStream_t st);
// doubles of the adjoint's workspace for nt sub-steps over npts points and ncol columns
int64_t mp_vjp_workspace_doubles(int nt, int64_t npts, int64_t ncol);
cudaError_t mp_launch_ensemble_mixed(const MpArgs* members, const int64_t* offs, int nm, int nz, int G, int grid,
                                     unsigned long long* counter, cudaStream_t st);

}  // namespace shield
