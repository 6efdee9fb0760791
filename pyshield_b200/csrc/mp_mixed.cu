// Mixed-precision form of the microphysics step: not built yet, so the
// entry point reports that the mode is unavailable.
#include "mp_launch.h"

namespace shield {
cudaError_t mp_launch_mixed(const MpArgs&, cudaStream_t) { return cudaErrorNotSupported; }
}  // namespace shield
