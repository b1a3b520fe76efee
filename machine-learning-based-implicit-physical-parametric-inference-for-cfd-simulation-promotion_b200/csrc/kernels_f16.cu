// kernels_f16.cu -- step kernels with f16 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_f16(const LaunchSet& L) { return launch_store<ST_F16>(L); }
}  // namespace ippi
