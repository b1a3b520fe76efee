// kernels_f32.cu -- step kernels with f32 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_f32(const LaunchSet& L) { return launch_store<ST_F32>(L); }
}  // namespace ippi
