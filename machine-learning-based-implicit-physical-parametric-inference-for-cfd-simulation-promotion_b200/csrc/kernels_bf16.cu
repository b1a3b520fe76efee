// kernels_bf16.cu -- step kernels with bf16 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_bf16(const LaunchSet& L) { return launch_store<ST_BF16>(L); }
}  // namespace ippi
