// kernels_bf16.cu -- step kernels with bf16 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_bf16(const LaunchSet& L) { return launch_store<ST_BF16>(L); }
cudaError_t prepare_bf16(size_t ib_smem) { return prepare_store<ST_BF16>(ib_smem); }
}  // namespace ippi
