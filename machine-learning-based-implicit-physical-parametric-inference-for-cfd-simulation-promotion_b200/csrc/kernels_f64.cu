// kernels_f64.cu -- step kernels with f64 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_f64(const LaunchSet& L) { return launch_store<ST_F64>(L); }
}  // namespace ippi
