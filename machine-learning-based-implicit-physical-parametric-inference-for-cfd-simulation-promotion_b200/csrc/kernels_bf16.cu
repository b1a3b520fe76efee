// kernels_bf16.cu -- step kernels with bf16 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_bf16(const LaunchSet& L) { return launch_store<ST_BF16>(L); }
cudaError_t band_setup_bf16() { return band_setup<ST_BF16>(); }
// device address of this module's copy of the fused network (c_mlp)
cudaError_t mlp_const_addr_bf16(void** p) { return cudaGetSymbolAddress(p, c_mlp); }
}  // namespace ippi
