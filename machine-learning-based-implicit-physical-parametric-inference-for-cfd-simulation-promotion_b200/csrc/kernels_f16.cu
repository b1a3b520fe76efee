// kernels_f16.cu -- step kernels with f16 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_f16(const LaunchSet& L) { return launch_store<ST_F16>(L); }
cudaError_t band_setup_f16() { return band_setup<ST_F16>(); }
// device address of this module's copy of the fused network (c_mlp)
cudaError_t mlp_const_addr_f16(void** p) { return cudaGetSymbolAddress(p, c_mlp); }
}  // namespace ippi
