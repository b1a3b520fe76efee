// kernels_f32.cu -- step kernels with f32 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_f32(const LaunchSet& L) { return launch_store<ST_F32>(L); }
cudaError_t band_setup_f32() { return band_setup<ST_F32>(); }
// device address of this module's copy of the fused network (c_mlp)
cudaError_t mlp_const_addr_f32(void** p) { return cudaGetSymbolAddress(p, c_mlp); }
}  // namespace ippi
