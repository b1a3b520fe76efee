// kernels_f64.cu -- step kernels with f64 population storage.
#include "kernels_impl.cuh"

namespace ippi {
cudaError_t launch_f64(const LaunchSet& L) { return launch_store<ST_F64>(L); }
cudaError_t band_setup_f64() { return band_setup<ST_F64>(); }
// device address of this module's copy of the fused network (c_mlp)
cudaError_t mlp_const_addr_f64(void** p) { return cudaGetSymbolAddress(p, c_mlp); }
}  // namespace ippi
