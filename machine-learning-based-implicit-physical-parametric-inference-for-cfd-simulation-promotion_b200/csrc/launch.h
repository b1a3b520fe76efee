// launch.h -- host-side launch descriptors shared by the per-storage kernel
// translation units (kernels_f64.cu, kernels_f32.cu, kernels_f16.cu,
// kernels_bf16.cu) and the C-ABI layer (ippi_lbm.cu).
#pragma once

#include "lbm_kernels.cuh"

namespace ippi {

struct LaunchSet {
    StepArgs step;
    dim3 grid;
    int coll, scene;
    // side-stream work: (prep -> band) and/or the IB chain, forked from and
    // joined to `stream`
    const PrepNode* prep;
    int nprep;
    bool band;
    BandArgs band_args;
    int band_blocks;
    bool ib;
    IbArgs ib_args;
    int ib_nst;          // 4 or 16 stencil nodes per marker
    int ib_passes;       // direct-forcing passes
    cudaStream_t stream, side;
    int side_prio;       // launch priority of the side-stream kernels
    cudaEvent_t fork, join;
    // optional device timing: events[0..3] around the bulk kernel and the
    // side-stream chain (only when not capturing)
    cudaEvent_t* events;
    // this step updates the running means (t >= avg_start): the bulk
    // kernel's averaging instance
    bool avg_on;
};

// Mesh::FindAndWriteTau's scan (tau_scan.cu) on device arrays
cudaError_t tau_scan_launch(const double* f, const double* m3, const double* tau, int nx, int ny, int n,
                            const int* xy, const double* target, int m_lo, int m_hi, double step,
                            double* best_dtau, double* best_err, cudaStream_t st);

cudaError_t launch_f64(const LaunchSet& L);
cudaError_t launch_f32(const LaunchSet& L);
cudaError_t launch_f16(const LaunchSet& L);
cudaError_t launch_bf16(const LaunchSet& L);

// allow band_kernel's dynamic shared memory (current device), per storage
cudaError_t band_setup_f64();
cudaError_t band_setup_f32();
cudaError_t band_setup_f16();
cudaError_t band_setup_bf16();

// device address (current device) of each storage module's constant-memory
// copy of the fused learned-tau network (c_mlp in lbm_common.cuh)
cudaError_t mlp_const_addr_f64(void** p);
cudaError_t mlp_const_addr_f32(void** p);
cudaError_t mlp_const_addr_f16(void** p);
cudaError_t mlp_const_addr_bf16(void** p);

}  // namespace ippi
