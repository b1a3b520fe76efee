// adjoint.h -- launchers of the reverse-mode step (adjoint.cu) used by the
// C-ABI layer (ippi_lbm.cu).  All adjoint arithmetic is FP64 on unshifted
// populations; the forward state is read in its storage type.
//
// One reverse step, for the step that maps f_in to f_out:
//   adj_state      f~ = stream + boundaries(f_in) and its moments (recompute)
//   adj_ib_fwd     the IB sub-step on f~ (recompute): marker velocities,
//                  forces, node force densities, corrected velocities
//   adj_collide    lam_f~ = (d f_out / d f~)^T lam_out per node, by dual
//                  numbers through the node's collision (tau model included);
//                  forced nodes also give lam of their corrected velocity and
//                  force density; g_tau = lam_out . d f_out / d tau
//   adj_ib_back    transposed spreading and interpolation: lam of the marker
//                  forces (plus the loss on the body forces) back to lam_f~
//   adj_stream     lam_in = (d f~ / d f_in)^T lam_f~: transposed pull,
//                  bounce-back, Zou-He inlet and NEE outlet, as a gather
//                  (every lam_in entry written once; no atomics)
#pragma once

#include "lbm_kernels.cuh"

namespace ippi {

struct AdjArgs {
    StepArgs s;          // geometry, parameters, tau model (f_in = the step's input)
    int storage;
    double* ft;          // [9][nn] post-stream populations f~
    double* m;           // [3][nn] rho, ux, uy of f~
    const double* lam_out;  // [9][nn] dL / d f_out
    double* lam_ft;      // [9][nn] dL / d f~
    double* lam_in;      // [9][nn] dL / d f_in (written by adj_stream)
    double* grad_tau;    // [nn] accumulated (tau field), or null
    double* xs;          // [nn][6] standardised features of learned nodes (else 0)
    double* up;          // [nn] dL / d softplus * out_scale of learned nodes (else 0)
    double* lin;         // [nn][8] learned tau linearised: value, d tau / d x[6], in-range flag
    const double* dldm;  // [3][nn] loss on the post-stream moments, or null
    // immersed boundary (null when no markers)
    const IbArgs* ib;    // host copy of the forward's tables
    int nst;             // stencil nodes per marker (4 bilinear, 16 Peskin)
    const int* fidx;     // [nn] forced-node index or -1
    const int* mbody;    // [nmark] body of each marker
    double* ib_rho;      // [nforced]
    double2* ib_us;      // [nforced] uncorrected velocity
    double2* ib_F;       // [nmark] marker force
    double2* ib_fn;      // [nforced] node force density
    double2* ib_uc;      // [nforced] corrected velocity
    double2* lam_uc;     // [nforced]
    double2* lam_fn;     // [nforced]
    double2* lam_ftot;   // [nforced]
    double* lam_rho;     // [nforced]
    double2* lam_F;      // [nmark]
    const double* dldF;  // [nbody][2] loss on this step's body forces, or null
    int collision;
    bool learned;
};

cudaError_t adj_state(const AdjArgs& A, cudaStream_t st);
cudaError_t adj_ib_fwd(const AdjArgs& A, cudaStream_t st);
cudaError_t adj_collide(const AdjArgs& A, cudaStream_t st);
cudaError_t adj_inject_moments(const AdjArgs& A, cudaStream_t st);
cudaError_t adj_ib_back(const AdjArgs& A, cudaStream_t st);
cudaError_t adj_stream(const AdjArgs& A, cudaStream_t st);
cudaError_t adj_ib_tables(const IbArgs& ib, int nx, int ny, int* fidx, int* mbody, cudaStream_t st);

// FP64 gradient with respect to the MLP parameters (lbm_common.cuh layout,
// weights w as FP32) of sum_s up[s] * softplus(MLP(xs[s])), added into
// grad[1313]; part holds mlp_grad_f64_partial_doubles() doubles

cudaError_t mlp_grad_upstream_f64(const double* xs, const double* up, int n, const float* w,
                                  double* part, double* grad, cudaStream_t st);
size_t mlp_grad_f64_partial_doubles();

}  // namespace ippi
