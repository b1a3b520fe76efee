// tau_scan.cu -- the implicit relaxation-time inference of the reference,
// Mesh::FindAndWriteTau (mesh.cpp:2625-2715), on the GPU.
//
// For a node and target moments (R, U, V), candidates dtau = m * step,
// m = m_lo .. m_hi (the reference: -10000 .. 10000, step 1e-5): each
// upstream neighbour relaxes with BGK at its tau + dtau,
//   fcol_k = (1 - 1/(tau + dtau)) fnew_k + feq_k / (tau + dtau),
// streams into the node, and the candidate's error is
//   |sum f - R| + |sum f e_x - U| + |sum f e_y - V|
// (momentum against the target velocity, as the reference compares them).
// The first minimum wins.  One warp per node: lane l takes m = m_lo + l,
// m_lo + l + 32, ...; the warp then reduces (error, m) lexicographically,
// which is the sequential first minimum.  This unit is compiled without FMA
// contraction and uses the reference's expression order, so its results
// equal a sequential FP64 scan bit for bit.
#include <climits>

#include "../../include/ippi_lbm.h"
#include "launch.h"

namespace ippi {
namespace {

constexpr int kScanWarps = 8;

// Lattice::Compute_feq (NodeAndLattice.cpp:124-149), same expression order
__device__ __forceinline__ void feq_ref(double rho, double ux, double uy, double* feq)
{
    const double w0 = rho * (4.0 / 9.0), w1 = rho / 9.0, w2 = rho / 36.0;
    const double uu = 1 - 1.5 * (ux * ux + uy * uy);
    feq[0] = w0 * (uu);
    feq[1] = w1 * (uu + 3.0 * (ux) + 4.5 * (ux) * (ux));
    feq[2] = w1 * (uu + 3.0 * (uy) + 4.5 * (uy) * (uy));
    feq[3] = w1 * (uu - 3.0 * (ux) + 4.5 * (ux) * (ux));
    feq[4] = w1 * (uu - 3.0 * (uy) + 4.5 * (uy) * (uy));
    feq[5] = w2 * (uu + 3.0 * (ux + uy) + 4.5 * (ux + uy) * (ux + uy));
    feq[6] = w2 * (uu - 3.0 * (ux - uy) + 4.5 * (ux - uy) * (ux - uy));
    feq[7] = w2 * (uu - 3.0 * (ux + uy) + 4.5 * (ux + uy) * (ux + uy));
    feq[8] = w2 * (uu + 3.0 * (ux - uy) + 4.5 * (ux - uy) * (ux - uy));
}

__global__ void __launch_bounds__(32 * kScanWarps) tau_scan_kernel(const double* __restrict__ f,
                                                                  const double* __restrict__ m3,
                                                                  const double* __restrict__ tau, int nx,
                                                                  int ny, int n, const int* __restrict__ xy,
                                                                  const double* __restrict__ target, int m_lo,
                                                                  int m_hi, double step, double* best_dtau,
                                                                  double* best_err)
{
    const int w = blockIdx.x * kScanWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (w >= n) return;  // the whole warp
    const long long nn = (long long)nx * ny;
    const int x = xy[2 * w], y = xy[2 * w + 1];
    double fn[9], fe[9], tn[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const long long g = (long long)(y - EY(k)) * nx + (x - EX(k));
        double feq[9];
        feq_ref(m3[g], m3[nn + g], m3[2 * nn + g], feq);
        fn[k] = f[k * nn + g];
        fe[k] = feq[k];
        tn[k] = tau[g];
    }
    const double R = target[3 * w], U = target[3 * w + 1], V = target[3 * w + 2];
    double best = 1e10;
    int bm = INT_MAX;
    for (int mm = m_lo + lane; mm <= m_hi; mm += 32) {
        const double d = (double)mm * step;
        double trho = 0, tu = 0, tv = 0;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const double c = (1.0 - 1.0 / (tn[k] + d)) * fn[k] + fe[k] / (tn[k] + d);
            trho += c;
            tu += c * (double)EX(k);
            tv += c * (double)EY(k);
        }
        const double err = fabs(trho - R) + fabs(tu - U) + fabs(tv - V);
        if (err < best) {
            best = err;
            bm = mm;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int om = __shfl_down_sync(0xffffffffu, bm, o);
        if (ob < best || (ob == best && om < bm)) {
            best = ob;
            bm = om;
        }
    }
    if (lane == 0) {
        best_dtau[w] = bm == INT_MAX ? 1e10 : (double)bm * step;
        best_err[w] = best;
    }
}

}  // namespace

cudaError_t tau_scan_launch(const double* f, const double* m3, const double* tau, int nx, int ny, int n,
                            const int* xy, const double* target, int m_lo, int m_hi, double step,
                            double* best_dtau, double* best_err, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    tau_scan_kernel<<<(n + kScanWarps - 1) / kScanWarps, 32 * kScanWarps, 0, st>>>(
        f, m3, tau, nx, ny, n, xy, target, m_lo, m_hi, step, best_dtau, best_err);
    return cudaGetLastError();
}

}  // namespace ippi

extern "C" int ippi_tau_scan_state(const double* f, const double* m3, const double* tau, int nx, int ny, int n,
                                   const int* xy, const double* target, int m_lo, int m_hi, double step,
                                   double* best_dtau, double* best_err, void* stream)
{
    if (!f || !m3 || !tau || nx < 3 || ny < 3 || n < 0 || (n > 0 && (!xy || !target || !best_dtau || !best_err)) ||
        m_lo > m_hi || !(step > 0))
        return IPPI_ERR_ARG;
    return ippi::tau_scan_launch(f, m3, tau, nx, ny, n, xy, target, m_lo, m_hi, step, best_dtau, best_err,
                                 (cudaStream_t)stream) == cudaSuccess
               ? IPPI_OK
               : IPPI_ERR_CUDA;
}
