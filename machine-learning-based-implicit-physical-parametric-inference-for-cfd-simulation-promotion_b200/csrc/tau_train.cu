// tau_train.cu -- training and batch inference kernels of the learned
// relaxation-time network (the MLP of lbm_common.cuh: 6 -> 32 tanh -> 32 tanh
// -> softplus), FP32, deterministic.
//
//   mlp_grad_kernel   each warp takes 32 samples at a time: one thread per
//                     sample runs the forward and backward pass and stages
//                     its activations and deltas in shared memory; then lane
//                     j accumulates row j of every weight gradient over the 32
//                     samples (dW2[j][:] += d2[s][j] h1[s][:], ...).  Warp
//                     sums are added in a fixed order into one partial per
//                     block.
//   mlp_grad_up_f64_kernel  the FP64 weight gradient of the adjoint (upstream
//                     gradients per sample): one warp per sample and one
//                     hidden neuron per lane, W2's row in registers, the other
//                     lanes' activations and deltas staged in shared memory and
//                     summed in four independent chains; samples whose
//                     upstream gradient is zero are skipped.
//   mlp_reduce_kernel the block partials summed in block order: gradient of
//                     the mean squared error and the loss
//   mlp_adam_kernel   Adam update, one thread per parameter
//   mlp_forward_kernel softplus outputs for a batch (evaluation)
#include <cuda_runtime.h>

#include "../../include/ippi_lbm.h"
#include "adjoint.h"
#include "lbm_common.cuh"

namespace {

using namespace ippi;

constexpr int kThreads = 128;                  // 4 warps
constexpr int kWarps = kThreads / 32;
constexpr int kRow = kMlpHid + 1;               // padded row of a 32-vector
constexpr int kXRow = kMlpIn + 1;
// per warp: x[32][7], h1/h2/d2/d1 [32][33], dout[32]
constexpr int kWarpFloats = 32 * kXRow + 4 * 32 * kRow + 32;
constexpr int kPartial = kMlpParams + 1;        // gradient + loss
template <typename R>
constexpr size_t grad_smem()
{
    return (size_t)(kWarps * kWarpFloats + kMlpParams + 3) * sizeof(R);
}
static_assert(kWarps * kWarpFloats >= kWarps * kPartial, "reduction buffer fits the staging area");

__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ double sigm(double z) { return 1.0 / (1.0 + exp(-z)); }
__device__ __forceinline__ float acc_tanh(float v) { return tanhf(v); }
__device__ __forceinline__ double acc_tanh(double v) { return tanh(v); }

// R: arithmetic type.  UP = false: Y holds targets, the loss is the mean
// squared error of softplus(z).  UP = true: Y holds upstream gradients
// dL/dsoftplus per sample (the loss is sum Y * softplus; no mean).
template <typename R, bool UP>
__global__ void __launch_bounds__(kThreads) mlp_grad_kernel(const R* __restrict__ X, const R* __restrict__ Y,
                                                             int n, const float* __restrict__ W,
                                                             R* __restrict__ part)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* sm = reinterpret_cast<R*>(sm_raw);
    R* ws = sm + kWarps * kWarpFloats;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int p = tid; p < kMlpParams; p += kThreads) ws[p] = R(W[p]);
    __syncthreads();
    R* base = sm + warp * kWarpFloats;
    R* xs = base;
    R* h1s = xs + 32 * kXRow;
    R* h2s = h1s + 32 * kRow;
    R* d2s = h2s + 32 * kRow;
    R* d1s = d2s + 32 * kRow;
    R* dos = d1s + 32 * kRow;

    const R inv_n = R(1) / (R)n;
    R gW2[kMlpHid], gW1[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpHid; i++) gW2[i] = R(0);
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) gW1[i] = R(0);
    R gb2 = 0, gb1 = 0, gw3 = 0, gb3 = 0, loss = 0;

    const int nchunks = (n + 31) / 32;
    for (int c = blockIdx.x * kWarps + warp; c < nchunks; c += gridDim.x * kWarps) {
        // ---- phase A: one sample per lane ----------------------------------
        const int s = c * 32 + lane;
        R x[kMlpIn], h1[kMlpHid], h2[kMlpHid];
        R dout = 0;
        if (s < n) {
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) x[i] = X[(size_t)s * kMlpIn + i];
        } else {
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) x[i] = 0;
        }
#pragma unroll
        for (int j = 0; j < kMlpHid; j++) {
            R a = ws[kMlpB1 + j];
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) a += ws[kMlpW1 + j * kMlpIn + i] * x[i];
            h1[j] = acc_tanh(a);
        }
        R z = ws[kMlpB3];
#pragma unroll
        for (int j = 0; j < kMlpHid; j++) {
            R a = ws[kMlpB2 + j];
#pragma unroll
            for (int i = 0; i < kMlpHid; i++) a += ws[kMlpW2 + j * kMlpHid + i] * h1[i];
            h2[j] = acc_tanh(a);
            z += ws[kMlpW3 + j] * h2[j];
        }
        if (s < n) {
            if (UP) {
                dout = Y[s] * sigm(z);
            } else {
                const R r = softplus(z) - Y[s];
                loss += r * r;
                dout = R(2) * r * sigm(z) * inv_n;
            }
        }
        // deltas: d2 = dout w3 (1 - h2^2); d1 = (W2^T d2) (1 - h1^2)
        R d2[kMlpHid];
#pragma unroll
        for (int j = 0; j < kMlpHid; j++) d2[j] = dout * ws[kMlpW3 + j] * (R(1) - h2[j] * h2[j]);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) xs[lane * kXRow + i] = x[i];
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) {
            R g = 0;
#pragma unroll
            for (int j = 0; j < kMlpHid; j++) g += ws[kMlpW2 + j * kMlpHid + i] * d2[j];
            d1s[lane * kRow + i] = g * (R(1) - h1[i] * h1[i]);
            h1s[lane * kRow + i] = h1[i];
            h2s[lane * kRow + i] = h2[i];
            d2s[lane * kRow + i] = d2[i];
        }
        dos[lane] = dout;
        __syncwarp();
        // ---- phase B: lane j accumulates row j over the 32 samples --------
        const int j = lane;
        for (int q = 0; q < 32; q++) {
            const R dj2 = d2s[q * kRow + j], dj1 = d1s[q * kRow + j], dq = dos[q];
#pragma unroll
            for (int i = 0; i < kMlpHid; i++) gW2[i] += dj2 * h1s[q * kRow + i];
            gb2 += dj2;
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) gW1[i] += dj1 * xs[q * kXRow + i];
            gb1 += dj1;
            gw3 += dq * h2s[q * kRow + j];
            gb3 += dq;
        }
        __syncwarp();
    }
    // ---- warp partials -> block partial (fixed order) -----------------------
    // the staging area is reused: warp w's gradient at sm[w * kPartial ...]
    R lsum = loss;
#pragma unroll
    for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    __syncthreads();
    R* g = sm + warp * kPartial;
    {
        const int j = lane;
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) g[kMlpW2 + j * kMlpHid + i] = gW2[i];
        g[kMlpB2 + j] = gb2;
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) g[kMlpW1 + j * kMlpIn + i] = gW1[i];
        g[kMlpB1 + j] = gb1;
        g[kMlpW3 + j] = gw3;
        if (j == 0) {
            g[kMlpB3] = gb3;
            g[kMlpParams] = lsum * inv_n;
        }
    }
    __syncthreads();
    for (int p = tid; p < kPartial; p += kThreads) {
        R v = 0;
        for (int w = 0; w < kWarps; w++) v += sm[w * kPartial + p];
        part[(size_t)blockIdx.x * kPartial + p] = v;
    }
}

// block partials summed in block order; ACC adds into grad instead of
// overwriting it
template <typename R, bool ACC>
__global__ void mlp_reduce_kernel(const R* __restrict__ part, int nblocks, R* __restrict__ grad,
                                  R* __restrict__ loss)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kPartial) return;
    R v = 0;
    for (int b = 0; b < nblocks; b++) v += part[(size_t)b * kPartial + p];
    if (p < kMlpParams) grad[p] = ACC ? grad[p] + v : v;
    else if (loss) *loss = v;
}

__global__ void mlp_adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                                float c2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.f - b1) * gp;
    const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

__global__ void __launch_bounds__(256) mlp_forward_kernel(const float* __restrict__ X, int n,
                                                          const float* __restrict__ W,
                                                          float* __restrict__ out)
{
    __shared__ __align__(16) float ws[kMlpParams + 3];
    for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) ws[p] = W[p];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) x[i] = X[(size_t)s * kMlpIn + i];
    float h1[kMlpHid];
#pragma unroll
    for (int j = 0; j < kMlpHid; j++) {
        float a = ws[kMlpB1 + j];
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) a += ws[kMlpW1 + j * kMlpIn + i] * x[i];
        h1[j] = tanhf(a);
    }
    float z = ws[kMlpB3];
#pragma unroll 4
    for (int j = 0; j < kMlpHid; j++) {
        float a = ws[kMlpB2 + j];
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) a += ws[kMlpW2 + j * kMlpHid + i] * h1[i];
        z += ws[kMlpW3 + j] * tanhf(a);
    }
    out[s] = softplus(z);
}

// The adjoint's weight gradient, FP64: sum over samples s of
// Y[s] * d softplus(z(x_s)) / dw.  One sample per warp at a time, lane j =
// neuron j of both hidden layers: row j of W2 in registers, its columns read
// from shared memory (conflict-free), the other lanes' activations by
// shuffle.  Lane j accumulates row j of dW2 and dW1 in registers; samples
// with Y[s] = 0 (outside the network's range) are skipped.  Warp partials
// are added in warp order into one partial per block, in the layout
// mlp_reduce_kernel expects.
__global__ void __launch_bounds__(kThreads) mlp_grad_up_f64_kernel(const double* __restrict__ X,
                                                                   const double* __restrict__ Y, int n,
                                                                   const float* __restrict__ W,
                                                                   double* __restrict__ part)
{
    // W2 during the sample loop, the warp partials after it
    __shared__ double smem[kWarps * kPartial];
    __shared__ double hs[kWarps][kMlpHid], ds[kWarps][kMlpHid];  // per warp: h1, then d2
    static_assert(kWarps * kPartial >= kMlpHid * kMlpHid, "W2 fits the partial buffer");
    double* w2s = smem;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int p = tid; p < kMlpHid * kMlpHid; p += kThreads) w2s[p] = double(W[kMlpW2 + p]);
    const int j = lane;
    double w1[kMlpIn], w2r[kMlpHid];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) w1[i] = double(W[kMlpW1 + j * kMlpIn + i]);
#pragma unroll
    for (int i = 0; i < kMlpHid; i++) w2r[i] = double(W[kMlpW2 + j * kMlpHid + i]);
    const double b1 = double(W[kMlpB1 + j]), b2 = double(W[kMlpB2 + j]), w3 = double(W[kMlpW3 + j]);
    const double b3 = double(W[kMlpB3]);
    __syncthreads();
    double gW2[kMlpHid], gW1[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpHid; i++) gW2[i] = 0.0;
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) gW1[i] = 0.0;
    double gb1 = 0.0, gb2 = 0.0, gw3 = 0.0, gb3 = 0.0;
    const int nw = gridDim.x * kWarps;
    for (int s = blockIdx.x * kWarps + warp; s < n; s += nw) {
        const double up = Y[s];
        if (up == 0.0) continue;  // the same sample on every lane
        double x[kMlpIn];
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) x[i] = X[(size_t)s * kMlpIn + i];
        double a1 = b1;
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) a1 += w1[i] * x[i];
        const double h1 = tanh(a1);
        // the other lanes' values through shared memory, summed in four
        // independent chains
        hs[warp][j] = h1;
        __syncwarp();
        double p2[4] = {b2, 0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) p2[i & 3] += w2r[i] * hs[warp][i];
        const double h2 = tanh((p2[0] + p2[1]) + (p2[2] + p2[3]));
        double z = w3 * h2;
#pragma unroll
        for (int o = 16; o; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
        z += b3;
        const double dout = up * sigm(z);
        const double d2 = dout * w3 * (1.0 - h2 * h2);
        ds[warp][j] = d2;
        __syncwarp();
        double p1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < kMlpHid; k++) p1[k & 3] += w2s[k * kMlpHid + j] * ds[warp][k];
        const double d1 = ((p1[0] + p1[1]) + (p1[2] + p1[3])) * (1.0 - h1 * h1);
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) gW2[i] += d2 * hs[warp][i];
        __syncwarp();  // hs / ds are rewritten for the next sample
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) gW1[i] += d1 * x[i];
        gb2 += d2;
        gb1 += d1;
        gw3 += dout * h2;
        gb3 += dout;
    }
    __syncthreads();  // W2 no longer read
    double* r = smem + warp * kPartial;
#pragma unroll
    for (int i = 0; i < kMlpHid; i++) r[kMlpW2 + j * kMlpHid + i] = gW2[i];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) r[kMlpW1 + j * kMlpIn + i] = gW1[i];
    r[kMlpB1 + j] = gb1;
    r[kMlpB2 + j] = gb2;
    r[kMlpW3 + j] = gw3;
    if (j == 0) {
        r[kMlpB3] = gb3;
        r[kMlpParams] = 0.0;
    }
    __syncthreads();
    for (int p = tid; p < kPartial; p += kThreads) {
        double v = 0.0;
        for (int w = 0; w < kWarps; w++) v += smem[w * kPartial + p];
        part[(size_t)blockIdx.x * kPartial + p] = v;
    }
}

bool g_grad_attr = false;

}  // namespace

namespace ippi {

size_t mlp_grad_f64_partial_doubles() { return (size_t)IPPI_MLP_GRAD_BLOCKS * kPartial; }

cudaError_t mlp_grad_upstream_f64(const double* xs, const double* up, int n, const float* w, double* part,
                                  double* grad, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    mlp_grad_up_f64_kernel<<<IPPI_MLP_GRAD_BLOCKS, kThreads, 0, st>>>(xs, up, n, w, part);
    mlp_reduce_kernel<double, true><<<(kPartial + 255) / 256, 256, 0, st>>>(part, IPPI_MLP_GRAD_BLOCKS, grad, nullptr);
    return cudaGetLastError();
}

}  // namespace ippi

extern "C" {

int ippi_mlp_param_count(void) { return kMlpParams; }

size_t ippi_mlp_scratch_floats(void) { return (size_t)IPPI_MLP_GRAD_BLOCKS * kPartial; }

int ippi_mlp_grad(const float* x, const float* y, int n, const float* w, float* grad, float* loss,
                  float* scratch, void* stream)
{
    if (!x || !y || !w || !grad || !scratch || n <= 0) return IPPI_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (!g_grad_attr) {
        if (cudaFuncSetAttribute(mlp_grad_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)grad_smem<float>()) != cudaSuccess)
            return IPPI_ERR_CUDA;
        g_grad_attr = true;
    }
    mlp_grad_kernel<float, false><<<IPPI_MLP_GRAD_BLOCKS, kThreads, grad_smem<float>(), st>>>(x, y, n, w, scratch);
    mlp_reduce_kernel<float, false><<<(kPartial + 255) / 256, 256, 0, st>>>(scratch, IPPI_MLP_GRAD_BLOCKS, grad,
                                                                           loss);
    return cudaGetLastError() == cudaSuccess ? IPPI_OK : IPPI_ERR_CUDA;
}

int ippi_mlp_adam(float* w, const float* grad, float* m, float* v, int step, float lr, float beta1,
                  float beta2, float eps, void* stream)
{
    if (!w || !grad || !m || !v || step < 1 || !(lr > 0)) return IPPI_ERR_ARG;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, grad, m, v, lr, beta1,
                                                                               beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? IPPI_OK : IPPI_ERR_CUDA;
}

int ippi_mlp_forward(const float* x, int n, const float* w, float* out, void* stream)
{
    if (!x || !w || !out || n < 0) return IPPI_ERR_ARG;
    if (n == 0) return IPPI_OK;
    mlp_forward_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(x, n, w, out);
    return cudaGetLastError() == cudaSuccess ? IPPI_OK : IPPI_ERR_CUDA;
}

}  // extern "C"
