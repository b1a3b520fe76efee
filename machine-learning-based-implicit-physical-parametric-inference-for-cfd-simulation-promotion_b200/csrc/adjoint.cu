// adjoint.cu -- the reverse-mode step (see adjoint.h for the stages).
// Channel scene (Zou-He inlet, NEE outlet, bounce-back walls), BGK / MRT / RR,
// tau constant, Smagorinsky, learned or a given field, IB with one
// direct-forcing pass.
#include "adjoint.h"

namespace ippi {
namespace {

constexpr int kT = 128;
constexpr int kDual = 14;  // f~[9], corrected u (2), force density (2), tau
using D = Dual<kDual>;

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ---- recompute: post-stream state of every node -----------------------------
template <int S>
__global__ void __launch_bounds__(kT) adj_state_kernel(const AdjArgs A)
{
    using C = typename Store<S>::C;
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const long long node = blockIdx.x * (long long)kT + threadIdx.x;
    if (node >= nn) return;
    const int x = (int)(node % a.nx), y = (int)(node / a.nx);
    C f[9], rho, ux, uy;
    node_state<S, SC_CHANNEL>(a, x, y, f, rho, ux, uy);
    const double rb = double(rbase<S>(a));
#pragma unroll
    for (int k = 0; k < 9; k++) A.ft[k * nn + node] = double(f[k]) + WK<double>(k) * rb;
    A.m[node] = double(rho);
    A.m[nn + node] = double(ux);
    A.m[2 * nn + node] = double(uy);
}

// ---- recompute: the IB sub-step (one direct-forcing pass) ------------------
__global__ void adj_ib_nodes_kernel(const AdjArgs A, IbArgs I)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= I.nforced) return;
    const long long nn = (long long)A.s.nx * A.s.ny;
    const int2 xy = I.fn_xy[n];
    const long long node = (long long)xy.y * A.s.nx + xy.x;
    A.ib_rho[n] = A.m[node];
    A.ib_us[n] = make_double2(A.m[nn + node], A.m[2 * nn + node]);
}

template <int NST>
__global__ void adj_ib_markers_kernel(const AdjArgs A, IbArgs I)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= I.nmark) return;
    double vx = 0.0, vy = 0.0;
#pragma unroll
    for (int q = 0; q < NST; q++) {
        const int n = I.st_node[m * 16 + q];
        const double2 w = I.st_w[m * 16 + q];
        vx += A.ib_us[n].x * w.x * w.y;
        vy += A.ib_us[n].y * w.x * w.y;
    }
    const double2 u = I.ub[m];
    A.ib_F[m] = make_double2(2.0 * (u.x - vx), 2.0 * (u.y - vy));
}

__global__ void adj_ib_spread_kernel(const AdjArgs A, IbArgs I)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= I.nforced) return;
    double fx = 0.0, fy = 0.0;
    for (int e = I.fn_ptr[n]; e < I.fn_ptr[n + 1]; e++) {
        const double2 d = A.ib_F[I.fe_marker[e]];
        const double2 w = I.fe_w[e];
        fx += d.x * w.x * w.y;
        fy += d.y * w.x * w.y;
    }
    const double r = A.ib_rho[n];
    A.ib_fn[n] = make_double2(fx, fy);
    A.ib_uc[n] = make_double2(A.ib_us[n].x + 0.5 * 1 * fx / r, A.ib_us[n].y + 0.5 * 1 * fy / r);
}

// ---- collision: vector-Jacobian product by dual numbers ---------------------
template <int CO, bool LRN>
__global__ void __launch_bounds__(kT) adj_collide_kernel(const AdjArgs A)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const long long node = blockIdx.x * (long long)kT + threadIdx.x;
    if (node >= nn) return;
    const int fi = A.fidx ? A.fidx[node] : -1;
    D f[9];
    double fv[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        fv[k] = A.ft[k * nn + node];
        f[k] = D::seed(fv[k], k);
    }
    D rho, ux, uy;
    macros<D>(f, D(0.0), rho, ux, uy);
    D fxd(0.0), fyd(0.0);
    if (fi >= 0) {
        ux = D::seed(A.ib_uc[fi].x, 9);
        uy = D::seed(A.ib_uc[fi].y, 10);
        fxd = D::seed(A.ib_fn[fi].x, 11);
        fyd = D::seed(A.ib_fn[fi].y, 12);
    }
    const D tau0(a.tau0), cs(a.cs);
    D tau = a.les == 3 ? D(a.tau_field[node]) : node_tau<D, LRN>(f, rho, ux, uy, D(0.0), a.les, tau0, cs, a.mlp);
    tau.d[13] += 1.0;
    collide_node<D, CO>(f, rho, ux, uy, D(0.0), tau);
    if (fi >= 0) add_force<D, CO>(f, ux, uy, fxd, fyd, tau0, tau);
    double lam[9];
#pragma unroll
    for (int k = 0; k < 9; k++) lam[k] = A.lam_out[k * nn + node];
    double g[kDual];
#pragma unroll
    for (int j = 0; j < kDual; j++) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 9; k++) s += lam[k] * f[k].d[j];
        g[j] = s;
    }
#pragma unroll
    for (int j = 0; j < 9; j++) A.lam_ft[j * nn + node] = g[j];
    if (fi >= 0) {
        A.lam_uc[fi] = make_double2(g[9], g[10]);
        A.lam_fn[fi] = make_double2(g[11], g[12]);
    }
    if (A.grad_tau && a.les == 3) A.grad_tau[node] += g[13];
    if (LRN && A.xs) {
        // the network path (features inside the training range) carries
        // dL/dw; the fallback does not
        double r = rho.v, vx = ux.v, vy = uy.v, pxx, pxy, pyy, x[kMlpIn];
        pi_neq<double>(fv, r, vx, vy, 0.0, pxx, pxy, pyy);
        mlp_features<double>(pxx, pxy, pyy, r, vx, vy, a.tau0, x);
        const float* st = a.mlp + kMlpParams;
        bool in = true;
        for (int i = 0; i < kMlpIn; i++) in = in && x[i] >= double(st[2 * kMlpIn + i]) && x[i] <= double(st[3 * kMlpIn + i]);
        for (int i = 0; i < kMlpIn; i++) A.xs[node * kMlpIn + i] = in ? (x[i] - double(st[i])) / double(st[kMlpIn + i]) : 0.0;
        A.up[node] = in ? g[13] * double(st[4 * kMlpIn]) : 0.0;
    }
}

// loss on the post-stream moments (rho, ux, uy) of the last step
__global__ void adj_inject_kernel(const AdjArgs A)
{
    const long long nn = (long long)A.s.nx * A.s.ny;
    const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (node >= nn) return;
    const double r = A.m[node], ux = A.m[nn + node], uy = A.m[2 * nn + node];
    const double gr = A.dldm[node], gx = A.dldm[nn + node], gy = A.dldm[2 * nn + node];
#pragma unroll
    for (int k = 0; k < 9; k++)
        A.lam_ft[k * nn + node] += gr + (gx * (EX(k) - ux) + gy * (EY(k) - uy)) / r;
}

// ---- IB adjoint --------------------------------------------------------------
__global__ void adj_ib_back1_kernel(const AdjArgs A, IbArgs I)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= I.nforced) return;
    const double r = A.ib_rho[n];
    const double2 luc = A.lam_uc[n], lfn = A.lam_fn[n], fn = A.ib_fn[n];
    // u_c = u* + f / (2 rho)
    A.lam_ftot[n] = make_double2(lfn.x + 0.5 * luc.x / r, lfn.y + 0.5 * luc.y / r);
    A.lam_rho[n] = -0.5 * (luc.x * fn.x + luc.y * fn.y) / (r * r);
}

template <int NST>
__global__ void adj_ib_back2_kernel(const AdjArgs A, IbArgs I)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= I.nmark) return;
    // f_n = sum_m F_m w_mn  ->  lam_F_m = sum_n w_mn lam_f_n
    double lx = 0.0, ly = 0.0;
    for (int q = 0; q < NST; q++) {
        const int n = I.st_node[m * 16 + q];
        const double2 w = I.st_w[m * 16 + q];
        lx += A.lam_ftot[n].x * w.x * w.y;
        ly += A.lam_ftot[n].y * w.x * w.y;
    }
    if (A.dldF) {
        // body force = -sum_m F_m ds_m
        const int b = A.mbody[m];
        lx -= I.ds[m] * A.dldF[2 * b];
        ly -= I.ds[m] * A.dldF[2 * b + 1];
    }
    A.lam_F[m] = make_double2(lx, ly);
}

__global__ void adj_ib_back3_kernel(const AdjArgs A, IbArgs I)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= I.nforced) return;
    const long long nn = (long long)A.s.nx * A.s.ny;
    // F_m = 2 (U_b - sum_n w_mn u*_n)  ->  lam_u*_n = lam_uc_n - 2 sum_m w_mn lam_F_m
    double lx = A.lam_uc[n].x, ly = A.lam_uc[n].y;
    for (int e = I.fn_ptr[n]; e < I.fn_ptr[n + 1]; e++) {
        const double2 l = A.lam_F[I.fe_marker[e]];
        const double2 w = I.fe_w[e];
        lx -= 2.0 * l.x * w.x * w.y;
        ly -= 2.0 * l.y * w.x * w.y;
    }
    const int2 xy = I.fn_xy[n];
    const long long node = (long long)xy.y * A.s.nx + xy.x;
    const double r = A.ib_rho[n], ux = A.ib_us[n].x, uy = A.ib_us[n].y, lr = A.lam_rho[n];
    // rho = sum f, u* = sum e f / rho
#pragma unroll
    for (int k = 0; k < 9; k++) A.lam_ft[k * nn + node] += lr + (lx * (EX(k) - ux) + ly * (EY(k) - uy)) / r;
}

// ---- transposed streaming and boundaries -----------------------------------
__device__ __forceinline__ void scatter_pull(const AdjArgs& A, int x, int y, const double* lam)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        if (lam[k] == 0.0) continue;
        const int sx = x - EX(k), sy = y - EY(k);
        if (sy < 0 || sy >= a.ny)
            atomicAdd(A.lam_in + OPP(k) * nn + (long long)y * a.nx + x, lam[k]);
        else if (sx >= 0)
            atomicAdd(A.lam_in + k * nn + (long long)sy * a.nx + sx, lam[k]);
    }
}

// transposed ch_fluid at (x, y): Zou-He (x = 0), then the pull
__device__ __forceinline__ void fluid_back(const AdjArgs& A, int x, int y, double* lam)
{
    const StepArgs& a = A.s;
    if (x == 0) {
        // the regularised Zou-He inlet is linear in the pulled populations:
        // its Jacobian from one dual evaluation, transposed onto lam
        using D9 = Dual<9>;
        D9 g[9];
#pragma unroll
        for (int k = 0; k < 9; k++) g[k] = D9::seed(0.0, k);
        zh_inlet<D9>(g, D9(inlet_profile<double>(y, a.ny, a.u_in)), D9(0.0));
        double lp[9];
#pragma unroll
        for (int j = 0; j < 9; j++) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++) v += lam[k] * g[k].d[j];
            lp[j] = v;
        }
#pragma unroll
        for (int k = 0; k < 9; k++) lam[k] = lp[k];
    }
    scatter_pull(A, x, y, lam);
}

__global__ void __launch_bounds__(kT) adj_stream_kernel(const AdjArgs A)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const long long node = blockIdx.x * (long long)kT + threadIdx.x;
    if (node >= nn) return;
    const int x = (int)(node % a.nx), y = (int)(node / a.nx);
    double lam[9];
#pragma unroll
    for (int k = 0; k < 9; k++) lam[k] = A.lam_ft[k * nn + node];
    if (x == a.nx - 1) {
        // NEE outlet: f~ = feq(rho0, ub) + fb - feq(rho_b, ub), fb = f~(nx-2, y)
        const long long b = node - 1;
        const double rb = A.m[b], ux = A.m[nn + b], uy = A.m[2 * nn + b];
        const double r0 = a.rho0;
        double gr = 0.0, gx = 0.0, gy = 0.0;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const double eu = EX(k) * ux + EY(k) * uy;
            const double w = WK<double>(k);
            const double fe1 = w * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * (ux * ux + uy * uy));
            gr -= lam[k] * fe1;
            // d feq / d u = w rho (3 e + 9 (e.u) e - 3 u)
            gx += lam[k] * (r0 - rb) * w * (3.0 * EX(k) + 9.0 * eu * EX(k) - 3.0 * ux);
            gy += lam[k] * (r0 - rb) * w * (3.0 * EY(k) + 9.0 * eu * EY(k) - 3.0 * uy);
        }
        double lb[9];
#pragma unroll
        for (int k = 0; k < 9; k++) lb[k] = lam[k] + gr + (gx * (EX(k) - ux) + gy * (EY(k) - uy)) / rb;
        fluid_back(A, a.nx - 2, y, lb);
    } else {
        fluid_back(A, x, y, lam);
    }
}

__global__ void adj_tables_kernel(IbArgs I, int nx, int* fidx, int* mbody)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < I.nforced) {
        const int2 xy = I.fn_xy[i];
        fidx[(long long)xy.y * nx + xy.x] = i;
    }
    if (i < I.nbody)
        for (int m = I.body_m[i].x; m < I.body_m[i].y; m++) mbody[m] = i;
}

}  // namespace

cudaError_t adj_state(const AdjArgs& A, cudaStream_t st)
{
    const long long nn = (long long)A.s.nx * A.s.ny;
    switch (A.storage) {
    case ST_F64: adj_state_kernel<ST_F64><<<blocks(nn, kT), kT, 0, st>>>(A); break;
    case ST_F32: adj_state_kernel<ST_F32><<<blocks(nn, kT), kT, 0, st>>>(A); break;
    case ST_F16: adj_state_kernel<ST_F16><<<blocks(nn, kT), kT, 0, st>>>(A); break;
    default: adj_state_kernel<ST_BF16><<<blocks(nn, kT), kT, 0, st>>>(A); break;
    }
    return cudaGetLastError();
}

cudaError_t adj_ib_fwd(const AdjArgs& A, cudaStream_t st)
{
    const IbArgs& I = *A.ib;
    adj_ib_nodes_kernel<<<blocks(I.nforced, kT), kT, 0, st>>>(A, I);
    if (A.nst == 16)
        adj_ib_markers_kernel<16><<<blocks(I.nmark, kT), kT, 0, st>>>(A, I);
    else
        adj_ib_markers_kernel<4><<<blocks(I.nmark, kT), kT, 0, st>>>(A, I);
    adj_ib_spread_kernel<<<blocks(I.nforced, kT), kT, 0, st>>>(A, I);
    return cudaGetLastError();
}

cudaError_t adj_collide(const AdjArgs& A, cudaStream_t st)
{
    const long long nn = (long long)A.s.nx * A.s.ny;
    const unsigned g = blocks(nn, kT);
    if (A.learned) {
        switch (A.collision) {
        case CO_MRT: adj_collide_kernel<CO_MRT, true><<<g, kT, 0, st>>>(A); break;
        case CO_RR: adj_collide_kernel<CO_RR, true><<<g, kT, 0, st>>>(A); break;
        default: adj_collide_kernel<CO_BGK, true><<<g, kT, 0, st>>>(A); break;
        }
    } else {
        switch (A.collision) {
        case CO_MRT: adj_collide_kernel<CO_MRT, false><<<g, kT, 0, st>>>(A); break;
        case CO_RR: adj_collide_kernel<CO_RR, false><<<g, kT, 0, st>>>(A); break;
        default: adj_collide_kernel<CO_BGK, false><<<g, kT, 0, st>>>(A); break;
        }
    }
    return cudaGetLastError();
}

cudaError_t adj_inject_moments(const AdjArgs& A, cudaStream_t st)
{
    const long long nn = (long long)A.s.nx * A.s.ny;
    adj_inject_kernel<<<blocks(nn, 256), 256, 0, st>>>(A);
    return cudaGetLastError();
}

cudaError_t adj_ib_back(const AdjArgs& A, cudaStream_t st)
{
    const IbArgs& I = *A.ib;
    adj_ib_back1_kernel<<<blocks(I.nforced, kT), kT, 0, st>>>(A, I);
    if (A.nst == 16)
        adj_ib_back2_kernel<16><<<blocks(I.nmark, kT), kT, 0, st>>>(A, I);
    else
        adj_ib_back2_kernel<4><<<blocks(I.nmark, kT), kT, 0, st>>>(A, I);
    adj_ib_back3_kernel<<<blocks(I.nforced, kT), kT, 0, st>>>(A, I);
    return cudaGetLastError();
}

cudaError_t adj_stream(const AdjArgs& A, cudaStream_t st)
{
    const long long nn = (long long)A.s.nx * A.s.ny;
    adj_stream_kernel<<<blocks(nn, kT), kT, 0, st>>>(A);
    return cudaGetLastError();
}

cudaError_t adj_ib_tables(const IbArgs& ib, int nx, int ny, int* fidx, int* mbody, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(fidx, 0xff, (size_t)nx * ny * sizeof(int), st);
    if (e != cudaSuccess) return e;
    const int n = std::max(ib.nforced, ib.nbody);
    if (n > 0) adj_tables_kernel<<<blocks(n, kT), kT, 0, st>>>(ib, nx, fidx, mbody);
    return cudaGetLastError();
}

}  // namespace ippi
