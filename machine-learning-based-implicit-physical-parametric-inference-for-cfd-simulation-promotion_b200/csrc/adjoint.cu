// adjoint.cu -- the reverse-mode step (see adjoint.h for the stages).
// Channel scene (Zou-He inlet, NEE outlet, bounce-back walls), BGK / MRT / RR,
// tau constant, Smagorinsky, learned or a given field, IB with one
// direct-forcing pass.
#include <algorithm>
#include <cstdlib>

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
// The 14 inputs' derivatives are carried kPass at a time: one forward pass
// of the node collision per group, with only that group's slots seeded.  A
// slot's arithmetic does not depend on the other slots, so the result is
// the one of a single 14-slot pass.  Four slots per pass keep the MRT
// instances nearly free of spills (the 14-slot form spilled 3 KB per
// thread, -Xptxas -v).
constexpr int kPass = 4;

// The learned relaxation time linearised at the node's scalar state, once
// per node for all passes: its value and d tau / d x_k with respect to the
// raw features (the network's forward and backward pass in FP64, the same
// arithmetic as the Dual overload of learned_tau).  in = false: outside the
// training range, the Smagorinsky fallback applies.
struct LrnLin {
    bool in;
    double v;
    double c[kMlpIn];
};

__device__ __forceinline__ LrnLin learned_lin(const float* __restrict__ w, const double* fv, double rho, double ux,
                                              double uy, double tau0)
{
    LrnLin r;
    const float* st = w + kMlpParams;
    double pxx, pxy, pyy, x[kMlpIn];
    pi_neq<double>(fv, rho, ux, uy, 0.0, pxx, pxy, pyy);
    mlp_features<double>(pxx, pxy, pyy, rho, ux, uy, tau0, x);
    r.in = true;
    for (int i = 0; i < kMlpIn; i++) {
        r.in = r.in && x[i] >= double(st[2 * kMlpIn + i]) && x[i] <= double(st[3 * kMlpIn + i]);
        x[i] = (x[i] - double(st[i])) / double(st[kMlpIn + i]);
    }
    if (!r.in) return r;
    double h1[kMlpHid], g2[kMlpHid];
    for (int j = 0; j < kMlpHid; j++) {
        double a = w[kMlpB1 + j];
        for (int i = 0; i < kMlpIn; i++) a += double(w[kMlpW1 + j * kMlpIn + i]) * x[i];
        h1[j] = tanh(a);
    }
    double z = w[kMlpB3];
    for (int j = 0; j < kMlpHid; j++) {
        double a = w[kMlpB2 + j];
        for (int i = 0; i < kMlpHid; i++) a += double(w[kMlpW2 + j * kMlpHid + i]) * h1[i];
        const double h2 = tanh(a);
        z += double(w[kMlpW3 + j]) * h2;
        g2[j] = double(w[kMlpW3 + j]) * (1.0 - h2 * h2);
    }
    double gx[kMlpIn] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < kMlpHid; i++) {
        double g1 = 0.0;
        for (int j = 0; j < kMlpHid; j++) g1 += double(w[kMlpW2 + j * kMlpHid + i]) * g2[j];
        g1 *= 1.0 - h1[i] * h1[i];
        for (int k = 0; k < kMlpIn; k++) gx[k] += double(w[kMlpW1 + i * kMlpIn + k]) * g1;
    }
    const double os = st[4 * kMlpIn];
    const double sig = 1.0 / (1.0 + exp(-z));
    r.v = tau0 + os * (fmax(z, 0.0) + log1p(exp(-fabs(z))));
    for (int k = 0; k < kMlpIn; k++) r.c[k] = os * sig * gx[k] / double(st[kMlpIn + k]);
    return r;
}

template <int CO, bool LRN, int j0>
__device__ __forceinline__ void collide_vjp_pass(const AdjArgs& A, long long node, int fi, const double* fv,
                                                 const double* lam, const LrnLin& lin, double* g)
{
    using P = Dual<kPass>;
    const StepArgs& a = A.s;
    // slots are compile-time constants: the duals stay in registers
    auto sd = [](double v, int q) {
        const int sl = q - j0;
        return (sl >= 0 && sl < kPass) ? P::seed(v, sl) : P(v);
    };
    P f[9];
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = sd(fv[k], k);
    P rho, ux, uy;
    macros<P>(f, P(0.0), rho, ux, uy);
    P fxd(0.0), fyd(0.0);
    if (fi >= 0) {
        ux = sd(A.ib_uc[fi].x, 9);
        uy = sd(A.ib_uc[fi].y, 10);
        fxd = sd(A.ib_fn[fi].x, 11);
        fyd = sd(A.ib_fn[fi].y, 12);
    }
    const P tau0(a.tau0), cs(a.cs);
    P tau;
    if (a.les == 3) {
        tau = P(a.tau_field[node]);
    } else if (LRN && lin.in) {
        P pxx, pxy, pyy, x[kMlpIn];
        pi_neq<P>(f, rho, ux, uy, P(0.0), pxx, pxy, pyy);
        mlp_features<P>(pxx, pxy, pyy, rho, ux, uy, tau0, x);
        tau = P(lin.v);
#pragma unroll
        for (int k = 0; k < kMlpIn; k++)
#pragma unroll
            for (int i = 0; i < kPass; i++) tau.d[i] += lin.c[k] * x[k].d[i];
    } else {
        // constant, Smagorinsky, or the learned model's Smagorinsky fallback
        tau = node_tau<P, false>(f, rho, ux, uy, P(0.0), a.les, tau0, cs);
    }
    if (13 - j0 >= 0 && 13 - j0 < kPass) tau.d[13 - j0] += 1.0;
    collide_node<P, CO>(f, rho, ux, uy, P(0.0), tau);
    if (fi >= 0) add_force<P, CO>(f, ux, uy, fxd, fyd, tau0, tau);
#pragma unroll
    for (int j = 0; j < kPass; j++) {
        if (j0 + j >= kDual) break;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 9; k++) s += lam[k] * f[k].d[j];
        g[j0 + j] = s;
    }
}

template <int CO, bool LRN>
__global__ void __launch_bounds__(kT) adj_collide_kernel(const AdjArgs A)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const long long node = blockIdx.x * (long long)kT + threadIdx.x;
    if (node >= nn) return;
    const int fi = A.fidx ? A.fidx[node] : -1;
    double fv[9], lam[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        fv[k] = A.ft[k * nn + node];
        lam[k] = A.lam_out[k * nn + node];
    }
    // the node's scalar moments (the IB-corrected velocity on forced nodes)
    double rv, uxv, uyv;
    macros<double>(fv, 0.0, rv, uxv, uyv);
    if (fi >= 0) {
        uxv = A.ib_uc[fi].x;
        uyv = A.ib_uc[fi].y;
    }
    LrnLin lin;
    lin.in = false;
    if (LRN && a.les == 2) lin = learned_lin(a.mlp, fv, rv, uxv, uyv, a.tau0);
    double g[kDual];
    static_assert(4 * kPass >= kDual, "four passes cover the inputs");
    collide_vjp_pass<CO, LRN, 0 * kPass>(A, node, fi, fv, lam, lin, g);
    collide_vjp_pass<CO, LRN, 1 * kPass>(A, node, fi, fv, lam, lin, g);
    collide_vjp_pass<CO, LRN, 2 * kPass>(A, node, fi, fv, lam, lin, g);
    collide_vjp_pass<CO, LRN, 3 * kPass>(A, node, fi, fv, lam, lin, g);
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
        double r = rv, vx = uxv, vy = uyv, pxx, pxy, pyy, x[kMlpIn];
        pi_neq<double>(fv, r, vx, vy, 0.0, pxx, pxy, pyy);
        mlp_features<double>(pxx, pxy, pyy, r, vx, vy, a.tau0, x);
        const float* st = a.mlp + kMlpParams;
        bool in = true;
        for (int i = 0; i < kMlpIn; i++) in = in && x[i] >= double(st[2 * kMlpIn + i]) && x[i] <= double(st[3 * kMlpIn + i]);
        for (int i = 0; i < kMlpIn; i++) A.xs[node * kMlpIn + i] = in ? (x[i] - double(st[i])) / double(st[kMlpIn + i]) : 0.0;
        A.up[node] = in ? g[13] * double(st[4 * kMlpIn]) : 0.0;
    }
}

// ---- the learned relaxation time linearised, one warp per node ---------------
// learned_lin's numbers for every node (value, d tau / d x[6] and the range
// flag into A.lin[node][8]), with lane j = neuron j of both hidden layers:
// row j of W2 in registers, its columns from shared memory, the other lanes'
// activations by shuffle.  The features are computed on every lane.
__global__ void __launch_bounds__(kT) adj_lin_kernel(const AdjArgs A)
{
    __shared__ double w2s[kMlpHid * kMlpHid];
    __shared__ double hs[kT / 32][kMlpHid], gs[kT / 32][kMlpHid];  // per warp: h1, then g2
    const StepArgs& a = A.s;
    const float* w = a.mlp;
    const float* st = w + kMlpParams;
    for (int p = threadIdx.x; p < kMlpHid * kMlpHid; p += kT) w2s[p] = double(w[kMlpW2 + p]);
    const int j = threadIdx.x & 31;
    double w1[kMlpIn], w2r[kMlpHid];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) w1[i] = double(w[kMlpW1 + j * kMlpIn + i]);
#pragma unroll
    for (int i = 0; i < kMlpHid; i++) w2r[i] = double(w[kMlpW2 + j * kMlpHid + i]);
    const double b1 = double(w[kMlpB1 + j]), b2 = double(w[kMlpB2 + j]), w3 = double(w[kMlpW3 + j]);
    const double b3 = double(w[kMlpB3]), os = double(st[4 * kMlpIn]);
    __syncthreads();
    const long long nn = (long long)a.nx * a.ny;
    const long long nw = (long long)gridDim.x * (kT / 32);
    // 32 nodes per round: lane l computes node base + l's features, then the
    // warp runs the network for each of the 32 in turn
    for (long long base = (blockIdx.x * (long long)(kT / 32) + (threadIdx.x >> 5)) * 32; base < nn;
         base += nw * 32) {
        const long long mine = base + j;
        double xl[kMlpIn];
        bool inl = false;
        // a node whose adjoint is zero contributes nothing: no network pass
        bool live = false;
        if (mine < nn)
#pragma unroll
            for (int k = 0; k < 9; k++) live = live || A.lam_out[k * nn + mine] != 0.0;
        if (live) {
            double f[9], rho, ux, uy, pxx, pxy, pyy;
#pragma unroll
            for (int k = 0; k < 9; k++) f[k] = A.ft[k * nn + mine];
            macros<double>(f, 0.0, rho, ux, uy);
            const int fi = A.fidx ? A.fidx[mine] : -1;
            if (fi >= 0) {
                ux = A.ib_uc[fi].x;
                uy = A.ib_uc[fi].y;
            }
            pi_neq<double>(f, rho, ux, uy, 0.0, pxx, pxy, pyy);
            mlp_features<double>(pxx, pxy, pyy, rho, ux, uy, a.tau0, xl);
            inl = true;
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) {
                inl = inl && xl[i] >= double(st[2 * kMlpIn + i]) && xl[i] <= double(st[3 * kMlpIn + i]);
                xl[i] = (xl[i] - double(st[i])) / double(st[kMlpIn + i]);
            }
        }
        const int nq = nn - base < 32 ? (int)(nn - base) : 32;
        // lane q keeps node base + q's z and d z / d x, and finishes it below
        double zm = 0.0, gm[kMlpIn] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < nq; q++) {
            const bool in = __shfl_sync(0xffffffffu, (int)inl, q) != 0;
            if (!in) continue;  // the same node on every lane
            double x[kMlpIn];
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) x[i] = __shfl_sync(0xffffffffu, xl[i], q);
            double a1 = b1;
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) a1 += w1[i] * x[i];
            const double h1 = tanh(a1);
            // the other lanes' values through shared memory, summed in four
            // independent chains
            const int wp = threadIdx.x >> 5;
            hs[wp][j] = h1;
            __syncwarp();
            double p2[4] = {b2, 0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < kMlpHid; i++) p2[i & 3] += w2r[i] * hs[wp][i];
            const double h2 = tanh((p2[0] + p2[1]) + (p2[2] + p2[3]));
            double z = w3 * h2;
#pragma unroll
            for (int o = 16; o; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
            z += b3;
            const double g2 = w3 * (1.0 - h2 * h2);
            gs[wp][j] = g2;
            __syncwarp();
            double p1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < kMlpHid; k++) p1[k & 3] += w2s[k * kMlpHid + j] * gs[wp][k];
            double g1 = (p1[0] + p1[1]) + (p1[2] + p1[3]);
            g1 *= 1.0 - h1 * h1;
            __syncwarp();  // hs / gs are rewritten for the next node
#pragma unroll
            for (int m = 0; m < kMlpIn; m++) {
                double v = w1[m] * g1;
#pragma unroll
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (j == q) gm[m] = v;
            }
            if (j == q) zm = z;
        }
        if (j < nq) {
            double* out = A.lin + mine * 8;
            if (inl) {
                const double sig = 1.0 / (1.0 + exp(-zm));
                out[0] = a.tau0 + os * (fmax(zm, 0.0) + log1p(exp(-fabs(zm))));
#pragma unroll
                for (int m = 0; m < kMlpIn; m++) out[1 + m] = os * sig * gm[m] / double(st[kMlpIn + m]);
                out[7] = 1.0;
            } else {
                out[7] = 0.0;
            }
        }
    }
}

// ---- MRT collision: the vector-Jacobian product in reverse mode --------------
// g = lambda^T d(out)/d(inputs) of collide_mrt (rb = 0) written out by hand:
// out = f - C a(m(f), rho, u, 1/tau) with the moment combinations m, the
// six relaxed moments a and their scatter C of collide_mrt.  Only the small
// pieces that are not linear in f use dual numbers: the relaxation time as
// a function of (f, rho, u) (Dual<12>) and the forcing term of forced nodes
// as a function of (u, F, tau) (Dual<5>).  Then the moments' adjoint:
// rho = sum f, u = j / rho (on forced nodes u is the corrected velocity, an
// input of its own).  The same derivatives as adj_collide_kernel<CO_MRT>
// to rounding, without its 14-slot duals.
template <bool LRN>
__global__ void __launch_bounds__(kT) adj_collide_mrt_kernel(const AdjArgs A)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const long long node = blockIdx.x * (long long)kT + threadIdx.x;
    if (node >= nn) return;
    const int fi = A.fidx ? A.fidx[node] : -1;
    double f[9], lam[9];
    bool live = false;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        f[k] = A.ft[k * nn + node];
        lam[k] = A.lam_out[k * nn + node];
        live = live || lam[k] != 0.0;
    }
    if (!live) {
        // lambda = 0: every product is zero (the relaxation time is not needed)
#pragma unroll
        for (int k = 0; k < 9; k++) A.lam_ft[k * nn + node] = 0.0;
        if (fi >= 0) {
            A.lam_uc[fi] = make_double2(0.0, 0.0);
            A.lam_fn[fi] = make_double2(0.0, 0.0);
        }
        if (LRN && A.xs) {
#pragma unroll
            for (int i = 0; i < kMlpIn; i++) A.xs[node * kMlpIn + i] = 0.0;
            A.up[node] = 0.0;
        }
        return;
    }
    double rho, ux, uy;
    macros<double>(f, 0.0, rho, ux, uy);
    double fx = 0.0, fy = 0.0;
    if (fi >= 0) {
        ux = A.ib_uc[fi].x;
        uy = A.ib_uc[fi].y;
        fx = A.ib_fn[fi].x;
        fy = A.ib_fn[fi].y;
    }
    // relaxation time and its gradient with respect to (f, rho, ux, uy)
    using T12 = Dual<12>;
    double tau, dtau[12];
#pragma unroll
    for (int i = 0; i < 12; i++) dtau[i] = 0.0;
    LrnLin lin;
    lin.in = false;
    if (a.les == 3) {
        tau = a.tau_field[node];
    } else if (a.les == 0 && !LRN) {
        tau = a.tau0;
    } else {
        T12 fd[9];
#pragma unroll
        for (int k = 0; k < 9; k++) fd[k] = T12::seed(f[k], k);
        const T12 rd = T12::seed(rho, 9), ud = T12::seed(ux, 10), vd = T12::seed(uy, 11);
        T12 pxx, pxy, pyy;
        pi_neq<T12>(fd, rd, ud, vd, T12(0.0), pxx, pxy, pyy);
        T12 td;
        if (LRN) {
            // linearised per node by adj_lin_kernel
            const double* l = A.lin + node * 8;
            lin.in = l[7] != 0.0;
            if (lin.in) {
                lin.v = l[0];
#pragma unroll
                for (int k = 0; k < kMlpIn; k++) lin.c[k] = l[1 + k];
            }
        }
        if (LRN && lin.in) {
            T12 x[kMlpIn];
            mlp_features<T12>(pxx, pxy, pyy, rd, ud, vd, T12(a.tau0), x);
            td = T12(lin.v);
#pragma unroll
            for (int k = 0; k < kMlpIn; k++)
#pragma unroll
                for (int i = 0; i < 12; i++) td.d[i] += lin.c[k] * x[k].d[i];
        } else {
            td = les_tau<T12>(pxx, pxy, pyy, rd, T12(a.tau0), T12(a.cs));
        }
        tau = td.v;
#pragma unroll
        for (int i = 0; i < 12; i++) dtau[i] = td.d[i];
    }
    // forward quantities of collide_mrt
    const double u2 = ux * ux + uy * uy, om = 1.0 / tau;
    const double m7 = (f[1] + f[3]) - (f[2] + f[4]);
    const double m8 = f[5] - f[6] + f[7] - f[8];
    const double k1 = 1.2 * (1.0 / 36.0), k2 = 1.1 * (1.0 / 36.0), k4 = 1.2 * (1.0 / 12.0);
    // adjoints of the relaxed moments a1 a2 a4 a6 a7 a8
    const double mu1 = -(-4.0 * lam[0] - lam[1] - lam[2] - lam[3] - lam[4] + 2.0 * (lam[5] + lam[6] + lam[7] + lam[8]));
    const double mu2 = -(4.0 * lam[0] - 2.0 * (lam[1] + lam[2] + lam[3] + lam[4]) + lam[5] + lam[6] + lam[7] + lam[8]);
    const double mu4 = -(-2.0 * lam[1] + 2.0 * lam[3] + lam[5] - lam[6] - lam[7] + lam[8]);
    const double mu6 = -(-2.0 * lam[2] + 2.0 * lam[4] + lam[5] + lam[6] - lam[7] - lam[8]);
    const double mu7 = -(lam[1] - lam[2] + lam[3] - lam[4]);
    const double mu8 = -(lam[5] - lam[6] + lam[7] - lam[8]);
    const double g1 = mu1 * k1, g2 = mu2 * k2, g4 = mu4 * k4, g6 = mu6 * k4, g7 = mu7 * om * 0.25,
                 g8 = mu8 * om * 0.25;
    double grho = g1 * (2.0 - 3.0 * u2) + g2 * (3.0 * u2 - 1.0) + g4 * ux + g6 * uy - g7 * (ux * ux - uy * uy) -
                  g8 * ux * uy;
    double gux = -6.0 * rho * ux * g1 + 6.0 * rho * ux * g2 + rho * g4 - 2.0 * rho * ux * g7 - rho * uy * g8;
    double guy = -6.0 * rho * uy * g1 + 6.0 * rho * uy * g2 + rho * g6 + 2.0 * rho * uy * g7 - rho * ux * g8;
    double gtau = -(mu7 * (m7 - rho * (ux * ux - uy * uy)) * 0.25 + mu8 * (m8 - rho * ux * uy) * 0.25) * om * om;
    double gf[9];
    gf[0] = lam[0] - 4.0 * g1 + 4.0 * g2;
    gf[1] = lam[1] - g1 - 2.0 * g2 - 2.0 * g4 + g7;
    gf[2] = lam[2] - g1 - 2.0 * g2 - 2.0 * g6 - g7;
    gf[3] = lam[3] - g1 - 2.0 * g2 + 2.0 * g4 + g7;
    gf[4] = lam[4] - g1 - 2.0 * g2 + 2.0 * g6 - g7;
    gf[5] = lam[5] + 2.0 * g1 + g2 + g4 + g6 + g8;
    gf[6] = lam[6] + 2.0 * g1 + g2 - g4 + g6 - g8;
    gf[7] = lam[7] + 2.0 * g1 + g2 - g4 - g6 + g8;
    gf[8] = lam[8] + 2.0 * g1 + g2 + g4 - g6 - g8;
    // the forcing term of a forced node, a function of (u, F, tau)
    double gfx = 0.0, gfy = 0.0;
    if (fi >= 0) {
        using T5 = Dual<5>;
        T5 z[9];
        add_force<T5, CO_MRT>(z, T5::seed(ux, 0), T5::seed(uy, 1), T5::seed(fx, 2), T5::seed(fy, 3), T5(a.tau0),
                              T5::seed(tau, 4));
        double gz[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 9; k++)
#pragma unroll
            for (int i = 0; i < 5; i++) gz[i] += lam[k] * z[k].d[i];
        gux += gz[0];
        guy += gz[1];
        gfx = gz[2];
        gfy = gz[3];
        gtau += gz[4];
    }
    // the relaxation time's dependence on (f, rho, u)
#pragma unroll
    for (int k = 0; k < 9; k++) gf[k] += gtau * dtau[k];
    grho += gtau * dtau[9];
    gux += gtau * dtau[10];
    guy += gtau * dtau[11];
    // the moments: rho = sum f; u = j / rho unless u is the corrected velocity
    if (fi >= 0) {
        A.lam_uc[fi] = make_double2(gux, guy);
        A.lam_fn[fi] = make_double2(gfx, gfy);
    } else {
        const double gjx = gux / rho, gjy = guy / rho;
        grho -= gux * ux / rho + guy * uy / rho;
#pragma unroll
        for (int k = 0; k < 9; k++) gf[k] += EX(k) * gjx + EY(k) * gjy;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) A.lam_ft[k * nn + node] = gf[k] + grho;
    if (A.grad_tau && a.les == 3) A.grad_tau[node] += gtau;
    if (LRN && A.xs) {
        double pxx, pxy, pyy, x[kMlpIn];
        pi_neq<double>(f, rho, ux, uy, 0.0, pxx, pxy, pyy);
        mlp_features<double>(pxx, pxy, pyy, rho, ux, uy, a.tau0, x);
        const float* st = a.mlp + kMlpParams;
        bool in = true;
        for (int i = 0; i < kMlpIn; i++) in = in && x[i] >= double(st[2 * kMlpIn + i]) && x[i] <= double(st[3 * kMlpIn + i]);
        for (int i = 0; i < kMlpIn; i++) A.xs[node * kMlpIn + i] = in ? (x[i] - double(st[i])) / double(st[kMlpIn + i]) : 0.0;
        A.up[node] = in ? gtau * double(st[4 * kMlpIn]) : 0.0;
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
// The pull maps (destination, direction) one to one onto (source, direction)
// except at the lattice's edges, whose maps are folded into the destination
// adjoint first (adj_edges_kernel, one thread per row):
//   outlet  x = nx-1 pulls nothing: its f~ is the NEE of node nx-2 (f~ =
//           feq(rho0, u_b) + f~_b - feq(rho_b, u_b)), so its adjoint is
//           transposed onto node nx-2's and then cleared;
//   inlet   x = 0: the regularised Zou-He map of the pulled populations is
//           linear; its transposed Jacobian (one dual evaluation) replaces
//           the node's adjoint;
// and walls, where a pull from beyond y bounces back (the source is the node
// itself, opposite direction).  adj_gather_kernel then writes every entry of
// lam_in from exactly one term: no atomics, the same bits on every run.
__global__ void __launch_bounds__(kT) adj_edges_kernel(const AdjArgs A)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const int y = blockIdx.x * kT + threadIdx.x;
    if (y >= a.ny) return;
    {
        const long long node = (long long)y * a.nx + (a.nx - 1), b = node - 1;
        double lam[9];
#pragma unroll
        for (int k = 0; k < 9; k++) lam[k] = A.lam_ft[k * nn + node];
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
#pragma unroll
        for (int k = 0; k < 9; k++) {
            A.lam_ft[k * nn + b] += lam[k] + gr + (gx * (EX(k) - ux) + gy * (EY(k) - uy)) / rb;
            A.lam_ft[k * nn + node] = 0.0;
        }
    }
    {
        const long long node = (long long)y * a.nx;
        using D9 = Dual<9>;
        D9 g[9];
#pragma unroll
        for (int k = 0; k < 9; k++) g[k] = D9::seed(0.0, k);
        zh_inlet<D9>(g, D9(inlet_profile<double>(y, a.ny, a.u_in)), D9(0.0));
        double lam[9];
#pragma unroll
        for (int k = 0; k < 9; k++) lam[k] = A.lam_ft[k * nn + node];
#pragma unroll
        for (int j = 0; j < 9; j++) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++) v += lam[k] * g[k].d[j];
            A.lam_ft[j * nn + node] = v;
        }
    }
}

// lam_in(x, y, j): the adjoint of the destination that pulled f_in_j(x, y) --
// (x + e_j) when that is inside the lattice in y (nothing beyond x), else the
// node itself in direction opp(j) (bounce-back)
__global__ void __launch_bounds__(kT) adj_gather_kernel(const AdjArgs A)
{
    const StepArgs& a = A.s;
    const long long nn = (long long)a.nx * a.ny;
    const long long node = blockIdx.x * (long long)kT + threadIdx.x;
    if (node >= nn) return;
    const int x = (int)(node % a.nx), y = (int)(node / a.nx);
#pragma unroll
    for (int j = 0; j < 9; j++) {
        const int dy = y + EY(j), dx = x + EX(j);
        double v;
        if (dy < 0 || dy >= a.ny)
            v = A.lam_ft[OPP(j) * nn + node];
        else
            v = (dx >= 0 && dx < a.nx) ? A.lam_ft[j * nn + (long long)dy * a.nx + dx] : 0.0;
        A.lam_in[j * nn + node] = v;
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
    // IPPI_TEST_ADJ_DUAL=1 (tests only): the dual-number MRT kernel, the
    // reference the reverse-mode one is compared with
    static const bool mrt_dual = [] {
        const char* e = std::getenv("IPPI_TEST_ADJ_DUAL");
        return e && e[0] == '1';
    }();
    if (A.collision == CO_MRT && !mrt_dual) {
        if (A.learned) {
            adj_lin_kernel<<<(unsigned)std::min<long long>(blocks(nn, kT), 148 * 16), kT, 0, st>>>(A);
            adj_collide_mrt_kernel<true><<<g, kT, 0, st>>>(A);
        } else {
            adj_collide_mrt_kernel<false><<<g, kT, 0, st>>>(A);
        }
        return cudaGetLastError();
    }
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
    adj_edges_kernel<<<blocks(A.s.ny, kT), kT, 0, st>>>(A);
    adj_gather_kernel<<<blocks(nn, kT), kT, 0, st>>>(A);
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
