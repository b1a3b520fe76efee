// lbm_common.cuh -- device-side building blocks of the D2Q9 step for sm_100a.
//
// Populations live in HBM as structure-of-arrays planes f[k][y][pitch] (x
// fastest).  FP32/FP16/BF16 storage keeps them shifted by w_k * rho0 (the
// lattice weight times the reference density) and FP16 additionally scaled by
// 1024, so the stored numbers are the small deviations from rest; arithmetic
// is FP32 on those shifted values.  FP64 storage keeps the reference's plain
// populations and FP64 arithmetic, for parity with the FP64 CPU path.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "dual.cuh"

namespace ippi {

enum { ST_F64 = 0, ST_F32 = 1, ST_F16 = 2, ST_BF16 = 3 };
enum { CO_BGK = 0, CO_MRT = 1, CO_RR = 2 };
enum { SC_REF = 0, SC_CHANNEL = 1 };

// per-node flags.  On the device: NF_DEFER (the bulk kernel skips the node,
// another kernel finishes it), NF_SOLID (a solid node: never updated) and
// NF_SBND (a fluid node with a link into a solid: halfway bounce-back on
// that link).  NF_EXPORT (boundary-net inputs) and NF_IB (immersed-boundary
// stencil nodes) live in the host-side tables only.
enum : uint8_t { NF_EXPORT = 1, NF_DEFER = 2, NF_IB = 4, NF_SOLID = 8, NF_SBND = 16 };

// step kernel modes
enum { MODE_STEP = 0, MODE_INIT = 1, MODE_MAT = 2, MODE_MAT_INIT = 3 };

// Resident 256-thread blocks per SM the step kernels are compiled for: 8 in
// FP32 arithmetic (32 registers), 4 in FP64 (64 registers: at 32 the FP64
// instances spilled 0.5-2.7 KB per thread), fewer with the learned network's
// hidden layer in registers.
template <int S, bool LRN>
constexpr int step_min_blocks()
{
    return LRN ? (S == ST_F64 ? 2 : 3) : (S == ST_F64 ? 4 : 8);
}

// D2Q9 velocity order of the reference (NodeAndLattice.cpp:3-13):
// 0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE.
__host__ __device__ constexpr int EX(int k)
{
    return k == 1 || k == 5 || k == 8 ? 1 : (k == 3 || k == 6 || k == 7 ? -1 : 0);
}
__host__ __device__ constexpr int EY(int k)
{
    return k == 2 || k == 5 || k == 6 ? 1 : (k == 4 || k == 7 || k == 8 ? -1 : 0);
}
__host__ __device__ constexpr int OPP(int k)
{
    return k == 0 ? 0 : (k <= 4 ? ((k + 1) % 4) + 1 : ((k - 5 + 2) % 4) + 5);
}
static_assert(OPP(1) == 3 && OPP(2) == 4 && OPP(3) == 1 && OPP(4) == 2, "opp");
static_assert(OPP(5) == 7 && OPP(6) == 8 && OPP(7) == 5 && OPP(8) == 6, "opp");

template <typename C>
__host__ __device__ constexpr C WK(int k)
{
    return k == 0 ? C(4.0 / 9.0) : (k <= 4 ? C(1.0 / 9.0) : C(1.0 / 36.0));
}

// device step counter / status word, one per lattice
// The kernels of a step with parity p read the user step number from t[p]
// and one thread of the bulk kernel writes t[p] + 1 into t[p ^ 1] for the
// next step, so concurrent kernels of one step never see a changing value.
struct Ctr {
    int t[2];         // user time step (feeds the averages), by step parity
    int err;          // 1 once rho left [0,10] or became NaN; 2 an IB barrier wait ran
                      // out; 3 a boundary-net weight copy wait ran out
    int err_t;        // first step where that happened
};

// ----------------------------------------------------------------------------
// storage traits
// ----------------------------------------------------------------------------
template <int S> struct Store;
template <> struct Store<ST_F64> {
    using T = double;
    using C = double;
    static constexpr bool kShift = false;
    __device__ static C ld(T v) { return v; }
    __device__ static T st(C v) { return v; }
};
template <> struct Store<ST_F32> {
    using T = float;
    using C = float;
    static constexpr bool kShift = true;
    __device__ static C ld(T v) { return v; }
    __device__ static T st(C v) { return v; }
};
template <> struct Store<ST_F16> {
    using T = __half;
    using C = float;
    static constexpr bool kShift = true;
    __device__ static C ld(T v) { return __half2float(v) * (1.0f / 1024.0f); }
    __device__ static T st(C v) { return __float2half_rn(v * 1024.0f); }
};
template <> struct Store<ST_BF16> {
    using T = __nv_bfloat16;
    using C = float;
    static constexpr bool kShift = true;
    __device__ static C ld(T v) { return __bfloat162float(v); }
    __device__ static T st(C v) { return __float2bfloat16_rn(v); }
};

// ----------------------------------------------------------------------------
// node physics (C = compute type).  `rb` is the population shift base: rho0
// for shifted storage, 0 for FP64.  Populations f[] are f_k - w_k * rb.
// ----------------------------------------------------------------------------

// Moments: rho = rb + sum f, u = sum f e / rho (zero below rho 1e-6), the
// rule of Lattice::CalMacro (NodeAndLattice.cpp:196-227).
template <typename C>
__device__ __forceinline__ void macros(const C* f, C rb, C& rho, C& ux, C& uy)
{
    C s = ((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7])) + f[8];
    C jx = (f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7]);
    C jy = (f[2] - f[4]) + (f[5] + f[6]) - (f[7] + f[8]);
    rho = rb + s;
    if (rho < C(1e-6)) {
        ux = C(0);
        uy = C(0);
    } else {
        C inv = C(1) / rho;
        ux = jx * inv;
        uy = jy * inv;
    }
}

// Second-order equilibrium (Lattice::Compute_feq, NodeAndLattice.cpp:124-149)
// in shifted form: feq_k - w_k rb = w_k (rho - rb) + w_k rho (3 eu + 4.5 eu^2 - 1.5 u^2).
template <typename C>
__device__ __forceinline__ void equilibrium(C rho, C ux, C uy, C rb, C* feq)
{
    const C dr = rho - rb;
    const C usq = C(1.5) * (ux * ux + uy * uy);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const C eu = C(EX(k)) * ux + C(EY(k)) * uy;
        feq[k] = WK<C>(k) * dr + WK<C>(k) * rho * (C(3) * eu + C(4.5) * eu * eu - usq);
    }
}

// Non-equilibrium stress Pi_neq = sum e e (f - feq) from moments: the
// second moments of the 2nd-order equilibrium are rho/3 + rho u u exactly.
template <typename C>
__device__ __forceinline__ void pi_neq(const C* f, C rho, C ux, C uy, C rb, C& pxx, C& pxy,
                                       C& pyy)
{
    const C dr3 = (rho - rb) * C(1.0 / 3.0);
    const C diag = f[5] + f[6] + f[7] + f[8];
    pxx = (f[1] + f[3] + diag) - dr3 - rho * ux * ux;
    pyy = (f[2] + f[4] + diag) - dr3 - rho * uy * uy;
    pxy = (f[5] - f[6] + f[7] - f[8]) - rho * ux * uy;
}

// Smagorinsky "hybrid" relaxation time (Mesh::CaculateLESTau, mesh.cpp:877-910):
// S = -3/(2 rho tau0) Pi_neq, Q = sqrt(2 S:S), tau = (sqrt(tau0^2 + 18 Cs^2 Q/rho) + tau0)/2.
template <typename C>
__device__ __forceinline__ C les_tau(C pxx, C pxy, C pyy, C rho, C tau0, C cs)
{
    const C c = C(-1.5) / (rho * tau0);
    const C sxx = pxx * c, sxy = pxy * c, syy = pyy * c;
    const C s2 = sxx * sxx + C(2) * sxy * sxy + syy * syy;
    const C q = sqrt(C(2) * s2);
    const C inv_rho = -c * tau0 * C(2.0 / 3.0);  // 1/rho without a second division
    const C g1 = tau0 * tau0 + C(18) * cs * cs * q * inv_rho;
    return (sqrt(g1) + tau0) * C(0.5);
}

// The closures of Mesh::CaculateLESTau left as alternatives in the reference
// (mesh.cpp:934-1071, 2113-2146), delta = 1.  g = (du/dx, du/dy, dv/dx,
// dv/dy), the forward differences of GetDuxDx .. GetDuyDy.
//
// WALE (mesh.cpp:934-967): Cw = 0.45,
// nu_t = Cw^2 (Gd:Gd)^3/2 / ((S:S)^5/2 + (Gd:Gd)^5/4 + 1e-12), tau = tau0 + 3 nu_t.
template <typename C>
__device__ __forceinline__ C wale_tau(const C* g, C tau0)
{
    const C gxx = g[0], gxy = g[1], gyx = g[2], gyy = g[3];
    const C sxy = C(0.5) * (gxy + gyx);
    const C ss = gxx * gxx + sxy * sxy + sxy * sxy + gyy * gyy;
    const C gxx2 = gxx * gxx + gxy * gyx, gxy2 = gxx * gxy + gxy * gyy;
    const C gyx2 = gyx * gxx + gyy * gyx, gyy2 = gyx * gxy + gyy * gyy;
    const C grr2 = gxx * gxx + gxy * gyx + gyx * gxy + gyy * gyy;
    const C dxx = C(0.5) * (gxx2 + gxx2) - grr2 / C(3.0);
    const C dxy = C(0.5) * (gxy2 + gyx2);
    const C dyy = C(0.5) * (gyy2 + gyy2) - grr2 / C(3.0);
    const C gg = dxx * dxx + dxy * dxy + dxy * dxy + dyy * dyy;
    // x^1.5 = x sqrt(x), x^2.5 = x^2 sqrt(x), x^1.25 = x sqrt(sqrt(x)): the
    // same values to rounding, without a general power
    const C rg = sqrt(gg), rs = sqrt(ss);
    const C vt = C(0.45 * 0.45) * (gg * rg) / (ss * ss * rs + gg * sqrt(rg) + C(1e-12));
    return tau0 + C(3) * vt;
}

// Coherent-structure model (mesh.cpp:1034-1071 with ComputeDynamicCs,
// 2113-2146): F = |Q/E| from the gradient's rotation and strain,
// C = F^3/2 (1 - F) / 11 (0.016 where E = 0), nu_t = C sqrt(2 Pi_neq:Pi_neq)
// on the unscaled non-equilibrium moments, tau = tau0 + 3 nu_t.
template <typename C>
__device__ __forceinline__ C csm_tau(const C* g, C pxx, C pxy, C pyy, C tau0)
{
    const C sxy = C(0.5) * (g[1] + g[2]);
    const C ss = g[0] * g[0] + sxy * sxy + sxy * sxy + g[3] * g[3];
    const C wxy = C(0.5) * (g[1] - g[2]);
    const C ww = C(2) * wxy * wxy;
    const C q = C(0.5) * (ww - ss), e = C(0.5) * (ww + ss);
    C ccsm = C(0.016);
    if (e != C(0)) {
        const C fcs = fabs(q / e);
        ccsm = (C(1) / C(11.0)) * (fcs * sqrt(fcs)) * (C(1) - fcs);
    }
    const C s2 = pxx * pxx + pxy * pxy + pxy * pxy + pyy * pyy;
    return tau0 + C(3) * (ccsm * sqrt(C(2) * s2));
}

// Wall-damped ("dynamic") Cs (mesh.cpp:968-1000): Cs = 3 / (1 + 1.71828^(6 -
// d)) at wall distance d, Q = sqrt(2 Pi_neq:Pi_neq) unscaled,
// tau = tau0 + (sqrt(tau0^2 + 18 Cs^2 Q / rho) - tau0) / 2.
template <typename C>
__device__ __forceinline__ C dyncs_tau(C pxx, C pxy, C pyy, C rho, C tau0, C dist)
{
    const C sc = C(3) / (C(1) + pow(C(1.71828), C(6) - dist));
    const C q = sqrt(C(2) * (pxx * pxx + pxy * pxy + pxy * pxy + pyy * pyy));
    return tau0 + (sqrt(tau0 * tau0 + C(18) * sc * sc * q / rho) - tau0) / C(2);
}

// BGK (Lattice::ComputeBGKCollision, NodeAndLattice.cpp:150-161).
template <typename C>
__device__ __forceinline__ void collide_bgk(C* f, const C* feq, C tau)
{
    const C om = C(1) / tau;
    const C a = C(1) - om;
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = a * f[k] + feq[k] * om;
}

// Regularised collision (Lattice::ComputeRRCollision, NodeAndLattice.cpp:228-288):
// fcol = feq + (1 - 1/tau) 4.5 w_k Q_k : Pi_neq,  Q_k = e_k e_k - I/3.
template <typename C>
__device__ __forceinline__ void collide_rr(C* f, const C* feq, C pxx, C pxy, C pyy, C tau)
{
    const C a = C(1) - C(1) / tau;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const C qxx = C(EX(k) * EX(k)) - C(1.0 / 3.0);
        const C qyy = C(EY(k) * EY(k)) - C(1.0 / 3.0);
        const C qxy = C(EX(k) * EY(k));
        const C f1 = C(4.5) * WK<C>(k) * (qxx * pxx + C(2) * qxy * pxy + qyy * pyy);
        f[k] = feq[k] + a * f1;
    }
}

// Lallemand-Luo MRT with the reference's rates s = {0, 1.2, 1.1, 0, 1.2, 0,
// 1.2, 1/tau, 1/tau} (NodeAndLattice.cpp:290-360).  Only the six
// non-conserved moments relax, so fcol = f - M^-1 S (m - m_eq) reduces to six
// moment differences and the columns of M^-1 = M^T diag(1/|row|^2).
template <typename C>
__device__ __forceinline__ void collide_mrt(C* f, C rho, C ux, C uy, C rb, C tau)
{
    const C dr = rho - rb;
    const C u2 = ux * ux + uy * uy;
    const C s15 = f[1] + f[2] + f[3] + f[4];
    const C s58 = f[5] + f[6] + f[7] + f[8];
    const C m1 = C(-4) * f[0] - s15 + C(2) * s58;
    const C m2 = C(4) * f[0] - C(2) * s15 + s58;
    const C m4 = C(-2) * (f[1] - f[3]) + (f[5] - f[6] - f[7] + f[8]);
    const C m6 = C(-2) * (f[2] - f[4]) + (f[5] + f[6] - f[7] - f[8]);
    const C m7 = (f[1] + f[3]) - (f[2] + f[4]);
    const C m8 = f[5] - f[6] + f[7] - f[8];
    const C om = C(1) / tau;
    const C a1 = C(1.2) * (m1 + C(2) * dr - C(3) * rho * u2) * C(1.0 / 36.0);
    const C a2 = C(1.1) * (m2 - dr + C(3) * rho * u2) * C(1.0 / 36.0);
    const C a4 = C(1.2) * (m4 + rho * ux) * C(1.0 / 12.0);
    const C a6 = C(1.2) * (m6 + rho * uy) * C(1.0 / 12.0);
    const C a7 = om * (m7 - rho * (ux * ux - uy * uy)) * C(0.25);
    const C a8 = om * (m8 - rho * ux * uy) * C(0.25);
    f[0] -= C(-4) * a1 + C(4) * a2;
    f[1] -= -a1 - C(2) * a2 - C(2) * a4 + a7;
    f[2] -= -a1 - C(2) * a2 - C(2) * a6 - a7;
    f[3] -= -a1 - C(2) * a2 + C(2) * a4 + a7;
    f[4] -= -a1 - C(2) * a2 + C(2) * a6 - a7;
    f[5] -= C(2) * a1 + a2 + a4 + a6 + a8;
    f[6] -= C(2) * a1 + a2 - a4 + a6 - a8;
    f[7] -= C(2) * a1 + a2 - a4 - a6 + a8;
    f[8] -= C(2) * a1 + a2 + a4 - a6 - a8;
}

// Guo forcing term (Lattice::Compute_Disforce, NodeAndLattice.cpp:162-195),
// with omega from the initial relaxation time: added to the post-collision
// populations of forced nodes.
template <typename C>
__device__ __forceinline__ void add_guo(C* f, C ux, C uy, C fx, C fy, C tau0)
{
    const C om = C(1) - C(0.5) * (C(1) / tau0);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const C eu = C(EX(k)) * ux + C(EY(k)) * uy;
        const C gx = (C(3) * (C(EX(k)) - ux) + C(9) * eu * C(EX(k))) * fx;
        const C gy = (C(3) * (C(EY(k)) - uy) + C(9) * eu * C(EY(k))) * fy;
        f[k] += WK<C>(k) * om * (gx + gy);
    }
}

// Forcing term of the IB force for the operator in use, added after the
// collision of a forced node (equilibrium at the corrected velocity
// u = u* + F / (2 rho)); each form adds exactly F to the node's momentum:
//   BGK  the Guo term above (omega from tau0, as Compute_Disforce)
//   MRT  the Guo source G in moment space, M^-1 (I - S/2) M G, written out
//        in the moment basis of collide_mrt: conserved jx, jy whole, e, eps,
//        qx, qy with 1 - s/2 = 0.4, 0.45, 0.4, 0.4, pxx, pxy with 1 - 1/(2 tau)
//   RR   first-order part of G halved, second-order part (1 - 1/(2 tau))
template <typename C, int CO>
__device__ __forceinline__ void add_force(C* f, C ux, C uy, C fx, C fy, C tau0, C tau)
{
    if (CO == CO_BGK) {
        add_guo<C>(f, ux, uy, fx, fy, tau0);
        return;
    }
    const C uF = ux * fx + uy * fy;
    const C om2 = C(1) - C(0.5) / tau;
    if (CO == CO_RR) {
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const C eu = C(EX(k)) * ux + C(EY(k)) * uy;
            const C eF = C(EX(k)) * fx + C(EY(k)) * fy;
            f[k] += WK<C>(k) * (C(1.5) * eF + om2 * (C(9) * eu * eF - C(3) * uF));
        }
        return;
    }
    // moments of G: e 6 uF, eps -6 uF, jx Fx, qx -Fx, jy Fy, qy -Fy,
    // pxx 2 (ux Fx - uy Fy), pxy ux Fy + uy Fx; a_m = (1 - s_m/2) G_m / |M_m|^2
    const C a1 = C(0.4 * 6.0 / 36.0) * uF;
    const C a2 = C(-0.45 * 6.0 / 36.0) * uF;
    const C a3 = fx * C(1.0 / 6.0), a5 = fy * C(1.0 / 6.0);
    const C a4 = fx * C(-0.4 / 12.0), a6 = fy * C(-0.4 / 12.0);
    const C a7 = om2 * C(0.5) * (ux * fx - uy * fy);
    const C a8 = om2 * C(0.25) * (ux * fy + uy * fx);
    f[0] += C(-4) * a1 + C(4) * a2;
    f[1] += -a1 - C(2) * a2 + a3 - C(2) * a4 + a7;
    f[2] += -a1 - C(2) * a2 + a5 - C(2) * a6 - a7;
    f[3] += -a1 - C(2) * a2 - a3 + C(2) * a4 + a7;
    f[4] += -a1 - C(2) * a2 - a5 + C(2) * a6 - a7;
    f[5] += C(2) * a1 + a2 + a3 + a4 + a5 + a6 + a8;
    f[6] += C(2) * a1 + a2 - a3 - a4 + a5 + a6 - a8;
    f[7] += C(2) * a1 + a2 - a3 - a4 - a5 - a6 + a8;
    f[8] += C(2) * a1 + a2 + a3 + a4 - a5 - a6 - a8;
}

// Relax one node's populations in place with the chosen operator.
template <typename C, int CO>
__device__ __forceinline__ void collide_node(C* f, C rho, C ux, C uy, C rb, C tau)
{
    if (CO == CO_MRT) {
        collide_mrt<C>(f, rho, ux, uy, rb, tau);
    } else {
        C feq[9];
        equilibrium<C>(rho, ux, uy, rb, feq);
        if (CO == CO_RR) {
            C pxx, pxy, pyy;
            pi_neq<C>(f, rho, ux, uy, rb, pxx, pxy, pyy);
            collide_rr<C>(f, feq, pxx, pxy, pyy, tau);
        } else {
            collide_bgk<C>(f, feq, tau);
        }
    }
}

// ---------------------------------------------------------------------------
// learned relaxation time: tau = tau0 + out_scale * softplus(MLP(features)),
// MLP 6 -> 32 tanh -> 32 tanh -> 1 with weights rounded to BF16 (held here
// as their exact FP32 values) and arithmetic in the compute type.
// Features of a node (post-stream state, Pi_neq as for the Smagorinsky model):
//   rho, |u|, Pi_neq_xx / |Pi|, Pi_neq_xy / |Pi|, Pi_neq_yy / |Pi|, |S|
// with |Pi| = sqrt(Pxx^2 + 2 Pxy^2 + Pyy^2), S = -3/(2 rho tau0) Pi_neq,
// |S| = sqrt(2 S:S).  Outside the training range [lo, hi] of any feature
// the node falls back to the Smagorinsky tau.
// Parameter block (floats): W1[32][6] b1[32] W2[32][32] b2[32] w3[32] b3,
// then mean[6] std[6] lo[6] hi[6] out_scale.
// ---------------------------------------------------------------------------
constexpr int kMlpIn = 6, kMlpHid = 32;
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpHid * kMlpIn, kMlpW2 = kMlpB1 + kMlpHid,
              kMlpB2 = kMlpW2 + kMlpHid * kMlpHid, kMlpW3 = kMlpB2 + kMlpHid, kMlpB3 = kMlpW3 + kMlpHid;
constexpr int kMlpParams = kMlpB3 + 1;  // 1313
constexpr int kMlpStats = 4 * kMlpIn + 1;
static_assert(kMlpParams == 1313, "MLP size");

// FP64 (parity path): libm-accurate tanh.  FP32: the hardware tanh
// (tanh.approx.f32, one MUFU op, max relative error about 2^-11): with BF16
// weights the network's own rounding is larger than that.
__device__ __forceinline__ double mlp_tanh(double v) { return tanh(v); }
__device__ __forceinline__ float mlp_tanh(float v)
{
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}
// softplus(z) = max(z, 0) + log(1 + exp(-|z|))
__device__ __forceinline__ double softplus(double z) { return fmax(z, 0.0) + log1p(exp(-fabs(z))); }
__device__ __forceinline__ float softplus(float z) { return fmaxf(z, 0.f) + log1pf(expf(-fabsf(z))); }

template <typename C>
__device__ __forceinline__ void mlp_features(C pxx, C pxy, C pyy, C rho, C ux, C uy, C tau0, C* x)
{
    const C c = C(-1.5) / (rho * tau0);
    const C sxx = pxx * c, sxy = pxy * c, syy = pyy * c;
    const C pn = sqrt(pxx * pxx + C(2) * pxy * pxy + pyy * pyy);
    const C inv = pn > C(0) ? C(1) / pn : C(0);
    x[0] = rho;
    x[1] = sqrt(ux * ux + uy * uy);
    x[2] = pxx * inv;
    x[3] = pxy * inv;
    x[4] = pyy * inv;
    x[5] = sqrt(C(2) * (sxx * sxx + C(2) * sxy * sxy + syy * syy));
}

// The network of the fused step kernels, in constant memory (one copy per
// compiled module; the host copies a handle's parameter block here on the
// handle's stream before its step kernels run).  The layer loops below are
// fully unrolled, so each weight is a constant-bank operand of its FMA: no
// load instruction and no wait on one.
static __constant__ float c_mlp[kMlpParams + kMlpStats];

// network output softplus(z) for standardised inputs x
template <typename C>
__device__ __forceinline__ C mlp_forward(const C* x)
{
    C h1[kMlpHid];
#pragma unroll
    for (int j = 0; j < kMlpHid; j++) {
        C a = C(c_mlp[kMlpB1 + j]);
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) a += C(c_mlp[kMlpW1 + j * kMlpIn + i]) * x[i];
        h1[j] = mlp_tanh(a);
    }
    C z = C(c_mlp[kMlpB3]);
#pragma unroll
    for (int j = 0; j < kMlpHid; j++) {
        C a = C(c_mlp[kMlpB2 + j]);
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) a += C(c_mlp[kMlpW2 + j * kMlpHid + i]) * h1[i];
        z += C(c_mlp[kMlpW3 + j]) * mlp_tanh(a);
    }
    return softplus(z);
}

// ---------------------------------------------------------------------------
// the same network with its 32 x 32 hidden layer on the tensor cores, for the
// 32 nodes of a warp at once (an opt-in per handle): every lane evaluates
// layer 1 for its own node (FMA, constant-memory weights) and writes the 32
// activations, rounded to BF16, as the A operand's row; the warp multiplies
// the 32 x 32 activation tile by W2^T with mma.sync m16n8k16 (BF16 inputs,
// FP32 accumulation: 2 node tiles x 4 output tiles x 2 k steps = 16 MMAs);
// each lane applies tanh and the output weights to the accumulator elements
// it holds, and the per-node sums meet in the node's lane through shuffles.
// The B operand (W2 as BF16 pairs in this lane's fragment order) and the
// lane's share of b2 / w3 come from a 4 KB table built on the host
// (MlpFrag).  All 32 lanes must call it together; the tile rows are 16-byte
// aligned (kTcRow words of 4 bytes).
// ---------------------------------------------------------------------------
constexpr int kTcRow = 20;  // 32-bit words per node row of the activation tile (16 + 4: no bank conflicts)

// The fragment table: kFragQ x 32 16-byte entries, entry [q][lane] (q-major,
// so each of a warp's eight loads is one coalesced 512-byte request):
//   q 0-3  W2 B fragments of the lane, words [k step][output tile][2] as BF16 pairs
//   q 4-7  per output tile q - 4: b2[c], b2[c + 1], w3[c], w3[c + 1] (FP32 bits),
//          c = 8 (q - 4) + 2 (lane & 3)
constexpr int kFragQ = 8;
struct MlpFrag {
    uint4 e[kFragQ][32];
};

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// z (before softplus) of this lane's node; x: standardised inputs; sh: the
// warp's 32 x kTcRow-word tile in shared memory
__device__ __forceinline__ float warp_mlp_tc(const float* x, uint32_t* sh, const MlpFrag* __restrict__ frag)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // this lane's fragments first: their loads run under layer 1
    uint4 fq[kFragQ];
#pragma unroll
    for (int q = 0; q < kFragQ; q++) fq[q] = __ldg(&frag->e[q][lane]);
    uint32_t* row = sh + lane * kTcRow;
#pragma unroll
    for (int v = 0; v < 4; v++) {
        uint32_t wd[4];
#pragma unroll
        for (int ww = 0; ww < 4; ww++) {
            float h[2];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int j = 2 * (4 * v + ww) + q;
                float s = c_mlp[kMlpB1 + j];
#pragma unroll
                for (int i = 0; i < kMlpIn; i++) s += c_mlp[kMlpW1 + j * kMlpIn + i] * x[i];
                h[q] = mlp_tanh(s);
            }
            const __nv_bfloat162 pr = __floats2bfloat162_rn(h[0], h[1]);  // low half: the even column
            wd[ww] = *reinterpret_cast<const uint32_t*>(&pr);
        }
        // 16-byte stores: at a 20-word row stride the 8 lanes of each phase hit distinct banks
        *reinterpret_cast<uint4*>(row + 4 * v) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
    }
    const uint32_t b[16] = {fq[0].x, fq[0].y, fq[0].z, fq[0].w, fq[1].x, fq[1].y, fq[1].z, fq[1].w,
                            fq[2].x, fq[2].y, fq[2].z, fq[2].w, fq[3].x, fq[3].y, fq[3].z, fq[3].w};
    float4 bw[4];
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
        bw[nt] = make_float4(__uint_as_float(fq[4 + nt].x), __uint_as_float(fq[4 + nt].y),
                             __uint_as_float(fq[4 + nt].z), __uint_as_float(fq[4 + nt].w));
    __syncwarp();
    float acc[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            acc[mt][nt][0] = acc[mt][nt][2] = bw[nt].x;
            acc[mt][nt][1] = acc[mt][nt][3] = bw[nt].y;
        }
#pragma unroll
    for (int kt = 0; kt < 2; kt++)
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const uint32_t* r0 = sh + (mt * 16 + g) * kTcRow + kt * 8 + t;
            const uint32_t* r1 = r0 + 8 * kTcRow;
            const uint32_t a0 = r0[0], a1 = r1[0], a2 = r0[4], a3 = r1[4];
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
                mma_bf16_16816(acc[mt][nt], a0, a1, a2, a3, b[(kt * 4 + nt) * 2], b[(kt * 4 + nt) * 2 + 1]);
        }
    // rows of this lane's accumulators: g, g + 8 (tile 0), 16 + g, 24 + g (tile 1)
    float p[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            p[2 * mt] += bw[nt].z * mlp_tanh(acc[mt][nt][0]) + bw[nt].w * mlp_tanh(acc[mt][nt][1]);
            p[2 * mt + 1] += bw[nt].z * mlp_tanh(acc[mt][nt][2]) + bw[nt].w * mlp_tanh(acc[mt][nt][3]);
        }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        p[q] += __shfl_xor_sync(0xffffffffu, p[q], 1);
        p[q] += __shfl_xor_sync(0xffffffffu, p[q], 2);
    }
    // node `lane` = 8 q + g' sits in row q of the lanes of group g'
    const int src = 4 * (lane & 7), q = lane >> 3;
    const float v0 = __shfl_sync(0xffffffffu, p[0], src), v1 = __shfl_sync(0xffffffffu, p[1], src);
    const float v2 = __shfl_sync(0xffffffffu, p[2], src), v3 = __shfl_sync(0xffffffffu, p[3], src);
    const float z = q == 0 ? v0 : q == 1 ? v1 : q == 2 ? v2 : v3;
    return z + c_mlp[kMlpB3];
}

// relaxation time from the network (constant memory), Smagorinsky where a
// feature leaves the training range
template <typename C>
__device__ __forceinline__ C learned_tau(C pxx, C pxy, C pyy, C rho, C ux, C uy, C tau0, C cs)
{
    constexpr int st = kMlpParams;
    C x[kMlpIn];
    mlp_features<C>(pxx, pxy, pyy, rho, ux, uy, tau0, x);
    bool in = true;
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) {
        in = in && x[i] >= C(c_mlp[st + 2 * kMlpIn + i]) && x[i] <= C(c_mlp[st + 3 * kMlpIn + i]);
        x[i] = (x[i] - C(c_mlp[st + i])) / C(c_mlp[st + kMlpIn + i]);
    }
    if (!in) return les_tau<C>(pxx, pxy, pyy, rho, tau0, cs);
    return tau0 + C(c_mlp[st + 4 * kMlpIn]) * mlp_forward<C>(x);
}

// The learned tau on dual numbers (adjoint): features carry their partial
// derivatives; the network runs in FP64 with a backward pass for dz/dx, and
// the chain rule gives the partial derivatives of tau.
template <int N>
__device__ Dual<N> learned_tau(Dual<N> pxx, Dual<N> pxy, Dual<N> pyy, Dual<N> rho, Dual<N> ux,
                               Dual<N> uy, Dual<N> tau0, Dual<N> cs, const float* __restrict__ w)
{
    using D = Dual<N>;
    const float* st = w + kMlpParams;
    D x[kMlpIn];
    mlp_features<D>(pxx, pxy, pyy, rho, ux, uy, tau0, x);
    bool in = true;
    for (int i = 0; i < kMlpIn; i++) {
        in = in && x[i].v >= double(st[2 * kMlpIn + i]) && x[i].v <= double(st[3 * kMlpIn + i]);
        x[i] = (x[i] - D(double(st[i]))) / D(double(st[kMlpIn + i]));
    }
    if (!in) return les_tau<D>(pxx, pxy, pyy, rho, tau0, cs);
    double h1[kMlpHid], g2[kMlpHid];
    for (int j = 0; j < kMlpHid; j++) {
        double a = w[kMlpB1 + j];
        for (int i = 0; i < kMlpIn; i++) a += double(w[kMlpW1 + j * kMlpIn + i]) * x[i].v;
        h1[j] = tanh(a);
    }
    double z = w[kMlpB3];
    for (int j = 0; j < kMlpHid; j++) {
        double a = w[kMlpB2 + j];
        for (int i = 0; i < kMlpHid; i++) a += double(w[kMlpW2 + j * kMlpHid + i]) * h1[i];
        const double h2 = tanh(a);
        z += double(w[kMlpW3 + j]) * h2;
        g2[j] = double(w[kMlpW3 + j]) * (1.0 - h2 * h2);  // dz / d(pre-activation 2)
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
    D t = tau0;
    t.v += os * (fmax(z, 0.0) + log1p(exp(-fabs(z))));
    for (int k = 0; k < kMlpIn; k++)
        for (int i = 0; i < N; i++) t.d[i] += os * sig * gx[k] * x[k].d[i];
    return t;
}

// whether a node's learned-model features lie inside the network's training
// range (the network sets tau there, Smagorinsky outside it): the same
// features and comparisons as learned_tau
template <typename C>
__device__ __forceinline__ bool learned_in_range(const C* f, C rho, C ux, C uy, C rb, C tau0)
{
    constexpr int st = kMlpParams;
    C pxx, pxy, pyy, x[kMlpIn];
    pi_neq<C>(f, rho, ux, uy, rb, pxx, pxy, pyy);
    mlp_features<C>(pxx, pxy, pyy, rho, ux, uy, tau0, x);
    bool in = true;
#pragma unroll
    for (int i = 0; i < kMlpIn; i++)
        in = in && x[i] >= C(c_mlp[st + 2 * kMlpIn + i]) && x[i] <= C(c_mlp[st + 3 * kMlpIn + i]);
    return in;
}

// relaxation time of a node's next collision: tau0, Smagorinsky, or (LRN)
// the learned model with its Smagorinsky fallback
template <typename C, bool LRN = false>
__device__ __forceinline__ C node_tau(const C* f, C rho, C ux, C uy, C rb, int les, C tau0, C cs)
{
    if (!LRN && !les) return tau0;
    C pxx, pxy, pyy;
    pi_neq<C>(f, rho, ux, uy, rb, pxx, pxy, pyy);
    if constexpr (LRN) return learned_tau(pxx, pxy, pyy, rho, ux, uy, tau0, cs);
    return les_tau<C>(pxx, pxy, pyy, rho, tau0, cs);
}

}  // namespace ippi
