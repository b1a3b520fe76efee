// lbm_kernels.cuh -- the time-step kernels (sm_100a).
//
// One time step is
//   step_kernel   every node that is not deferred: pull-stream the 9
//                 post-collision populations of its neighbours, apply the
//                 boundary rule of its kind, take the moments, Smagorinsky
//                 tau + collision, store the 9 new post-collision
//                 populations.  HBM traffic per node: 9 loads + 9 stores.
// and, on a side stream running concurrently with it,
//   prep_kernel   the post-stream state of the boundary nets' input nodes
//                 into side buffers
//   band_kernel   (flat plate with boundary nets) the nets' MLP on the band
//                 nodes, then their collision
//   ib_*          (immersed boundary) stencil-node states, interpolation and
//                 direct forcing, spreading and velocity correction, forced
//                 collision with the Guo term, per-body force sums
// A node is "deferred" when its collision needs moments of other nodes of
// the same step (net inputs, marker forces); step_kernel skips it and the
// side-stream kernels own it.  All kernels of a step read only the previous
// field and write disjoint nodes of the next one.
//
// The stored state between steps is the post-collision field; one launch of
// step_kernel performs Mesh::Streaming + Mesh::BoundaryCondition of step t
// (mesh.cpp:192-356) and the LES + collision loop of step t+1
// (mesh.cpp:386-437).
#pragma once

#include "lbm_common.cuh"

namespace ippi {

constexpr int kBlockX = 256;
// rows (in groups of 2^row_shift) with any flagged tile, one bit each, as a
// kernel parameter: the bulk kernel reads the tile flags only in those rows
constexpr int kRowMaskWords = 128;

struct StepArgs {
    const void* f_in;   // post-collision populations of the previous step
    void* f_out;        // post-collision populations of this step
    long long pitch;    // row pitch (elements)
    long long plane;    // plane stride (elements)
    int nx, ny;
    int les;
    int plate_x0;
    double tau0, cs, u_in, rho0;
    float f_tau0, f_cs, f_u_in, f_rho0;  // the same in FP32 (no conversions per node)
    const uint8_t* tile;  // [gy][gx] 1 = some node of this block is deferred
    int tiles_x;
    const uint8_t* nflag; // [ny][nx] NF_* bits
    void* side_f;         // [nslots][9] compute type: fnew of deferred nodes
    void* side_m;         // [2][nslots][3] compute type: rho, ux, uy (by step parity)
    int nslots;
    void* corner;         // flat plate: [2][12] fixed bottom corners (f[9], rho, ux, uy)
    void* avg;            // [3][ny][nx] compute type: running means of ux, uy, rho
    int avg_start;
    Ctr* ctr;
    int mode;             // MODE_*
    int par;              // step parity: side-buffer half and ctr->t entry
    int fixed_t;          // step number for the MAT modes
    const double* init_m; // [3][ny][nx] initial rho, ux, uy (INIT modes)
    const float* mlp;     // learned tau: parameters + feature statistics in device memory (the
                          // adjoint reads them here; the LRN step kernels read the copy in
                          // constant memory, c_mlp)
    const MlpFrag* mlp_frag; // learned tau on the tensor cores (bulk row segments): per-lane W2
                          // fragments, b2 and w3; null = the FMA network
    const double* tau_field; // les == 3: relaxation time per node [ny][nx]
    void* mac;            // les 4, 5: [2][ny][nx] compute type, ux and uy of this step's
                          // post-stream (and IB-corrected) state, for the velocity gradient
    const double* wall_dist; // les 6: distance to the wall per node [ny][nx]
    unsigned rowmask[kRowMaskWords]; // bit (y >> row_shift): a tile of row y is flagged
    int row_shift;
    double* dl_f;         // MAT: fnew [9][ny][nx]
    double* dl_m;         // MAT: rho, ux, uy, boundary-net flag [4][ny][nx]
    double* dl_tau;       // MAT: tau of the next collision [ny][nx]
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
// a run parameter in the compute type (FP64 or its FP32 copy)
template <typename C> __device__ __forceinline__ C prm(double d, float f);
template <> __device__ __forceinline__ double prm<double>(double d, float) { return d; }
template <> __device__ __forceinline__ float prm<float>(double, float f) { return f; }

// element offsets fit in 32 bits (ippi_create bounds 9 * pitch * ny)
template <int S>
__device__ __forceinline__ typename Store<S>::C ldf(const StepArgs& a, int k, int x, int y)
{
    using T = typename Store<S>::T;
    const T* p = reinterpret_cast<const T*>(a.f_in);
    return Store<S>::ld(__ldg(p + (unsigned)(k * (int)a.plane + y * (int)a.pitch + x)));
}

template <int S>
__device__ __forceinline__ void stf(const StepArgs& a, int k, int x, int y, typename Store<S>::C v)
{
    using T = typename Store<S>::T;
    T* p = reinterpret_cast<T*>(a.f_out);
    p[(unsigned)(k * (int)a.plane + y * (int)a.pitch + x)] = Store<S>::st(v);
}

template <int S>
__device__ __forceinline__ typename Store<S>::C rbase(const StepArgs& a)
{
    using C = typename Store<S>::C;
    return Store<S>::kShift ? prm<C>(a.rho0, a.f_rho0) : C(0);
}

// plain pull of all 9 populations (all sources inside the lattice)
template <int S>
__device__ __forceinline__ void pull(const StepArgs& a, int x, int y, typename Store<S>::C* f)
{
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = ldf<S>(a, k, x - EX(k), y - EY(k));
}

// non-equilibrium extrapolation: f(A) = feq(A) + f(B) - feq(B)
template <typename C>
__device__ __forceinline__ void nee(C* f, C rhoA, C uxA, C uyA, C rhoB, C uxB, C uyB, C rb)
{
    C ea[9], eb[9];
    equilibrium<C>(rhoA, uxA, uyA, rb, ea);
    equilibrium<C>(rhoB, uxB, uyB, rb, eb);
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = (ea[k] + f[k]) - eb[k];
}

// ---------------------------------------------------------------------------
// flat-plate scene (Mesh::JudgeStyle mesh.cpp:1398-1425 and
// Mesh::BoundaryCondition mesh.cpp:228-356, one rank, global coordinates)
// ---------------------------------------------------------------------------
enum RefKind { RK_FLUID, RK_INLET, RK_OUTLET, RK_TOP, RK_TOP_IN, RK_TOP_OUT, RK_BOT_SPEC,
               RK_BOT_NEE, RK_FIXED };

__host__ __device__ __forceinline__ int ref_kind(int x, int y, int nx, int ny, int plate_x0)
{
    if (y == 0 && (x == 0 || x == nx - 1)) return RK_FIXED;  // 'i'/'o' corners never updated
    if (x == 0) return y == ny - 1 ? RK_TOP_IN : RK_INLET;
    if (x == nx - 1) return y == ny - 1 ? RK_TOP_OUT : RK_OUTLET;
    if (y == ny - 1) return RK_TOP;
    if (y == 0) return x < plate_x0 ? RK_BOT_SPEC : RK_BOT_NEE;
    return RK_FLUID;
}

__host__ __device__ __forceinline__ char ref_style(int x, int y, int nx, int ny, int plate_x0)
{
    switch (ref_kind(x, y, nx, ny, plate_x0)) {
    case RK_FIXED: return x == 0 ? 'i' : 'o';
    case RK_INLET:
    case RK_TOP_IN: return 'i';
    case RK_OUTLET:
    case RK_TOP_OUT: return 'o';
    case RK_TOP: return 'u';
    case RK_BOT_SPEC: return 'm';
    case RK_BOT_NEE: return 'd';
    default: return 'f';
    }
}

// pulled fluid node (x, y) with its moments
template <int S>
__device__ __forceinline__ void ref_fluid(const StepArgs& a, int x, int y, typename Store<S>::C* f,
                                          typename Store<S>::C& rho, typename Store<S>::C& ux,
                                          typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    pull<S>(a, x, y, f);
    macros<C>(f, rbase<S>(a), rho, ux, uy);
}

// inlet node (0, y), 1 <= y <= ny-2: rho = 1, u = (u_in, 0), NEE from (1, y)
template <int S>
__device__ __forceinline__ void ref_inlet(const StepArgs& a, int y, typename Store<S>::C* f,
                                          typename Store<S>::C& rho, typename Store<S>::C& ux,
                                          typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    C rb, ub, vb;
    ref_fluid<S>(a, 1, y, f, rb, ub, vb);
    rho = C(1);
    ux = prm<C>(a.u_in, a.f_u_in);
    uy = C(0);
    nee<C>(f, rho, ux, uy, rb, ub, vb, rbase<S>(a));
}

// outlet node (nx-1, y), 1 <= y <= ny-2: rho = 1, u = u(nx-2, y), NEE
template <int S>
__device__ __forceinline__ void ref_outlet(const StepArgs& a, int y, typename Store<S>::C* f,
                                           typename Store<S>::C& rho, typename Store<S>::C& ux,
                                           typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    C rb, ub, vb;
    ref_fluid<S>(a, a.nx - 2, y, f, rb, ub, vb);
    rho = C(1);
    ux = ub;
    uy = vb;
    nee<C>(f, rho, ux, uy, rb, ub, vb, rbase<S>(a));
}

template <int S>
__device__ void ref_state(const StepArgs& a, int x, int y, typename Store<S>::C* f,
                          typename Store<S>::C& rho, typename Store<S>::C& ux,
                          typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    const C rbs = rbase<S>(a);
    const int kind = ref_kind(x, y, a.nx, a.ny, a.plate_x0);
    switch (kind) {
    case RK_FLUID: ref_fluid<S>(a, x, y, f, rho, ux, uy); break;
    case RK_INLET: ref_inlet<S>(a, y, f, rho, ux, uy); break;
    case RK_OUTLET: ref_outlet<S>(a, y, f, rho, ux, uy); break;
    case RK_TOP: {
        C rb, ub, vb;
        ref_fluid<S>(a, x, a.ny - 2, f, rb, ub, vb);
        rho = C(1);
        ux = ub;
        uy = vb;
        nee<C>(f, rho, ux, uy, rb, ub, vb, rbs);
    } break;
    case RK_TOP_IN: {
        C rb, ub, vb;
        ref_inlet<S>(a, a.ny - 2, f, rb, ub, vb);
        rho = C(1);
        ux = ub;
        uy = vb;
        nee<C>(f, rho, ux, uy, rb, ub, vb, rbs);
    } break;
    case RK_TOP_OUT: {
        C rb, ub, vb;
        ref_outlet<S>(a, a.ny - 2, f, rb, ub, vb);
        rho = C(1);
        ux = ub;
        uy = vb;
        nee<C>(f, rho, ux, uy, rb, ub, vb, rbs);
    } break;
    case RK_BOT_SPEC: {
        // specular reflection pulls of mesh.cpp:327-335
        f[0] = ldf<S>(a, 0, x, 0);
        f[1] = ldf<S>(a, 1, x - 1, 0);
        f[2] = ldf<S>(a, 4, x, 1);
        f[3] = ldf<S>(a, 3, x + 1, 0);
        f[4] = ldf<S>(a, 4, x, 1);
        f[5] = ldf<S>(a, 8, x - 1, 1);
        f[6] = ldf<S>(a, 7, x + 1, 1);
        f[7] = ldf<S>(a, 7, x + 1, 1);
        f[8] = ldf<S>(a, 8, x - 1, 1);
        macros<C>(f, rbs, rho, ux, uy);
    } break;
    case RK_BOT_NEE: {
        C rb, ub, vb;
        ref_fluid<S>(a, x, 1, f, rb, ub, vb);
        rho = rb;
        ux = C(0);
        uy = C(0);
        nee<C>(f, rho, ux, uy, rb, ub, vb, rbs);
    } break;
    default: {  // RK_FIXED: populations and moments as initialised
        const C* c = reinterpret_cast<const C*>(a.corner) + (x == 0 ? 0 : 12);
#pragma unroll
        for (int k = 0; k < 9; k++) f[k] = c[k];
        rho = c[9];
        ux = c[10];
        uy = c[11];
    } break;
    }
}

// ---------------------------------------------------------------------------
// channel scene: halfway bounce-back walls at y = -1/2 and ny - 1/2,
// parabolic Zou-He velocity inlet at x = 0, the reference's NEE outlet
// (rho0, u from x = nx-2) at x = nx-1.
// ---------------------------------------------------------------------------
template <typename C>
__device__ __forceinline__ C inlet_profile(int y, int ny, C umax)
{
    const C H = C(ny);
    const C yy = C(y) + C(0.5);
    return C(4) * umax * yy * (H - yy) / (H * H);
}

// Zou-He velocity inlet (west, velocity (u, 0)): the unknowns 1, 5, 8 and
// the density of Zou & He (1997) -- in shifted populations rho - rb =
// (S + rb u)/(1 - u), the rest unchanged -- then the regularised
// reconstruction of Latt & Chopard (2008): every population from the
// equilibrium at (rho, u, 0) plus the second-order projection of the
// non-equilibrium part.  The plain Zou-He completion with BGK diverges at
// tau = 0.53 in a 400 x 100 channel (it is stable from about 0.55); the
// regularised one does not.  Linear in the pulled populations for fixed u.
template <typename C>
__device__ __forceinline__ void zh_inlet(C* f, C u, C rbs)
{
    const C sk = f[0] + f[2] + f[4] + C(2) * (f[3] + f[6] + f[7]);
    const C r = rbs + (sk + rbs * u) / (C(1) - u);
    f[1] = f[3] + C(2.0 / 3.0) * r * u;
    f[5] = f[7] - C(0.5) * (f[2] - f[4]) + C(1.0 / 6.0) * r * u;
    f[8] = f[6] + C(0.5) * (f[2] - f[4]) + C(1.0 / 6.0) * r * u;
    C pxx, pxy, pyy, fe[9];
    pi_neq<C>(f, r, u, C(0), rbs, pxx, pxy, pyy);
    equilibrium<C>(r, u, C(0), rbs, fe);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const C qxx = C(EX(k) * EX(k)) - C(1.0 / 3.0);
        const C qyy = C(EY(k) * EY(k)) - C(1.0 / 3.0);
        const C qxy = C(EX(k) * EY(k));
        f[k] = fe[k] + C(4.5) * WK<C>(k) * (qxx * pxx + C(2) * qxy * pxy + qyy * pyy);
    }
}

template <int S>
__device__ __forceinline__ void ch_pull(const StepArgs& a, int x, int y, typename Store<S>::C* f)
{
    if (x >= 1 && y >= 1 && y <= a.ny - 2) {  // x <= nx - 2 for every caller
        pull<S>(a, x, y, f);
        return;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const int sx = x - EX(k), sy = y - EY(k);
        if (sy < 0 || sy >= a.ny)
            f[k] = ldf<S>(a, OPP(k), x, y);
        else if (sx < 0)
            f[k] = 0;
        else
            f[k] = ldf<S>(a, k, sx, sy);
    }
}

template <int S>
__device__ __forceinline__ void ch_fluid(const StepArgs& a, int x, int y, typename Store<S>::C* f,
                                         typename Store<S>::C& rho, typename Store<S>::C& ux,
                                         typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    const C rbs = rbase<S>(a);
    ch_pull<S>(a, x, y, f);
    if (x == 0) zh_inlet<C>(f, inlet_profile<C>(y, a.ny, prm<C>(a.u_in, a.f_u_in)), rbs);
    macros<C>(f, rbs, rho, ux, uy);
}

template <int S>
__device__ void ch_state(const StepArgs& a, int x, int y, typename Store<S>::C* f,
                         typename Store<S>::C& rho, typename Store<S>::C& ux,
                         typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    if (x == a.nx - 1) {
        C rb, ub, vb;
        ch_fluid<S>(a, a.nx - 2, y, f, rb, ub, vb);
        rho = prm<C>(a.rho0, a.f_rho0);
        ux = ub;
        uy = vb;
        nee<C>(f, rho, ux, uy, rb, ub, vb, rbase<S>(a));
    } else {
        ch_fluid<S>(a, x, y, f, rho, ux, uy);
    }
}
// ---------------------------------------------------------------------------
// shared epilogue pieces
// ---------------------------------------------------------------------------
__device__ __forceinline__ void flag_error(Ctr* c, int t)
{
    if (atomicExch(&c->err, 1) == 0) c->err_t = t;
}

__device__ __forceinline__ int step_time(const StepArgs& a)
{
    return a.mode >= MODE_MAT ? a.fixed_t : __ldcg(&a.ctr->t[a.par]);
}

// pull of an interior fluid node next to solid nodes: a population whose
// source is solid is the node's own opposite post-collision population
// (halfway bounce-back, as the reference's 'b' nodes next to 's' nodes)
template <int S>
__device__ __forceinline__ void solid_pull(const StepArgs& a, int x, int y, typename Store<S>::C* f)
{
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const int sx = x - EX(k), sy = y - EY(k);
        f[k] = (a.nflag[sy * a.nx + sx] & NF_SOLID) ? ldf<S>(a, OPP(k), x, y) : ldf<S>(a, k, sx, sy);
    }
}

// velocity gradient (du/dx, du/dy, dv/dx, dv/dy) by forward differences of
// the stored velocities: GetDuxDx / GetDuyDx (mesh.cpp:1659-1724, 1795-1864)
// give 0 in the last column and towards a solid node, GetDuxDy / GetDuyDy
// (mesh.cpp:1725-1794, 1865-1934) from the second-to-last row up and towards
// a solid node
template <int S>
__device__ __forceinline__ void vel_grad(const StepArgs& a, int x, int y, typename Store<S>::C* g)
{
    using C = typename Store<S>::C;
    const C* m = reinterpret_cast<const C*>(a.mac);
    const int pl = a.nx * a.ny, node = y * a.nx + x;
    const C u0 = m[node], v0 = m[pl + node];
    g[0] = g[1] = g[2] = g[3] = C(0);
    if (x < a.nx - 1 && !(a.nflag[node + 1] & NF_SOLID)) {
        g[0] = m[node + 1] - u0;
        g[2] = m[pl + node + 1] - v0;
    }
    if (y + 1 < a.ny - 1 && !(a.nflag[node + a.nx] & NF_SOLID)) {
        g[1] = m[node + a.nx] - u0;
        g[3] = m[pl + node + a.nx] - v0;
    }
}

// relaxation time of the given field (3) and of the closures 4 (WALE), 5
// (coherent structure), 6 (wall-damped Cs), from the post-stream state
// f / rho / u of node (x, y)
template <int S>
__device__ __forceinline__ typename Store<S>::C ext_tau(const StepArgs& a, int x, int y,
                                                         const typename Store<S>::C* f,
                                                         typename Store<S>::C rho, typename Store<S>::C ux,
                                                         typename Store<S>::C uy, typename Store<S>::C rb)
{
    using C = typename Store<S>::C;
    if (a.les == 3) return C(a.tau_field[y * a.nx + x]);
    const C tau0 = prm<C>(a.tau0, a.f_tau0);
    C g[4];
    if (a.les == 4) {
        vel_grad<S>(a, x, y, g);
        return wale_tau<C>(g, tau0);
    }
    C pxx, pxy, pyy;
    pi_neq<C>(f, rho, ux, uy, rb, pxx, pxy, pyy);
    if (a.les == 5) {
        vel_grad<S>(a, x, y, g);
        return csm_tau<C>(g, pxx, pxy, pyy, tau0);
    }
    return dyncs_tau<C>(pxx, pxy, pyy, rho, tau0, C(a.wall_dist[y * a.nx + x]));
}

// post-stream state of node (x, y): the boundary rule of its kind and its
// moments, or (INIT modes) the equilibrium of the initial moments
template <int S, int SC>
__device__ __forceinline__ void node_state(const StepArgs& a, int x, int y, typename Store<S>::C* f,
                                           typename Store<S>::C& rho, typename Store<S>::C& ux,
                                           typename Store<S>::C& uy)
{
    using C = typename Store<S>::C;
    if (a.mode == MODE_INIT || a.mode == MODE_MAT_INIT) {
        // Lattice::InitialLatticeFeq: populations at equilibrium of the given moments
        const long long node = (long long)y * a.nx + x;
        const long long pl = (long long)a.nx * a.ny;
        rho = C(a.init_m[node]);
        ux = C(a.init_m[pl + node]);
        uy = C(a.init_m[2 * pl + node]);
        equilibrium<C>(rho, ux, uy, rbase<S>(a), f);
        if (SC == SC_REF && a.mode == MODE_INIT &&
            ref_kind(x, y, a.nx, a.ny, a.plate_x0) == RK_FIXED) {
            C* c = reinterpret_cast<C*>(a.corner) + (x == 0 ? 0 : 12);
#pragma unroll
            for (int q = 0; q < 9; q++) c[q] = f[q];
            c[9] = rho;
            c[10] = ux;
            c[11] = uy;
        }
    } else if (SC == SC_REF) {
        ref_state<S>(a, x, y, f, rho, ux, uy);
    } else {
        ch_state<S>(a, x, y, f, rho, ux, uy);
    }
}

// averages, error check and download outputs of one node's post-stream state
template <int S>
__device__ __forceinline__ void node_epilogue(const StepArgs& a, long long node, int t,
                                              const typename Store<S>::C* f,
                                              typename Store<S>::C rho, typename Store<S>::C ux,
                                              typename Store<S>::C uy)
{
    using C = typename Store<S>::C;
    const long long pl = (long long)a.nx * a.ny;
    if (a.mode < MODE_MAT) {
        if (a.mode == MODE_STEP && t >= a.avg_start) {
            // Mesh::ComputeAvgVelocity (mesh.cpp:1969-1971)
            C* av = reinterpret_cast<C*>(a.avg);
            const C n0 = C(t - a.avg_start), n1 = C(t - a.avg_start + 1);
            av[node] = (av[node] * n0 + ux) / n1;
            av[pl + node] = (av[pl + node] * n0 + uy) / n1;
            av[2 * pl + node] = (av[2 * pl + node] * n0 + rho) / n1;
        }
        // Mesh::ErrorCatch (mesh.cpp:2103): rho outside [0, 10]; NaN too
        if (!(rho <= C(10) && rho >= C(0))) flag_error(a.ctr, t);
    } else {
        const C rbs = rbase<S>(a);
#pragma unroll
        for (int q = 0; q < 9; q++) a.dl_f[q * pl + node] = double(f[q] + WK<C>(q) * rbs);
        a.dl_m[node] = double(rho);
        a.dl_m[pl + node] = double(ux);
        a.dl_m[2 * pl + node] = double(uy);
    }
}

// ---------------------------------------------------------------------------
// the fused stream + boundary + collide kernel (every node not deferred)
// ---------------------------------------------------------------------------
// (the learned-tau variant keeps the network's hidden layer in registers:
// fewer resident blocks)
template <int S, int CO, int SC, bool LRN, int XT = 0>
__global__ void __launch_bounds__(kBlockX, (step_min_blocks<S, LRN>())) step_kernel(const StepArgs a)
{
    using C = typename Store<S>::C;
    const int x = blockIdx.x * kBlockX + threadIdx.x;
    const int y = blockIdx.y;
    const int t = step_time(a);
    if (x < a.nx) {
        const long long node = (long long)y * a.nx + x;
        uint8_t nf = 0;
        if (a.tile[blockIdx.y * a.tiles_x + blockIdx.x]) nf = a.nflag[node];
        const bool deferred = nf & NF_DEFER;
        if ((nf & NF_SOLID) && a.mode >= MODE_MAT) {
            // a solid node reads as fluid at rest
            const long long pl = (long long)a.nx * a.ny;
#pragma unroll
            for (int q = 0; q < 9; q++) a.dl_f[q * pl + node] = WK<double>(q) * a.rho0;
            a.dl_m[node] = a.rho0;
            a.dl_m[pl + node] = 0.0;
            a.dl_m[2 * pl + node] = 0.0;
            a.dl_tau[node] = a.tau0;
        } else if ((!deferred && !(nf & NF_SOLID)) || a.mode == MODE_INIT) {
            const C rbs = rbase<S>(a);
            C f[9], rho, ux, uy;
            if ((nf & NF_SBND) && a.mode != MODE_INIT && a.mode != MODE_MAT_INIT) {
                solid_pull<S>(a, x, y, f);
                macros<C>(f, rbs, rho, ux, uy);
            } else {
                node_state<S, SC>(a, x, y, f, rho, ux, uy);
            }
            if (!deferred) {
                node_epilogue<S>(a, node, t, f, rho, ux, uy);
                const C tau = XT            ? ext_tau<S>(a, x, y, f, rho, ux, uy, rbs)
                              : a.les == 3 ? C(a.tau_field[node])
                                           : node_tau<C, LRN>(f, rho, ux, uy, rbs, a.les, prm<C>(a.tau0, a.f_tau0),
                                                              prm<C>(a.cs, a.f_cs));
                if (a.mode >= MODE_MAT) {
                    a.dl_tau[node] = double(tau);
                    if (LRN)  // 1 where the network set tau, 0 where Smagorinsky did
                        a.dl_m[3ll * a.nx * a.ny + node] =
                            learned_in_range<C>(f, rho, ux, uy, rbs, prm<C>(a.tau0, a.f_tau0)) ? 1.0 : 0.0;
                } else {
                    collide_node<C, CO>(f, rho, ux, uy, rbs, tau);
#pragma unroll
                    for (int q = 0; q < 9; q++) stf<S>(a, q, x, y, f[q]);
                }
            }
        }
    }
    if (a.mode < MODE_MAT && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        a.ctr->t[a.par ^ 1] = t + 1;
}

// ---------------------------------------------------------------------------
// the same for normal steps (MODE_STEP), without the INIT / download paths:
// the parameters are copied into registers once, node indices are 32-bit
// (ippi_create bounds 9 * pitch * ny below 2^31), and an interior node pulls
// its 9 populations from one base pointer at constant plane offsets.  Edge
// nodes take the boundary rule of the scene.
// ---------------------------------------------------------------------------
// One 256-node row segment (bx, by) of a normal step: pull (or the node's
// boundary rule), moments, relaxation time, collision, stores.  Everything
// that is not the node's own pull, collision and stores is kept out of the
// common instance: the flag tables are read only in rows the parameter mask
// marks, the step counter only by the averaging instances (AV, chosen per
// step on the host) and on the error path, the per-node relaxation-time
// field only by the XT instances.  At 8 blocks of 256 threads per SM the
// kernel has 32 registers, and each extra branch with its own loads cost
// 1-3 % of the step (measured interleaved).
template <int S, int CO, int SC, bool LRN, int XT, int AV>
__device__ __forceinline__ void bulk_tile(const StepArgs& a, int bx, int by, int tx)
{
    using C = typename Store<S>::C;
    using T = typename Store<S>::T;
    const int x = bx * kBlockX + tx, y = by;
    const int nx = a.nx, ny = a.ny;
    const int pitch = (int)a.pitch, plane = (int)a.plane;
    const int node = y * nx + x;
    const int rbit = y >> a.row_shift;
    const bool row_flagged = (a.rowmask[rbit >> 5] >> (rbit & 31)) & 1u;
    // the whole segment interior, in a row without flagged tiles (decided
    // once per block): no per-node bound, flag or boundary-kind test
    const bool interior_seg = !row_flagged && bx >= 1 && (bx + 1) * kBlockX <= nx - 1 && y >= 1 && y <= ny - 2;
    const C rbs = rbase<S>(a);
    C f[9], rho, ux, uy;
    const int cell = y * pitch + x;
    if (interior_seg) {
        const T* p = reinterpret_cast<const T*>(a.f_in) + cell;
#pragma unroll
        for (int k = 0; k < 9; k++) f[k] = Store<S>::ld(__ldg(p + (k * plane - EY(k) * pitch - EX(k))));
        macros<C>(f, rbs, rho, ux, uy);
    } else {
        if (x >= nx) return;
        uint8_t nf = 0;
        if (row_flagged && a.tile[by * a.tiles_x + bx]) nf = a.nflag[node];
        if (nf & (NF_DEFER | NF_SOLID)) return;
        if (nf & NF_SBND) {
            solid_pull<S>(a, x, y, f);
            macros<C>(f, rbs, rho, ux, uy);
        } else if (x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2) {
            const T* p = reinterpret_cast<const T*>(a.f_in) + cell;
#pragma unroll
            for (int k = 0; k < 9; k++) f[k] = Store<S>::ld(__ldg(p + (k * plane - EY(k) * pitch - EX(k))));
            macros<C>(f, rbs, rho, ux, uy);
        } else if (SC == SC_REF) {
            ref_state<S>(a, x, y, f, rho, ux, uy);
        } else {
            ch_state<S>(a, x, y, f, rho, ux, uy);
        }
    }
    // Mesh::ErrorCatch (mesh.cpp:2103): rho outside [0, 10]; NaN too
    const bool bad = !(rho <= C(10) && rho >= C(0));
    const C tau = XT ? ext_tau<S>(a, x, y, f, rho, ux, uy, rbs)
                     : node_tau<C, LRN>(f, rho, ux, uy, rbs, a.les, prm<C>(a.tau0, a.f_tau0),
                                        prm<C>(a.cs, a.f_cs));
    if (AV) {
        // Mesh::ComputeAvgVelocity (mesh.cpp:1969-1971) of the post-stream
        // moments, which the collision below overwrites in f only
        const int t = __ldcg(&a.ctr->t[a.par]);
        C* av = reinterpret_cast<C*>(a.avg);
        const int pl = nx * ny;
        const C n0 = C(t - a.avg_start), n1 = C(t - a.avg_start + 1);
        av[node] = (av[node] * n0 + ux) / n1;
        av[pl + node] = (av[pl + node] * n0 + uy) / n1;
        av[2 * pl + node] = (av[2 * pl + node] * n0 + rho) / n1;
    }
    collide_node<C, CO>(f, rho, ux, uy, rbs, tau);
    T* q = reinterpret_cast<T*>(a.f_out) + cell;
#pragma unroll
    for (int k = 0; k < 9; k++) q[k * plane] = Store<S>::st(f[k]);
    if (bad) flag_error(a.ctr, __ldcg(&a.ctr->t[a.par]));
}

// The learned-tau row segment with the network's hidden layer on the tensor
// cores (warp_mlp_tc): the same pull, moments, collision and stores as
// bulk_tile, but every lane of a warp reaches the network together -- lanes
// beyond the lattice or on deferred / solid nodes run it on dummy features
// and store nothing.
template <int S, int CO, int SC, int AV>
__device__ __forceinline__ void bulk_tile_tc(const StepArgs& a, int bx, int by, int tx)
{
    using C = typename Store<S>::C;
    using T = typename Store<S>::T;
    static_assert(S != ST_F64, "the tensor-core network is for FP32 arithmetic");
    __shared__ __align__(16) uint32_t h1s[kBlockX / 32][32 * kTcRow];
    const int x = bx * kBlockX + tx, y = by;
    const int nx = a.nx, ny = a.ny;
    const int pitch = (int)a.pitch, plane = (int)a.plane;
    bool active = x < nx;
    const int node = y * nx + x;
    uint8_t nf = 0;
    const int rbit = y >> a.row_shift;
    if (active && ((a.rowmask[rbit >> 5] >> (rbit & 31)) & 1u) && a.tile[by * a.tiles_x + bx]) nf = a.nflag[node];
    if (nf & (NF_DEFER | NF_SOLID)) active = false;
    const C rbs = rbase<S>(a);
    C f[9], rho = C(1), ux = C(0), uy = C(0);
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = C(0);
    const int cell = y * pitch + x;
    if (active) {
        if (nf & NF_SBND) {
            solid_pull<S>(a, x, y, f);
            macros<C>(f, rbs, rho, ux, uy);
        } else if (x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2) {
            const T* p = reinterpret_cast<const T*>(a.f_in) + cell;
#pragma unroll
            for (int k = 0; k < 9; k++) f[k] = Store<S>::ld(__ldg(p + (k * plane - EY(k) * pitch - EX(k))));
            macros<C>(f, rbs, rho, ux, uy);
        } else if (SC == SC_REF) {
            ref_state<S>(a, x, y, f, rho, ux, uy);
        } else {
            ch_state<S>(a, x, y, f, rho, ux, uy);
        }
    }
    const C tau0 = prm<C>(a.tau0, a.f_tau0), cs = prm<C>(a.cs, a.f_cs);
    C pxx, pxy, pyy;
    pi_neq<C>(f, rho, ux, uy, rbs, pxx, pxy, pyy);
    // features, range and standardisation as learned_tau
    constexpr int st = kMlpParams;
    C xs[kMlpIn];
    mlp_features<C>(pxx, pxy, pyy, rho, ux, uy, tau0, xs);
    bool in = active;
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) {
        in = in && xs[i] >= C(c_mlp[st + 2 * kMlpIn + i]) && xs[i] <= C(c_mlp[st + 3 * kMlpIn + i]);
        xs[i] = active ? (xs[i] - C(c_mlp[st + i])) / C(c_mlp[st + kMlpIn + i]) : C(0);
    }
    __syncwarp();
    const float z = warp_mlp_tc(xs, h1s[tx >> 5], a.mlp_frag);
    if (!active) return;
    const bool bad = !(rho <= C(10) && rho >= C(0));
    const C tau = in ? tau0 + C(c_mlp[st + 4 * kMlpIn]) * softplus(z) : les_tau<C>(pxx, pxy, pyy, rho, tau0, cs);
    if (AV) {
        const int t = __ldcg(&a.ctr->t[a.par]);
        C* av = reinterpret_cast<C*>(a.avg);
        const int pl = nx * ny;
        const C n0 = C(t - a.avg_start), n1 = C(t - a.avg_start + 1);
        av[node] = (av[node] * n0 + ux) / n1;
        av[pl + node] = (av[pl + node] * n0 + uy) / n1;
        av[2 * pl + node] = (av[2 * pl + node] * n0 + rho) / n1;
    }
    collide_node<C, CO>(f, rho, ux, uy, rbs, tau);
    T* q = reinterpret_cast<T*>(a.f_out) + cell;
#pragma unroll
    for (int k = 0; k < 9; k++) q[k * plane] = Store<S>::st(f[k]);
    if (bad) flag_error(a.ctr, __ldcg(&a.ctr->t[a.par]));
}

// a learned-tau row segment: the tensor-core network when the handle holds
// one (a warp-uniform kernel parameter), else bulk_tile's FMA network
template <int S, int CO, int SC, bool LRN, int XT, int AV>
__device__ __forceinline__ void bulk_tile_any(const StepArgs& a, int bx, int by, int tx)
{
    if constexpr (LRN && S != ST_F64 && XT == 0) {
        if (a.mlp_frag) {
            bulk_tile_tc<S, CO, SC, AV>(a, bx, by, tx);
            return;
        }
    }
    bulk_tile<S, CO, SC, LRN, XT, AV>(a, bx, by, tx);
}

// a normal step without immersed boundary work in the same launch: one
// block per row segment; block (0, 0) advances the step counter
template <int S, int CO, int SC, bool LRN, int XT = 0, int AV = 0>
__global__ void __launch_bounds__(kBlockX, (step_min_blocks<S, LRN>())) step_fast(const StepArgs ap)
{
    // When launched as a programmatic dependent (the boundary-net step), the
    // grid's last block waits for its primary to complete, so the grid cannot
    // complete before it; it is scheduled last and waits on a grid that was
    // resident before any bulk block started, so there is no circular wait.
    // Without a primary the wait returns at once.
    if (blockIdx.x == gridDim.x - 1 && blockIdx.y == gridDim.y - 1 && threadIdx.x == 0)
        asm volatile("griddepcontrol.wait;" ::: "memory");
    bulk_tile_any<S, CO, SC, LRN, XT, AV>(ap, blockIdx.x, blockIdx.y, threadIdx.x);
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        ap.ctr->t[ap.par ^ 1] = __ldcg(&ap.ctr->t[ap.par]) + 1;
}

// ---------------------------------------------------------------------------
// side-stream prep: post-stream state of the nodes other kernels need --
// inputs of the boundary nets and IB stencil nodes (moments into side_m) and
// deferred nodes (populations into side_f, plus their averages / outputs).
// Runs concurrently with step_kernel: both only read f_in.
// ---------------------------------------------------------------------------
struct PrepNode {
    int x, y, slot, flags;
};

template <int S, int SC>
__global__ void __launch_bounds__(256, (step_min_blocks<S, false>())) prep_kernel(const StepArgs a, const PrepNode* nodes, int n)
{
    using C = typename Store<S>::C;
    // band_kernel, when launched as this grid's programmatic dependent, may
    // start now: it waits for this grid's results itself
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PrepNode pn = nodes[i];
    const int t = step_time(a);
    C f[9], rho, ux, uy;
    node_state<S, SC>(a, pn.x, pn.y, f, rho, ux, uy);
    C* sm = reinterpret_cast<C*>(a.side_m) + ((long long)a.par * a.nslots + pn.slot) * 3;
    sm[0] = rho;
    sm[1] = ux;
    sm[2] = uy;
    if (pn.flags & NF_DEFER) {
        C* sf = reinterpret_cast<C*>(a.side_f) + (long long)pn.slot * 9;
#pragma unroll
        for (int q = 0; q < 9; q++) sf[q] = f[q];
        node_epilogue<S>(a, (long long)pn.y * a.nx + pn.x, t, f, rho, ux, uy);
    }
}

// ---------------------------------------------------------------------------
// boundary nets (Mesh::NNmodel_Type00..07, mesh.cpp:2767-3259)
//
// One block evaluates one net (Linear(nin,128)+ReLU, 6 x (Linear(128,128)+
// ReLU), Linear(128,1)) on up to band_nodes band nodes, each linear layer as
// tensor-core products D[128 outputs][N nodes] = W x act^T by tcgen05.mma
// (kind::f16: FP16 operands, FP32 accumulators in tensor memory; M = 128,
// N = 48 or 96, K = 16 per instruction).  FP32 accuracy from two FP16 parts: every
// operand is x = hi + lo 2^-11 with hi = fp16(x) and lo = fp16((x - hi) 2^11)
// (round to nearest; the scaled remainder stays clear of FP16's subnormals),
// and a product is hi.hi + (hi.lo + lo.hi) 2^-11 (lo.lo is below FP32
// rounding): 22 significant bits per operand, as many as two TF32 parts, in
// half the instructions and bytes.  The weights come split from the host;
// the activations are split when they are written.  The tensor cores' FP32
// accumulation is not IEEE round-to-nearest, so the large hi.hi terms go to
// two accumulators of 64 inputs each, which the epilogue adds with ordinary
// FP32 adds; the scaled small terms share a third.  The output layer is an
// FP32 dot product.
//
// Shared memory: two layer buffers of hi and lo weight planes (32 KB each,
// the canonical K-major no-swizzle layout of the instruction's A operand,
// prepared on the host; layer l + 2 is copied in by TMA bulk copies as soon
// as layer l's products are done), the activation planes (B operand, hi and
// lo), the output layer's partial sums and the mbarriers.  One thread issues
// the products; sixteen warps run the epilogue (warp w reads accumulator
// lanes 32 (w % 4) .. and a quarter of the nodes).  Every wait is bounded.
// ---------------------------------------------------------------------------
constexpr int kBandWarps = 16;
constexpr int kBandThreads = 32 * kBandWarps;
constexpr int kHidden = 128;                       // M of each product: one layer's outputs
constexpr int kBandIn = 16;                        // layer-1 inputs, zero-padded
constexpr float kBandLoScale = 2048.f;             // 2^11: the lo parts' scale
// per-net device layout: FP16 planes (layer 1 hi, lo [128 x 16]; layers 2..7
// hi, lo [128 x 128]), then FP32 b1[128], bh[6][128], wo[128]
constexpr int kBandL1Plane = kHidden * kBandIn;    // halves
constexpr int kBandLayerPlane = kHidden * kHidden; // halves
constexpr int kBandOffHid = 2 * kBandL1Plane;
constexpr int kBandHalves = kBandOffHid + 12 * kBandLayerPlane;
constexpr int kBandF32B1 = 0, kBandF32Bh = kHidden, kBandF32Wo = 7 * kHidden, kBandF32 = 8 * kHidden;
static_assert(kBandHalves % 8 == 0, "16-byte aligned FP32 part");
// A operand (weights), K-major no swizzle: 8-row x 16-byte core matrices,
// rows (outputs) 16 B apart, row groups of 8 128 B apart, k groups of 8
// (16 B) 2 KB apart
constexpr uint32_t kBandWSbo = 128, kBandWLbo = (kHidden / 8) * 128;
__host__ __device__ constexpr int band_w_index(int m, int k)  // half index in a weight plane
{
    return (k >> 3) * (int)(kBandWLbo / 2) + (m >> 3) * 64 + (m & 7) * 8 + (k & 7);
}
// shared memory (bytes): weight buffer b at b * kBandSmWBuf, hi plane then lo
constexpr int kBandSmWPlane = kBandLayerPlane * 2;
constexpr int kBandSmWBuf = 2 * kBandSmWPlane;

// Band nodes per block, N of each product: 96 with FP64 storage (there the
// bulk step is the longer leg, and fewer band blocks leave it more of the
// GPU), 48 otherwise (there the nets are the longer leg).  On the 2401 x 501
// plate 64 and 96 nodes per block made the FP32 step 30.1 and 34.2 us
// against 29.5; 48 and 128 made the FP64 step 45.4 and 44.2 us against 41.0.
__host__ __device__ constexpr int band_nodes(int storage) { return storage == ST_F64 ? 96 : 48; }

// The block's layout for N = NB nodes.
template <int NB>
struct BandShape {
    // B operand (activations), K-major no swizzle with N = NB rows; the
    // k-group stride is padded by 16 B so that a warp's 32 features land in
    // 16 banks
    static constexpr uint32_t ASbo = 128, ALbo = (NB / 8) * 128 + 16;
    static constexpr int ActPlane = (kHidden / 8) * ALbo;
    // shared memory (bytes): the two weight buffers, the activation planes,
    // [4][NB] output partial sums, [NB] net outputs, 3 mbarriers and the
    // tensor-memory address
    static constexpr int SmAH = 2 * kBandSmWBuf;
    static constexpr int SmAL = SmAH + ActPlane;
    static constexpr int SmRed = SmAL + ActPlane;
    static constexpr int SmOut = SmRed + 4 * NB * 4;
    static constexpr int SmBar = SmOut + NB * 4;
    static constexpr size_t SmemBytes = (size_t)SmBar + 3 * 8 + 8;
    // tensor memory: big accumulators at columns 0 and Acc, the small one at 2 Acc
    static constexpr uint32_t Acc = NB <= 64 ? 64 : 128;
    static constexpr uint32_t TmemCols = NB <= 64 ? 256 : 512;
    static constexpr uint32_t AccSmall = 2 * Acc;
    // the epilogue: warp w takes features 32 (w % 4) .. of nodes WarpNodes
    // (w / 4) .., in chunks of Chunk (at most 16: one reduce-scatter)
    static constexpr int WarpNodes = NB / 4;
    static constexpr int Chunk = WarpNodes <= 16 ? WarpNodes : (WarpNodes % 16 == 0 ? 16 : 12);
    // instruction descriptor (kind::f16): D F32 (bit 4), A and B F16 (0 at
    // bits 7, 10), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
    static constexpr uint32_t Idesc = (1u << 4) | ((uint32_t)(NB >> 3) << 17) | ((uint32_t)(kHidden >> 4) << 24);
    static_assert(NB % 16 == 0 && NB <= 128, "tcgen05 N, accumulators Acc columns apart");
    static_assert(WarpNodes % Chunk == 0 && Chunk % 4 == 0, "epilogue chunks");
    static_assert(ActPlane % 16 == 0 && SmBar % 8 == 0, "band_kernel shared-memory layout");
    static_assert(SmemBytes <= 227 * 1024, "band_kernel shared memory");
    static_assert(SmemBytes > 114 * 1024, "one band block per SM: two would share tensor memory");
    // byte offset of (node n, feature k) in an activation plane
    __device__ static uint32_t a_offset(int n, int k)
    {
        return (uint32_t)(k >> 3) * ALbo + (uint32_t)(n >> 3) * 128 + (uint32_t)(n & 7) * 16 + (uint32_t)(k & 7) * 2;
    }
};
template <int S>
using BandShapeOf = BandShape<band_nodes(S)>;

struct BandNode {
    int x, y, slot, nin;   // nin = 15 or 9
    int nb_slot[5];
    int nb_stale;          // bit q: neighbour q reads the previous step's moments
};

struct BandNet {
    const uint16_t* w16;    // kBandHalves FP16 plane values, 16-byte aligned
    const float* w32;       // kBandF32 biases and output weights
    float bo;
    int nin;
};

struct BandArgs {
    const BandNode* nodes;
    const int2* work;       // per block: (first node, count <= band_nodes); all of one net type
    const int* work_type;
    const int* in_slot;     // per block, node and neighbour q: 2 slot + (reads the previous step), or -1
    BandNet net[8];
    StepArgs s;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// `bytes` (a multiple of 16) from this GPU's global memory into shared memory
// by the TMA engine; completes `bytes` of the mbarrier's expected transfer
__device__ __forceinline__ void band_copy(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// one layer's two weight planes (hi at the buffer, lo one plane after it);
// the mbarrier's phase completes when both have landed
__device__ __forceinline__ void band_planes_async(uint32_t buf, const uint16_t* hi, uint32_t plane_bytes,
                                                  uint64_t* bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(2 * plane_bytes)
                 : "memory");
    band_copy(buf, hi, plane_bytes, bar);
    band_copy(buf + kBandSmWPlane, reinterpret_cast<const char*>(hi) + plane_bytes, plane_bytes, bar);
}

// wait for phase `parity` of an mbarrier, at most 2^22 polls (each poll may
// suspend the thread for a while); false when the limit ran out
__device__ __forceinline__ bool band_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// x = hi + lo 2^-11, hi and lo FP16 (round to nearest even)
__device__ __forceinline__ void f16_split(float x, __half& hi, __half& lo)
{
    hi = __float2half_rn(x);
    lo = __float2half_rn((x - __half2float(hi)) * kBandLoScale);
}

// shared-memory matrix descriptor: K-major, no swizzle, start / leading
// (k-group) / stride (8-row group) byte offsets in 16-byte units, version 1
__device__ __forceinline__ uint64_t band_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// D (tensor memory) = A x B^T (+ D when acc), issued by one thread
__device__ __forceinline__ void band_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// the mbarrier's arrival once every product this thread issued is done
__device__ __forceinline__ void band_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// one layer's products from weight buffer `wb` (K = 16 ksteps): big
// accumulator c <- hi.hi of inputs 64 c .. 64 c + 63; the small one <- hi.lo
// + lo.hi (scaled by 2^11); the mbarrier arrives when all are done
template <int NB>
__device__ __forceinline__ void band_layer_mma(uint32_t tmem, uint32_t wb, uint32_t ah, uint32_t al, int ksteps,
                                               uint64_t* bar)
{
    using B = BandShape<NB>;
    const uint32_t wl = wb + kBandSmWPlane;
    for (int ks = 0; ks < ksteps; ks++)
        band_mma(tmem + B::Acc * (uint32_t)(ks >> 2), band_desc(wb + ks * 2 * kBandWLbo, kBandWLbo, kBandWSbo),
                 band_desc(ah + ks * 2 * B::ALbo, B::ALbo, B::ASbo), B::Idesc, (ks & 3) != 0);
    for (int ks = 0; ks < ksteps; ks++)
        band_mma(tmem + B::AccSmall, band_desc(wb + ks * 2 * kBandWLbo, kBandWLbo, kBandWSbo),
                 band_desc(al + ks * 2 * B::ALbo, B::ALbo, B::ASbo), B::Idesc, ks != 0);
    for (int ks = 0; ks < ksteps; ks++)
        band_mma(tmem + B::AccSmall, band_desc(wl + ks * 2 * kBandWLbo, kBandWLbo, kBandWSbo),
                 band_desc(ah + ks * 2 * B::ALbo, B::ALbo, B::ASbo), B::Idesc, 1u);
    band_commit(bar);
}

// (FP64 storage: 2 in the launch bounds caps the kernel at 64 registers, so a
// band block leaves room for four of the bulk kernel's longer FP64 blocks on
// its SM; the FP32-class instances keep their registers, as the nets are the
// longer leg there.  Shared memory keeps band blocks one per SM.)
template <int S, int CO>
__global__ void __launch_bounds__(kBandThreads, S == ST_F64 ? 2 : 1) band_kernel(const BandArgs ba)
{
    using C = typename Store<S>::C;
    constexpr int NB = band_nodes(S);
    using BS = BandShape<NB>;
    const StepArgs& a = ba.s;
    extern __shared__ __align__(1024) unsigned char band_smem[];
    const uint32_t sb = smem_u32(band_smem);
    float* red = reinterpret_cast<float*>(band_smem + BS::SmRed);
    float* outv = reinterpret_cast<float*>(band_smem + BS::SmOut);
    // bar[0] / bar[1]: weight buffer 0 / 1 landed; bar[2]: a layer's products done
    uint64_t* bar = reinterpret_cast<uint64_t*>(band_smem + BS::SmBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 3);
    const int2 w = ba.work[blockIdx.x];
    const BandNet& net = ba.net[ba.work_type[blockIdx.x]];
    const uint16_t* __restrict__ w16 = net.w16;
    const float* __restrict__ w32 = net.w32;
    const C* sm_cur = reinterpret_cast<const C*>(a.side_m) + (long long)a.par * a.nslots * 3;
    const C* sm_old = reinterpret_cast<const C*>(a.side_m) + (long long)(a.par ^ 1) * a.nslots * 3;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // the bulk kernel, when launched as this grid's programmatic dependent,
    // may start once every block of this grid is resident
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    if (tid == 0) {
#pragma unroll
        for (int i = 0; i < 3; i++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[i])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // layer 1 into buffer 0, layer 2 into buffer 1
        band_planes_async(sb, w16, kBandL1Plane * 2, &bar[0]);
        band_planes_async(sb + kBandSmWBuf, w16 + kBandOffHid, kBandLayerPlane * 2, &bar[1]);
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(BS::TmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // inputs: (u_x, u_y, rho) of each neighbour cast to float (mesh.cpp:2805-2808);
    // item i < 5 NB fills inputs 3 q .. 3 q + 2 of node i / 5 (q =
    // i % 5), the next NB items the zero padding (input 15)
    static_assert(kBandIn == 16, "input staging");
    // prep_kernel's moments and populations: complete once its grid is (a
    // no-op without a programmatic primary)
    asm volatile("griddepcontrol.wait;" ::: "memory");
#pragma unroll
    for (int i = tid; i < 6 * NB; i += kBandThreads) {
        if (i < 5 * NB) {
            const int n = i / 5, q = i % 5;
            const int code = __ldg(ba.in_slot + (size_t)blockIdx.x * NB * 5 + i);
            float v[3] = {0.f, 0.f, 0.f};
            if (code >= 0) {
                const C* mm = ((code & 1) ? sm_old : sm_cur) + (long long)(code >> 1) * 3;
                v[0] = float(mm[1]);
                v[1] = float(mm[2]);
                v[2] = float(mm[0]);
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                __half hi, lo;
                f16_split(v[c], hi, lo);
                *reinterpret_cast<__half*>(band_smem + BS::SmAH + BS::a_offset(n, 3 * q + c)) = hi;
                *reinterpret_cast<__half*>(band_smem + BS::SmAL + BS::a_offset(n, 3 * q + c)) = lo;
            }
        } else {
            const int n = i - 5 * NB;
            *reinterpret_cast<__half*>(band_smem + BS::SmAH + BS::a_offset(n, 15)) = __float2half_rn(0.f);
            *reinterpret_cast<__half*>(band_smem + BS::SmAL + BS::a_offset(n, 15)) = __float2half_rn(0.f);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    bool ok = true;
    const int qd = warp & 3, k = 32 * qd + lane;  // this thread's output feature in the epilogue
    const int nb0 = BS::WarpNodes * (warp >> 2);  // and its first node
    const uint32_t trow0 = tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)nb0;
    const float wo = __ldg(w32 + kBandF32Wo + k);
    float bias = __ldg(w32 + kBandF32B1 + k);
#pragma unroll 1
    for (int l = 0; l < 7; l++) {
        const int b = l & 1;
        // the next layer's bias, a layer ahead of its use
        const float bias_next = l < 6 ? __ldg(w32 + kBandF32Bh + l * kHidden + k) : 0.f;
        if (tid == 0) {
            ok = band_wait(&bar[b], (l >> 1) & 1) && ok;
            tc_fence_after();
            band_layer_mma<NB>(tmem, sb + b * kBandSmWBuf, sb + BS::SmAH, sb + BS::SmAL,
                           l == 0 ? kBandIn / 16 : kHidden / 16, &bar[2]);
            if (l + 2 < 7) {
                // layer l + 2 into this buffer once the products here are done
                ok = band_wait(&bar[2], l & 1) && ok;
                band_planes_async(sb + b * kBandSmWBuf, w16 + kBandOffHid + (size_t)(l + 1) * 2 * kBandLayerPlane,
                                  kBandLayerPlane * 2, &bar[b]);
            }
        }
        __syncwarp();
        ok = band_wait(&bar[2], l & 1) && ok;
        __syncwarp();  // the tensor-memory loads below are warp-collective
        tc_fence_after();
        // epilogue: bias + the three accumulators, ReLU; split into the next
        // layer's activation planes, or (last layer) the output layer's
        // partial sums over this warp's 32 features
        constexpr int CH = BS::Chunk, NP = CH / 4;
#pragma unroll 1
        for (int h = 0; h < BS::WarpNodes / CH; h++) {
            const int nb = nb0 + CH * h;
            const uint32_t trow = trow0 + (uint32_t)(CH * h);
            uint32_t r[NP][3][4];
#pragma unroll
            for (int p = 0; p < NP; p++)
#pragma unroll
                for (int c = 0; c < 3; c++) tmem_ld4(trow + BS::Acc * (uint32_t)c + 4u * (uint32_t)p, r[p][c]);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[16];
#pragma unroll
            for (int p = 0; p < NP; p++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    float x = bias + __uint_as_float(r[p][0][j]);
                    if (l > 0) x += __uint_as_float(r[p][1][j]);
                    v[4 * p + j] = fmaxf(fmaf(__uint_as_float(r[p][2][j]), 1.f / kBandLoScale, x), 0.f);
                }
            if (l < 6) {
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    __half hi, lo;
                    f16_split(v[j], hi, lo);
                    *reinterpret_cast<__half*>(band_smem + BS::SmAH + BS::a_offset(nb + j, k)) = hi;
                    *reinterpret_cast<__half*>(band_smem + BS::SmAL + BS::a_offset(nb + j, k)) = lo;
                }
            } else {
                // output layer: the warp's 32 features of v * wo summed per
                // node by a reduce-scatter (lane L ends with node L % 16)
#pragma unroll
                for (int j = 0; j < 16; j++) v[j] = j < CH ? v[j] * wo : 0.f;
#pragma unroll
                for (int o = 8; o >= 1; o >>= 1) {
                    const bool up = lane & o;
#pragma unroll
                    for (int i = 0; i < o; i++) {
                        const float send = up ? v[i] : v[i + o];
                        const float keep = up ? v[i + o] : v[i];
                        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                    }
                }
                v[0] += __shfl_xor_sync(0xffffffffu, v[0], 16);
                if (lane < CH) red[qd * NB + nb + lane] = v[0];
            }
        }
        bias = bias_next;
        tc_fence_before();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
    }
    for (int n = tid; n < NB; n += kBandThreads)
        outv[n] = ((red[n] + red[NB + n]) + (red[2 * NB + n] + red[3 * NB + n])) + net.bo;
    if (__syncthreads_or(!ok) && tid == 0) {
        // a wait of some thread ran out: report it, and give what may still
        // be in flight one more bounded wait before the tensor memory is freed
        atomicExch(&a.ctr->err, 3);
        band_wait(&bar[2], 0);
        band_wait(&bar[0], 1);
        band_wait(&bar[1], 0);
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BS::TmemCols)
                     : "memory");
    }


    // tau (net output if >= 0.501, else Smagorinsky; mesh.cpp:2821-2827,
    // 392-396) and the collision of the band node
    if (tid < w.y) {
        const BandNode& bn = ba.nodes[w.x + tid];
        const double nn_tau = (double)outv[tid];
        const C* sf = reinterpret_cast<const C*>(a.side_f) + (long long)bn.slot * 9;
        const C* mm = sm_cur + (long long)bn.slot * 3;
        C f[9];
#pragma unroll
        for (int q = 0; q < 9; q++) f[q] = sf[q];
        const C rho = mm[0], ux = mm[1], uy = mm[2];
        const C rbs = rbase<S>(a);
        const bool use_nn = nn_tau >= 0.501;
        const long long node = (long long)bn.y * a.nx + bn.x;
        const C tau = use_nn       ? C(nn_tau)
                      : a.les == 3 ? C(a.tau_field[node])
                                   : node_tau<C>(f, rho, ux, uy, rbs, a.les, prm<C>(a.tau0, a.f_tau0),
                                                 prm<C>(a.cs, a.f_cs));
        if (a.mode >= MODE_MAT) {
            a.dl_tau[node] = double(tau);
            a.dl_m[3ll * a.nx * a.ny + node] = use_nn ? 1.0 : 0.0;
        } else {
            collide_node<C, CO>(f, rho, ux, uy, rbs, tau);
#pragma unroll
            for (int q = 0; q < 9; q++) stf<S>(a, q, bn.x, bn.y, f[q]);
        }
    }
}

// ---------------------------------------------------------------------------
// immersed boundary (mesh.cpp:514-832, 1244-1281 and NodeAndLattice.cpp:162-195)
// as one sequence of phases over kIbCtas blocks, separated by barriers
// (release / acquire: global-memory writes of one phase are visible to every
// block in the next):
//   nodes    post-stream state of every stencil node, from the previous field
//            (the bulk kernel skips these nodes)
//   markers  InterpolateVel + CalParticleForce: F_m = 2 (U_b - sum u delta)
//   spread   SpreadForce + UpdateVelocity: node force, u += F / (2 rho)
//            (markers and spread repeat for each direct-forcing pass)
//   finish   per-body force sums (FP64 fixed-order tree, one block per body)
//            and the forced nodes' collision with the corrected velocity and
//            the operator's forcing term
// In a normal step the phases run in the first IbArgs::nib blocks of the
// step's one launch (step_ib_fused, a global-memory barrier): kIbCtas, or
// more where there are many forced nodes (one block per kIbNodesPerBlock of
// them, at most one per SM, all of them in the launch's first wave); alone
// (ib_fused) they
// run as one thread-block cluster with cluster barriers.  Launched beside the
// bulk kernel on another stream instead, the IB work only found free SMs
// once the bulk kernel drained; as a separate cluster kernel with the bulk
// kernel as its programmatic dependent, the launch pair cost about 5 us per
// step more than one launch.
// ---------------------------------------------------------------------------
constexpr int kIbThreads = 128;  // threads per CTA of the IB cluster
constexpr int kIbCtas = 8;       // CTAs per cluster (portable cluster size)
constexpr int kIbNodesPerBlock = 512;  // forced nodes per IB block of step_ib_fused
constexpr int kIbMaxBlocks = 148;      // IB blocks of step_ib_fused at most (one per SM)

struct IbArgs {
    int nmark, nforced, nbody;
    // markers, sorted by body
    const double2* ub;          // prescribed velocity
    const double* ds;           // arc length (force weight)
    const int* st_node;         // [nmark][16] stencil -> forced-node index
    const double2* st_w;        // [nmark][16] (wa, wb): contribution (v * wa) * wb
    const int2* body_m;         // per body: (first marker, end marker)
    // forced nodes, CSR node -> (marker, wa, wb) in marker order
    const int* fn_slot;         // side-buffer slot
    const int2* fn_xy;
    const int* fn_ptr;          // [nforced + 1]
    const int* fe_marker;
    const double2* fe_w;
    // work arrays
    double* rho;                // per forced node
    double* ucx;
    double* ucy;
    double* fx;
    double* fy;
    double2* dmf;               // per marker: force of the current pass
    double2* mft;               // per marker: total force
    // outputs
    double* force_now;          // [nbody][2]
    double* force_hist;         // [hist_cap][nbody][2]
    int hist_cap;
    unsigned long long* bar;    // GridBar arrival counter (step_ib_fused)
    int bar_extra;              // arrivals each GridBar waits for beyond its blocks:
                                // 0, or > 0 in the test that lets the wait run out
    int nib;                    // IB blocks of step_ib_fused (kIbCtas .. kIbMaxBlocks)
    StepArgs s;
};

// cluster-wide barrier: arrive (release) + wait (acquire)
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

template <int S, int SC>
__device__ __forceinline__ void ib_node_item(const IbArgs& ia, int n, int t)
{
    using C = typename Store<S>::C;
    const StepArgs& a = ia.s;
    const int2 xy = ia.fn_xy[n];
    C f[9], rho, ux, uy;
    node_state<S, SC>(a, xy.x, xy.y, f, rho, ux, uy);
    C* sf = reinterpret_cast<C*>(a.side_f) + (long long)ia.fn_slot[n] * 9;
#pragma unroll
    for (int q = 0; q < 9; q++) sf[q] = f[q];
    node_epilogue<S>(a, (long long)xy.y * a.nx + xy.x, t, f, rho, ux, uy);
    ia.rho[n] = double(rho);
    ia.ucx[n] = double(ux);
    ia.ucy[n] = double(uy);
    ia.fx[n] = 0.0;
    ia.fy[n] = 0.0;
}

template <int NST>
__device__ __forceinline__ void ib_marker_item(const IbArgs& ia, int m, bool first_pass)
{
    double vx = 0.0, vy = 0.0;
#pragma unroll
    for (int q = 0; q < NST; q++) {
        const int sn = ia.st_node[m * 16 + q];
        const double2 sw = ia.st_w[m * 16 + q];
        vx += ia.ucx[sn] * sw.x * sw.y;
        vy += ia.ucy[sn] * sw.x * sw.y;
    }
    const double2 u = ia.ub[m];
    const double2 d = make_double2(2.0 * (u.x - vx), 2.0 * (u.y - vy));
    ia.dmf[m] = d;
    const double2 tot = first_pass ? make_double2(0.0, 0.0) : ia.mft[m];
    ia.mft[m] = make_double2(tot.x + d.x, tot.y + d.y);
}

__device__ __forceinline__ void ib_spread_item(const IbArgs& ia, int n)
{
    // the node's markers in CSR (marker) order, kIbGather at a time with all
    // loads of a group issued together: two memory round trips per group
    // instead of two per marker
    constexpr int kIbGather = 8;
    double dfx = 0.0, dfy = 0.0;
    const int e1 = ia.fn_ptr[n + 1];
    for (int e0 = ia.fn_ptr[n]; e0 < e1; e0 += kIbGather) {
        int mk[kIbGather];
        double2 wq[kIbGather], d[kIbGather];
#pragma unroll
        for (int j = 0; j < kIbGather; j++) {
            const bool on = e0 + j < e1;
            mk[j] = on ? ia.fe_marker[e0 + j] : 0;
            wq[j] = on ? ia.fe_w[e0 + j] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int j = 0; j < kIbGather; j++) d[j] = e0 + j < e1 ? ia.dmf[mk[j]] : make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < kIbGather; j++)
            if (e0 + j < e1) {
                dfx += d[j].x * wq[j].x * wq[j].y;
                dfy += d[j].y * wq[j].x * wq[j].y;
            }
    }
    const double r = ia.rho[n];
    ia.ucx[n] = ia.ucx[n] + 0.5 * 1 * dfx / r;
    ia.ucy[n] = ia.ucy[n] + 0.5 * 1 * dfy / r;
    ia.fx[n] += dfx;
    ia.fy[n] += dfy;
}

// body force -sum F ds over the body's markers: fixed-order tree over the CTA
template <int NT>
__device__ __forceinline__ void ib_body_sum(const IbArgs& ia, int b, int t, double (*red)[NT])
{
    const StepArgs& a = ia.s;
    const int tid = threadIdx.x;
    const int2 mr = ia.body_m[b];
    double sx = 0.0, sy = 0.0;
    for (int m = mr.x + tid; m < mr.y; m += NT) {
        sx -= ia.mft[m].x * ia.ds[m];
        sy -= ia.mft[m].y * ia.ds[m];
    }
    red[0][tid] = sx;
    red[1][tid] = sy;
    __syncthreads();
    for (int w = NT / 2; w; w >>= 1) {
        if (tid < w) {
            red[0][tid] += red[0][tid + w];
            red[1][tid] += red[1][tid + w];
        }
        __syncthreads();
    }
    if (tid == 0) {
        ia.force_now[2 * b] = red[0][0];
        ia.force_now[2 * b + 1] = red[1][0];
        if (a.mode == MODE_STEP || a.mode == MODE_INIT) {
            const long long h = (long long)(((t % ia.hist_cap) + ia.hist_cap) % ia.hist_cap);
            ia.force_hist[(h * ia.nbody + b) * 2] = red[0][0];
            ia.force_hist[(h * ia.nbody + b) * 2 + 1] = red[1][0];
        }
    }
    __syncthreads();  // red is reused by the next body
}

// collision of a forced node with the corrected velocity and forcing term
template <int S, int CO, bool LRN, int XT>
__device__ __forceinline__ void ib_collide_item(const IbArgs& ia, int n)
{
    using C = typename Store<S>::C;
    const StepArgs& a = ia.s;
    const C* sf = reinterpret_cast<const C*>(a.side_f) + (long long)ia.fn_slot[n] * 9;
    C f[9];
#pragma unroll
    for (int q = 0; q < 9; q++) f[q] = sf[q];
    const C rho = C(ia.rho[n]);
    const C ux = C(ia.ucx[n]), uy = C(ia.ucy[n]);
    const C rbs = rbase<S>(a);
    const int2 xy = ia.fn_xy[n];
    const C tau = XT            ? ext_tau<S>(a, xy.x, xy.y, f, rho, ux, uy, rbs)
                  : a.les == 3 ? C(a.tau_field[(long long)xy.y * a.nx + xy.x])
                               : node_tau<C, LRN>(f, rho, ux, uy, rbs, a.les, prm<C>(a.tau0, a.f_tau0),
                                                  prm<C>(a.cs, a.f_cs));
    if (a.mode >= MODE_MAT) {
        a.dl_tau[(long long)xy.y * a.nx + xy.x] = double(tau);
        if (LRN)
            a.dl_m[3ll * a.nx * a.ny + (long long)xy.y * a.nx + xy.x] =
                learned_in_range<C>(f, rho, ux, uy, rbs, prm<C>(a.tau0, a.f_tau0)) ? 1.0 : 0.0;
    } else {
        collide_node<C, CO>(f, rho, ux, uy, rbs, tau);
        add_force<C, CO>(f, ux, uy, C(ia.fx[n]), C(ia.fy[n]), prm<C>(a.tau0, a.f_tau0), tau);
#pragma unroll
        for (int q = 0; q < 9; q++) stf<S>(a, q, xy.x, xy.y, f[q]);
    }
}

// Barrier between the IB phases of the IB blocks.  ClusterBar: the kIbCtas
// blocks form one thread-block cluster (the hardware co-schedules it).
// GridBar: the blocks are the first nblk blocks of the step kernel; a
// monotonic 64-bit arrival counter in global memory, nbar barriers per
// launch, so each launch starts from a multiple of nblk * nbar (the first
// barrier cannot complete before every block has read it; the host zeroes
// the counter whenever a handle's nblk changes).  The wait is
// bounded: after 1 s (or kBarSpins polls) the block records the barrier
// error (Ctr::err = 2) and goes on, so a launch never hangs.  The IB blocks are
// the lowest block indices of a launch on an otherwise idle stream and the
// other blocks never wait on them, so they are resident long before then.
struct ClusterBar {
    __device__ __forceinline__ void operator()() { cluster_sync(); }
};

constexpr int kBarSpins = 1 << 26;                  // polls, and
constexpr unsigned long long kBarNanos = 1000000000ull;  // 1 s of waiting at most

struct GridBar {
    unsigned long long* ctr;
    unsigned long long base;
    int k;
    Ctr* err;
    int extra;
    int nblk;
    __device__ __forceinline__ void operator()()
    {
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(ctr, 1ull);
            k++;
            const unsigned long long target = base + (unsigned long long)k * (nblk + extra);
            int it = 0;
            unsigned long long v, t0, now;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            do {
                asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(ctr) : "memory");
                if (v >= target) break;
                __nanosleep(64);
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
            } while (++it < kBarSpins && now - t0 < kBarNanos);
            if (v < target) atomicExch(&err->err, 2);
            __threadfence();
        } else {
            k++;
        }
        __syncthreads();
    }
};

// The force part of the IB sub-step in nblk blocks of NT threads (block
// blk): stencil-node states, direct-forcing passes, the corrected
// velocities into the gradient field (WALE / coherent model; with a barrier
// after them when SYNC_MAC, for collisions in the same launch), body sums.
template <int S, int SC, int NST, int XT, int NT, bool SYNC_MAC, typename Bar>
__device__ __forceinline__ void ib_force_phases(const IbArgs& ia, int passes, int blk, int nblk,
                                                double (*red)[NT], Bar& bar, int t)
{
    const int T = nblk * NT;
    const int g = blk * NT + threadIdx.x;
    for (int n = g; n < ia.nforced; n += T) ib_node_item<S, SC>(ia, n, t);
    bar();
    for (int p = 0; p < passes; p++) {
        for (int m = g; m < ia.nmark; m += T) ib_marker_item<NST>(ia, m, p == 0);
        bar();
        for (int n = g; n < ia.nforced; n += T) ib_spread_item(ia, n);
        bar();
    }
    if (XT && (ia.s.les == 4 || ia.s.les == 5)) {
        using C = typename Store<S>::C;
        C* m = reinterpret_cast<C*>(ia.s.mac);
        const int pl = ia.s.nx * ia.s.ny;
        for (int n = g; n < ia.nforced; n += T) {
            const int2 xy = ia.fn_xy[n];
            m[xy.y * ia.s.nx + xy.x] = C(ia.ucx[n]);
            m[pl + xy.y * ia.s.nx + xy.x] = C(ia.ucy[n]);
        }
        if (SYNC_MAC) bar();
    }
    for (int b = blk; b < ia.nbody; b += nblk) ib_body_sum<NT>(ia, b, t, red);
}

// The IB sub-step of one launch, in nblk blocks of NT threads (block blk):
// the force part, then the forced nodes' collisions.
template <int S, int SC, int CO, bool LRN, int NST, int XT, int NT, typename Bar>
__device__ __forceinline__ void ib_phases(const IbArgs& ia, int passes, int blk, int nblk, double (*red)[NT],
                                          Bar& bar)
{
    const int T = nblk * NT;
    const int g = blk * NT + threadIdx.x;
    const int t = step_time(ia.s);
    // the step counter of the next step (a bulk kernel beside this one does
    // not write it; the others write the same value)
    if (ia.s.mode == MODE_STEP && g == 0) ia.s.ctr->t[ia.s.par ^ 1] = t + 1;
    ib_force_phases<S, SC, NST, XT, NT, true>(ia, passes, blk, nblk, red, bar, t);
    for (int n = g; n < ia.nforced; n += T) ib_collide_item<S, CO, LRN, XT>(ia, n);
}

// the IB sub-step alone, launched as exactly one cluster (gridDim.x ==
// kIbCtas): initialisation and download modes, timed and boundary-net steps
template <int S, int SC, int CO, bool LRN, int NST, int XT = 0>
__global__ void __launch_bounds__(kIbThreads) ib_fused(const IbArgs ia, int passes)
{
    __shared__ double red[2][kIbThreads];
    ClusterBar bar;
    ib_phases<S, SC, CO, LRN, NST, XT, kIbThreads>(ia, passes, blockIdx.x, gridDim.x, red, bar);
}

// A normal step with markers in ONE launch: blocks 0 .. nib-1 perform the
// IB sub-step (GridBar between its phases), the rest are the bulk row
// segments (block nib + by * tiles_x + bx).  The IB blocks are
// dispatched first, so they run beside the bulk blocks from the start, and
// the step ends when the launch does.
template <int S, int SC, int CO, bool LRN, int NST, int XT, int AV>
__global__ void __launch_bounds__(kBlockX, (step_min_blocks<S, LRN>())) step_ib_fused(const IbArgs ia, int passes)
{
    __shared__ double red[2][kBlockX];
    __shared__ unsigned long long s_base;
    const int nib = ia.nib;
    if ((int)blockIdx.x < nib) {
        const unsigned long long nbar =
            1ull + 2ull * (unsigned long long)passes + ((XT && (ia.s.les == 4 || ia.s.les == 5)) ? 1ull : 0ull);
        if (threadIdx.x == 0) {
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(ia.bar) : "memory");
            s_base = v - v % (nbar * (unsigned long long)nib);
        }
        __syncthreads();
        GridBar bar{ia.bar, s_base, 0, ia.s.ctr, ia.bar_extra, nib};
        ib_phases<S, SC, CO, LRN, NST, XT, kBlockX>(ia, passes, blockIdx.x, nib, red, bar);
        return;
    }
    const int tile = blockIdx.x - nib;
    const int by = tile / ia.s.tiles_x, bx = tile - by * ia.s.tiles_x;
    bulk_tile_any<S, CO, SC, LRN, XT, AV>(ia.s, bx, by, threadIdx.x);
}

// the post-stream velocity of node (x, y) into StepArgs::mac (closures 4,
// 5): the state the step's collision sees, before the IB correction
template <int S, int SC>
__device__ __forceinline__ void mac_node(const StepArgs& a, int x, int y, bool skip_forced)
{
    using C = typename Store<S>::C;
    if (x >= a.nx) return;
    const int node = y * a.nx + x, pl = a.nx * a.ny;
    const uint8_t nf = a.nflag[node];
    if (skip_forced && (nf & NF_DEFER)) return;  // written by the IB blocks
    C f[9], rho, ux = C(0), uy = C(0);
    if (nf & NF_SOLID) {
    } else if ((nf & NF_SBND) && a.mode != MODE_INIT && a.mode != MODE_MAT_INIT) {
        solid_pull<S>(a, x, y, f);
        macros<C>(f, rbase<S>(a), rho, ux, uy);
    } else {
        node_state<S, SC>(a, x, y, f, rho, ux, uy);
    }
    C* m = reinterpret_cast<C*>(a.mac);
    m[node] = ux;
    m[pl + node] = uy;
}

template <int S, int SC>
__global__ void __launch_bounds__(kBlockX) mac_kernel(const StepArgs a)
{
    mac_node<S, SC>(a, blockIdx.x * kBlockX + threadIdx.x, blockIdx.y, false);
}

// WALE / coherent model with markers, a normal step in two launches.  First:
// blocks 0 .. kIbCtas-1 the force part of the IB sub-step (GridBar between
// phases; the corrected velocities into the gradient field), the others the
// post-stream velocities of every other node.  Second: blocks 0 ..
// kIbCtas-1 the forced nodes' collisions, the others the bulk row segments;
// every velocity the gradients read is final by then.
template <int S, int SC, int NST>
__global__ void __launch_bounds__(kBlockX, (step_min_blocks<S, false>())) mac_ib_fused(const IbArgs ia, int passes)
{
    __shared__ double red[2][kBlockX];
    __shared__ unsigned long long s_base;
    if (blockIdx.x < kIbCtas) {
        const unsigned long long nbar = 1ull + 2ull * (unsigned long long)passes;
        if (threadIdx.x == 0) {
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(ia.bar) : "memory");
            s_base = v - v % (nbar * kIbCtas);
        }
        __syncthreads();
        GridBar bar{ia.bar, s_base, 0, ia.s.ctr, ia.bar_extra, kIbCtas};
        const int t = step_time(ia.s);
        if (ia.s.mode == MODE_STEP && blockIdx.x == 0 && threadIdx.x == 0) ia.s.ctr->t[ia.s.par ^ 1] = t + 1;
        ib_force_phases<S, SC, NST, 1, kBlockX, false>(ia, passes, blockIdx.x, kIbCtas, red, bar, t);
        return;
    }
    const int tile = blockIdx.x - kIbCtas;
    const int by = tile / ia.s.tiles_x, bx = tile - by * ia.s.tiles_x;
    mac_node<S, SC>(ia.s, bx * kBlockX + threadIdx.x, by, true);
}

template <int S, int SC, int CO, bool LRN, int AV>
__global__ void __launch_bounds__(kBlockX, (step_min_blocks<S, LRN>())) collide_ib_fused(const IbArgs ia)
{
    if (blockIdx.x < kIbCtas) {
        for (int n = blockIdx.x * kBlockX + threadIdx.x; n < ia.nforced; n += kIbCtas * kBlockX)
            ib_collide_item<S, CO, LRN, 1>(ia, n);
        return;
    }
    const int tile = blockIdx.x - kIbCtas;
    const int by = tile / ia.s.tiles_x, bx = tile - by * ia.s.tiles_x;
    bulk_tile<S, CO, SC, LRN, 1, AV>(ia.s, bx, by, threadIdx.x);
}

// ---------------------------------------------------------------------------
// small utility kernels
// ---------------------------------------------------------------------------
static __global__ void style_kernel(uint8_t* out, int nx, int ny, int plate_x0, int scene,
                                   const uint8_t* nflag)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny) return;
    const int x = (int)(i % nx), y = (int)(i / nx);
    if (nflag[i] & (NF_SOLID | NF_SBND)) {
        out[i] = (uint8_t)((nflag[i] & NF_SOLID) ? 's' : 'b');  // JudgeStyle's solid / boundary
        return;
    }
    if (scene == SC_REF) {
        out[i] = (uint8_t)ref_style(x, y, nx, ny, plate_x0);
    } else {
        out[i] = (uint8_t)(x == 0 ? 'i' : (x == nx - 1 ? 'o' : ((y == 0 || y == ny - 1) ? 'w' : 'f')));
    }
}

// Momentum exchange on solid links (Mesh::OutputCd, mesh.cpp:1461-1526):
// F = sum over fluid nodes x and directions k with x + e_k solid of
// e_k (fnew_opp(k)(x) + fcol_k(x)); fnew is the materialised post-stream
// field (FP64), fcol the post-collision field the last step started from.
// One block, fixed-order tree: deterministic.
template <int S>
__global__ void __launch_bounds__(256) solid_force_kernel(const StepArgs a, const int2* links, int nlink,
                                                         const double* fnew, double* out)
{
    __shared__ double red[2][256];
    const int tid = threadIdx.x;
    const long long pl = (long long)a.nx * a.ny;
    const double rb = double(rbase<S>(a));
    double sx = 0.0, sy = 0.0;
    for (int l = tid; l < nlink; l += 256) {
        const int node = links[l].x, k = links[l].y;
        const int x = node % a.nx, y = node / a.nx;
        const double fc = double(ldf<S>(a, k, x, y)) + WK<double>(k) * rb;
        const double v = fnew[OPP(k) * pl + node] + fc;
        sx += EX(k) * v;
        sy += EY(k) * v;
    }
    red[0][tid] = sx;
    red[1][tid] = sy;
    __syncthreads();
    for (int w = 128; w; w >>= 1) {
        if (tid < w) {
            red[0][tid] += red[0][tid + w];
            red[1][tid] += red[1][tid + w];
        }
        __syncthreads();
    }
    if (tid == 0) {
        out[0] = red[0][0];
        out[1] = red[1][0];
    }
}

template <typename C>
__global__ void to_double_kernel(const C* in, double* out, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = double(in[i]);
}

// element-wise type conversion (grid-stride), for the FP32 host-buffer calls
template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ in, B* __restrict__ out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = B(in[i]);
}

// deterministic FP64 sum: per-block partial sums, then one block
static __global__ void sum_partial_kernel(const double* in, long long n, double* part)
{
    __shared__ double red[256];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        s += in[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// run diagnostics of the materialised moments m = [rho, ux, uy, net flag]
// [ny][nx] over the non-solid nodes: out[0] = bit pattern of the largest |u|
// (non-negative doubles order as their bit patterns, and a NaN's pattern lies
// above every number's, so one NaN shows), out[1] / out[2] = nodes with the
// net flag set / clear (learned model only).  out[] is zeroed by the caller.
static __global__ void diag_kernel(const double* __restrict__ m, const uint8_t* __restrict__ nflag, long long nn,
                                   int learned, unsigned long long* out)
{
    unsigned long long mx = 0, net = 0, fb = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        if (nflag[i] & NF_SOLID) continue;
        const double ux = m[nn + i], uy = m[2 * nn + i];
        const unsigned long long b = (unsigned long long)__double_as_longlong(sqrt(ux * ux + uy * uy));
        mx = b > mx ? b : mx;
        if (learned) {
            if (m[3 * nn + i] != 0.0) net++;
            else fb++;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = v > mx ? v : mx;
        net += __shfl_xor_sync(0xffffffffu, net, o);
        fb += __shfl_xor_sync(0xffffffffu, fb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, mx);
        if (learned) {
            atomicAdd(out + 1, net);
            atomicAdd(out + 2, fb);
        }
    }
}

}  // namespace ippi
