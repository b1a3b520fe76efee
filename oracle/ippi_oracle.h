/*
 * ippi_oracle.h -- FP64 CPU restatement of the IPPI-LBM D2Q9 time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against.  Only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py may load it; the product library never links or calls it.
 *
 * What it restates (file:line in the reference project IPPI-LBM/):
 *   - node flags            Mesh::JudgeStyle        mesh.cpp:1391-1454
 *   - initial populations   Lattice::InitialLatticeFeq NodeAndLattice.cpp:69-123
 *   - equilibrium           Lattice::Compute_feq    NodeAndLattice.cpp:124-149
 *   - BGK / MRT / RR        NodeAndLattice.cpp:150-161, 290-360, 228-288
 *   - macroscopics          Lattice::CalMacro       NodeAndLattice.cpp:196-227
 *   - Smagorinsky "hybrid"  Mesh::CaculateLESTau    mesh.cpp:852-911
 *   - step order            Mesh::OneLBMStep        mesh.cpp:357-513
 *   - pull streaming        Mesh::Streaming         mesh.cpp:192-226
 *   - NEE/specular BCs      Mesh::BoundaryCondition mesh.cpp:228-356
 *   - learned boundary tau  Mesh::NNmodel_Type00..07 mesh.cpp:2767-3259
 *   - error check           Mesh::ErrorCatch        mesh.cpp:2101-2111
 *   - time averages         Mesh::ComputeAvgVelocity mesh.cpp:1954-1974
 *   - IB markers/interp/force/spread/update
 *                           mesh.cpp:173-191, 552-655, 514-551, 656-832, 1244-1281
 *   - Peskin 4-point delta  Mesh::DiracDelta        mesh.cpp:1354-1389
 *   - Guo forcing term      Lattice::Compute_Disforce NodeAndLattice.cpp:162-195
 * and, for the channel scene that has no reference code (parabolic Zou-He
 * inlet, zero-gradient outlet, halfway bounce-back walls), the same
 * published schemes the CUDA kernels implement.
 *
 * Parity pin: the flat-plate step (flags, BGK/MRT/RR + Smagorinsky, NEE and
 * specular boundaries, averages, IB primitives) is pinned against the
 * reference sources compiled by oracle/build_ref.sh (tests/golden fixtures
 * and tests/test_oracle.py); the boundary networks are pinned against
 * outputs of the shipped TorchScript nets (tests/golden/band_net_golden.npz).
 * The channel scene is pinned only by analytic known-answer tests.
 */
#ifndef IPPI_ORACLE_H
#define IPPI_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* Threads of the per-node loops (collision, streaming, averages, velocity
 * update): OpenMP over columns, with each node's arithmetic unchanged, so
 * results do not depend on the count.  1 when built without OpenMP. */
int orc_threads(void);

typedef struct {
    int nx, ny;          /* global lattice (reference Nx, Ny)                    */
    int collision;       /* 0 BGK, 1 MRT, 2 RR                                   */
    int bc_set;          /* 0 reference flat plate (NEE), 1 channel (ZH/ZG/BB)   */
    int les_model;       /* 0 constant tau0, 1 Smagorinsky "hybrid", 2 learned,
                            3 given tau per node (orc_set_tau_field), 4 WALE,
                            5 coherent structure, 6 wall-damped Cs
                            (orc_set_wall_distance)                              */
    double tau0;         /* startTau                                              */
    double cs;           /* Smagorinsky constant                                 */
    double u_in;         /* inlet velocity (flat plate) / u_max (channel)         */
    double rho0;         /* reference density (1.0)                              */
    int plate_x0;        /* bottom wall: specular for x < plate_x0, NEE no-slip after */
    int avg_start;       /* startAvg                                              */
    int delta_kernel;    /* 0 bilinear 2x2, 1 Peskin 4x4                          */
    int mdf_iters;       /* direct-forcing passes per step (>=1)                  */
} orc_params;

enum { ORC_F = 0, ORC_RHO = 1, ORC_UX = 2, ORC_UY = 3, ORC_TAU = 4,
       ORC_AVG_U = 5, ORC_AVG_V = 6, ORC_AVG_RHO = 7, ORC_FLAGS = 8,
       ORC_NNFLAG = 9 };

orc* orc_create(const orc_params* p);
void orc_destroy(orc* s);
/* rho/ux/uy are [ny][nx] row-major (x fastest); NULL means rho=1, u=0. */
void orc_init_macros(orc* s, const double* rho, const double* ux, const double* uy);
/* Markers: xy[2n], ub[2n] (prescribed marker velocity), body[n] (or NULL), ds[n]
 * (or NULL for 1).  Returns 0, or -1 if a stencil node lies closer than 3
 * nodes to the lattice edge. */
int orc_set_markers(orc* s, int n, const double* xy, const double* ub,
                    const int* body, const double* ds);
/* TorchScript-layout weights of one boundary net (see band-net layout). */
int orc_load_band_net(orc* s, int type, const float* w, size_t n);
/* Advance nsteps reference time steps, numbered t0 .. t0+nsteps-1.
 * Returns 0, or -3 when ErrorCatch fired (rho outside [0,10] or NaN). */
int orc_step(orc* s, int nsteps, int t0);
/* Fields on the global grid, x fastest: F is [9][ny][nx], the rest [ny][nx].
 * TAU / NNFLAG give the relaxation time the next collision will use. */
void orc_get(orc* s, int field, double* out);
/* Force on each body (lattice units, FP64) from an IB sub-step evaluated on
 * the current velocity field (state untouched), and the mass sum(rho). */
int orc_forces(orc* s, double* force_xy, double* mass);
/* One IB sub-step on the current state (interpolate, force, spread, velocity
 * update) for unit parity with the reference IB primitives: writes marker
 * velocities vref[2n], marker forces mforce[2n], node forces nforce[2][ny][nx]
 * and leaves the corrected velocity in the state.  Any pointer may be NULL. */
void orc_ib_probe(orc* s, double* vref, double* mforce, double* nforce);
int orc_num_bodies(orc* s);

/* Solid nodes (channel scene): solid[ny][nx] != 0, at least 3 nodes from
 * the edges, or NULL to remove them.  Fluid links into a solid take halfway
 * bounce-back; solid nodes read as fluid at rest.  Returns 0 or -1. */
int orc_set_solid(orc* s, const unsigned char* solid);
/* Momentum-exchange force on the solids after the last step
 * (Mesh::OutputCd's sum, before its scaling). */
void orc_solid_force(orc* s, double* force_xy);

/* Building blocks exposed for unit tests. */
double orc_peskin_phi(double r);
float orc_band_forward(const float* w, int nin, const float* in);
/* stencil of one marker: writes up to 16 (x,y,weight) triples, returns count */
int orc_marker_stencil(int delta_kernel, double mx, double my,
                       int* xs, int* ys, double* ws);
/* One collision on a single node (fnew[9], rho, ux, uy, tau) -> fcol[9]. */
void orc_collide_node(int collision, const double* fnew, double rho, double ux,
                      double uy, double tau, double* fcol);
double orc_les_tau(const double* fnew, double rho, double ux, double uy,
                   double tau0, double cs);
/* IB forcing term added after one collision of a forced node (per operator,
 * see force_term in ippi_oracle.c) -> lf[9]. */
void orc_force_node(int collision, double ux, double uy, double fx, double fy, double tau0,
                    double tau, double* lf);

/* Learned relaxation time (no reference code; les_model 2): network
 * parameters w[1313] (the FP32 values of the BF16 weights: W1[32][6] b1[32]
 * W2[32][32] b2[32] w3[32] b3) and stats[25] (mean[6] std[6] lo[6] hi[6]
 * out_scale).  Returns 0, or -1 on a bad size. */
int orc_load_tau_mlp(orc* s, const float* w, size_t n, const float* stats, size_t nstats);
/* wall distance per node for les_model 6 (wall-damped Cs): [ny][nx] global. */
int orc_set_wall_distance(orc* s, const double* d);
/* tau per node for les_model 3: [ny][nx] global. */
int orc_set_tau_field(orc* s, const double* tau);
/* Mesh::FindAndWriteTau's scan (mesh.cpp:2625-2715) over candidates m_lo..m_hi
 * (dtau = m * step) for n nodes xy[n][2] with targets target[n][3]; state
 * f [9][ny][nx], m3 [3][ny][nx] (rho, ux, uy), tau [ny][nx]. */
void orc_tau_scan_state(const double* f, const double* m3, const double* tau, int nx, int ny,
                        int n, const int* xy, const double* target, int m_lo, int m_hi,
                        double step, double* best_dtau, double* best_err);
/* tau0 + out_scale * softplus(MLP(features)), Smagorinsky outside [lo, hi];
 * p = the 1338 parameters + statistics as doubles */
double orc_learned_tau(const double* fnew, double rho, double ux, double uy,
                       double tau0, double cs, const double* p);

#ifdef __cplusplus
}
#endif
#endif
