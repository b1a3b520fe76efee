/*
 * ippi_lbm.h -- C ABI of the B200 D2Q9 time step (libippi_lbm.so).
 *
 * The reference (IPPI-LBM) has no plugin or FFI: its boundary is the C++
 * class API that main.cpp calls.  These entry points are what that API's
 * methods bind to in the drop-in host layer (host/mesh.cpp):
 *
 *   ippi_create        Mesh::InitialLatMesh + Mesh::JudgeStyle
 *                      (mesh.cpp:60-171, 1391-1454); Parameter.h switches
 *                      (Parameter.h:8-21) and main.cpp constants (main.cpp:12-65)
 *                      become ippi_params fields
 *   ippi_init_macros   Lattice::InitialLatticeFeq over the mesh
 *                      (NodeAndLattice.cpp:69-123; mesh.cpp:159-166)
 *   ippi_reequilibrate the same in the middle of a run, as
 *                      Mesh::ManageDataFromXflow / XflowABS do
 *                      (mesh.cpp:2391-2398, 2615-2620)
 *   ippi_set_markers   Mesh::InitialIBParticle (mesh.cpp:173-191) -- the IB
 *                      sub-step InterpolateVel / CalParticleForce / SpreadForce /
 *                      UpdateVelocity (mesh.cpp:552, 514, 656, 1244) then runs
 *                      inside every ippi_step
 *   ippi_load_band_net the model loads of Mesh::NNmodel_Type00..07
 *                      (mesh.cpp:2767-3259): weights once, not per call
 *   ippi_step          Mesh::OneLBMStep (mesh.cpp:357-513) followed by
 *                      Mesh::ComputeAvgVelocity (mesh.cpp:1954-1974), nsteps times
 *   ippi_download      the LatMesh fields read by Mesh::WriteDatFluid
 *                      (mesh.cpp:1180-1243) and the flags of JudgeStyle
 *   ippi_forces        the marker force sums of Mesh::OutputCd's role
 *                      (mesh.cpp:1461-1526), from the IB marker forces, FP64
 *   ippi_last_error    cerr messages of the reference (e.g. ErrorCatch,
 *                      mesh.cpp:2101-2111, which called MPI_Abort)
 *
 * Conventions: every call returns IPPI_OK (0) or a negative IPPI_ERR_* code
 * and never throws.  A handle owns all of its device memory and one CUDA
 * stream; host pointers are borrowed for the duration of the call.  A handle
 * is not thread-safe.  Arrays on the lattice are row-major [ny][nx] (x
 * fastest); populations are [9][ny][nx] in the reference's D2Q9 order
 * (0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE).
 */
#ifndef IPPI_LBM_H
#define IPPI_LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IPPI_ABI_VERSION 3

/* status codes */
#define IPPI_OK 0
#define IPPI_ERR_ARG (-1)      /* bad argument (sizes, enum values, tau <= 0.5) */
#define IPPI_ERR_CUDA (-2)     /* a CUDA call failed; see ippi_last_error       */
#define IPPI_ERR_DIVERGED (-3) /* rho left [0,10] or became NaN (ErrorCatch)    */
#define IPPI_ERR_STATE (-4)    /* call not valid in the handle's current state  */
#define IPPI_ERR_NOMEM (-5)    /* device allocation failed                      */

/* collision operator (Parameter.h SRTLBM / MRT / RRLBM) */
#define IPPI_BGK 0
#define IPPI_MRT 1
#define IPPI_RR 2
/* population storage; arithmetic is FP64 for IPPI_F64, FP32 otherwise, on
 * populations shifted by w_k * rho0 */
#define IPPI_F64 0
#define IPPI_F32 1
#define IPPI_F16 2
#define IPPI_BF16 3
/* boundary set */
#define IPPI_BC_REF_NEE 0   /* the reference's flat-plate scene (mesh.cpp:228-356) */
#define IPPI_BC_CHANNEL 1   /* Zou-He parabolic inlet, NEE outlet, bounce-back walls */
/* subgrid model */
#define IPPI_LES_NONE 0
#define IPPI_LES_SMAGORINSKY 1 /* SmagorinskyByHybrid, mesh.cpp:852-911 */
#define IPPI_LES_LEARNED 2     /* per-node network (ippi_load_tau_mlp), Smagorinsky
                                  outside its training range; channel scene only */
#define IPPI_LES_FIELD 3       /* a given relaxation time per node (ippi_set_tau_field);
                                  channel scene */
/* The closures the reference keeps as alternatives in Mesh::CaculateLESTau
 * (channel scene only): */
#define IPPI_LES_WALE 4        /* WALE on forward-difference velocity gradients,
                                  mesh.cpp:934-967 */
#define IPPI_LES_CSM 5         /* coherent-structure Cs (ComputeDynamicCs), mesh.cpp:1034-1071,
                                  2113-2146 */
#define IPPI_LES_DYNAMIC 6     /* wall-damped Cs = 3 / (1 + 1.71828^(6 - d)),
                                  mesh.cpp:968-1000; d from ippi_set_wall_distance */
/* IB interpolation/spreading kernel */
#define IPPI_DELTA_BILINEAR 0 /* mesh.cpp:606-644 (default of Parameter.h) */
#define IPPI_DELTA_PESKIN4 1  /* Dirac_Delta, mesh.cpp:555-605, 1354-1389 */

/* fields for ippi_download */
#define IPPI_FIELD_F 0       /* fnew after the last step, double [9][ny][nx]   */
#define IPPI_FIELD_RHO 1     /* double [ny][nx]                                 */
#define IPPI_FIELD_UX 2
#define IPPI_FIELD_UY 3
#define IPPI_FIELD_TAU 4     /* relaxation time the next collision uses        */
#define IPPI_FIELD_AVG_U 5   /* time averages of ComputeAvgVelocity            */
#define IPPI_FIELD_AVG_V 6
#define IPPI_FIELD_AVG_RHO 7
#define IPPI_FIELD_FLAGS 8   /* uint8 [ny][nx]: JudgeStyle chars f i o m d u (w) */
#define IPPI_FIELD_NNFLAG 9  /* double [ny][nx]: 1 where a boundary net sets tau;
                                with IPPI_LES_LEARNED, 1 where the learned network
                                set it (0: Smagorinsky fallback, solid nodes) */

typedef struct ippi_lbm ippi_lbm;

typedef struct {
    int nx, ny;          /* lattice (main.cpp:20-21 Nx, Ny)                   */
    int collision;       /* IPPI_BGK / IPPI_MRT / IPPI_RR                     */
    int storage;         /* IPPI_F64 / IPPI_F32 / IPPI_F16 / IPPI_BF16        */
    int bc_set;          /* IPPI_BC_REF_NEE / IPPI_BC_CHANNEL                 */
    int les_model;       /* IPPI_LES_NONE / IPPI_LES_SMAGORINSKY              */
    double tau0;         /* startTau (main.cpp:43)                            */
    double cs;           /* Smagorinsky constant (main.cpp:12)                */
    double u_in;         /* flat plate: inlet velocity (mesh.cpp:244 uses 0.1);
                            channel: centre-line velocity u_max               */
    double rho0;         /* reference density and population shift (1.0)    */
    int plate_x0;        /* flat plate: specular bottom for x < plate_x0
                            (mesh.cpp:1413 uses 400)                          */
    int avg_start;       /* startAvg (main.cpp:54)                            */
    int delta_kernel;    /* IPPI_DELTA_BILINEAR / IPPI_DELTA_PESKIN4          */
    int mdf_iters;       /* direct-forcing passes per step, >= 1              */
    int device;          /* CUDA device ordinal                               */
} ippi_params;

/* ABI version of the loaded library (IPPI_ABI_VERSION). */
int ippi_abi_version(void);

/* Fill *p with the reference's defaults: BGK, F64, flat plate, Smagorinsky,
 * tau0 from main.cpp:43 for the given size, cs 0.173, u_in 0.1, rho0 1,
 * plate_x0 400, avg_start 30000, bilinear delta, one forcing pass. */
void ippi_params_default(ippi_params* p, int nx, int ny);

/* Create a lattice (flags, buffers, stream) initialised to rho = 1, u = 0. */
int ippi_create(const ippi_params* p, ippi_lbm** out);
int ippi_destroy(ippi_lbm* h);

/* Set rho/u on every node and the populations to their equilibrium
 * (InitialLatticeFeq).  NULL arrays mean rho = 1 / u = 0.  Resets averages. */
int ippi_init_macros(ippi_lbm* h, const double* rho, const double* ux, const double* uy);

/* ippi_init_macros for FP32 host arrays: the Lattice fields of the
 * reference's SINGLE build (Parameter.h REAL = float) that InitialLatticeFeq
 * reads (NodeAndLattice.cpp:69-123).  The values are widened to FP64 on the
 * device; half the bytes cross the bus. */
int ippi_init_macros_f32(ippi_lbm* h, const float* rho, const float* ux, const float* uy);
/* Lattice::InitialLatticeFeq on every node in the middle of a run (the
 * reference's ManageDataFromXflow / XflowABS, mesh.cpp:2391-2398, 2615-2620):
 * populations replaced by the equilibrium of the given moments (NULL: rho 1,
 * u 0), with the running means and the force history kept.  Needs a step
 * taken. */
int ippi_reequilibrate(ippi_lbm* h, const double* rho, const double* ux, const double* uy);

/* Immersed-boundary markers: positions xy[2n], prescribed velocities ub[2n]
 * (NULL = at rest), body id per marker body[n] (NULL = all 0), arc length per
 * marker ds[n] (NULL = 1, the reference's force omits the area factor,
 * mesh.cpp:527).  Every stencil node must lie at least 3 nodes inside the
 * lattice.  n = 0 removes the markers. */
int ippi_set_markers(ippi_lbm* h, int n, const double* xy, const double* ub,
                     const int* body, const double* ds);

/* Weights of boundary net `type` (0..7) in TorchScript parameter order of
 * NNmodel/AutoT0<type>.pt: hidden_layer1 weight[128][nin], bias[128],
 * hidden_layer2..7 weight[128][128], bias[128], output_layer weight[1][128],
 * bias[1]; nin = 15 for types 1, 3, 5, 7 and 9 for 0, 2, 4, 6.  The nets act
 * with the BGK operator only, as in the reference.  They are evaluated with
 * FP32 accuracy on the tensor cores (every operand as two FP16 parts, FP32
 * sums): outputs agree with libtorch's FP32 forward to about 1e-7. */
int ippi_load_band_net(ippi_lbm* h, int type, const float* w, size_t n);

/* Advance nsteps time steps numbered t0, t0+1, ... (t feeds the averages,
 * mesh.cpp:1958-1971).  Returns IPPI_ERR_DIVERGED if rho left [0,10] or became
 * NaN in any of them.  Synchronises the handle's stream. */
int ippi_step(ippi_lbm* h, int nsteps, int t0);

/* No counterpart in the reference (measurement): ippi_step with device
 * timing.  The steps are queued behind a short hold on the handle's stream
 * (about 0.5 ms of GPU time), so they run back to back however slowly the host
 * issues them, and *ms receives the milliseconds between CUDA events recorded
 * on that stream just before the first step and just after the last.  A
 * pending initial collision runs before the timed region. */
int ippi_step_timed(ippi_lbm* h, int nsteps, int t0, double* ms);

/* The Smagorinsky constant of the following steps: the Cs argument of
 * Mesh::OneLBMStep, passed on to Mesh::CaculateLESTau each step (mesh.cpp
 * 357, 852-911).  cs >= 0; changing it rebuilds the step graphs. */
int ippi_set_les_cs(ippi_lbm* h, double cs);

/* Copy a field to host memory; bytes must equal the field's size. */
int ippi_download(ippi_lbm* h, int field, void* host, size_t bytes);

/* ippi_download into FP32 host memory, the LatMesh fields WriteDatFluid reads
 * under the reference's SINGLE build (mesh.cpp:1180-1243 with REAL = float):
 * any field but IPPI_FIELD_FLAGS, rounded to FP32 on the device; bytes must
 * equal the field's element count times 4. */
int ippi_download_f32(ippi_lbm* h, int field, float* host, size_t bytes);

/* Force on each body (lattice units, FP64, computed by the IB sub-step on the
 * current velocity field): force_xy[2 * nbody] = (Fx, Fy); *nbody receives
 * the body count (may be NULL).  mass (may be NULL) receives sum(rho) over
 * the lattice in FP64. */
int ippi_forces(ippi_lbm* h, double* force_xy, int* nbody, double* mass);

/* Per-step body forces recorded by the IB sub-step: out[step][body][2] for
 * the last min(max_steps, recorded) steps; returns the number of steps
 * written (>= 0) or an error code. */
int ippi_force_history(ippi_lbm* h, double* out, int max_steps);

/* The CUDA stream the handle launches on (a cudaStream_t), for event timing. */
int ippi_get_stream(ippi_lbm* h, void** stream);

/* Device timing of `nsteps` steps launched one by one with CUDA events around
 * each launch: average milliseconds of the bulk stream-collide kernel, and of
 * the side-stream chain (prep + boundary nets, or prep + IB) that runs
 * concurrently with it, reported in ms_band when nets are active and in
 * ms_ib when markers are (0 when absent).  Advances the simulation like
 * ippi_step. */
int ippi_profile_steps(ippi_lbm* h, int nsteps, int t0, double* ms_bulk,
                       double* ms_band, double* ms_ib);

/* No counterpart in the reference: the learned relaxation time
 * (IPPI_LES_LEARNED).  tau = tau0 + out_scale * softplus(MLP(x)) with
 * x = (features - mean) / std and the MLP 6 -> 32 tanh -> 32 tanh -> 1.
 * Features of a node, from its post-stream state (Pi_neq as in the
 * Smagorinsky model, S = -3/(2 rho tau0) Pi_neq):
 *   rho, |u|, Pi_xx/|Pi|, Pi_xy/|Pi|, Pi_yy/|Pi|, |S| = sqrt(2 S:S)
 * with |Pi| = sqrt(Pi_xx^2 + 2 Pi_xy^2 + Pi_yy^2).  Nodes with any feature
 * outside [lo, hi] take the Smagorinsky tau.
 * w_bf16[1313]: BF16 bit patterns of W1[32][6] b1[32] W2[32][32] b2[32]
 * w3[32] b3 (row-major, out x in).  stats[25]: mean[6] std[6] lo[6] hi[6]
 * out_scale.
 * The step kernels read the network from the device's constant memory, which
 * holds one network at a time: calls that run them for a learned-model
 * handle hold a per-device lock until their stream has drained, and copy
 * the handle's network in when another one is there.  Learned-model handles
 * on one device therefore take turns, also across host threads.  The record
 * of which network the constant memory holds assumes the device's primary
 * context lives as long as the process (no cudaDeviceReset between calls). */
#define IPPI_MLP_PARAMS 1313
#define IPPI_MLP_STATS 25
int ippi_load_tau_mlp(ippi_lbm* h, const uint16_t* w_bf16, size_t n, const float* stats,
                      size_t nstats);

/* No counterpart in the reference: the learned tau's 32 x 32 hidden layer on
 * the tensor cores (on != 0) or on FP32 FMA (0, the default) in the step's
 * bulk row segments.  On the tensor cores each warp multiplies its 32 nodes'
 * layer-1 activations, rounded to BF16, by the BF16 weights with FP32
 * accumulation (mma.sync m16n8k16); the IB-forced nodes, downloads and the
 * adjoint keep the FMA network, and the adjoint refuses to run while this is
 * on.  IPPI_LES_LEARNED with FP32 / FP16 / BF16 storage only. */
int ippi_set_learned_tensor_cores(ippi_lbm* h, int on);

/* No counterpart in the reference: the relaxation time of every node for
 * IPPI_LES_FIELD, tau[ny][nx] (host, each > 0.5) -- the parameter field of
 * the adjoint's tau gradient. */
int ippi_set_tau_field(ippi_lbm* h, const double* tau);

/* Filtered snapshot of the current state for training the learned tau:
 * box filter over factor x factor blocks (nx, ny multiples of factor) into
 * out[6][ny/factor][nx/factor] (host, FP64): rho_bar, ux_bar, uy_bar
 * (density-weighted), Sxx, Sxy, Syy of the effective stress
 *   Sigma = box(sigma) - (box(rho u u) - rho_bar u_bar u_bar),
 *   sigma = -(1 - 1/(2 tau)) Pi_neq  (the lattice's deviatoric stress),
 * i.e. the stress a coarse lattice must carry to reproduce the filtered
 * fine-lattice momentum flux. */
int ippi_filter_snapshot(ippi_lbm* h, int factor, double* out, size_t bytes);

/* Training kernels of the learned tau (FP32, device pointers, enqueued on
 * `stream`; deterministic for a given n).
 * ippi_mlp_grad: x[n][6] standardised features, y[n] targets of
 *   softplus(MLP(x)) (offset / out_scale), w[1313] FP32 parameters ->
 *   grad[1313] of the mean squared error and *loss (may be NULL); scratch
 *   holds ippi_mlp_scratch_floats() floats.
 * ippi_mlp_adam: one Adam step (step >= 1) on w with moments m, v.
 * ippi_mlp_forward: out[n] = softplus(MLP(x)). */
#define IPPI_MLP_GRAD_BLOCKS 296
int ippi_mlp_param_count(void);
size_t ippi_mlp_scratch_floats(void);
int ippi_mlp_grad(const float* x, const float* y, int n, const float* w, float* grad, float* loss,
                  float* scratch, void* stream);
int ippi_mlp_adam(float* w, const float* grad, float* m, float* v, int step, float lr, float beta1,
                  float beta2, float eps, void* stream);
int ippi_mlp_forward(const float* x, int n, const float* w, float* out, void* stream);

/* ippi_load_tau_mlp with FP32 weights used as given (no BF16 rounding):
 * for gradient checks and end-to-end training through the solver. */
int ippi_load_tau_mlp_f32(ippi_lbm* h, const float* w, size_t n, const float* stats, size_t nstats);

/* No counterpart in the reference: reverse-mode gradients through the step
 * (channel scene; BGK / MRT / RR; tau constant, Smagorinsky, learned or a
 * field; immersed boundary with one direct-forcing pass).
 * ippi_adjoint_forward advances nsteps steps numbered t0.. like ippi_step,
 * keeping the state before every ckpt_every-th step on the device.
 * ippi_adjoint_backward then returns, for the loss L whose partial
 * derivatives are
 *   dl_dforce[nsteps][nbody][2]  dL / d(body force of each step) (may be NULL)
 *   dl_dmacro[3][ny][nx]        dL / d(rho, ux, uy) of the last step's
 *                               post-stream state, i.e. the fields
 *                               ippi_download gives after the rollout (may be NULL),
 * the gradients (host arrays, FP64, each may be NULL):
 *   grad_tau[ny][nx]   with respect to the tau field (IPPI_LES_FIELD)
 *   grad_mlp[1313]     with respect to the network weights (IPPI_LES_LEARNED)
 *   grad_f0[9][ny][nx] with respect to the populations before the first step
 * Each segment of ckpt_every steps is recomputed from its checkpoint with the
 * forward kernels; the reverse sweep is FP64. */
int ippi_adjoint_forward(ippi_lbm* h, int nsteps, int t0, int ckpt_every);
int ippi_adjoint_backward(ippi_lbm* h, const double* dl_dforce, const double* dl_dmacro,
                          double* grad_tau, double* grad_mlp, double* grad_f0);

/* Implicit relaxation-time inference, Mesh::FindAndWriteTau (mesh.cpp:2625-
 * 2715): for each of n interior nodes xy[n][2] and target moments
 * target[n][3] (rho, u, v), the dtau = m * step, m = m_lo .. m_hi (the
 * reference: -10000 .. 10000, 1e-5), for which the 9 upstream neighbours,
 * relaxed with BGK at their tau + dtau and streamed into the node, give
 * moments closest to the target in |rho - R| + |jx - U| + |jy - V| (first
 * minimum).  best_dtau[n], best_err[n] are host arrays.  ippi_tau_scan uses
 * the handle's current post-stream state (populations, moments, the tau of
 * the next collision); ippi_tau_scan_state takes that state as device arrays
 * f[9][ny][nx], m3[3][ny][nx], tau[ny][nx] (and device xy, target, outputs),
 * enqueued on `stream`.  The scan reproduces the sequential FP64 scan bit for
 * bit. */
int ippi_tau_scan(ippi_lbm* h, int n, const int* xy, const double* target, int m_lo, int m_hi,
                  double step, double* best_dtau, double* best_err);
int ippi_tau_scan_state(const double* f, const double* m3, const double* tau, int nx, int ny, int n,
                        const int* xy, const double* target, int m_lo, int m_hi, double step,
                        double* best_dtau, double* best_err, void* stream);

/* Solid nodes (the reference's 's' style): solid[ny][nx] != 0 marks a solid
 * node, at least 3 nodes inside the lattice (channel scene).  Fluid nodes
 * with a link into a solid ('b') take halfway bounce-back on it; solid nodes
 * are not updated and download as fluid at rest.  n = 0 removes them.
 * ippi_solid_force: the momentum-exchange force on the solids after the
 * last step, Mesh::OutputCd (mesh.cpp:1461-1526): the sum over 'b' nodes and
 * directions k into a solid of e_k (fnew_opp(k) + fcol_k), FP64, as the
 * reference sums it (before its 1/(rho U^2 R) scaling). */
int ippi_set_solid(ippi_lbm* h, const uint8_t* solid, size_t n);
int ippi_solid_force(ippi_lbm* h, double* force_xy);

/* IPPI_LES_DYNAMIC: the wall distance d[ny][nx] of every node (Mesh::
 * SetNormalDis, mesh.cpp:1935-1953, computes it for the cylinder). */
int ippi_set_wall_distance(ippi_lbm* h, const double* dist);

/* No counterpart in the reference (its state is written only as Tecplot
 * text, mesh.cpp:1180-1233).  Diagnostics of the state after the last step,
 * for a metrics log: the largest |u| over the non-solid nodes (NaN once the
 * state holds a NaN), and with IPPI_LES_LEARNED the number of non-solid nodes
 * whose relaxation time the network set and the number where the features
 * left its training range and Smagorinsky set it (both 0 for other models).
 * Any output may be NULL.  Synchronises. */
int ippi_diagnostics(ippi_lbm* h, double* max_u, long long* net_nodes, long long* fallback_nodes);

/* No counterpart in the reference (it has no restart path).  Checkpoint and
 * resume of the evolving state: both population buffers (the current one and
 * the input of the last step, which downloads re-run), the running means, the
 * flat-plate corner values, the drag/lift of the last step and the force
 * history, and the step bookkeeping (last user step, internal step count).
 * The configuration is not saved: the resuming handle is created and set up
 * (parameters, markers, solid mask, wall distance, tau field or network) as
 * the saving one was; a hash of the parameters, markers and solid mask in the
 * checkpoint must match, and so must the FP64 mass the state gives when its
 * last step is re-run under the resuming handle's configuration.  The buffer
 * also carries a hash of its payload.  Layout: a fixed header then the raw
 * device sections, native byte order.
 *
 * ippi_state_bytes: size of the checkpoint of this handle.
 * ippi_save_state: write it into host[bytes] (bytes >= ippi_state_bytes);
 *   IPPI_ERR_STATE before the handle's first step.
 * ippi_load_state: restore from host[bytes]; *last_step (may be NULL) gets the
 *   user step number of the saved state's last step, so stepping resumes at
 *   *last_step + 1.  IPPI_ERR_ARG on a bad magic, version, size, hash or mass;
 *   on a mass mismatch the handle holds the loaded state but must not be
 *   trusted.  Synchronise. */
int ippi_state_bytes(ippi_lbm* h, size_t* bytes);
int ippi_save_state(ippi_lbm* h, void* host, size_t bytes);
int ippi_load_state(ippi_lbm* h, const void* host, size_t bytes, int* last_step);

/* Last error message of the handle (or of the library when h is NULL). */
int ippi_last_error(ippi_lbm* h, char* buf, size_t n);

/* No counterpart in the reference.  Deterministic FP64 sum of a density
 * field rho[ny][nx] (device memory) into *mass (device memory), enqueued on
 * `stream` (a cudaStream_t, NULL = default stream), without allocating any
 * device memory: for callers that cannot call cudaMalloc where they need the
 * mass checksum (device memory owned by another allocator, such as a
 * framework's caching allocator or a fixed arena reserved at start-up, and
 * loops that forbid allocation after start-up).  Its scratch is a fixed
 * device array of IPPI_NOALLOC_MAX_ROWS row sums that the library keeps on
 * every GPU it is loaded on until the process exits; ny beyond that is
 * rejected with IPPI_ERR_ARG.  The first call on a device looks up that
 * array's device address and keeps it, so make that first call before any
 * stream capture; the kept address assumes the device's primary context
 * lives as long as the process (no cudaDeviceReset between calls).  Calls
 * share the array: calls that overlap on the GPU race.  A launch error
 * already pending from the caller's earlier work is left pending (not
 * cleared) and makes the call return IPPI_ERR_CUDA. */
#define IPPI_NOALLOC_MAX_ROWS 16384
int ippi_mass_noalloc(const double* rho, int nx, int ny, double* mass, void* stream);

#ifdef __cplusplus
}
#endif
#endif
