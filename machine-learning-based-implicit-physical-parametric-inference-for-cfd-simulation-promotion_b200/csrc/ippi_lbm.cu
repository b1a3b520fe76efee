// ippi_lbm.cu -- the C ABI of include/ippi_lbm.h: lattice handle, device
// buffers, side-buffer tables for the boundary nets and the immersed
// boundary, step launches captured in CUDA graphs, downloads.
//
// Device layout (one handle):
//   f[2]      populations, [9][ny][pitch] in the storage type, ping-pong;
//             buffer `cur` holds the latest post-collision field and the
//             other one the field before it (needed to reconstruct the
//             post-stream state for downloads)
//   nflag     uint8 [ny][nx], slot int32 [ny][nx], tile uint8 [ny][gx]:
//             nodes whose moments other kernels read (net inputs, marker
//             stencils) or whose collision is finished by another kernel
//   side_f    [nslots][9], side_m [2][nslots][3] (compute type)
//   avg       [3][ny][nx] running means (compute type)
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/ippi_lbm.h"
#include "adjoint.h"
#include "launch.h"

using namespace ippi;

namespace {

char g_last_error[512] = "";

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct NetHost {
    bool loaded = false;
    int nin = 0;
    std::vector<float> w;  // TorchScript order
};

}  // namespace

struct ippi_lbm {
    ippi_params p;
    int S;          // storage
    int csize;      // bytes of the compute type
    int tsize;      // bytes of the storage type
    cudaStream_t st = nullptr;
    long long pitch = 0, plane = 0;
    int gx = 0;
    void* f[2] = {nullptr, nullptr};
    int cur = 0;
    Ctr* ctr = nullptr;
    Ctr* ctr_h = nullptr;  // pinned mirror
    cudaStream_t side = nullptr;   // concurrent prep / net / IB kernels
    int side_prio = 0;             // their launch priority (the device's highest)
    cudaEvent_t fork = nullptr, join = nullptr;
    uint8_t* nflag = nullptr;
    uint8_t* tile = nullptr;
    int nslots = 0;
    PrepNode* prep_d = nullptr;    // nodes whose post-stream state the side kernels need
    int nprep = 0;
    int ib_nst = 4;
    bool ib_active = false;
    void* side_f = nullptr;
    void* side_m = nullptr;
    void* corner = nullptr;
    void* avg = nullptr;
    double* init_m = nullptr;
    float* io32 = nullptr;    // [9][ny][nx] staging of the FP32 host-buffer calls
    bool pending_init = true;
    int last_t = 0;     // user step number of the last executed step
    int kcount = 0;     // internal steps executed (init counts as k = 0)
    // materialised download fields (valid until the next step)
    double* dl = nullptr;     // [9 + 4 + 1][ny][nx]: f, rho ux uy nnflag, tau
    bool dl_valid = false;
    uint8_t* dl_flags = nullptr;
    double* red = nullptr;    // reduction partials
    // boundary nets
    NetHost nets[8];
    float* net_dev[8] = {};
    std::vector<BandNode> band_nodes;
    BandNode* band_nodes_d = nullptr;
    int2* band_work_d = nullptr;
    int* band_type_d = nullptr;
    int* band_in_d = nullptr;  // [blocks][band_nodes][5] net input slots
    int band_blocks = 0;
    // immersed boundary
    int nmark = 0, nbody = 0, nforced = 0, hist_cap = 0;
    std::vector<double> mk_xy, mk_ub, mk_ds;
    std::vector<int> mk_body;
    std::vector<DevBuf> ib_bufs;
    IbArgs ib{};
    double* force_now = nullptr;
    double* force_hist = nullptr;
    long long hist_written = 0;
    // learned tau: parameters (FP32 values of the BF16 weights) + statistics
    float* mlp_dev = nullptr;
    std::vector<float> mlp_host;   // the loaded parameters + statistics (FP32 values)
    bool mlp_tc = false;           // hidden layer on the tensor cores (ippi_set_learned_tensor_cores)
    MlpFrag* mlp_frag = nullptr;   // lane fragments of W2, b2, w3 for warp_mlp_tc
    unsigned long long mlp_version = 0;  // unique per network load (g_mlp_serial)
    double* tau_field = nullptr;  // IPPI_LES_FIELD: [ny][nx]
    unsigned long long* ib_bar = nullptr;  // arrival counter of the one-launch step's IB blocks
    void* mac = nullptr;          // IPPI_LES_WALE / CSM: [2][ny][nx] compute type, velocities
    double* wall_dist = nullptr;  // IPPI_LES_DYNAMIC: [ny][nx]
    // hashes of the inputs a checkpoint presumes besides the parameters: the
    // tau field, the learned network (weights and statistics), the wall
    // distance (0 = never set)
    uint64_t tau_field_hash = 0, mlp_hash = 0, wall_hash = 0;
    // solid nodes (halfway bounce-back) and their momentum-exchange links
    std::vector<uint8_t> solid;   // [ny][nx] or empty
    int2* solid_links = nullptr;  // (fluid node, direction into the solid)
    int nlinks = 0;
    double* solid_out = nullptr;
    // adjoint: the recorded rollout (checkpoints every K steps) and work buffers
    struct Adjoint {
        bool ready = false;
        int nsteps = 0, t0 = 0, K = 0;
        std::vector<void*> ck;   // state before steps 0, K, 2K, ...
        std::vector<void*> seg;  // recomputed inputs of one segment
        std::vector<void*> work; // everything else, freed together
    } adj;
    bool no_avg = false;         // forward recomputes must not touch the averages
    // graphs of two steps and of one step: [start buffer][step parity]
    // step graphs by [start buffer][parity of the first step][averaging]
    cudaGraphExec_t graph[2][2][2] = {};
    cudaGraphExec_t graph1[2][2][2] = {};
    // rows with flagged tiles (StepArgs::rowmask / row_shift)
    unsigned rowmask[kRowMaskWords] = {};
    int row_shift = 0;
    char err[512] = "";
};

// Initial moment table [3][nn]: fills the fields the caller did not give
// (rho = 1, u = 0) and records the first node with rho <= 0 (or NaN) or a
// non-finite velocity in *bad (all ones when there is none).
__global__ void init_fields_kernel(double* m, long long nn, int has_rho, int has_ux, int has_uy,
                                   unsigned long long* bad)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        if (!has_rho) m[i] = 1.0;
        if (!has_ux) m[nn + i] = 0.0;
        if (!has_uy) m[2 * nn + i] = 0.0;
        if (!(m[i] > 0) || !isfinite(m[nn + i]) || !isfinite(m[2 * nn + i]))
            atomicMin(bad, (unsigned long long)i);
    }
}

// Box filter of the materialised post-stream state over fac x fac blocks
// (ippi_filter_snapshot).  dl planes: f[0..8], rho 9, ux 10, uy 11, tau 13.
__global__ void filter_snapshot_kernel(const double* dl, int nx, int ny, int fac, double* out)
{
    const int cx = blockIdx.x * blockDim.x + threadIdx.x, cy = blockIdx.y;
    const int mx = nx / fac, my = ny / fac;
    if (cx >= mx || cy >= my) return;
    const long long nn = (long long)nx * ny;
    double r = 0, jx = 0, jy = 0, txx = 0, txy = 0, tyy = 0, sxx = 0, sxy = 0, syy = 0;
    for (int dy = 0; dy < fac; dy++)
        for (int dx = 0; dx < fac; dx++) {
            const long long n = (long long)(cy * fac + dy) * nx + (cx * fac + dx);
            const double* f = dl + n;
            const double rho = dl[9 * nn + n], ux = dl[10 * nn + n], uy = dl[11 * nn + n];
            const double tau = dl[13 * nn + n];
            const double d = f[5 * nn] + f[6 * nn] + f[7 * nn] + f[8 * nn];
            const double pxx = f[1 * nn] + f[3 * nn] + d - rho / 3 - rho * ux * ux;
            const double pyy = f[2 * nn] + f[4 * nn] + d - rho / 3 - rho * uy * uy;
            const double pxy = f[5 * nn] - f[6 * nn] + f[7 * nn] - f[8 * nn] - rho * ux * uy;
            const double c = -(1.0 - 0.5 / tau);
            sxx += c * pxx;
            sxy += c * pxy;
            syy += c * pyy;
            r += rho;
            jx += rho * ux;
            jy += rho * uy;
            txx += rho * ux * ux;
            txy += rho * ux * uy;
            tyy += rho * uy * uy;
        }
    const double inv = 1.0 / ((double)fac * fac);
    const double rb = r * inv, ub = jx / r, vb = jy / r;
    const long long m = (long long)mx * my, o = (long long)cy * mx + cx;
    out[o] = rb;
    out[m + o] = ub;
    out[2 * m + o] = vb;
    out[3 * m + o] = sxx * inv - (txx * inv - rb * ub * ub);
    out[4 * m + o] = sxy * inv - (txy * inv - rb * ub * vb);
    out[5 * m + o] = syy * inv - (tyy * inv - rb * vb * vb);
}

namespace {

int fail(ippi_lbm* h, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) snprintf(h->err, sizeof h->err, "%s", buf);
    snprintf(g_last_error, sizeof g_last_error, "%s", buf);
    return code;
}

#define CK(h, call)                                                                     \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(h, e_ == cudaErrorMemoryAllocation ? IPPI_ERR_NOMEM : IPPI_ERR_CUDA, \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

template <typename P>
cudaError_t dalloc(P** p, size_t bytes)
{
    return cudaMalloc((void**)p, bytes ? bytes : 16);
}

void dfree(void* p)
{
    if (p) cudaFree(p);
}

// FP32 value -> BF16 bits, round to nearest even (finite values)
uint16_t bf16_bits(float v)
{
    uint32_t u;
    std::memcpy(&u, &v, 4);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

// The lane fragments of warp_mlp_tc from a parameter block (lbm_common.cuh
// layout): for lane (g = lane / 4, t = lane % 4), k step kt and output tile
// nt, the B registers of mma.m16n8k16 hold W2[n][k], W2[n][k + 1] and
// W2[n][k + 8], W2[n][k + 9] as BF16 pairs (n = 8 nt + g, k = 16 kt + 2 t,
// the smaller k in the low half); then b2 and w3 at columns c, c + 1
// (c = 8 nt + 2 t), the accumulator columns the lane holds.
MlpFrag mlp_fragments(const float* w)
{
    MlpFrag fr;
    for (int lane = 0; lane < 32; lane++) {
        const int g = lane >> 2, t = lane & 3;
        uint32_t words[16];
        for (int kt = 0; kt < 2; kt++)
            for (int nt = 0; nt < 4; nt++) {
                const int n = 8 * nt + g, k = 16 * kt + 2 * t;
                const float* row = w + kMlpW2 + n * kMlpHid;
                words[(kt * 4 + nt) * 2] = bf16_bits(row[k]) | ((uint32_t)bf16_bits(row[k + 1]) << 16);
                words[(kt * 4 + nt) * 2 + 1] = bf16_bits(row[k + 8]) | ((uint32_t)bf16_bits(row[k + 9]) << 16);
            }
        for (int q = 0; q < 4; q++)
            fr.e[q][lane] = make_uint4(words[4 * q], words[4 * q + 1], words[4 * q + 2], words[4 * q + 3]);
        auto bits = [](float v) {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            return u;
        };
        for (int nt = 0; nt < 4; nt++) {
            const int c = 8 * nt + 2 * t;
            fr.e[4 + nt][lane] = make_uint4(bits(w[kMlpB2 + c]), bits(w[kMlpB2 + c + 1]), bits(w[kMlpW3 + c]),
                                            bits(w[kMlpW3 + c + 1]));
        }
    }
    return fr;
}

// grid of the grid-stride conversion kernels: 256-thread blocks, at most
// 32 per SM of a 148-SM device
unsigned convert_blocks(size_t n)
{
    return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 32));
}

void drop_graphs(ippi_lbm* h)
{
    for (int b = 0; b < 2; b++)
        for (int q = 0; q < 2; q++)
            for (int v = 0; v < 2; v++)
                for (cudaGraphExec_t* g : {&h->graph[b][q][v], &h->graph1[b][q][v]})
                    if (*g) {
                        cudaGraphExecDestroy(*g);
                        *g = nullptr;
                    }
}

void adjoint_free(ippi_lbm* h)
{
    for (auto* v : {&h->adj.ck, &h->adj.seg, &h->adj.work}) {
        for (void* p : *v) dfree(p);
        v->clear();
    }
    h->adj.ready = false;
}

// NVTX range over a library call: shown by profilers that record NVTX, a
// no-op otherwise
class Range {
public:
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// The fused learned-tau kernels read the network from their storage module's
// constant memory (c_mlp), which holds one network per device at a time.  The
// calls that launch those kernels hold the device's lock (MlpLock), copy the
// handle's network there on the handle's stream when another one is loaded
// (mlp_const_ready), and drain the stream before they let go of the lock, so
// learned handles on one device take turns even across host threads.  The
// record of which network each module holds assumes the device's primary
// context (and with it the constant memory) lives as long as the process: a
// cudaDeviceReset between calls is not supported.
constexpr int kMaxDevices = 64;
std::recursive_mutex g_mlp_mu[kMaxDevices];
unsigned long long g_mlp_loaded[kMaxDevices][4] = {};  // network version in each storage module
std::atomic<unsigned long long> g_mlp_serial{0};

class MlpLock {
public:
    explicit MlpLock(ippi_lbm* h)
    {
        if (h && h->p.les_model == IPPI_LES_LEARNED && h->mlp_dev && h->p.device >= 0 &&
            h->p.device < kMaxDevices) {
            h_ = h;
            g_mlp_mu[h->p.device].lock();
        }
    }
    ~MlpLock()
    {
        if (!h_) return;
        cudaStreamSynchronize(h_->st);
        g_mlp_mu[h_->p.device].unlock();
    }
    MlpLock(const MlpLock&) = delete;
    MlpLock& operator=(const MlpLock&) = delete;

private:
    ippi_lbm* h_ = nullptr;
};

// with the device's lock held and the device current: the handle's network
// into the constant memory of its storage module, if another one is there
int mlp_const_ready(ippi_lbm* h)
{
    if (h->p.les_model != IPPI_LES_LEARNED || !h->mlp_dev) return IPPI_OK;
    if (h->p.device < 0 || h->p.device >= kMaxDevices)
        return fail(h, IPPI_ERR_ARG, "learned tau on device %d (at most %d devices)", h->p.device, kMaxDevices);
    unsigned long long& loaded = g_mlp_loaded[h->p.device][h->S];
    if (loaded == h->mlp_version) return IPPI_OK;
    void* dst = nullptr;
    cudaError_t e;
    switch (h->S) {
    case ST_F64: e = mlp_const_addr_f64(&dst); break;
    case ST_F32: e = mlp_const_addr_f32(&dst); break;
    case ST_F16: e = mlp_const_addr_f16(&dst); break;
    default: e = mlp_const_addr_bf16(&dst); break;
    }
    CK(h, e);
    nvtxMarkA("ippi tau network to constant memory");
    CK(h, cudaMemcpyAsync(dst, h->mlp_dev, (size_t)(kMlpParams + kMlpStats) * sizeof(float),
                          cudaMemcpyDeviceToDevice, h->st));
    loaded = h->mlp_version;
    return IPPI_OK;
}

cudaError_t launch(const LaunchSet& L, int S)
{
    switch (S) {
    case ST_F64: return launch_f64(L);
    case ST_F32: return launch_f32(L);
    case ST_F16: return launch_f16(L);
    default: return launch_bf16(L);
    }
}

// Mesh::DiracDelta (mesh.cpp:1367-1384), same expressions as the oracle
double peskin_phi(double x)
{
    if (std::fabs(x) < 1) {
        double R = 1.0 + 4.0 * std::fabs(x) - 4 * (x * x);
        return (1.0 / 8.0) * (3.0 - 2.0 * std::fabs(x) + std::sqrt(R));
    } else if (std::fabs(x) < 2) {
        double R = -7.0 + 12.0 * std::fabs(x) - 4 * (x * x);
        return (1.0 / 8.0) * (5.0 - 2.0 * std::fabs(x) - std::sqrt(R));
    }
    return 0;
}

// Marker stencil of InterpolateVel / SpreadForce (mesh.cpp:566-585, 618-638):
// node (X, Y) contributes (value * wa) * wb.
int marker_stencil(int kernel, double mx, double my, int* xs, int* ys, double* wa, double* wb)
{
    const int XInt = (int)mx, YInt = (int)my;
    int n = 0;
    if (kernel == IPPI_DELTA_PESKIN4) {
        for (int X = XInt - 1; X <= XInt + 2; X++)
            for (int Y = YInt - 1; Y <= YInt + 2; Y++) {
                xs[n] = X;
                ys[n] = Y;
                wa[n] = peskin_phi(mx - X) * peskin_phi(my - Y);
                wb[n] = 1.0;
                n++;
            }
    } else {
        for (int X = XInt; X <= XInt + 1; X++)
            for (int Y = YInt; Y <= YInt + 1; Y++) {
                xs[n] = X;
                ys[n] = Y;
                wa[n] = 1 - std::fabs(mx - X);
                wb[n] = 1 - std::fabs(my - Y);
                n++;
            }
    }
    return n;
}

// ---------------------------------------------------------------------------
// boundary-net band: nodes, neighbour references, call order
// ---------------------------------------------------------------------------
struct NbRef {
    int x, y;
    bool stale;
};

// Node list and neighbour order of Mesh::NNmodel_TypeXX in global
// coordinates (reference local column i = x + 1).  Neighbours at x = -1 /
// x = nx are the halo columns, which hold the other edge column's moments
// from the previous step (mesh.cpp:493-498 with the periodic ring).
void band_type_nodes(int type, int nx, int ny, std::vector<std::pair<int2, std::vector<NbRef>>>& out)
{
    auto ref = [&](int x, int y) {
        if (x < 0) return NbRef{nx - 1, y, true};
        if (x >= nx) return NbRef{0, y, true};
        return NbRef{x, y, false};
    };
    auto add = [&](int x, int y, std::initializer_list<int2> nb) {
        std::vector<NbRef> v;
        for (auto q : nb) v.push_back(ref(q.x, q.y));
        out.push_back({make_int2(x, y), v});
    };
    switch (type) {
    case 0: add(0, 0, {{0, 1}, {1, 1}, {1, 0}}); break;
    case 2: add(0, ny - 1, {{0, ny - 2}, {1, ny - 2}, {1, ny - 1}}); break;
    case 4: add(nx - 1, ny - 1, {{nx - 2, ny - 1}, {nx - 2, ny - 2}, {nx - 1, ny - 2}}); break;
    case 6: add(nx - 1, 0, {{nx - 1, 1}, {nx - 2, 1}, {nx - 2, 0}}); break;
    case 1:
        for (int y = 1; y < ny - 1; y++) add(0, y, {{0, y + 1}, {1, y + 1}, {1, y}, {1, y - 1}, {0, y - 1}});
        break;
    case 5:
        for (int y = 1; y < ny - 1; y++)
            add(nx - 1, y, {{nx - 1, y + 1}, {nx - 2, y + 1}, {nx - 2, y}, {nx - 2, y - 1}, {nx - 1, y - 1}});
        break;
    case 3:
        for (int x = 0; x < nx; x++) {
            int y = ny - 2;
            add(x, y, {{x + 1, y}, {x + 1, y - 1}, {x, y - 1}, {x - 1, y - 1}, {x - 1, y}});
        }
        break;
    case 7:
        for (int x = 0; x < nx; x++) {
            int y = 1;
            add(x, y, {{x - 1, y}, {x - 1, y + 1}, {x, y + 1}, {x + 1, y + 1}, {x + 1, y}});
        }
        break;
    }
}

bool nets_active(const ippi_lbm* h)
{
    if (h->p.collision != IPPI_BGK || h->p.bc_set != IPPI_BC_REF_NEE) return false;
    for (int t = 0; t < 8; t++)
        if (h->nets[t].loaded) return true;
    return false;
}

// ---------------------------------------------------------------------------
// rebuild of flags, slots, side buffers, band and IB tables
// ---------------------------------------------------------------------------
int rebuild(ippi_lbm* h)
{
    const int nx = h->p.nx, ny = h->p.ny;
    const size_t nn = (size_t)nx * ny;
    drop_graphs(h);
    std::vector<uint8_t> flag(nn, 0);
    std::vector<int> slot(nn, -1);
    auto id = [&](int x, int y) { return (size_t)y * nx + x; };

    // band nodes: the last loaded type covering a node decides (call order
    // 00 01 02 04 05 06 03 07, mesh.cpp:364-379)
    struct BandEntry {
        int type;
        std::vector<NbRef> nb;
    };
    std::map<size_t, BandEntry> band;
    if (nets_active(h)) {
        static const int order[8] = {0, 1, 2, 4, 5, 6, 3, 7};
        for (int oi = 0; oi < 8; oi++) {
            int t = order[oi];
            if (!h->nets[t].loaded) continue;
            std::vector<std::pair<int2, std::vector<NbRef>>> lst;
            band_type_nodes(t, nx, ny, lst);
            for (auto& e : lst) band[id(e.first.x, e.first.y)] = BandEntry{t, e.second};
        }
        for (auto& kv : band) {
            flag[kv.first] |= NF_EXPORT | NF_DEFER;
            for (auto& r : kv.second.nb) flag[id(r.x, r.y)] |= NF_EXPORT;
        }
    }

    // immersed boundary: stencil nodes are exported and deferred
    std::vector<int> fn_of_node;  // node -> forced index
    std::vector<int> st_node;     // [nmark][16] node ids
    std::vector<double> st_wa, st_wb;
    const int nst = h->p.delta_kernel == IPPI_DELTA_PESKIN4 ? 16 : 4;
    const int nm = h->nmark;
    if (nm > 0) {
        st_node.assign((size_t)nm * 16, -1);
        st_wa.assign((size_t)nm * 16, 0.0);
        st_wb.assign((size_t)nm * 16, 0.0);
        for (int m = 0; m < nm; m++) {
            int xs[16], ys[16];
            double wa[16], wb[16];
            int c = marker_stencil(h->p.delta_kernel, h->mk_xy[2 * m], h->mk_xy[2 * m + 1], xs, ys, wa, wb);
            for (int q = 0; q < c; q++) {
                st_node[(size_t)m * 16 + q] = (int)id(xs[q], ys[q]);
                st_wa[(size_t)m * 16 + q] = wa[q];
                st_wb[(size_t)m * 16 + q] = wb[q];
                flag[id(xs[q], ys[q])] |= NF_IB | NF_DEFER;
            }
        }
    }

    // solid nodes and the fluid nodes with a link into one
    std::vector<uint8_t> sflag(nn, 0);
    std::vector<int2> links;
    if (!h->solid.empty()) {
        for (size_t i = 0; i < nn; i++)
            if (h->solid[i]) sflag[i] = NF_SOLID;
        for (int y = 1; y < ny - 1; y++)
            for (int x = 1; x < nx - 1; x++) {
                if (h->solid[id(x, y)]) continue;
                for (int k = 1; k < 9; k++)
                    if (h->solid[id(x + EX(k), y + EY(k))]) {
                        sflag[id(x, y)] = NF_SBND;
                        links.push_back(make_int2((int)id(x, y), k));
                    }
            }
        for (size_t i = 0; i < nn; i++)
            if (sflag[i] && (flag[i] & (NF_IB | NF_EXPORT)))
                return fail(h, IPPI_ERR_ARG, "an IB stencil or boundary-net node touches the solid (node %zu)", i);
    }
    dfree(h->solid_links);
    h->solid_links = nullptr;
    h->nlinks = (int)links.size();
    if (!links.empty()) {
        CK(h, dalloc(&h->solid_links, links.size() * sizeof(int2)));
        CK(h, cudaMemcpy(h->solid_links, links.data(), links.size() * sizeof(int2), cudaMemcpyHostToDevice));
    }

    // slots in row-major order; boundary-net nodes (inputs and band) are
    // prep nodes, IB stencil nodes are computed by the IB kernel itself
    int ns = 0;
    std::vector<PrepNode> prep;
    for (size_t i = 0; i < nn; i++)
        if (flag[i]) {
            slot[i] = ns++;
            if (flag[i] & NF_EXPORT)
                prep.push_back(PrepNode{(int)(i % nx), (int)(i / nx), slot[i], flag[i]});
        }
    h->nslots = ns;

    // the bulk kernel only needs to know which nodes it must skip
    std::vector<uint8_t> defer(nn, 0);
    std::vector<uint8_t> tile((size_t)h->gx * ny, 0);
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            const uint8_t d = (uint8_t)((flag[id(x, y)] & NF_DEFER) | sflag[id(x, y)]);
            if (d) {
                defer[id(x, y)] = d;
                tile[(size_t)y * h->gx + x / kBlockX] = 1;
            }
        }

    // rows holding a flagged tile, in groups of 2^row_shift rows per bit
    h->row_shift = 0;
    while (((ny - 1) >> h->row_shift) >= kRowMaskWords * 32) h->row_shift++;
    std::memset(h->rowmask, 0, sizeof h->rowmask);
    for (int y = 0; y < ny; y++)
        for (int bx = 0; bx < h->gx; bx++)
            if (tile[(size_t)y * h->gx + bx]) {
                const int r = y >> h->row_shift;
                h->rowmask[r >> 5] |= 1u << (r & 31);
            }
    CK(h, cudaMemcpy(h->nflag, defer.data(), nn, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(h->tile, tile.data(), tile.size(), cudaMemcpyHostToDevice));
    dfree(h->prep_d);
    h->prep_d = nullptr;
    h->nprep = (int)prep.size();
    CK(h, dalloc(&h->prep_d, std::max<size_t>(prep.size(), 1) * sizeof(PrepNode)));
    if (!prep.empty())
        CK(h, cudaMemcpy(h->prep_d, prep.data(), prep.size() * sizeof(PrepNode), cudaMemcpyHostToDevice));
    dfree(h->side_f);
    dfree(h->side_m);
    h->side_f = h->side_m = nullptr;
    CK(h, dalloc(&h->side_f, (size_t)std::max(ns, 1) * 9 * h->csize));
    CK(h, dalloc(&h->side_m, (size_t)std::max(ns, 1) * 6 * h->csize));
    {
        // the previous-step moments read by the first steps' nets are the
        // halo's initial rho = 1, u = 0 (mesh.cpp:88-101)
        std::vector<char> init((size_t)std::max(ns, 1) * 6 * h->csize, 0);
        for (int s = 0; s < 2 * std::max(ns, 1); s++) {
            if (h->csize == 8)
                ((double*)init.data())[3 * s] = 1.0;
            else
                ((float*)init.data())[3 * s] = 1.0f;
        }
        CK(h, cudaMemcpy(h->side_m, init.data(), init.size(), cudaMemcpyHostToDevice));
    }

    // band tables
    dfree(h->band_nodes_d);
    dfree(h->band_work_d);
    dfree(h->band_type_d);
    dfree(h->band_in_d);
    h->band_in_d = nullptr;
    h->band_nodes_d = nullptr;
    h->band_work_d = nullptr;
    h->band_type_d = nullptr;
    h->band_blocks = 0;
    if (!band.empty()) {
        std::vector<BandNode> nodes;
        std::vector<int2> work;
        std::vector<int> wtype;
        std::vector<int> in_slot;  // per block, node and neighbour: 2 slot + stale, or -1
        const int nb_blk = band_nodes(h->p.storage);  // band nodes per block of band_kernel
        for (int t = 0; t < 8; t++) {
            int first = (int)nodes.size();
            for (auto& kv : band) {
                if (kv.second.type != t) continue;
                BandNode b{};
                b.x = (int)(kv.first % nx);
                b.y = (int)(kv.first / nx);
                b.slot = slot[kv.first];
                b.nin = (int)kv.second.nb.size() * 3;
                b.nb_stale = 0;
                for (size_t q = 0; q < kv.second.nb.size(); q++) {
                    const NbRef& r = kv.second.nb[q];
                    b.nb_slot[q] = slot[id(r.x, r.y)];
                    if (r.stale) b.nb_stale |= 1 << q;
                }
                nodes.push_back(b);
            }
            for (int s0 = first; s0 < (int)nodes.size(); s0 += nb_blk) {
                work.push_back(make_int2(s0, std::min(nb_blk, (int)nodes.size() - s0)));
                wtype.push_back(t);
                for (int n = 0; n < nb_blk; n++)
                    for (int q = 0; q < 5; q++) {
                        int code = -1;
                        if (s0 + n < (int)nodes.size() && 3 * q < nodes[s0 + n].nin)
                            code = 2 * nodes[s0 + n].nb_slot[q] + ((nodes[s0 + n].nb_stale >> q) & 1);
                        in_slot.push_back(code);
                    }
            }
        }
        h->band_nodes = nodes;
        CK(h, dalloc(&h->band_nodes_d, nodes.size() * sizeof(BandNode)));
        CK(h, dalloc(&h->band_work_d, work.size() * sizeof(int2)));
        CK(h, dalloc(&h->band_type_d, wtype.size() * sizeof(int)));
        CK(h, dalloc(&h->band_in_d, in_slot.size() * sizeof(int)));
        CK(h, cudaMemcpy(h->band_in_d, in_slot.data(), in_slot.size() * sizeof(int), cudaMemcpyHostToDevice));
        CK(h, cudaMemcpy(h->band_nodes_d, nodes.data(), nodes.size() * sizeof(BandNode), cudaMemcpyHostToDevice));
        CK(h, cudaMemcpy(h->band_work_d, work.data(), work.size() * sizeof(int2), cudaMemcpyHostToDevice));
        CK(h, cudaMemcpy(h->band_type_d, wtype.data(), wtype.size() * sizeof(int), cudaMemcpyHostToDevice));
        h->band_blocks = (int)work.size();
        const int st = h->p.storage;
        CK(h, st == IPPI_F64   ? band_setup_f64()
              : st == IPPI_F32 ? band_setup_f32()
              : st == IPPI_F16 ? band_setup_f16()
                               : band_setup_bf16());
    }

    // immersed-boundary tables
    for (auto& b : h->ib_bufs) dfree(b.p);
    h->ib_bufs.clear();
    h->nforced = 0;
    h->ib_active = false;
    if (nm > 0) {
        // markers sorted by body, keeping their order within a body
        std::vector<int> morder(nm);
        for (int m = 0; m < nm; m++) morder[m] = m;
        std::stable_sort(morder.begin(), morder.end(),
                         [&](int a, int b) { return h->mk_body[a] < h->mk_body[b]; });
        const int nb = h->nbody;
        std::vector<int2> body_m(nb, make_int2(0, 0));
        for (int mi = 0; mi < nm; mi++) {
            const int b = h->mk_body[morder[mi]];
            if (mi == 0 || h->mk_body[morder[mi - 1]] != b) body_m[b].x = mi;
            body_m[b].y = mi + 1;
        }
        // forced nodes in first-use order; CSR entries in marker order, the
        // accumulation order of SpreadForce (mesh.cpp:757-781)
        std::vector<int> fnode, fptr(1, 0), fe_marker, st_loc((size_t)nm * 16, 0);
        std::vector<double2> fe_w, st_w((size_t)nm * 16, make_double2(0, 0));
        std::map<int, int> forced_index;
        std::vector<std::vector<std::pair<int, double2>>> entries;
        for (int mi = 0; mi < nm; mi++) {
            const int m = morder[mi];
            for (int q = 0; q < nst; q++) {
                const int nd = st_node[(size_t)m * 16 + q];
                auto it = forced_index.find(nd);
                int fi;
                if (it == forced_index.end()) {
                    fi = (int)fnode.size();
                    forced_index[nd] = fi;
                    fnode.push_back(nd);
                    entries.emplace_back();
                } else {
                    fi = it->second;
                }
                const double2 w = make_double2(st_wa[(size_t)m * 16 + q], st_wb[(size_t)m * 16 + q]);
                entries[fi].push_back({mi, w});
                st_loc[(size_t)mi * 16 + q] = fi;
                st_w[(size_t)mi * 16 + q] = w;
            }
        }
        for (auto& e : entries) {
            for (auto& pr : e) {
                fe_marker.push_back(pr.first);
                fe_w.push_back(pr.second);
            }
            fptr.push_back((int)fe_marker.size());
        }
        const int nf = (int)fnode.size();
        std::vector<int> fn_slot(nf);
        std::vector<int2> fn_xy(nf);
        for (int i = 0; i < nf; i++) {
            fn_slot[i] = slot[fnode[i]];
            fn_xy[i] = make_int2(fnode[i] % nx, fnode[i] / nx);
        }
        std::vector<double2> ub(nm);
        std::vector<double> ds(nm);
        for (int mi = 0; mi < nm; mi++) {
            const int m = morder[mi];
            ub[mi] = make_double2(h->mk_ub[2 * m], h->mk_ub[2 * m + 1]);
            ds[mi] = h->mk_ds[m];
        }
        auto up = [&](const void* src, size_t bytes) -> void* {
            DevBuf b;
            b.bytes = bytes;
            if (dalloc(&b.p, bytes) != cudaSuccess) return nullptr;
            if (src && cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
            if (!src) cudaMemset(b.p, 0, bytes);
            h->ib_bufs.push_back(b);
            return b.p;
        };
        IbArgs& I = h->ib;
        I = IbArgs{};
        I.nmark = nm;
        I.nforced = nf;
        I.nbody = nb;
        I.ub = (const double2*)up(ub.data(), nm * sizeof(double2));
        I.ds = (const double*)up(ds.data(), nm * sizeof(double));
        I.st_node = (const int*)up(st_loc.data(), st_loc.size() * sizeof(int));
        I.st_w = (const double2*)up(st_w.data(), st_w.size() * sizeof(double2));
        I.body_m = (const int2*)up(body_m.data(), body_m.size() * sizeof(int2));
        I.fn_slot = (const int*)up(fn_slot.data(), nf * sizeof(int));
        I.fn_xy = (const int2*)up(fn_xy.data(), nf * sizeof(int2));
        I.fn_ptr = (const int*)up(fptr.data(), fptr.size() * sizeof(int));
        I.fe_marker = (const int*)up(fe_marker.data(), fe_marker.size() * sizeof(int));
        I.fe_w = (const double2*)up(fe_w.data(), fe_w.size() * sizeof(double2));
        I.rho = (double*)up(nullptr, nf * sizeof(double));
        I.ucx = (double*)up(nullptr, nf * sizeof(double));
        I.ucy = (double*)up(nullptr, nf * sizeof(double));
        I.fx = (double*)up(nullptr, nf * sizeof(double));
        I.fy = (double*)up(nullptr, nf * sizeof(double));
        I.dmf = (double2*)up(nullptr, nm * sizeof(double2));
        I.mft = (double2*)up(nullptr, nm * sizeof(double2));
        h->hist_cap = (int)std::max<long long>(16, std::min<long long>(1 << 16, (1ll << 24) / std::max(1, nb)));
        I.force_now = (double*)up(nullptr, (size_t)nb * 2 * sizeof(double));
        I.force_hist = (double*)up(nullptr, (size_t)h->hist_cap * nb * 2 * sizeof(double));
        I.hist_cap = h->hist_cap;
        // IB blocks of the one-launch step: one per kIbNodesPerBlock forced
        // nodes, kIbCtas .. kIbMaxBlocks; the barrier counter restarts at 0,
        // a multiple of every launch's arrivals
        I.nib = (int)std::min<long long>(kIbMaxBlocks, std::max<long long>(kIbCtas, (nf + kIbNodesPerBlock - 1) /
                                                                                      kIbNodesPerBlock));
        CK(h, cudaMemset(h->ib_bar, 0, sizeof(unsigned long long)));
        for (auto& b : h->ib_bufs)
            if (!b.p) return fail(h, IPPI_ERR_NOMEM, "IB table allocation failed");
        h->force_now = I.force_now;
        h->force_hist = I.force_hist;
        h->hist_written = 0;
        h->nforced = nf;
        h->ib_nst = nst;
        h->ib_active = true;
    }
    h->dl_valid = false;
    return IPPI_OK;
}

// ---------------------------------------------------------------------------
// launches
// ---------------------------------------------------------------------------
LaunchSet make_launch(ippi_lbm* h, int mode, const void* fin, void* fout, int par)
{
    LaunchSet L{};
    StepArgs& a = L.step;
    a.f_in = fin;
    a.f_out = fout;
    a.pitch = h->pitch;
    a.plane = h->plane;
    a.nx = h->p.nx;
    a.ny = h->p.ny;
    a.les = h->p.les_model;
    a.mlp = h->mlp_dev;
    a.mlp_frag = h->mlp_tc ? h->mlp_frag : nullptr;
    a.tau_field = h->tau_field;
    a.mac = h->mac;
    a.wall_dist = h->wall_dist;
    std::memcpy(a.rowmask, h->rowmask, sizeof a.rowmask);
    a.row_shift = h->row_shift;
    a.plate_x0 = h->p.plate_x0;
    a.tau0 = h->p.tau0;
    a.cs = h->p.cs;
    a.u_in = h->p.u_in;
    a.rho0 = h->p.rho0;
    a.f_tau0 = (float)h->p.tau0;
    a.f_cs = (float)h->p.cs;
    a.f_u_in = (float)h->p.u_in;
    a.f_rho0 = (float)h->p.rho0;
    a.tile = h->tile;
    a.tiles_x = h->gx;
    a.nflag = h->nflag;
    a.side_f = h->side_f;
    a.side_m = h->side_m;
    a.nslots = h->nslots;
    a.corner = h->corner;
    a.avg = h->avg;
    a.avg_start = h->no_avg ? 0x7fffffff : h->p.avg_start;
    a.ctr = h->ctr;
    a.mode = mode;
    a.par = par;
    a.fixed_t = h->last_t;
    a.init_m = h->init_m;
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    a.dl_f = h->dl;
    a.dl_m = h->dl ? h->dl + 9 * nn : nullptr;
    a.dl_tau = h->dl ? h->dl + 13 * nn : nullptr;
    L.grid = dim3(h->gx, h->p.ny);
    L.coll = h->p.collision;
    L.scene = h->p.bc_set == IPPI_BC_CHANNEL ? SC_CHANNEL : SC_REF;
    L.stream = h->st;
    L.side = h->side;
    L.side_prio = h->side_prio;
    L.fork = h->fork;
    L.join = h->join;
    L.prep = h->prep_d;
    L.nprep = h->nprep;
    L.band = h->band_blocks > 0;
    L.ib = h->ib_active;
    if (L.band) {
        BandArgs& B = L.band_args;
        B.nodes = h->band_nodes_d;
        B.work = h->band_work_d;
        B.work_type = h->band_type_d;
        B.in_slot = h->band_in_d;
        for (int t = 0; t < 8; t++) {
            if (!h->nets[t].loaded) continue;
            char* base = reinterpret_cast<char*>(h->net_dev[t]);
            B.net[t].w16 = reinterpret_cast<const uint16_t*>(base);
            B.net[t].w32 = reinterpret_cast<const float*>(base + (size_t)kBandHalves * 2);
            B.net[t].nin = h->nets[t].nin;
            B.net[t].bo = h->nets[t].w.back();
        }
        B.s = a;
        L.band_blocks = h->band_blocks;
    }
    if (L.ib) {
        L.ib_args = h->ib;
        L.ib_args.bar = h->ib_bar;
        // IPPI_TEST_IB_BARRIER_EXTRA=n (tests only): every IB barrier of the
        // one-launch step waits for n arrivals that never come, runs out
        // after its poll limit and reports the timeout
        static const int bar_extra = [] {
            const char* e = std::getenv("IPPI_TEST_IB_BARRIER_EXTRA");
            return e ? std::max(0, std::atoi(e)) : 0;
        }();
        L.ib_args.bar_extra = bar_extra;
        L.ib_args.s = a;
        L.ib_nst = h->ib_nst;
        L.ib_passes = std::max(1, h->p.mdf_iters);
    }
    return L;
}

// the user step number t of the next step, into the counter entry of its parity
int set_time(ippi_lbm* h, int t)
{
    const int par = h->kcount & 1;
    h->ctr_h->t[par] = t;
    CK(h, cudaMemcpyAsync(&h->ctr->t[par], &h->ctr_h->t[par], sizeof(int), cudaMemcpyHostToDevice, h->st));
    return IPPI_OK;
}

// every launch computes relaxation times: the learned model needs its network
int tau_ready(ippi_lbm* h)
{
    if (h->p.les_model == IPPI_LES_LEARNED && !h->mlp_dev)
        return fail(h, IPPI_ERR_STATE, "learned tau selected but no network loaded (ippi_load_tau_mlp)");
    if (h->p.les_model == IPPI_LES_FIELD && !h->tau_field)
        return fail(h, IPPI_ERR_STATE, "tau field selected but none set (ippi_set_tau_field)");
    if (h->p.les_model == IPPI_LES_DYNAMIC && !h->wall_dist)
        return fail(h, IPPI_ERR_STATE, "wall-damped closure selected but no wall distance set (ippi_set_wall_distance)");
    return IPPI_OK;
}

// the first collision, from the equilibrium of the initial moments (k = 0)
int run_init(ippi_lbm* h)
{
    if (int rc = tau_ready(h)) return rc;
    Range range("ippi initial collision");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    std::memset(h->ctr_h, 0, sizeof(Ctr));
    CK(h, cudaMemcpyAsync(h->ctr, h->ctr_h, sizeof(Ctr), cudaMemcpyHostToDevice, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    LaunchSet L = make_launch(h, MODE_INIT, nullptr, h->f[0], 0);
    CK(h, launch(L, h->S));
    h->cur = 0;
    h->kcount = 1;
    h->last_t = 0;
    h->pending_init = false;
    h->dl_valid = false;
    return IPPI_OK;
}

// n (1 or 2) steps starting from buffer b with parity q, with or without
// the running means (av), as one CUDA graph
int build_graph(ippi_lbm* h, int n, int b, int q, int av)
{
    cudaGraph_t g;
    cudaGraphExec_t& slot = n == 2 ? h->graph[b][q][av] : h->graph1[b][q][av];
    CK(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    LaunchSet L0 = make_launch(h, MODE_STEP, h->f[b], h->f[b ^ 1], q);
    L0.avg_on = av;
    cudaError_t e0 = launch(L0, h->S), e1 = cudaSuccess;
    if (n == 2) {
        LaunchSet L1 = make_launch(h, MODE_STEP, h->f[b ^ 1], h->f[b], q ^ 1);
        L1.avg_on = av;
        e1 = launch(L1, h->S);
    }
    cudaError_t ec = cudaStreamEndCapture(h->st, &g);
    if (e0 != cudaSuccess || e1 != cudaSuccess || ec != cudaSuccess)
        return fail(h, IPPI_ERR_CUDA, "graph capture failed: %s",
                    cudaGetErrorString(e0 ? e0 : (e1 ? e1 : ec)));
    cudaError_t ei = cudaGraphInstantiate(&slot, g, 0);
    cudaGraphDestroy(g);
    CK(h, ei);
    return IPPI_OK;
}

// post-stream state of the last step (populations, moments, next tau) into
// the download buffers: the last step re-run from its input field with its
// outputs redirected (nothing of the state changes)
int materialize(ippi_lbm* h)
{
    if (h->dl_valid) return IPPI_OK;
    if (int rc = tau_ready(h)) return rc;
    Range range("ippi materialize (download pass)");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    if (!h->dl) CK(h, dalloc(&h->dl, 14 * nn * sizeof(double)));
    CK(h, cudaMemsetAsync(h->dl + 12 * nn, 0, nn * sizeof(double), h->st));  // net-flag plane
    LaunchSet L;
    if (h->pending_init) {
        h->last_t = 0;
        L = make_launch(h, MODE_MAT_INIT, nullptr, nullptr, 0);
    } else {
        L = make_launch(h, MODE_MAT, h->f[h->cur ^ 1], nullptr, (h->kcount - 1) & 1);
    }
    CK(h, launch(L, h->S));
    CK(h, cudaStreamSynchronize(h->st));
    h->dl_valid = true;
    return IPPI_OK;
}

// ---------------------------------------------------------------------------
// checkpoint layout: a fixed header, then the device sections in this order
// ---------------------------------------------------------------------------
constexpr char kCkpMagic[8] = {'I', 'P', 'P', 'I', 'C', 'K', 'P', '1'};

struct CkpHeader {
    char magic[8];
    uint32_t abi, header_bytes;
    uint64_t config_hash;
    int32_t nx, ny, storage, nbody, hist_cap, cur;
    int64_t kcount, last_t, hist_written;
    uint64_t f_bytes, avg_bytes, corner_bytes, force_bytes, hist_bytes;
    double mass;            // FP64 mass of the state (ippi_forces), re-checked on load
    uint64_t payload_hash;  // ckp_hash of everything after the header
};

struct CkpLayout {
    size_t f, avg, corner, force, hist, total;
};

struct CkpSection {
    void* dev;
    size_t bytes;
};

CkpLayout ckp_layout(const ippi_lbm* h)
{
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    CkpLayout L;
    L.f = (size_t)9 * h->plane * h->tsize;
    L.avg = 3 * nn * h->csize;
    L.corner = 24 * (size_t)h->csize;
    L.force = h->force_now ? (size_t)h->nbody * 2 * sizeof(double) : 0;
    L.hist = h->force_hist ? (size_t)h->hist_cap * h->nbody * 2 * sizeof(double) : 0;
    L.total = sizeof(CkpHeader) + 2 * L.f + L.avg + L.corner + L.force + L.hist;
    return L;
}

std::vector<CkpSection> ckp_sections(ippi_lbm* h, const CkpLayout& L)
{
    return {{h->f[0], L.f},         {h->f[1], L.f},          {h->avg, L.avg},
            {h->corner, L.corner}, {h->force_now, L.force}, {h->force_hist, L.hist}};
}

// FNV-1a over 64-bit words (bytes for the tail), each step followed by a
// right xor-shift so that high bits reach the low ones
uint64_t ckp_hash(const unsigned char* p, size_t n, uint64_t x = 0xcbf29ce484222325ull)
{
    constexpr uint64_t prime = 0x100000001b3ull;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        x = (x ^ w) * prime;
        x ^= x >> 29;
    }
    for (; i < n; i++) x = (x ^ p[i]) * prime;
    return x;
}

// what the saved state presumes of the handle: parameters (not the device),
// markers, solid mask, and what sets the relaxation times -- the tau field,
// the learned network, the wall distance and the boundary nets
uint64_t ckp_config_hash(const ippi_lbm* h)
{
    const ippi_params& p = h->p;
    uint64_t x = 0xcbf29ce484222325ull;
    auto put = [&](const void* v, size_t n) { x = ckp_hash(static_cast<const unsigned char*>(v), n, x); };
    const int32_t ints[] = {p.nx, p.ny, p.collision, p.storage, p.bc_set, p.les_model,
                            p.plate_x0, p.avg_start, p.delta_kernel, p.mdf_iters, h->nbody, h->hist_cap};
    const double dbl[] = {p.tau0, p.cs, p.u_in, p.rho0};
    put(ints, sizeof ints);
    put(dbl, sizeof dbl);
    put(h->mk_xy.data(), h->mk_xy.size() * sizeof(double));
    put(h->mk_ub.data(), h->mk_ub.size() * sizeof(double));
    put(h->mk_ds.data(), h->mk_ds.size() * sizeof(double));
    put(h->mk_body.data(), h->mk_body.size() * sizeof(int));
    put(h->solid.data(), h->solid.size());
    const uint64_t tau_inputs[] = {h->tau_field_hash, h->mlp_hash, h->wall_hash};
    put(tau_inputs, sizeof tau_inputs);
    for (int t = 0; t < 8; t++) {
        if (!h->nets[t].loaded) continue;
        put(&t, sizeof t);
        put(h->nets[t].w.data(), h->nets[t].w.size() * sizeof(float));
    }
    return x;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int ippi_abi_version(void) { return IPPI_ABI_VERSION; }

void ippi_params_default(ippi_params* p, int nx, int ny)
{
    std::memset(p, 0, sizeof *p);
    p->nx = nx;
    p->ny = ny;
    p->collision = IPPI_BGK;
    p->storage = IPPI_F64;
    p->bc_set = IPPI_BC_REF_NEE;
    p->les_model = IPPI_LES_SMAGORINSKY;
    p->tau0 = 0.5 + 6.0 * ((ny * 0.1) / 5e5);  // main.cpp:38-43
    p->cs = 0.173;
    p->u_in = 0.1;
    p->rho0 = 1.0;
    p->plate_x0 = 400;
    p->avg_start = 30000;
    p->delta_kernel = IPPI_DELTA_BILINEAR;
    p->mdf_iters = 1;
    p->device = 0;
}

int ippi_create(const ippi_params* p, ippi_lbm** out)
{
    if (!p || !out) return fail(nullptr, IPPI_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->nx < 4 || p->ny < 4) return fail(nullptr, IPPI_ERR_ARG, "lattice must be at least 4 x 4");
    if (9ll * (((long long)p->nx + 63) / 64 * 64) * p->ny >= (1ll << 31))
        return fail(nullptr, IPPI_ERR_ARG, "lattice too large for 32-bit population offsets");
    if (p->collision < 0 || p->collision > 2) return fail(nullptr, IPPI_ERR_ARG, "bad collision");
    if (p->storage < 0 || p->storage > 3) return fail(nullptr, IPPI_ERR_ARG, "bad storage");
    if (p->bc_set < 0 || p->bc_set > 1) return fail(nullptr, IPPI_ERR_ARG, "bad bc_set");
    if (p->les_model < 0 || p->les_model > 6) return fail(nullptr, IPPI_ERR_ARG, "bad les_model");
    if (p->les_model == IPPI_LES_LEARNED && p->bc_set != IPPI_BC_CHANNEL)
        return fail(nullptr, IPPI_ERR_ARG, "the learned relaxation time is built for the channel scene");
    if (p->les_model >= IPPI_LES_FIELD && p->bc_set != IPPI_BC_CHANNEL)
        return fail(nullptr, IPPI_ERR_ARG,
                    "the tau field and the WALE, coherent and wall-damped closures are built for the channel scene");
    if (p->delta_kernel < 0 || p->delta_kernel > 1) return fail(nullptr, IPPI_ERR_ARG, "bad delta_kernel");
    if (!(p->tau0 > 0.5)) return fail(nullptr, IPPI_ERR_ARG, "tau0 must exceed 0.5");
    if (!(p->rho0 > 0)) return fail(nullptr, IPPI_ERR_ARG, "rho0 must be positive");
    if (p->bc_set == IPPI_BC_CHANNEL && !(std::fabs(p->u_in) < 0.5))
        return fail(nullptr, IPPI_ERR_ARG, "channel inlet velocity must be below 0.5");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, IPPI_ERR_CUDA, "no CUDA device available");
    if (p->device < 0 || p->device >= ndev) return fail(nullptr, IPPI_ERR_ARG, "bad device ordinal");

    ippi_lbm* h = new ippi_lbm();
    h->p = *p;
    if (h->p.mdf_iters < 1) h->p.mdf_iters = 1;
    h->S = p->storage;
    h->csize = p->storage == IPPI_F64 ? 8 : 4;
    h->tsize = p->storage == IPPI_F64 ? 8 : (p->storage == IPPI_F32 ? 4 : 2);
    const int nx = p->nx, ny = p->ny;
    const size_t nn = (size_t)nx * ny;
    h->pitch = ((long long)nx + 63) / 64 * 64;
    h->plane = h->pitch * ny;
    h->gx = (nx + kBlockX - 1) / kBlockX;
    int rc = IPPI_OK;
    auto bail = [&](int code) {
        ippi_destroy(h);
        return code;
    };
    if (cudaSetDevice(p->device) != cudaSuccess) return bail(fail(nullptr, IPPI_ERR_CUDA, "cudaSetDevice failed"));
    int lo_prio = 0, hi_prio = 0;
    cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    // the side stream (a handful of small blocks) outranks the bulk kernel so
    // its blocks are scheduled as soon as an SM has room
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, hi_prio) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(nullptr, IPPI_ERR_CUDA, "stream creation failed"));
    h->side_prio = hi_prio;
    const size_t fbytes = (size_t)9 * h->plane * h->tsize;
    for (int b = 0; b < 2; b++)
        if (dalloc(&h->f[b], fbytes) != cudaSuccess || cudaMemset(h->f[b], 0, fbytes) != cudaSuccess)
            return bail(fail(nullptr, IPPI_ERR_NOMEM, "population buffers (%zu bytes each)", fbytes));
    if (dalloc(&h->ctr, sizeof(Ctr)) != cudaSuccess || cudaMallocHost(&h->ctr_h, sizeof(Ctr)) != cudaSuccess ||
        dalloc(&h->nflag, nn) != cudaSuccess ||
        dalloc(&h->tile, (size_t)h->gx * ny) != cudaSuccess ||
        dalloc(&h->corner, 24 * (size_t)h->csize) != cudaSuccess ||
        dalloc(&h->avg, 3 * nn * h->csize) != cudaSuccess ||
        dalloc(&h->init_m, 3 * nn * sizeof(double)) != cudaSuccess ||
        dalloc(&h->red, 4096 * sizeof(double)) != cudaSuccess)
        return bail(fail(nullptr, IPPI_ERR_NOMEM, "device allocation failed"));
    if (dalloc(&h->ib_bar, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(h->ib_bar, 0, sizeof(unsigned long long)) != cudaSuccess)
        return bail(fail(nullptr, IPPI_ERR_NOMEM, "device allocation failed"));
    if ((p->les_model == IPPI_LES_WALE || p->les_model == IPPI_LES_CSM) &&
        (dalloc(&h->mac, 2 * nn * h->csize) != cudaSuccess || cudaMemset(h->mac, 0, 2 * nn * h->csize) != cudaSuccess))
        return bail(fail(nullptr, IPPI_ERR_NOMEM, "velocity field for the gradient closures"));
    cudaMemset(h->ctr, 0, sizeof(Ctr));
    cudaMemset(h->corner, 0, 24 * (size_t)h->csize);
    rc = rebuild(h);
    if (rc != IPPI_OK) return bail(rc);
    rc = ippi_init_macros(h, nullptr, nullptr, nullptr);
    if (rc != IPPI_OK) return bail(rc);
    *out = h;
    return IPPI_OK;
}

int ippi_destroy(ippi_lbm* h)
{
    if (!h) return IPPI_OK;
    if (h->st) cudaStreamSynchronize(h->st);
    drop_graphs(h);
    adjoint_free(h);
    for (int b = 0; b < 2; b++) dfree(h->f[b]);
    dfree(h->mlp_dev);
    dfree(h->mlp_frag);
    dfree(h->tau_field);
    dfree(h->mac);
    dfree(h->wall_dist);
    dfree(h->ib_bar);
    dfree(h->solid_links);
    dfree(h->solid_out);
    dfree(h->ctr);
    if (h->ctr_h) cudaFreeHost(h->ctr_h);
    dfree(h->nflag);
    dfree(h->prep_d);
    dfree(h->tile);
    dfree(h->side_f);
    dfree(h->side_m);
    dfree(h->corner);
    dfree(h->avg);
    dfree(h->init_m);
    dfree(h->io32);
    dfree(h->dl);
    dfree(h->dl_flags);
    dfree(h->red);
    for (int t = 0; t < 8; t++) dfree(h->net_dev[t]);
    dfree(h->band_nodes_d);
    dfree(h->band_work_d);
    dfree(h->band_type_d);
    dfree(h->band_in_d);
    for (auto& b : h->ib_bufs) dfree(b.p);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return IPPI_OK;
}

namespace {
int init_macros(ippi_lbm* h, const double* rho, const double* ux, const double* uy, bool keep_means);
int init_macros_f32(ippi_lbm* h, const float* rho, const float* ux, const float* uy);
}

int ippi_init_macros_f32(ippi_lbm* h, const float* rho, const float* ux, const float* uy)
{
    return init_macros_f32(h, rho, ux, uy);
}

int ippi_init_macros(ippi_lbm* h, const double* rho, const double* ux, const double* uy)
{
    return init_macros(h, rho, ux, uy, false);
}

int ippi_reequilibrate(ippi_lbm* h, const double* rho, const double* ux, const double* uy)
{
    if (h && h->pending_init) return fail(h, IPPI_ERR_STATE, "no step taken yet (use ippi_init_macros)");
    return init_macros(h, rho, ux, uy, true);
}

namespace {
// Defaults for the fields the caller did not give, the validity check and
// the pending initial collision, once the given fields are in init_m.
int init_macros_finish(ippi_lbm* h, bool has_rho, bool has_ux, bool has_uy, bool keep_means)
{
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(h->red);
    CK(h, cudaMemsetAsync(bad, 0xff, sizeof *bad, h->st));
    init_fields_kernel<<<std::min<size_t>((nn + 255) / 256, 4096), 256, 0, h->st>>>(
        h->init_m, (long long)nn, has_rho, has_ux, has_uy, bad);
    CK(h, cudaGetLastError());
    if (!keep_means) CK(h, cudaMemsetAsync(h->avg, 0, 3 * nn * h->csize, h->st));
    unsigned long long first_bad = 0;
    CK(h, cudaMemcpyAsync(&first_bad, bad, sizeof first_bad, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    if (first_bad != ~0ull)
        return fail(h, IPPI_ERR_ARG, "initial rho must be positive and u finite (node %llu)", first_bad);
    // the step graphs read the initial fields only through MODE_INIT, which
    // is launched outside them: they stay valid
    h->pending_init = true;
    h->dl_valid = false;
    if (!keep_means) h->hist_written = 0;
    return IPPI_OK;
}

int init_macros(ippi_lbm* h, const double* rho, const double* ux, const double* uy, bool keep_means)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    CK(h, cudaSetDevice(h->p.device));
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    if (!h->init_m) CK(h, dalloc(&h->init_m, 3 * nn * sizeof(double)));
    // host fields straight into the device table (fast from pinned memory),
    // defaults and the validity check on the device
    const double* src[3] = {rho, ux, uy};
    for (int q = 0; q < 3; q++)
        if (src[q])
            CK(h, cudaMemcpyAsync(h->init_m + q * nn, src[q], nn * sizeof(double),
                                  cudaMemcpyHostToDevice, h->st));
    return init_macros_finish(h, rho != nullptr, ux != nullptr, uy != nullptr, keep_means);
}

int init_macros_f32(ippi_lbm* h, const float* rho, const float* ux, const float* uy)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    CK(h, cudaSetDevice(h->p.device));
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    if (!h->init_m) CK(h, dalloc(&h->init_m, 3 * nn * sizeof(double)));
    if (!h->io32) CK(h, dalloc(&h->io32, 9 * nn * sizeof(float)));
    // FP32 host fields into the staging planes, widened on the device
    const float* src[3] = {rho, ux, uy};
    for (int q = 0; q < 3; q++)
        if (src[q]) {
            CK(h, cudaMemcpyAsync(h->io32 + q * nn, src[q], nn * sizeof(float), cudaMemcpyHostToDevice,
                                  h->st));
            convert_kernel<float, double><<<convert_blocks(nn), 256, 0, h->st>>>(
                h->io32 + q * nn, h->init_m + q * nn, (long long)nn);
            CK(h, cudaGetLastError());
        }
    return init_macros_finish(h, rho != nullptr, ux != nullptr, uy != nullptr, false);
}
}  // namespace

int ippi_set_markers(ippi_lbm* h, int n, const double* xy, const double* ub, const int* body,
                     const double* ds)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (n < 0 || (n > 0 && !xy)) return fail(h, IPPI_ERR_ARG, "bad marker arrays");
    const int nst = h->p.delta_kernel == IPPI_DELTA_PESKIN4 ? 16 : 4;
    int nbody = 0;
    for (int m = 0; m < n; m++) {
        const double mx = xy[2 * m], my = xy[2 * m + 1];
        if (!(mx >= 0 && mx < h->p.nx && my >= 0 && my < h->p.ny))
            return fail(h, IPPI_ERR_ARG, "marker %d outside the lattice", m);
        int xs[16], ys[16];
        double wa[16], wb[16];
        int c = marker_stencil(h->p.delta_kernel, mx, my, xs, ys, wa, wb);
        for (int q = 0; q < c; q++)
            if (xs[q] < 3 || xs[q] > h->p.nx - 4 || ys[q] < 3 || ys[q] > h->p.ny - 4)
                return fail(h, IPPI_ERR_ARG, "marker %d stencil is closer than 3 nodes to the edge", m);
        const int b = body ? body[m] : 0;
        if (b < 0) return fail(h, IPPI_ERR_ARG, "negative body id");
        nbody = std::max(nbody, b + 1);
        (void)nst;
    }
    const int keep_n = h->nmark, keep_nb = h->nbody;
    std::vector<double> keep_xy = h->mk_xy, keep_ub = h->mk_ub, keep_ds = h->mk_ds;
    std::vector<int> keep_body = h->mk_body;
    h->nmark = n;
    h->nbody = n > 0 ? nbody : 0;
    h->mk_xy.assign(xy, xy + 2 * (size_t)n);
    h->mk_ub.assign(2 * (size_t)n, 0.0);
    if (ub) h->mk_ub.assign(ub, ub + 2 * (size_t)n);
    h->mk_ds.assign(n, 1.0);
    if (ds) h->mk_ds.assign(ds, ds + n);
    h->mk_body.assign(n, 0);
    if (body) h->mk_body.assign(body, body + n);
    CK(h, cudaStreamSynchronize(h->st));
    int rc = rebuild(h);
    if (rc) {
        // rejected (a stencil on a solid): keep the previous markers
        h->nmark = keep_n;
        h->nbody = keep_nb;
        h->mk_xy = keep_xy;
        h->mk_ub = keep_ub;
        h->mk_ds = keep_ds;
        h->mk_body = keep_body;
        rebuild(h);
    }
    return rc;
}

int ippi_load_band_net(ippi_lbm* h, int type, const float* w, size_t n)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (type < 0 || type > 7 || !w) return fail(h, IPPI_ERR_ARG, "bad net type");
    const int nin = (type % 2 == 0) ? 9 : 15;
    const size_t need = (size_t)kHidden * nin + kHidden + 6 * (kHidden * kHidden + kHidden) + kHidden + 1;
    if (n != need) return fail(h, IPPI_ERR_ARG, "net %d expects %zu floats, got %zu", type, need, n);
    NetHost& net = h->nets[type];
    net.loaded = true;
    net.nin = nin;
    net.w.assign(w, w + n);
    // device layout (band_kernel's tensor-core operands): every weight
    // matrix as two FP16 planes hi = fp16(W), lo = fp16((W - hi) 2^11)
    // (round to nearest even), each in the instruction's K-major no-swizzle
    // A layout (band_w_index):
    //   layer 1 hi, lo [128 x 16, inputs beyond nin zero];
    //   layers 2..7 hi, lo [128 x 128] each;
    // then FP32 b1[128], bh[6][128], wo[128]
    auto planes = [](uint16_t* hi, uint16_t* lo, const float* W, int nin_, int kpad) {
        for (int m = 0; m < kHidden; m++)
            for (int k = 0; k < kpad; k++) {
                const float x = k < nin_ ? W[(size_t)m * nin_ + k] : 0.f;
                const __half xh = __float2half_rn(x);
                const __half xl = __float2half_rn((x - __half2float(xh)) * kBandLoScale);
                std::memcpy(&hi[band_w_index(m, k)], &xh, 2);
                std::memcpy(&lo[band_w_index(m, k)], &xl, 2);
            }
    };
    const float* p = w;
    std::vector<uint16_t> d16((size_t)kBandHalves, 0);
    std::vector<float> d32((size_t)kBandF32, 0.f);
    planes(d16.data(), d16.data() + kBandL1Plane, p, nin, kBandIn);
    p += kHidden * nin;
    for (int j = 0; j < kHidden; j++) d32[kBandF32B1 + j] = p[j];
    p += kHidden;
    for (int l = 0; l < 6; l++) {
        const float* W = p + (size_t)l * (kHidden * kHidden + kHidden);
        uint16_t* hi = d16.data() + kBandOffHid + (size_t)l * 2 * kBandLayerPlane;
        planes(hi, hi + kBandLayerPlane, W, kHidden, kHidden);
        for (int j = 0; j < kHidden; j++) d32[kBandF32Bh + l * kHidden + j] = W[kHidden * kHidden + j];
    }
    p += 6 * (size_t)(kHidden * kHidden + kHidden);
    for (int j = 0; j < kHidden; j++) d32[kBandF32Wo + j] = p[j];
    std::vector<char> d(d16.size() * 2 + d32.size() * 4);
    std::memcpy(d.data(), d16.data(), d16.size() * 2);
    std::memcpy(d.data() + d16.size() * 2, d32.data(), d32.size() * 4);
    CK(h, cudaStreamSynchronize(h->st));
    dfree(h->net_dev[type]);
    h->net_dev[type] = nullptr;
    CK(h, dalloc(&h->net_dev[type], d.size()));
    CK(h, cudaMemcpy(h->net_dev[type], d.data(), d.size(), cudaMemcpyHostToDevice));
    return rebuild(h);
}

namespace {
// Queue nsteps steps numbered t0.. on the handle's stream (graph launches
// only; nothing waits).  The caller holds the network lock.
int enqueue_steps(ippi_lbm* h, int nsteps, int t0)
{
    if (h->pending_init) {
        int rc = run_init(h);
        if (rc) return rc;
    }
    int rc = set_time(h, t0);
    if (rc) return rc;
    // two steps per graph, one where the averaging starts between them and
    // for an odd last step (a driver calling once per step)
    const long long avs = h->no_avg ? 0x7fffffffll : (long long)h->p.avg_start;
    for (int done = 0; done < nsteps;) {
        const long long t = (long long)t0 + done;
        const int q = (int)((h->kcount + done) & 1);
        const int av = t >= avs;
        const int n = (nsteps - done >= 2 && (av || t + 1 < avs)) ? 2 : 1;
        cudaGraphExec_t& g = n == 2 ? h->graph[h->cur][q][av] : h->graph1[h->cur][q][av];
        if (!g) {
            rc = build_graph(h, n, h->cur, q, av);
            if (rc) return rc;
        }
        CK(h, cudaGraphLaunch(g, h->st));
        if (n == 1) h->cur ^= 1;
        done += n;
    }
    h->kcount += nsteps;
    h->last_t = t0 + nsteps - 1;
    h->hist_written += nsteps;
    h->dl_valid = false;
    return IPPI_OK;
}

// Drain the stream after queued steps and report their status word.
int finish_steps(ippi_lbm* h)
{
    CK(h, cudaMemcpyAsync(h->ctr_h, h->ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    if (h->ctr_h->err == 2)
        return fail(h, IPPI_ERR_CUDA, "an immersed-boundary barrier timed out (blocks not co-resident)");
    if (h->ctr_h->err == 3)
        return fail(h, IPPI_ERR_CUDA, "a boundary-net weight copy did not complete in time");
    if (h->ctr_h->err)
        return fail(h, IPPI_ERR_DIVERGED, "Simulation Error! rho left [0,10] at step %d", h->ctr_h->err_t);
    return IPPI_OK;
}

// Holds the stream for about `ns` nanoseconds of %globaltimer (at most 2^22
// polls), so that work queued behind it starts back to back.
__global__ void hold_kernel(long long ns)
{
    long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (int i = 0; i < (1 << 22); i++) {
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 >= ns) break;
        __nanosleep(1000);
    }
}
}  // namespace

int ippi_step(ippi_lbm* h, int nsteps, int t0)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (int rc = tau_ready(h)) return rc;
    if (nsteps < 0) return fail(h, IPPI_ERR_ARG, "negative step count");
    if (nsteps == 0) return IPPI_OK;
    CK(h, cudaSetDevice(h->p.device));
    Range range("ippi_step");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    if (int rc = enqueue_steps(h, nsteps, t0)) return rc;
    return finish_steps(h);
}

int ippi_step_timed(ippi_lbm* h, int nsteps, int t0, double* ms)
{
    if (!h || !ms) return fail(h, IPPI_ERR_ARG, "null argument");
    if (int rc = tau_ready(h)) return rc;
    if (nsteps <= 0) return fail(h, IPPI_ERR_ARG, "nsteps must be positive");
    CK(h, cudaSetDevice(h->p.device));
    Range range("ippi_step_timed");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    if (h->pending_init) {
        // the initial collision is not part of the timed steps
        if (int rc = run_init(h)) return rc;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(h, cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        CK(h, ce);
    }
    hold_kernel<<<1, 1, 0, h->st>>>(500000);
    int rc = IPPI_OK;
    ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaEventRecord(e0, h->st);
    if (ce == cudaSuccess) rc = enqueue_steps(h, nsteps, t0);
    if (ce == cudaSuccess && rc == IPPI_OK) ce = cudaEventRecord(e1, h->st);
    if (ce != cudaSuccess) rc = fail(h, IPPI_ERR_CUDA, "timed step: %s", cudaGetErrorString(ce));
    const int rf = finish_steps(h);
    if (rc == IPPI_OK) rc = rf;
    if (rc == IPPI_OK) {
        float f = 0.f;
        ce = cudaEventElapsedTime(&f, e0, e1);
        if (ce != cudaSuccess) rc = fail(h, IPPI_ERR_CUDA, "timed step: %s", cudaGetErrorString(ce));
        *ms = f;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int ippi_profile_steps(ippi_lbm* h, int nsteps, int t0, double* ms_bulk, double* ms_band, double* ms_ib)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (int rc = tau_ready(h)) return rc;
    if (nsteps <= 0) return fail(h, IPPI_ERR_ARG, "nsteps must be positive");
    CK(h, cudaSetDevice(h->p.device));
    Range range("ippi_profile_steps");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    if (h->pending_init) {
        int rc = run_init(h);
        if (rc) return rc;
    }
    int rc = set_time(h, t0);
    if (rc) return rc;
    std::vector<cudaEvent_t> ev((size_t)nsteps * 4);
    for (auto& e : ev) CK(h, cudaEventCreate(&e));
    for (int s = 0; s < nsteps; s++) {
        LaunchSet L = make_launch(h, MODE_STEP, h->f[h->cur], h->f[h->cur ^ 1], (h->kcount + s) & 1);
        L.avg_on = (long long)t0 + s >= (long long)L.step.avg_start;
        L.events = &ev[(size_t)s * 4];
        CK(h, launch(L, h->S));
        h->cur ^= 1;
    }
    CK(h, cudaStreamSynchronize(h->st));
    CK(h, cudaStreamSynchronize(h->side));
    // bulk kernel: events 0-1 on the main stream; side chain (prep + nets /
    // IB), concurrent with it: events 2-3 on the side stream
    double tb = 0, tn = 0, ti = 0;
    const bool band = h->band_blocks > 0, ib = h->ib_active;
    const bool side = h->nprep > 0 || band || ib;
    for (int s = 0; s < nsteps; s++) {
        float ms;
        cudaEventElapsedTime(&ms, ev[s * 4 + 0], ev[s * 4 + 1]);
        tb += ms;
        if (side) {
            cudaEventElapsedTime(&ms, ev[s * 4 + 2], ev[s * 4 + 3]);
            if (band) tn += ms;
            if (ib) ti += ms;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    h->kcount += nsteps;
    h->last_t = t0 + nsteps - 1;
    h->hist_written += nsteps;
    h->dl_valid = false;
    if (ms_bulk) *ms_bulk = tb / nsteps;
    if (ms_band) *ms_band = tn / nsteps;
    if (ms_ib) *ms_ib = ti / nsteps;
    CK(h, cudaMemcpy(h->ctr_h, h->ctr, sizeof(Ctr), cudaMemcpyDeviceToHost));
    if (h->ctr_h->err == 2)
        return fail(h, IPPI_ERR_CUDA, "an immersed-boundary barrier timed out (blocks not co-resident)");
    if (h->ctr_h->err == 3)
        return fail(h, IPPI_ERR_CUDA, "a boundary-net weight copy did not complete in time");
    if (h->ctr_h->err)
        return fail(h, IPPI_ERR_DIVERGED, "Simulation Error! rho left [0,10] at step %d", h->ctr_h->err_t);
    return IPPI_OK;
}

int ippi_download(ippi_lbm* h, int field, void* host, size_t bytes)
{
    if (!h || !host) return fail(h, IPPI_ERR_ARG, "null argument");
    CK(h, cudaSetDevice(h->p.device));
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    size_t need = field == IPPI_FIELD_F ? 9 * nn * sizeof(double)
                                        : (field == IPPI_FIELD_FLAGS ? nn : nn * sizeof(double));
    if (field < 0 || field > 9) return fail(h, IPPI_ERR_ARG, "bad field %d", field);
    if (bytes != need) return fail(h, IPPI_ERR_ARG, "field %d needs %zu bytes, got %zu", field, need, bytes);
    switch (field) {
    case IPPI_FIELD_FLAGS: {
        if (!h->dl_flags) CK(h, dalloc(&h->dl_flags, nn));
        style_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, h->st>>>(
            h->dl_flags, h->p.nx, h->p.ny, h->p.plate_x0,
            h->p.bc_set == IPPI_BC_CHANNEL ? SC_CHANNEL : SC_REF, h->nflag);
        CK(h, cudaGetLastError());
        CK(h, cudaMemcpyAsync(host, h->dl_flags, nn, cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
        return IPPI_OK;
    }
    case IPPI_FIELD_AVG_U:
    case IPPI_FIELD_AVG_V:
    case IPPI_FIELD_AVG_RHO: {
        const size_t off = (size_t)(field - IPPI_FIELD_AVG_U) * nn;
        if (h->csize == 8) {
            CK(h, cudaMemcpyAsync(host, (double*)h->avg + off, nn * 8, cudaMemcpyDeviceToHost, h->st));
        } else {
            if (!h->dl) CK(h, dalloc(&h->dl, 14 * nn * sizeof(double)));
            h->dl_valid = false;
            to_double_kernel<float><<<(unsigned)((nn + 255) / 256), 256, 0, h->st>>>((const float*)h->avg + off,
                                                                                      h->dl, (long long)nn);
            CK(h, cudaGetLastError());
            CK(h, cudaMemcpyAsync(host, h->dl, nn * 8, cudaMemcpyDeviceToHost, h->st));
        }
        CK(h, cudaStreamSynchronize(h->st));
        return IPPI_OK;
    }
    default: break;
    }
    int rc = materialize(h);
    if (rc) return rc;
    const double* src;
    switch (field) {
    case IPPI_FIELD_F: src = h->dl; break;
    case IPPI_FIELD_RHO: src = h->dl + 9 * nn; break;
    case IPPI_FIELD_UX: src = h->dl + 10 * nn; break;
    case IPPI_FIELD_UY: src = h->dl + 11 * nn; break;
    case IPPI_FIELD_NNFLAG: src = h->dl + 12 * nn; break;
    default: src = h->dl + 13 * nn; break;  // TAU
    }
    CK(h, cudaMemcpy(host, src, need, cudaMemcpyDeviceToHost));
    return IPPI_OK;
}

int ippi_download_f32(ippi_lbm* h, int field, float* host, size_t bytes)
{
    if (!h || !host) return fail(h, IPPI_ERR_ARG, "null argument");
    CK(h, cudaSetDevice(h->p.device));
    if (field < 0 || field > 9 || field == IPPI_FIELD_FLAGS)
        return fail(h, IPPI_ERR_ARG, "bad field %d for an FP32 download", field);
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    const size_t n = field == IPPI_FIELD_F ? 9 * nn : nn;
    if (bytes != n * sizeof(float))
        return fail(h, IPPI_ERR_ARG, "field %d needs %zu bytes, got %zu", field, n * sizeof(float), bytes);
    if (!h->io32) CK(h, dalloc(&h->io32, 9 * nn * sizeof(float)));
    const float* src = h->io32;
    if (field >= IPPI_FIELD_AVG_U && field <= IPPI_FIELD_AVG_RHO) {
        const size_t off = (size_t)(field - IPPI_FIELD_AVG_U) * nn;
        if (h->csize == 4) {
            src = (const float*)h->avg + off;
        } else {
            convert_kernel<double, float><<<convert_blocks(nn), 256, 0, h->st>>>((const double*)h->avg + off,
                                                                                h->io32, (long long)nn);
            CK(h, cudaGetLastError());
        }
    } else {
        int rc = materialize(h);
        if (rc) return rc;
        const size_t plane = field == IPPI_FIELD_F      ? 0
                             : field == IPPI_FIELD_RHO  ? 9
                             : field == IPPI_FIELD_UX   ? 10
                             : field == IPPI_FIELD_UY   ? 11
                             : field == IPPI_FIELD_NNFLAG ? 12
                                                        : 13;  // TAU
        convert_kernel<double, float><<<convert_blocks(n), 256, 0, h->st>>>(h->dl + plane * nn, h->io32,
                                                                           (long long)n);
        CK(h, cudaGetLastError());
    }
    CK(h, cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return IPPI_OK;
}

int ippi_forces(ippi_lbm* h, double* force_xy, int* nbody, double* mass)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    CK(h, cudaSetDevice(h->p.device));
    if (nbody) *nbody = h->nbody;
    if (h->pending_init && (force_xy || mass)) {
        int rc = materialize(h);
        if (rc) return rc;
    }
    if (force_xy && h->nbody > 0) {
        CK(h, cudaStreamSynchronize(h->st));
        CK(h, cudaMemcpy(force_xy, h->force_now, (size_t)h->nbody * 2 * sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (mass) {
        int rc = materialize(h);
        if (rc) return rc;
        const size_t nn = (size_t)h->p.nx * h->p.ny;
        const int nblk = 1024;
        sum_partial_kernel<<<nblk, 256, 0, h->st>>>(h->dl + 9 * nn, (long long)nn, h->red);
        sum_partial_kernel<<<1, 256, 0, h->st>>>(h->red, nblk, h->red + nblk);
        CK(h, cudaGetLastError());
        CK(h, cudaMemcpyAsync(mass, h->red + nblk, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
    }
    return IPPI_OK;
}

int ippi_force_history(ippi_lbm* h, double* out, int max_steps)
{
    if (!h || (!out && max_steps > 0)) return fail(h, IPPI_ERR_ARG, "null argument");
    if (h->nbody == 0) return 0;
    CK(h, cudaSetDevice(h->p.device));
    CK(h, cudaStreamSynchronize(h->st));
    const long long avail = std::min<long long>(h->hist_written + (h->pending_init ? 0 : 1), h->hist_cap);
    const int n = (int)std::min<long long>(avail, max_steps);
    const int nb = h->nbody;
    // the ring slots of steps last_t - n + 1 .. last_t: at most two runs
    const size_t row = (size_t)nb * 2 * sizeof(double);
    int i = 0;
    while (i < n) {
        const long long t = (long long)h->last_t - (n - 1) + i;
        const long long slot = ((t % h->hist_cap) + h->hist_cap) % h->hist_cap;
        const int run = (int)std::min<long long>(n - i, h->hist_cap - slot);
        CK(h, cudaMemcpy(out + (size_t)i * nb * 2, h->force_hist + (size_t)slot * nb * 2, run * row,
                         cudaMemcpyDeviceToHost));
        i += run;
    }
    return n;
}

int ippi_get_stream(ippi_lbm* h, void** stream)
{
    if (!h || !stream) return fail(h, IPPI_ERR_ARG, "null argument");
    *stream = (void*)h->st;
    return IPPI_OK;
}

int ippi_diagnostics(ippi_lbm* h, double* max_u, long long* net_nodes, long long* fallback_nodes)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    CK(h, cudaSetDevice(h->p.device));
    int rc = materialize(h);
    if (rc) return rc;
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    const int learned = h->p.les_model == IPPI_LES_LEARNED;
    unsigned long long* out = reinterpret_cast<unsigned long long*>(h->red);
    CK(h, cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), h->st));
    const unsigned nblk = (unsigned)std::min<size_t>((nn + 255) / 256, 4 * 148);
    diag_kernel<<<nblk, 256, 0, h->st>>>(h->dl + 9 * nn, h->nflag, (long long)nn, learned, out);
    CK(h, cudaGetLastError());
    unsigned long long r[3];
    CK(h, cudaMemcpyAsync(r, out, sizeof r, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    if (max_u) std::memcpy(max_u, &r[0], sizeof(double));
    if (net_nodes) *net_nodes = (long long)r[1];
    if (fallback_nodes) *fallback_nodes = (long long)r[2];
    return IPPI_OK;
}

int ippi_state_bytes(ippi_lbm* h, size_t* bytes)
{
    if (!h || !bytes) return fail(h, IPPI_ERR_ARG, "null argument");
    *bytes = ckp_layout(h).total;
    return IPPI_OK;
}

int ippi_save_state(ippi_lbm* h, void* host, size_t bytes)
{
    if (!h || !host) return fail(h, IPPI_ERR_ARG, "null argument");
    const CkpLayout L = ckp_layout(h);
    if (bytes < L.total) return fail(h, IPPI_ERR_ARG, "checkpoint needs %zu bytes, got %zu", L.total, bytes);
    CK(h, cudaSetDevice(h->p.device));
    if (h->pending_init) return fail(h, IPPI_ERR_STATE, "no state to save before the first step");
    Range range("ippi_save_state");
    CkpHeader hd{};
    std::memcpy(hd.magic, kCkpMagic, sizeof hd.magic);
    hd.abi = IPPI_ABI_VERSION;
    hd.header_bytes = sizeof(CkpHeader);
    hd.config_hash = ckp_config_hash(h);
    hd.nx = h->p.nx;
    hd.ny = h->p.ny;
    hd.storage = h->p.storage;
    hd.nbody = h->nbody;
    hd.hist_cap = h->hist_cap;
    hd.cur = h->cur;
    hd.kcount = h->kcount;
    hd.last_t = h->last_t;
    hd.hist_written = h->hist_written;
    hd.f_bytes = L.f;
    hd.avg_bytes = L.avg;
    hd.corner_bytes = L.corner;
    hd.force_bytes = L.force;
    hd.hist_bytes = L.hist;
    int rc = ippi_forces(h, nullptr, nullptr, &hd.mass);
    if (rc) return rc;
    CK(h, cudaStreamSynchronize(h->st));
    unsigned char* p = static_cast<unsigned char*>(host) + sizeof(CkpHeader);
    for (const CkpSection& s : ckp_sections(h, L)) {
        if (s.bytes) CK(h, cudaMemcpy(p, s.dev, s.bytes, cudaMemcpyDeviceToHost));
        p += s.bytes;
    }
    hd.payload_hash = ckp_hash(static_cast<unsigned char*>(host) + sizeof(CkpHeader), L.total - sizeof(CkpHeader));
    std::memcpy(host, &hd, sizeof hd);
    return IPPI_OK;
}

int ippi_load_state(ippi_lbm* h, const void* host, size_t bytes, int* last_step)
{
    if (!h || !host) return fail(h, IPPI_ERR_ARG, "null argument");
    if (bytes < sizeof(CkpHeader)) return fail(h, IPPI_ERR_ARG, "checkpoint shorter than its header");
    CkpHeader hd;
    std::memcpy(&hd, host, sizeof hd);
    if (std::memcmp(hd.magic, kCkpMagic, sizeof hd.magic) != 0) return fail(h, IPPI_ERR_ARG, "not a checkpoint");
    if (hd.abi != IPPI_ABI_VERSION || hd.header_bytes != sizeof(CkpHeader))
        return fail(h, IPPI_ERR_ARG, "checkpoint of ABI %u, this library is %d", hd.abi, IPPI_ABI_VERSION);
    const CkpLayout L = ckp_layout(h);
    if (hd.nx != h->p.nx || hd.ny != h->p.ny || hd.storage != h->p.storage || hd.nbody != h->nbody ||
        hd.hist_cap != h->hist_cap || hd.f_bytes != L.f || hd.avg_bytes != L.avg || hd.corner_bytes != L.corner ||
        hd.force_bytes != L.force || hd.hist_bytes != L.hist)
        return fail(h, IPPI_ERR_ARG, "checkpoint of a %dx%d lattice (storage %d, %d bodies) does not fit this handle",
                    hd.nx, hd.ny, hd.storage, hd.nbody);
    if (bytes < L.total) return fail(h, IPPI_ERR_ARG, "checkpoint truncated (%zu of %zu bytes)", bytes, L.total);
    if (hd.config_hash != ckp_config_hash(h))
        return fail(h, IPPI_ERR_ARG, "checkpoint of another configuration (parameters, markers or solid mask)");
    if (hd.cur != 0 && hd.cur != 1) return fail(h, IPPI_ERR_ARG, "checkpoint buffer index %d", hd.cur);
    const unsigned char* p = static_cast<const unsigned char*>(host) + sizeof(CkpHeader);
    if (ckp_hash(p, L.total - sizeof(CkpHeader)) != hd.payload_hash)
        return fail(h, IPPI_ERR_ARG, "checkpoint payload hash mismatch (corrupted)");
    CK(h, cudaSetDevice(h->p.device));
    Range range("ippi_load_state");
    CK(h, cudaStreamSynchronize(h->st));
    for (const CkpSection& s : ckp_sections(h, L)) {
        if (s.bytes) CK(h, cudaMemcpy(s.dev, p, s.bytes, cudaMemcpyHostToDevice));
        p += s.bytes;
    }
    std::memset(h->ctr_h, 0, sizeof(Ctr));
    CK(h, cudaMemcpy(h->ctr, h->ctr_h, sizeof(Ctr), cudaMemcpyHostToDevice));
    h->cur = hd.cur;
    h->kcount = (int)hd.kcount;
    h->last_t = (int)hd.last_t;
    h->hist_written = hd.hist_written;
    h->pending_init = false;
    h->dl_valid = false;
    double mass = 0.0;
    int rc = ippi_forces(h, nullptr, nullptr, &mass);
    if (rc) return rc;
    if (std::memcmp(&mass, &hd.mass, sizeof mass) != 0)
        return fail(h, IPPI_ERR_ARG, "checkpoint mass %.17g, this configuration gives %.17g", hd.mass, mass);
    if (last_step) *last_step = h->last_t;
    return IPPI_OK;
}

int ippi_last_error(ippi_lbm* h, char* buf, size_t n)
{
    if (!buf || n == 0) return IPPI_ERR_ARG;
    snprintf(buf, n, "%s", h ? h->err : g_last_error);
    return IPPI_OK;
}

}  // extern "C"

namespace {
// the tensor-core fragments of the loaded network, on the device
int upload_mlp_frag(ippi_lbm* h)
{
    if (h->mlp_host.size() < (size_t)kMlpParams) return IPPI_OK;
    const MlpFrag fr = mlp_fragments(h->mlp_host.data());
    if (!h->mlp_frag) CK(h, dalloc(&h->mlp_frag, sizeof(MlpFrag)));
    CK(h, cudaMemcpy(h->mlp_frag, &fr, sizeof(MlpFrag), cudaMemcpyHostToDevice));
    return IPPI_OK;
}
}  // namespace

int ippi_set_learned_tensor_cores(ippi_lbm* h, int on)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (on && h->p.les_model != IPPI_LES_LEARNED)
        return fail(h, IPPI_ERR_STATE, "tensor cores for the learned tau need les_model IPPI_LES_LEARNED");
    if (on && h->p.storage == IPPI_F64)
        return fail(h, IPPI_ERR_ARG, "the tensor-core network is for FP32 arithmetic (not FP64 storage)");
    CK(h, cudaSetDevice(h->p.device));
    CK(h, cudaStreamSynchronize(h->st));
    h->mlp_tc = on != 0;
    if (h->mlp_tc)
        if (int rc = upload_mlp_frag(h)) return rc;
    drop_graphs(h);
    return IPPI_OK;
}

int ippi_load_tau_mlp(ippi_lbm* h, const uint16_t* w_bf16, size_t n, const float* stats, size_t nstats)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (!w_bf16 || !stats || n != (size_t)IPPI_MLP_PARAMS || nstats != (size_t)IPPI_MLP_STATS)
        return fail(h, IPPI_ERR_ARG, "tau network: %d BF16 weights and %d statistics expected", IPPI_MLP_PARAMS,
                    IPPI_MLP_STATS);
    std::vector<float> blob(IPPI_MLP_PARAMS + IPPI_MLP_STATS);
    for (int i = 0; i < IPPI_MLP_PARAMS; i++) {
        const uint32_t bits = (uint32_t)w_bf16[i] << 16;
        std::memcpy(&blob[i], &bits, 4);
        if (!std::isfinite(blob[i])) return fail(h, IPPI_ERR_ARG, "tau network weight %d is not finite", i);
    }
    for (int i = 0; i < IPPI_MLP_STATS; i++) blob[IPPI_MLP_PARAMS + i] = stats[i];
    for (int i = 0; i < 6; i++)
        if (!(stats[6 + i] > 0) || !(stats[12 + i] <= stats[18 + i]) || !std::isfinite(stats[i]))
            return fail(h, IPPI_ERR_ARG, "tau network statistics of feature %d are invalid", i);
    if (!(stats[24] > 0) || !std::isfinite(stats[24])) return fail(h, IPPI_ERR_ARG, "out_scale must be positive");
    CK(h, cudaSetDevice(h->p.device));
    CK(h, cudaStreamSynchronize(h->st));
    if (!h->mlp_dev) CK(h, dalloc(&h->mlp_dev, blob.size() * sizeof(float)));
    CK(h, cudaMemcpy(h->mlp_dev, blob.data(), blob.size() * sizeof(float), cudaMemcpyHostToDevice));
    h->mlp_version = ++g_mlp_serial;
    h->mlp_hash = ckp_hash(reinterpret_cast<const unsigned char*>(blob.data()), blob.size() * sizeof(float),
                           0x6d6c70ull);
    h->mlp_host = blob;
    if (h->mlp_tc)
        if (int rc = upload_mlp_frag(h)) return rc;
    // step graphs captured before the first load hold a null network pointer
    drop_graphs(h);
    h->dl_valid = false;
    return IPPI_OK;
}

int ippi_filter_snapshot(ippi_lbm* h, int factor, double* out, size_t bytes)
{
    if (!h || !out) return fail(h, IPPI_ERR_ARG, "null argument");
    const int nx = h->p.nx, ny = h->p.ny;
    if (factor < 1 || nx % factor || ny % factor)
        return fail(h, IPPI_ERR_ARG, "filter factor %d must divide %d and %d", factor, nx, ny);
    const size_t m = (size_t)(nx / factor) * (ny / factor);
    if (bytes != 6 * m * sizeof(double)) return fail(h, IPPI_ERR_ARG, "filtered snapshot needs %zu bytes", 6 * m * sizeof(double));
    CK(h, cudaSetDevice(h->p.device));
    if (int rc = materialize(h)) return rc;
    double* d = nullptr;
    CK(h, dalloc(&d, 6 * m * sizeof(double)));
    const dim3 grid((nx / factor + 127) / 128, ny / factor);
    filter_snapshot_kernel<<<grid, 128, 0, h->st>>>(h->dl, nx, ny, factor, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, 6 * m * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    dfree(d);
    CK(h, e);
    return IPPI_OK;
}

int ippi_set_tau_field(ippi_lbm* h, const double* tau)
{
    if (!h || !tau) return fail(h, IPPI_ERR_ARG, "null argument");
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    for (size_t i = 0; i < nn; i++)
        if (!(tau[i] > 0.5) || !std::isfinite(tau[i]))
            return fail(h, IPPI_ERR_ARG, "tau field must exceed 0.5 (node %zu)", i);
    CK(h, cudaSetDevice(h->p.device));
    CK(h, cudaStreamSynchronize(h->st));
    if (!h->tau_field) CK(h, dalloc(&h->tau_field, nn * sizeof(double)));
    CK(h, cudaMemcpy(h->tau_field, tau, nn * sizeof(double), cudaMemcpyHostToDevice));
    h->tau_field_hash = ckp_hash(reinterpret_cast<const unsigned char*>(tau), nn * sizeof(double), 0x746175ull);
    drop_graphs(h);
    h->dl_valid = false;
    return IPPI_OK;
}

// ---------------------------------------------------------------------------
// adjoint
// ---------------------------------------------------------------------------
int ippi_load_tau_mlp_f32(ippi_lbm* h, const float* w, size_t n, const float* stats, size_t nstats)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (!w || n != (size_t)IPPI_MLP_PARAMS) return fail(h, IPPI_ERR_ARG, "tau network: %d weights expected", IPPI_MLP_PARAMS);
    std::vector<uint16_t> dummy(IPPI_MLP_PARAMS, 0);
    int rc = ippi_load_tau_mlp(h, dummy.data(), n, stats, nstats);  // validates and allocates
    if (rc) return rc;
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(w[i])) return fail(h, IPPI_ERR_ARG, "tau network weight %zu is not finite", i);
    CK(h, cudaMemcpy(h->mlp_dev, w, n * sizeof(float), cudaMemcpyHostToDevice));
    std::copy(w, w + n, h->mlp_host.begin());
    if (h->mlp_tc)
        if (int rc2 = upload_mlp_frag(h)) return rc2;
    h->mlp_version = ++g_mlp_serial;
    h->mlp_hash = ckp_hash(reinterpret_cast<const unsigned char*>(stats), nstats * sizeof(float),
                           ckp_hash(reinterpret_cast<const unsigned char*>(w), n * sizeof(float), 0x6d6c7033ull));
    return IPPI_OK;
}

int ippi_adjoint_forward(ippi_lbm* h, int nsteps, int t0, int ckpt_every)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (nsteps < 1 || ckpt_every < 1) return fail(h, IPPI_ERR_ARG, "nsteps and ckpt_every must be positive");
    if (h->p.bc_set != IPPI_BC_CHANNEL) return fail(h, IPPI_ERR_STATE, "the adjoint is built for the channel scene");
    if (!h->solid.empty()) return fail(h, IPPI_ERR_STATE, "the adjoint does not take solid nodes");
    if (h->p.les_model >= IPPI_LES_WALE)
        return fail(h, IPPI_ERR_STATE, "the adjoint takes the relaxation-time models 0-3");
    if (h->mlp_tc)
        return fail(h, IPPI_ERR_STATE, "the adjoint linearises the FMA network: switch the tensor cores off");
    if (h->ib_active && h->p.mdf_iters != 1)
        return fail(h, IPPI_ERR_STATE, "the adjoint supports one direct-forcing pass (mdf_iters = 1)");
    if (h->ib_active && (long long)nsteps > h->hist_cap)
        return fail(h, IPPI_ERR_ARG, "rollout longer than the force history (%d steps)", h->hist_cap);
    if (int rc = tau_ready(h)) return rc;
    CK(h, cudaSetDevice(h->p.device));
    Range range("ippi_adjoint_forward");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    adjoint_free(h);
    if (h->pending_init) {
        int rc = run_init(h);
        if (rc) return rc;
    }
    const size_t fbytes = (size_t)9 * h->plane * h->tsize;
    const int nck = (nsteps + ckpt_every - 1) / ckpt_every;
    for (int i = 0; i < nck; i++) {
        void* p = nullptr;
        if (dalloc(&p, fbytes) != cudaSuccess) {
            adjoint_free(h);
            return fail(h, IPPI_ERR_NOMEM, "adjoint checkpoints (%d x %zu bytes)", nck, fbytes);
        }
        h->adj.ck.push_back(p);
        CK(h, cudaMemcpyAsync(p, h->f[h->cur], fbytes, cudaMemcpyDeviceToDevice, h->st));
        const int n = std::min(ckpt_every, nsteps - i * ckpt_every);
        int rc = ippi_step(h, n, t0 + i * ckpt_every);
        if (rc) {
            adjoint_free(h);
            return rc;
        }
    }
    h->adj.nsteps = nsteps;
    h->adj.t0 = t0;
    h->adj.K = ckpt_every;
    h->adj.ready = true;
    return IPPI_OK;
}

int ippi_adjoint_backward(ippi_lbm* h, const double* dl_dforce, const double* dl_dmacro, double* grad_tau,
                          double* grad_mlp, double* grad_f0)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (!h->adj.ready) return fail(h, IPPI_ERR_STATE, "no recorded rollout (ippi_adjoint_forward)");
    if (grad_tau && h->p.les_model != IPPI_LES_FIELD)
        return fail(h, IPPI_ERR_STATE, "grad_tau needs the tau-field model (IPPI_LES_FIELD)");
    if (grad_mlp && h->p.les_model != IPPI_LES_LEARNED)
        return fail(h, IPPI_ERR_STATE, "grad_mlp needs the learned model (IPPI_LES_LEARNED)");
    CK(h, cudaSetDevice(h->p.device));
    Range range("ippi_adjoint_backward");
    MlpLock lock(h);
    if (int rc = mlp_const_ready(h)) return rc;
    const int nx = h->p.nx, ny = h->p.ny, nsteps = h->adj.nsteps, K = h->adj.K;
    const size_t nn = (size_t)nx * ny;
    const size_t fbytes = (size_t)9 * h->plane * h->tsize;
    auto& W = h->adj.work;
    auto get = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (dalloc(&p, bytes) != cudaSuccess) p = nullptr;
        W.push_back(p);  // a failed allocation stays as a null entry
        if (p) cudaMemsetAsync(p, 0, bytes, h->st);
        return p;
    };
    // work buffers (freed with the record)
    for (void* p : W) dfree(p);
    W.clear();
    for (void* p : h->adj.seg) dfree(p);
    h->adj.seg.clear();
    for (int i = 1; i < K && i < nsteps; i++) {
        void* p = nullptr;
        if (dalloc(&p, fbytes) != cudaSuccess) return fail(h, IPPI_ERR_NOMEM, "adjoint segment buffers");
        h->adj.seg.push_back(p);
    }
    AdjArgs A{};
    A.storage = h->S;
    A.collision = h->p.collision;
    A.learned = h->p.les_model == IPPI_LES_LEARNED;
    A.ft = (double*)get(9 * nn * sizeof(double));
    A.m = (double*)get(3 * nn * sizeof(double));
    double* la = (double*)get(9 * nn * sizeof(double));
    double* lb = (double*)get(9 * nn * sizeof(double));
    A.lam_ft = (double*)get(9 * nn * sizeof(double));
    A.grad_tau = grad_tau ? (double*)get(nn * sizeof(double)) : nullptr;
    A.lin = A.learned ? (double*)get(nn * 8 * sizeof(double)) : nullptr;
    double* gmlp = nullptr;
    double* part = nullptr;
    if (grad_mlp) {
        A.xs = (double*)get(nn * 6 * sizeof(double));
        A.up = (double*)get(nn * sizeof(double));
        gmlp = (double*)get(IPPI_MLP_PARAMS * sizeof(double));
        part = (double*)get(mlp_grad_f64_partial_doubles() * sizeof(double));
    }
    double* dldm = nullptr;
    if (dl_dmacro) {
        dldm = (double*)get(3 * nn * sizeof(double));
        if (dldm) CK(h, cudaMemcpyAsync(dldm, dl_dmacro, 3 * nn * sizeof(double), cudaMemcpyHostToDevice, h->st));
    }
    double* dldF = nullptr;
    IbArgs I = h->ib;
    if (h->ib_active) {
        const int nf = h->nforced, nm = h->nmark;
        A.ib = &I;
        A.nst = h->ib_nst;
        A.fidx = (int*)get(nn * sizeof(int));
        A.mbody = (int*)get(std::max(nm, 1) * sizeof(int));
        A.ib_rho = (double*)get(nf * sizeof(double));
        A.lam_rho = (double*)get(nf * sizeof(double));
        A.ib_us = (double2*)get(nf * sizeof(double2));
        A.ib_fn = (double2*)get(nf * sizeof(double2));
        A.ib_uc = (double2*)get(nf * sizeof(double2));
        A.lam_uc = (double2*)get(nf * sizeof(double2));
        A.lam_fn = (double2*)get(nf * sizeof(double2));
        A.lam_ftot = (double2*)get(nf * sizeof(double2));
        A.ib_F = (double2*)get(nm * sizeof(double2));
        A.lam_F = (double2*)get(nm * sizeof(double2));
        if (dl_dforce) {
            const size_t nb = (size_t)nsteps * h->nbody * 2;
            dldF = (double*)get(nb * sizeof(double));
            if (dldF) CK(h, cudaMemcpyAsync(dldF, dl_dforce, nb * sizeof(double), cudaMemcpyHostToDevice, h->st));
        }
    }
    for (void* p : W)
        if (!p) return fail(h, IPPI_ERR_NOMEM, "adjoint work buffers");
    if (h->ib_active) CK(h, adj_ib_tables(I, nx, ny, const_cast<int*>(A.fidx), const_cast<int*>(A.mbody), h->st));

    h->no_avg = true;
    int rc = IPPI_OK;
    const int nck = (int)h->adj.ck.size();
    for (int seg = nck - 1; seg >= 0 && rc == IPPI_OK; seg--) {
        const int s0 = seg * K, s1 = std::min(s0 + K, nsteps);
        std::vector<const void*> in(s1 - s0);
        in[0] = h->adj.ck[seg];
        // recompute the segment's step inputs with the forward kernels
        h->ctr_h->t[0] = h->adj.t0 + s0;
        cudaMemcpyAsync(&h->ctr->t[0], &h->ctr_h->t[0], sizeof(int), cudaMemcpyHostToDevice, h->st);
        for (int s = s0; s < s1 - 1; s++) {
            void* out = h->adj.seg[s - s0];
            LaunchSet L = make_launch(h, MODE_STEP, in[s - s0], out, (s - s0) & 1);
            cudaError_t e = launch(L, h->S);
            if (e != cudaSuccess) {
                rc = fail(h, IPPI_ERR_CUDA, "adjoint recompute: %s", cudaGetErrorString(e));
                break;
            }
            in[s - s0 + 1] = out;
        }
        for (int s = s1 - 1; s >= s0 && rc == IPPI_OK; s--) {
            A.s = make_launch(h, MODE_STEP, in[s - s0], nullptr, 0).step;
            A.lam_out = la;
            A.lam_in = lb;
            A.dldm = dldm;
            A.dldF = dldF ? dldF + (size_t)s * h->nbody * 2 : nullptr;
            cudaError_t e = adj_state(A, h->st);
            if (e == cudaSuccess && h->ib_active) e = adj_ib_fwd(A, h->st);
            if (e == cudaSuccess) e = adj_collide(A, h->st);
            if (e == cudaSuccess && dldm && s == nsteps - 1) e = adj_inject_moments(A, h->st);
            if (e == cudaSuccess && gmlp) e = mlp_grad_upstream_f64(A.xs, A.up, (int)nn, h->mlp_dev, part, gmlp, h->st);
            if (e == cudaSuccess && h->ib_active) e = adj_ib_back(A, h->st);
            if (e == cudaSuccess) e = adj_stream(A, h->st);  // writes every entry of lb
            if (e != cudaSuccess) rc = fail(h, IPPI_ERR_CUDA, "adjoint step %d: %s", s, cudaGetErrorString(e));
            std::swap(la, lb);
        }
    }
    h->no_avg = false;
    if (rc) return rc;
    if (grad_f0) CK(h, cudaMemcpyAsync(grad_f0, la, 9 * nn * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    if (grad_tau) CK(h, cudaMemcpyAsync(grad_tau, A.grad_tau, nn * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    if (grad_mlp) CK(h, cudaMemcpyAsync(grad_mlp, gmlp, IPPI_MLP_PARAMS * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    CK(h, cudaGetLastError());
    return IPPI_OK;
}

int ippi_tau_scan(ippi_lbm* h, int n, const int* xy, const double* target, int m_lo, int m_hi, double step,
                  double* best_dtau, double* best_err)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (n < 0 || (n > 0 && (!xy || !target || !best_dtau || !best_err)) || m_lo > m_hi || !(step > 0))
        return fail(h, IPPI_ERR_ARG, "bad tau-scan arguments");
    if (n == 0) return IPPI_OK;
    const int nx = h->p.nx, ny = h->p.ny;
    for (int q = 0; q < n; q++)
        if (xy[2 * q] < 1 || xy[2 * q] > nx - 2 || xy[2 * q + 1] < 1 || xy[2 * q + 1] > ny - 2)
            return fail(h, IPPI_ERR_ARG, "tau-scan node %d is not an interior node", q);
    CK(h, cudaSetDevice(h->p.device));
    if (int rc = materialize(h)) return rc;
    const size_t nn = (size_t)nx * ny;
    int* dxy = nullptr;
    double *dt = nullptr, *dout = nullptr;
    cudaError_t e = dalloc(&dxy, 2 * (size_t)n * sizeof(int));
    if (e == cudaSuccess) e = dalloc(&dt, 3 * (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = dalloc(&dout, 2 * (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dxy, xy, 2 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, target, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->st);
    // the materialised post-stream state: f planes 0..8, rho/ux/uy 9..11,
    // tau of the next collision 13
    if (e == cudaSuccess)
        e = tau_scan_launch(h->dl, h->dl + 9 * nn, h->dl + 13 * nn, nx, ny, n, dxy, dt, m_lo, m_hi, step, dout,
                            dout + n, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(best_dtau, dout, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(best_err, dout + n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    dfree(dxy);
    dfree(dt);
    dfree(dout);
    CK(h, e);
    return IPPI_OK;
}

int ippi_set_solid(ippi_lbm* h, const uint8_t* solid, size_t n)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    const int nx = h->p.nx, ny = h->p.ny;
    const size_t nn = (size_t)nx * ny;
    if (n == 0) {
        h->solid.clear();
        return rebuild(h);
    }
    if (!solid || n != nn) return fail(h, IPPI_ERR_ARG, "solid mask needs nx * ny = %zu entries", nn);
    if (h->p.bc_set != IPPI_BC_CHANNEL) return fail(h, IPPI_ERR_ARG, "solid nodes are built for the channel scene");
    for (size_t i = 0; i < nn; i++) {
        const int x = (int)(i % nx), y = (int)(i / nx);
        if (solid[i] && (x < 3 || x > nx - 4 || y < 3 || y > ny - 4))
            return fail(h, IPPI_ERR_ARG, "solid node %zu is closer than 3 nodes to the lattice edge", i);
    }
    std::vector<uint8_t> keep = h->solid;
    h->solid.assign(solid, solid + nn);
    for (auto& v : h->solid) v = v ? 1 : 0;
    int rc = rebuild(h);
    if (rc) {
        h->solid = keep;
        rebuild(h);
    }
    return rc;
}

int ippi_solid_force(ippi_lbm* h, double* force_xy)
{
    if (!h || !force_xy) return fail(h, IPPI_ERR_ARG, "null argument");
    if (h->nlinks == 0) {
        force_xy[0] = force_xy[1] = 0.0;
        return IPPI_OK;
    }
    if (h->pending_init) return fail(h, IPPI_ERR_STATE, "no step taken yet");
    CK(h, cudaSetDevice(h->p.device));
    if (int rc = materialize(h)) return rc;
    if (!h->solid_out) CK(h, dalloc(&h->solid_out, 2 * sizeof(double)));
    // the last step started from f[cur ^ 1]: its post-collision field
    const StepArgs a = make_launch(h, MODE_STEP, h->f[h->cur ^ 1], nullptr, 0).step;
    switch (h->S) {
    case ST_F64: solid_force_kernel<ST_F64><<<1, 256, 0, h->st>>>(a, h->solid_links, h->nlinks, h->dl, h->solid_out); break;
    case ST_F32: solid_force_kernel<ST_F32><<<1, 256, 0, h->st>>>(a, h->solid_links, h->nlinks, h->dl, h->solid_out); break;
    case ST_F16: solid_force_kernel<ST_F16><<<1, 256, 0, h->st>>>(a, h->solid_links, h->nlinks, h->dl, h->solid_out); break;
    default: solid_force_kernel<ST_BF16><<<1, 256, 0, h->st>>>(a, h->solid_links, h->nlinks, h->dl, h->solid_out); break;
    }
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(force_xy, h->solid_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return IPPI_OK;
}

int ippi_set_les_cs(ippi_lbm* h, double cs)
{
    if (!h) return fail(nullptr, IPPI_ERR_ARG, "null handle");
    if (!(cs >= 0) || !std::isfinite(cs)) return fail(h, IPPI_ERR_ARG, "Cs must be finite and >= 0");
    if (cs == h->p.cs) return IPPI_OK;
    CK(h, cudaSetDevice(h->p.device));
    CK(h, cudaStreamSynchronize(h->st));
    h->p.cs = cs;
    drop_graphs(h);  // the step graphs hold the constant as a kernel parameter
    h->dl_valid = false;
    return IPPI_OK;
}

int ippi_set_wall_distance(ippi_lbm* h, const double* dist)
{
    if (!h || !dist) return fail(h, IPPI_ERR_ARG, "null argument");
    const size_t nn = (size_t)h->p.nx * h->p.ny;
    for (size_t i = 0; i < nn; i++)
        if (!std::isfinite(dist[i])) return fail(h, IPPI_ERR_ARG, "wall distance must be finite (node %zu)", i);
    CK(h, cudaSetDevice(h->p.device));
    CK(h, cudaStreamSynchronize(h->st));
    if (!h->wall_dist) CK(h, dalloc(&h->wall_dist, nn * sizeof(double)));
    CK(h, cudaMemcpy(h->wall_dist, dist, nn * sizeof(double), cudaMemcpyHostToDevice));
    h->wall_hash = ckp_hash(reinterpret_cast<const unsigned char*>(dist), nn * sizeof(double), 0x77616c6cull);
    drop_graphs(h);
    h->dl_valid = false;
    return IPPI_OK;
}
