/*
 * ref_driver.cpp -- C entry points around the reference's own Mesh class,
 * compiled together with the reference sources by oracle/build_ref.sh into
 * oracle/_ref/libippi_ref_<variant>.so.  TEST INFRASTRUCTURE ONLY: it is the
 * checker for the oracle restatement and the timed CPU reference arm.
 *
 * It does what the reference driver main.cpp:52-116 does -- set the Mesh
 * fields, InitialLatMesh, JudgeStyle, then OneLBMStep + ComputeAvgVelocity
 * per step -- with the constants taken from the caller, ranks run as threads
 * through the in-process MPI stand-in, and the state read back on the global
 * grid.  Two adjustments keep the reference runnable, both documented:
 *   - JudgeStyle writes LatMesh[i][Ny].u (mesh.cpp:1438), one element past
 *     each column; the columns are given spare capacity first so that write
 *     lands in owned memory and corrupts nothing (the value is never read);
 *   - the boundary nets are served by the torch stand-in (ref_shim/torch),
 *     or, in the libtorch build (ref_torch/), by libtorch itself loading the
 *     shipped TorchScript archives.
 */
#include "mesh.h"

#include <cstring>
#include <functional>
#include <pthread.h>

namespace {

struct RefSim {
    int nx, ny, ranks, nx_p, rem;
    double tau, cs, u_in;
    int avg_start;
    ippi_mpi_world world;
    std::vector<Mesh> mesh;
    int last_error = 0;
};

/* global x of local column i on rank r (main.cpp:71-83, mesh.cpp:103-108) */
inline int global_x(const RefSim* s, int r, int i) { return (i - 1) + s->nx_p * r; }

struct RankJob {
    RefSim* s;
    int r;
    std::function<void(int)>* fn;
    int err;
};

void* rank_main(void* p)
{
    RankJob* j = (RankJob*)p;
    ippi_mpi_enter(&j->s->world, j->r);
    // one intra-op thread per rank, as the reference's ranks run under
    // OMP_NUM_THREADS=1 (its own at::set_num_threads(1) is commented out,
    // mesh.cpp:2776); with libtorch each net call is pinned to the rank's core
    at::set_num_threads(1);
    try {
        (*j->fn)(j->r);
    } catch (const ippi_mpi_abort&) {
        j->err = -3;
    }
    return nullptr;
}

/* One thread per rank, each with a 256 MiB stack (the reference keeps
 * per-node work arrays on the stack; thread stacks inherited from a host
 * process can be small). */
int run_ranks(RefSim* s, std::function<void(int)> fn)
{
    std::vector<pthread_t> th(s->ranks);
    std::vector<RankJob> jobs(s->ranks);
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, (size_t)256 << 20);
    for (int r = 0; r < s->ranks; r++) {
        jobs[r] = RankJob{s, r, &fn, 0};
        pthread_create(&th[r], &attr, rank_main, &jobs[r]);
    }
    pthread_attr_destroy(&attr);
    for (int r = 0; r < s->ranks; r++) pthread_join(th[r], nullptr);
    for (auto& j : jobs)
        if (j.err) return j.err;
    return 0;
}

}  // namespace

extern "C" {

void* ref_create(int nx, int ny, double tau, double cs, double u_in, int avg_start, int ranks)
{
    RefSim* s = new RefSim();
    s->nx = nx;
    s->ny = ny;
    s->ranks = ranks < 1 ? 1 : ranks;
    s->tau = tau;
    s->cs = cs;
    s->u_in = u_in;
    s->avg_start = avg_start;
    s->world.size = s->ranks;
    s->mesh.resize(s->ranks);
    int CoreNum = s->ranks;
    int Nx_p, PartitionRemainderFlag = 0;
    if (nx % CoreNum == 0) {
        Nx_p = nx / CoreNum;
    } else {
        Nx_p = nx / CoreNum;
        PartitionRemainderFlag = Nx_p + nx % CoreNum;
    }
    s->nx_p = Nx_p;
    s->rem = PartitionRemainderFlag;
    run_ranks(s, [&](int r) {
        Mesh& m = s->mesh[r];
        Point2D center = {400, 620};
        Point2D vel = {(REAL)u_in, 0};
        m.startAvg = avg_start;
        m.center = center;
        m.radius = 20;
        m.startTau = tau;
        m.startU = vel;
        m.MyrankID = r;
        m.MyCoreNum = CoreNum;
        m.stepH = 0;
        m.stepL = 0;
        m.StartCs = cs;
        m.LatmeshSizeNx = nx;
        m.LatmeshSizeNy = ny;
        m.InitialLatMesh(Nx_p, ny, tau, vel, 1.0, r, CoreNum, PartitionRemainderFlag);
        MPI_Barrier(MPI_COMM_WORLD);
        for (auto& col : m.LatMesh) col.reserve(col.size() + 1);
        m.JudgeStyle(center, 20, r, CoreNum);
        m.ParallelSize = Nx_p;
        MPI_Barrier(MPI_COMM_WORLD);
    });
    return s;
}

void ref_destroy(void* h) { delete (RefSim*)h; }

/* Overwrite rho/u of every interior node and reset its populations to
 * equilibrium with InitialLatticeFeq -- what ManageDataFromXflow does
 * (mesh.cpp:2189-2413) with external data.  Arrays are [ny][nx]. */
void ref_init_macros(void* h, const double* rho, const double* ux, const double* uy)
{
    RefSim* s = (RefSim*)h;
    for (int r = 0; r < s->ranks; r++) {
        Mesh& m = s->mesh[r];
        int NX = (int)m.LatMesh.size();
        for (int i = 1; i < NX - 1; i++)
            for (int j = 0; j < s->ny; j++) {
                size_t g = (size_t)j * s->nx + global_x(s, r, i);
                Lattice& L = m.LatMesh[i][j];
                L.rho = rho ? rho[g] : 1.0;
                L.u.x = ux ? ux[g] : 0.0;
                L.u.y = uy ? uy[g] : 0.0;
                L.InitialLatticeFeq();
            }
    }
}

/* main.cpp:105-216: OneLBMStep, barrier, ComputeAvgVelocity, barrier. */
int ref_step(void* h, int nsteps, int t0)
{
    RefSim* s = (RefSim*)h;
    return run_ranks(s, [&](int r) {
        Mesh& m = s->mesh[r];
        for (int t = t0; t < t0 + nsteps; ++t) {
            m.OneLBMStep(r, s->ranks, (REAL)s->cs, (REAL)1, t);
            MPI_Barrier(MPI_COMM_WORLD);
            m.ComputeAvgVelocity(t);
            MPI_Barrier(MPI_COMM_WORLD);
        }
    });
}

/* field ids as the oracle's: 0 F[9][ny][nx], 1 rho, 2 ux, 3 uy, 4 tau,
 * 5 avg_u, 6 avg_v, 7 avg_rho, 8 style char, 9 NNflag */
void ref_get(void* h, int field, double* out)
{
    RefSim* s = (RefSim*)h;
    size_t plane = (size_t)s->nx * s->ny;
    for (int r = 0; r < s->ranks; r++) {
        Mesh& m = s->mesh[r];
        int NX = (int)m.LatMesh.size();
        for (int i = 1; i < NX - 1; i++)
            for (int j = 0; j < s->ny; j++) {
                const Lattice& L = m.LatMesh[i][j];
                size_t g = (size_t)j * s->nx + global_x(s, r, i);
                switch (field) {
                case 0:
                    for (int k = 0; k < 9; k++) out[k * plane + g] = L.fnew[k];
                    break;
                case 1: out[g] = L.rho; break;
                case 2: out[g] = L.u.x; break;
                case 3: out[g] = L.u.y; break;
                case 4: out[g] = L.tau; break;
                case 5: out[g] = L.avg_u; break;
                case 6: out[g] = L.avg_v; break;
                case 7: out[g] = L.avg_density; break;
                case 8: out[g] = (double)(unsigned char)L.style; break;
                case 9: out[g] = L.NNflag ? 1.0 : 0.0; break;
                default: out[g] = 0; break;
                }
            }
    }
}

/* IB primitives of one rank, in the order an IB step would call them:
 * InitialIBParticle (mesh.cpp:173) -> InterpolateVel (552) ->
 * CalParticleForce (514) -> SpreadForce (656) -> UpdateVelocity (1244).
 * Outputs marker positions xy[2n], interpolated velocities vref[2n], marker
 * forces mforce[2n] and node forces nforce[2][ny][nx]; the corrected u stays
 * in the mesh (read it with ref_get). */
int ref_ib_probe(void* h, int n, double radius, double cx, double cy,
                 double* xy, double* vref, double* mforce, double* nforce)
{
    RefSim* s = (RefSim*)h;
    if (s->ranks != 1) return -1;
    return run_ranks(s, [&](int r) {
        Mesh& m = s->mesh[r];
        Point2D pv = {0, 0};
        m.InitialIBParticle(n, radius, cx, cy, pv);
        m.InterpolateVel(r, s->ranks, s->nx_p);
        m.CalParticleForce((int)radius);
        m.SpreadForce(r, s->ranks, s->nx_p);
        m.UpdateVelocity(r, s->ranks);
        for (int q = 0; q < n; q++) {
            xy[2 * q] = m.IBParticle[q].position.x;
            xy[2 * q + 1] = m.IBParticle[q].position.y;
            vref[2 * q] = m.IBParticle[q].vel_ref.x;
            vref[2 * q + 1] = m.IBParticle[q].vel_ref.y;
            mforce[2 * q] = m.IBParticle[q].force.x;
            mforce[2 * q + 1] = m.IBParticle[q].force.y;
        }
        size_t plane = (size_t)s->nx * s->ny;
        int NX = (int)m.LatMesh.size();
        for (int i = 1; i < NX - 1; i++)
            for (int j = 0; j < s->ny; j++) {
                size_t g = (size_t)j * s->nx + global_x(s, r, i);
                nforce[g] = m.LatMesh[i][j].force.x;
                nforce[plane + g] = m.LatMesh[i][j].force.y;
            }
    });
}

}  // extern "C"
