// mesh.cpp -- Mesh over the C ABI of include/ippi_lbm.h.  Method by method
// the reference's IPPI-LBM/mesh.cpp entry points that its driver calls; the
// time step itself (streaming, boundaries, LES, collision, IB, nets,
// averages, error check) is one ippi_step call on the GPU.
#include "mesh.h"

#include <sys/stat.h>

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>

namespace {

const char* field_err(ippi_lbm* h)
{
    static char buf[512];
    ippi_last_error(h, buf, sizeof buf);
    return buf;
}

}  // namespace

Mesh::Mesh() {}

Mesh::~Mesh()
{
    if (h_) ippi_destroy(h_);
}

bool Mesh::check(int rc, const char* what)
{
    if (rc == IPPI_OK) return true;
    if (rc == IPPI_ERR_DIVERGED) {
        // Mesh::ErrorCatch (mesh.cpp:2101-2111)
        cerr << "Simulation Error!" << endl;
        errorflag = 1;
    } else {
        cerr << what << ": " << field_err(h_) << endl;
    }
    if (AbortOnError) std::exit(1);
    return false;
}

// Mesh::InitialLatMesh (mesh.cpp:60-171): the whole lattice on one GPU, rho =
// Rho, u = 0, populations at equilibrium.  Nx is LatmeshSizeNx when set,
// else the slab width of the single rank.
void Mesh::InitialLatMesh(int Nx_P, int Ny, double tau, Point2D StartVel, double Rho, int RankID,
                          int CoreNum, int PartitionRemainderFlag)
{
    if (RankID != 0 || CoreNum != 1) {
        cerr << "InitialLatMesh: one GPU holds the lattice; run one rank (RankID 0, CoreNum 1)" << endl;
        if (AbortOnError) std::exit(1);
        return;
    }
    const int nx = LatmeshSizeNx > 0 ? LatmeshSizeNx : (PartitionRemainderFlag ? PartitionRemainderFlag : Nx_P);
    ippi_params p;
    ippi_params_default(&p, nx, Ny);
    p.collision = Collision;
    p.storage = Storage;
    p.bc_set = BoundarySet;
    p.les_model = LesModel;
    p.tau0 = tau;
    p.cs = StartCs;
    p.u_in = StartVel.x;
    p.rho0 = Rho;
    p.plate_x0 = PlateX0;
    p.avg_start = startAvg;
    p.delta_kernel = DeltaKernel;
    p.mdf_iters = MdfIters;
    p.device = Device;
    if (h_) ippi_destroy(h_);
    h_ = nullptr;
    if (!check(ippi_create(&p, &h_), "ippi_create")) return;
    cs_ = p.cs;
    for (bool& b : net_loaded_) b = false;
    nx_ = nx;
    ny_ = Ny;
    LatmeshSizeNx = nx;
    LatmeshSizeNy = Ny;
    ParallelSize = nx;
    if (Rho != 1.0) {
        std::vector<double> r((size_t)nx * Ny, Rho);
        if (!check(ippi_init_macros(h_, r.data(), nullptr, nullptr), "ippi_init_macros")) return;
    }
    tau_field_.clear();
    if (LesModel == IPPI_LES_FIELD) {
        // the tau-field model starts from every node's TauAtBeginning
        tau_field_.assign((size_t)nx * Ny, tau);
        if (!check(ippi_set_tau_field(h_, tau_field_.data()), "ippi_set_tau_field")) return;
    }
    LatMesh.assign(nx + 2, vector<Lattice>(Ny));
    for (int i = 0; i < nx + 2; i++)
        for (int j = 0; j < Ny; j++) {
            Lattice& L = LatMesh[i][j];
            L.pos = {i - 1, j};
            L.rho = (REAL)Rho;
            L.tau = L.TauAtBeginning = (REAL)tau;
            L.u = {0, 0};
            L.InitialLatticeFeq();
        }
    synced_ = synced_f_ = false;
}

void Mesh::SetInitialField(const double* rho, const double* ux, const double* uy)
{
    if (!h_) return;
    check(ippi_init_macros(h_, rho, ux, uy), "ippi_init_macros");
    synced_ = synced_f_ = false;
}

bool Mesh::LoadBandNet(int type, const float* w, size_t n)
{
    if (!h_ || !check(ippi_load_band_net(h_, type, w, n), "ippi_load_band_net")) return false;
    net_loaded_[type] = true;
    synced_ = synced_f_ = false;
    return true;
}

// Mesh::InitialIBParticle (mesh.cpp:173-191): NumNodes markers on the circle,
// marker i at (X + R sin(2 pi i / N), Y + R cos(2 pi i / N)), prescribed
// velocity ParticleVel.  Each marker carries its arc length 2 pi R / N so
// the body force is the boundary integral (the reference's marker force
// leaves that factor out, mesh.cpp:527-528).
void Mesh::InitialIBParticle(int NumNodes, double Radius, double ParticlePositionX,
                             double ParticlePositionY, Point2D ParticleVel)
{
    IBParticle.assign(NumNodes, Particlenode());
    std::vector<double> xy(2 * (size_t)NumNodes), ub(2 * (size_t)NumNodes), ds(NumNodes);
    for (int i = 0; i < NumNodes; i++) {
        Particlenode& P = IBParticle[i];
        P.position.x = (REAL)(ParticlePositionX + Radius * std::sin(2. * M_PI * (double)i / NumNodes));
        P.position.y = (REAL)(ParticlePositionY + Radius * std::cos(2. * M_PI * (double)i / NumNodes));
        P.position_ref = P.position;
        P.vel = ParticleVel;
        P.center = {(REAL)ParticlePositionX, (REAL)ParticlePositionY};
        xy[2 * i] = P.position.x;
        xy[2 * i + 1] = P.position.y;
        ub[2 * i] = ParticleVel.x;
        ub[2 * i + 1] = ParticleVel.y;
        ds[i] = 2. * M_PI * Radius / NumNodes;
    }
    center = {(REAL)ParticlePositionX, (REAL)ParticlePositionY};
    radius = Radius;
    marker_ds_ = ds;
    if (h_) check(ippi_set_markers(h_, NumNodes, xy.data(), ub.data(), nullptr, ds.data()), "ippi_set_markers");
}

// Mesh::JudgeStyle (mesh.cpp:1391-1454): the node kinds follow from the
// boundary set chosen at InitialLatMesh; this reads them into the mirror.
void Mesh::JudgeStyle(Point2D CylinderCenter1, REAL Radius, int RankID, int CoreNum)
{
    (void)RankID;
    (void)CoreNum;
    center = CylinderCenter1;
    radius = Radius;
    if (!h_) return;
    if (SolidCylinder) {
        std::vector<unsigned char> m((size_t)nx_ * ny_, 0);
        for (int y = 0; y < ny_; y++)
            for (int x = 0; x < nx_; x++) {
                const double dx = x - (double)CylinderCenter1.x, dy = y - (double)CylinderCenter1.y;
                m[(size_t)y * nx_ + x] = dx * dx + dy * dy <= (double)Radius * Radius;
            }
        if (!SetSolid(m.data())) return;
    }
    std::vector<unsigned char> fl((size_t)nx_ * ny_);
    if (!check(ippi_download(h_, IPPI_FIELD_FLAGS, fl.data(), fl.size()), "ippi_download")) return;
    for (int x = 0; x < nx_; x++)
        for (int y = 0; y < ny_; y++) LatMesh[x + 1][y].style = (char)fl[(size_t)y * nx_ + x];
}

// Mesh::OneLBMStep (mesh.cpp:357-513): one step numbered t.  Cs and Pr are
// fixed at InitialLatMesh (StartCs); RankID / CoreNum are 0 / 1.
void Mesh::OneLBMStep(int RankID, int CoreNum, REAL Cs, REAL Pr, int t)
{
    (void)RankID;
    (void)CoreNum;
    (void)Pr;  // unused by the reference's active closure too (mesh.cpp:852-911)
    // the per-call Smagorinsky constant, as CaculateLESTau receives it
    if (h_ && (double)Cs != cs_) {
        if (!check(ippi_set_les_cs(h_, (double)Cs), "ippi_set_les_cs")) return;
        cs_ = (double)Cs;
    }
    RunSteps(t, 1);
}

void Mesh::RunSteps(int t0, int n)
{
    if (!h_ || n <= 0) return;
    check(ippi_step(h_, n, t0), "ippi_step");
    last_t_ = t0 + n - 1;
    synced_ = synced_f_ = false;
}

// Mesh::ComputeAvgVelocity (mesh.cpp:1954-1974): the running means of u, v
// and rho from step startAvg on are updated inside every step on the GPU.
void Mesh::ComputeAvgVelocity(int t) { (void)t; }

void Mesh::Sync(bool with_f)
{
    if (!h_) return;
    const size_t nn = (size_t)nx_ * ny_;
    std::vector<double> buf(nn);
    auto get = [&](int field, auto&& put) {
        if (!check(ippi_download(h_, field, buf.data(), nn * sizeof(double)), "ippi_download")) return;
        for (int y = 0; y < ny_; y++)
            for (int x = 0; x < nx_; x++) put(LatMesh[x + 1][y], buf[(size_t)y * nx_ + x]);
    };
    get(IPPI_FIELD_RHO, [](Lattice& L, double v) { L.rho = (REAL)v; L.p = (REAL)(v / 3.0); });
    get(IPPI_FIELD_UX, [](Lattice& L, double v) { L.u.x = (REAL)v; });
    get(IPPI_FIELD_UY, [](Lattice& L, double v) { L.u.y = (REAL)v; });
    get(IPPI_FIELD_TAU, [](Lattice& L, double v) { L.tau = (REAL)v; });
    get(IPPI_FIELD_AVG_U, [](Lattice& L, double v) { L.avg_u = v; });
    get(IPPI_FIELD_AVG_V, [](Lattice& L, double v) { L.avg_v = v; });
    get(IPPI_FIELD_AVG_RHO, [](Lattice& L, double v) { L.avg_density = v; });
    get(IPPI_FIELD_NNFLAG, [](Lattice& L, double v) { L.NNflag = v != 0; });
    if (with_f) {
        std::vector<double> f(9 * nn);
        if (check(ippi_download(h_, IPPI_FIELD_F, f.data(), f.size() * sizeof(double)), "ippi_download"))
            for (int k = 0; k < 9; k++)
                for (int y = 0; y < ny_; y++)
                    for (int x = 0; x < nx_; x++)
                        LatMesh[x + 1][y].fnew[k] = (REAL)f[k * nn + (size_t)y * nx_ + x];
        synced_f_ = true;
    }
    synced_ = true;
}

void Mesh::ensure_synced()
{
    if (!synced_) Sync(false);
}

// Mesh::ErrorCatch (mesh.cpp:2101-2111) on the mirror; the step checks every
// node on the GPU already (ippi_step reports IPPI_ERR_DIVERGED).
void Mesh::ErrorCatch(int i, int j)
{
    ensure_synced();
    const double r = LatMesh[i][j].rho;
    if (r > 10 || r < 0) {
        cerr << "Simulation Error!" << endl;
        errorflag = 1;
        if (AbortOnError) std::exit(1);
    }
}

// Mesh::InitialFile (mesh.cpp:1170-1179)
void Mesh::InitialFile()
{
    ::mkdir("fluid", 0755);
    ::mkdir("particle", 0755);
    ::mkdir("cp", 0755);
}

// Mesh::WriteDatFluid (mesh.cpp:1180-1243): Tecplot point data, x-major, one
// line per node: X Y Density U V avgu avgv tau avgRho
void Mesh::WriteDatFluid(int t, int RankID, int NX, int CoreNum)
{
    (void)CoreNum;
    ensure_synced();
    std::ostringstream name;
    name << "fluid/fluid_t" << t << "_" << RankID << ".dat";
    std::ofstream out(name.str());
    if (RankID == 0) {
        out << "TITLE = \"Simulation of Fluid State at Time " << t << "\"\n";
        out << "VARIABLES = \"X\" \"Y\" \"Density\" \"U\" \"V\" \"avgu\" \"avgv\" \"tau\" \"avgRho\" \n";
        out << "ZONE T=\"Time " << t << "\", ";
        out << "I=" << ny_ << ", J=" << NX << ", K=1, ";
        out << "DATAPACKING=POINT, ZONETYPE=Ordered\n";
    }
    for (int X = 1; X < nx_ + 1; ++X)
        for (int Y = 0; Y < ny_; ++Y) {
            const Lattice& L = LatMesh[X][Y];
            out << L.pos.x << " " << L.pos.y << " " << L.rho << " " << L.u.x << " " << L.u.y << " "
                << L.avg_u << " " << L.avg_v << " " << L.tau << " " << L.avg_density << "\n";
        }
}

namespace {
// MergeDatFluid / MergeAvgu (mesh.cpp:1320-1353, 2069-2098): concatenate the
// per-rank files and delete them
void merge(const std::string& base, const std::string& merged, int CoreNum)
{
    std::ofstream out(merged);
    for (int i = 0; i <= CoreNum; ++i) {
        const std::string in_name = base + std::to_string(i) + ".dat";
        std::ifstream in(in_name);
        if (!in) continue;
        out << in.rdbuf();
        in.close();
        std::remove(in_name.c_str());
    }
}
}  // namespace

void Mesh::MergeDatFluid(int t, int CoreNum)
{
    merge("fluid/fluid_t" + std::to_string(t) + "_", "fluid/fluid_Merged_" + std::to_string(t) + ".dat",
          CoreNum);
}

// Mesh::WriteAvgu (mesh.cpp:2010-2068): inner rows, style code 0 fluid, 1
// solid, 2 boundary, 3 other kinds
void Mesh::WriteAvgu(int t, int RankID, int NX, int CoreNum)
{
    (void)CoreNum;
    ensure_synced();
    std::ostringstream name;
    name << "fluid/Avgu_" << t << "_" << RankID << ".dat";
    std::ofstream out(name.str());
    if (RankID == 0) {
        out << "TITLE = \"Simulation of Fluid State at Time " << t << "\"\n";
        out << "VARIABLES = \"X\" \"Y\" \"AvgdDenstiy\" \"U\" \"V\" \"avgy\" \"avgv\" \"Style\" \n";
        out << "ZONE T=\"Time " << t << "\", ";
        out << "I=" << ny_ - 2 << ", J=" << NX << ", K=1, ";
        out << "DATAPACKING=POINT, ZONETYPE=Ordered\n";
    }
    for (int X = 1; X < nx_ + 1; ++X)
        for (int Y = 1; Y < ny_ - 1; ++Y) {
            const Lattice& L = LatMesh[X][Y];
            const int code = L.style == 'f' ? 0 : L.style == 's' ? 1 : L.style == 'b' ? 2 : 3;
            out << L.pos.x << " " << L.pos.y << " " << L.rho << " " << L.u.x << " " << L.u.y << " "
                << L.avg_u << " " << L.avg_v << " " << code << "\n";
        }
}

void Mesh::MergeAvgu(int t, int CoreNum)
{
    merge("fluid/Avgu_" + std::to_string(t) + "_", "fluid/fluid_avg_" + std::to_string(t) + ".dat", CoreNum);
}

// Mesh::WriteDatParticle (mesh.cpp:1283-1317): the marker polyline
void Mesh::WriteDatParticle(int t)
{
    std::ostringstream name;
    name << "particle/particle_t" << t << ".dat";
    std::ofstream out(name.str());
    const size_t n = IBParticle.size();
    out << "TITLE = \"Particle State at Time " << t << "\"\n";
    out << "VARIABLES = \"X\" \"Y\" \"Z\"\n";
    out << "ZONE T=\"Particle\", N=" << n << ", E=" << n;
    out << ", DATAPACKING=POINT, ZONETYPE=FELINESEG\n";
    out << "Nodes=" << n << ", Elements=" << n << "\n";
    for (size_t i = 0; i < n; ++i) out << IBParticle[i].position.x << " " << IBParticle[i].position.y << " 0\n";
    for (size_t i = 0; i + 1 < n; ++i) out << i + 1 << " " << i + 2 << "\n";
    if (n) out << 1 << " " << n << "\n";
}

// Mesh::GetSt (mesh.cpp:1975-2009): velocity profiles at x = 9.33 stepH and
// x = 12 stepH appended to particle/5.33H_<t>.dat and particle/8.0H_<t>.dat
void Mesh::GetSt(int t)
{
    ensure_synced();
    for (int i = 1; i < nx_ + 1; i++)
        for (int j = 0; j < ny_; j++) {
            const Lattice& L = LatMesh[i][j];
            const char* which[2] = {"5.33H_", "8.0H_"};
            const double at[2] = {9.33 * stepH, 12.0 * stepH};
            for (int q = 0; q < 2; q++)
                if (L.pos.x == at[q]) {
                    std::ofstream out("particle/" + std::string(which[q]) + std::to_string(t) + ".dat",
                                      std::ios::app);
                    out << L.pos.y * 0.005 << " " << L.u.x << " " << L.u.y << " " << L.avg_u << " "
                        << L.avg_v << std::endl;
                }
        }
}

bool Mesh::SetSolid(const unsigned char* solid)
{
    if (!h_) return false;
    const size_t nn = solid ? (size_t)nx_ * ny_ : 0;
    return check(ippi_set_solid(h_, solid, nn), "ippi_set_solid");
}

// Mesh::OutputCd (mesh.cpp:1461-1526): momentum exchange over the links from
// 'b' nodes into 's' nodes after the last step, Cd / Cl = F / (0.5 U^2 2R)
// with U = startU.x; "t cd cl" appended to particle/CD_CL.dat.
void Mesh::OutputCd(int RankID, int CoreNum, int time, double Radius)
{
    (void)CoreNum;
    double f[2] = {0, 0};
    if (!h_ || !check(ippi_solid_force(h_, f), "ippi_solid_force")) return;
    const double q = 0.5 * (double)startU.x * (double)startU.x * 2 * Radius;
    const double cd = f[0] / q, cl = f[1] / q;
    if (RankID == 0) {
        cerr << "cd:" << cd << " " << "cl:" << cl << endl;
        std::ofstream out("particle/CD_CL.dat", std::ios::app);
        out << time << " " << cd << " " << cl << endl;
    }
}

// Mesh::ComputeCp (mesh.cpp:1642-1655) keeps, on every 'b' node, the running
// mean from step startcp of (p - 1/3) / (0.5 U^2), p = rho / 3.  It is linear
// in rho, so it is the mean density the step accumulates from startAvg on,
// taken through the same map: startcp must equal startAvg.
void Mesh::ComputeCp(int startcp, int t)
{
    if (t < startcp) return;
    if (cp_start_ != startcp && startcp != startAvg)
        cerr << "ComputeCp: the pressure mean starts at startAvg = " << startAvg << ", not " << startcp << endl;
    cp_start_ = startcp;
}

// Mesh::OutputCp (mesh.cpp:1575-1597): "x y cp" of every 'b' node (interior
// columns) to cp/cp_<time>_<rank>.dat
void Mesh::OutputCp(int RankID, int CoreNum, int time, double Radius)
{
    (void)CoreNum;
    (void)Radius;
    ensure_synced();
    const double q = 0.5 * (double)startU.x * (double)startU.x;
    const bool have = cp_start_ >= 0 && last_t_ >= startAvg;
    std::ostringstream name;
    name << "cp/cp_" << time << "_" << RankID << ".dat";
    std::ofstream out(name.str());
    for (int i = 1; i < nx_ + 1; i++)
        for (int j = 0; j < ny_; j++) {
            Lattice& L = LatMesh[i][j];
            if (L.style != 'b') continue;
            L.cp = have ? (L.avg_density / 3.0 - 1.0 / 3.0) / q : 0.0;
            out << L.pos.x << " " << L.pos.y << " " << L.cp << "\n";
        }
}

// Mesh::MergeCp (mesh.cpp:1598-1641): cp/cp_<t>_<r>.dat of every rank into
// cp/cp_Merged_<t>.dat, the parts removed (empty parts skipped)
void Mesh::MergeCp(int t, int CoreNum)
{
    std::ofstream merged("cp/cp_Merged_" + std::to_string(t) + ".dat");
    for (int r = 0; r < CoreNum; r++) {
        const std::string part = "cp/cp_" + std::to_string(t) + "_" + std::to_string(r) + ".dat";
        {
            std::ifstream in(part);
            if (!in) continue;
            if (in.peek() != std::ifstream::traits_type::eof()) merged << in.rdbuf();
        }
        std::remove(part.c_str());
    }
}

// Mesh::GetDuxDx .. GetDuyDy (mesh.cpp:1659-1934) on the mirror: forward
// differences; 0 towards a solid node, in the last column and from the
// second-to-last row up.  The device closures use the same rule.
double Mesh::GetDuxDx(int i, int j)
{
    ensure_synced();
    const int imax = i + 1, Nx = (int)LatMesh.size();
    if (LatMesh[imax][j].style == 's' || imax == Nx - 1) return 0.0;
    return (LatMesh[imax][j].u.x - LatMesh[i][j].u.x) / 1.0;
}

double Mesh::GetDuxDy(int i, int j)
{
    ensure_synced();
    const int jmax = j + 1, Ny = (int)LatMesh[0].size();
    if (jmax >= Ny - 1 || LatMesh[i][jmax].style == 's') return 0.0;
    return (LatMesh[i][jmax].u.x - LatMesh[i][j].u.x) / 1.0;
}

double Mesh::GetDuyDx(int i, int j)
{
    ensure_synced();
    const int imax = i + 1, Nx = (int)LatMesh.size();
    if (LatMesh[imax][j].style == 's' || imax == Nx - 1) return 0.0;
    return (LatMesh[imax][j].u.y - LatMesh[i][j].u.y) / 1.0;
}

double Mesh::GetDuyDy(int i, int j)
{
    ensure_synced();
    const int jmax = j + 1, Ny = (int)LatMesh[0].size();
    if (jmax >= Ny - 1 || LatMesh[i][jmax].style == 's') return 0.0;
    return (LatMesh[i][jmax].u.y - LatMesh[i][j].u.y) / 1.0;
}

// Mesh::SetNormalDis (mesh.cpp:1935-1953): distance of every non-solid node
// to the cylinder surface, measured from the mirror index (i, j) as the
// reference does (for one rank: x + 1, y); handed to the wall-damped closure
void Mesh::SetNormalDis()
{
    const int Nx = (int)LatMesh.size(), Ny = (int)LatMesh[0].size();
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            if (LatMesh[i][j].style == 's') continue;
            const double x = i, y = j, lx = center.x, ly = center.y;
            LatMesh[i][j].normalDis = std::sqrt((x - lx) * (x - lx) + (y - ly) * (y - ly)) - radius;
        }
    if (!h_ || LesModel != IPPI_LES_DYNAMIC) return;
    std::vector<double> d((size_t)nx_ * ny_);
    for (int y = 0; y < ny_; y++)
        for (int x = 0; x < nx_; x++) d[(size_t)y * nx_ + x] = LatMesh[x + 1][y].normalDis;
    check(ippi_set_wall_distance(h_, d.data()), "ippi_set_wall_distance");
}

// Mesh::ComputeDynamicCs (mesh.cpp:2113-2146): the coherent-structure
// coefficient of node (i, j) from the mirror's velocities
double Mesh::ComputeDynamicCs(int i, int j)
{
    const double Sxx = 0.5 * (GetDuxDx(i, j) + GetDuxDx(i, j));
    const double Sxy = 0.5 * (GetDuxDy(i, j) + GetDuyDx(i, j));
    const double Syx = Sxy;
    const double Syy = 0.5 * (GetDuyDy(i, j) + GetDuyDy(i, j));
    const double SS = Sxx * Sxx + Sxy * Sxy + Syx * Syx + Syy * Syy;
    const double Wxy = 0.5 * (GetDuxDy(i, j) - GetDuyDx(i, j));
    const double WW = 2 * Wxy * Wxy;
    const double Q = 0.5 * (WW - SS), E = 0.5 * (WW + SS);
    if (E == 0) return LatMesh[i][j].CoherentCS = 0.016;
    const double F = std::fabs(Q / E);
    return LatMesh[i][j].CoherentCS = (1 / 11.0) * std::pow(F, 1.5) * (1 - F);
}

// ---------------------------------------------------------------------------
// XFlow coupling.  The reference matches every node against every point
// (O(nodes x points), mesh.cpp:2368-2390); a point lands on exactly one node,
// so here each point finds its node directly.  Relaxation times written by
// these methods reach the collision under the tau-field model
// (IPPI_LES_FIELD); under the others the collision recomputes tau every step,
// as the reference's does, and they stay in the mirror.
// ---------------------------------------------------------------------------

// Mesh::ReadXflowdata (mesh.cpp:2413-2547)
vector<PointData> Mesh::ReadXflowdata(int t)
{
    std::vector<PointData> pts;
    const std::string name = XflowDir + "/pb_" + std::to_string(t + XflowStepOffset) + ".csv";
    if (!ippi_host::read_xflow_csv(name, pts)) cerr << "cannot open " << name << endl;
    ippi_host::clip_xflow(pts, MyrankID, MyCoreNum, ParallelSize, LatmeshSizeNx);
    return pts;
}

void Mesh::set_tau_node(int x, int y, double tau)
{
    if (LesModel != IPPI_LES_FIELD) return;
    if (tau_field_.empty()) {
        // the relaxation times the mirror holds
        tau_field_.resize((size_t)nx_ * ny_);
        for (int yy = 0; yy < ny_; yy++)
            for (int xx = 0; xx < nx_; xx++) tau_field_[(size_t)yy * nx_ + xx] = LatMesh[xx + 1][yy].tau;
    }
    tau_field_[(size_t)y * nx_ + x] = tau;
}

void Mesh::upload_tau_field()
{
    if (h_ && LesModel == IPPI_LES_FIELD && !tau_field_.empty())
        check(ippi_set_tau_field(h_, tau_field_.data()), "ippi_set_tau_field");
}

// Lattice::InitialLatticeFeq on every node from the mirror's rho and u
void Mesh::reequilibrate_mirror()
{
    if (!h_) return;
    const size_t nn = (size_t)nx_ * ny_;
    std::vector<double> m(3 * nn);
    for (int y = 0; y < ny_; y++)
        for (int x = 0; x < nx_; x++) {
            const Lattice& L = LatMesh[x + 1][y];
            const size_t g = (size_t)y * nx_ + x;
            m[g] = L.rho;
            m[nn + g] = L.u.x;
            m[2 * nn + g] = L.u.y;
        }
    if (last_t_ > 0)
        check(ippi_reequilibrate(h_, m.data(), m.data() + nn, m.data() + 2 * nn), "ippi_reequilibrate");
    else
        check(ippi_init_macros(h_, m.data(), m.data() + nn, m.data() + 2 * nn), "ippi_init_macros");
    synced_ = synced_f_ = false;
}

// Mesh::ManageDataFromXflow (mesh.cpp:2189-2399): the imported rho, u and
// tau = 3 nu + 1/2 on the nodes the points land on, then every node at the
// equilibrium of its moments
void Mesh::ManageDataFromXflow(int t)
{
    const std::vector<PointData> pts = ReadXflowdata(t);
    ensure_synced();
    for (const PointData& p : pts) {
        int x, y;
        if (!ippi_host::xflow_node(p, nx_, ny_, &x, &y)) continue;
        Lattice& L = LatMesh[x + 1][y];
        L.absU.x = (REAL)(L.u.x - p.ux);
        L.absU.y = (REAL)(L.u.y - p.uy);
        L.absRHO = (REAL)(L.rho - p.TotalPressure);
        L.u.x = (REAL)p.ux;
        L.u.y = (REAL)p.uy;
        L.rho = (REAL)p.TotalPressure;
        L.tau = (REAL)(3 * p.viscosity + 0.5);
        set_tau_node(x, y, L.tau);
    }
    reequilibrate_mirror();
    upload_tau_field();
}

// Mesh::XflowABS (mesh.cpp:2585-2624): differences to the imported state on
// the nodes the points land on, then every node at the equilibrium of its
// moments
void Mesh::XflowABS(int t)
{
    const std::vector<PointData> pts = ReadXflowdata(t);
    ensure_synced();
    for (const PointData& p : pts) {
        int x, y;
        if (!ippi_host::xflow_node(p, nx_, ny_, &x, &y)) continue;
        Lattice& L = LatMesh[x + 1][y];
        L.absU.x = (REAL)(L.u.x - p.ux);
        L.absU.y = (REAL)(L.u.y - p.uy);
        L.absRHO = (REAL)(L.rho - p.TotalPressure);
        L.xflowtau = p.viscosity * 3.0 + 0.5;
        L.abstau = L.tau - L.xflowtau;
    }
    reequilibrate_mirror();
}

// Mesh::ChangeTauFromXflow (mesh.cpp:2717-2766): tau = 1/2 + 3 nu on every
// node, and the mean square velocity and density differences appended to
// cp/InletMSE.dat.  The reference carries the last matched point's values
// into nodes no point lands on (from uninitialised ones before the first
// match); here the carry starts from nu = (startTau - 1/2) / 3 and zero
// errors.  Nodes are visited x-major over the lattice columns.
void Mesh::ChangeTauFromXflow(int t)
{
    const std::vector<PointData> pts = ReadXflowdata(t);
    ensure_synced();
    std::vector<int> at((size_t)nx_ * ny_, -1);
    for (size_t q = 0; q < pts.size(); q++) {
        int x, y;
        if (ippi_host::xflow_node(pts[q], nx_, ny_, &x, &y)) at[(size_t)y * nx_ + x] = (int)q;
    }
    double nu = (startTau - 0.5) / 3.0, ev = 0, er = 0, total_v = 0, total_r = 0;
    for (int x = 0; x < nx_; x++)
        for (int y = 0; y < ny_; y++) {
            Lattice& L = LatMesh[x + 1][y];
            const int q = at[(size_t)y * nx_ + x];
            if (q >= 0) {
                const PointData& p = pts[q];
                nu = p.viscosity;
                ev = (L.u.x - p.ux) * (L.u.x - p.ux) + (L.u.y - p.uy) * (L.u.y - p.uy);
                er = (L.rho - p.TotalPressure) * (L.rho - p.TotalPressure);
            }
            total_v += ev;
            total_r += er;
            L.tau = (REAL)(0.5 + 3.0 * nu);
            set_tau_node(x, y, L.tau);
        }
    upload_tau_field();
    const double n = (double)nx_ * ny_;
    std::ofstream out("cp/InletMSE.dat", std::ios::app);
    out << t << " " << total_v / n << " " << total_r / n << endl;
}

// Mesh::FindAndWriteTau (mesh.cpp:2625-2715): the dtau in [-0.1, 0.1] (step
// 1e-5) whose BGK relaxation of the 9 upstream neighbours best reproduces the
// imported moments of step t + 1 at node (i, j) of the mirror (column i =
// x + 1), scanned on the GPU (ippi_tau_scan); the 9 neighbours' tau += dtau;
// "t dtau tau_0 .. tau_8" appended to cp/BestTau.dat
void Mesh::FindAndWriteTau(int i, int j, int t)
{
    static const int e[9][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
    if (!h_) return;
    const int x = i - 1, y = j;
    const std::vector<PointData> pts = ReadXflowdata(t + 1);
    double target[3];
    bool found = false;
    for (const PointData& p : pts) {
        int px, py;
        if (ippi_host::xflow_node(p, nx_, ny_, &px, &py) && px == x && py == y) {
            target[0] = p.TotalPressure;
            target[1] = p.ux;
            target[2] = p.uy;
            found = true;
        }
    }
    if (!found) {
        cerr << "FindAndWriteTau: no XFlow point on node (" << x << ", " << y << ") at step " << t + 1 << endl;
        return;
    }
    const int xy[2] = {x, y};
    double best = 0, err = 0;
    if (!check(ippi_tau_scan(h_, 1, xy, target, -10000, 10000, 1e-5, &best, &err), "ippi_tau_scan")) return;
    ensure_synced();
    for (int k = 0; k < 9; k++) {
        Lattice& L = LatMesh[i + e[k][0]][j + e[k][1]];
        L.tau = (REAL)(L.tau + best);
        set_tau_node(x + e[k][0], y + e[k][1], L.tau);
    }
    upload_tau_field();
    if (MyrankID == 0) {
        cerr << "Timestep:" << t << " " << "BestTau:" << best << endl;
        std::ofstream out("cp/BestTau.dat", std::ios::app);
        out << t << " " << best << " ";
        for (int k = 0; k < 9; k++) out << LatMesh[i + e[k][0]][j + e[k][1]].tau << " ";
        out << endl;
    }
}

int Mesh::BodyForces(double* fxy, int max_bodies)
{
    if (!h_) return 0;
    int nb = 0;
    if (!check(ippi_forces(h_, nullptr, &nb, nullptr), "ippi_forces")) return 0;
    std::vector<double> f(2 * (size_t)std::max(nb, 1));
    if (!check(ippi_forces(h_, f.data(), &nb, nullptr), "ippi_forces")) return 0;
    for (int b = 0; b < nb && b < max_bodies; b++) {
        fxy[2 * b] = f[2 * b];
        fxy[2 * b + 1] = f[2 * b + 1];
    }
    for (size_t m = 0; m < IBParticle.size() && nb > 0; m++) IBParticle[m].force = {0, 0};
    return nb;
}

void Mesh::DragLift(double U, double D, double* cd, double* cl)
{
    double f[2] = {0, 0};
    BodyForces(f, 1);
    const double q = 0.5 * U * U * D;
    *cd = f[0] / q;
    *cl = f[1] / q;
}

void Mesh::OutputForces(int t, double U, double D)
{
    double f[2] = {0, 0};
    BodyForces(f, 1);
    const double q = 0.5 * U * U * D;
    std::ofstream out("particle/forces.dat", std::ios::app);
    out.precision(12);
    out << t << " " << f[0] << " " << f[1] << " " << f[0] / q << " " << f[1] / q << "\n";
}

// ---------------------------------------------------------------------------
// additions: checkpoint / resume and the metrics log (no reference code; the
// reference writes Tecplot text only and has no restart path)
// ---------------------------------------------------------------------------
bool Mesh::SaveCheckpoint(const std::string& path)
{
    if (!h_) return false;
    size_t n = 0;
    if (!check(ippi_state_bytes(h_, &n), "ippi_state_bytes")) return false;
    std::vector<unsigned char> buf(n);
    if (!check(ippi_save_state(h_, buf.data(), n), "ippi_save_state")) return false;
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::binary | std::ios::trunc);
        if (!out.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)n)) {
            cerr << "cannot write " << tmp << endl;
            return false;
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        cerr << "cannot rename " << tmp << " to " << path << endl;
        return false;
    }
    return true;
}

int Mesh::LoadCheckpoint(const std::string& path)
{
    if (!h_) return -1;
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) {
        cerr << "cannot read " << path << endl;
        return -1;
    }
    const std::streamsize n = in.tellg();
    std::vector<unsigned char> buf((size_t)n);
    in.seekg(0);
    if (!in.read(reinterpret_cast<char*>(buf.data()), n)) {
        cerr << "cannot read " << path << endl;
        return -1;
    }
    int last = -1;
    if (!check(ippi_load_state(h_, buf.data(), buf.size(), &last), "ippi_load_state")) return -1;
    last_t_ = last;
    synced_ = synced_f_ = false;
    return last;
}

void Mesh::LogMetrics(const std::string& path, int t, double mlups, double U, double D)
{
    if (!h_) return;
    int nb = 0;
    double mass = 0, f[2] = {0, 0};
    if (!check(ippi_forces(h_, nullptr, &nb, &mass), "ippi_forces")) return;
    if (nb > 0) BodyForces(f, 1);
    double max_u = 0;
    long long net = 0, fallback = 0;
    if (!check(ippi_diagnostics(h_, &max_u, &net, &fallback), "ippi_diagnostics")) return;
    const int bytes = Storage == IPPI_F64 ? 144 : (Storage == IPPI_F32 ? 72 : 36);
    std::ofstream out(path, std::ios::app);
    out.precision(17);
    auto num = [&](double v) -> std::ostream& {
        if (std::isfinite(v)) out << v;
        else out << "null";
        return out;
    };
    const double q = 0.5 * U * U * D;
    out << "{\"step\": " << t << ", \"mlups\": ";
    num(mlups) << ", \"hbm_gbs\": ";
    num(mlups * bytes * 1e-3) << ", \"mass\": ";
    num(mass) << ", \"cd\": ";
    if (nb > 0 && q > 0) {
        num(f[0] / q) << ", \"cl\": ";
        num(f[1] / q);
    } else {
        out << "null, \"cl\": null";
    }
    out << ", \"max_u\": ";
    num(max_u) << ", \"tau_net_nodes\": " << net << ", \"tau_fallback_nodes\": " << fallback << "}\n";
}

// ---------------------------------------------------------------------------
// sub-steps of the fused GPU step
// ---------------------------------------------------------------------------
void Mesh::fused_only(const char* what, const char* why)
{
    cerr << "Mesh::" << what << ": " << why << "; nothing was changed" << endl;
    errorflag = 1;
}

static const char* kFused =
    "runs inside OneLBMStep, whose one GPU launch pulls the populations, applies the boundary "
    "rules, the immersed-boundary forcing and the collision together, so it cannot run on its own";

void Mesh::Streaming(int RankID, int CoreNum)
{
    (void)RankID;
    (void)CoreNum;
    fused_only("Streaming", kFused);
}
void Mesh::BoundaryCondition(int RankID, int CoreNum)
{
    (void)RankID;
    (void)CoreNum;
    fused_only("BoundaryCondition", kFused);
}
void Mesh::SpreadForce(int RankID, int CoreNum, int Nx_P)
{
    (void)RankID;
    (void)CoreNum;
    (void)Nx_P;
    fused_only("SpreadForce", kFused);
}
void Mesh::UpdateVelocity(int RankID, int CoreNum)
{
    (void)RankID;
    (void)CoreNum;
    fused_only("UpdateVelocity", kFused);
}
void Mesh::XflowBoundary(int t)
{
    (void)t;
    fused_only("XflowBoundary",
               "it overwrites the stored rho and u of non-fluid nodes, which the GPU step does not keep "
               "(every step derives them from the populations)");
}

// ---------------------------------------------------------------------------
// read-side IB and LES steps on the mirror
// ---------------------------------------------------------------------------
// Mesh::DiracDelta (mesh.cpp:1354-1385): Peskin's 4-point kernel
REAL Mesh::DiracDelta(REAL x)
{
    const double a = std::fabs((double)x);
    if (a < 1.0) return (REAL)((3.0 - 2.0 * a + std::sqrt(1.0 + 4.0 * a - 4.0 * a * a)) / 8.0);
    if (a < 2.0) return (REAL)((5.0 - 2.0 * a - std::sqrt(-7.0 + 12.0 * a - 4.0 * a * a)) / 8.0);
    return (REAL)0;
}
REAL Mesh::DiracDeltaD2Q9(REAL x, REAL y) { return DiracDelta(x) * DiracDelta(y); }
REAL Mesh::GetDis2D(REAL x1, REAL y1, REAL x2, REAL y2)
{
    const double dx = (double)x2 - x1, dy = (double)y2 - y1;
    return (REAL)std::sqrt(dx * dx + dy * dy);
}
double Mesh::ComputeDistance(double x0, double y0, double x1, double y1)
{
    const double dx = x1 - x0, dy = y1 - y0;
    const double ex = x0 - center.x, ey = y0 - center.y;
    const double len = std::sqrt(dx * dx + dy * dy);
    if (len == 0.0) return std::sqrt(ex * ex + ey * ey);
    return std::fabs(dx * ey - dy * ex) / len;
}
void Mesh::FilterLBM(int i, int j)
{
    (void)i;
    (void)j;
}
bool Mesh::isAvailable(int i, int j)
{
    if (LatMesh.empty() || i < 0 || i >= (int)LatMesh.size() || j < 0 || j >= (int)LatMesh[0].size()) return false;
    return LatMesh[i][j].style != 's';
}

// Mesh::InterpolateVel (mesh.cpp:552-655) for one rank: markers outside
// [x of column 1, x of the last halo column) get 0; the stencil around
// column (int)x + 1, row (int)y is 4 x 4 with Peskin's kernel or 2 x 2
// bilinear
void Mesh::InterpolateVel(int RankID, int CoreNum, int Nx_P)
{
    (void)RankID;
    (void)CoreNum;
    (void)Nx_P;
    if (!h_ || LatMesh.empty()) return;
    ensure_synced();
    const int NX = (int)LatMesh.size(), NY = (int)LatMesh[0].size();
    for (Particlenode& P : IBParticle) {
        P.vel_ref = {0, 0};
        if (P.position.x < LatMesh[1][0].pos.x || P.position.x >= LatMesh[NX - 1][0].pos.x) continue;
        const int xi = (int)P.position.x + 1, yi = (int)P.position.y;
        const bool peskin = DeltaKernel == IPPI_DELTA_PESKIN4;
        const int lo = peskin ? -1 : 0, hi = peskin ? 2 : 1;
        for (int X = xi + lo; X <= xi + hi; X++)
            for (int Y = yi + lo; Y <= yi + hi; Y++) {
                if (X < 0 || X >= NX || Y < 0 || Y >= NY) continue;
                const Lattice& L = LatMesh[X][Y];
                const REAL dx = P.position.x - L.pos.x, dy = P.position.y - L.pos.y;
                const REAL w = peskin ? DiracDeltaD2Q9(dx, dy) : (REAL)((1 - std::fabs(dx)) * (1 - std::fabs(dy)));
                P.vel_ref.x += L.u.x * w;
                P.vel_ref.y += L.u.y * w;
            }
    }
}

// Mesh::CalParticleForce (mesh.cpp:514-531, direct forcing): F = 2 (U_b - U*),
// without the area factor, as the reference
void Mesh::CalParticleForce(int Radius)
{
    (void)Radius;
    for (Particlenode& P : IBParticle) {
        P.force.x = 2 * (P.vel.x - P.vel_ref.x);
        P.force.y = 2 * (P.vel.y - P.vel_ref.y);
    }
}

// Mesh::CaculateLESTau's active closure (SmagorinskyByHybrid, mesh.cpp
// 852-911) for node (i, j) of the mirror: Pi = sum e e (fnew - feq),
// S = -3 / (2 rho tau0) Pi, Q = sqrt(2 S:S),
// tau = (sqrt(tau0^2 + 18 Cs^2 Q / rho) + tau0) / 2 with tau0 = startTau
void Mesh::CaculateLESTau(int i, int j, REAL Cs, REAL Pr, int RankID, int CoreNum)
{
    (void)Pr;
    (void)RankID;
    (void)CoreNum;
    if (!h_ || !isAvailable(i, j)) return;
    if (!synced_f_) Sync(true);
    Lattice& L = LatMesh[i][j];
    const double rho = L.rho, ux = L.u.x, uy = L.u.y;
    static const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    static const double w[9] = {4. / 9, 1. / 9, 1. / 9, 1. / 9, 1. / 9, 1. / 36, 1. / 36, 1. / 36, 1. / 36};
    double pxx = 0, pxy = 0, pyy = 0;
    for (int k = 0; k < 9; k++) {
        const double eu = ex[k] * ux + ey[k] * uy;
        const double feq = w[k] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * (ux * ux + uy * uy));
        const double d = (double)L.fnew[k] - feq;
        pxx += ex[k] * ex[k] * d;
        pxy += ex[k] * ey[k] * d;
        pyy += ey[k] * ey[k] * d;
    }
    const double tau0 = startTau > 0 ? startTau : (double)L.TauAtBeginning;
    const double c = -3.0 / (2.0 * rho * tau0);
    const double sxx = c * pxx, sxy = c * pxy, syy = c * pyy;
    const double q = std::sqrt(2.0 * (sxx * sxx + 2.0 * sxy * sxy + syy * syy));
    L.tau = (REAL)((std::sqrt(tau0 * tau0 + 18.0 * (double)Cs * Cs * q / rho) + tau0) / 2.0);
}

// Mesh::UpdateBoundary (mesh.cpp:1527-1534): each marker moves by its
// interpolated velocity; the GPU step takes the new positions
void Mesh::UpdateBoundary()
{
    if (IBParticle.empty()) return;
    const int n = (int)IBParticle.size();
    std::vector<double> xy(2 * (size_t)n), ub(2 * (size_t)n);
    for (int m = 0; m < n; m++) {
        Particlenode& P = IBParticle[m];
        P.position.x += P.vel_ref.x;
        P.position.y += P.vel_ref.y;
        xy[2 * m] = P.position.x;
        xy[2 * m + 1] = P.position.y;
        ub[2 * m] = P.vel.x;
        ub[2 * m + 1] = P.vel.y;
    }
    if (h_)
        check(ippi_set_markers(h_, n, xy.data(), ub.data(), nullptr,
                               marker_ds_.size() == (size_t)n ? marker_ds_.data() : nullptr),
              "ippi_set_markers");
}

// ---------------------------------------------------------------------------
// boundary nets: evaluated inside every step once loaded
// ---------------------------------------------------------------------------
int Mesh::nn_model(int type)
{
    if (!h_ || !net_loaded_[type]) {
        cerr << "Mesh::NNmodel_Type0" << type << ": net AutoT0" << type
             << " has no weights (LoadBandNet); its nodes use the Smagorinsky tau" << endl;
        return -1;
    }
    Sync(false);  // tau and NNflag the next collision uses, nets included
    return 0;
}
int Mesh::NNmodel_Type00(int t) { (void)t; return nn_model(0); }
int Mesh::NNmodel_Type01(int t) { (void)t; return nn_model(1); }
int Mesh::NNmodel_Type02(int t) { (void)t; return nn_model(2); }
int Mesh::NNmodel_Type03(int t) { (void)t; return nn_model(3); }
int Mesh::NNmodel_Type04(int t) { (void)t; return nn_model(4); }
int Mesh::NNmodel_Type05(int t) { (void)t; return nn_model(5); }
int Mesh::NNmodel_Type06(int t) { (void)t; return nn_model(6); }
int Mesh::NNmodel_Type07(int t) { (void)t; return nn_model(7); }
