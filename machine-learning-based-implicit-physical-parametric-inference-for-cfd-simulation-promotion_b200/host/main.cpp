// main.cpp -- the driver of IPPI-LBM/main.cpp over the GPU Mesh: the same
// settings (main.cpp:12-65), the same call sequence (InitialLatMesh,
// JudgeStyle, OneLBMStep + ComputeAvgVelocity every step, WriteDatFluid +
// MergeDatFluid every SaveStep steps) and the same output files, on one GPU
// (RankID 0, CoreNum 1).  The reference's constants are the defaults; the
// options below override them.
//
//   ippi_main [--scene plate|channel] [--nx N] [--ny N] [--steps N]
//             [--save N] [--avg N] [--re R] [--u U] [--cs C]
//             [--cylinder X Y D] [--markers N] [--solid] [--cp START]
//             [--nets DIR] [--init FILE] [--batched] [--print N] [--device N]
//             [--xflow DIR] [--xflow-offset N] [--xflow-init] [--xflow-abs N]
//             [--les none|smagorinsky|wale|csm|dynamic]
//             [--checkpoint FILE] [--resume FILE] [--metrics FILE]
//
//   plate    the reference's scene: flat plate, NEE inlet u = --u, Re 5e5,
//            tau = 0.5 + 6 (Ny U / Re) (main.cpp:37-43)
//   channel  Zou-He parabolic inlet (u_max = --u), NEE outlet, bounce-back
//            walls; with --cylinder an IB cylinder of diameter D,
//            nu = U D / Re, tau = 3 nu + 1/2; its body force goes to
//            particle/forces.dat every step
//   --solid        the cylinder as solid nodes (halfway bounce-back) instead
//                  of IB markers; Mesh::OutputCd's momentum-exchange Cd / Cl
//                  go to particle/CD_CL.dat every step (every save point
//                  with --batched)
//   --cp START     with --solid: surface pressure coefficient averaged from
//                  step START (= --avg) to cp/cp_Merged_<t>.dat at save points
//   --nets DIR     boundary nets AutoT0<k>.f32 (raw float32 TorchScript
//                  parameters) for the plate scene
//   --init FILE    initial rho, ux, uy as 3 x Ny x Nx float64 (raw)
//   --batched      advance between save points in one call (CUDA graphs)
//                  instead of one OneLBMStep call per step
//   --les NAME     the relaxation-time closure (default: Parameter.h's);
//                  wale / csm / dynamic are the alternatives the reference
//                  keeps in Mesh::CaculateLESTau (channel scene); dynamic
//                  damps Cs with the distance to the --cylinder surface
//                  (Mesh::SetNormalDis)
//   --xflow DIR    XFlow exports DIR/pb_<t + offset>.csv (offset 10014, or
//                  --xflow-offset); --xflow-init: Mesh::ManageDataFromXflow
//                  after step 1; --xflow-abs N: Mesh::XflowABS every N steps
//                  (the coupling blocks of the reference's main.cpp:132-156)
//   --checkpoint FILE  the device state (Mesh::SaveCheckpoint) at every save
//                  point and after the last step
//   --resume FILE  continue from such a checkpoint, set up with the same
//                  options, at the step after the one it holds
//   --metrics FILE a JSON line (Mesh::LogMetrics) at every --print step
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "mesh.h"

using namespace std;

namespace {

struct Options {
    string scene = "plate";
    int nx = 2401, ny = 501;
    int steps = 200000, save = 20000, avg = 30000;
    double re = 5e5, u = 0.1, cs = 0.173;
    bool cylinder = false;
    double cx = 0, cy = 0, d = 0;
    int markers = 0;
    bool solid = false;
    int cp = -1;
    string xflow;
    int xflow_offset = 10014;
    bool xflow_init = false;
    int xflow_abs = 0;
    int les = -1;
    string nets, init;
    string checkpoint, resume, metrics;
    bool batched = false;
    int print = 1;
    int device = 0;
};

bool parse(int argc, char** argv, Options& o)
{
    for (int i = 1; i < argc; i++) {
        string a = argv[i];
        auto need = [&](int n) {
            if (i + n >= argc) {
                cerr << a << " needs " << n << " value(s)" << endl;
                return false;
            }
            return true;
        };
        if (a == "--scene" && need(1)) o.scene = argv[++i];
        else if (a == "--nx" && need(1)) o.nx = atoi(argv[++i]);
        else if (a == "--ny" && need(1)) o.ny = atoi(argv[++i]);
        else if (a == "--steps" && need(1)) o.steps = atoi(argv[++i]);
        else if (a == "--save" && need(1)) o.save = atoi(argv[++i]);
        else if (a == "--avg" && need(1)) o.avg = atoi(argv[++i]);
        else if (a == "--re" && need(1)) o.re = atof(argv[++i]);
        else if (a == "--u" && need(1)) o.u = atof(argv[++i]);
        else if (a == "--cs" && need(1)) o.cs = atof(argv[++i]);
        else if (a == "--cylinder" && need(3)) {
            o.cylinder = true;
            o.cx = atof(argv[++i]);
            o.cy = atof(argv[++i]);
            o.d = atof(argv[++i]);
        } else if (a == "--markers" && need(1)) o.markers = atoi(argv[++i]);
        else if (a == "--solid") o.solid = true;
        else if (a == "--xflow" && need(1)) o.xflow = argv[++i];
        else if (a == "--xflow-offset" && need(1)) o.xflow_offset = atoi(argv[++i]);
        else if (a == "--xflow-init") o.xflow_init = true;
        else if (a == "--xflow-abs" && need(1)) o.xflow_abs = atoi(argv[++i]);
        else if (a == "--les" && need(1)) {
            const string m = argv[++i];
            o.les = m == "none" ? IPPI_LES_NONE : m == "smagorinsky" ? IPPI_LES_SMAGORINSKY
                    : m == "wale" ? IPPI_LES_WALE : m == "csm" ? IPPI_LES_CSM
                    : m == "dynamic" ? IPPI_LES_DYNAMIC : -2;
            if (o.les == -2) return false;
        }
        else if (a == "--cp" && need(1)) o.cp = atoi(argv[++i]);
        else if (a == "--checkpoint" && need(1)) o.checkpoint = argv[++i];
        else if (a == "--resume" && need(1)) o.resume = argv[++i];
        else if (a == "--metrics" && need(1)) o.metrics = argv[++i];
        else if (a == "--nets" && need(1)) o.nets = argv[++i];
        else if (a == "--init" && need(1)) o.init = argv[++i];
        else if (a == "--batched") o.batched = true;
        else if (a == "--print" && need(1)) o.print = atoi(argv[++i]);
        else if (a == "--device" && need(1)) o.device = atoi(argv[++i]);
        else if (a == "--help" || a == "-h") return false;
        else {
            cerr << "unknown option " << a << endl;
            return false;
        }
    }
    return o.scene == "plate" || o.scene == "channel";
}

bool read_floats(const string& path, vector<float>& w)
{
    ifstream in(path, ios::binary | ios::ate);
    if (!in) return false;
    const streamsize n = in.tellg();
    w.resize((size_t)n / sizeof(float));
    in.seekg(0);
    return bool(in.read(reinterpret_cast<char*>(w.data()), n));
}

}  // namespace

int main(int argc, char* argv[])
{
    Options o;
    if (!parse(argc, argv, o)) {
        cerr << "usage: ippi_main [--scene plate|channel] [--nx N] [--ny N] [--steps N] [--save N]\n"
                "                 [--avg N] [--re R] [--u U] [--cs C] [--cylinder X Y D] [--markers N]\n"
                "                 [--solid] [--cp START] [--nets DIR] [--init FILE] [--batched]\n"
                "                 [--print N] [--device N] [--xflow DIR] [--xflow-offset N]\n"
                "                 [--xflow-init] [--xflow-abs N] [--les none|smagorinsky|wale|csm|dynamic]\n"
                "                 [--checkpoint FILE] [--resume FILE] [--metrics FILE]"
             << endl;
        return 2;
    }
    const int RankID = 0, CoreNum = 1;
    REAL Cs = (REAL)o.cs;
    REAL Pr = 1;
    const int Nx = o.nx, Ny = o.ny;
    Point2D StartVel{(REAL)o.u, 0};
    const REAL Rho = 1.0;
    const bool channel = o.scene == "channel";
    // main.cpp:43 for the plate; 3 nu + 1/2 with nu = U D / Re for the cylinder
    const double tau = channel && o.cylinder ? 3.0 * (o.u * o.d / o.re) + 0.5
                                             : 0.5 + 6.0 * ((Ny * StartVel.x) / o.re);

    Mesh mesh;
    mesh.startAvg = o.avg;
    mesh.center = {(REAL)o.cx, (REAL)o.cy};
    mesh.radius = o.d / 2;
    mesh.startTau = tau;
    mesh.startU = StartVel;
    mesh.MyrankID = RankID;
    mesh.MyCoreNum = CoreNum;
    mesh.StartCs = Cs;
    mesh.LatmeshSizeNx = Nx;
    mesh.LatmeshSizeNy = Ny;
    mesh.Device = o.device;
    if (o.les >= 0) mesh.LesModel = o.les;
    if (!o.xflow.empty()) mesh.XflowDir = o.xflow;
    mesh.XflowStepOffset = o.xflow_offset;
    if (channel) {
        mesh.BoundarySet = IPPI_BC_CHANNEL;
        mesh.DeltaKernel = IPPI_DELTA_PESKIN4;
    }
    mesh.InitialFile();

    mesh.InitialLatMesh(Nx, Ny, tau, StartVel, Rho, RankID, CoreNum, 0);
    const bool solid = channel && o.cylinder && o.solid;
    mesh.SolidCylinder = solid;
    mesh.JudgeStyle(mesh.center, (REAL)mesh.radius, RankID, CoreNum);
    if (mesh.LesModel == IPPI_LES_DYNAMIC) mesh.SetNormalDis();
    if (!o.init.empty()) {
        vector<double> m(3 * (size_t)Nx * Ny);
        ifstream in(o.init, ios::binary);
        if (!in.read(reinterpret_cast<char*>(m.data()), m.size() * sizeof(double))) {
            cerr << "cannot read " << o.init << endl;
            return 1;
        }
        const size_t nn = (size_t)Nx * Ny;
        mesh.SetInitialField(m.data(), m.data() + nn, m.data() + 2 * nn);
    }
    if (channel && o.cylinder && !solid) {
        const int n = o.markers > 0 ? o.markers : (int)std::ceil(M_PI * o.d);
        mesh.InitialIBParticle(n, o.d / 2, o.cx, o.cy, Point2D{0, 0});
        mesh.WriteDatParticle(0);
    }
    if (!o.nets.empty())
        for (int k : {1, 3, 5, 7}) {
            vector<float> w;
            const string path = o.nets + "/AutoT0" + to_string(k) + ".f32";
            if (read_floats(path, w)) mesh.LoadBandNet(k, w.data(), w.size());
            else cerr << "no net " << path << " (type " << k << " keeps Smagorinsky)" << endl;
        }

    cout << "=====================" << endl;
    cout << "L = " << Nx << " x " << Ny << endl;
    cout << "U = " << StartVel.x << endl;
    cout << "Re = " << o.re << endl;
    cout << "Tau = " << tau << endl;
    cout << endl;
    cout << "Start Computing" << endl;

    const bool forces = channel && o.cylinder && !solid;
    int first = 1;
    if (!o.resume.empty()) {
        const int last = mesh.LoadCheckpoint(o.resume);
        if (last < 0) return 1;
        first = last + 1;
        cout << "Resumed at step " << first << " from " << o.resume << endl;
    }
    auto t_mark = std::chrono::steady_clock::now();
    int s_mark = first - 1;
    for (int t = first; t <= o.steps;) {
        int n = 1;
        if (o.batched) {
            // up to the next save point
            n = o.save > 0 ? std::min(o.steps - t + 1, o.save - (t - 1) % o.save) : o.steps - t + 1;
            // stop where a coupling hook runs
            if (o.xflow_init && t == 1) n = 1;
            if (o.xflow_abs > 0) n = std::min(n, o.xflow_abs - (t - 1) % o.xflow_abs);
            mesh.RunSteps(t, n);
            if (solid) mesh.OutputCd(RankID, CoreNum, t + n - 1, mesh.radius);
            if (forces) {
                vector<double> hist(2 * (size_t)n);
                const int got = ippi_force_history(mesh.Handle(), hist.data(), n);
                ofstream out("particle/forces.dat", ios::app);
                out.precision(12);
                const double q = 0.5 * o.u * o.u * o.d;
                for (int s = 0; s < got; s++)
                    out << t + n - got + s << " " << hist[2 * s] << " " << hist[2 * s + 1] << " "
                        << hist[2 * s] / q << " " << hist[2 * s + 1] / q << "\n";
            }
        } else {
            mesh.OneLBMStep(RankID, CoreNum, Cs, Pr, t);
            if (forces) mesh.OutputForces(t, o.u, o.d);
            if (solid) mesh.OutputCd(RankID, CoreNum, t, mesh.radius);
        }
        t += n;
        const int last = t - 1;
        if (o.xflow_init && last == 1) mesh.ManageDataFromXflow(last);
        if (o.xflow_abs > 0 && last % o.xflow_abs == 0) mesh.XflowABS(last);
        if (solid && o.cp >= 0) mesh.ComputeCp(o.cp, last);
        if (o.save > 0 && last % o.save == 0) {
            mesh.WriteDatFluid(last, RankID, Nx, CoreNum);
            mesh.MergeDatFluid(last, CoreNum);
            if (solid && o.cp >= 0) {
                mesh.OutputCp(RankID, CoreNum, last, mesh.radius);
                mesh.MergeCp(last, CoreNum);
            }
        }
        mesh.ComputeAvgVelocity(last);
        const bool report = o.print > 0 && (last % o.print == 0 || last == o.steps);
        if (report) cout << "Compute Step:" << " " << last << endl;
        if (!o.metrics.empty() && report) {
            const auto now = std::chrono::steady_clock::now();
            const double sec = std::chrono::duration<double>(now - t_mark).count();
            const double mlups = sec > 0 ? (double)Nx * Ny * (last - s_mark) / sec * 1e-6 : 0.0;
            mesh.LogMetrics(o.metrics, last, mlups, o.u, o.d);
            t_mark = std::chrono::steady_clock::now();
            s_mark = last;
        }
        if (!o.checkpoint.empty() && ((o.save > 0 && last % o.save == 0) || last == o.steps) &&
            !mesh.SaveCheckpoint(o.checkpoint))
            return 1;
    }
    return mesh.errorflag;
}
