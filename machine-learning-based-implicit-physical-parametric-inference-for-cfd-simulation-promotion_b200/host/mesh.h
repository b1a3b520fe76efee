// mesh.h -- the reference's Mesh class (IPPI-LBM/mesh.h:32-114) as a host
// object over the B200 time step (include/ippi_lbm.h).
//
// Same public fields and the same call sequence as the reference's driver
// (main.cpp): set the fields, InitialLatMesh, JudgeStyle, optionally
// InitialIBParticle, then OneLBMStep / ComputeAvgVelocity every step and
// WriteDatFluid + MergeDatFluid every SaveStep steps.  Differences:
//   * one GPU holds the whole lattice: RankID / CoreNum are accepted and
//     must be 0 / 1 (no MPI slabs, no halo exchange);
//   * the node state lives on the GPU; LatMesh is its host mirror, refreshed
//     by Sync() and by the methods that read it;
//   * ComputeAvgVelocity is fused into the step (the averages start at
//     startAvg) and only refreshes nothing on the host;
//   * RunSteps(t0, n) advances n steps in one call (CUDA graphs, one
//     synchronisation) for drivers that need no per-step host work;
//   * a diverged run (ErrorCatch: rho outside [0, 10]) prints the reference's
//     message and sets errorflag; with AbortOnError (default) it exits like
//     the reference's MPI_Abort.
#pragma once
#ifndef MESH_H
#define MESH_H
#define _USE_MATH_DEFINES
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "NodeAndLattice.h"
#include "xflow.h"

class Mesh {
public:
    Mesh();
    ~Mesh();
    Mesh(const Mesh&) = delete;
    Mesh& operator=(const Mesh&) = delete;

    vector<Particlenode> IBParticle;
    vector<vector<Lattice>> LatMesh;  // [NX = Nx + 2][Ny], halo columns 0 and NX - 1
    int LatmeshSizeNx = 0;
    int LatmeshSizeNy = 0;
    Point2D center{0, 0};
    double radius = 0;
    const double eps = 1.0e-9;
    double startTau = 0;
    Point2D startU{0, 0};
    int MyrankID = 0;
    int MyCoreNum = 1;
    int stepH = 0, stepL = 0;
    int startAvg = 0;
    double StartCs = 0;
    int errorflag = 0;
    int ParallelSize = 0;

    // settings with no field in the reference (Parameter.h gives the defaults)
    int BoundarySet = IPPI_BC_REF_NEE;  // IPPI_BC_CHANNEL: Zou-He inlet, walls
    int Collision = ippi_host::kCollision;
    int Storage = ippi_host::kStorage;
    int LesModel = ippi_host::kLes;
    int DeltaKernel = ippi_host::kDelta;
    int MdfIters = 1;
    int PlateX0 = 400;  // flat plate: specular bottom for x < PlateX0 (mesh.cpp:1413)
    int Device = 0;
    bool AbortOnError = true;
    std::string XflowDir = "Xflowdata_pingban_every_1_step";  // mesh.cpp:2197
    int XflowStepOffset = 10014;                               // mesh.cpp:2192

    // ---- the reference's API ------------------------------------------
    void InitialLatMesh(int Nx_P, int Ny, double tau, Point2D StartVel, double Rho, int RankID,
                        int CoreNum, int PartitionRemainderFlag);
    void InitialIBParticle(int NumNodes, double Radius, double ParticlePositionX,
                           double ParticlePositionY, Point2D ParticleVel);
    void JudgeStyle(Point2D CylinderCenter1, REAL Radius, int RankID, int CoreNum);
    void OneLBMStep(int RankID, int CoreNum, REAL Cs, REAL Pr, int t);
    void ComputeAvgVelocity(int t);
    void ErrorCatch(int i, int j);
    void InitialFile();
    void WriteDatFluid(int t, int RankID, int NX, int CoreNum);
    void MergeDatFluid(int t, int CoreNum);
    void WriteAvgu(int t, int RankID, int NX, int CoreNum);
    void MergeAvgu(int t, int CoreNum);
    void WriteDatParticle(int t);
    void GetSt(int t);
    void OutputCd(int RankID, int CoreNum, int time, double Radius);
    void OutputCp(int RankID, int CoreNum, int time, double Radius);
    void MergeCp(int t, int CoreNum);
    void ComputeCp(int startcp, int t);
    // velocity-gradient helpers and the closures' per-node inputs on the
    // mirror (mesh.cpp:1659-1953, 2113-2146); SetNormalDis also hands the
    // distances to the wall-damped closure (IPPI_LES_DYNAMIC)
    double GetDuxDx(int i, int j);
    double GetDuxDy(int i, int j);
    double GetDuyDx(int i, int j);
    double GetDuyDy(int i, int j);
    void SetNormalDis();
    double ComputeDynamicCs(int i, int j);
    // XFlow coupling (mesh.cpp:2189-2766); files XflowDir/pb_<t + XflowStepOffset>.csv
    vector<PointData> ReadXflowdata(int t);
    void ManageDataFromXflow(int t);
    void XflowABS(int t);
    void FindAndWriteTau(int i, int j, int t);
    void ChangeTauFromXflow(int t);
    // The step's sub-steps (mesh.cpp:192-356, 656-832, 1244-1281, 2548-2584).
    // OneLBMStep performs them in one fused launch on the GPU, so they cannot
    // run on their own: each prints why on stderr, sets errorflag and
    // changes nothing.
    void Streaming(int RankID, int CoreNum);
    void BoundaryCondition(int RankID, int CoreNum);
    void SpreadForce(int RankID, int CoreNum, int Nx_P);
    void UpdateVelocity(int RankID, int CoreNum);
    void XflowBoundary(int t);
    // Read-side IB and LES steps on the host mirror (the GPU step runs its
    // own each step): InterpolateVel fills IBParticle[m].vel_ref from the
    // current velocity field (Peskin 4-point or bilinear, as DeltaKernel),
    // CalParticleForce sets IBParticle[m].force = 2 (vel - vel_ref), and
    // CaculateLESTau sets LatMesh[i][j].tau to the Smagorinsky tau of the
    // node's populations with the given Cs (mesh.cpp:514-655, 852-911)
    void InterpolateVel(int RankID, int CoreNum, int Nx_P);
    void CalParticleForce(int Radius);
    void CaculateLESTau(int i, int j, REAL Cs, REAL Pr, int RankID, int CoreNum);
    // moves each marker by its vel_ref and hands the new positions to the
    // GPU step (mesh.cpp:1527-1534)
    void UpdateBoundary();
    // the Peskin 4-point kernel phi(x) and phi(x) phi(y) (mesh.cpp:1354-1389)
    REAL DiracDelta(REAL x);
    REAL DiracDeltaD2Q9(REAL x, REAL y);
    REAL GetDis2D(REAL x1, REAL y1, REAL x2, REAL y2);
    // distance from `center` to the line through (x0, y0) and (x1, y1); the
    // reference's body (mesh.cpp:1536-1550) is unfinished and returns nothing
    double ComputeDistance(double x0, double y0, double x1, double y1);
    void FilterLBM(int i, int j);  // empty in the reference (mesh.cpp:2166-2169)
    bool isAvailable(int i, int j);
    // The boundary nets run inside every OneLBMStep once their weights are
    // loaded (LoadBandNet).  NNmodel_Type0<n>(t) refreshes LatMesh's tau and
    // NNflag from the GPU (the values the next collision uses) and returns
    // 0, or returns -1 with a message when net n has no weights.
    int NNmodel_Type00(int t);
    int NNmodel_Type01(int t);
    int NNmodel_Type02(int t);
    int NNmodel_Type03(int t);
    int NNmodel_Type04(int t);
    int NNmodel_Type05(int t);
    int NNmodel_Type06(int t);
    int NNmodel_Type07(int t);

    // ---- additions ----------------------------------------------------
    // JudgeStyle marks the nodes within Radius of CylinderCenter1 as solid
    // ('s', halfway bounce-back; their fluid neighbours become 'b'), the
    // cylinder OutputCd / OutputCp read (channel scene)
    bool SolidCylinder = false;
    // solid nodes from a mask solid[Ny][Nx] (NULL removes them)
    bool SetSolid(const unsigned char* solid);
    // initial macroscopic fields rho/ux/uy[Ny][Nx] (NULL: rho 1, u 0)
    void SetInitialField(const double* rho, const double* ux, const double* uy);
    // boundary net weights (NNmodel/AutoT0<type>.pt in TorchScript order)
    bool LoadBandNet(int type, const float* w, size_t n);
    // n steps numbered t0 .. t0 + n - 1
    void RunSteps(int t0, int n);
    // refresh LatMesh from the device (populations too when with_f)
    void Sync(bool with_f = false);
    // per-body force of the last step (FP64); returns the body count
    int BodyForces(double* fxy, int max_bodies);
    // drag / lift coefficients -sum(F) / (0.5 U^2 D) of body 0
    void DragLift(double U, double D, double* cd, double* cl);
    // one line "t Fx Fy Cd Cl" appended to particle/forces.dat
    void OutputForces(int t, double U, double D);
    // checkpoint of the device state written to `path` (ippi_save_state,
    // through a temporary file renamed over it); false on error
    bool SaveCheckpoint(const std::string& path);
    // resume from a checkpoint file (ippi_load_state) into a mesh set up as
    // the saving one was; returns the last step it holds, -1 on error
    int LoadCheckpoint(const std::string& path);
    // one JSON line appended to `path`: step, MLUPS and HBM GB/s of the
    // steps since the previous line, FP64 mass, Cd / Cl of body 0 (U, D;
    // null without markers), max |u|, and the learned tau's network /
    // fallback node counts (ippi_diagnostics)
    void LogMetrics(const std::string& path, int t, double mlups, double U, double D);
    ippi_lbm* Handle() { return h_; }

private:
    ippi_lbm* h_ = nullptr;
    int nx_ = 0, ny_ = 0;
    bool synced_ = false;
    int last_t_ = 0;
    std::vector<double> init_rho_, init_ux_, init_uy_;
    int cp_start_ = -1;
    std::vector<double> tau_field_;  // the tau-field model's tau[Ny][Nx]
    std::vector<double> marker_ds_;  // arc length per marker (ippi_set_markers)
    bool net_loaded_[8] = {};
    bool synced_f_ = false;           // LatMesh fnew is current too
    double cs_ = -1;                  // Smagorinsky constant on the device
    void fused_only(const char* what, const char* why);
    int nn_model(int type);
    void reequilibrate_mirror();
    void set_tau_node(int x, int y, double tau);
    void upload_tau_field();
    bool check(int rc, const char* what);
    void ensure_synced();
};
#endif
