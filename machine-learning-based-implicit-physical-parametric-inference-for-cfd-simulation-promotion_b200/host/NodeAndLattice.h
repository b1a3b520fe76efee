// NodeAndLattice.h -- host-side node types (IPPI-LBM/NodeAndLattice.h:9-88).
//
// In the reference every Lattice object holds the live state of its node and
// the solver works on vector<vector<Lattice>>.  Here the live state is on the
// GPU (structure-of-arrays population planes behind ippi_lbm); a Lattice is
// the host mirror of one node, filled by Mesh::Sync() (and by the methods
// that read the mirror: WriteDatFluid, WriteAvgu, GetSt, ErrorCatch).  The
// per-node helpers kept here (CalMacro, Compute_feq, InitialLatticeFeq) act
// on the mirror for post-processing; the collision operators run only on the
// device.
#ifndef NODEANDLATTICE_H
#define NODEANDLATTICE_H

#include <vector>

#include "Point2D.h"

using namespace std;

class Particlenode {
public:
    Point2D position{0, 0};
    Point2D position_ref{0, 0};
    Point2D vel_ref{0, 0};  // velocity interpolated at the marker
    Point2D vel{0, 0};      // prescribed marker velocity
    Point2D force{0, 0};    // marker force of the last step
    Point2D center{0, 0};
    void UpdateParticleBoundary() {}  // markers are fixed (the reference's is empty too)
};

class Lattice {
public:
    Lattice() : feq(9, 0), fcol(9, 0), fnew(9, 0), lat_force(9, 0) {}

    REAL rho = 1;
    Point2D u = {0, 0};
    Position2D pos = {0, 0};
    REAL p = REAL(1.0 / 3.0);
    REAL tau = 0;
    REAL TauAtBeginning = 0;
    Point2D force = {0, 0};
    vector<REAL> feq;
    vector<REAL> fcol;
    vector<REAL> fnew;  // populations after the last step (Mesh::Sync with populations)
    vector<REAL> lat_force;
    double Cs = 0.0;
    double avg_u = 0;
    double avg_v = 0;
    double avg_density = 0;
    double cp = 0;  // time-averaged pressure coefficient ('b' nodes, Mesh::OutputCp)
    // differences to the imported XFlow state (Mesh::ManageDataFromXflow,
    // XflowABS): u - u_xflow, rho - rho_xflow, tau - (3 nu_xflow + 1/2)
    Point2D absU = {0, 0};
    REAL absRHO = 0;
    double xflowtau = 0;
    double abstau = 0;
    double normalDis = 0;   // distance to the cylinder surface (Mesh::SetNormalDis)
    double CoherentCS = 0;  // coherent-structure coefficient (Mesh::ComputeDynamicCs)
    char style = 'f';
    bool NNflag = false;

    // rho, u, p from fnew (Lattice::CalMacro, NodeAndLattice.cpp:196-227)
    void CalMacro();
    // second-order equilibrium of (rho, u) into feq (NodeAndLattice.cpp:124-149)
    void Compute_feq();
    // fnew = fcol = feq(rho, u) (NodeAndLattice.cpp:69-123)
    void InitialLatticeFeq();
};

#endif
