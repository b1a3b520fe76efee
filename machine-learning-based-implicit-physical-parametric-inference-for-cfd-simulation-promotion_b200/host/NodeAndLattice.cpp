// NodeAndLattice.cpp -- host-side helpers of the node mirror.
#include "NodeAndLattice.h"

namespace {
const int kE[9][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
const double kW[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
}  // namespace

// Lattice::CalMacro (NodeAndLattice.cpp:196-227): moments of fnew, u = 0 when
// rho < 1e-6, p = rho / 3
void Lattice::CalMacro()
{
    double r = 0, mx = 0, my = 0;
    for (int k = 0; k < 9; k++) {
        r += fnew[k];
        mx += fnew[k] * kE[k][0];
        my += fnew[k] * kE[k][1];
    }
    rho = (REAL)r;
    if (r < 1e-6) {
        u = {0, 0};
    } else {
        u.x = (REAL)(mx / r);
        u.y = (REAL)(my / r);
    }
    p = (REAL)(r / 3.0);
}

// second-order equilibrium w_k rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u.u)
void Lattice::Compute_feq()
{
    feq.resize(9);
    const double uu = 1 - 1.5 * ((double)u.x * u.x + (double)u.y * u.y);
    for (int k = 0; k < 9; k++) {
        const double eu = kE[k][0] * (double)u.x + kE[k][1] * (double)u.y;
        feq[k] = (REAL)(kW[k] * rho * (uu + 3.0 * eu + 4.5 * eu * eu));
    }
}

void Lattice::InitialLatticeFeq()
{
    Compute_feq();
    fnew = feq;
    fcol = feq;
}
