// xflow.h -- the XFlow point-cloud exports the reference imports
// (Mesh::ManageDataFromXflow / ReadXflowdata, mesh.cpp:2189-2547).
//
// One CSV per step, a header line, then one line per point with at least 14
// comma-separated fields: id, x, y, z, VelocityModule, StaticPressure, (skip),
// TotalPressure, (skip), viscosity, ux, uy, uz, and one more separator.  The
// reader keeps the reference's rules:
//   * a line that does not parse that way is skipped;
//   * x, y are rounded to 1e-3 m, then x -> (x + 0.4) / DX and y -> y / DX
//     (DX = 1e-3 m per lattice unit); velocities -> v / 340.112 / sqrt(3);
//     TotalPressure -> (StaticPressure + 101325) / 101325 (a density);
//   * points with the same (x, y) are merged: each later one is averaged into
//     the running value, (kept + new) / 2, field by field;
//   * points outside the rank's x range are dropped.
// The merged points keep the order of their first appearance (the reference
// lists them in unordered_map order; every point lands on its own node, so
// the order changes nothing).
#ifndef IPPI_XFLOW_H
#define IPPI_XFLOW_H

#include <string>
#include <vector>

// the reference's record (mesh.h:20-32): vx, vy, vz hold the position
struct PointData {
    double VelocityModule = 0;
    double StaticPress = 0;
    double TotalPressure = 0;
    double viscosity = 0;
    double ux = 0, uy = 0, uz = 0;
    double vx = 0, vy = 0, vz = 0;
};

namespace ippi_host {
constexpr double kXflowDX = 0.001;      // m per lattice unit (mesh.cpp:2271)
constexpr double kXflowSound = 340.112;  // m/s (mesh.cpp:2272)

// parse, convert and merge one file; false when it cannot be opened
bool read_xflow_csv(const std::string& path, std::vector<PointData>& out);
// keep the points of rank `rank` of `ncore` slabs of `parallel_size`
// columns, nx_total columns in all (mesh.cpp:2348-2360)
void clip_xflow(std::vector<PointData>& pts, int rank, int ncore, int parallel_size, int nx_total);
// the node (x, y) a point lands on: |vx - x| < DX and |vy - y| < DX
bool xflow_node(const PointData& p, int nx, int ny, int* x, int* y);
}  // namespace ippi_host

#endif
