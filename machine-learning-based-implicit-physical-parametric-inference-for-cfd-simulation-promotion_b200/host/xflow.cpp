// xflow.cpp -- reader of the XFlow point-cloud exports (see xflow.h).
#include "xflow.h"

#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <utility>

namespace ippi_host {

namespace {
// one data line (mesh.cpp:2222-2236): every number followed by one
// separator character, the same extraction rules as the reference's stream
bool parse_line(const std::string& line, PointData& p)
{
    std::istringstream ss(line);
    double skip = 0;
    char sep = 0;
    double* fields[13] = {&skip,         &p.vx, &p.vy, &p.vz, &p.VelocityModule, &p.StaticPress, &skip,
                          &p.TotalPressure, &skip, &p.viscosity, &p.ux, &p.uy, &p.uz};
    for (double* f : fields)
        if (!(ss >> *f >> sep)) return false;
    return true;
}

void average_into(PointData& kept, const PointData& p)
{
    // mesh.cpp:2301-2321: sum, then halve
    kept.VelocityModule = (kept.VelocityModule + p.VelocityModule) / 2.0;
    kept.StaticPress = (kept.StaticPress + p.StaticPress) / 2.0;
    kept.TotalPressure = (kept.TotalPressure + p.TotalPressure) / 2.0;
    kept.ux = (kept.ux + p.ux) / 2.0;
    kept.uy = (kept.uy + p.uy) / 2.0;
    kept.uz = (kept.uz + p.uz) / 2.0;
    kept.vz = (kept.vz + p.vz) / 2.0;
    kept.viscosity = (kept.viscosity + p.viscosity) / 2.0;
}
}  // namespace

bool read_xflow_csv(const std::string& path, std::vector<PointData>& out)
{
    out.clear();
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    std::getline(in, line);  // header
    std::map<std::pair<double, double>, size_t> seen;
    while (std::getline(in, line)) {
        PointData p;
        if (!parse_line(line, p)) continue;
        // RoundToThreeDecimalPlaces (mesh.cpp:41-46), then lattice units
        // (mesh.cpp:2274-2287)
        p.vx = std::round(p.vx * 1000.0) / 1000.0;
        p.vy = std::round(p.vy * 1000.0) / 1000.0;
        p.vx = (p.vx + 0.4) / kXflowDX;
        p.vy = p.vy / kXflowDX;
        p.vz = p.vz / kXflowDX;
        p.VelocityModule = p.VelocityModule / kXflowSound / std::sqrt(3.0);
        p.ux = p.ux / kXflowSound / std::sqrt(3.0);
        p.uy = p.uy / kXflowSound / std::sqrt(3.0);
        p.uz = p.uz / kXflowSound / std::sqrt(3.0);
        p.TotalPressure = (p.StaticPress + 101325) / 101325;
        const auto key = std::make_pair(p.vx, p.vy);
        auto it = seen.find(key);
        if (it == seen.end()) {
            seen.emplace(key, out.size());
            out.push_back(p);
        } else {
            average_into(out[it->second], p);
        }
    }
    return true;
}

void clip_xflow(std::vector<PointData>& pts, int rank, int ncore, int parallel_size, int nx_total)
{
    int lo = rank * parallel_size;
    int hi = (rank + 1) * parallel_size + 2;
    if (rank == ncore - 1) hi = nx_total;
    if (rank == 0) lo -= 2;
    std::vector<PointData> keep;
    keep.reserve(pts.size());
    for (const PointData& p : pts)
        if (!(p.vx < lo - 0.5 || p.vx > hi + 0.5)) keep.push_back(p);
    pts.swap(keep);
}

bool xflow_node(const PointData& p, int nx, int ny, int* x, int* y)
{
    const double rx = std::nearbyint(p.vx), ry = std::nearbyint(p.vy);
    if (!(std::fabs(p.vx - rx) < kXflowDX && std::fabs(p.vy - ry) < kXflowDX)) return false;
    if (rx < 0 || rx > nx - 1 || ry < 0 || ry > ny - 1) return false;
    *x = (int)rx;
    *y = (int)ry;
    return true;
}

}  // namespace ippi_host
