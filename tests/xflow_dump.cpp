// Test harness: the host XFlow reader's merged, clipped points, one per
// line with every field at full precision, and the node each lands on.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "xflow.h"

int main(int argc, char** argv)
{
    if (argc != 4) return 2;
    const int nx = std::atoi(argv[2]), ny = std::atoi(argv[3]);
    std::vector<PointData> pts;
    if (!ippi_host::read_xflow_csv(argv[1], pts)) return 1;
    ippi_host::clip_xflow(pts, 0, 1, nx, nx);
    for (const PointData& p : pts) {
        int x = -1, y = -1;
        if (!ippi_host::xflow_node(p, nx, ny, &x, &y)) x = y = -1;
        std::printf("%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %d\n", p.vx, p.vy, p.vz,
                    p.VelocityModule, p.StaticPress, p.TotalPressure, p.viscosity, p.ux, p.uy, p.uz, x, y);
    }
    return 0;
}
