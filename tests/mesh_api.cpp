// Test harness: the Mesh methods of the reference's class that the time step
// fuses or that act on the host mirror (host/mesh.h).
//   mesh_api cpu              helpers and refusals (no GPU call)
//   mesh_api gpu NETDIR       flat plate with net 3: per-call Cs, the
//                             Smagorinsky tau of CaculateLESTau against the
//                             device's, NNmodel_Type0x; channel cylinder:
//                             InterpolateVel / CalParticleForce / UpdateBoundary
// Prints "key value..." lines for the Python side to check.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mesh.h"

static std::vector<float> read_f32(const std::string& path)
{
    std::vector<float> w;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return w;
    float buf[4096];
    size_t r;
    while ((r = std::fread(buf, sizeof(float), 4096, f)) > 0) w.insert(w.end(), buf, buf + r);
    std::fclose(f);
    return w;
}

static int cpu()
{
    Mesh m;
    m.AbortOnError = false;
    for (double x : {0.0, 0.25, 0.5, 1.0, 1.5, 1.999, 2.0, -0.75, -1.25})
        std::printf("delta %.17g %.17g\n", x, (double)m.DiracDelta((REAL)x));
    std::printf("delta2 %.17g\n", (double)m.DiracDeltaD2Q9((REAL)0.3, (REAL)-1.2));
    std::printf("dis %.17g\n", (double)m.GetDis2D(1, 2, 4, 6));
    m.center = {3, 4};
    std::printf("linedist %.17g\n", m.ComputeDistance(0, 0, 10, 0));
    std::printf("pointdist %.17g\n", m.ComputeDistance(0, 0, 0, 0));
    std::printf("available_empty %d\n", (int)m.isAvailable(0, 0));
    m.FilterLBM(1, 1);
    std::printf("errorflag_before %d\n", m.errorflag);
    m.Streaming(0, 1);
    std::printf("errorflag_after %d\n", m.errorflag);
    m.errorflag = 0;
    m.BoundaryCondition(0, 1);
    m.SpreadForce(0, 1, 10);
    m.UpdateVelocity(0, 1);
    m.XflowBoundary(1);
    std::printf("errorflag_all %d\n", m.errorflag);
    std::printf("nn_unloaded %d\n", m.NNmodel_Type03(1));
    return 0;
}

static int gpu(const std::string& netdir)
{
    // flat plate with net 3 (main.cpp's scene, 416 x 24)
    {
        Mesh m;
        m.Storage = IPPI_F64;
        m.Collision = IPPI_BGK;
        m.LesModel = IPPI_LES_SMAGORINSKY;
        m.LatmeshSizeNx = 416;
        m.LatmeshSizeNy = 24;
        m.startTau = 0.52;
        m.StartCs = 0.173;
        m.InitialLatMesh(416, 24, 0.52, Point2D{0.1, 0}, 1.0, 0, 1, 0);
        m.JudgeStyle(Point2D{0, 0}, 0, 0, 1);
        std::vector<float> w = read_f32(netdir + "/AutoT03.f32");
        if (!m.LoadBandNet(3, w.data(), w.size())) return 3;
        for (int t = 1; t <= 6; t++) m.OneLBMStep(0, 1, (REAL)(t <= 3 ? 0.173 : 0.3), 0, t);
        m.Sync(true);
        const int i = 201, j = 10;  // interior column 201 (x = 200), row 10
        std::printf("device_tau %.17g\n", (double)m.LatMesh[i][j].tau);
        m.CaculateLESTau(i, j, (REAL)0.3, 0, 0, 1);
        std::printf("host_tau %.17g\n", (double)m.LatMesh[i][j].tau);
        std::printf("nn03 %d\n", m.NNmodel_Type03(6));
        int flags = 0;
        for (int x = 1; x <= 416; x++) flags += m.LatMesh[x][22].NNflag ? 1 : 0;
        std::printf("nnflags_row22 %d\n", flags);
        m.AbortOnError = false;
        std::printf("nn01 %d\n", m.NNmodel_Type01(6));
    }
    // channel cylinder: markers read back, then moved
    {
        Mesh m;
        m.BoundarySet = IPPI_BC_CHANNEL;
        m.Storage = IPPI_F64;
        m.Collision = IPPI_MRT;
        m.DeltaKernel = IPPI_DELTA_PESKIN4;
        m.LatmeshSizeNx = 160;
        m.LatmeshSizeNy = 48;
        m.startTau = 0.56;
        m.StartCs = 0.1;
        m.InitialLatMesh(160, 48, 0.56, Point2D{0.05, 0}, 1.0, 0, 1, 0);
        m.JudgeStyle(Point2D{0, 0}, 0, 0, 1);
        m.InitialIBParticle(38, 6.0, 40.3, 24.1, Point2D{0, 0});
        for (int t = 1; t <= 20; t++) m.OneLBMStep(0, 1, (REAL)0.1, 0, t);
        m.InterpolateVel(0, 1, 160);
        m.CalParticleForce(6);
        for (int q = 0; q < 38; q += 9)
            std::printf("marker %d %.17g %.17g %.17g %.17g %.17g %.17g\n", q, (double)m.IBParticle[q].position.x,
                        (double)m.IBParticle[q].position.y, (double)m.IBParticle[q].vel_ref.x,
                        (double)m.IBParticle[q].vel_ref.y, (double)m.IBParticle[q].force.x,
                        (double)m.IBParticle[q].force.y);
        // the velocity field the interpolation read
        FILE* f = std::fopen("u_field.txt", "w");
        for (int y = 0; y < 48; y++)
            for (int x = 0; x < 160; x++)
                std::fprintf(f, "%.17g %.17g\n", (double)m.LatMesh[x + 1][y].u.x, (double)m.LatMesh[x + 1][y].u.y);
        std::fclose(f);
        const double x0 = m.IBParticle[0].position.x + m.IBParticle[0].vel_ref.x;
        m.UpdateBoundary();
        std::printf("moved %.17g %.17g\n", (double)m.IBParticle[0].position.x, x0);
        m.OneLBMStep(0, 1, (REAL)0.1, 0, 21);
        std::printf("errorflag %d\n", m.errorflag);
    }
    return 0;
}

int main(int argc, char** argv)
{
    if (argc >= 2 && std::string(argv[1]) == "cpu") return cpu();
    if (argc >= 3 && std::string(argv[1]) == "gpu") return gpu(argv[2]);
    return 2;
}
