// Test harness: the host Mesh's XFlow methods on a small channel under the
// tau-field model.  ChangeTauFromXflow(1) before the first step, two steps,
// FindAndWriteTau at node (x, y) for step 2 (the targets of step 3), one more
// step, then the fluid file of step 3.
//   xflow_mesh DIR OFFSET NX NY X Y
#include <cstdlib>
#include <iostream>

#include "mesh.h"

int main(int argc, char** argv)
{
    if (argc != 7) return 2;
    const int nx = std::atoi(argv[3]), ny = std::atoi(argv[4]), x = std::atoi(argv[5]), y = std::atoi(argv[6]);
    Mesh mesh;
    mesh.XflowDir = argv[1];
    mesh.XflowStepOffset = std::atoi(argv[2]);
    mesh.BoundarySet = IPPI_BC_CHANNEL;
    mesh.LesModel = IPPI_LES_FIELD;
    mesh.Collision = IPPI_BGK;
    mesh.Storage = IPPI_F64;
    mesh.startTau = 0.76;
    mesh.startU = {0.05, 0};
    mesh.StartCs = 0.1;
    mesh.LatmeshSizeNx = nx;
    mesh.LatmeshSizeNy = ny;
    mesh.InitialFile();
    mesh.InitialLatMesh(nx, ny, 0.76, Point2D{0.05, 0}, 1.0, 0, 1, 0);
    mesh.JudgeStyle(mesh.center, 0, 0, 1);
    mesh.ChangeTauFromXflow(1);
    mesh.RunSteps(1, 2);
    mesh.FindAndWriteTau(x + 1, y, 2);
    mesh.RunSteps(3, 1);
    mesh.WriteDatFluid(3, 0, nx, 1);
    mesh.MergeDatFluid(3, 1);
    return mesh.errorflag;
}
