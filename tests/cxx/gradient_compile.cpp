// Compile check of the C++ adapters for the post-solve steps, in the
// reference's spellings: LocalSmoothingGradient<Physics>(feSystem) and
// ZZGradientRecovery<Physics>(feSystem) followed by feSystem.getSolutionGradient()
// (include/assembly/LocalSmoothingGradient.hpp:20-94, ZZGradientRecovery.hpp:33-140),
// SimulationOutput(name, BackendType::VTU).captureFrame(feSystem)
// (include/output/SimulationOutput.hpp:22-116) and Mesh(fname) of a Gmsh file.
#include "yafel_gpu/yafel_gpu.hpp"

using namespace yafel::gpu;

Vector<double> smoothed_gradient(FESystem &feSystem) {
    LocalSmoothingGradient<PoissonEquation<2>>(feSystem);
    return feSystem.getSolutionGradient().download();
}

Vector<double> zz_gradient(FESystem &feSystem) {
    ZZGradientRecovery<PoissonEquation<3>>(feSystem);
    return feSystem.getSolutionGradient().download();
}

void write_output(FESystem &feSystem) {
    SimulationOutput out("solution", BackendType::VTU);
    out.captureFrame(feSystem);
}

int read_mesh_cells(const std::string &fname) { return read_gmsh(fname).nCells(); }
