// Compile check of the C++ adapter for gradient recovery: the reference's
// spelling LocalSmoothingGradient<Physics>(feSystem) followed by
// feSystem.getSolutionGradient() (include/assembly/LocalSmoothingGradient.hpp:20-94).
#include "yafel_gpu/yafel_gpu.hpp"

using namespace yafel::gpu;

Vector<double> smoothed_gradient(FESystem &feSystem) {
    LocalSmoothingGradient<PoissonEquation<2>>(feSystem);
    return feSystem.getSolutionGradient().download();
}
