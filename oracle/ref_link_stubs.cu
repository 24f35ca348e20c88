// ref_link_stubs.cu -- link-only definitions for the reference harness.
//
// TEST INFRASTRUCTURE ONLY.  The harness compiles the reference's
// src/ContactSolver.cu to launch its xpbdContactSDFKernel.  That translation
// unit also refers to methods of other reference classes (the voxel SDF
// builder, whose source does not compile with this toolchain, the spatial
// hash, the FEM solver and the coating model) from ContactSolver members the
// harness never calls.  These definitions only satisfy the linker: each stops
// the process if it is ever reached.
#include <cstdio>
#include <cstdlib>

#include "FEMSolver.cuh"
#include "SharedSpatialHash.h"
#include "ToolCoatingModel.cuh"
#include "ToolSDF.h"

namespace {
[[noreturn]] void unreachable(const char* what) {
    std::fprintf(stderr, "reference harness: %s is not part of the harness\n", what);
    std::abort();
}
}  // namespace

namespace edgepredict {

ToolSDF::~ToolSDF() {}
bool ToolSDF::build(const std::vector<FEMNode>&, const std::vector<Triangle>&, double, int) {
    unreachable("ToolSDF::build");
}
bool ToolSDF::rebuild(const std::vector<Vec3>&, const std::vector<Triangle>&, double, int) {
    unreachable("ToolSDF::rebuild");
}
void ToolSDF::setToolTransform(float, float, float, float, float) { unreachable("ToolSDF::setToolTransform"); }

SharedSpatialHash::~SharedSpatialHash() {}
void SharedSpatialHash::build(FEMNodeGPU*, int, const HashConfig&, cudaStream_t) {
    unreachable("SharedSpatialHash::build");
}
void SharedSpatialHash::scatterResults(FEMNodeGPU*, cudaStream_t) { unreachable("SharedSpatialHash::scatterResults"); }

std::vector<FEMNodeGPU> FEMSolver::getNodes() { unreachable("FEMSolver::getNodes"); }

void ToolCoatingModel::updateWear(int, double, double, double, WearZone, double) {
    unreachable("ToolCoatingModel::updateWear");
}
double ToolCoatingModel::getWearDepth(int) const { unreachable("ToolCoatingModel::getWearDepth"); }
double ToolCoatingModel::getCraterWear(int) const { unreachable("ToolCoatingModel::getCraterWear"); }
double ToolCoatingModel::getFlankWear(int) const { unreachable("ToolCoatingModel::getFlankWear"); }
bool ToolCoatingModel::isSubstrateExposed(int) const { unreachable("ToolCoatingModel::isSubstrateExposed"); }

}  // namespace edgepredict
