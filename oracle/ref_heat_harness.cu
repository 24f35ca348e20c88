// ref_heat_harness.cu -- runs the REFERENCE's own grid heat diffusion kernel,
// unmodified.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file with the
// reference sources where they lie into oracle/_ref/libmpm_ref.so, next to
// ref_harness.cu.  mpmDiffuseTemperatureKernel lives in an unnamed namespace of
// src/MPMWorkpieceSolver.cu, so this translation unit includes that file and
// launches the kernel on a grid built from node masses and T m.
#include "src/MPMWorkpieceSolver.cu"

#include <cstdint>
#include <cstdio>
#include <vector>

#include "mpm_oracle.h"

namespace {
char g_heat_err[256] = {0};
}

extern "C" {

const char* ref_heat_last_error(void) { return g_heat_err; }

// One launch of mpmDiffuseTemperatureKernel (src/MPMWorkpieceSolver.cu:208-262)
// over an nx*ny*nz grid (x fastest) with the given node masses and T m, with
// alpha = k / (rho_phys cp) as MPMWorkpieceSolver::step computes it (:751-752).
// tm is overwritten with the kernel's temperatureMass.
int ref_heat_diffuse(const orc_params* p, const double* mass, double* tm, double dt) {
    using namespace edgepredict;
    const int64_t nn = (int64_t)p->nx * p->ny * p->nz;
    std::vector<MPMGridNodeGPU> h((size_t)nn);
    for (int64_t i = 0; i < nn; ++i) {
        h[i].mass = mass[i];
        h[i].temperatureMass = tm[i];
    }
    MPMGridParams gp;
    gp.cellSize = p->dx;
    gp.minX = p->ox; gp.minY = p->oy; gp.minZ = p->oz;
    gp.nx = p->nx; gp.ny = p->ny; gp.nz = p->nz;
    const double alpha = p->thermal_conductivity / (p->rho_phys * p->cp);
    MPMGridNodeGPU* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(MPMGridNodeGPU) * (size_t)(nn > 0 ? nn : 1));
    if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), sizeof(MPMGridNodeGPU) * (size_t)nn, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nn > 0) {
        const int block = 256;
        mpmDiffuseTemperatureKernel<<<(int)((nn + block - 1) / block), block>>>(d, (int)nn, gp, alpha, dt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, sizeof(MPMGridNodeGPU) * (size_t)nn, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        snprintf(g_heat_err, sizeof(g_heat_err), "ref_heat_diffuse: %s", cudaGetErrorString(e));
        return -1;
    }
    for (int64_t i = 0; i < nn; ++i) tm[i] = h[i].temperatureMass;
    return 0;
}

}  // extern "C"
