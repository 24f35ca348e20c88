// ref_heat_harness.cu -- runs the REFERENCE's own MPMWorkpieceSolver kernels,
// unmodified: its grid heat diffusion alone, and its whole step.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file with the
// reference sources where they lie into oracle/_ref/libmpm_ref.so, next to
// ref_harness.cu.  mpmDiffuseTemperatureKernel lives in an unnamed namespace of
// src/MPMWorkpieceSolver.cu, so this translation unit includes that file and
// launches the kernels directly.
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

// nsteps steps of MPMWorkpieceSolver::step (src/MPMWorkpieceSolver.cu:727-781)
// launched kernel by kernel on the fixed grid of p (the solver's own grid
// rebuild from the particle bounds every 25 steps and its compaction are
// host-side domain management and are not run): clearMPMGridKernel,
// mpmP2GKernel, mpmGridUpdateKernel with the tool samples at the pose of the
// step (p0 + v t + offset), mpmDiffuseTemperatureKernel when k / (rho cp) > 0,
// mpmG2PKernel, and chipFractureAndSeparationKernel on even step counts with
// the tool tip at pose + tool_tip_dz.  The material constants are filled as
// MPMWorkpieceSolver::initialize fills them (:422-452).  s->extf (or zero) is
// the particles' force MPMParticleGPU::f.  Particles in and out by state.
int ref_ws_run(const orc_params* p, const orc_ws_params* wp, orc_state* s, const orc_tool_samples* tool, double dt,
               int nsteps, int64_t step0, double t0, double* contact_force) {
    using namespace edgepredict;
    const int n = s->n;
    std::vector<MPMParticleGPU> h((size_t)n);
    for (int i = 0; i < n; ++i) {
        MPMParticleGPU& q = h[i];
        q.x = s->x[i]; q.y = s->y[i]; q.z = s->z[i];
        q.vx = s->vx[i]; q.vy = s->vy[i]; q.vz = s->vz[i];
        q.fx = s->extf ? s->extf[3 * i] : 0.0;
        q.fy = s->extf ? s->extf[3 * i + 1] : 0.0;
        q.fz = s->extf ? s->extf[3 * i + 2] : 0.0;
        q.mass = s->mass[i];
        q.volume = s->vol[i];
        q.density = s->mass[i] / s->vol[i];
        q.temperature = s->T[i];
        q.plasticStrain = s->eps[i];
        q.strainRate = s->edot[i];
        q.damage = s->D[i];
        q.residualStress = s->sres[i];
        const double* sg = s->sig + 6 * (int64_t)i;
        const double* bs = s->bs + 6 * (int64_t)i;
        q.stress_xx = sg[0]; q.stress_yy = sg[1]; q.stress_zz = sg[2];
        q.stress_xy = sg[3]; q.stress_xz = sg[4]; q.stress_yz = sg[5];
        q.backstress_xx = bs[0]; q.backstress_yy = bs[1]; q.backstress_zz = bs[2];
        q.backstress_xy = bs[3]; q.backstress_xz = bs[4]; q.backstress_yz = bs[5];
        q.id = s->id[i];
        q.status = static_cast<ParticleStatus>(s->status[i]);
    }
    MPMGridParams gp;
    gp.cellSize = p->dx;
    gp.minX = p->ox; gp.minY = p->oy; gp.minZ = p->oz;
    gp.nx = p->nx; gp.ny = p->ny; gp.nz = p->nz;
    MPMMaterialParams mat;
    mat.density = p->rho_phys;
    mat.young = p->E;
    mat.poisson = p->nu;
    mat.shear = mat.young / (2.0 * (1.0 + mat.poisson));
    mat.bulk = mat.young / (3.0 * (1.0 - 2.0 * mat.poisson));
    mat.specificHeat = p->cp;
    mat.meltTemp = p->Tm;
    mat.refTemp = p->Tamb;
    mat.jcA = p->A; mat.jcB = p->B; mat.jcN = p->n; mat.jcC = p->C; mat.jcM = p->m;
    mat.refStrainRate = p->edot0;
    mat.failureStrain = wp->failure_strain;
    mat.damageThreshold = p->Dth;
    mat.criticalPlasticStrain = wp->critical_plastic_strain;
    mat.thermalChipRatio = wp->thermal_chip_ratio;
    mat.toolContactRadius = wp->tool_contact_radius;
    mat.contactDamping = wp->contact_damping;
    mat.maxContactTempRise = wp->max_contact_temp_rise;
    mat.thermalConductivity = p->thermal_conductivity;
    mat.kinematicHardeningModulus = p->Hkin;
    mat.thermalClampEnabled = wp->thermal_clamp;
    const int64_t nn = (int64_t)gp.nx * gp.ny * gp.nz;
    const int ns = tool ? tool->n : 0;
    MPMParticleGPU* d = nullptr;
    MPMGridNodeGPU* dg = nullptr;
    Vec3* dsm = nullptr;
    double* dforce = nullptr;
    std::vector<Vec3> smp((size_t)(ns > 0 ? ns : 1));
    cudaError_t e = cudaMalloc(&d, sizeof(MPMParticleGPU) * (size_t)(n > 0 ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&dg, sizeof(MPMGridNodeGPU) * (size_t)(nn > 0 ? nn : 1));
    if (e == cudaSuccess) e = cudaMalloc(&dsm, sizeof(Vec3) * smp.size());
    if (e == cudaSuccess) e = cudaMalloc(&dforce, sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), sizeof(MPMParticleGPU) * (size_t)n, cudaMemcpyHostToDevice);
    const int block = 256;
    const int pGrid = (n + block - 1) / block, nGrid = (int)((nn + block - 1) / block);
    const double alpha = (p->cp > 0.0) ? p->thermal_conductivity / (p->rho_phys * p->cp) : 0.0;
    for (int k = 0; k < nsteps && e == cudaSuccess; ++k) {
        const double t = t0 + (double)k * dt;
        const double pr[3] = {p->tool_p0[0] + p->tool_v[0] * t, p->tool_p0[1] + p->tool_v[1] * t,
                              p->tool_p0[2] + p->tool_v[2] * t};
        for (int q = 0; q < ns; ++q) smp[q] = Vec3(pr[0] + tool->ox[q], pr[1] + tool->oy[q], pr[2] + tool->oz[q]);
        if (ns > 0) e = cudaMemcpy(dsm, smp.data(), sizeof(Vec3) * (size_t)ns, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) break;
        clearMPMGridKernel<<<nGrid, block>>>(dg, (int)nn);
        if (n > 0) mpmP2GKernel<<<pGrid, block>>>(d, n, dg, gp);
        cudaMemset(dforce, 0, sizeof(double));
        mpmGridUpdateKernel<<<nGrid, block>>>(dg, (int)nn, ns > 0 ? dsm : nullptr, ns, gp, mat, p->fixture_thickness,
                                              dt, dforce);
        if (alpha > 0.0) mpmDiffuseTemperatureKernel<<<nGrid, block>>>(dg, (int)nn, gp, alpha, dt);
        if (n > 0) mpmG2PKernel<<<pGrid, block>>>(d, n, dg, gp, mat, dt);
        if (((step0 + k) % 2) == 0 && n > 0)
            chipFractureAndSeparationKernel<<<pGrid, block>>>(d, n, pr[0], pr[1], pr[2] + p->tool_tip_dz, gp.cellSize,
                                                              mat.damageThreshold, mat.criticalPlasticStrain);
        e = cudaDeviceSynchronize();
    }
    double fsum = 0.0;
    if (e == cudaSuccess) e = cudaMemcpy(&fsum, dforce, sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, sizeof(MPMParticleGPU) * (size_t)n, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (dg) cudaFree(dg);
    if (dsm) cudaFree(dsm);
    if (dforce) cudaFree(dforce);
    if (e != cudaSuccess) {
        snprintf(g_heat_err, sizeof(g_heat_err), "ref_ws_run: %s", cudaGetErrorString(e));
        return -1;
    }
    if (contact_force) *contact_force = fsum;
    for (int i = 0; i < n; ++i) {
        const MPMParticleGPU& q = h[i];
        s->x[i] = q.x; s->y[i] = q.y; s->z[i] = q.z;
        s->vx[i] = q.vx; s->vy[i] = q.vy; s->vz[i] = q.vz;
        if (s->extf) { s->extf[3 * i] = q.fx; s->extf[3 * i + 1] = q.fy; s->extf[3 * i + 2] = q.fz; }
        s->T[i] = q.temperature;
        s->eps[i] = q.plasticStrain;
        s->edot[i] = q.strainRate;
        s->D[i] = q.damage;
        s->sres[i] = q.residualStress;
        double* sg = s->sig + 6 * (int64_t)i;
        double* bs = s->bs + 6 * (int64_t)i;
        sg[0] = q.stress_xx; sg[1] = q.stress_yy; sg[2] = q.stress_zz;
        sg[3] = q.stress_xy; sg[4] = q.stress_xz; sg[5] = q.stress_yz;
        bs[0] = q.backstress_xx; bs[1] = q.backstress_yy; bs[2] = q.backstress_zz;
        bs[3] = q.backstress_xy; bs[4] = q.backstress_xz; bs[5] = q.backstress_yz;
        s->status[i] = static_cast<int32_t>(q.status);
    }
    return 0;
}

}  // extern "C"
