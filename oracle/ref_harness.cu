// ref_harness.cu -- runs the REFERENCE's own MPM kernels, unmodified.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference sources where they lie (include path = the reference root) into
// oracle/_ref/libmpm_ref.so.  Nothing here is part of the product library.
//
// The reference solver class cannot express the benchmark grids: its domain is
// hard-wired to a 0.2 m cube and dx >= 0.5 mm (src/MPMSolver.cu:840-846), and
// its step graph captures host stack scalars (:1073-1075).  So this harness
// includes the reference translation unit and launches its kernels directly,
// in the order that MPMSolver::step captures them (src/MPMSolver.cu:1092-1164):
//   lodClassify? -> resetGrid -> p2g -> updateGrid -> fixtureBC? ->
//   (rasterizeTool -> applyGridCollision)? -> g2p -> (detectShearBands ->
//   applyAdiabaticHeating)? -> bounds -> resetExtForce, then
//   chipFractureAndSeparation on even steps.
#include "src/MPMSolver.cu"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mpm_oracle.h"

using namespace edgepredict;

namespace {

char g_err[512] = {0};

#define HCHECK(call)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            snprintf(g_err, sizeof(g_err), "%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                     cudaGetErrorString(e_));                                                     \
            return -1;                                                                            \
        }                                                                                         \
    } while (0)

// The reference kernels hard-code these; a run whose parameters differ is not
// a run of the reference and is refused.
int check_reference_constants(const orc_params* p) {
    if (p->mass_threshold != 1e-12 || p->gravity_z != -9.81 || p->apic_dinv_factor != 3.0 ||
        p->apic_decay != 0.99 || p->deps_cap != 0.05 || p->dT_cap != 50.0 ||
        p->plasticity_mode != ORC_PLAST_EXPLICIT || p->chip_every != 2 ||
        (p->tool_mode != ORC_TOOL_NONE && p->tool_mode != ORC_TOOL_RASTER) ||
        p->fixture_damping != 1e7) {
        snprintf(g_err, sizeof(g_err), "parameters outside what the reference kernels implement");
        return -2;
    }
    // applyAdiabaticHeatingKernel compares the absolute temperature with 25.5
    // (src/AdiabaticShearModel.cu:123)
    if (p->asb_enabled && p->Tamb + p->asb_touch_rise != 25.5) {
        snprintf(g_err, sizeof(g_err), "the reference's shear model needs Tamb + touch rise = 25.5");
        return -2;
    }
    return 0;
}

// AdiabaticShearModel::initialize (src/AdiabaticShearModel.cu:229-241) with
// the solver's material.
ShearBandParams make_shear_params(const orc_params* p) {
    ShearBandParams b;
    b.criticalStrainRate = p->asb_critical_rate;
    b.softeningThreshold = 0.95;
    b.taylorQuinney = p->asb_taylor_quinney;
    b.thermalDiffusivity = 2.9e-6;
    b.bandWidth = 20e-6;
    b.maxTempRatio = p->asb_max_temp_ratio;
    b.meltingTemp = p->Tm;
    b.specificHeat = p->cp;
    b.density = p->rho_phys;
    return b;
}

MPMKernelConfig make_config(const orc_params* p) {
    MPMKernelConfig c;
    c.dx = p->dx;
    c.invDx = 1.0 / p->dx;
    c.youngsModulus = p->E;
    c.poissonsRatio = p->nu;
    c.density = p->rho_phys;
    c.physicalDensity = p->rho_phys;
    c.specificHeat = p->cp;
    c.taylorQuinney = p->beta;
    c.meltingPoint = p->Tm;
    c.ambientTemp = p->Tamb;
    c.jc_A = p->A; c.jc_B = p->B; c.jc_n = p->n; c.jc_C = p->C; c.jc_m = p->m;
    c.kinematicHardeningModulus = p->Hkin;
    c.jc_D1 = p->D1; c.jc_D2 = p->D2; c.jc_D3 = p->D3; c.jc_D4 = p->D4; c.jc_D5 = p->D5;
    c.damageThreshold = p->Dth;
    c.referenceStrainRate = p->edot0;
    c.lodActiveRadius = p->lod_active_r;
    c.lodNearRadius = p->lod_near_r;
    return c;
}

void soa_to_aos(const orc_state* s, std::vector<MPMParticle>& a) {
    a.resize(s->n);
    for (int i = 0; i < s->n; ++i) {
        MPMParticle& q = a[i];
        q.x = s->x[i]; q.y = s->y[i]; q.z = s->z[i];
        q.vx = s->vx[i]; q.vy = s->vy[i]; q.vz = s->vz[i];
        if (s->extf) { q.ext_fx = s->extf[3 * i]; q.ext_fy = s->extf[3 * i + 1]; q.ext_fz = s->extf[3 * i + 2]; }
        q.mass = s->mass[i]; q.volume = s->vol[i]; q.temperature = s->T[i];
        for (int k = 0; k < 9; ++k) { q.F[k] = s->F[9 * i + k]; q.F_p[k] = s->Fp[9 * i + k]; q.C[k] = s->C[9 * i + k]; }
        const double* sg = s->sig + 6 * i;
        q.stress_xx = sg[0]; q.stress_yy = sg[1]; q.stress_zz = sg[2];
        q.stress_xy = sg[3]; q.stress_xz = sg[4]; q.stress_yz = sg[5];
        const double* b = s->bs + 6 * i;
        q.backstress_xx = b[0]; q.backstress_yy = b[1]; q.backstress_zz = b[2];
        q.backstress_xy = b[3]; q.backstress_xz = b[4]; q.backstress_yz = b[5];
        q.plasticStrain = s->eps[i]; q.strainRate = s->edot[i]; q.damage = s->D[i]; q.residualStress = s->sres[i];
        q.id = s->id[i];
        q.status = static_cast<ParticleStatus>(s->status[i]);
        q.lodZone = static_cast<LODZone>(s->lod ? s->lod[i] : 0);
        q.asbCounter = static_cast<uint8_t>(s->asb ? s->asb[i] : 0);
    }
}

void aos_to_soa(const std::vector<MPMParticle>& a, orc_state* s) {
    for (int i = 0; i < s->n; ++i) {
        const MPMParticle& q = a[i];
        s->x[i] = q.x; s->y[i] = q.y; s->z[i] = q.z;
        s->vx[i] = q.vx; s->vy[i] = q.vy; s->vz[i] = q.vz;
        if (s->extf) { s->extf[3 * i] = q.ext_fx; s->extf[3 * i + 1] = q.ext_fy; s->extf[3 * i + 2] = q.ext_fz; }
        s->T[i] = q.temperature;
        for (int k = 0; k < 9; ++k) { s->F[9 * i + k] = q.F[k]; s->Fp[9 * i + k] = q.F_p[k]; s->C[9 * i + k] = q.C[k]; }
        double* sg = s->sig + 6 * i;
        sg[0] = q.stress_xx; sg[1] = q.stress_yy; sg[2] = q.stress_zz;
        sg[3] = q.stress_xy; sg[4] = q.stress_xz; sg[5] = q.stress_yz;
        double* b = s->bs + 6 * i;
        b[0] = q.backstress_xx; b[1] = q.backstress_yy; b[2] = q.backstress_zz;
        b[3] = q.backstress_xy; b[4] = q.backstress_xz; b[5] = q.backstress_yz;
        s->eps[i] = q.plasticStrain; s->edot[i] = q.strainRate; s->D[i] = q.damage; s->sres[i] = q.residualStress;
        s->status[i] = static_cast<int32_t>(q.status);
        if (s->lod) s->lod[i] = static_cast<int32_t>(q.lodZone);
        if (s->asb) s->asb[i] = static_cast<int32_t>(q.asbCounter);
    }
}

// Device-side handle for one reference run.
struct RefRun {
    MPMParticle* d_p = nullptr;
    MPMGridNode* d_g = nullptr;
    FEMNodeGPU* d_tool = nullptr;
    FEMNodeGPU* d_tool_start = nullptr;
    FEMNodeGPU* d_tool_end = nullptr;
    double* d_bmin = nullptr;
    double* d_bmax = nullptr;
    int n = 0, ntool = 0;
    int64_t nn = 0;
    cudaStream_t st = nullptr;
    ~RefRun() {
        if (d_p) cudaFree(d_p);
        if (d_g) cudaFree(d_g);
        if (d_tool) cudaFree(d_tool);
        if (d_tool_start) cudaFree(d_tool_start);
        if (d_tool_end) cudaFree(d_tool_end);
        if (d_bmin) cudaFree(d_bmin);
        if (d_bmax) cudaFree(d_bmax);
        if (st) cudaStreamDestroy(st);
    }
};

// One reference step on stream st, in the captured order.  Tool nodes must
// already hold this step's positions.
void launch_step(RefRun& r, const orc_params* p, const MPMKernelConfig& cfg, double dt, int64_t counter,
                 const double tip[3], const double* hBmin, const double* hBmax) {
    int3 dims = make_int3(p->nx, p->ny, p->nz);
    Vec3 dmin(p->ox, p->oy, p->oz);
    const int T = 256;
    const int gb = (int)((r.nn + T - 1) / T);
    const int pb = (r.n + T - 1) / T;
    if (p->lod_enabled)
        lodClassifyKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, Vec3(tip[0], tip[1], tip[2]), cfg.lodActiveRadius, cfg.lodNearRadius);
    resetGridKernel<<<gb, T, 0, r.st>>>(r.d_g, (int)r.nn);
    p2gKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, r.d_g, dims, cfg, dmin);
    updateGridKernel<<<gb, T, 0, r.st>>>(r.d_g, (int)r.nn, dt);
    if (p->fixture_thickness > 0.0)
        applyFixtureBCKernel<<<gb, T, 0, r.st>>>(r.d_g, dims, p->oz, p->dx, p->fixture_thickness, p->fixture_damping, dt);
    if (r.ntool > 0) {
        rasterizeToolKernel<<<(r.ntool + 255) / 256, 256, 0, r.st>>>(r.d_tool, r.ntool, r.d_g, dims, cfg, dmin);
        applyGridCollisionKernel<<<gb, T, 0, r.st>>>(r.d_g, (int)r.nn, dt);
    }
    g2pKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, r.d_g, dims, cfg, dt, dmin);
    if (p->asb_enabled) {
        // AdiabaticShearModel::update (src/AdiabaticShearModel.cu:262-279)
        const ShearBandParams sb = make_shear_params(p);
        detectShearBandsKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, sb);
        applyAdiabaticHeatingKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, sb, dt);
    }
    cudaMemcpyAsync(r.d_bmin, hBmin, 3 * sizeof(double), cudaMemcpyHostToDevice, r.st);
    cudaMemcpyAsync(r.d_bmax, hBmax, 3 * sizeof(double), cudaMemcpyHostToDevice, r.st);
    updateParticleBoundsKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, r.d_bmin, r.d_bmin + 1, r.d_bmin + 2, r.d_bmax,
                                                  r.d_bmax + 1, r.d_bmax + 2);
    resetExternalForceKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n);
    if (p->chip_sep_enabled && (counter % 2) == 0)
        chipFractureAndSeparationKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, tip[2], p->dx, p->Dth, 1e-6);
}

void fill_tool(const orc_params* p, const orc_tool_samples* tool, double t, std::vector<FEMNodeGPU>& nodes) {
    nodes.resize(tool ? tool->n : 0);
    for (size_t i = 0; i < nodes.size(); ++i) {
        double pr[3];
        for (int d = 0; d < 3; ++d) pr[d] = p->tool_p0[d] + p->tool_v[d] * t;
        nodes[i].x = pr[0] + tool->ox[i];
        nodes[i].y = pr[1] + tool->oy[i];
        nodes[i].z = pr[2] + tool->oz[i];
        nodes[i].vx = p->tool_v[0];
        nodes[i].vy = p->tool_v[1];
        nodes[i].vz = p->tool_v[2];
    }
}

int setup(RefRun& r, const orc_params* p, int n, int ntool) {
    r.n = n;
    r.ntool = ntool;
    r.nn = (int64_t)p->nx * p->ny * p->nz;
    HCHECK(cudaStreamCreateWithFlags(&r.st, cudaStreamNonBlocking));
    HCHECK(cudaMalloc(&r.d_p, sizeof(MPMParticle) * (size_t)(n > 0 ? n : 1)));
    HCHECK(cudaMalloc(&r.d_g, sizeof(MPMGridNode) * (size_t)r.nn));
    HCHECK(cudaMalloc(&r.d_bmin, 3 * sizeof(double)));
    HCHECK(cudaMalloc(&r.d_bmax, 3 * sizeof(double)));
    if (ntool > 0) {
        HCHECK(cudaMalloc(&r.d_tool, sizeof(FEMNodeGPU) * ntool));
        HCHECK(cudaMalloc(&r.d_tool_start, sizeof(FEMNodeGPU) * ntool));
        HCHECK(cudaMalloc(&r.d_tool_end, sizeof(FEMNodeGPU) * ntool));
    }
    return 0;
}

// MPMParticle defaults (its constructor) with the given position, status,
// id, mass, volume and temperature: the state MPMSolver::initializeParticleBox
// writes (src/MPMSolver.cu:1315-1327).
__global__ void fill_particles(MPMParticle* out, const double* x, const double* y, const double* z, const int* status,
                               int n, double mass, double vol, double T0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    MPMParticle p;
    p.x = x[i]; p.y = y[i]; p.z = z[i];
    p.mass = mass; p.volume = vol; p.density = mass / vol; p.temperature = T0;
    p.id = i;
    p.status = static_cast<ParticleStatus>(status[i]);
    out[i] = p;
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err; }

int ref_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int ref_sizeof_particle(void) { return (int)sizeof(MPMParticle); }
int ref_sizeof_gridnode(void) { return (int)sizeof(MPMGridNode); }

// Run nsteps reference steps on the state s (host SoA, updated in place).
// Tool node positions are recomputed on the host each step as
// (p0 + v*t) + offset with t = t0 + k*dt.
int ref_run(const orc_params* p, orc_state* s, const orc_tool_samples* tool, double dt, int nsteps,
            long long step0, double t0) {
    int rc = check_reference_constants(p);
    if (rc) return rc;
    const int ntool = (p->tool_mode == ORC_TOOL_RASTER && tool) ? tool->n : 0;
    RefRun r;
    if ((rc = setup(r, p, s->n, ntool))) return rc;
    std::vector<MPMParticle> h;
    soa_to_aos(s, h);
    HCHECK(cudaMemcpy(r.d_p, h.data(), sizeof(MPMParticle) * (size_t)s->n, cudaMemcpyHostToDevice));
    MPMKernelConfig cfg = make_config(p);
    const double inf = std::numeric_limits<double>::infinity();
    double hBmin[3] = {inf, inf, inf}, hBmax[3] = {-inf, -inf, -inf};
    std::vector<FEMNodeGPU> nodes;
    for (int k = 0; k < nsteps; ++k) {
        const double t = t0 + (double)k * dt;
        double tip[3];
        for (int d = 0; d < 3; ++d) tip[d] = p->tool_p0[d] + p->tool_v[d] * t;
        tip[2] += p->tool_tip_dz;
        if (ntool > 0) {
            fill_tool(p, tool, t, nodes);
            HCHECK(cudaMemcpyAsync(r.d_tool, nodes.data(), sizeof(FEMNodeGPU) * ntool, cudaMemcpyHostToDevice, r.st));
        }
        launch_step(r, p, cfg, dt, step0 + k, tip, hBmin, hBmax);
        HCHECK(cudaStreamSynchronize(r.st));
        HCHECK(cudaGetLastError());
    }
    HCHECK(cudaMemcpy(h.data(), r.d_p, sizeof(MPMParticle) * (size_t)s->n, cudaMemcpyDeviceToHost));
    aos_to_soa(h, s);
    return 0;
}

// Reference-compatible stats through the reference's own kernel
// (computeParticleStatsKernel, src/MPMSolver.cu:729-788): out = {max stress,
// max T, kinetic, "internal"}.
// AdiabaticShearModel::update (src/AdiabaticShearModel.cu:262-279) once over
// the particles of s, with the solver material of p.
int ref_asb_heat(const orc_params* p, orc_state* s, double dt) {
    std::vector<MPMParticle> a;
    soa_to_aos(s, a);
    const int n = s->n;
    MPMParticle* d = nullptr;
    HCHECK(cudaMalloc(&d, sizeof(MPMParticle) * (size_t)(n > 0 ? n : 1)));
    cudaError_t e = cudaMemcpy(d, a.data(), sizeof(MPMParticle) * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) {
        const ShearBandParams sb = make_shear_params(p);
        const int pb = (n + 255) / 256;
        detectShearBandsKernel<<<pb, 256>>>(d, n, sb);
        applyAdiabaticHeatingKernel<<<pb, 256>>>(d, n, sb, dt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(a.data(), d, sizeof(MPMParticle) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "ref_asb_heat: %s", cudaGetErrorString(e));
        return -1;
    }
    aos_to_soa(a, s);
    return 0;
}

int ref_stats(orc_state* s, double out[4]) {
    std::vector<MPMParticle> h;
    soa_to_aos(s, h);
    MPMParticle* d = nullptr;
    double* r = nullptr;
    HCHECK(cudaMalloc(&d, sizeof(MPMParticle) * (size_t)(s->n > 0 ? s->n : 1)));
    HCHECK(cudaMalloc(&r, 4 * sizeof(double)));
    HCHECK(cudaMemcpy(d, h.data(), sizeof(MPMParticle) * (size_t)s->n, cudaMemcpyHostToDevice));
    HCHECK(cudaMemset(r, 0, 4 * sizeof(double)));
    computeParticleStatsKernel<<<(s->n + 255) / 256, 256>>>(d, s->n, r, r + 1, r + 2, r + 3);
    HCHECK(cudaGetLastError());
    HCHECK(cudaMemcpy(out, r, 4 * sizeof(double), cudaMemcpyDeviceToHost));
    cudaFree(d);
    cudaFree(r);
    return 0;
}

// Timed reference run for the benchmark's reference arm: the state is uploaded
// once, then `warmup` untimed and `steps` timed steps run as the reference
// runs them -- the per-step launch sequence captured into one CUDA graph
// (src/MPMSolver.cu:1077-1157), chip separation launched outside the graph on
// even steps, and the tool nodes moved by the reference's own
// interpolateToolNodesKernel (:494-504).  Returns device milliseconds of the
// timed steps in *ms_out and leaves the final state in s.
static int bench_loaded(RefRun& r, const orc_params* p, const orc_tool_samples* tool, double dt, int warmup,
                        int steps, double* ms_out);

int ref_bench(const orc_params* p, orc_state* s, const orc_tool_samples* tool, double dt, int warmup, int steps,
              double* ms_out) {
    int rc = check_reference_constants(p);
    if (rc) return rc;
    const int ntool = (p->tool_mode == ORC_TOOL_RASTER && tool) ? tool->n : 0;
    RefRun r;
    if ((rc = setup(r, p, s->n, ntool))) return rc;
    {
        std::vector<MPMParticle> h;
        soa_to_aos(s, h);
        HCHECK(cudaMemcpy(r.d_p, h.data(), sizeof(MPMParticle) * (size_t)s->n, cudaMemcpyHostToDevice));
    }
    if ((rc = bench_loaded(r, p, tool, dt, warmup, steps, ms_out))) return rc;
    std::vector<MPMParticle> h(s->n);
    HCHECK(cudaMemcpy(h.data(), r.d_p, sizeof(MPMParticle) * (size_t)s->n, cudaMemcpyDeviceToHost));
    aos_to_soa(h, s);
    return 0;
}

// Same timing from particle positions only (large workloads): the AoS array is
// filled on the device.  Returns the count of non-INACTIVE particles at the
// end in *n_live.
int ref_bench_positions(const orc_params* p, const double* x, const double* y, const double* z, const int* status,
                        int n, double mass, double vol, double T0, const orc_tool_samples* tool, double dt,
                        int warmup, int steps, double* ms_out, long long* n_live) {
    int rc = check_reference_constants(p);
    if (rc) return rc;
    const int ntool = (p->tool_mode == ORC_TOOL_RASTER && tool) ? tool->n : 0;
    RefRun r;
    if ((rc = setup(r, p, n, ntool))) return rc;
    double *dx_ = nullptr, *dy_ = nullptr, *dz_ = nullptr;
    int* ds = nullptr;
    HCHECK(cudaMalloc(&dx_, 8 * (size_t)n));
    HCHECK(cudaMalloc(&dy_, 8 * (size_t)n));
    HCHECK(cudaMalloc(&dz_, 8 * (size_t)n));
    HCHECK(cudaMalloc(&ds, 4 * (size_t)n));
    HCHECK(cudaMemcpy(dx_, x, 8 * (size_t)n, cudaMemcpyHostToDevice));
    HCHECK(cudaMemcpy(dy_, y, 8 * (size_t)n, cudaMemcpyHostToDevice));
    HCHECK(cudaMemcpy(dz_, z, 8 * (size_t)n, cudaMemcpyHostToDevice));
    HCHECK(cudaMemcpy(ds, status, 4 * (size_t)n, cudaMemcpyHostToDevice));
    fill_particles<<<(n + 255) / 256, 256>>>(r.d_p, dx_, dy_, dz_, ds, n, mass, vol, T0);
    HCHECK(cudaGetLastError());
    HCHECK(cudaDeviceSynchronize());
    cudaFree(dx_); cudaFree(dy_); cudaFree(dz_); cudaFree(ds);
    if ((rc = bench_loaded(r, p, tool, dt, warmup, steps, ms_out))) return rc;
    int* dcnt = nullptr;
    int active = 0, chip = 0;
    HCHECK(cudaMalloc(&dcnt, 2 * sizeof(int)));
    HCHECK(cudaMemset(dcnt, 0, 2 * sizeof(int)));
    countParticleStatusKernel<<<(n + 255) / 256, 256>>>(r.d_p, n, dcnt, dcnt + 1);
    HCHECK(cudaMemcpy(&active, dcnt, sizeof(int), cudaMemcpyDeviceToHost));
    HCHECK(cudaMemcpy(&chip, dcnt + 1, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(dcnt);
    *n_live = (long long)active + chip;
    return 0;
}

static int bench_loaded(RefRun& r, const orc_params* p, const orc_tool_samples* tool, double dt, int warmup,
                        int steps, double* ms_out) {
    const int ntool = r.ntool;
    const int total = warmup + steps;
    std::vector<FEMNodeGPU> nodes;
    if (ntool > 0) {
        fill_tool(p, tool, 0.0, nodes);
        HCHECK(cudaMemcpy(r.d_tool_start, nodes.data(), sizeof(FEMNodeGPU) * ntool, cudaMemcpyHostToDevice));
        fill_tool(p, tool, dt * total, nodes);
        HCHECK(cudaMemcpy(r.d_tool_end, nodes.data(), sizeof(FEMNodeGPU) * ntool, cudaMemcpyHostToDevice));
    }
    MPMKernelConfig cfg = make_config(p);
    const double inf = std::numeric_limits<double>::infinity();
    // the bounds sentinels that each step copies host->device (the reference
    // copies them from its stack, src/MPMSolver.cu:1073-1075, :1134-1135);
    // pinned here so that the captured copy is valid for the whole run
    double* hB = nullptr;
    HCHECK(cudaMallocHost(&hB, 6 * sizeof(double)));
    double* hBmin = hB;
    double* hBmax = hB + 3;
    for (int d = 0; d < 3; ++d) { hBmin[d] = inf; hBmax[d] = -inf; }
    double tip0[3] = {p->tool_p0[0], p->tool_p0[1], p->tool_p0[2] + p->tool_tip_dz};

    // capture the per-step graph (without chip separation, which the reference
    // launches outside the graph)
    orc_params pg = *p;
    pg.chip_sep_enabled = 0;
    cudaGraph_t graph;
    cudaGraphExec_t exec = nullptr;
    HCHECK(cudaStreamBeginCapture(r.st, cudaStreamCaptureModeThreadLocal));
    launch_step(r, &pg, cfg, dt, 1, tip0, hBmin, hBmax);
    HCHECK(cudaStreamEndCapture(r.st, &graph));
    HCHECK(cudaGraphInstantiate(&exec, graph, nullptr, nullptr, 0));
    cudaGraphDestroy(graph);

    cudaEvent_t e0, e1;
    HCHECK(cudaEventCreate(&e0));
    HCHECK(cudaEventCreate(&e1));
    const int T = 256, pb = (r.n + T - 1) / T;
    for (int k = 0; k < total; ++k) {
        if (k == warmup) HCHECK(cudaEventRecord(e0, r.st));
        if (ntool > 0)
            interpolateToolNodesKernel<<<(ntool + 255) / 256, 256, 0, r.st>>>(r.d_tool, r.d_tool_start, r.d_tool_end,
                                                                           ntool, (double)k / (double)total);
        HCHECK(cudaGraphLaunch(exec, r.st));
        if (p->chip_sep_enabled && (k % 2) == 0) {
            double tz = p->tool_p0[2] + p->tool_v[2] * (dt * k) + p->tool_tip_dz;
            chipFractureAndSeparationKernel<<<pb, T, 0, r.st>>>(r.d_p, r.n, tz, p->dx, p->Dth, 1e-6);
        }
    }
    HCHECK(cudaEventRecord(e1, r.st));
    HCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    HCHECK(cudaEventElapsedTime(&ms, e0, e1));
    *ms_out = ms;
    cudaGraphExecDestroy(exec);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeHost(hB);
    return 0;
}

}  // extern "C"
