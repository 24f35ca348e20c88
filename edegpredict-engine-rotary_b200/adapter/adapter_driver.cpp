// adapter_driver.cpp -- a plain C entry layer over MPMSolverB200, so that the
// GPU tests and bench.py can drive the drop-in adapter the way
// SimulationEngine does (src/SimulationEngine.cpp:495-536): tool pose, the
// blended FEM-node motion, one step() per sub-step, syncMetrics() per macro
// step, and the particle array handed to ContactSolver / CFD.
//
// Built with the adapter inside the reference tree (the reference's headers
// and its src/Config.cpp for initialize(Config)) into
// adapter/_build/libmpm_adapter.so; see build.py --adapter.
#include <cstddef>
#include <cstring>
#include <string>

#include "Config.h"
#include "MPMSolverB200.h"

using edgepredict::FEMNodeGPU;
using edgepredict::MPMParticle;
using edgepredict::MPMSolverB200;
using edgepredict::Vec3;

namespace {
MPMSolverB200* S(void* a) { return static_cast<MPMSolverB200*>(a); }
thread_local std::string g_err;
}  // namespace

extern "C" {

void* mad_create(int max_particles) { return new MPMSolverB200(max_particles); }

void mad_destroy(void* a) { delete S(a); }

int mad_status(void* a) { return (int)S(a)->lastStatus(); }

const char* mad_error(void* a) {
    g_err = S(a)->lastError();
    return g_err.c_str();
}

// Config::loadFromString + setPrecision + initialize (src/main.cpp:307-330).
int mad_initialize_json(void* a, const char* json, int precision) {
    edgepredict::Config c;
    try {
        c.loadFromString(json ? json : "{}");
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
    S(a)->setPrecision(precision);
    return S(a)->initialize(c) ? 0 : -1;
}

int mad_initialize_params(void* a, const mpm_params* p) { return p && S(a)->initializeWithParams(*p) ? 0 : -1; }

int mad_init_box(void* a, const double mn[3], const double mx[3], double spacing) {
    S(a)->initializeParticleBox(Vec3(mn[0], mn[1], mn[2]), Vec3(mx[0], mx[1], mx[2]), spacing);
    return S(a)->getParticleCount() > 0 ? 0 : -1;
}

// tool (may be NULL): candidates inside its analytic shape are left out.
int mad_init_seeded_box(void* a, const int32_t c0[3], const int32_t c1[3], int ppc, uint64_t seed, int fixed_layers,
                        double T0, const mpm_tool_desc* tool) {
    return S(a)->initializeSeededBox(c0, c1, ppc, seed, fixed_layers, T0, tool) ? 0 : -1;
}

int mad_particle_count(void* a) { return S(a)->getParticleCount(); }

void mad_set_tool_position(void* a, const double p[3]) { S(a)->setToolPosition(Vec3(p[0], p[1], p[2])); }

void mad_set_tool_nodes(void* a, void* d_nodes, int n) { S(a)->setToolNodes(static_cast<FEMNodeGPU*>(d_nodes), n); }

void mad_begin_interp(void* a, void* d_nodes, int n) {
    S(a)->beginInterpolatedToolMotion(static_cast<FEMNodeGPU*>(d_nodes), n);
}

void mad_interp_substep(void* a, void* d_nodes, double alpha) {
    S(a)->interpolateToolForSubStep(static_cast<FEMNodeGPU*>(d_nodes), alpha);
}

void mad_end_interp(void* a, void* d_nodes) { S(a)->endInterpolatedToolMotion(static_cast<FEMNodeGPU*>(d_nodes)); }

void mad_step(void* a, double dt) { S(a)->step(dt); }

int mad_pending(void* a) { return S(a)->pendingSteps(); }

void mad_flush(void* a) { S(a)->flush(); }

// syncMetrics, then the IMetricsProvider getters (max stress, max
// temperature, kinetic, internal) and the library's full metrics.
void mad_sync_metrics(void* a, double iface[4], mpm_metrics* full) {
    S(a)->syncMetrics();
    if (iface) {
        iface[0] = S(a)->getMaxStress();
        iface[1] = S(a)->getMaxTemperature();
        iface[2] = S(a)->getTotalKineticEnergy();
        iface[3] = S(a)->getTotalInternalEnergy();
    }
    if (full) *full = S(a)->getMetrics();
}

// getParticles() into dst (504-byte records); returns the records written.
int64_t mad_get_particles(void* a, void* dst, int64_t cap_bytes) {
    const std::vector<MPMParticle> v = S(a)->getParticles();
    const int64_t n = (int64_t)v.size();
    if (!dst || cap_bytes < n * (int64_t)sizeof(MPMParticle)) return -1;
    if (n) std::memcpy(dst, v.data(), (size_t)n * sizeof(MPMParticle));
    return n;
}

void* mad_device_particles(void* a) { return S(a)->getDeviceParticles(); }

void* mad_stream(void* a) { return S(a)->getComputeStream(); }

double mad_stable_dt(void* a) { return S(a)->getStableTimeStep(); }

void mad_set_cfl(void* a, double cfl) { S(a)->setAdaptiveCFL(cfl); }

double mad_time(void* a) { return S(a)->getCurrentTime(); }

void* mad_handle(void* a) { return S(a)->handle(); }

// sizeof(FEMNodeGPU) and the byte offsets of x, y, z, vx, vy, vz.
int mad_fem_node_layout(int32_t* size, int32_t off[6]) {
    *size = (int32_t)sizeof(FEMNodeGPU);
    off[0] = (int32_t)offsetof(FEMNodeGPU, x);
    off[1] = (int32_t)offsetof(FEMNodeGPU, y);
    off[2] = (int32_t)offsetof(FEMNodeGPU, z);
    off[3] = (int32_t)offsetof(FEMNodeGPU, vx);
    off[4] = (int32_t)offsetof(FEMNodeGPU, vy);
    off[5] = (int32_t)offsetof(FEMNodeGPU, vz);
    return (int)sizeof(MPMParticle);
}

}  // extern "C"
