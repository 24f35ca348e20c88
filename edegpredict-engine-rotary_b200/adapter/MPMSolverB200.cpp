// MPMSolverB200.cpp -- see MPMSolverB200.h.  Every call forwards to the C ABI
// of libmpm_b200.so; reference behaviour is cited per member.
#include "MPMSolverB200.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <iostream>
#include <limits>

#include "Config.h"

namespace edgepredict {

static_assert(sizeof(MPMParticle) == 504, "mpm_export_aos writes 504-byte MPMParticle records");

MPMSolverB200::MPMSolverB200(int maxParticles) : m_maxParticles(maxParticles) {
    mpm_params_default(&m_params);
}

MPMSolverB200::~MPMSolverB200() {
    flush();   // the reference would have run the steps it was given
    if (m_deviceMirror) cudaFree(m_deviceMirror);
    if (m_startNodes) cudaFree(m_startNodes);
    if (m_h) mpm_destroy(m_h);
}

bool MPMSolverB200::check(mpm_status s) {
    m_status = s;
    if (s == MPM_OK) return true;
    const char* msg = mpm_last_error(m_h);
    m_error = std::string(mpm_status_string(s)) + ": " + (msg ? msg : "");
    std::cerr << "[MPMSolverB200] " << m_error << std::endl;
    return false;
}

// MPMSolver::initialize (src/MPMSolver.cu:832-915): the same Config fields,
// the same 0.2 m cube around the origin and the same dx rule.  Device memory
// is taken when the workpiece is created (particle mass and volume depend on
// its spacing).
bool MPMSolverB200::initialize(const Config& config) {
    flush();
    const auto& sph = config.getSPH();
    const auto& mat = config.getMaterial();
    const int precision = m_params.precision;
    mpm_params_default(&m_params);
    m_params.precision = precision;
    m_params.dx = std::max(sph.smoothingRadius * 2.0, 0.0005);
    const double lo = -0.1, hi = 0.1;
    m_domainMin = Vec3(lo, lo, lo);
    const int n = (int)((hi - lo) / m_params.dx) + 1;
    m_params.nx = m_params.ny = m_params.nz = n;
    m_params.origin[0] = m_params.origin[1] = m_params.origin[2] = lo;
    m_params.E = mat.youngsModulus;
    m_params.nu = mat.poissonsRatio;
    m_params.rho_phys = mat.density;
    m_density = mat.density * sph.numericalMassScalingFactor;
    m_params.cp = mat.specificHeat;
    m_params.beta = 0.9;
    m_params.Tm = mat.meltingPoint;
    m_params.Tamb = config.getMachining().ambientTemperature;
    m_params.jc_A = mat.jc_A;
    m_params.jc_B = mat.jc_B;
    m_params.jc_n = mat.jc_n;
    m_params.jc_C = mat.jc_C;
    m_params.jc_m = mat.jc_m;
    m_params.D1 = sph.jc_D1;
    m_params.D2 = sph.jc_D2;
    m_params.D3 = sph.jc_D3;
    m_params.D4 = sph.jc_D4;
    m_params.D5 = sph.jc_D5;
    m_params.D_th = sph.damageThreshold;
    m_params.edot0 = sph.referenceStrainRate;
    m_params.lod_active_r = sph.lodActiveRadius;
    m_params.lod_near_r = sph.lodNearRadius;
    m_params.lod_enabled = sph.lodEnabled ? 1 : 0;
    m_params.fixture_thickness = config.getMachineSetup().fixtureLayerThickness;
    m_params.fixture_damping = 1e7;
    m_initialized = true;
    return true;
}

bool MPMSolverB200::ensureHandle(double spacing) {
    if (!m_initialized) return false;
    flush();
    if (m_h) {
        mpm_destroy(m_h);
        m_h = nullptr;
    }
    m_params.particle_volume = spacing * spacing * spacing;
    m_params.particle_mass = m_density * m_params.particle_volume;
    return check(mpm_create(&m_params, m_maxParticles, nullptr, &m_h));
}

// The library's own parameters (any grid), for workpieces the reference's
// initialize cannot express; the inertial density is params.rho_phys.
bool MPMSolverB200::initializeWithParams(const mpm_params& params) {
    flush();
    if (m_h) {
        mpm_destroy(m_h);
        m_h = nullptr;
    }
    m_numParticles = 0;
    m_params = params;
    m_density = params.rho_phys;
    m_domainMin = Vec3(params.origin[0], params.origin[1], params.origin[2]);
    m_initialized = check(mpm_create(&m_params, m_maxParticles, nullptr, &m_h));
    return m_initialized;
}

bool MPMSolverB200::initializeSeededBox(const int32_t c0[3], const int32_t c1[3], int ppc, uint64_t seed,
                                        int fixedLayers, double T0, const mpm_tool_desc* removeInside) {
    flush();
    if (!m_h) return false;
    int64_t n = 0;
    if (!check(mpm_init_box(m_h, c0, c1, ppc, seed, 0, fixedLayers, T0, removeInside))) return false;
    if (!check(mpm_get_counts(m_h, &n, nullptr, nullptr))) return false;
    m_numParticles = (int)n;
    m_time = 0.0;
    push();
    return true;
}

bool MPMSolverB200::uploadLattice(const std::vector<double>& x, const std::vector<double>& y,
                                  const std::vector<double>& z, const std::vector<int32_t>& status) {
    const int64_t n = (int64_t)x.size();
    std::vector<double> T((size_t)n, m_params.Tamb);
    mpm_particles_soa soa{};
    soa.elem = 8;
    soa.x = const_cast<double*>(x.data());
    soa.y = const_cast<double*>(y.data());
    soa.z = const_cast<double*>(z.data());
    soa.temperature = T.data();
    soa.status = const_cast<int32_t*>(status.data());
    if (!check(mpm_upload(m_h, &soa, n))) return false;
    m_numParticles = (int)n;
    push();
    return true;
}

// MPMSolver::initializeParticleBox (src/MPMSolver.cu:1297-1336): a lattice of
// the given spacing from minBounds up to maxBounds (inclusive), the lowest 10 %
// of the height FIXED_BOUNDARY, ambient temperature.
void MPMSolverB200::initializeParticleBox(const Vec3& minBounds, const Vec3& maxBounds, double spacing) {
    m_numParticles = 0;
    if (!(spacing > 0.0) || !ensureHandle(spacing)) return;
    const double zfix = minBounds.z + (maxBounds.z - minBounds.z) * 0.1;
    std::vector<double> x, y, z;
    std::vector<int32_t> st;
    for (double pz = minBounds.z; pz <= maxBounds.z; pz += spacing)
        for (double py = minBounds.y; py <= maxBounds.y; py += spacing)
            for (double px = minBounds.x; px <= maxBounds.x && (int)x.size() < m_maxParticles; px += spacing) {
                x.push_back(px);
                y.push_back(py);
                z.push_back(pz);
                st.push_back(pz <= zfix ? MPM_FIXED : MPM_ACTIVE);
            }
    uploadLattice(x, y, z, st);
    m_metrics.bounds_min[0] = minBounds.x; m_metrics.bounds_min[1] = minBounds.y; m_metrics.bounds_min[2] = minBounds.z;
    m_metrics.bounds_max[0] = maxBounds.x; m_metrics.bounds_max[1] = maxBounds.y; m_metrics.bounds_max[2] = maxBounds.z;
}

// MPMSolver::initializeCylindricalWorkpiece (src/MPMSolver.cu:1338-1381): a
// lattice disc stack below `center` along -z (the reference ignores `axis`),
// the lowest 10 % of the length FIXED_BOUNDARY.
void MPMSolverB200::initializeCylindricalWorkpiece(const Vec3& center, double radius, double length, double spacing,
                                                   int axis) {
    (void)axis;
    m_numParticles = 0;
    if (!(spacing > 0.0) || !ensureHandle(spacing)) return;
    const double zfix = center.z - length * 0.1, r2 = radius * radius;
    std::vector<double> x, y, z;
    std::vector<int32_t> st;
    for (double dz = 0; dz <= length; dz += spacing)
        for (double dy = -radius; dy <= radius; dy += spacing)
            for (double dx = -radius; dx <= radius && (int)x.size() < m_maxParticles; dx += spacing) {
                if (dx * dx + dy * dy > r2) continue;
                x.push_back(center.x + dx);
                y.push_back(center.y + dy);
                z.push_back(center.z - dz);
                st.push_back(center.z - dz <= zfix ? MPM_FIXED : MPM_ACTIVE);
            }
    uploadLattice(x, y, z, st);
    m_metrics.bounds_min[0] = center.x - radius; m_metrics.bounds_min[1] = center.y - radius;
    m_metrics.bounds_min[2] = center.z - length;
    m_metrics.bounds_max[0] = center.x + radius; m_metrics.bounds_max[1] = center.y + radius;
    m_metrics.bounds_max[2] = center.z;
}

// The tool source the next sub-step reads: the blended FEM nodes while a
// blended motion is on (interpolateToolForSubStep's alpha), else the nodes
// of setToolNodes (or none).
MPMSolverB200::ToolSource MPMSolverB200::currentSource() const {
    ToolSource t;
    t.end = m_toolNodes;
    if (m_interpActive && m_startNodes) {
        t.start = m_startNodes;
        t.alpha = m_interpAlpha;
    }
    return t;
}

// rasterizeToolKernel + applyGridCollisionKernel (src/MPMSolver.cu:444-492)
// read the FEM tool's device nodes on every step: the library does the same
// from the node records (mpm_set_tool_nodes), with no host copy.
void MPMSolverB200::setToolNodes(FEMNodeGPU* nodes, int numNodes) {
    flush();
    m_toolNodes = nodes;
    m_numToolNodes = numNodes;
}

// beginInterpolatedToolMotion / interpolateToolForSubStep /
// endInterpolatedToolMotion (src/MPMSolver.cu:976-1000): the nodes of each
// sub-step blend linearly from a snapshot taken here (a device-to-device
// copy, as the reference takes it) to the current FEM nodes; the blend itself
// runs on the device inside the raster launch of every step.
void MPMSolverB200::beginInterpolatedToolMotion(FEMNodeGPU* femNodes, int numNodes) {
    flush();
    const size_t bytes = sizeof(FEMNodeGPU) * (size_t)std::max(numNodes, 0);
    if (bytes > m_startNodesBytes) {
        if (m_startNodes) cudaFree(m_startNodes);
        m_startNodes = nullptr;
        m_startNodesBytes = 0;
        if (cudaMalloc(&m_startNodes, bytes) != cudaSuccess) {
            m_status = MPM_OOM;
            m_error = "tool node snapshot: out of memory";
            m_interpActive = false;
            return;
        }
        m_startNodesBytes = bytes;
    }
    cudaStream_t st = getComputeStream();
    cudaError_t e = bytes ? cudaMemcpyAsync(m_startNodes, femNodes, bytes, cudaMemcpyDeviceToDevice, st)
                          : cudaSuccess;
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        m_status = MPM_CUDA_ERROR;
        m_error = std::string("tool node snapshot: ") + cudaGetErrorString(e);
        m_interpActive = false;
        return;
    }
    m_toolNodes = femNodes;
    m_numToolNodes = numNodes;
    m_interpActive = true;
    m_interpAlpha = 0.0;
}

void MPMSolverB200::interpolateToolForSubStep(FEMNodeGPU* femNodes, double alpha) {
    // part of the sub-step sequence: no flush unless the node array changes
    if (femNodes != m_toolNodes) flush();
    m_toolNodes = femNodes;
    m_interpAlpha = alpha;
}

void MPMSolverB200::endInterpolatedToolMotion(FEMNodeGPU* femNodes) {
    flush();
    m_toolNodes = femNodes;
    m_interpActive = false;
    m_interpAlpha = 0.0;
}

// MPMSolver::step (src/MPMSolver.cu:1062-1168): one step of dt; nothing
// before a workpiece exists.  Queued: a sub-step joins the queue when it has
// the queue's dt and its tool source continues the queue's (the same node
// arrays, and a blend weight one per-step increment further); otherwise the
// queue runs first.
void MPMSolverB200::step(double dt) {
    if (!m_initialized || !m_h || m_numParticles == 0) return;
    const ToolSource t = currentSource();
    if (m_pendingSteps > 0) {
        bool join = dt == m_pendingDt && t.start == m_runSource.start && t.end == m_runSource.end;
        if (join && t.start) {
            const double want = m_pendingSteps == 1 ? t.alpha
                                                    : m_runSource.alpha + m_pendingSteps * m_runDalpha;
            join = std::fabs(t.alpha - want) <= 1e-12 * std::max(1.0, std::fabs(want));
            if (join && m_pendingSteps == 1) m_runDalpha = t.alpha - m_runSource.alpha;
        }
        if (!join || m_pendingSteps >= kMaxQueuedSteps) flush();
    }
    if (m_pendingSteps == 0) {
        m_pendingDt = dt;
        m_runSource = t;
        m_runDalpha = 0.0;
    }
    ++m_pendingSteps;
    m_time += dt;
}

// The queued sub-steps as one library call: the tool pose (chip separation
// and LOD read its tip, src/MPMSolver.cu:1160-1162), the node source of the
// first queued sub-step with the per-step blend increment, then the steps.
bool MPMSolverB200::runQueue() {
    const int n = m_pendingSteps;
    m_pendingSteps = 0;
    mpm_tool_desc t{};
    t.mode = m_runSource.end ? MPM_TOOL_RASTER : MPM_TOOL_NONE;
    t.shape = MPM_SHAPE_CYLINDER_Y;
    t.position[0] = m_toolPosition.x; t.position[1] = m_toolPosition.y; t.position[2] = m_toolPosition.z;
    if (!check(mpm_set_tool(m_h, &t))) return false;
    if (m_runSource.end) {
        mpm_tool_nodes tn{};
        tn.start = m_runSource.start;
        tn.end = m_runSource.end;
        tn.n = m_numToolNodes;
        tn.stride = (int32_t)sizeof(FEMNodeGPU);
        tn.off_pos[0] = (int32_t)offsetof(FEMNodeGPU, x);
        tn.off_pos[1] = (int32_t)offsetof(FEMNodeGPU, y);
        tn.off_pos[2] = (int32_t)offsetof(FEMNodeGPU, z);
        tn.off_vel[0] = (int32_t)offsetof(FEMNodeGPU, vx);
        tn.off_vel[1] = (int32_t)offsetof(FEMNodeGPU, vy);
        tn.off_vel[2] = (int32_t)offsetof(FEMNodeGPU, vz);
        tn.alpha0 = m_runSource.alpha;
        tn.dalpha = m_runDalpha;
        if (!check(mpm_set_tool_nodes(m_h, &tn))) return false;
    }
    return check(mpm_step(m_h, m_pendingDt, n));
}

void MPMSolverB200::flush() {
    if (m_pendingSteps == 0 || !m_h) {
        m_pendingSteps = 0;
        return;
    }
    pull();
    runQueue();
    push();
}

// The live mirror: writes of the reference's consumers come in before a step
// or a read (pull), the state goes out after steps (push).
void MPMSolverB200::pull() {
    if (!m_mirrorLive || !m_h || !m_deviceMirror || m_numParticles == 0) return;
    check(mpm_import_aos(m_h, m_deviceMirror, (int64_t)m_deviceMirrorBytes, MPM_AOS_WRITABLE));
}

void MPMSolverB200::push() {
    if (!m_mirrorLive || !m_h || m_numParticles == 0 || !ensureMirror()) return;
    check(mpm_export_aos(m_h, m_deviceMirror, (int64_t)((size_t)m_numParticles * sizeof(MPMParticle))));
}

bool MPMSolverB200::ensureMirror() {
    const size_t bytes = (size_t)m_numParticles * sizeof(MPMParticle);
    if (bytes <= m_deviceMirrorBytes && m_deviceMirror) return true;
    if (m_deviceMirror) cudaFree(m_deviceMirror);
    m_deviceMirror = nullptr;
    m_deviceMirrorBytes = 0;
    if (cudaMalloc(&m_deviceMirror, bytes) != cudaSuccess) {
        m_status = MPM_OOM;
        m_error = "device particle mirror: out of memory";
        m_mirrorLive = false;
        return false;
    }
    m_deviceMirrorBytes = bytes;
    return true;
}

// getStableTimeStep (src/MPMSolver.cu:1170-1178): CFL * dx / max(c, 1) with
// c = sqrt(E / inertial density), at least 1e-10 s.
double MPMSolverB200::getStableTimeStep() const {
    const double c = std::sqrt(m_params.E / m_density);
    return std::max(m_cfl * m_params.dx / std::max(c, 1.0), 1e-10);
}

double MPMSolverB200::getWaveSpeed() const { return std::sqrt(m_params.E / m_density); }
double MPMSolverB200::getPhysicalWaveSpeed() const { return std::sqrt(m_params.E / m_params.rho_phys); }

// getHighestFrequency (src/MPMSolver.cu:1188-1197): c_phys / (2 dx).
double MPMSolverB200::getHighestFrequency() const {
    return getPhysicalWaveSpeed() / (2.0 * std::max(m_params.dx, 1e-10));
}

void MPMSolverB200::reset() {
    flush();
    m_time = 0.0;
    if (m_h) check(mpm_reset_clock(m_h));
}

void MPMSolverB200::getBounds(double& minX, double& minY, double& minZ, double& maxX, double& maxY,
                              double& maxZ) const {
    minX = m_metrics.bounds_min[0]; minY = m_metrics.bounds_min[1]; minZ = m_metrics.bounds_min[2];
    maxX = m_metrics.bounds_max[0]; maxY = m_metrics.bounds_max[1]; maxZ = m_metrics.bounds_max[2];
}

// syncMetrics (src/MPMSolver.cu:1239-1259) and the cached bounds.
void MPMSolverB200::syncMetrics() {
    if (!m_h || m_numParticles == 0) return;
    flush();
    pull();
    mpm_metrics m{};
    const mpm_status s = mpm_sync_metrics(m_h, &m);
    if (s == MPM_NUMERIC) {
        // The workpiece's error word is set (a NaN or Inf state, or a Newton
        // return that did not converge).  The kill zone has taken the NaN
        // particles out of the reductions, so the peaks alone would look
        // healthy: report them as NaN, which SimulationHealthMonitor::check
        // turns into its NAN_CORRUPTION halt
        // (include/SimulationHealthMonitor.h:321-328), as a NaN would in the
        // reference.  Not run by the tests (they compile against the
        // reference's headers, which only this container has).
        m.ref_max_stress = std::numeric_limits<double>::quiet_NaN();
        m.ref_max_temperature = std::numeric_limits<double>::quiet_NaN();
        m_metrics = m;
        check(s);
        return;
    }
    if (check(s)) m_metrics = m;
}

void MPMSolverB200::applyHeatFlux(double, double, double, double) {}

double MPMSolverB200::getTemperatureAt(double x, double y, double z) const {
    double best = 1e30, T = m_params.Tamb;
    for (const MPMParticle& p : m_hostParticles) {
        if (p.status != ParticleStatus::ACTIVE) continue;
        const double dx = p.x - x, dy = p.y - y, dz = p.z - z, d = dx * dx + dy * dy + dz * dz;
        if (d < best) {
            best = d;
            T = p.temperature;
        }
    }
    return T;
}

// setParticleTemperatures (src/MPMSolver.cu:1267-1277): count <= particles.
void MPMSolverB200::setParticleTemperatures(const double* temperatures, int count) {
    if (!m_h || !temperatures || count <= 0 || count > m_numParticles) return;
    flush();
    pull();
    if (check(mpm_set_temperatures(m_h, temperatures, count))) push();
}

std::vector<MPMParticle> MPMSolverB200::getParticles() {
    flush();
    pull();
    m_hostParticles.assign((size_t)m_numParticles, MPMParticle());
    if (m_h && m_numParticles > 0 &&
        !check(mpm_export_aos(m_h, m_hostParticles.data(), (int64_t)m_hostParticles.size() * 504)))
        m_hostParticles.clear();
    return m_hostParticles;
}

// The reference hands out its own particle array (include/MPMSolver.cuh:
// 143, used by ContactSolver at src/ContactSolver.cu:1131 and by CFD chip
// coupling at src/SimulationEngine.cpp:1012): here the live mirror.
MPMParticle* MPMSolverB200::getDeviceParticles() {
    if (!m_h || m_numParticles == 0) return nullptr;
    flush();
    pull();   // writes since the last export, when the mirror is already out
    if (!ensureMirror()) return nullptr;
    m_mirrorLive = true;
    if (!check(mpm_export_aos(m_h, m_deviceMirror, (int64_t)((size_t)m_numParticles * sizeof(MPMParticle)))))
        return nullptr;
    return m_deviceMirror;
}

// The handle's stream, after the queued sub-steps are issued on it.
cudaStream_t MPMSolverB200::getComputeStream() const {
    const_cast<MPMSolverB200*>(this)->flush();
    void* s = nullptr;
    if (m_h) mpm_get_stream(m_h, &s);
    return static_cast<cudaStream_t>(s);
}

void MPMSolverB200::applyExternalForce(const Vec3& center, double radius, const Vec3& force) {
    if (!m_h) return;
    flush();
    const double c[3] = {center.x, center.y, center.z}, f[3] = {force.x, force.y, force.z};
    check(mpm_apply_external_force(m_h, c, radius, f));
}

// setDynamicMassScaling (src/MPMSolver.cu:1211-1225): inertial density =
// max(physical * factor, physical); thermal terms keep the physical density.
void MPMSolverB200::setDynamicMassScaling(double factor) {
    if (!(factor > 0.0)) return;
    flush();
    m_density = std::max(m_params.rho_phys * factor, m_params.rho_phys);
    if (m_h) check(mpm_set_mass_scaling(m_h, factor));
}

// getMeltingParticleCount (src/MPMSolver.cu:1388-1402, countMeltingParticles-
// Kernel :790-800): ACTIVE particles within 1 degree of the melting point,
// counted on the host copy of the particles.
int MPMSolverB200::getMeltingParticleCount(double meltingPoint) {
    getParticles();
    int n = 0;
    for (const MPMParticle& p : m_hostParticles)
        if (p.status == ParticleStatus::ACTIVE && p.temperature >= meltingPoint - 1.0) ++n;
    return n;
}

}  // namespace edgepredict
