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
    if (m_deviceMirror) cudaFree(m_deviceMirror);
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
    if (m_h) {
        mpm_destroy(m_h);
        m_h = nullptr;
    }
    m_params.particle_volume = spacing * spacing * spacing;
    m_params.particle_mass = m_density * m_params.particle_volume;
    return check(mpm_create(&m_params, m_maxParticles, nullptr, &m_h));
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

bool MPMSolverB200::readToolNodes(const FEMNodeGPU* nodes, int n, std::vector<double>& px, std::vector<double>& py,
                                  std::vector<double>& pz, double vel[3]) {
    std::vector<FEMNodeGPU> h((size_t)n);
    cudaError_t e = cudaMemcpy(h.data(), nodes, sizeof(FEMNodeGPU) * (size_t)n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        m_status = MPM_CUDA_ERROR;
        m_error = std::string("tool nodes: ") + cudaGetErrorString(e);
        return false;
    }
    px.resize((size_t)n); py.resize((size_t)n); pz.resize((size_t)n);
    vel[0] = vel[1] = vel[2] = 0.0;
    for (int i = 0; i < n; ++i) {
        px[i] = h[i].x; py[i] = h[i].y; pz[i] = h[i].z;
        vel[0] += h[i].vx; vel[1] += h[i].vy; vel[2] += h[i].vz;
    }
    if (n > 0) for (int a = 0; a < 3; ++a) vel[a] /= n;
    return true;
}

// rasterizeToolKernel + applyGridCollisionKernel (src/MPMSolver.cu:444-492):
// the tool nodes as raster samples about the tool tip; the grid takes the
// tool's mean node velocity (equal to every node's for a translating tool).
bool MPMSolverB200::pushToolSamples(const std::vector<double>& px, const std::vector<double>& py,
                                    const std::vector<double>& pz, const double vel[3]) {
    const size_t n = px.size();
    std::vector<double> ox(n), oy(n), oz(n);
    for (size_t i = 0; i < n; ++i) {
        ox[i] = px[i] - m_toolPosition.x;
        oy[i] = py[i] - m_toolPosition.y;
        oz[i] = pz[i] - m_toolPosition.z;
    }
    mpm_tool_desc t{};
    t.mode = MPM_TOOL_RASTER;
    t.shape = MPM_SHAPE_CYLINDER_Y;
    t.position[0] = m_toolPosition.x; t.position[1] = m_toolPosition.y; t.position[2] = m_toolPosition.z;
    t.velocity[0] = vel[0]; t.velocity[1] = vel[1]; t.velocity[2] = vel[2];
    t.tip_dz = 0.0;
    t.n_samples = (int32_t)n;
    t.sample_dx = ox.data(); t.sample_dy = oy.data(); t.sample_dz = oz.data();
    return check(mpm_set_tool(m_h, &t));
}

void MPMSolverB200::setToolNodes(FEMNodeGPU* nodes, int numNodes) {
    m_toolNodes = nodes;
    m_numToolNodes = numNodes;
}

// beginInterpolatedToolMotion / interpolateToolForSubStep /
// endInterpolatedToolMotion (include/MPMSolver.cuh:91-110): positions blend
// linearly between the snapshot and the current FEM nodes over a macro step.
void MPMSolverB200::beginInterpolatedToolMotion(FEMNodeGPU* femNodes, int numNodes) {
    double v[3];
    m_interpActive = readToolNodes(femNodes, numNodes, m_interpStart[0], m_interpStart[1], m_interpStart[2], v);
    m_toolNodes = femNodes;
    m_numToolNodes = numNodes;
}

void MPMSolverB200::interpolateToolForSubStep(FEMNodeGPU* femNodes, double alpha) {
    m_toolNodes = femNodes;
    m_interpAlpha = std::min(std::max(alpha, 0.0), 1.0);
}

void MPMSolverB200::endInterpolatedToolMotion(FEMNodeGPU* femNodes) {
    m_toolNodes = femNodes;
    m_interpActive = false;
    m_interpAlpha = 1.0;
}

// MPMSolver::step (src/MPMSolver.cu:1062-1168): one step of dt; nothing
// before a workpiece exists.
void MPMSolverB200::step(double dt) {
    if (!m_initialized || !m_h || m_numParticles == 0) return;
    if (m_toolNodes && m_numToolNodes > 0) {
        std::vector<double> px, py, pz;
        double vel[3];
        if (!readToolNodes(m_toolNodes, m_numToolNodes, px, py, pz, vel)) return;
        if (m_interpActive && m_interpStart[0].size() == px.size()) {
            const double a = m_interpAlpha;
            for (size_t i = 0; i < px.size(); ++i) {
                px[i] = m_interpStart[0][i] + a * (px[i] - m_interpStart[0][i]);
                py[i] = m_interpStart[1][i] + a * (py[i] - m_interpStart[1][i]);
                pz[i] = m_interpStart[2][i] + a * (pz[i] - m_interpStart[2][i]);
            }
        }
        if (!pushToolSamples(px, py, pz, vel)) return;
    }
    if (check(mpm_step(m_h, dt, 1))) m_time += dt;
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
    check(mpm_set_temperatures(m_h, temperatures, count));
}

std::vector<MPMParticle> MPMSolverB200::getParticles() {
    m_hostParticles.assign((size_t)m_numParticles, MPMParticle());
    if (m_h && m_numParticles > 0 &&
        !check(mpm_export_aos(m_h, m_hostParticles.data(), (int64_t)m_hostParticles.size() * 504)))
        m_hostParticles.clear();
    return m_hostParticles;
}

MPMParticle* MPMSolverB200::getDeviceParticles() {
    if (!m_h || m_numParticles == 0) return nullptr;
    const size_t bytes = (size_t)m_numParticles * sizeof(MPMParticle);
    if (bytes > m_deviceMirrorBytes) {
        if (m_deviceMirror) cudaFree(m_deviceMirror);
        m_deviceMirror = nullptr;
        m_deviceMirrorBytes = 0;
        if (cudaMalloc(&m_deviceMirror, bytes) != cudaSuccess) {
            m_status = MPM_OOM;
            m_error = "device particle mirror: out of memory";
            return nullptr;
        }
        m_deviceMirrorBytes = bytes;
    }
    if (!check(mpm_export_aos(m_h, m_deviceMirror, (int64_t)bytes))) return nullptr;
    return m_deviceMirror;
}

cudaStream_t MPMSolverB200::getComputeStream() const {
    void* s = nullptr;
    if (m_h) mpm_get_stream(m_h, &s);
    return static_cast<cudaStream_t>(s);
}

void MPMSolverB200::applyExternalForce(const Vec3& center, double radius, const Vec3& force) {
    if (!m_h) return;
    const double c[3] = {center.x, center.y, center.z}, f[3] = {force.x, force.y, force.z};
    check(mpm_apply_external_force(m_h, c, radius, f));
}

// setDynamicMassScaling (src/MPMSolver.cu:1211-1225): inertial density =
// max(physical * factor, physical); thermal terms keep the physical density.
void MPMSolverB200::setDynamicMassScaling(double factor) {
    if (!(factor > 0.0)) return;
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
