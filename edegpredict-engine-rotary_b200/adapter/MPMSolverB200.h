// MPMSolverB200.h -- drop-in for edgepredict::MPMSolver (include/MPMSolver.cuh:76-268)
// on top of libmpm_b200.so (include/mpm_capi.h).
//
// Built inside the reference tree: it includes the reference's own headers
// (IPhysicsSolver.h, Types.h, Config.h) and links libmpm_b200.so.  It
// implements IPhysicsSolver / IMetricsProvider / IThermalCoupling
// (include/IPhysicsSolver.h:24-149) and the MPMSolver members that
// SimulationEngine, ContactSolver and the exporters call, with the same names
// and meanings.  Where the reference returns void/bool and swallows errors,
// so does this class; the last C-ABI status and message are kept
// (lastStatus(), lastError()).
//
// Sub-stepping.  SimulationEngine calls step(microDt) once per sub-step with
// only interpolateToolForSubStep between the calls (src/SimulationEngine.cpp:
// 515-524).  step() queues the sub-step; the queue runs as ONE multi-step
// call of the library (one fused launch per step, replayable from a CUDA
// graph) at the next call of any other member, or when dt or the tool
// source changes.  The FEM tool nodes are rasterised on the device from
// their own device records with the sub-step blend done there
// (mpm_set_tool_nodes): no host copy of the nodes and no synchronisation per
// sub-step.  getComputeStream() runs the queue first, so work that the
// caller orders after it on that stream sees every step.
//
// The device mirror.  getDeviceParticles() hands out an MPMParticle array,
// as the reference hands out its own d_particles, which ContactSolver and CFD
// chip coupling write in place.  Once handed out it stays live: before every
// step and every read the writes in it are imported (mpm_import_aos:
// positions, velocities, temperatures, statuses and ext_f), and after every
// batch of steps it is exported again.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "IPhysicsSolver.h"
#include "Types.h"
#include "mpm_capi.h"

namespace edgepredict {

class Config;

class MPMSolverB200 : public IPhysicsSolver, public IMetricsProvider, public IThermalCoupling {
public:
    // maxParticles: handle capacity (the reference's m_maxParticles default is 5,000,000).
    explicit MPMSolverB200(int maxParticles = 5000000);
    ~MPMSolverB200() override;
    MPMSolverB200(const MPMSolverB200&) = delete;
    MPMSolverB200& operator=(const MPMSolverB200&) = delete;

    // ---- IPhysicsSolver
    std::string getName() const override { return "MPMSolverB200"; }
    bool initialize(const Config& config) override;
    void step(double dt) override;
    double getStableTimeStep() const override;
    double getCurrentTime() const override { return m_time; }
    bool isInitialized() const override { return m_initialized; }
    void reset() override;
    void getBounds(double& minX, double& minY, double& minZ, double& maxX, double& maxY,
                   double& maxZ) const override;
    int getNodeCount() const override { return m_params.nx * m_params.ny * m_params.nz; }
    int getParticleCount() const override { return m_numParticles; }

    // ---- IMetricsProvider (values of the last syncMetrics)
    double getMaxStress() const override { return m_metrics.ref_max_stress; }
    double getMaxTemperature() const override { return m_metrics.ref_max_temperature; }
    double getTotalKineticEnergy() const override { return m_metrics.ref_kinetic; }
    double getTotalInternalEnergy() const override { return m_metrics.ref_internal; }
    void syncMetrics() override;

    // ---- IThermalCoupling
    // A no-op, as in the reference (src/MPMSolver.cu:1261-1265).
    void applyHeatFlux(double x, double y, double z, double heatFlux) override;
    // Temperature of the nearest ACTIVE particle of the last getParticles().
    double getTemperatureAt(double x, double y, double z) const override;
    void setParticleTemperatures(const double* temperatures, int count) override;

    // ---- MPMSolver members used by SimulationEngine / ContactSolver / exporters
    void initializeParticleBox(const Vec3& minBounds, const Vec3& maxBounds, double spacing);
    void initializeCylindricalWorkpiece(const Vec3& center, double radius, double length, double spacing,
                                        int axis = 2);
    std::vector<MPMParticle> getParticles();
    // The particles in the MPMParticle layout in device memory, writable in
    // place: writes reach the solver before its next step or read (positions,
    // velocities, temperatures, statuses, ext_f).  The pointer stays valid
    // until a larger workpiece is initialised.
    MPMParticle* getDeviceParticles();
    cudaStream_t getComputeStream() const;
    const Vec3& getDomainMin() const { return m_domainMin; }

    // Tool: FEM nodes on the device, rasterised onto the grid every step
    // (setToolNodes, include/MPMSolver.cuh:86-89), and the tool-tip position
    // used by chip separation and LOD.
    void setToolNodes(FEMNodeGPU* nodes, int numNodes);
    void beginInterpolatedToolMotion(FEMNodeGPU* femNodes, int numNodes);
    void interpolateToolForSubStep(FEMNodeGPU* femNodes, double alpha);
    void endInterpolatedToolMotion(FEMNodeGPU* femNodes);
    void setToolPosition(const Vec3& pos) { m_toolPosition = pos; }
    Vec3 getToolPosition() const { return m_toolPosition; }

    void applyExternalForce(const Vec3& center, double radius, const Vec3& force);
    void setLODEnabled(bool enabled) { m_params.lod_enabled = enabled ? 1 : 0; }
    void setDynamicMassScaling(double factor);
    double getHighestFrequency() const;
    double getWaveSpeed() const;
    double getPhysicalWaveSpeed() const;
    void setAdaptiveCFL(double cfl) { m_cfl = cfl > 0.01 ? cfl : 0.01; }
    double getAdaptiveCFL() const { return m_cfl; }
    double getSmoothingRadius() const { return m_params.dx * 1.5; }
    int getMeltingParticleCount(double meltingPoint);

    // ---- this build
    // Arithmetic of the bulk state: MPM_PREC_F32 (default) or MPM_PREC_F64.
    // Takes effect at the next workpiece initialisation.
    void setPrecision(int precision) { m_params.precision = precision; }
    // A workpiece on a grid the reference's initialize(Config) cannot express
    // (its domain is the 0.2 m cube with dx >= 0.5 mm, src/MPMSolver.cu:
    // 840-846): the library's parameters as given, then a seeded box of
    // cells [c0, c1) with ppc particles per cell (mpm_init_box), leaving out
    // the candidates inside removeInside's analytic shape when it is given.
    bool initializeWithParams(const mpm_params& params);
    bool initializeSeededBox(const int32_t c0[3], const int32_t c1[3], int ppc, uint64_t seed, int fixedLayers,
                             double T0, const mpm_tool_desc* removeInside = nullptr);
    // Runs the queued sub-steps now (every other member does this first).
    void flush();
    int pendingSteps() const { return m_pendingSteps; }
    mpm_handle* handle() { return m_h; }
    const mpm_metrics& getMetrics() const { return m_metrics; }
    mpm_status lastStatus() const { return m_status; }
    std::string lastError() const { return m_error; }

private:
    // The tool source of one sub-step: FEM records end (blended from start by
    // alpha when start is set).
    struct ToolSource {
        const FEMNodeGPU* start = nullptr;
        const FEMNodeGPU* end = nullptr;
        double alpha = 0.0;
    };
    bool check(mpm_status s);
    bool ensureHandle(double spacing);
    bool uploadLattice(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
                       const std::vector<int32_t>& status);
    ToolSource currentSource() const;
    bool runQueue();
    void pull();
    void push();
    bool ensureMirror();
    // A queue longer than this runs without waiting for an observation.
    static constexpr int kMaxQueuedSteps = 64;

    mpm_params m_params{};
    mpm_handle* m_h = nullptr;
    int m_maxParticles;
    int m_numParticles = 0;
    bool m_initialized = false;
    double m_time = 0.0;
    double m_cfl = 0.2;
    double m_density = 7850.0;       // inertial density (physical x mass scaling)
    Vec3 m_domainMin;
    Vec3 m_toolPosition;
    FEMNodeGPU* m_toolNodes = nullptr;       // the nodes a step reads (setToolNodes / the blend's end)
    int m_numToolNodes = 0;
    FEMNodeGPU* m_startNodes = nullptr;      // the blend's start snapshot (device, owned)
    size_t m_startNodesBytes = 0;
    bool m_interpActive = false;
    double m_interpAlpha = 0.0;
    // queued sub-steps: count, their dt, the first one's tool source and the
    // blend weight added per sub-step
    int m_pendingSteps = 0;
    double m_pendingDt = 0.0;
    ToolSource m_runSource;
    double m_runDalpha = 0.0;
    mpm_metrics m_metrics{};
    std::vector<MPMParticle> m_hostParticles;
    MPMParticle* m_deviceMirror = nullptr;
    size_t m_deviceMirrorBytes = 0;
    bool m_mirrorLive = false;
    mpm_status m_status = MPM_OK;
    std::string m_error;
};

}  // namespace edgepredict
