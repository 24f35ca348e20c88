// mpm_engine.h -- host engine behind the C ABI: owns the device state of one
// or more workpiece instances and drives the step kernel.  Not a public
// header; the ABI is include/mpm_capi.h.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/mpm_capi.h"
#include "mpm_device.cuh"
#include "mpm_internal.h"

namespace mpmb {

// A tool SDF as a 3D texture (trilinear filtering, clamp addressing,
// unnormalised coordinates), shared by the copies of an instance record.
struct ToolSdfTex {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    int n[3] = {0, 0, 0};
    float origin[3] = {0, 0, 0}, voxel = 0.0f, cos_a = 1.0f, sin_a = 0.0f;
    ~ToolSdfTex() {
        if (tex) cudaDestroyTextureObject(tex);
        if (arr) cudaFreeArray(arr);
    }
};

struct InstHost {
    mpm_params p;
    mpm_tool_desc tool;
    std::vector<double> samples;  // raster samples: x..., y..., z...
    int64_t cap = 0, np = 0, pbase = 0;
    int64_t nn = 0, grid_off = 0;  // grid nodes and offset (in nodes) in the grid pools
    int nbx = 0, nby = 0, nbz = 0;
    int bin0 = 0;                  // first bin of the instance in the engine's bin table
    int since = 0;                 // G2P steps since the re-bin that last moved its particles
    bool rebin_now = false;        // positions changed outside a step: bin from them at the next re-bin
    double time = 0.0, dt = 0.0;
    int64_t step = 0;
    double* d_samples = nullptr;
    int n_samples = 0;
    int samples_cap = 0;    // samples d_samples holds room for (set_tool reuses it)
    double sbox[6] = {0, 0, 0, 0, 0, 0};   // the samples' offset box: x, y, z min, then max
    // raster from FEM node records in device memory (mpm_set_tool_nodes)
    bool has_nodes = false;
    mpm_tool_nodes nodes{};
    int64_t nodes_step0 = 0;  // step counter when the node source was set
    double ext_c[3] = {0, 0, 0}, ext_r = 0.0, ext_f[3] = {0, 0, 0};
    bool ext_pending = false;
    double tool_t0 = 0.0;   // time at which the tool descriptor was set
    std::shared_ptr<ToolSdfTex> sdf;   // voxel tool SDF for the contact (null: analytic SDF)
    int fresh = 0;          // particles uploaded or generated, not yet binned
    // A checkpoint load failed after it began to overwrite the particle
    // arrays: the state is part old, part new.  Steps refuse the handle until
    // an upload, a generated box or a complete checkpoint load replaces it.
    bool broken = false;
    // An AoS import brought per-particle external forces for the next step
    // (device array indexed pbase + upload order).
    bool pext_pending = false;
};

class EngineBase {
   public:
    virtual ~EngineBase() = default;
    std::string err;
    virtual mpm_status init_box(int inst, const int32_t c0[3], const int32_t c1[3], int32_t ppc, uint64_t seed,
                                uint32_t instance, int32_t fixed_layers, double T0, const mpm_tool_desc* tool) = 0;
    virtual mpm_status upload(int inst, const mpm_particles_soa* host, int64_t n) = 0;
    virtual mpm_status download(int inst, mpm_particles_soa* host) = 0;
    virtual mpm_status export_aos(int inst, void* dst, int64_t bytes) = 0;
    virtual mpm_status import_aos(int inst, const void* src, int64_t bytes, uint32_t fields) = 0;
    virtual mpm_status set_tool(int inst, const mpm_tool_desc* t) = 0;
    virtual mpm_status set_tool_sdf(int inst, const mpm_tool_sdf* s) = 0;
    virtual mpm_status set_tool_nodes(int inst, const mpm_tool_nodes* n) = 0;
    // MPMWorkpieceSolver's step semantics for the whole handle (NULL: back to
    // MPMSolver's).
    virtual mpm_status set_workpiece_semantics(const mpm_workpiece_params* p) = 0;
    virtual mpm_status step(int32_t nsteps, const double* dt_per_inst) = 0;
    virtual mpm_status metrics(int inst, mpm_metrics* out) = 0;
    virtual mpm_status set_mass_scaling(int inst, double f) = 0;
    virtual mpm_status ext_force(int inst, const double c[3], double r, const double f[3]) = 0;
    virtual mpm_status set_temps(int inst, const double* T, int64_t count) = 0;
    virtual mpm_status reset_clock(int inst) = 0;
    // Appends n_add instances and drops the listed ones; kept instances keep
    // their state (indices of the instances after a dropped one shift down).
    virtual mpm_status get_config(mpm_launch_config* c) = 0;
    virtual mpm_status set_config(const mpm_launch_config* c) = 0;
    virtual mpm_status autotune(const double* dt_per_inst, mpm_launch_config* best) = 0;
    virtual mpm_status reserve(int64_t particles, int64_t nodes, int64_t keys, int64_t bins, int max_inst,
                               bool backstress) = 0;
    virtual mpm_status change_instances(const mpm_params* params, const int64_t* caps, int n_add,
                                        const int32_t* remove, int n_remove, int* first) = 0;
    virtual mpm_status sync() = 0;
    // Status of every instance from its error word (MPM_OK, MPM_NUMERIC; all
    // MPM_TIMEOUT when a bounded wait gave up); synchronises the stream.
    virtual mpm_status inst_statuses(int32_t* out, int n) = 0;
    // Checkpoint of one instance (format: mpm_checkpoint.h).
    virtual mpm_status checkpoint_bytes(int inst, int64_t* bytes) = 0;
    virtual mpm_status checkpoint_save(int inst, void* buf, int64_t bytes) = 0;
    virtual mpm_status checkpoint_load(int inst, const void* buf, int64_t bytes) = 0;
    virtual int n_inst() const = 0;
    virtual const InstHost& inst(int i) const = 0;
    virtual cudaStream_t stream() const = 0;
    virtual int64_t launches() const = 0;
    virtual mpm_status profile_enable(bool on) = 0;
    virtual mpm_status profile_read(double* ms, int64_t* n) = 0;
};

// Creates an engine for n instances (all of the same precision; n may be 0,
// params[0] then only sets the precision and launch defaults).  Returns
// nullptr with a message in `err` on failure.
std::unique_ptr<EngineBase> make_engine(const mpm_params* params, const int64_t* caps, int n, cudaStream_t st,
                                        mpm_status* status, std::string* err);

mpm_status check_params(const mpm_params* p, std::string* err);

}  // namespace mpmb

// The opaque C handle.
struct mpm_handle {
    std::unique_ptr<mpmb::EngineBase> eng;
};
