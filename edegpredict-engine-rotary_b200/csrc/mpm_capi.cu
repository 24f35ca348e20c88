// mpm_capi.cu -- the extern "C" entry points of include/mpm_capi.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mpm_capi.h"
#include "mpm_engine.h"

namespace {

std::string& lib_err() {
    static thread_local std::string e;
    return e;
}

mpm_status fail(mpm_handle* h, mpm_status s, const std::string& m) {
    if (h && h->eng) h->eng->err = m;
    lib_err() = m;
    return s;
}

mpm_status ret(mpm_handle* h, mpm_status s) {
    if (s != MPM_OK && h && h->eng) lib_err() = h->eng->err;
    return s;
}

#define NEED_H(h)                                                              \
    do {                                                                       \
        if (!(h) || !(h)->eng) return fail(nullptr, MPM_INVALID_ARG, "handle is NULL"); \
    } while (0)

}  // namespace

namespace mpmb {
void set_lib_error(const std::string& m) { lib_err() = m; }
}  // namespace mpmb

extern "C" {

mpm_status mpm_params_default(mpm_params* p) {
    if (!p) return fail(nullptr, MPM_INVALID_ARG, "params is NULL");
    std::memset(p, 0, sizeof(*p));
    p->abi_version = MPM_ABI_VERSION;
    p->precision = MPM_PREC_F32;
    p->plasticity = MPM_PLAST_EXPLICIT;
    // MPMKernelConfig defaults (include/MPMSolver.cuh:64-73)
    p->E = 200e9;
    p->nu = 0.3;
    p->rho_phys = 7850.0;
    p->cp = 475.0;
    p->beta = 0.9;
    p->Tm = 1500.0;
    p->Tamb = 25.0;
    p->jc_A = 595e6;
    p->jc_B = 580e6;
    p->jc_n = 0.133;
    p->jc_C = 0.023;
    p->jc_m = 1.03;
    p->edot0 = 1.0;
    p->H_kin = 0.0;
    p->D1 = 0.06; p->D2 = 3.31; p->D3 = -1.96; p->D4 = 0.018; p->D5 = 0.58;
    p->D_th = 1.0;
    // MPMSolver members and constants (include/MPMSolver.cuh:253-254, src/MPMSolver.cu:16, :890)
    p->fixture_thickness = 0.002;
    p->fixture_damping = 1e7;
    p->gravity_z = -9.81;
    p->mass_threshold = 1e-12;
    p->apic_dinv_factor = 3.0;
    p->apic_decay = 0.99;
    p->deps_cap = 0.05;
    p->dT_cap = 50.0;
    p->lod_enabled = 0;
    p->lod_active_r = 0.002;
    p->lod_near_r = 0.01;
    p->chip_every = 2;
    p->newton_tol = 1e-12;
    p->newton_maxit = 60;
    p->schedule = MPM_SCHED_FUSED;
    p->sort_every = 16;
    p->threads_per_block = 128;
    // ContactConfig defaults (include/ContactSolver.cuh:30-34); off until contact_every > 0
    p->contact_every = 0;
    p->contact_radius = 0.0002;
    p->contact_friction = 0.3;
    p->contact_heat_partition = 0.5;
    // AdiabaticShearConfig defaults (include/Types.h:90-94); off as in the reference
    p->asb_enabled = 0;
    p->asb_critical_rate = 1e4;
    p->asb_taylor_quinney = 0.9;
    p->asb_max_temp_ratio = 0.9;
    p->asb_touch_rise = 0.5;
    // MPMMaterialParams::thermalConductivity (include/MPMWorkpieceSolver.cuh:88); off
    p->heat_conduction = 0;
    p->thermal_conductivity = 42.6;
    return MPM_OK;
}

mpm_status mpm_create(const mpm_params* p, int64_t capacity, void* stream, mpm_handle** out) {
    if (!out) return fail(nullptr, MPM_INVALID_ARG, "out is NULL");
    *out = nullptr;
    mpm_status s = MPM_OK;
    std::string e;
    auto eng = mpmb::make_engine(p, &capacity, 1, (cudaStream_t)stream, &s, &e);
    if (!eng) return fail(nullptr, s, e);
    *out = new mpm_handle{std::move(eng)};
    return MPM_OK;
}

mpm_status mpm_destroy(mpm_handle* h) {
    delete h;
    return MPM_OK;
}

mpm_status mpm_init_box(mpm_handle* h, const int32_t c0[3], const int32_t c1[3], int32_t ppc, uint64_t seed,
                        uint32_t instance, int32_t fixed_layers, double T0, const mpm_tool_desc* tool) {
    NEED_H(h);
    if (!c0 || !c1) return fail(h, MPM_INVALID_ARG, "cell box is NULL");
    return ret(h, h->eng->init_box(0, c0, c1, ppc, seed, instance, fixed_layers, T0, tool));
}

mpm_status mpm_upload(mpm_handle* h, const mpm_particles_soa* host, int64_t n) {
    NEED_H(h);
    return ret(h, h->eng->upload(0, host, n));
}

mpm_status mpm_download(mpm_handle* h, mpm_particles_soa* host) {
    NEED_H(h);
    return ret(h, h->eng->download(0, host));
}

mpm_status mpm_export_aos(mpm_handle* h, void* dst, int64_t dst_bytes) {
    NEED_H(h);
    return ret(h, h->eng->export_aos(0, dst, dst_bytes));
}

mpm_status mpm_import_aos(mpm_handle* h, const void* src, int64_t src_bytes, uint32_t fields) {
    NEED_H(h);
    return ret(h, h->eng->import_aos(0, src, src_bytes, fields));
}

mpm_status mpm_set_tool(mpm_handle* h, const mpm_tool_desc* tool) {
    NEED_H(h);
    return ret(h, h->eng->set_tool(0, tool));
}

mpm_status mpm_set_tool_nodes(mpm_handle* h, const mpm_tool_nodes* nodes) {
    NEED_H(h);
    return ret(h, h->eng->set_tool_nodes(0, nodes));
}

mpm_status mpm_set_workpiece_semantics(mpm_handle* h, const mpm_workpiece_params* params) {
    NEED_H(h);
    return ret(h, h->eng->set_workpiece_semantics(params));
}

mpm_status mpm_step(mpm_handle* h, double dt, int32_t nsteps) {
    NEED_H(h);
    if (h->eng->n_inst() == 1) return ret(h, h->eng->step(nsteps, &dt));
    std::vector<double> dts((size_t)h->eng->n_inst(), dt);
    return ret(h, h->eng->step(nsteps, dts.data()));
}

mpm_status mpm_stable_dt(const mpm_handle* h, double cfl, double* dt) {
    if (!h || !h->eng || !dt) return fail(nullptr, MPM_INVALID_ARG, "handle or output is NULL");
    const mpm_params& p = h->eng->inst(0).p;
    const double rho = p.particle_mass / p.particle_volume;
    const double c = std::sqrt(p.E / rho);
    *dt = std::fmax(cfl * p.dx / std::fmax(c, 1.0), 1e-10);
    return MPM_OK;
}

mpm_status mpm_sync_metrics(mpm_handle* h, mpm_metrics* out) {
    NEED_H(h);
    return ret(h, h->eng->metrics(0, out));
}

mpm_status mpm_set_mass_scaling(mpm_handle* h, double factor) {
    NEED_H(h);
    return ret(h, h->eng->set_mass_scaling(0, factor));
}

mpm_status mpm_apply_external_force(mpm_handle* h, const double center[3], double radius, const double force[3]) {
    NEED_H(h);
    return ret(h, h->eng->ext_force(0, center, radius, force));
}

mpm_status mpm_set_temperatures(mpm_handle* h, const double* temperatures, int64_t count) {
    NEED_H(h);
    return ret(h, h->eng->set_temps(0, temperatures, count));
}

mpm_status mpm_get_counts(const mpm_handle* h, int64_t* n_particles, int64_t* n_steps, double* time) {
    if (!h || !h->eng) return fail(nullptr, MPM_INVALID_ARG, "handle is NULL");
    const auto& x = h->eng->inst(0);
    if (n_particles) *n_particles = x.np;
    if (n_steps) *n_steps = x.step;
    if (time) *time = x.time;
    return MPM_OK;
}

mpm_status mpm_get_stream(const mpm_handle* h, void** stream) {
    if (!h || !h->eng || !stream) return fail(nullptr, MPM_INVALID_ARG, "handle or output is NULL");
    *stream = (void*)h->eng->stream();
    return MPM_OK;
}

mpm_status mpm_reset_clock(mpm_handle* h) {
    NEED_H(h);
    return ret(h, h->eng->reset_clock(0));
}

// ---------------------------------------------------------------- batched form

#define NEED_I(h, i)                                                                                  \
    do {                                                                                              \
        NEED_H(h);                                                                                    \
        if ((i) < 0 || (i) >= (h)->eng->n_inst()) return fail(h, MPM_INVALID_ARG, "instance index out of range"); \
    } while (0)

mpm_status mpm_batch_create(const mpm_params* params, const int64_t* capacities, int32_t n_instances, void* stream,
                            mpm_handle** out) {
    if (!out) return fail(nullptr, MPM_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!params || !capacities || n_instances <= 0)
        return fail(nullptr, MPM_INVALID_ARG, "a batch needs at least one instance");
    mpm_status s = MPM_OK;
    std::string e;
    auto eng = mpmb::make_engine(params, capacities, n_instances, (cudaStream_t)stream, &s, &e);
    if (!eng) return fail(nullptr, s, e);
    *out = new mpm_handle{std::move(eng)};
    return MPM_OK;
}

mpm_status mpm_batch_count(const mpm_handle* h, int32_t* n_instances) {
    if (!h || !h->eng || !n_instances) return fail(nullptr, MPM_INVALID_ARG, "handle or output is NULL");
    *n_instances = h->eng->n_inst();
    return MPM_OK;
}

mpm_status mpm_batch_init_box(mpm_handle* h, int32_t inst, const int32_t c0[3], const int32_t c1[3], int32_t ppc,
                              uint64_t seed, uint32_t instance_key, int32_t fixed_layers, double T0,
                              const mpm_tool_desc* tool_at_t0) {
    NEED_I(h, inst);
    if (!c0 || !c1) return fail(h, MPM_INVALID_ARG, "cell box is NULL");
    return ret(h, h->eng->init_box(inst, c0, c1, ppc, seed, instance_key, fixed_layers, T0, tool_at_t0));
}

mpm_status mpm_batch_upload(mpm_handle* h, int32_t inst, const mpm_particles_soa* host, int64_t n) {
    NEED_I(h, inst);
    return ret(h, h->eng->upload(inst, host, n));
}

mpm_status mpm_batch_download(mpm_handle* h, int32_t inst, mpm_particles_soa* host) {
    NEED_I(h, inst);
    return ret(h, h->eng->download(inst, host));
}

mpm_status mpm_batch_export_aos(mpm_handle* h, int32_t inst, void* dst, int64_t dst_bytes) {
    NEED_I(h, inst);
    return ret(h, h->eng->export_aos(inst, dst, dst_bytes));
}

mpm_status mpm_batch_import_aos(mpm_handle* h, int32_t inst, const void* src, int64_t src_bytes, uint32_t fields) {
    NEED_I(h, inst);
    return ret(h, h->eng->import_aos(inst, src, src_bytes, fields));
}

mpm_status mpm_set_tool_sdf(mpm_handle* h, const mpm_tool_sdf* sdf) {
    NEED_H(h);
    return ret(h, h->eng->set_tool_sdf(0, sdf));
}

mpm_status mpm_batch_set_tool_nodes(mpm_handle* h, int32_t inst, const mpm_tool_nodes* nodes) {
    NEED_I(h, inst);
    return ret(h, h->eng->set_tool_nodes(inst, nodes));
}

mpm_status mpm_batch_set_tool_sdf(mpm_handle* h, int32_t inst, const mpm_tool_sdf* sdf) {
    NEED_I(h, inst);
    return ret(h, h->eng->set_tool_sdf(inst, sdf));
}

mpm_status mpm_batch_set_tool(mpm_handle* h, int32_t inst, const mpm_tool_desc* tool) {
    NEED_I(h, inst);
    return ret(h, h->eng->set_tool(inst, tool));
}

mpm_status mpm_batch_step(mpm_handle* h, const double* dt, int32_t nsteps) {
    NEED_H(h);
    if (!dt) return fail(h, MPM_INVALID_ARG, "dt is NULL");
    return ret(h, h->eng->step(nsteps, dt));
}

mpm_status mpm_batch_sync_metrics(mpm_handle* h, int32_t inst, mpm_metrics* out) {
    NEED_I(h, inst);
    return ret(h, h->eng->metrics(inst, out));
}

mpm_status mpm_checkpoint_bytes(mpm_handle* h, int32_t inst, int64_t* bytes) {
    NEED_I(h, inst);
    if (!bytes) return fail(h, MPM_INVALID_ARG, "bytes is NULL");
    return ret(h, h->eng->checkpoint_bytes(inst, bytes));
}

mpm_status mpm_checkpoint_save(mpm_handle* h, int32_t inst, void* buf, int64_t bytes) {
    NEED_I(h, inst);
    return ret(h, h->eng->checkpoint_save(inst, buf, bytes));
}

mpm_status mpm_checkpoint_load(mpm_handle* h, int32_t inst, const void* buf, int64_t bytes) {
    NEED_I(h, inst);
    return ret(h, h->eng->checkpoint_load(inst, buf, bytes));
}

mpm_status mpm_batch_instance_status(mpm_handle* h, int32_t* status, int32_t n) {
    NEED_H(h);
    if (!status) return fail(h, MPM_INVALID_ARG, "status array is NULL");
    return ret(h, h->eng->inst_statuses(status, n));
}

mpm_status mpm_batch_get_counts(const mpm_handle* h, int32_t inst, int64_t* n_particles, int64_t* n_steps,
                                double* time) {
    if (!h || !h->eng) return fail(nullptr, MPM_INVALID_ARG, "handle is NULL");
    if (inst < 0 || inst >= h->eng->n_inst()) return fail(nullptr, MPM_INVALID_ARG, "instance index out of range");
    const auto& x = h->eng->inst(inst);
    if (n_particles) *n_particles = x.np;
    if (n_steps) *n_steps = x.step;
    if (time) *time = x.time;
    return MPM_OK;
}

mpm_status mpm_batch_change(mpm_handle* h, const mpm_params* add, const int64_t* add_capacities, int32_t n_add,
                            const int32_t* remove, int32_t n_remove, int32_t* first_added) {
    NEED_H(h);
    if (n_add < 0 || n_remove < 0) return fail(h, MPM_INVALID_ARG, "negative count");
    if (n_add > 0 && (!add || !add_capacities)) return fail(h, MPM_INVALID_ARG, "new instances need parameters");
    if (n_remove > 0 && !remove) return fail(h, MPM_INVALID_ARG, "remove list is NULL");
    int first = 0;
    mpm_status s = h->eng->change_instances(add, add_capacities, n_add, remove, n_remove, &first);
    if (s == MPM_OK && first_added) *first_added = first;
    return ret(h, s);
}

mpm_status mpm_get_launch_config(const mpm_handle* h, mpm_launch_config* out) {
    if (!h || !h->eng || !out) return fail(nullptr, MPM_INVALID_ARG, "handle or output is NULL");
    return h->eng->get_config(out);
}

mpm_status mpm_set_launch_config(mpm_handle* h, const mpm_launch_config* cfg) {
    NEED_H(h);
    return ret(h, h->eng->set_config(cfg));
}

mpm_status mpm_autotune(mpm_handle* h, const double* dt, mpm_launch_config* chosen) {
    NEED_H(h);
    if (!dt) return fail(h, MPM_INVALID_ARG, "dt is NULL");
    return ret(h, h->eng->autotune(dt, chosen));
}

mpm_status mpm_selftest_bounded_wait(int64_t limit_ns, void* stream) {
    if (limit_ns < 1000000 || limit_ns > 1000000000)
        return fail(nullptr, MPM_INVALID_ARG, "limit_ns must be in [1e6, 1e9]");
    std::string e;
    const mpm_status s = mpmb::wait_selftest(limit_ns, (cudaStream_t)stream, &e);
    lib_err() = e;
    return s;
}

mpm_status mpm_profile_enable(mpm_handle* h, int32_t enable) {
    NEED_H(h);
    return ret(h, h->eng->profile_enable(enable != 0));
}

mpm_status mpm_profile_read(mpm_handle* h, double* kernel_ms, int64_t* kernel_launches) {
    NEED_H(h);
    if (!kernel_ms || !kernel_launches) return fail(h, MPM_INVALID_ARG, "output is NULL");
    return ret(h, h->eng->profile_read(kernel_ms, kernel_launches));
}

mpm_status mpm_launch_count(const mpm_handle* h, int64_t* count) {
    if (!h || !h->eng || !count) return fail(nullptr, MPM_INVALID_ARG, "handle or output is NULL");
    *count = h->eng->launches();
    return MPM_OK;
}

const char* mpm_last_error(const mpm_handle* h) {
    if (h && h->eng && !h->eng->err.empty()) return h->eng->err.c_str();
    return lib_err().c_str();
}

const char* mpm_status_string(mpm_status s) {
    switch (s) {
        case MPM_OK: return "MPM_OK";
        case MPM_INVALID_ARG: return "MPM_INVALID_ARG";
        case MPM_OOM: return "MPM_OOM";
        case MPM_CUDA_ERROR: return "MPM_CUDA_ERROR";
        case MPM_NUMERIC: return "MPM_NUMERIC";
        case MPM_OUT_OF_GRID: return "MPM_OUT_OF_GRID";
        case MPM_TIMEOUT: return "MPM_TIMEOUT";
        case MPM_NOT_SUPPORTED: return "MPM_NOT_SUPPORTED";
        case MPM_CAPACITY: return "MPM_CAPACITY";
        case MPM_CANCELLED: return "MPM_CANCELLED";
    }
    return "unknown";
}

}  // extern "C"
