// mpm_server.cu -- the serving loop's C ABI (include/mpm_capi.h, mpm_server_*):
// the scheduler of mpm_server_core.h over one batch engine whose pools are
// reserved from the HBM budget when the server is created.
#include <cuda_runtime.h>

#include <chrono>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mpm_capi.h"
#include "mpm_engine.h"
#include "mpm_internal.h"
#include "mpm_server_core.h"

namespace mpmb {
namespace {

// The scheduler's engine operations on the GPU engine.
struct GpuOps {
    EngineBase* e = nullptr;
    mpm_status change(const std::vector<mpm_params>& add, const std::vector<int64_t>& caps,
                      const std::vector<int32_t>& remove, int* first) {
        return e->change_instances(add.data(), caps.data(), (int)add.size(), remove.data(), (int)remove.size(),
                                   first);
    }
    mpm_status init(int inst, const mpm_request& r, int64_t* np) {
        const mpm_status s = e->init_box(inst, r.c0, r.c1, r.ppc, r.seed, r.instance_key, r.fixed_layers, r.T0,
                                         r.tool.mode != MPM_TOOL_NONE ? &r.tool : nullptr);
        *np = e->inst(inst).np;
        return s;
    }
    mpm_status step(int k, const std::vector<double>& dts) { return e->step(k, dts.data()); }
    mpm_status metrics(int inst, mpm_metrics* m) { return e->metrics(inst, m); }
    mpm_status health(std::vector<int32_t>& st) { return e->inst_statuses(st.data(), (int)st.size()); }
    mpm_status save(int inst, std::vector<unsigned char>* buf) {
        int64_t n = 0;
        mpm_status s = e->checkpoint_bytes(inst, &n);
        if (s != MPM_OK) return s;
        buf->resize((size_t)n);
        return e->checkpoint_save(inst, buf->data(), n);
    }
    mpm_status restore(int inst, const std::vector<unsigned char>& buf, int64_t* np) {
        const mpm_status s = e->checkpoint_load(inst, buf.data(), (int64_t)buf.size());
        *np = e->inst(inst).np;
        return s;
    }
};

mpm_status fail(mpm_status s, const std::string& m) {
    set_lib_error("mpm_server: " + m);
    return s;
}

}  // namespace
}  // namespace mpmb

struct mpm_server {
    mpm_server_config cfg{};
    std::unique_ptr<mpmb::EngineBase> eng;
    mpmb::GpuOps ops;
    std::unique_ptr<mpmb::Scheduler<mpmb::GpuOps>> sched;
    std::chrono::steady_clock::time_point t0;
};

extern "C" {

mpm_status mpm_server_footprint(const mpm_server_config* cfg, const mpm_request* req, int64_t* bytes) {
    if (!cfg || !req || !bytes) return mpmb::fail(MPM_INVALID_ARG, "NULL argument");
    const mpmb::Footprint f = mpmb::request_footprint(*req);
    const mpmb::PoolBytes b = mpmb::pool_bytes(cfg->precision, cfg->backstress != 0, cfg->deterministic != 0);
    *bytes = (int64_t)(f.particles * b.particle + f.nodes * b.node + f.keys * b.key + f.bins * b.bin);
    return MPM_OK;
}

mpm_status mpm_server_create(const mpm_server_config* cfg, void* stream, mpm_server** out) {
    using namespace mpmb;
    if (!cfg || !out) return fail(MPM_INVALID_ARG, "config or output is NULL");
    *out = nullptr;
    if (cfg->precision != MPM_PREC_F32 && cfg->precision != MPM_PREC_F64)
        return fail(MPM_INVALID_ARG, "precision must be F32 or F64");
    if (cfg->hbm_budget_bytes < ((int64_t)1 << 26)) return fail(MPM_INVALID_ARG, "hbm_budget_bytes below 64 MiB");
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return fail(MPM_CUDA_ERROR, "cudaMemGetInfo failed (no device?)");
    }
    if ((size_t)cfg->hbm_budget_bytes > free_b)
        return fail(MPM_OOM, "hbm_budget_bytes (" + std::to_string(cfg->hbm_budget_bytes) +
                                 ") exceeds free device memory (" + std::to_string(free_b) + ")");
    // an engine without instances; params only set the precision
    mpm_params tmpl;
    mpm_params_default(&tmpl);
    tmpl.precision = cfg->precision;
    tmpl.nx = tmpl.ny = tmpl.nz = 8;
    tmpl.dx = 1e-4;
    tmpl.particle_mass = tmpl.particle_volume = 1.0;
    mpm_status s = MPM_OK;
    std::string e;
    auto eng = make_engine(&tmpl, nullptr, 0, (cudaStream_t)stream, &s, &e);
    if (!eng) return fail(s, e);
    const Pools pools =
        pools_for_budget(cfg->hbm_budget_bytes, cfg->precision, cfg->backstress != 0, cfg->deterministic != 0);
    const int max_res = cfg->max_resident > 0 ? cfg->max_resident : 4096;
    s = eng->reserve(pools.particles, pools.nodes, pools.keys, pools.bins, max_res, cfg->backstress != 0);
    if (s != MPM_OK) return fail(s, "reserving the pools: " + eng->err);
    mpm_launch_config lc;
    eng->get_config(&lc);
    lc.use_graph = cfg->use_graph ? 1 : 0;
    lc.deterministic = cfg->deterministic ? 1 : 0;
    eng->set_config(&lc);
    auto* srv = new mpm_server;
    srv->cfg = *cfg;
    srv->eng = std::move(eng);
    srv->ops.e = srv->eng.get();
    srv->t0 = std::chrono::steady_clock::now();
    const auto t0 = srv->t0;
    srv->sched = std::make_unique<Scheduler<GpuOps>>(
        &srv->ops, pools, cfg->max_chunk, max_res,
        [t0]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); },
        cfg->max_resident_particles);
    *out = srv;
    return MPM_OK;
}

mpm_status mpm_server_destroy(mpm_server* s) {
    delete s;
    return MPM_OK;
}

mpm_status mpm_server_submit(mpm_server* s, const mpm_request* req, int64_t* id) {
    using namespace mpmb;
    if (!s || !req) return fail(MPM_INVALID_ARG, "server or request is NULL");
    std::string e;
    mpm_status st = check_params(&req->params, &e);
    if (st != MPM_OK) return fail(st, "request params: " + e);
    if (req->params.precision != s->cfg.precision) return fail(MPM_INVALID_ARG, "request precision differs from the server's");
    if (req->params.H_kin > 0.0 && !s->cfg.backstress)
        return fail(MPM_NOT_SUPPORTED, "H_kin > 0 needs a server created with backstress = 1");
    if (req->tool.mode == MPM_TOOL_RASTER)
        return fail(MPM_NOT_SUPPORTED, "raster tools are not served (the samples are not kept); use an SDF tool");
    st = s->sched->submit(*req, id);
    if (st == MPM_CAPACITY) return fail(st, "the request's footprint exceeds the server's pools");
    if (st != MPM_OK) return fail(st, "nsteps >= 0, finite dt > 0, ppc > 0 and a finite T0 required");
    return MPM_OK;
}

mpm_status mpm_server_tick(mpm_server* s, int32_t* n_resident) {
    if (!s) return mpmb::fail(MPM_INVALID_ARG, "server is NULL");
    mpmb::Range nvtx_range("mpm.server_tick");
    const mpm_status st = s->sched->tick(n_resident);
    if (st != MPM_OK) return mpmb::fail(st, s->eng->err);
    return MPM_OK;
}

mpm_status mpm_server_poll(mpm_server* s, int64_t id, mpm_result* out) {
    if (!s || !out) return mpmb::fail(MPM_INVALID_ARG, "server or output is NULL");
    const mpm_status st = s->sched->poll(id, out);
    if (st != MPM_OK) return mpmb::fail(st, "unknown request id");
    return MPM_OK;
}

mpm_status mpm_server_cancel(mpm_server* s, int64_t id) {
    if (!s) return mpmb::fail(MPM_INVALID_ARG, "server is NULL");
    const mpm_status st = s->sched->cancel(id);
    if (st != MPM_OK) return mpmb::fail(st, "unknown request id");
    return MPM_OK;
}

mpm_status mpm_server_preempt(mpm_server* s, int64_t id) {
    if (!s) return mpmb::fail(MPM_INVALID_ARG, "server is NULL");
    const mpm_status st = s->sched->preempt(id);
    if (st != MPM_OK) return mpmb::fail(st, "unknown request id or the request is not running");
    return MPM_OK;
}

mpm_status mpm_server_stats_get(mpm_server* s, mpm_server_stats* out) {
    if (!s || !out) return mpmb::fail(MPM_INVALID_ARG, "server or output is NULL");
    *out = s->sched->stats();
    return MPM_OK;
}

}  // extern "C"
