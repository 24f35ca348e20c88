// mpm_engine.cu -- host engine: device memory, TMA descriptors, the step
// schedule, re-binning, upload/download and metrics.  One engine holds one or
// more workpiece instances (the plain C ABI uses one).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "mpm_engine.h"
#include "mpm_checkpoint.h"

namespace mpmb {

namespace {

typedef CUresult (*PFN_encodeTiled_t)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                      const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

PFN_encodeTiled_t encode_fn() {
    static PFN_encodeTiled_t fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_encodeTiled_t)p;
    }
    return fn;
}

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                                \
            return e_ == cudaErrorMemoryAllocation ? MPM_OOM : MPM_CUDA_ERROR;                       \
        }                                                                                            \
    } while (0)

#define MS(call)                     \
    do {                             \
        mpm_status s_ = (call);      \
        if (s_ != MPM_OK) return s_; \
    } while (0)

}  // namespace

mpm_status check_params(const mpm_params* p, std::string* err) {
    auto bad = [&](const char* m) {
        *err = m;
        return MPM_INVALID_ARG;
    };
    if (!p) return bad("params is NULL");
    if (p->abi_version != MPM_ABI_VERSION) return bad("params.abi_version does not match MPM_ABI_VERSION");
    if (p->precision != MPM_PREC_F32 && p->precision != MPM_PREC_F64) return bad("precision must be F32 or F64");
    if (p->nx < 8 || p->ny < 8 || p->nz < 8) return bad("grid needs at least 8 nodes per axis");
    if ((int64_t)p->nx * p->ny * p->nz > (int64_t)1 << 31) return bad("grid larger than 2^31 nodes");
    if (!(p->dx > 0.0) || !std::isfinite(p->dx)) return bad("dx must be positive");
    if (!(p->particle_mass > 0.0) || !(p->particle_volume > 0.0)) return bad("particle mass and volume must be positive");
    if (!(p->E > 0.0) || !(p->nu > -1.0 && p->nu < 0.5)) return bad("E > 0 and -1 < nu < 0.5 required");
    if (!(p->D_th > 0.0)) return bad("D_th must be positive");
    if (p->plasticity != MPM_PLAST_EXPLICIT && p->plasticity != MPM_PLAST_NEWTON) return bad("plasticity mode");
    if (p->schedule != MPM_SCHED_FUSED && p->schedule != MPM_SCHED_SPLIT) return bad("schedule");
    if (p->threads_per_block < 0 || p->threads_per_block > 256 || (p->threads_per_block % 32) != 0)
        return bad("threads_per_block must be 0 or a multiple of 32 up to 256");
    if (p->contact_every < 0) return bad("contact_every must be >= 0");
    if (p->contact_every > 0 && (!(p->contact_radius > 0.0) || !(p->contact_friction >= 0.0) ||
                                 !(p->contact_heat_partition >= 0.0 && p->contact_heat_partition <= 1.0)))
        return bad("contact needs radius > 0, friction >= 0 and 0 <= heat partition <= 1");
    if (p->asb_enabled && (!(p->asb_critical_rate >= 0.0) || !(p->asb_taylor_quinney >= 0.0) ||
                           !(p->asb_max_temp_ratio > 0.0) || !(p->asb_touch_rise >= 0.0)))
        return bad("adiabatic shear model needs critical rate >= 0, Taylor-Quinney >= 0, max temperature ratio > 0 "
                   "and touch rise >= 0");
    if (p->heat_conduction && (!(p->thermal_conductivity >= 0.0) || !(p->rho_phys * p->cp > 0.0)))
        return bad("heat conduction needs thermal_conductivity >= 0 and rho_phys * cp > 0");
    return MPM_OK;
}

template <typename R>
class Engine final : public EngineBase {
   public:
    std::vector<InstHost> I;
    cudaStream_t st = nullptr;
    bool own_st = false;
    int64_t cap_total = 0, nn_total = 0, nkeys = 0;
    // allocated sizes (grow-only)
    int64_t pcap_alloc = -1, pcap_alloc_next = 0, nn_alloc = 0, scan_alloc = 0, map_alloc = 0;
    int64_t slot_alloc[4] = {0, 0, 0, 0}, key_alloc[2] = {0, 0}, bin_alloc[6] = {0, 0, 0, 0, 0, 0};
    int64_t inst_alloc[3] = {0, 0, 0};
    RelayoutMap* d_map = nullptr;
    void* pbuf[2] = {nullptr, nullptr};
    PState<R> ps[2];
    int cur = 0;
    bool has_K = false;
    V4<R>* gpool[2] = {nullptr, nullptr};
    // heat conduction node arrays, beside the grids: T m scatter (two buffers, paired with
    // gpool) and the node temperatures after the diffusion step
    R* tpool[3] = {nullptr, nullptr, nullptr};
    int32_t* mask_pool = nullptr;     // raster marks per grid node (Inst::tool_mask)
    Inst<R>* d_inst = nullptr;
    std::vector<Inst<R>> h_inst;
    int32_t *d_key_base = nullptr, *d_bin_key = nullptr, *d_bin_inst = nullptr, *d_bin_local = nullptr;
    int64_t* d_inst_pbase = nullptr;
    int32_t *d_key = nullptr, *d_rank = nullptr, *d_newbin = nullptr, *d_count = nullptr, *d_offset = nullptr;
    int32_t* d_perm = nullptr;     // re-bin: source slot of every destination slot, then its upload position
    int64_t perm_alloc = 0;
    int32_t *d_flag = nullptr, *d_flag_scan = nullptr, *d_scan_tmp = nullptr;
    double* d_pos = nullptr;
    Work* d_work = nullptr;
    int* d_nwork = nullptr;
    int max_work = 0;
    int* d_err = nullptr;          // the handle's error word (ERR_TIMEOUT)
    int* d_ierr = nullptr;         // one error word per instance (ERR_NUMERIC, ERR_NEWTON)
    int64_t ierr_alloc = 0;
    unsigned long long* d_ctr = nullptr;
    static constexpr size_t kCtrBytes = 4 * sizeof(unsigned long long) + 2 * sizeof(double);
    double *d_stat_part = nullptr, *d_stat_out = nullptr;
    int stat_blocks = 0;
    void* d_stage = nullptr;
    size_t stage_bytes = 0;
    V4<R>* d_pext = nullptr;       // per-particle external force of an AoS import (pbase + upload order)
    int64_t pext_alloc = 0;
    int* d_flags = nullptr;        // AoS import: [0] a particle moved, [1] records with an invalid status
    bool ws_on = false;            // MPMWorkpieceSolver's step semantics
    mpm_workpiece_params ws{};
    int32_t* d_gen = nullptr;
    size_t gen_bytes = 0;
    bool binned = false;
    int64_t n_sorts = 0;
    int64_t launch_base = 0;
    int sort_every = 16, threads = 128, ctas_per_sm = 4, prec_ = MPM_PREC_F32;
    static constexpr int kDefaultPassChunk = 1;
    int pass_chunk = kDefaultPassChunk;   // FP32 particles per pass of the step kernel / 128
    bool use_graph = false;
    int rbuf = 0;
    // deterministic mode (mpm_launch_config.deterministic): every work item's
    // node tile (kPartCh x kTileNodes values), the escaped fixed-point node
    // sums (kPartCh x nn_total) and their per-bin marks
    bool det = true;
    R* d_part = nullptr;
    int64_t part_alloc = 0;
    unsigned long long* d_esc = nullptr;
    int64_t esc_alloc = 0;
    int32_t* d_esc_flag = nullptr;
    int64_t esc_flag_alloc = 0;
    // step-kernel timing (mpm_profile_enable)
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;

    void prof_begin() {
        if (!prof) return;
        if (ev_used + 2 > ev_pool.size()) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            ev_pool.push_back(a);
            ev_pool.push_back(b);
        }
        cudaEventRecord(ev_pool[ev_used], st);
    }
    void prof_end() {
        if (!prof) return;
        cudaEventRecord(ev_pool[ev_used + 1], st);
        ev_used += 2;
    }
    mpm_status profile_enable(bool on) override {
        prof = on;
        return MPM_OK;
    }
    mpm_status profile_read(double* ms, int64_t* n) override {
        CK(cudaStreamSynchronize(st));
        double tot = 0.0;
        for (size_t k = 0; k + 1 < ev_used; k += 2) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, ev_pool[k], ev_pool[k + 1]));
            tot += t;
        }
        *ms = tot;
        *n = (int64_t)(ev_used / 2);
        ev_used = 0;
        return MPM_OK;
    }

    ~Engine() override {
        if (st) cudaStreamSynchronize(st);
        drop_graphs();
        void* ptrs[] = {pbuf[0], pbuf[1], gpool[0], gpool[1], tpool[0], tpool[1], tpool[2], mask_pool, d_inst,
                        d_key_base, d_bin_key, d_bin_inst,
                        d_bin_local,
                        d_inst_pbase, d_key, d_rank, d_newbin, d_count, d_offset, d_flag, d_flag_scan, d_scan_tmp,
                        d_pos, d_work, d_nwork, d_err, d_ierr, d_ctr, d_stat_part, d_stat_out, d_stage, d_gen,
                        d_map, d_perm, d_part, d_esc, d_esc_flag, d_pext, d_flags};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        for (auto& x : I)
            if (x.d_samples) cudaFree(x.d_samples);
        for (auto e : ev_pool) cudaEventDestroy(e);
        if (own_st && st) cudaStreamDestroy(st);
    }

    int n_inst() const override { return (int)I.size(); }
    const InstHost& inst(int i) const override { return I[i]; }
    cudaStream_t stream() const override { return st; }
    int64_t launches() const override { return launch_counter() - launch_base; }

    // ---------------------------------------------------------------- setup

    mpm_status init(const mpm_params* params, const int64_t* caps, int n, cudaStream_t stream_in) {
        launch_base = launch_counter();
        std::vector<InstHost> nI;
        mpm_status s = check_params(&params[0], &err);
        if (s != MPM_OK) return s;
        prec_ = params[0].precision;
        s = make_insts(params, caps, n, &nI);
        if (s != MPM_OK) return s;
        sort_every = params[0].sort_every > 0 ? params[0].sort_every : 16;
        threads = params[0].threads_per_block > 0 ? params[0].threads_per_block : 128;
        if (stream_in) {
            st = stream_in;
        } else {
            CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            own_st = true;
        }
        CK(cudaMalloc(&d_nwork, sizeof(int)));
        CK(cudaMemsetAsync(d_nwork, 0, sizeof(int), st));
        CK(cudaMalloc(&d_err, sizeof(int)));
        CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
        // counters: [0] escaped updates, [1] yields, [2] contacts, [3] adiabatic shear heatings,
        // then two FP64 sums (contact friction work, contact normal force)
        CK(cudaMalloc(&d_ctr, kCtrBytes));
        CK(cudaMemsetAsync(d_ctr, 0, kCtrBytes, st));
        stat_blocks = 148 * 8;   // 8 CTAs per SM of the metrics reduction (more loads in flight)
        CK(cudaMalloc(&d_stat_part, sizeof(double) * kStatSlots * stat_blocks));
        CK(cudaMalloc(&d_stat_out, sizeof(double) * kStatSlots));
        return relayout(std::move(nI), std::vector<int>(n, -1));
    }

    // Host records of new instances (validated, default tool, clock at 0).
    mpm_status make_insts(const mpm_params* params, const int64_t* caps, int n, std::vector<InstHost>* out) {
        out->assign(n, InstHost{});
        for (int i = 0; i < n; ++i) {
            mpm_status s = check_params(&params[i], &err);
            if (s != MPM_OK) return s;
            if (params[i].precision != prec_) {
                err = "all instances of an engine share one precision";
                return MPM_INVALID_ARG;
            }
            if (caps[i] < 0 || caps[i] > ((int64_t)1 << 31) - 1) {
                err = "capacity out of range";
                return MPM_INVALID_ARG;
            }
            InstHost& x = (*out)[i];
            x.p = params[i];
            x.cap = caps[i];
            x.tool = mpm_tool_desc{};
            x.tool.mode = MPM_TOOL_NONE;
        }
        return MPM_OK;
    }

    // Grow-only device buffer: reallocates (contents dropped) when `need`
    // elements do not fit, with a quarter of headroom.
    template <typename T>
    mpm_status grow(T*& p, int64_t& have, int64_t need, bool headroom = true) {
        need = std::max<int64_t>(need, 1);
        if (p && need <= have) return MPM_OK;
        if (p) cudaFree(p);
        p = nullptr;
        const int64_t n = headroom ? need + need / 4 : need;
        CK(cudaMalloc(&p, sizeof(T) * n));
        have = n;
        return MPM_OK;
    }

    static constexpr bool kPosLo = sizeof(R) == 4;   // FP32 state keeps position low parts
    static size_t pstate_bytes(int64_t cp, bool withK) {
        const size_t v4 = sizeof(V4<R>);
        return (12 + (kPosLo ? 1 : 0)) * al256(v4 * cp) + (withK ? 2 * al256(v4 * cp) : 0) + al256(sizeof(R) * cp) +
               2 * al256(cp) + 4 * al256(4 * cp);
    }
    static void carve(void* base, int64_t cp, bool withK, PState<R>& s) {
        char* q = (char*)base;
        const size_t v4 = sizeof(V4<R>);
        auto take = [&](size_t bytes) {
            void* r = q;
            q += al256(bytes);
            return r;
        };
        for (int k = 0; k < 6; ++k) s.A[k] = (V4<R>*)take(v4 * cp);
        for (int k = 0; k < 4; ++k) s.B[k] = (V4<R>*)take(v4 * cp);
        for (int k = 0; k < 2; ++k) s.S[k] = (V4<R>*)take(v4 * cp);
        for (int k = 0; k < 2; ++k) s.K[k] = withK ? (V4<R>*)take(v4 * cp) : nullptr;
        s.X = kPosLo ? (V4<R>*)take(v4 * cp) : nullptr;
        s.sres = (R*)take(sizeof(R) * cp);
        s.status = (uint8_t*)take(cp);
        s.asb = (uint8_t*)take(cp);
        s.id = (int32_t*)take(4 * cp);
        s.bin = (int32_t*)take(4 * cp);
        s.orig = (int32_t*)take(4 * cp);
        s.skey = (int32_t*)take(4 * cp);
    }

    // Replaces the instance set by nI; from[j] is the old index of new
    // instance j (-1: new, empty).  Instances are laid out contiguously in
    // the new order: particle slots [pbase, pbase + cap), grid nodes, sort keys
    // (bin*64 + cell per bin, then the INACTIVE sentinel and the unused-slot
    // pad) and bins.  The particles of kept instances move to their new slots
    // in one copy into the other state buffer; grids are not carried (every
    // step call starts from a cleared grid).  Allocations only grow.  The next
    // step re-bins.
    mpm_status relayout(std::vector<InstHost> nI, const std::vector<int>& from) {
        Range nvtx_range("mpm.relayout");
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        const int n = (int)nI.size();
        // error words follow their instances; new instances start clean
        std::vector<int> old_words(I.size(), 0), words(n, 0);
        if (!I.empty() && d_ierr)
            CK(cudaMemcpy(old_words.data(), d_ierr, sizeof(int) * I.size(), cudaMemcpyDeviceToHost));
        for (int j = 0; j < n; ++j)
            if (from[j] >= 0) words[j] = old_words[from[j]];
        std::vector<RelayoutMap> map(n);
        std::vector<char> kept(I.size(), 0);
        bool any_kept = false;
        for (int j = 0; j < n; ++j) {
            map[j].old_pbase = 0;
            map[j].np = 0;
            if (from[j] >= 0) {
                kept[from[j]] = 1;
                map[j].old_pbase = I[from[j]].pbase;
                map[j].np = I[from[j]].np;
                any_kept |= I[from[j]].np > 0;
            }
        }
        for (size_t i = 0; i < I.size(); ++i)
            if (!kept[i] && I[i].d_samples) {
                cudaFree(I[i].d_samples);
                I[i].d_samples = nullptr;
            }
        I = std::move(nI);
        // layout
        int64_t pb = 0, go = 0, kb = 0;
        bool wantK = false;
        std::vector<int32_t> key_base(n), bin_key, bin_inst, bin_local;
        std::vector<int64_t> inst_pbase(n);
        for (int i = 0; i < n; ++i) {
            InstHost& x = I[i];
            // a pending imported per-particle force is indexed by the old slot
            // range: an instance change drops it
            x.pext_pending = false;
            x.pbase = pb;
            pb += x.cap;
            x.nn = (int64_t)x.p.nx * x.p.ny * x.p.nz;
            x.grid_off = go;
            go += x.nn;
            x.nbx = (x.p.nx + kBin - 1) / kBin;
            x.nby = (x.p.ny + kBin - 1) / kBin;
            x.nbz = (x.p.nz + kBin - 1) / kBin;
            const int64_t nbins = (int64_t)x.nbx * x.nby * x.nbz;
            x.bin0 = (int)bin_key.size();
            key_base[i] = (int32_t)kb;
            for (int64_t b = 0; b < nbins; ++b) {
                bin_key.push_back((int32_t)(kb + b * kCellsPerBin));
                bin_inst.push_back(i);
                bin_local.push_back((int32_t)b);
            }
            kb += nbins * kCellsPerBin + 2;
            inst_pbase[i] = x.pbase;
            map[i].new_pbase = x.pbase;
            wantK |= x.p.H_kin > 0.0;
        }
        if (kb > ((int64_t)1 << 31) - 1 || pb > ((int64_t)1 << 31) - 1) {
            err = "too many bins or particles for one engine";
            return MPM_CAPACITY;
        }
        cap_total = pb;
        nn_total = go;
        nkeys = kb;
        max_work = (int)bin_key.size();
        const int64_t cp = std::max<int64_t>(cap_total, 1);
        // particle state: copy kept instances into the other buffer (or into
        // new, larger buffers)
        const bool had = pcap_alloc >= 0;
        const bool newbufs = !had || cap_total > pcap_alloc || (wantK && !has_K);
        PState<R> dst[2];
        void* nbuf[2] = {nullptr, nullptr};
        const bool withK = wantK || has_K;
        if (newbufs) {
            const int64_t cnew = had ? std::max<int64_t>(cp, pcap_alloc + pcap_alloc / 4) : cp;
            const size_t bytes = pstate_bytes(cnew, withK);
            for (int b = 0; b < 2; ++b) {
                cudaError_t e = cudaMalloc(&nbuf[b], bytes);
                if (e != cudaSuccess) {
                    if (nbuf[0]) cudaFree(nbuf[0]);
                    cudaGetLastError();
                    err = std::string("particle state: ") + cudaGetErrorString(e);
                    return e == cudaErrorMemoryAllocation ? MPM_OOM : MPM_CUDA_ERROR;
                }
                carve(nbuf[b], cnew, withK, dst[b]);
                if (withK) {
                    CK(cudaMemsetAsync(dst[b].K[0], 0, sizeof(V4<R>) * cnew, st));
                    CK(cudaMemsetAsync(dst[b].K[1], 0, sizeof(V4<R>) * cnew, st));
                }
            }
            pcap_alloc_next = cnew;
        }
        if (had && any_kept) {
            MS(grow(d_map, map_alloc, n));
            CK(cudaMemcpyAsync(d_map, map.data(), sizeof(RelayoutMap) * n, cudaMemcpyHostToDevice, st));
            launch_relayout<R>(ps[cur], newbufs ? dst[0] : ps[cur ^ 1], d_map, n, cap_total, st);
        }
        if (newbufs) {
            CK(cudaStreamSynchronize(st));
            for (int b = 0; b < 2; ++b) {
                if (pbuf[b]) cudaFree(pbuf[b]);
                pbuf[b] = nbuf[b];
                ps[b] = dst[b];
            }
            pcap_alloc = pcap_alloc_next;
            has_K = withK;
            cur = 0;
        } else if (had && any_kept) {
            cur ^= 1;
        }
        // grids and tool masks (not carried across a relayout)
        if (nn_total > nn_alloc) {
            CK(cudaStreamSynchronize(st));
            for (int b = 0; b < 2; ++b) {
                if (gpool[b]) cudaFree(gpool[b]);
                gpool[b] = nullptr;
            }
            for (int b = 0; b < 3; ++b) {
                if (tpool[b]) cudaFree(tpool[b]);
                tpool[b] = nullptr;
            }
            if (mask_pool) cudaFree(mask_pool);
            mask_pool = nullptr;
            const int64_t nn = std::max<int64_t>(nn_total + nn_total / 4, 1);
            for (int b = 0; b < 2; ++b) CK(cudaMalloc(&gpool[b], sizeof(V4<R>) * nn));
            for (int b = 0; b < 3; ++b) CK(cudaMalloc(&tpool[b], sizeof(R) * nn));
            CK(cudaMalloc(&mask_pool, sizeof(int32_t) * nn));
            nn_alloc = nn;
        }
        if (nn_total > 0) {
            CK(cudaMemsetAsync(gpool[0], 0, sizeof(V4<R>) * nn_total, st));
            CK(cudaMemsetAsync(gpool[1], 0, sizeof(V4<R>) * nn_total, st));
            for (int b = 0; b < 3; ++b) CK(cudaMemsetAsync(tpool[b], 0, sizeof(R) * nn_total, st));
            CK(cudaMemsetAsync(mask_pool, 0, sizeof(int32_t) * nn_total, st));
        }
        rbuf = 0;
        // sort scratch, key and bin tables
        MS(grow(d_key, slot_alloc[0], cp));
        MS(grow(d_rank, slot_alloc[1], cp));
        MS(grow(d_newbin, slot_alloc[2], cp));
        MS(grow(d_perm, perm_alloc, 2 * cp));
        MS(grow(d_pos, slot_alloc[3], 3 * cp));
        MS(grow(d_count, key_alloc[0], nkeys + 1));
        MS(grow(d_offset, key_alloc[1], nkeys + 1));
        const int64_t nb_tot = std::max<int64_t>(max_work, 1);
        MS(grow(d_flag, bin_alloc[0], nb_tot + 1));
        MS(grow(d_flag_scan, bin_alloc[1], nb_tot + 1));
        MS(grow(d_bin_key, bin_alloc[2], nb_tot));
        MS(grow(d_bin_inst, bin_alloc[3], nb_tot));
        MS(grow(d_bin_local, bin_alloc[4], nb_tot));
        MS(grow(d_work, bin_alloc[5], nb_tot));
        MS(grow(d_scan_tmp, scan_alloc, std::max<int64_t>(scan_tmp_size(nkeys + 1), scan_tmp_size(cp))));
        MS(grow(d_key_base, inst_alloc[0], n));
        MS(grow(d_inst_pbase, inst_alloc[1], n));
        MS(grow(d_inst, inst_alloc[2], n));
        MS(grow(d_ierr, ierr_alloc, n));
        if (n > 0) CK(cudaMemcpyAsync(d_ierr, words.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        if (n > 0) {
            CK(cudaMemcpyAsync(d_key_base, key_base.data(), 4 * n, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_inst_pbase, inst_pbase.data(), 8 * n, cudaMemcpyHostToDevice, st));
        }
        if (!bin_key.empty()) {
            CK(cudaMemcpyAsync(d_bin_key, bin_key.data(), 4 * bin_key.size(), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_bin_inst, bin_inst.data(), 4 * bin_inst.size(), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_bin_local, bin_local.data(), 4 * bin_local.size(), cudaMemcpyHostToDevice, st));
        }
        CK(cudaMemsetAsync(d_nwork, 0, sizeof(int), st));
        // instance table with TMA descriptors
        h_inst.assign(n, Inst<R>{});
        for (int i = 0; i < n; ++i) {
            mpm_status s = build_inst(i);
            if (s != MPM_OK) return s;
        }
        if (n > 0) CK(cudaMemcpyAsync(d_inst, h_inst.data(), sizeof(Inst<R>) * n, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        binned = false;
        return MPM_OK;
    }

    // Allocates every pool for the given totals up front (only while the
    // engine holds no instance), so that later instance changes within them
    // never reallocate.
    mpm_status reserve(int64_t particles, int64_t nodes, int64_t keys, int64_t bins, int max_inst,
                       bool backstress) override {
        if (!I.empty()) {
            err = "reserve needs an engine without instances";
            return MPM_INVALID_ARG;
        }
        if (particles < 1 || nodes < 1 || keys < 1 || bins < 1 || max_inst < 1) {
            err = "reserve sizes must be positive";
            return MPM_INVALID_ARG;
        }
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        for (int b = 0; b < 2; ++b) {
            if (pbuf[b]) cudaFree(pbuf[b]);
            pbuf[b] = nullptr;
        }
        for (int b = 0; b < 2; ++b) {
            CK(cudaMalloc(&pbuf[b], pstate_bytes(particles, backstress)));
            carve(pbuf[b], particles, backstress, ps[b]);
            if (backstress) {
                CK(cudaMemsetAsync(ps[b].K[0], 0, sizeof(V4<R>) * particles, st));
                CK(cudaMemsetAsync(ps[b].K[1], 0, sizeof(V4<R>) * particles, st));
            }
        }
        pcap_alloc = particles;
        has_K = backstress;
        cur = 0;
        for (int b = 0; b < 2; ++b) {
            if (gpool[b]) cudaFree(gpool[b]);
            gpool[b] = nullptr;
            CK(cudaMalloc(&gpool[b], sizeof(V4<R>) * nodes));
            CK(cudaMemsetAsync(gpool[b], 0, sizeof(V4<R>) * nodes, st));
        }
        for (int b = 0; b < 3; ++b) {
            if (tpool[b]) cudaFree(tpool[b]);
            tpool[b] = nullptr;
            CK(cudaMalloc(&tpool[b], sizeof(R) * nodes));
            CK(cudaMemsetAsync(tpool[b], 0, sizeof(R) * nodes, st));
        }
        if (mask_pool) cudaFree(mask_pool);
        mask_pool = nullptr;
        CK(cudaMalloc(&mask_pool, sizeof(int32_t) * nodes));
        nn_alloc = nodes;
        MS(grow(d_key, slot_alloc[0], particles, false));
        MS(grow(d_rank, slot_alloc[1], particles, false));
        MS(grow(d_newbin, slot_alloc[2], particles, false));
        MS(grow(d_perm, perm_alloc, 2 * particles, false));
        MS(grow(d_pos, slot_alloc[3], 3 * particles, false));
        MS(grow(d_count, key_alloc[0], keys + 1, false));
        MS(grow(d_offset, key_alloc[1], keys + 1, false));
        MS(grow(d_flag, bin_alloc[0], bins + 1, false));
        MS(grow(d_flag_scan, bin_alloc[1], bins + 1, false));
        MS(grow(d_bin_key, bin_alloc[2], bins, false));
        MS(grow(d_bin_inst, bin_alloc[3], bins, false));
        MS(grow(d_bin_local, bin_alloc[4], bins, false));
        MS(grow(d_work, bin_alloc[5], bins, false));
        MS(grow(d_scan_tmp, scan_alloc, std::max<int64_t>(scan_tmp_size(keys + 1), scan_tmp_size(particles)), false));
        MS(grow(d_key_base, inst_alloc[0], max_inst, false));
        MS(grow(d_inst_pbase, inst_alloc[1], max_inst, false));
        MS(grow(d_inst, inst_alloc[2], max_inst, false));
        MS(grow(d_ierr, ierr_alloc, max_inst, false));
        MS(grow(d_map, map_alloc, max_inst, false));
        CK(cudaStreamSynchronize(st));
        return MPM_OK;
    }

    // Adds instances at the end and drops the listed ones (state of the
    // others is kept).  New instances start empty; fill them with init_box or
    // upload.  Returns the index of the first added instance in *first.
    mpm_status change_instances(const mpm_params* params, const int64_t* caps, int n_add, const int32_t* remove,
                                int n_remove, int* first) override {
        // uploaded-but-unbinned positions sit in per-slot scratch that the
        // relayout does not move: bin them first
        if (!I.empty()) MS(ensure_binned());
        std::vector<InstHost> add;
        if (n_add > 0) {
            mpm_status s = make_insts(params, caps, n_add, &add);
            if (s != MPM_OK) return s;
        }
        std::vector<char> drop(I.size(), 0);
        for (int k = 0; k < n_remove; ++k) {
            if (remove[k] < 0 || remove[k] >= (int)I.size()) {
                err = "instance index out of range";
                return MPM_INVALID_ARG;
            }
            drop[remove[k]] = 1;
        }
        std::vector<InstHost> nI;
        std::vector<int> from;
        for (int i = 0; i < (int)I.size(); ++i)
            if (!drop[i]) {
                nI.push_back(I[i]);
                from.push_back(i);
            }
        if (first) *first = (int)nI.size();
        for (auto& x : add) {
            nI.push_back(x);
            from.push_back(-1);
        }
        return relayout(std::move(nI), from);
    }

    mpm_status build_inst(int i) {
        InstHost& x = I[i];
        const mpm_params& p = x.p;
        Inst<R>& d = h_inst[i];
        std::memset((void*)&d, 0, sizeof(d));
        PFN_encodeTiled_t enc = encode_fn();
        if (!enc) {
            err = "cuTensorMapEncodeTiled is not available from the driver";
            return MPM_CUDA_ERROR;
        }
        const size_t es = sizeof(R);
        for (int b = 0; b < 2; ++b) {
            d.grid[b] = gpool[b] + x.grid_off;
            cuuint64_t dims[4] = {4, (cuuint64_t)p.nx, (cuuint64_t)p.ny, (cuuint64_t)p.nz};
            cuuint64_t strides[3] = {4 * es, 4 * es * (cuuint64_t)p.nx, 4 * es * (cuuint64_t)p.nx * p.ny};
            cuuint32_t box[4] = {4, (cuuint32_t)kTile, (cuuint32_t)kTile, (cuuint32_t)kTile};
            cuuint32_t estr[4] = {1, 1, 1, 1};
            CUresult r = enc(&d.tmap[b], es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                             (void*)d.grid[b], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) {
                err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
                return MPM_CUDA_ERROR;
            }
        }
        fill_mutable(i);
        return MPM_OK;
    }

    // Every field except the TMA descriptors and grid pointers (which depend
    // only on the grid layout).
    void fill_mutable(int i) {
        InstHost& x = I[i];
        const mpm_params& p = x.p;
        Inst<R>& d = h_inst[i];
        d.tool_mask = mask_pool + x.grid_off;
        d.samples = x.d_samples;
        d.n_samples = x.n_samples;
        d.tn_start = x.has_nodes ? static_cast<const unsigned char*>(x.nodes.start) : nullptr;
        d.tn_end = x.has_nodes ? static_cast<const unsigned char*>(x.nodes.end) : nullptr;
        d.tn_n = x.has_nodes ? x.nodes.n : 0;
        d.tn_stride = x.nodes.stride;
        for (int a = 0; a < 3; ++a) {
            d.tn_off[a] = x.nodes.off_pos[a];
            d.tn_off[3 + a] = x.nodes.off_vel[a];
        }
        d.tn_a0 = x.nodes.alpha0;
        d.tn_da = x.nodes.dalpha;
        d.tn_step0 = x.nodes_step0;
        d.ierr = d_ierr + i;
        d.tm[0] = tpool[0] + x.grid_off;
        d.tm[1] = tpool[1] + x.grid_off;
        d.tn = tpool[2] + x.grid_off;
        d.gbase = x.grid_off;
        d.nx = p.nx; d.ny = p.ny; d.nz = p.nz;
        d.nbx = x.nbx; d.nby = x.nby; d.nbz = x.nbz;
        d.nbins = x.nbx * x.nby * x.nbz;
        d.bin0 = x.bin0;
        d.rebin_first = std::max(sort_every - x.since, 0);
        d.rebin_now = x.rebin_now ? 1 : 0;
        d.nn = x.nn;
        if (det && d_esc) {
            d.esc = d_esc + x.grid_off;
            d.esc_stride = std::max<int64_t>(nn_total, 1);
            d.esc_flag = d_esc_flag + x.bin0;
            d.esc_scale = std::ldexp(1.0, 40) / std::max(p.particle_mass, 1e-300);
        } else {
            d.esc = nullptr;
            d.esc_flag = nullptr;
        }
        d.dx = p.dx; d.ox = p.origin[0]; d.oy = p.origin[1]; d.oz = p.origin[2];
        d.dt = x.dt; d.t0 = x.time; d.step0 = x.step;
        const double mu = p.E / (2.0 * (1.0 + p.nu));
        const double lam = p.E * p.nu / ((1.0 + p.nu) * (1.0 - 2.0 * p.nu));
        d.mu = (R)mu; d.lam = (R)lam;
        d.pmass = (R)p.particle_mass; d.pvol = (R)p.particle_volume;
        d.A = (R)p.jc_A; d.B = (R)p.jc_B; d.n = (R)p.jc_n; d.C = (R)p.jc_C; d.m = (R)p.jc_m;
        d.edot0 = (R)std::max(p.edot0, 1e-12);
        d.Hkin = (R)p.H_kin;
        d.D1 = (R)p.D1; d.D2 = (R)p.D2; d.D3 = (R)p.D3; d.D4c = (R)p.D4; d.D5 = (R)p.D5; d.Dth = (R)p.D_th;
        d.Tspan = (R)std::max(p.Tm - p.Tamb, 1.0);
        // flow stress of an unheated particle: (A + B eps^n)(1 + C ln es)(1 - 0) with eps >= 0 and
        // es >= 1e-5, so Y >= A (1 + C ln 1e-5) when A > 0, B >= 0, C >= 0 (with a margin far above
        // the rounding of Y); 0 disables the bound
        {
            const double rt_lo = 1.0 + p.jc_C * std::log(1e-5);
            d.ylo = (p.jc_A > 0.0 && p.jc_B >= 0.0 && p.jc_C >= 0.0 && rt_lo > 0.0)
                        ? (R)(p.jc_A * rt_lo * (1.0 - 1e-4))
                        : R(0);
        }
        d.dTmax = (R)(p.Tm - p.Tamb);
        d.heat = (R)(p.beta / std::max(p.rho_phys * p.cp, 1e-12));
        d.apic = (R)p.apic_dinv_factor;
        d.decay = (R)p.apic_decay;
        d.deps_cap = (R)p.deps_cap;
        d.dT_cap = (R)p.dT_cap;
        d.fix_thick = p.fixture_thickness; d.fix_damp = p.fixture_damping;
        d.grav = p.gravity_z; d.mthr = p.mass_threshold;
        d.lod = p.lod_enabled; d.plast = p.plasticity;
        d.lod_r1 = p.lod_active_r; d.lod_r2 = p.lod_near_r;
        d.chip_every = p.chip_every;
        d.contact_every = p.contact_every > 0 ? p.contact_every : 0;
        d.contact_r = p.contact_radius;
        d.contact_mu = p.contact_friction;
        d.contact_hp = p.contact_heat_partition;
        d.rho_phys = p.rho_phys;
        // MPMWorkpieceSolver::step: alpha = k / (rho cp) (src/MPMWorkpieceSolver.cu:751-752)
        d.sdf_on = x.sdf ? 1 : 0;
        if (x.sdf) {
            d.sdf_tex = (unsigned long long)x.sdf->tex;
            for (int a = 0; a < 3; ++a) { d.sdf_n[a] = x.sdf->n[a]; d.sdf_o[a] = x.sdf->origin[a]; }
            d.sdf_vox = x.sdf->voxel; d.sdf_cos = x.sdf->cos_a; d.sdf_sin = x.sdf->sin_a;
        }
        // MPMWorkpieceSolver diffuses whenever k / (rho cp) > 0 (src/MPMWorkpieceSolver.cu:750-760)
        d.heat_on = (ws_on ? (p.thermal_conductivity > 0.0 && p.cp > 0.0 && p.rho_phys > 0.0) : p.heat_conduction != 0)
                        ? 1 : 0;
        d.ws_shear = (R)(p.E / (2.0 * (1.0 + p.nu)));
        d.ws_bulk = (R)(p.E / (3.0 * (1.0 - 2.0 * p.nu)));
        d.ws_fail = (R)ws.failure_strain;
        d.ws_crit_eps = (R)ws.critical_plastic_strain;
        d.ws_chip_ratio = (R)ws.thermal_chip_ratio;
        d.ws_damping = (R)ws.contact_damping;
        d.ws_max_rise = (R)ws.max_contact_temp_rise;
        d.ws_clamp = ws.thermal_clamp ? 1 : 0;
        d.ws_contact_r = ws.tool_contact_radius;
        for (int a = 0; a < 6; ++a) d.ws_sbox[a] = x.sbox[a];
        d.heat_c = p.thermal_conductivity / (p.rho_phys * p.cp) * x.dt / (p.dx * p.dx);
        d.Tamb = (R)p.Tamb;
        d.cp = p.cp;
        // applyAdiabaticHeatingKernel constants (src/AdiabaticShearModel.cu:131-176)
        d.asb_on = p.asb_enabled ? 1 : 0;
        d.asb_rise = (R)p.asb_touch_rise;
        d.asb_min_rate = (R)std::max(p.asb_critical_rate * 0.5, 5000.0);
        d.asb_crit = (R)p.asb_critical_rate;
        d.asb_heat = (R)(p.asb_taylor_quinney / std::max(p.rho_phys * p.cp, 1e-12));
        d.asb_Tcap = (R)(p.asb_max_temp_ratio * p.Tm - p.Tamb);
        d.newton_maxit = p.newton_maxit > 0 ? p.newton_maxit : 60;
        d.newton_tol = p.newton_tol > 0 ? p.newton_tol : 1e-12;
        const mpm_tool_desc& t = x.tool;
        d.tool_mode = t.mode; d.tool_shape = t.shape;
        for (int a = 0; a < 3; ++a) { d.tool_p0[a] = t.position[a]; d.tool_v[a] = t.velocity[a]; }
        d.tool_t0 = x.tool_t0;
        d.tool_r = t.radius; d.tool_rake = t.rake; d.tool_clear = t.clearance; d.tool_tip_dz = t.tip_dz;
        d.tool_sg = std::sin(t.rake); d.tool_cg = std::cos(t.rake);
        d.tool_sa = std::sin(t.clearance); d.tool_ca = std::cos(t.clearance);
        for (int a = 0; a < 3; ++a) { d.ext_c[a] = x.ext_c[a]; d.ext_f[a] = x.ext_f[a]; }
        d.ext_r = x.ext_pending ? x.ext_r : 0.0;
        d.pext = x.pext_pending ? d_pext : nullptr;
        d.pbase = x.pbase; d.np = x.np; d.pcap = x.cap;
        d.fresh = x.fresh;
    }

    mpm_status push_insts() {
        for (int i = 0; i < (int)I.size(); ++i) fill_mutable(i);
        CK(cudaMemcpyAsync(d_inst, h_inst.data(), sizeof(Inst<R>) * I.size(), cudaMemcpyHostToDevice, st));
        return MPM_OK;
    }

    // ---------------------------------------------------------------- binning

    // Deterministic mode: the stored node tiles and the escaped sums, grown
    // outside any graph capture and zeroed when grown (k_node_sum clears what
    // it reads).  fill_mutable points the instances into them.
    mpm_status det_scratch() {
        const int64_t items = std::max<int64_t>(max_work, 1);
        const int64_t nodes = std::max<int64_t>(nn_total, 1);
        if (part_alloc >= items * kPartCh * kTileNodes && esc_alloc >= kPartCh * nodes && esc_flag_alloc >= items)
            return MPM_OK;
        CK(cudaStreamSynchronize(st));   // nothing in flight uses the old buffers
        MS(grow(d_part, part_alloc, items * kPartCh * kTileNodes, false));
        MS(grow(d_esc, esc_alloc, kPartCh * nodes, false));
        MS(grow(d_esc_flag, esc_flag_alloc, items, false));
        CK(cudaMemsetAsync(d_esc, 0, sizeof(unsigned long long) * esc_alloc, st));
        CK(cudaMemsetAsync(d_esc_flag, 0, sizeof(int32_t) * esc_flag_alloc, st));
        return MPM_OK;
    }

    // The re-bin before a step call after an upload, a generation, a load or
    // a change of the instance set: fresh instances are binned from their
    // positions, every other instance keeps the layout its last re-bin gave
    // it (so an instance's layout, and with it every sum of its steps, does
    // not depend on when other instances arrive or on a checkpoint reload).
    mpm_status rebin() {
        Range nvtx_range("mpm.rebin");
        CK(cudaMemsetAsync(d_count, 0, 4 * (nkeys + 1), st));
        launch_pad_counts<R>(d_inst, (int)I.size(), d_key_base, d_count, st);
        // (the atomic mode keeps no layout: every instance is binned from its
        // positions, and all share one re-bin phase from here)
        launch_bin_count<R>(d_inst, (int)I.size(), ps[cur], d_key_base, true, d_pos, d_key, d_rank, d_count, d_newbin,
                            cap_total, det ? 0 : -1, sort_every, det, st);
        exclusive_scan(d_count, d_offset, nkeys, d_scan_tmp, st);
        launch_bin_scatter<R>(ps[cur], ps[cur ^ 1], d_inst, (int)I.size(), d_key, d_rank, d_offset, d_key_base,
                              d_newbin, true, d_pos, has_K, cap_total, d_perm, d_bin_key, max_work, st);
        build_work(d_offset, d_bin_key, d_bin_inst, d_bin_local, d_inst_pbase, max_work, d_flag, d_flag_scan,
                   d_scan_tmp, d_work, d_nwork, st);
        cur ^= 1;
        ++n_sorts;
        binned = true;
        bool any_fresh = false;
        bool any_now = false;
        for (auto& x : I) {
            any_fresh |= (x.fresh != 0);
            any_now |= x.rebin_now;
            if (x.fresh || x.rebin_now || !det) x.since = 0;
            x.fresh = 0;
            x.rebin_now = false;
        }
        any_fresh |= any_now;
        if (any_fresh) return push_insts();
        return MPM_OK;
    }

    mpm_status ensure_binned() {
        bool any_fresh = false;
        for (const auto& x : I) any_fresh |= (x.fresh != 0);
        if (!binned || any_fresh) return rebin();
        return MPM_OK;
    }

    // ---------------------------------------------------------------- particles in

    mpm_status init_box(int i, const int32_t c0[3], const int32_t c1[3], int32_t ppc, uint64_t seed, uint32_t instance,
                        int32_t fixed_layers, double T0, const mpm_tool_desc* tool) override {
        Range nvtx_range("mpm.init_box");
        InstHost& x = I[i];
        for (int a = 0; a < 3; ++a)
            if (c1[a] <= c0[a] || c0[a] < 0) {
                err = "empty or negative cell box";
                return MPM_INVALID_ARG;
            }
        if (ppc <= 0) {
            err = "ppc must be positive";
            return MPM_INVALID_ARG;
        }
        if (!std::isfinite(T0)) {
            err = "T0 must be finite";
            return MPM_INVALID_ARG;
        }
        const int64_t ncand = (int64_t)(c1[0] - c0[0]) * (c1[1] - c0[1]) * (c1[2] - c0[2]) * ppc;
        if (ncand > x.cap) {
            err = "box holds more candidates than the instance capacity";
            return MPM_CAPACITY;
        }
        x.time = 0.0;
        x.step = 0;
        if (tool) {
            mpm_status s = set_tool(i, tool);
            if (s != MPM_OK) return s;
        }
        const size_t need = 4 * (size_t)(2 * ncand + 2);
        if (gen_bytes < need) {
            if (d_gen) cudaFree(d_gen);
            d_gen = nullptr;
            CK(cudaMalloc(&d_gen, need));
            gen_bytes = need;
        }
        int32_t* flag = d_gen;
        int32_t* idx = d_gen + ncand + 1;
        int32_t* tmp = nullptr;
        CK(cudaMalloc(&tmp, 4 * scan_tmp_size(ncand)));
        Inst<R> P = h_inst[i];
        const int tool_check = (tool && tool->mode != MPM_TOOL_NONE) ? 1 : 0;
        launch_gen<R>(P, c0, c1, ppc, seed, instance, fixed_layers, T0 - x.p.Tamb, tool_check, flag, idx, tmp, ps[cur],
                      x.pbase, d_pos, st);
        int32_t lastf = 0, lasti = 0;
        CK(cudaMemcpyAsync(&lastf, flag + ncand - 1, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&lasti, idx + ncand - 1, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        cudaFree(tmp);
        x.np = (int64_t)lasti + lastf;
        x.fresh = 1;
        x.broken = false;
        x.pext_pending = false;
        CK(cudaMemsetAsync(d_ierr + i, 0, sizeof(int), st));   // a new state starts without errors
        CK(cudaGetLastError());
        return push_insts();  // binned by the next call that needs it
    }

    static size_t fbytes(const void* p, int elem, int64_t n, int per) { return p ? al256((size_t)elem * n * per) : 0; }

    mpm_status upload(int i, const mpm_particles_soa* h, int64_t n) override {
        Range nvtx_range("mpm.upload");
        InstHost& x = I[i];
        if (!h || (h->elem != 4 && h->elem != 8)) {
            err = "particles.elem must be 4 or 8";
            return MPM_INVALID_ARG;
        }
        if (n < 0 || n > x.cap) {
            err = "particle count exceeds the capacity";
            return MPM_CAPACITY;
        }
        if (n > 0 && (!h->x || !h->y || !h->z)) {
            err = "positions are required";
            return MPM_INVALID_ARG;
        }
        const int e = h->elem;
        struct F { const void* src; size_t per; const void** dst; };
        DevSoA d{};
        d.elem = e;
        F fs[] = {{h->x, 1, &d.x}, {h->y, 1, &d.y}, {h->z, 1, &d.z}, {h->vx, 1, &d.vx}, {h->vy, 1, &d.vy},
                  {h->vz, 1, &d.vz}, {h->F, 9, &d.F}, {h->Fp, 9, &d.Fp}, {h->C, 9, &d.C}, {h->stress, 6, &d.stress},
                  {h->backstress, 6, &d.bs}, {h->plastic_strain, 1, &d.eps}, {h->strain_rate, 1, &d.edot},
                  {h->temperature, 1, &d.T}, {h->damage, 1, &d.D}, {h->residual_stress, 1, &d.sres}};
        size_t need = 0;
        for (auto& f : fs) need += fbytes(f.src, e, n, (int)f.per);
        need += (h->status ? al256(4 * n) : 0) + (h->id ? al256(4 * n) : 0);
        if (stage_bytes < need) {
            if (d_stage) cudaFree(d_stage);
            d_stage = nullptr;
            CK(cudaMalloc(&d_stage, need));
            stage_bytes = need;
        }
        char* q = (char*)d_stage;
        for (auto& f : fs) {
            if (!f.src) { *f.dst = nullptr; continue; }
            const size_t b = (size_t)e * n * f.per;
            CK(cudaMemcpyAsync(q, f.src, b, cudaMemcpyHostToDevice, st));
            *f.dst = q;
            q += al256(b);
        }
        d.status = nullptr;
        d.id = nullptr;
        if (h->status) {
            CK(cudaMemcpyAsync(q, h->status, 4 * n, cudaMemcpyHostToDevice, st));
            d.status = (const int32_t*)q;
            q += al256(4 * n);
        }
        if (h->id) {
            CK(cudaMemcpyAsync(q, h->id, 4 * n, cudaMemcpyHostToDevice, st));
            d.id = (const int32_t*)q;
            q += al256(4 * n);
        }
        launch_import<R>(d, n, x.p.origin[0], x.p.origin[1], x.p.origin[2], x.p.dx, x.p.Tamb, ps[cur], x.pbase, d_pos,
                         st);
        x.np = n;
        x.fresh = 1;
        x.broken = false;
        x.pext_pending = false;
        CK(cudaMemsetAsync(d_ierr + i, 0, sizeof(int), st));   // a new state starts without errors
        CK(cudaGetLastError());
        return push_insts();  // binned by the next call that needs it
    }

    // ---------------------------------------------------------------- particles out

    mpm_status download(int i, mpm_particles_soa* h) override {
        Range nvtx_range("mpm.download");
        InstHost& x = I[i];
        if (!h || (h->elem != 4 && h->elem != 8)) {
            err = "particles.elem must be 4 or 8";
            return MPM_INVALID_ARG;
        }
        mpm_status s = ensure_binned();
        if (s != MPM_OK) return s;
        const int64_t n = x.np;
        const int e = h->elem;
        struct F { void* dst; size_t per; void** dev; };
        DevSoAOut o{};
        o.elem = e;
        F fs[] = {{h->x, 1, &o.x}, {h->y, 1, &o.y}, {h->z, 1, &o.z}, {h->vx, 1, &o.vx}, {h->vy, 1, &o.vy},
                  {h->vz, 1, &o.vz}, {h->F, 9, &o.F}, {h->Fp, 9, &o.Fp}, {h->C, 9, &o.C}, {h->stress, 6, &o.stress},
                  {h->backstress, 6, &o.bs}, {h->plastic_strain, 1, &o.eps}, {h->strain_rate, 1, &o.edot},
                  {h->temperature, 1, &o.T}, {h->damage, 1, &o.D}, {h->residual_stress, 1, &o.sres}};
        size_t need = 0;
        for (auto& f : fs) need += fbytes(f.dst, e, n, (int)f.per);
        need += (h->status ? al256(4 * n) : 0) + (h->id ? al256(4 * n) : 0);
        if (stage_bytes < need) {
            CK(cudaStreamSynchronize(st));
            if (d_stage) cudaFree(d_stage);
            d_stage = nullptr;
            CK(cudaMalloc(&d_stage, need));
            stage_bytes = need;
        }
        char* q = (char*)d_stage;
        for (auto& f : fs) {
            if (!f.dst) { *f.dev = nullptr; continue; }
            *f.dev = q;
            q += al256((size_t)e * n * f.per);
        }
        o.status = nullptr;
        o.id = nullptr;
        if (h->status) { o.status = (int32_t*)q; q += al256(4 * n); }
        if (h->id) { o.id = (int32_t*)q; q += al256(4 * n); }
        launch_export<R>(d_inst + i, ps[cur], x.pbase, n, x.p.Tamb, o, st);
        for (auto& f : fs)
            if (f.dst) CK(cudaMemcpyAsync(f.dst, *f.dev, (size_t)e * n * f.per, cudaMemcpyDeviceToHost, st));
        if (h->status) CK(cudaMemcpyAsync(h->status, o.status, 4 * n, cudaMemcpyDeviceToHost, st));
        if (h->id) CK(cudaMemcpyAsync(h->id, o.id, 4 * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return inst_status(i);
    }

    mpm_status export_aos(int i, void* dst, int64_t bytes) override {
        Range nvtx_range("mpm.export_aos");
        InstHost& x = I[i];
        if (!dst || bytes < x.np * 504) {
            err = "destination smaller than np * sizeof(MPMParticle) (504 bytes)";
            return MPM_INVALID_ARG;
        }
        mpm_status s = ensure_binned();
        if (s != MPM_OK) return s;
        cudaPointerAttributes at{};
        const bool dev = cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeDevice;
        cudaGetLastError();
        void* out = dst;
        if (!dev) {
            const size_t need = (size_t)504 * std::max<int64_t>(x.np, 1);
            if (stage_bytes < need) {
                CK(cudaStreamSynchronize(st));
                if (d_stage) cudaFree(d_stage);
                d_stage = nullptr;
                CK(cudaMalloc(&d_stage, need));
                stage_bytes = need;
            }
            out = d_stage;
        }
        launch_export_aos<R>(d_inst + i, ps[cur], x.pbase, x.np, x.p.Tamb, x.p.rho_phys, out, st);
        if (!dev) CK(cudaMemcpyAsync(dst, out, (size_t)504 * x.np, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return inst_status(i);
    }

    mpm_status import_aos(int i, const void* src, int64_t bytes, uint32_t fields) override {
        Range nvtx_range("mpm.import_aos");
        InstHost& x = I[i];
        if (!src || bytes < x.np * 504) {
            err = "source smaller than np * sizeof(MPMParticle) (504 bytes)";
            return MPM_INVALID_ARG;
        }
        if (fields & ~(uint32_t)MPM_AOS_WRITABLE) {
            err = "unknown MPM_AOS_* field bits";
            return MPM_INVALID_ARG;
        }
        if (fields == 0 || x.np == 0) return MPM_OK;
        // positions are re-expressed in the bins the export was taken from
        MS(ensure_binned());
        cudaPointerAttributes at{};
        const bool dev = cudaPointerGetAttributes(&at, src) == cudaSuccess &&
                         (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
        cudaGetLastError();
        const void* in = src;
        if (!dev) {
            const size_t need = (size_t)504 * x.np;
            if (stage_bytes < need) {
                CK(cudaStreamSynchronize(st));
                if (d_stage) cudaFree(d_stage);
                d_stage = nullptr;
                CK(cudaMalloc(&d_stage, need));
                stage_bytes = need;
            }
            CK(cudaMemcpyAsync(d_stage, src, need, cudaMemcpyHostToDevice, st));
            in = d_stage;
        }
        if (!d_flags) CK(cudaMalloc(&d_flags, 2 * sizeof(int)));
        if ((fields & MPM_AOS_EXT_FORCE) && pext_alloc < cap_total) {
            CK(cudaStreamSynchronize(st));
            MS(grow(d_pext, pext_alloc, cap_total, false));
        }
        CK(cudaMemsetAsync(d_flags, 0, 2 * sizeof(int), st));
        launch_import_aos<R>(d_inst + i, ps[cur], x.pbase, x.np, x.p.Tamb, fields,
                             in, (fields & MPM_AOS_EXT_FORCE) ? d_pext : nullptr, d_flags, st);
        int h[2] = {0, 0};
        CK(cudaMemcpyAsync(h, d_flags, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        if (h[0]) {   // moved particles: re-bin the instance from its positions before the next step
            binned = false;
            I[i].rebin_now = true;
        }
        if (fields & MPM_AOS_EXT_FORCE) x.pext_pending = true;
        MS(push_insts());
        if (h[1]) {
            err = std::to_string(h[1]) + " records have a status outside 0..4 (kept their status)";
            return MPM_INVALID_ARG;
        }
        return MPM_OK;
    }

    // ---------------------------------------------------------------- tool

    // The voxel tool SDF as a 3D texture set up as ToolSDF::createTexture does
    // (src/ToolSDF.cu:534-567): float texels, trilinear filtering, clamp
    // addressing, unnormalised coordinates.
    mpm_status set_tool_sdf(int i, const mpm_tool_sdf* s) override {
        InstHost& x = I[i];
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        if (!s) {
            x.sdf.reset();
            return push_insts();
        }
        if (!s->values || s->nx < 2 || s->ny < 2 || s->nz < 2 || s->nx > 1024 || s->ny > 1024 || s->nz > 1024 ||
            !(s->voxel > 0.0f) || !std::isfinite(s->angle)) {
            err = "tool SDF: values, 2..1024 voxels per axis and a positive voxel edge";
            return MPM_INVALID_ARG;
        }
        auto t = std::make_shared<ToolSdfTex>();
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
        const cudaExtent ext = make_cudaExtent(s->nx, s->ny, s->nz);
        CK(cudaMalloc3DArray(&t->arr, &ch, ext));
        cudaMemcpy3DParms cp = {};
        cp.srcPtr = make_cudaPitchedPtr((void*)s->values, s->nx * sizeof(float), s->nx, s->ny);
        cp.dstArray = t->arr;
        cp.extent = ext;
        cp.kind = cudaMemcpyHostToDevice;
        CK(cudaMemcpy3D(&cp));
        cudaResourceDesc rd = {};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = t->arr;
        cudaTextureDesc td = {};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        CK(cudaCreateTextureObject(&t->tex, &rd, &td, nullptr));
        t->n[0] = s->nx; t->n[1] = s->ny; t->n[2] = s->nz;
        for (int a = 0; a < 3; ++a) t->origin[a] = s->origin[a];
        t->voxel = s->voxel;
        t->cos_a = std::cos(s->angle);
        t->sin_a = std::sin(s->angle);
        x.sdf = std::move(t);
        return push_insts();
    }

    mpm_status set_tool(int i, const mpm_tool_desc* t) override {
        InstHost& x = I[i];
        if (!t || t->mode < MPM_TOOL_NONE || t->mode > MPM_TOOL_SDF_SLIP || t->shape < 0 || t->shape > 1) {
            err = "invalid tool descriptor";
            return MPM_INVALID_ARG;
        }
        if (t->mode == MPM_TOOL_RASTER && t->n_samples > 0 && (!t->sample_dx || !t->sample_dy || !t->sample_dz)) {
            err = "raster tool needs sample offsets";
            return MPM_INVALID_ARG;
        }
        x.tool = *t;
        x.tool.sample_dx = x.tool.sample_dy = x.tool.sample_dz = nullptr;
        x.tool_t0 = x.time;
        if (t->mode == MPM_TOOL_RASTER) {
            const int ns = std::max(t->n_samples, 0);
            // the samples live in one device buffer, reused while it is large
            // enough: a captured step graph reads them through the instance
            // record and stays valid
            if (ns > x.samples_cap) {
                CK(cudaStreamSynchronize(st));   // nothing in flight reads the old buffer
                if (x.d_samples) cudaFree(x.d_samples);
                x.d_samples = nullptr;
                x.samples_cap = 0;
                CK(cudaMalloc(&x.d_samples, 3 * sizeof(double) * ns));
                x.samples_cap = ns;
            }
            x.n_samples = ns;
            for (int a = 0; a < 3; ++a) { x.sbox[a] = 0.0; x.sbox[3 + a] = 0.0; }
            if (ns > 0) {
                const double* c[3] = {t->sample_dx, t->sample_dy, t->sample_dz};
                for (int a = 0; a < 3; ++a) {
                    x.sbox[a] = x.sbox[3 + a] = c[a][0];
                    for (int q = 1; q < ns; ++q) {
                        x.sbox[a] = std::min(x.sbox[a], c[a][q]);
                        x.sbox[3 + a] = std::max(x.sbox[3 + a], c[a][q]);
                    }
                }
                CK(cudaMemcpyAsync(x.d_samples, t->sample_dx, 8 * ns, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(x.d_samples + ns, t->sample_dy, 8 * ns, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(x.d_samples + 2 * ns, t->sample_dz, 8 * ns, cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
            }
        } else {
            x.has_nodes = false;
        }
        return push_insts();
    }

    // The raster tool from FEM node records in device memory (mpm_tool_nodes).
    mpm_status set_tool_nodes(int i, const mpm_tool_nodes* n) override {
        InstHost& x = I[i];
        if (!n) {
            x.has_nodes = false;
            return push_insts();
        }
        if (!n->end || n->n <= 0 || n->stride < 24) {
            err = "tool nodes: end records, n > 0 and a stride of at least 24 bytes required";
            return MPM_INVALID_ARG;
        }
        for (int a = 0; a < 3; ++a)
            if (n->off_pos[a] < 0 || n->off_pos[a] + 8 > n->stride || n->off_vel[a] < 0 ||
                n->off_vel[a] + 8 > n->stride || (n->off_pos[a] % 8) != 0 || (n->off_vel[a] % 8) != 0) {
                err = "tool nodes: field offsets must be 8-byte aligned and inside a record";
                return MPM_INVALID_ARG;
            }
        if ((n->stride % 8) != 0 || (reinterpret_cast<uintptr_t>(n->end) % 8) != 0 ||
            (reinterpret_cast<uintptr_t>(n->start) % 8) != 0) {
            err = "tool nodes: records must be 8-byte aligned";
            return MPM_INVALID_ARG;
        }
        if (!std::isfinite(n->alpha0) || !std::isfinite(n->dalpha)) {
            err = "tool nodes: alpha0 and dalpha must be finite";
            return MPM_INVALID_ARG;
        }
        x.nodes = *n;
        x.has_nodes = true;
        x.nodes_step0 = x.step;
        x.tool.mode = MPM_TOOL_RASTER;
        return push_insts();
    }

    // ---------------------------------------------------------------- step

    // Points the raster tool of an instance marks per step (samples or FEM
    // nodes; 0: no raster tool).
    static int raster_points(const InstHost& x) {
        if (x.tool.mode != MPM_TOOL_RASTER) return 0;
        return x.has_nodes ? x.nodes.n : x.n_samples;
    }

    // The tool masks of step k of the call: cleared, then marked by the
    // raster kernel, which reads the pose (or the node records and their
    // blend) from the instance record, so the sequence replays from a graph.
    void raster_all(int k) {
        bool any = false;
        for (const auto& x : I) any |= raster_points(x) > 0;
        if (!any) return;
        Range nvtx_range("mpm.tool_raster");
        for (int i = 0; i < (int)I.size(); ++i) {
            const InstHost& x = I[i];
            const int np = raster_points(x);
            if (np <= 0) continue;
            cudaMemsetAsync(mask_pool + x.grid_off, 0, sizeof(int32_t) * x.nn, st);
            launch_raster<R>(d_inst, i, k, np, st);
        }
    }

    mpm_status step(int32_t N, const double* dts) override {
        Range nvtx_range("mpm.step");
        if (N < 0) {
            err = "nsteps must be >= 0";
            return MPM_INVALID_ARG;
        }
        if (N == 0) return MPM_OK;
        for (int i = 0; i < (int)I.size(); ++i) {
            if (!(dts[i] > 0.0) || !std::isfinite(dts[i])) {
                err = "dt must be positive";
                return MPM_INVALID_ARG;
            }
            if (I[i].broken) {
                err = "workpiece " + std::to_string(i) + " was left part-loaded by a failed checkpoint load; "
                      "upload, generate or load it again";
                return MPM_INVALID_ARG;
            }
            I[i].dt = dts[i];
        }
        mpm_status s = ensure_binned();
        if (s != MPM_OK) return s;
        if (det) MS(det_scratch());
        s = push_insts();
        if (s != MPM_OK) return s;
        bool ext = false;
        for (auto& x : I) ext |= x.ext_pending || x.pext_pending;
        // the raster launches' sizes are part of a captured graph
        std::vector<int> rsig(I.size());
        for (size_t q = 0; q < I.size(); ++q) rsig[q] = raster_points(I[q]);
        if (rsig != raster_sig) {
            drop_graphs();
            raster_sig = rsig;
        }
        if (ws_on)
            s = issue_ws_steps(N, ext);
        else if (use_graph && !prof && max_work > 0)
            s = step_graph(N, ext);
        else
            s = issue_steps(N, ext);
        if (s != MPM_OK) return s;
        for (auto& x : I) {
            x.time += (double)N * x.dt;
            x.step += N;
            x.ext_pending = false;
            x.pext_pending = false;
        }
        CK(cudaGetLastError());
        return MPM_OK;
    }

    // The launches of one step call.  Fused schedule: N+1 launches (P2G of
    // step 0, then G2P k + P2G k+1, then G2P of step N-1); split: 2N.  Only
    // device work and host counters (re-bin cadence, buffer parity), so the
    // sequence can be captured in a graph.
    mpm_status issue_steps(int32_t N, bool ext) {
        mpm_status s = MPM_OK;
        const size_t gbytes = sizeof(V4<R>) * nn_total;
        const bool fused = I[0].p.schedule == MPM_SCHED_FUSED;
        int w = rbuf;
        // point k of the call: the instances whose re-bin phase falls on k are
        // re-binned (the others keep their layout); last[i] = the call's last
        // such point of instance i
        std::vector<int> last(I.size(), -1);
        // The atomic mode re-bins every instance whenever one is due, so the
        // instances keep one shared phase: a batch of workpieces admitted at
        // different steps would otherwise re-bin (and move every particle)
        // at nearly every step.
        auto maybe_sort = [&](int k) -> mpm_status {
            bool any = false;
            for (size_t i = 0; i < I.size(); ++i) {
                const int f = std::max(sort_every - I[i].since, 0);
                if (k >= f && (k - f) % sort_every == 0) {
                    any = true;
                    last[i] = k;
                }
            }
            if (any && !det)
                for (size_t i = 0; i < I.size(); ++i) last[i] = k;
            return any ? rebin_regular(det ? k : -1) : MPM_OK;
        };
        const int cps = ctas_per_sm;
        int xk = 0, heat = 0;
        for (const InstHost& x : I) {
            xk |= (x.p.asb_enabled || x.p.heat_conduction || (x.sdf && x.p.contact_every > 0)) ? 1 : 0;
            heat |= x.p.heat_conduction ? 1 : 0;
        }
        // Default mode: the grid buffer a P2G launch writes starts at zero, and
        // so does its T m buffer; the launch adds its tiles with atomics.
        // Deterministic mode: the launch stores its tiles and k_node_sum writes
        // every node of the buffer from them.
        auto clear = [&](int b) -> mpm_status {
            if (det) return MPM_OK;
            CK(cudaMemsetAsync(gpool[b], 0, gbytes, st));
            if (heat) CK(cudaMemsetAsync(tpool[b], 0, sizeof(R) * nn_total, st));
            return MPM_OK;
        };
        const int64_t part_items = part_alloc / (kPartCh * kTileNodes);
        auto node_sum = [&](int b) {
            if (det)
                launch_node_sum<R>(d_inst, d_bin_inst, d_bin_local, d_flag, d_flag_scan, d_part, part_items, b,
                                   max_work, st);
        };
        auto p2g_args = [&](StepArgs a) {
            a.part = det ? d_part : nullptr;
            a.chunk = pass_chunk;
            return a;
        };
        // heat conduction: the diffusion step on grid buffer b before the G2P that reads it
        auto diffuse = [&](int b) {
            if (heat) launch_heat_diffuse<R>(d_inst, (int)I.size(), b, nn_total, st);
        };
        if (fused) {
            if ((s = clear(w)) != MPM_OK) return s;
            const StepArgs a = p2g_args(StepArgs{0, 0, N == 1 ? 1 : 0, ext ? 1 : 0, 0, xk});
            launch_step<R>(d_inst, d_work, d_nwork, max_work, ps[cur], a, w, false, true, threads, cps, d_err, d_ctr,
                           st);
            node_sum(w);
            for (int k = 0; k + 1 < N; ++k) {
                if ((s = maybe_sort(k)) != MPM_OK) return s;
                if ((s = clear(w ^ 1)) != MPM_OK) return s;
                raster_all(k);
                diffuse(w);
                const StepArgs b = p2g_args(StepArgs{k, 0, (k + 2 == N) ? 1 : 0, 0, k + 1, xk});
                prof_begin();
                launch_step<R>(d_inst, d_work, d_nwork, max_work, ps[cur], b, w, true, true, threads, cps, d_err,
                               d_ctr, st);
                prof_end();
                node_sum(w ^ 1);
                w ^= 1;
            }
            // the last point: a split of these steps into several calls re-bins
            // at the same steps as one call
            if ((s = maybe_sort(N - 1)) != MPM_OK) return s;
            raster_all(N - 1);
            diffuse(w);
            StepArgs c{N - 1, 1, 0, 0, N - 1, xk};
            c.chunk = pass_chunk;
            launch_step<R>(d_inst, d_work, d_nwork, max_work, ps[cur], c, w, true, false, threads, cps, d_err, d_ctr,
                           st);
        } else {
            for (int k = 0; k < N; ++k) {
                if ((s = maybe_sort(k)) != MPM_OK) return s;
                if ((s = clear(w)) != MPM_OK) return s;
                const StepArgs a = p2g_args(StepArgs{k, 0, 1, (ext && k == 0) ? 1 : 0, k, xk});
                prof_begin();
                launch_step<R>(d_inst, d_work, d_nwork, max_work, ps[cur], a, w, false, true, threads, cps, d_err,
                               d_ctr, st);
                prof_end();
                node_sum(w);
                raster_all(k);
                diffuse(w);
                StepArgs c{k, 1, 0, 0, k, xk};
                c.chunk = pass_chunk;
                prof_begin();
                launch_step<R>(d_inst, d_work, d_nwork, max_work, ps[cur], c, w, true, false, threads, cps, d_err,
                               d_ctr, st);
                prof_end();
            }
        }
        // G2P steps since each instance's last re-bin
        for (size_t i = 0; i < I.size(); ++i) I[i].since = last[i] >= 0 ? N - last[i] : I[i].since + N;
        rbuf = w;
        return MPM_OK;
    }

    // MPMWorkpieceSolver's step, N times: clear grid buffer 0 and its T m, then
    // P2G, the grid update (contact force of the step into the metrics'
    // contact-force slot), the diffusion step, G2P and chip separation.
    mpm_status issue_ws_steps(int32_t N, bool ext) {
        std::vector<int64_t> np(I.size()), nn(I.size());
        for (size_t i = 0; i < I.size(); ++i) {
            np[i] = I[i].np;
            nn[i] = I[i].nn;
        }
        int diffuse = 0;
        for (const auto& h : h_inst) diffuse |= h.heat_on;
        double* fsum = reinterpret_cast<double*>(d_ctr + 4) + 1;
        for (int k = 0; k < N; ++k) {
            CK(cudaMemsetAsync(gpool[0], 0, sizeof(V4<R>) * nn_total, st));
            CK(cudaMemsetAsync(tpool[0], 0, sizeof(R) * nn_total, st));
            CK(cudaMemsetAsync(fsum, 0, sizeof(double), st));
            launch_ws_step<R>(d_inst, np, nn, ps[cur], k, (ext && k == 0) ? 1 : 0, diffuse, fsum, st,
                              &launch_heat_diffuse<R>, nn_total);
        }
        rbuf = 0;
        return MPM_OK;
    }

    mpm_status set_workpiece_semantics(const mpm_workpiece_params* p) override {
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        if (!p) {
            if (ws_on) {   // positions drifted from their bins: re-bin for the fused kernel
                binned = false;
                for (auto& x : I) x.rebin_now = true;
            }
            ws_on = false;
            return push_insts();
        }
        if (!(p->tool_contact_radius >= 0.0) || !std::isfinite(p->failure_strain) ||
            !std::isfinite(p->critical_plastic_strain) || !std::isfinite(p->thermal_chip_ratio) ||
            !(p->contact_damping >= 0.0) || !(p->max_contact_temp_rise >= 0.0)) {
            err = "workpiece semantics: finite constants, non-negative radius, damping and cap required";
            return MPM_INVALID_ARG;
        }
        ws = *p;
        ws_on = true;
        return push_insts();
    }

    // ---------------------------------------------------------------- graphs

    // A captured step call, valid for one layout and launch configuration; the
    // host counters it leaves behind are replayed with it.
    struct GraphEntry {
        int32_t N;
        std::vector<int> since0;   // the instances' re-bin phases before the call
        int cur0, rbuf0, ext;
        cudaGraphExec_t exec;
        std::vector<int> since1;   // ... and after it
        int64_t sorts, launches;
        int cur1, rbuf1;
        uint64_t use;
    };
    std::vector<GraphEntry> graphs;
    std::vector<int> raster_sig;   // raster points per instance when the graphs were captured
    uint64_t graph_clock = 0;
    static constexpr size_t kMaxGraphs = 32;

    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }

    mpm_status step_graph(int32_t N, bool ext) {
        Range nvtx_range("mpm.graph");
        std::vector<int> since(I.size());
        for (size_t i = 0; i < I.size(); ++i) since[i] = I[i].since;
        for (auto& g : graphs) {
            if (g.N == N && g.since0 == since && g.cur0 == cur && g.rbuf0 == rbuf && g.ext == (int)ext) {
                CK(cudaGraphLaunch(g.exec, st));
                for (size_t i = 0; i < I.size(); ++i) I[i].since = g.since1[i];
                n_sorts += g.sorts;
                cur = g.cur1;
                rbuf = g.rbuf1;
                launch_counter() += g.launches;
                g.use = ++graph_clock;
                return MPM_OK;
            }
        }
        GraphEntry e{};
        e.N = N;
        e.since0 = since;
        e.cur0 = cur;
        e.rbuf0 = rbuf;
        e.ext = (int)ext;
        const int64_t sorts0 = n_sorts, l0 = launch_counter();
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        mpm_status s = issue_steps(N, ext);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (s != MPM_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (ce != cudaSuccess) {
            err = std::string("step graph capture: ") + cudaGetErrorString(ce);
            return MPM_CUDA_ERROR;
        }
        ce = cudaGraphInstantiate(&e.exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            err = std::string("step graph instantiate: ") + cudaGetErrorString(ce);
            return MPM_CUDA_ERROR;
        }
        CK(cudaGraphLaunch(e.exec, st));
        e.since1.resize(I.size());
        for (size_t i = 0; i < I.size(); ++i) e.since1[i] = I[i].since;
        e.sorts = n_sorts - sorts0;
        e.launches = launch_counter() - l0;
        e.cur1 = cur;
        e.rbuf1 = rbuf;
        e.use = ++graph_clock;
        if (graphs.size() >= kMaxGraphs) {
            size_t old = 0;
            for (size_t k = 1; k < graphs.size(); ++k)
                if (graphs[k].use < graphs[old].use) old = k;
            cudaGraphExecDestroy(graphs[old].exec);
            graphs.erase(graphs.begin() + old);
        }
        graphs.push_back(e);
        return MPM_OK;
    }

    // ---------------------------------------------------------------- launch configuration

    mpm_status get_config(mpm_launch_config* c) override {
        c->ctas_per_sm = ctas_per_sm;
        c->sort_every = sort_every;
        c->use_graph = use_graph ? 1 : 0;
        c->deterministic = det ? 1 : 0;
        c->pass_size = pass_chunk * 128;
        return MPM_OK;
    }

    mpm_status set_config(const mpm_launch_config* c) override {
        if (!c || c->ctas_per_sm < 1 || c->ctas_per_sm > 8 || c->sort_every < 1 || c->sort_every > 1024 ||
            (c->deterministic != 0 && c->deterministic != 1) ||
            (c->pass_size != 0 && c->pass_size != 128 && c->pass_size != 256 && c->pass_size != 512)) {
            err = "launch config: ctas_per_sm in [1, 8], sort_every in [1, 1024], deterministic 0 or 1, pass_size "
                  "0, 128, 256 or 512";
            return MPM_INVALID_ARG;
        }
        const int chunk = c->pass_size ? c->pass_size / 128 : kDefaultPassChunk;
        if (c->ctas_per_sm != ctas_per_sm || c->sort_every != sort_every || (c->deterministic != 0) != det ||
            chunk != pass_chunk)
            drop_graphs();
        pass_chunk = chunk;
        det = c->deterministic != 0;
        ctas_per_sm = c->ctas_per_sm;
        sort_every = c->sort_every;
        use_graph = c->use_graph != 0;
        if (!use_graph) drop_graphs();
        return MPM_OK;
    }

    // Times the candidates over real steps and keeps the fastest: the pass
    // size first (16 steps each at the current CTAs and cadence), then, at the
    // fastest pass size, CTAs per SM x re-bin cadence over one re-bin period
    // each.  The trial steps advance the simulation like any other steps.
    mpm_status autotune(const double* dts, mpm_launch_config* best) override {
        const int cand_pass[3] = {128, 256, 512};
        const int cand_ctas[3] = {2, 3, 4};
        const int cand_sort[3] = {8, 16, 32};
        mpm_launch_config cur_cfg{};
        get_config(&cur_cfg);
        mpm_launch_config win = cur_cfg;
        double win_ms = 1e300;
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        // n steps of candidate c, then the re-bin that ends the period: ms per step
        auto trial = [&](const mpm_launch_config& c, int n, double* per) -> mpm_status {
            mpm_status s = set_config(&c);
            if (s != MPM_OK) return s;
            for (auto& x : I) x.since = 0;
            cudaEventRecord(e0, st);
            if ((s = step(n, dts)) != MPM_OK) return s;
            if ((s = rebin_regular(-1)) != MPM_OK) return s;
            for (auto& x : I) x.since = 0;
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                err = "autotune: event sync failed";
                return MPM_CUDA_ERROR;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            *per = ms / n;
            return MPM_OK;
        };
        mpm_status s = MPM_OK;
        for (int a = 0; a < 3 && s == MPM_OK; ++a) {
            mpm_launch_config c = cur_cfg;
            c.pass_size = cand_pass[a];
            double per = 0.0;
            if ((s = trial(c, 16, &per)) != MPM_OK) break;
            if (per < win_ms) {
                win_ms = per;
                win = c;
            }
        }
        const int pass = win.pass_size;
        win_ms = 1e300;
        for (int a = 0; a < 3 && s == MPM_OK; ++a)
            for (int b = 0; b < 3 && s == MPM_OK; ++b) {
                mpm_launch_config c = cur_cfg;
                c.pass_size = pass;
                c.ctas_per_sm = cand_ctas[a];
                c.sort_every = cand_sort[b];
                double per = 0.0;
                if ((s = trial(c, cand_sort[b], &per)) != MPM_OK) break;
                if (per < win_ms) {
                    win_ms = per;
                    win = c;
                }
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (s != MPM_OK) return s;
        s = set_config(&win);
        if (best) *best = win;
        return s == MPM_OK ? device_status() : s;
    }

    // The re-bin at point kpt of a step call: the instances whose re-bin
    // phase falls on kpt are binned from their positions, the others keep
    // their layout (kpt < 0: every instance is re-binned).
    mpm_status rebin_regular(int kpt) {
        Range nvtx_range("mpm.rebin");
        // positions are bin-local (no instance is fresh here)
        CK(cudaMemsetAsync(d_count, 0, 4 * (nkeys + 1), st));
        launch_pad_counts<R>(d_inst, (int)I.size(), d_key_base, d_count, st);
        launch_bin_count<R>(d_inst, (int)I.size(), ps[cur], d_key_base, false, d_pos, d_key, d_rank, d_count,
                            d_newbin, cap_total, kpt, sort_every, false, st);
        exclusive_scan(d_count, d_offset, nkeys, d_scan_tmp, st);
        launch_bin_scatter<R>(ps[cur], ps[cur ^ 1], d_inst, (int)I.size(), d_key, d_rank, d_offset, d_key_base,
                              d_newbin, false, d_pos, has_K, cap_total, d_perm, d_bin_key, max_work, st);
        build_work(d_offset, d_bin_key, d_bin_inst, d_bin_local, d_inst_pbase, max_work, d_flag, d_flag_scan,
                   d_scan_tmp, d_work, d_nwork, st);
        cur ^= 1;
        ++n_sorts;
        return MPM_OK;
    }

    // ---------------------------------------------------------------- metrics

    // Status from the error words of the handle (ERR_TIMEOUT) and of
    // instances [i0, i1).  Synchronises the stream.
    mpm_status word_status(int i0, int i1, std::vector<int>* words = nullptr) {
        int e = 0;
        std::vector<int> w((size_t)std::max(i1 - i0, 0), 0);
        CK(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        if (!w.empty()) CK(cudaMemcpyAsync(w.data(), d_ierr + i0, sizeof(int) * w.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (e & ERR_NEWTON) {
            // a thread saw Newton returns fail in more than one instance: every
            // instance that runs the Newton return is marked (on the device, so
            // that the mark stays with the instance) and the handle's bit cleared
            const unsigned char one = 1;
            for (size_t k = 0; k < I.size(); ++k)
                if (I[k].p.plasticity == MPM_PLAST_NEWTON) {
                    CK(cudaMemcpyAsync(reinterpret_cast<unsigned char*>(d_ierr + k) + 1, &one, 1,
                                       cudaMemcpyHostToDevice, st));
                    if ((int)k >= i0 && (int)k < i1) w[k - i0] |= ERR_NEWTON;
                }
            e &= ~ERR_NEWTON;
            CK(cudaMemcpyAsync(d_err, &e, sizeof(int), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        if (words) *words = w;
        if (e & ERR_TIMEOUT) {
            err = "a bounded device wait timed out (TMA tile load)";
            return MPM_TIMEOUT;
        }
        for (size_t k = 0; k < w.size(); ++k) {
            if (!w[k]) continue;
            const std::string who = "instance " + std::to_string(i0 + (int)k) + ": ";
            err = who + ((w[k] & 0xff) ? "a NaN or Inf in the particle state" : "a Newton return did not converge");
            return MPM_NUMERIC;
        }
        return MPM_OK;
    }
    mpm_status device_status() { return word_status(0, (int)I.size()); }
    mpm_status inst_status(int i) { return word_status(i, i + 1); }

    mpm_status inst_statuses(int32_t* out, int n) override {
        if (!out || n < (int)I.size()) {
            err = "status array NULL or shorter than the instance count";
            return MPM_INVALID_ARG;
        }
        std::vector<int> w;
        const mpm_status s = word_status(0, (int)I.size(), &w);
        if (s != MPM_OK && s != MPM_TIMEOUT && s != MPM_NUMERIC) return s;
        for (size_t k = 0; k < w.size(); ++k)
            out[k] = s == MPM_TIMEOUT ? MPM_TIMEOUT : (w[k] ? MPM_NUMERIC : MPM_OK);
        return MPM_OK;
    }

    mpm_status metrics(int i, mpm_metrics* out) override {
        Range nvtx_range("mpm.metrics");
        if (!out) {
            err = "metrics output is NULL";
            return MPM_INVALID_ARG;
        }
        InstHost& x = I[i];
        mpm_status s = ensure_binned();
        if (s != MPM_OK) return s;
        const double mu = x.p.E / (2.0 * (1.0 + x.p.nu));
        const double K = x.p.E / (3.0 * (1.0 - 2.0 * x.p.nu));
        // at least 4 particles per thread (256-thread CTAs), at most stat_blocks CTAs
        const int nb = (int)std::max<int64_t>(1, std::min<int64_t>(stat_blocks, (x.np + 4 * 256 - 1) / (4 * 256)));
        launch_stats<R>(d_inst + i, ps[cur], x.pbase, x.np, mu, K, x.p.rho_phys, x.p.cp, x.p.Tamb, d_stat_part, nb,
                        d_stat_out, st);
        double v[kStatSlots];
        unsigned long long ctr[4];
        double fsum[2];
        CK(cudaMemcpyAsync(v, d_stat_out, sizeof(v), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ctr, d_ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(fsum, d_ctr + 4, sizeof(fsum), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        // a NaN or Inf that never reached the positions (a temperature, stress or
        // plastic strain of a live particle) shows in the FP64 sums: it marks the
        // instance's word too (byte 0)
        bool finite = true;
        for (int k : {0, 1, 2, 3, 4, 5, 6, 10, 13, 14}) finite = finite && std::isfinite(v[k]);
        if (!finite) {
            const unsigned char one = 1;
            CK(cudaMemcpyAsync(d_ierr + i, &one, 1, cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        std::memset(out, 0, sizeof(*out));
        out->mass = v[0];
        out->momentum[0] = v[1]; out->momentum[1] = v[2]; out->momentum[2] = v[3];
        out->kinetic = v[4];
        out->internal_elastic = v[5];
        out->thermal = v[6];
        out->max_temperature = x.p.Tamb + (std::isfinite(v[7]) ? v[7] : 0.0);
        out->max_von_mises = v[8];
        out->max_plastic_strain = std::isfinite(v[9]) ? v[9] : 0.0;
        const double nlive = (double)x.np - v[18];
        out->mean_plastic_strain = nlive > 0 ? v[10] / nlive : 0.0;
        out->ref_max_stress = v[11];
        out->ref_max_temperature = v[12];
        out->ref_kinetic = v[13];
        out->ref_internal = v[14];
        out->n_active = (int64_t)v[15];
        out->n_chip = (int64_t)v[16];
        out->n_fixed = (int64_t)v[17];
        out->n_inactive = (int64_t)v[18];
        for (int a = 0; a < 3; ++a) {
            out->bounds_min[a] = v[19 + a];
            out->bounds_max[a] = v[22 + a];
        }
        out->n_escaped = (int64_t)ctr[0];
        out->n_sorts = n_sorts;
        out->n_yielded = (int64_t)ctr[1];
        out->n_contacts = (int64_t)ctr[2];
        out->contact_work = fsum[0];
        out->contact_force = fsum[1];
        out->n_asb_heated = (int64_t)ctr[3];
        return inst_status(i);
    }

    // ---------------------------------------------------------------- misc

    mpm_status set_mass_scaling(int i, double f) override {
        InstHost& x = I[i];
        if (!(f > 0.0)) {
            err = "mass scaling factor must be positive";
            return MPM_INVALID_ARG;
        }
        const double rho = std::max(x.p.rho_phys * f, x.p.rho_phys);
        x.p.particle_mass = rho * x.p.particle_volume;
        return push_insts();
    }
    mpm_status ext_force(int i, const double c[3], double r, const double f[3]) override {
        InstHost& x = I[i];
        if (!c || !f || !(r > 0.0)) {
            err = "external force needs a center, a positive radius and a force";
            return MPM_INVALID_ARG;
        }
        for (int a = 0; a < 3; ++a) { x.ext_c[a] = c[a]; x.ext_f[a] = f[a]; }
        x.ext_r = r;
        x.ext_pending = true;
        return MPM_OK;
    }
    mpm_status set_temps(int i, const double* T, int64_t count) override {
        InstHost& x = I[i];
        if (!T || count < 0 || count > x.np) {
            err = "temperature count out of range";
            return MPM_INVALID_ARG;
        }
        mpm_status s = ensure_binned();
        if (s != MPM_OK) return s;
        double* d = nullptr;
        CK(cudaMalloc(&d, 8 * std::max<int64_t>(count, 1)));
        CK(cudaMemcpyAsync(d, T, 8 * count, cudaMemcpyHostToDevice, st));
        launch_set_temps<R>(ps[cur], x.pbase, x.np, d, count, x.p.Tamb, st);
        CK(cudaStreamSynchronize(st));
        cudaFree(d);
        return MPM_OK;
    }
    // ---------------------------------------------------------------- checkpoints

    // Device pointer (at the instance's first slot) and bytes per particle of
    // every array of a checkpoint, in the order of ckpt_array_elem.
    std::vector<std::pair<char*, size_t>> ckpt_arrays(const PState<R>& s, int64_t pbase) const {
        const size_t v4 = sizeof(V4<R>);
        std::vector<std::pair<char*, size_t>> a;
        for (int k = 0; k < 6; ++k) a.push_back({(char*)(s.A[k] + pbase), v4});
        for (int k = 0; k < 4; ++k) a.push_back({(char*)(s.B[k] + pbase), v4});
        for (int k = 0; k < 2; ++k) a.push_back({(char*)(s.S[k] + pbase), v4});
        if (has_K)
            for (int k = 0; k < 2; ++k) a.push_back({(char*)(s.K[k] + pbase), v4});
        if (kPosLo) a.push_back({(char*)(s.X + pbase), v4});
        a.push_back({(char*)(s.sres + pbase), sizeof(R)});
        a.push_back({(char*)(s.status + pbase), 1});
        a.push_back({(char*)(s.asb + pbase), 1});
        a.push_back({(char*)(s.id + pbase), 4});
        a.push_back({(char*)(s.bin + pbase), 4});
        a.push_back({(char*)(s.orig + pbase), 4});
        a.push_back({(char*)(s.skey + pbase), 4});
        return a;
    }
    int ckpt_samples(const InstHost& x) const { return x.tool.mode == MPM_TOOL_RASTER ? x.n_samples : 0; }

    mpm_status checkpoint_bytes(int i, int64_t* bytes) override {
        const InstHost& x = I[i];
        *bytes = (int64_t)(sizeof(CkptHeader) + ckpt_payload_bytes(prec_, has_K, x.np, ckpt_samples(x)));
        return MPM_OK;
    }

    mpm_status checkpoint_save(int i, void* buf, int64_t bytes) override {
        Range nvtx_range("mpm.checkpoint_save");
        MS(ensure_binned());
        InstHost& x = I[i];
        const int ns = ckpt_samples(x);
        const uint64_t pay = ckpt_payload_bytes(prec_, has_K, x.np, ns);
        if (!buf || bytes < (int64_t)(sizeof(CkptHeader) + pay)) {
            err = "checkpoint buffer NULL or smaller than mpm_checkpoint_bytes";
            return MPM_INVALID_ARG;
        }
        unsigned char* q = static_cast<unsigned char*>(buf) + sizeof(CkptHeader);
        for (const auto& a : ckpt_arrays(ps[cur], x.pbase)) {
            if (x.np > 0) CK(cudaMemcpyAsync(q, a.first, a.second * x.np, cudaMemcpyDeviceToHost, st));
            q += a.second * x.np;
        }
        if (ns > 0) CK(cudaMemcpyAsync(q, x.d_samples, 24 * (size_t)ns, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CkptHeader h;
        std::memset(&h, 0, sizeof(h));
        std::memcpy(h.magic, kCkptMagic, sizeof(kCkptMagic));
        h.version = kCkptVersion;
        h.abi_version = MPM_ABI_VERSION;
        h.precision = prec_;
        h.has_K = has_K ? 1 : 0;
        h.n_samples = ns;
        h.np = x.np;
        h.since_rebin = x.since;
        h.step = x.step;
        h.time = x.time;
        h.tool_t0 = x.tool_t0;
        h.dt = x.dt;
        h.payload_bytes = pay;
        h.checksum = ckpt_checksum(static_cast<const unsigned char*>(buf) + sizeof(CkptHeader), pay);
        h.params = x.p;
        h.tool = x.tool;
        h.tool.sample_dx = h.tool.sample_dy = h.tool.sample_dz = nullptr;
        std::memcpy(buf, &h, sizeof(h));
        return MPM_OK;
    }

    mpm_status checkpoint_load(int i, const void* buf, int64_t bytes) override {
        Range nvtx_range("mpm.checkpoint_load");
        InstHost& x = I[i];
        CkptHeader h;
        mpm_status s = ckpt_check(buf, bytes, prec_, has_K, x.p.nx, x.p.ny, x.p.nz, x.cap, &h, &err);
        if (s != MPM_OK) return s;
        if ((s = check_params(&h.params, &err)) != MPM_OK) return s;
        if (h.params.H_kin > 0.0 && !has_K) {
            err = "checkpoint uses backstress (H_kin > 0); the handle has no backstress state";
            return MPM_NOT_SUPPORTED;
        }
        CK(cudaStreamSynchronize(st));   // nothing in flight uses the instance's slots
        // The one allocation (the raster samples) comes before anything of the
        // instance is overwritten: a refusal here leaves the old state whole.
        double* samples = nullptr;
        if (h.n_samples > 0) CK(cudaMalloc(&samples, 24 * (size_t)h.n_samples));
        // From here on a failure leaves the particle arrays part old, part new:
        // the instance is marked broken, and steps refuse it until a complete
        // state replaces it.
        x.broken = true;
        const unsigned char* q = static_cast<const unsigned char*>(buf) + sizeof(CkptHeader);
        const int64_t n = h.np;
        auto copy_in = [&]() -> mpm_status {
            for (const auto& a : ckpt_arrays(ps[cur], x.pbase)) {
                const bool is_K = has_K && !h.has_K && (a.first == (char*)(ps[cur].K[0] + x.pbase) ||
                                                        a.first == (char*)(ps[cur].K[1] + x.pbase));
                if (is_K) {
                    // a checkpoint without backstress into a handle that has it: zero
                    if (n > 0) CK(cudaMemsetAsync(a.first, 0, a.second * n, st));
                    continue;
                }
                if (n > 0) CK(cudaMemcpyAsync(a.first, q, a.second * n, cudaMemcpyHostToDevice, st));
                q += a.second * n;
            }
            if (h.n_samples > 0)
                CK(cudaMemcpyAsync(samples, q, 24 * (size_t)h.n_samples, cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(d_ierr + i, 0, sizeof(int), st));
            CK(cudaStreamSynchronize(st));
            return MPM_OK;
        };
        if ((s = copy_in()) != MPM_OK) {
            if (samples) cudaFree(samples);
            err = "checkpoint load failed part-way; the workpiece must be uploaded or loaded again (" + err + ")";
            return s;
        }
        if (x.d_samples) cudaFree(x.d_samples);   // the stream is idle (synchronised above)
        x.d_samples = samples;
        x.n_samples = h.n_samples > 0 ? h.n_samples : 0;
        x.samples_cap = x.n_samples;
        x.has_nodes = false;   // a node source (device pointers) is not part of a checkpoint
        x.broken = false;
        x.p = h.params;
        x.tool = h.tool;
        x.np = n;
        x.since = std::max(h.since_rebin, 0);
        x.rebin_now = false;
        x.step = h.step;
        x.time = h.time;
        x.tool_t0 = h.tool_t0;
        x.dt = h.dt;
        x.fresh = 0;
        x.ext_pending = false;
        x.pext_pending = false;
        binned = false;   // the next call re-bins; the loaded instance keeps its saved layout
        return push_insts();
    }

    mpm_status reset_clock(int i) override {
        I[i].time = 0.0;
        I[i].step = 0;
        I[i].tool_t0 = 0.0;
        return push_insts();
    }
    mpm_status sync() override {
        CK(cudaStreamSynchronize(st));
        return device_status();
    }
};

std::unique_ptr<EngineBase> make_engine(const mpm_params* params, const int64_t* caps, int n, cudaStream_t st,
                                        mpm_status* status, std::string* err) {
    if (!params || n < 0 || (n > 0 && !caps)) {
        *status = MPM_INVALID_ARG;
        *err = "no instances";
        return nullptr;
    }
    if (params[0].precision == MPM_PREC_F64) {
        auto e = std::make_unique<Engine<double>>();
        *status = e->init(params, caps, n, st);
        if (*status != MPM_OK) {
            *err = e->err;
            return nullptr;
        }
        return e;
    }
    auto e = std::make_unique<Engine<float>>();
    *status = e->init(params, caps, n, st);
    if (*status != MPM_OK) {
        *err = e->err;
        return nullptr;
    }
    return e;
}

}  // namespace mpmb
