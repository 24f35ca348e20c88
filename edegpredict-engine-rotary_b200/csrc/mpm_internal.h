// mpm_internal.h -- launchers shared by the C ABI (mpm_capi.cu) and the
// kernels (mpm_step.cu, mpm_aux.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/mpm_capi.h"
#include "mpm_device.cuh"

namespace mpmb {

// An NVTX range over a scope: the step's phases show by name on the timeline
// of Nsight Systems or any other NVTX tool; without a tool attached the push
// and pop are calls to no-ops.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Device copies of an upload (NULL field = MPMParticle default).
struct DevSoA {
    int elem;  // 4 or 8
    const void *x, *y, *z, *vx, *vy, *vz, *F, *Fp, *C, *stress, *bs, *eps, *edot, *T, *D, *sres;
    const int32_t *status, *id;
};

struct DevSoAOut {
    int elem;
    void *x, *y, *z, *vx, *vy, *vz, *F, *Fp, *C, *stress, *bs, *eps, *edot, *T, *D, *sres;
    int32_t *status, *id;
};

// MPMParticle, include/Types.h:199-266 (504 bytes): the byte layout that the
// reference's ContactSolver, CFD coupling and exporters read.
struct AosParticle {
    double x, y, z, vx, vy, vz, fx, fy, fz, ext_fx, ext_fy, ext_fz;
    double density, pressure, volume, mass, temperature;
    double F[9], F_p[9], C[9];
    double stress_xx, stress_yy, stress_zz, stress_xy, stress_xz, stress_yz;
    double backstress_xx, backstress_yy, backstress_zz, backstress_xy, backstress_xz, backstress_yz;
    double plasticStrain, strainRate, damage, residualStress;
    int32_t id, status, cellHash, lodZone, lastUpdateStep;
    uint8_t asbCounter;
};
static_assert(sizeof(AosParticle) == 504, "MPMParticle layout is 504 bytes");

// One instance of a relayout: its first slot in the new layout, its first
// slot in the old one and the particles to carry over (0 for a new instance).
struct RelayoutMap {
    int64_t new_pbase, old_pbase, np;
};

// Number of stats accumulators (see k_stats).
constexpr int kStatSlots = 32;

// One heat-conduction diffusion step on grid buffer b of every instance that
// conducts heat (node temperatures into Inst::tn).
template <typename R>
void launch_heat_diffuse(const Inst<R>* insts, int n_inst, int b, int64_t total, cudaStream_t st);

template <typename R>
void launch_step(const Inst<R>* insts, const Work* work, const int* n_work, int max_work, const PState<R>& ps,
                 const StepArgs& a, int rbuf, bool g2p, bool p2g, int threads, int ctas_per_sm, int* err,
                 unsigned long long* counters, cudaStream_t st);

// Deterministic mode: the grid buffer b of every instance from the node
// tiles the step launch stored per work item (part, part_items items) and the
// escaped fixed-point sums; one CTA per two bins of the batch bin table.
template <typename R>
void launch_node_sum(const Inst<R>* insts, const int32_t* bin_inst, const int32_t* bin_local, const int32_t* flag,
                     const int32_t* flag_scan, const R* part, int64_t part_items, int b, int nbins_total,
                     cudaStream_t st);

template <typename R>
void launch_bin_count(const Inst<R>* insts, int n_inst, const PState<R>& ps, const int32_t* key_base, bool initial,
                      const double* pos_scratch, int32_t* key, int32_t* rank, int32_t* count, int32_t* newbin,
                      int64_t np, int kpt, int sort_every, bool keep_all, cudaStream_t st);

// The re-bin's move: every particle to its slot in the new layout, each
// cell's particles in the order of their old slots (bin_key: the first key
// of each of the nbins_total bins of the bin table).
template <typename R>
void launch_bin_scatter(const PState<R>& src, const PState<R>& dst, const Inst<R>* insts, int n_inst,
                        const int32_t* key, const int32_t* rank, const int32_t* offset, const int32_t* key_base,
                        const int32_t* newbin, bool initial, const double* pos_scratch, bool has_K, int64_t np,
                        int32_t* perm, const int32_t* bin_key, int nbins_total, cudaStream_t st);
// (perm holds 2 np int32: the permutation, then its sources' upload positions)

template <typename R>
void launch_pad_counts(const Inst<R>* insts, int n_inst, const int32_t* key_base, int32_t* count, cudaStream_t st);

// The raster tool of instance i at step k of the current call (samples or FEM
// node records, pose and blend from the instance record) into its tool mask;
// npoints = samples or nodes.
template <typename R>
void launch_raster(const Inst<R>* insts, int i, int k, int npoints, cudaStream_t st);

template <typename R>
void launch_import(const DevSoA& in, int64_t n, double ox, double oy, double oz, double dx, double Tamb,
                   const PState<R>& ps, int64_t pbase, double* pos_scratch, cudaStream_t st);

// Seeded box generator: writes the kept candidates at [pbase, pbase + kept).
// flag/idx hold ncand int32 each; scan_tmp >= scan_tmp_size(ncand).
template <typename R>
void launch_gen(const Inst<R>& P, const int32_t c0[3], const int32_t c1[3], int ppc, uint64_t seed, uint32_t inst,
                int fixed_layers, double dT0, int tool_check, int32_t* flag, int32_t* idx, int32_t* scan_tmp,
                const PState<R>& ps, int64_t pbase, double* pos_scratch, cudaStream_t st);

template <typename R>
void launch_export(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double Tamb,
                   const DevSoAOut& out, cudaStream_t st);

template <typename R>
void launch_export_aos(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double Tamb,
                       double rho, void* out, cudaStream_t st);

// Reads `fields` (MPM_AOS_*) of n MPMParticle records (device memory, upload
// order) back into the particle state; the external force goes to pext
// (indexed pbase + upload order).  flags[0]: a particle moved (re-bin);
// flags[1]: records whose status is outside 0..4.
template <typename R>
void launch_import_aos(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double Tamb,
                       uint32_t fields, const void* in, V4<R>* pext, int* flags, cudaStream_t st);

// One step of MPMWorkpieceSolver's semantics for every instance (np, nn:
// particles and nodes of each): P2G into grid buffer 0 and tm[0], the grid
// update (contact force into *fsum), diffuse_fn when diffuse, G2P and chip
// separation.  use_ext: the first step of a call (pending external forces).
template <typename R>
void launch_ws_step(const Inst<R>* insts, const std::vector<int64_t>& np, const std::vector<int64_t>& nn,
                    const PState<R>& ps, int k, int use_ext, int diffuse, double* fsum, cudaStream_t st,
                    void (*diffuse_fn)(const Inst<R>*, int, int, int64_t, cudaStream_t), int64_t nn_total);

template <typename R>
void launch_stats(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double mu, double K,
                  double rho, double cp, double Tamb, double* partial, int nblocks, double* out, cudaStream_t st);

// Copies particles [old_pbase, old_pbase + np) of every instance of `map`
// (sorted by new_pbase) from src to [new_pbase, ...) of dst; total = slots of
// the new layout.
template <typename R>
void launch_relayout(const PState<R>& src, const PState<R>& dst, const RelayoutMap* map, int n_inst, int64_t total,
                     cudaStream_t st);

template <typename R>
void launch_set_temps(const PState<R>& ps, int64_t pbase, int64_t n, const double* T, int64_t count, double Tamb,
                      cudaStream_t st);

// Device-wide exclusive scan of n int32 (in -> out), tmp >= scan_tmp_size(n).
int64_t scan_tmp_size(int64_t n);
void exclusive_scan(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t st);
// Ordered work list (one item per non-empty bin) from the key offsets; the
// bin table gives each global bin its first key, instance and local index.
void build_work(const int32_t* offset, const int32_t* bin_key, const int32_t* bin_inst, const int32_t* bin_local,
                const int64_t* inst_pbase, int64_t nbins_total, int32_t* flag, int32_t* flag_scan, int32_t* tmp,
                Work* work, int* n_work, cudaStream_t st);
void fill_i32(int32_t* p, int32_t v, int64_t n, cudaStream_t st);

// Kernel launches issued by this process (all handles and the handle-free
// entry points), counted atomically: any host thread may launch.
std::atomic<int64_t>& launch_counter();

// The calling thread's error string, returned by mpm_last_error(NULL).
void set_lib_error(const std::string& m);

// Runs a kernel whose bounded mbarrier wait (the one guarding the step
// kernel's tile loads) must give up after limit_ns: MPM_TIMEOUT when it did.
mpm_status wait_selftest(int64_t limit_ns, cudaStream_t st, std::string* err);

}  // namespace mpmb
