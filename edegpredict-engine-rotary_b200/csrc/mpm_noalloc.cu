// mpm_noalloc.cu -- mpm_metrics_aos_noalloc: the workpiece metrics of a
// device array of MPMParticle records (include/Types.h:199-266, 504 bytes),
// reduced on the GPU without allocating anything.
//
// Who needs it: code that holds the reference's particle array on the device
// (the reference solver's own d_particles, a ContactSolver or exporter buffer,
// or mpm_export_aos written to device memory) and cannot create a handle --
// mpm_create allocates device state for the particles, and some callers may
// not allocate at all (a fixed device-memory budget carved up at start-up, a
// real-time loop that must not enter the allocator, a process whose memory
// pool is full).  The reference computes these quantities on the host after
// copying every particle back (MPMSolver::syncMetrics, src/MPMSolver.cu:
// 1239-1259, over getParticles); here they come back as one 256-byte result.
//
// Scratch: one file-scope device array, g_metrics_scratch, holding a row of
// kStatSlots FP64 partials per block and one result row.  Each block reduces a
// fixed range of kRecordsPerBlock records, so n is limited to
// kMaxBlocks * kRecordsPerBlock = 67,108,864 particles (1 MiB of scratch);
// larger n is refused with MPM_CAPACITY before anything is launched.  Nothing
// in the scratch has to start at zero: every call writes each partial row and
// the result row before it reads them.  Because the ranges are fixed, the
// summation order -- and so the result -- depends only on n and the data.
//
// Every call looks up the scratch's device address on the current device
// (cudaGetSymbolAddress, which on the first call also loads this library's
// kernels onto that device) and checks the lookup; nothing is cached, so a
// cudaDeviceReset, a torn-down primary context or another current context
// gets the address that is valid in it.  The call synchronises its stream,
// so it cannot be made while that stream is being captured.  The scratch is
// shared by every caller on a device, so calls on one device must not
// overlap: two calls in flight at once (from two host threads, or on two
// streams) race on it and both results are wrong.  Each call waits for its
// own result before returning.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/mpm_capi.h"
#include "mpm_internal.h"

namespace mpmb {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int64_t kRecordsPerBlock = 16384;
constexpr int kMaxBlocks = 4096;
constexpr int64_t kMaxRecords = kMaxBlocks * kRecordsPerBlock;  // 67,108,864

// kMaxBlocks partial rows, then the result row.
__device__ __align__(256) double g_metrics_scratch[(kMaxBlocks + 1) * kStatSlots];

// Slot layout of the reduction (the same as the handle path's k_stats):
//  0 mass 1-3 momentum 4 kinetic 5 elastic 6 thermal 7 max dT 8 max vm 9 max eps
//  10 sum eps 11 ref max stress 12 ref max T 13 ref kinetic 14 ref internal
//  15 n active 16 n chip 17 n fixed 18 n inactive 19-21 bmin 22-24 bmax
__device__ __forceinline__ bool slot_is_min(int q) { return q >= 19 && q < 22; }
__device__ __forceinline__ bool slot_is_max(int q) {
    return q == 7 || q == 8 || q == 9 || q == 11 || q == 12 || (q >= 22 && q < 25);
}
__device__ __forceinline__ double slot_combine(int q, double a, double b) {
    return slot_is_min(q) ? fmin(a, b) : (slot_is_max(q) ? fmax(a, b) : a + b);
}

// Block b reduces records [b*kRecordsPerBlock, min(n, (b+1)*kRecordsPerBlock))
// into partial row b.  Mass, volume, density and temperature are read per
// record (the reference stores them per particle).
__global__ void __launch_bounds__(kNoAllocThreads) k_aos_stats(const AosParticle* __restrict__ rec, int64_t n,
                                                               double mu, double K, double cp, double Tamb,
                                                               double* __restrict__ partial) {
    __shared__ double sh[kStatSlots][kNoAllocThreads / 32];
    double acc[kStatSlots];
    for (int q = 0; q < kStatSlots; ++q) acc[q] = 0.0;
    acc[7] = -INFINITY; acc[9] = -INFINITY;
    for (int q = 19; q < 22; ++q) acc[q] = INFINITY;
    for (int q = 22; q < 25; ++q) acc[q] = -INFINITY;
    const int64_t lo = (int64_t)blockIdx.x * kRecordsPerBlock;
    const int64_t hi = min(n, lo + kRecordsPerBlock);
    for (int64_t i = lo + threadIdx.x; i < hi; i += kNoAllocThreads) {
        const AosParticle& r = rec[i];
        const int st = __ldg(&r.status);
        if (st == ST_INACTIVE) { acc[18] += 1.0; continue; }
        if (st == ST_ACTIVE) acc[15] += 1.0;
        else if (st == ST_CHIP) acc[16] += 1.0;
        else if (st == ST_FIXED) acc[17] += 1.0;
        const double m = __ldg(&r.mass), V = __ldg(&r.volume), rho = __ldg(&r.density);
        const double sxx = __ldg(&r.stress_xx), syy = __ldg(&r.stress_yy), szz = __ldg(&r.stress_zz);
        const double sxy = __ldg(&r.stress_xy), sxz = __ldg(&r.stress_xz), syz = __ldg(&r.stress_yz);
        const double tr = sxx + syy + szz;
        const double dx_ = sxx - tr / 3.0, dy_ = syy - tr / 3.0, dz_ = szz - tr / 3.0;
        const double vm = sqrt(1.5 * (dx_ * dx_ + dy_ * dy_ + dz_ * dz_ + 2.0 * (sxy * sxy + sxz * sxz + syz * syz)));
        const double vx = __ldg(&r.vx), vy = __ldg(&r.vy), vz = __ldg(&r.vz);
        const double v2 = vx * vx + vy * vy + vz * vz;
        const double dT = __ldg(&r.temperature) - Tamb, eps = __ldg(&r.plasticStrain);
        acc[0] += m;
        acc[1] += m * vx; acc[2] += m * vy; acc[3] += m * vz;
        acc[4] += 0.5 * m * v2;
        const double pr = tr / 3.0;
        acc[5] += V * (vm * vm / (6.0 * mu) + pr * pr / (2.0 * K));
        acc[6] += rho * V * cp * dT;
        acc[7] = fmax(acc[7], dT);
        acc[8] = fmax(acc[8], vm);
        acc[9] = fmax(acc[9], eps);
        acc[10] += eps;
        if (st == ST_ACTIVE || st == ST_CHIP) {
            // computeParticleStatsKernel (src/MPMSolver.cu:729-788): its fixed
            // 80 GPa shear modulus is part of the reported quantity
            acc[11] = fmax(acc[11], vm);
            acc[12] = fmax(acc[12], Tamb + dT);
            acc[13] += 0.5 * m * v2;
            acc[14] += (vm * vm * m) / (6.0 * 80e9) + V * eps * vm;
            const double xw[3] = {__ldg(&r.x), __ldg(&r.y), __ldg(&r.z)};
            for (int q = 0; q < 3; ++q) {
                acc[19 + q] = fmin(acc[19 + q], xw[q]);
                acc[22 + q] = fmax(acc[22 + q], xw[q]);
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kStatSlots; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v = slot_combine(q, v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) sh[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < kStatSlots) {
        const int q = threadIdx.x;
        double v = sh[q][0];
        for (int w = 1; w < kNoAllocThreads / 32; ++w) v = slot_combine(q, v, sh[q][w]);
        partial[(int64_t)blockIdx.x * kStatSlots + q] = v;
    }
}

// One warp: lane q combines partial rows 0..nb-1 of slot q in row order and
// writes slot q of the result row.
__global__ void k_aos_stats_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= kStatSlots) return;
    double v = partial[q];
    for (int b = 1; b < nb; ++b) v = slot_combine(q, v, partial[(int64_t)b * kStatSlots + q]);
    out[q] = v;
}

mpm_status fail(mpm_status s, const std::string& m) {
    set_lib_error("mpm_metrics_aos_noalloc: " + m);
    return s;
}

// Device address of g_metrics_scratch in the current context of the current
// device.  Looked up on every call rather than cached per device ordinal: a
// cached address would outlive a cudaDeviceReset or a primary-context
// teardown, and would belong to another context when the caller makes a
// non-primary context current, and a kernel given it would write through a
// stale or foreign pointer.
mpm_status scratch_on_current_device(double** out) {
    int dev = -1;
    cudaError_t rc = cudaGetDevice(&dev);
    if (rc != cudaSuccess) return fail(MPM_CUDA_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(rc));
    void* p = nullptr;
    rc = cudaGetSymbolAddress(&p, g_metrics_scratch);
    if (rc != cudaSuccess || !p)
        return fail(MPM_CUDA_ERROR, std::string("cudaGetSymbolAddress(g_metrics_scratch) on device ") +
                                        std::to_string(dev) + ": " + cudaGetErrorString(rc));
    *out = static_cast<double*>(p);
    return MPM_OK;
}

}  // namespace
}  // namespace mpmb

extern "C" mpm_status mpm_metrics_aos_noalloc(const mpm_params* p, const void* d_particles, int64_t n, void* stream,
                                              mpm_metrics* out) {
    using namespace mpmb;
    if (!p || !out) return fail(MPM_INVALID_ARG, "params or output is NULL");
    if (p->abi_version != MPM_ABI_VERSION) return fail(MPM_INVALID_ARG, "params.abi_version does not match MPM_ABI_VERSION");
    if (!(p->E > 0.0) || !(p->nu > -1.0 && p->nu < 0.5)) return fail(MPM_INVALID_ARG, "E > 0 and -1 < nu < 0.5 required");
    if (n < 0) return fail(MPM_INVALID_ARG, "n is negative");
    if (n > kMaxRecords)
        return fail(MPM_CAPACITY, "n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                                      std::to_string(kMaxRecords) + " particles (" + std::to_string(kMaxBlocks) +
                                      " blocks x " + std::to_string(kRecordsPerBlock) +
                                      "); use mpm_sync_metrics on a handle instead");
    if (n > 0 && !d_particles) return fail(MPM_INVALID_ARG, "d_particles is NULL");
    if (reinterpret_cast<uintptr_t>(d_particles) % 8 != 0) return fail(MPM_INVALID_ARG, "d_particles is not 8-byte aligned");

    double* scratch = nullptr;
    mpm_status s = scratch_on_current_device(&scratch);
    if (s != MPM_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = n > 0 ? (int)((n + kRecordsPerBlock - 1) / kRecordsPerBlock) : 1;
    double* result = scratch + (int64_t)kMaxBlocks * kStatSlots;
    const double mu = p->E / (2.0 * (1.0 + p->nu));
    const double K = p->E / (3.0 * (1.0 - 2.0 * p->nu));
    k_aos_stats<<<nb, kNoAllocThreads, 0, st>>>(static_cast<const AosParticle*>(d_particles), n, mu, K, p->cp,
                                                p->Tamb, scratch);
    k_aos_stats_final<<<1, 32, 0, st>>>(scratch, nb, result);
    launch_counter() += 2;
    cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess) return fail(MPM_CUDA_ERROR, std::string("launch: ") + cudaGetErrorString(rc));
    double v[kStatSlots];
    rc = cudaMemcpyAsync(v, result, sizeof(v), cudaMemcpyDeviceToHost, st);
    if (rc == cudaSuccess) rc = cudaStreamSynchronize(st);
    if (rc != cudaSuccess) return fail(MPM_CUDA_ERROR, std::string("result copy: ") + cudaGetErrorString(rc));

    std::memset(out, 0, sizeof(*out));
    out->mass = v[0];
    out->momentum[0] = v[1]; out->momentum[1] = v[2]; out->momentum[2] = v[3];
    out->kinetic = v[4];
    out->internal_elastic = v[5];
    out->thermal = v[6];
    out->max_temperature = p->Tamb + (std::isfinite(v[7]) ? v[7] : 0.0);
    out->max_von_mises = v[8];
    out->max_plastic_strain = std::isfinite(v[9]) ? v[9] : 0.0;
    const double nlive = (double)n - v[18];
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
    return MPM_OK;
}
