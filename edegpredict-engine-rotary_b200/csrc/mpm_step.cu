// mpm_step.cu -- the MPM step kernel for sm_100a.
//
// One CTA takes one bin (4^3 stencil-base cells = the particles whose 3^3
// quadratic stencils start inside the bin) at a time:
//   G2P part  : the bin's 6^3 node tile of the previous grid is fetched by TMA
//               into shared memory; the grid update (gravity, fixture damping,
//               tool boundary) is applied per node while it is staged; each
//               particle gathers v, the APIC moments and the velocity gradient
//               through separable tensor-product contractions, then moves and
//               updates C, F - I and the strain rate (restates g2pKernel,
//               reference src/MPMSolver.cu:506-605, and chip separation :1002-1060).
//   P2G part  : the Johnson-Cook return (p2gKernel :123-365) and the APIC
//               scatter of mass and momentum+force impulse into a shared-memory
//               tile (:370-421), pre-reduced there by shared atomics; the tile
//               is then flushed into the next grid with one 128-bit vector
//               atomic per node.
// FUSED schedule: launch k runs G2P of step k and P2G of step k+1 on the same
// particle without a round trip through memory (velocity, C and strain rate
// stay in registers), so a step costs one pass over the particles.  SPLIT
// schedule: separate P2G and G2P launches per step, like the reference.
#include <cuda.h>
#include <cuda_runtime.h>

#include "mpm_device.cuh"
#include "mpm_internal.h"

namespace mpmb {

// Bounds-checked builds (-DMPMB_CHECKED, libmpm_b200_checked.so): every index
// the step kernels derive from data is checked before it is used; a failed
// check counts, records the first site and index (mpm_check_report) and skips
// the access, so no check traps.  Default builds compile every check away.
enum : int { kSiteParticle = 1, kSiteFlush = 2, kSiteScatter = 3, kSiteGather = 4, kSiteHeat = 5, kSiteBin = 6,
             kSiteNodeSum = 7, kSitePart = 8 };
#ifdef MPMB_CHECKED
struct CheckRecord {
    unsigned long long count;
    long long index;
    int site;
    int pad;
};
static __device__ CheckRecord g_check;
__device__ __noinline__ bool check_fail(int site, long long index) {
    if (atomicAdd(&g_check.count, 1ull) == 0ull) {
        g_check.site = site;
        g_check.index = index;
    }
    return false;
}
#define MPMB_CHECK(cond, site, index) ((cond) ? true : check_fail((site), (long long)(index)))
#else
#define MPMB_CHECK(cond, site, index) true
#endif

// ------------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Particle state is read and written once per step: streaming loads and
// stores (evict-first) keep L1 for the register spills and L2 for the grid
// tiles and stored node tiles (1.7 % off the fused step on 33.5 M particles,
// 1.5 % on the 512-workpiece batch).  FP64 keeps plain accesses.
__device__ __forceinline__ float4 ldcs4(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ D4 ldcs4(const D4* p) { return *p; }
__device__ __forceinline__ void stcs4(float4* p, const float4 v) { __stcs(p, v); }
__device__ __forceinline__ void stcs4(D4* p, const D4 v) { *p = v; }
__device__ __forceinline__ void tmap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}
// 4-D tiled TMA load (no multicast): coordinates innermost first.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the mbarrier phase with a time limit (ns); false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = gtimer();
    while (!mbar_try_wait(bar, parity)) {
        if (gtimer() - t0 > limit_ns) return false;
    }
    return true;
}

// Self-test of mbar_wait_bounded: one thread waits on an mbarrier that nothing
// arrives at (no copy in flight), gives up after limit_ns, invalidates the
// barrier and records the outcome (1: gave up, 0: completed).
__global__ void k_wait_selftest(uint64_t limit_ns, int* out) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    const bool done = mbar_wait_bounded(&bar, 0, limit_ns);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar)) : "memory");
    *out = done ? 0 : 1;
}

mpm_status wait_selftest(int64_t limit_ns, cudaStream_t st, std::string* err) {
    int* d = nullptr;
    int h = -1;
    cudaError_t e = cudaMalloc(&d, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0xff, sizeof(int), st);
    if (e == cudaSuccess) {
        k_wait_selftest<<<1, 32, 0, st>>>((uint64_t)limit_ns, d);
        ++launch_counter();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        *err = std::string("bounded-wait self-test: ") + cudaGetErrorString(e);
        return MPM_CUDA_ERROR;
    }
    if (h != 1) {
        *err = "bounded-wait self-test: the wait did not give up";
        return MPM_CUDA_ERROR;
    }
    *err = "bounded-wait self-test: the device wait gave up after its limit (expected)";
    return MPM_TIMEOUT;
}

template <typename R> __device__ __forceinline__ void vec_atomic_add(V4<R>* dst, R a, R b, R c, R d);
template <> __device__ __forceinline__ void vec_atomic_add<float>(float4* dst, float a, float b, float c, float d) {
    atomicAdd(dst, make_float4(a, b, c, d));  // one 128-bit vector reduction (sm_90+)
}
template <> __device__ __forceinline__ void vec_atomic_add<double>(D4* dst, double a, double b, double c, double d) {
    atomicAdd(&dst->x, a);
    atomicAdd(&dst->y, b);
    atomicAdd(&dst->z, c);
    atomicAdd(&dst->w, d);
}

// ------------------------------------------------------------------ grid node update

// Grid update of one node, restating updateGridKernel (src/MPMSolver.cu:424-442),
// applyFixtureBCKernel (:82-110) and the tool boundary: rasterizeToolKernel +
// applyGridCollisionKernel (:444-492) in raster mode, or the analytic SDF.
// Nodes at or below the mass threshold have zero velocity and contribute
// nothing to the gather, as g2pKernel skips them (:543).
template <typename R> struct NV {
    R x, y, z;
};

template <typename R>
__device__ __forceinline__ NV<R> node_vel_inl(const Inst<R>& P, const V4<R> g, int gx, int gy, int gz, double pr0,
                                              double pr2) {
    const R m = g.x;
    NV<R> out{R(0), R(0), R(0)};
    if (!(m > (R)P.mthr)) return out;
    R vx = g.y / m, vy = g.z / m, vz = (g.w + m * (R)(P.grav * P.dt)) / m;
    if (P.fix_thick > 0.0) {
        const double zr = ds(node_coord(gz, P.dx, P.oz), P.oz) / P.fix_thick;
        if (zr <= 1.0) {
            if (gz == 0) {
                vx = vy = vz = R(0);
            } else if (zr > 0.0) {
                const double s = dm(dm(P.fix_damp, ds(1.0, zr)), ds(1.0, zr));
                const R f = (R)(1.0 / da(1.0, dm(s, P.dt)));
                vx *= f; vy *= f; vz *= f;
            }
        }
    }
    if (P.tool_mode == TOOL_RASTER) {
        const int32_t mk = P.tool_mask[gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz)];
        if (mk) {
            if (P.tn_end) {
                // the velocity of the tool node that marked it
                const unsigned char* r = P.tn_end + (int64_t)(mk - 1) * P.tn_stride;
                vx = (R)*reinterpret_cast<const double*>(r + P.tn_off[3]);
                vy = (R)*reinterpret_cast<const double*>(r + P.tn_off[4]);
                vz = (R)*reinterpret_cast<const double*>(r + P.tn_off[5]);
            } else {
                vx = (R)P.tool_v[0]; vy = (R)P.tool_v[1]; vz = (R)P.tool_v[2];
            }
        }
    } else if ((P.tool_mode == TOOL_SDF_STICKY || P.tool_mode == TOOL_SDF_SLIP) &&
               !tool_far(P, node_coord(gx, P.dx, P.ox), node_coord(gz, P.dx, P.oz), pr0, pr2)) {
        double nrm[3];
        const double phi = tool_sdf(P, node_coord(gx, P.dx, P.ox), node_coord(gz, P.dx, P.oz), pr0, pr2, nrm);
        if (phi <= 0.0) {
            if (P.tool_mode == TOOL_SDF_STICKY) {
                vx = (R)P.tool_v[0]; vy = (R)P.tool_v[1]; vz = (R)P.tool_v[2];
            } else {
                const double rx = ds((double)vx, P.tool_v[0]), ry = ds((double)vy, P.tool_v[1]),
                             rz = ds((double)vz, P.tool_v[2]);
                const double vn = da(da(dm(rx, nrm[0]), dm(ry, nrm[1])), dm(rz, nrm[2]));
                if (vn < 0.0) {
                    vx = (R)ds((double)vx, dm(vn, nrm[0]));
                    vy = (R)ds((double)vy, dm(vn, nrm[1]));
                    vz = (R)ds((double)vz, dm(vn, nrm[2]));
                }
            }
        }
    }
    out.x = vx; out.y = vy; out.z = vz;
    return out;
}

// Out-of-line copy for the slow-path gather (keeps its 27 node updates small).
template <typename R>
__device__ __noinline__ NV<R> node_vel(const Inst<R>& P, const V4<R> g, int gx, int gy, int gz, double pr0, double pr2) {
    return node_vel_inl<R>(P, g, gx, gy, gz, pr0, pr2);
}

// ------------------------------------------------------------------ gather (G2P)

// Separable contraction over the 3x3x3 stencil from the velocity tile:
//   v_a   = sum w v_a,  M_ab = sum w v_a o_b  (o = stencil offset 0,1,2),
//   L_ab  = sum v_a dw_b  (cell units).
// k (z) first: Z0 = sum wz v, Z1 = sum k wz v, Z2 = sum dwz v; then j; then i.
// Node velocity tile of a bin, one 16-byte (FP32) record per node at
// vidx(x, y, z) = x + 12 y + 72 z: the 8 lanes of a quarter warp (cells x 0-3,
// y = 2m, 2m + 1 of one z layer) read 8 distinct 4-bank groups, so a warp's
// 128-bit gathers are conflict-free.
constexpr int kVY = 12, kVZ = 72, kVPlane = kVZ * kTile;
__device__ __forceinline__ int vidx(int x, int y, int z) { return x + kVY * y + kVZ * z; }

template <typename R>
__device__ __forceinline__ void gather_tile(const V4<R>* vel, int base, const R (&w)[3][3], const R (&dw)[3][3],
                                            R v[3], R M[3][3], R L[3][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        v[c] = R(0);
#pragma unroll
        for (int b = 0; b < 3; ++b) { M[c][b] = R(0); L[c][b] = R(0); }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R Y00[3] = {0, 0, 0}, Y01[3] = {0, 0, 0}, Y02[3] = {0, 0, 0}, Y10[3] = {0, 0, 0}, Y20[3] = {0, 0, 0};
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R Z0[3] = {0, 0, 0}, Z1[3] = {0, 0, 0}, Z2[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const V4<R> node = vel[base + i + kVY * j + kVZ * k];
                const R vn[3] = {node.x, node.y, node.z};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const R vv = vn[c];
                    Z0[c] = fma(w[2][k], vv, Z0[c]);
                    if (k == 1) Z1[c] = fma(w[2][1], vv, Z1[c]);
                    if (k == 2) Z1[c] = fma(R(2) * w[2][2], vv, Z1[c]);
                    Z2[c] = fma(dw[2][k], vv, Z2[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                Y00[c] = fma(w[1][j], Z0[c], Y00[c]);
                if (j) Y01[c] = fma(R(j) * w[1][j], Z0[c], Y01[c]);
                Y02[c] = fma(dw[1][j], Z0[c], Y02[c]);
                Y10[c] = fma(w[1][j], Z1[c], Y10[c]);
                Y20[c] = fma(w[1][j], Z2[c], Y20[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            v[c] = fma(w[0][i], Y00[c], v[c]);
            if (i) M[c][0] = fma(R(i) * w[0][i], Y00[c], M[c][0]);
            L[c][0] = fma(dw[0][i], Y00[c], L[c][0]);
            M[c][1] = fma(w[0][i], Y01[c], M[c][1]);
            L[c][1] = fma(w[0][i], Y02[c], L[c][1]);
            M[c][2] = fma(w[0][i], Y10[c], M[c][2]);
            L[c][2] = fma(w[0][i], Y20[c], L[c][2]);
        }
    }
}

// Same sums for a particle whose stencil left its bin's tile: nodes are read
// and updated straight from the grid (rare; the re-bin brings it back).  Out
// of line, with its inputs and result by value, so that the hot path keeps
// its arrays in registers.
template <typename R> struct GatherOut {
    R v[3], M[3][3], L[3][3];
};

template <typename R>
__device__ __noinline__ GatherOut<R> gather_global(const Inst<R>& P, const V4<R>* __restrict__ grid, int g0x, int g0y,
                                                   int g0z, R x0, R x1, R x2, double pr0, double pr2) {
    GatherOut<R> o;
    R w[3][3], dw[3][3];
    int gb[3];
    gb[0] = g0x + bspline(x0, w[0], dw[0]);
    gb[1] = g0y + bspline(x1, w[1], dw[1]);
    gb[2] = g0z + bspline(x2, w[2], dw[2]);
    for (int c = 0; c < 3; ++c) {
        o.v[c] = R(0);
        for (int b = 0; b < 3; ++b) { o.M[c][b] = R(0); o.L[c][b] = R(0); }
    }
    // the 27 node loads first, all in flight together, then the node updates
    V4<R> gv[27];
    bool in[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int gx = gb[0] + q / 9, gy = gb[1] + (q / 3) % 3, gz = gb[2] + q % 3;
        const int64_t gi = gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz);
        in[q] = gx >= 0 && gx < P.nx && gy >= 0 && gy < P.ny && gz >= 0 && gz < P.nz &&
                MPMB_CHECK(gi >= 0 && gi < P.nn, kSiteGather, gi);
        gv[q] = in[q] ? grid[gi] : mk4<R>(R(0), R(0), R(0), R(0));
    }
    for (int i = 0; i < 3; ++i) {
        const int gx = gb[0] + i;
        for (int j = 0; j < 3; ++j) {
            const int gy = gb[1] + j;
            for (int k = 0; k < 3; ++k) {
                const int gz = gb[2] + k;
                if (!in[i * 9 + j * 3 + k]) continue;
                const NV<R> nv = node_vel(P, gv[i * 9 + j * 3 + k], gx, gy, gz, pr0, pr2);
                const R vv[3] = {nv.x, nv.y, nv.z};
                const R ww = w[0][i] * w[1][j] * w[2][k];
                const R g0 = dw[0][i] * w[1][j] * w[2][k], g1 = w[0][i] * dw[1][j] * w[2][k],
                        g2 = w[0][i] * w[1][j] * dw[2][k];
                for (int c = 0; c < 3; ++c) {
                    o.v[c] += ww * vv[c];
                    o.M[c][0] += ww * vv[c] * R(i);
                    o.M[c][1] += ww * vv[c] * R(j);
                    o.M[c][2] += ww * vv[c] * R(k);
                    o.L[c][0] += vv[c] * g0;
                    o.L[c][1] += vv[c] * g1;
                    o.L[c][2] += vv[c] * g2;
                }
            }
        }
    }
    return o;
}

// ------------------------------------------------------------------ scatter (P2G)

// Momentum + impulse at node (i,j,k):
//   p_a = w_ijk (Q_a + R_ax i + R_ay j + R_az k) + S_ax dwx wy wz + S_ay wx dwy wz + S_az wx wy dwz
// with Q = m (v - dx C d), R = m dx C, S = -dt V J sigma / dx.  Separable in k.
// Scatter of a particle whose stencil left its bin's tile: straight into the
// grid with vector atomics (rare; out of line, inputs by value).
template <typename R> struct ScatterIn {
    R xi[3], Q[3], Rm[9], S[9];
    int g0[3];
};

// Deterministic mode: channel ch of node gi gets v in fixed point (rounded to
// a multiple of 1/esc_scale, clamped to +-4e18 units; integer adds commute, so
// the escaped sums do not depend on the order of the particles).
template <typename R>
__device__ __forceinline__ void esc_add(const Inst<R>& P, int64_t gi, int ch, R v) {
    const double q = fmin(fmax((double)v * P.esc_scale, -4.0e18), 4.0e18);
    atomicAdd(&P.esc[ch * P.esc_stride + gi], (unsigned long long)__double2ll_rn(q));
}
// ... and marks the bin whose 4x4x4 core holds node (gx, gy, gz) for k_node_sum.
template <typename R> __device__ __forceinline__ void esc_mark(const Inst<R>& P, int gx, int gy, int gz) {
    P.esc_flag[gx / kBin + P.nbx * (gy / kBin + P.nby * (gz / kBin))] = 1;
}

template <typename R>
__device__ __noinline__ void scatter_global(const Inst<R>& P, V4<R>* __restrict__ grid, const ScatterIn<R> in, R m) {
    R w[3][3], dw[3][3];
    int gb[3];
    for (int a = 0; a < 3; ++a) gb[a] = in.g0[a] + bspline(in.xi[a], w[a], dw[a]);
    for (int i = 0; i < 3; ++i) {
        const int gx = gb[0] + i;
        if (gx < 0 || gx >= P.nx) continue;
        for (int j = 0; j < 3; ++j) {
            const int gy = gb[1] + j;
            if (gy < 0 || gy >= P.ny) continue;
            for (int k = 0; k < 3; ++k) {
                const int gz = gb[2] + k;
                if (gz < 0 || gz >= P.nz) continue;
                const R ww = w[0][i] * w[1][j] * w[2][k];
                const R g0 = dw[0][i] * w[1][j] * w[2][k], g1 = w[0][i] * dw[1][j] * w[2][k],
                        g2 = w[0][i] * w[1][j] * dw[2][k];
                R p[3];
                for (int a = 0; a < 3; ++a)
                    p[a] = ww * (in.Q[a] + in.Rm[a * 3] * R(i) + in.Rm[a * 3 + 1] * R(j) + in.Rm[a * 3 + 2] * R(k)) +
                           in.S[a * 3] * g0 + in.S[a * 3 + 1] * g1 + in.S[a * 3 + 2] * g2;
                const int64_t gi = gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz);
                if (!MPMB_CHECK(gi >= 0 && gi < P.nn, kSiteScatter, gi)) continue;
                if (P.esc) {
                    esc_add<R>(P, gi, 0, ww * m);
                    esc_add<R>(P, gi, 1, p[0]);
                    esc_add<R>(P, gi, 2, p[1]);
                    esc_add<R>(P, gi, 3, p[2]);
                    esc_mark<R>(P, gx, gy, gz);
                } else {
                    vec_atomic_add<R>(&grid[gi], ww * m, p[0], p[1], p[2]);
                }
            }
        }
    }
}

// Heat conduction on the global paths (particles whose stencil left the bin
// tile): the T m scatter into the write buffer, and the temperature gather
// over the nodes with m > 1e-18 (sum of w T and of w), as the tile paths do.
template <typename R>
__device__ __noinline__ void scatter_T_global(const Inst<R>& P, R* __restrict__ tw, int g0x, int g0y, int g0z, R x0,
                                              R x1, R x2, R mT) {
    R w[3][3], dw[3][3];
    int gb[3];
    gb[0] = g0x + bspline(x0, w[0], dw[0]);
    gb[1] = g0y + bspline(x1, w[1], dw[1]);
    gb[2] = g0z + bspline(x2, w[2], dw[2]);
    for (int i = 0; i < 3; ++i) {
        const int gx = gb[0] + i;
        if (gx < 0 || gx >= P.nx) continue;
        for (int j = 0; j < 3; ++j) {
            const int gy = gb[1] + j;
            if (gy < 0 || gy >= P.ny) continue;
            for (int k = 0; k < 3; ++k) {
                const int gz = gb[2] + k;
                if (gz < 0 || gz >= P.nz) continue;
                const int64_t gi = gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz);
                if (!MPMB_CHECK(gi >= 0 && gi < P.nn, kSiteHeat, gi)) continue;
                if (P.esc) {
                    esc_add<R>(P, gi, 4, w[0][i] * w[1][j] * w[2][k] * mT);
                    esc_mark<R>(P, gx, gy, gz);
                } else {
                    atomicAdd(&tw[gi], w[0][i] * w[1][j] * w[2][k] * mT);
                }
            }
        }
    }
}

template <typename R> struct TSum {
    R ts, ws;
};

template <typename R>
__device__ __noinline__ TSum<R> gather_T_global(const Inst<R>& P, const V4<R>* __restrict__ grid, int g0x, int g0y,
                                                int g0z, R x0, R x1, R x2) {
    R w[3][3], dw[3][3];
    int gb[3];
    gb[0] = g0x + bspline(x0, w[0], dw[0]);
    gb[1] = g0y + bspline(x1, w[1], dw[1]);
    gb[2] = g0z + bspline(x2, w[2], dw[2]);
    TSum<R> o{R(0), R(0)};
    for (int i = 0; i < 3; ++i) {
        const int gx = gb[0] + i;
        if (gx < 0 || gx >= P.nx) continue;
        for (int j = 0; j < 3; ++j) {
            const int gy = gb[1] + j;
            if (gy < 0 || gy >= P.ny) continue;
            for (int k = 0; k < 3; ++k) {
                const int gz = gb[2] + k;
                if (gz < 0 || gz >= P.nz) continue;
                const int64_t q = gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz);
                const R ww = w[0][i] * w[1][j] * w[2][k];
                if (!(ww > R(0)) || !(grid[q].x > R(1e-18))) continue;
                o.ts += P.tn[q] * ww;
                o.ws += ww;
            }
        }
    }
    return o;
}

// ------------------------------------------------------------------ Johnson-Cook

// Consistent return (extension of this build), FP64: q - 3 mu dg = Y(eps + dg)
// on [0, q/3mu], Newton steps safeguarded by bisection; rate and temperature
// terms frozen at the step start.  Returns false when it did not converge.
__device__ __noinline__ bool newton_return(double q, double mu, double eps0, double A, double B, double n, double rt,
                                           double tt, double tol_rel, int maxit, double* out) {
    double lo = 0.0, hi = q / (3.0 * mu);
    double x = (q - (A + B * pow(eps0, n)) * rt * tt) / (3.0 * mu);
    if (!(x > lo)) x = 0.5 * (lo + hi);
    if (x > hi) x = hi;
    const double tol = tol_rel * q;
    for (int it = 0; it < maxit; ++it) {
        const double e = eps0 + x;
        const double fx = q - 3.0 * mu * x - (A + B * pow(e, n)) * rt * tt;
        if (fabs(fx) <= tol) { *out = x; return true; }
        if (fx > 0.0) lo = x; else hi = x;
        const double dY = (e > 0.0) ? B * n * pow(e, n - 1.0) * rt * tt : (double)INFINITY;
        const double d = -3.0 * mu - dY;
        double xn = x - fx / d;
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (hi - lo <= 1e-15 * hi) { *out = xn; return true; }
        x = xn;
    }
    *out = x;
    return false;
}

// det(I + X) - 1 without cancellation.
template <typename R> __device__ __forceinline__ R detm1(const R X[9]) {
    const R tr = X[0] + X[4] + X[8];
    const R i2 = X[0] * X[4] - X[1] * X[3] + X[0] * X[8] - X[2] * X[6] + X[4] * X[8] - X[5] * X[7];
    const R i3 = X[0] * (X[4] * X[8] - X[5] * X[7]) - X[1] * (X[3] * X[8] - X[5] * X[6]) +
                 X[2] * (X[3] * X[7] - X[4] * X[6]);
    return tr + i2 + i3;
}

struct JCOut {
    bool ran, yielded, to_chip;
};

// Elastic stress and Johnson-Cook return of one ACTIVE particle, restating
// p2gKernel (src/MPMSolver.cu:164-365) on F - I and F_p - I:
//   F_e - I = (H - Hp)(I + Hp)^-1,  J - 1 = det(I + E) - 1 (clamped to +-0.1),
//   B - I = E + E^T + E E^T,  sigma = mu/J (B - I) + lambda (J - 1) I.
// The return rescales only the diagonal and upper off-diagonal entries of the
// deviator (:239-248); the lower entries yx, zx, zy keep their trial values and
// enter the force (:406-408) and the F_p update (:282-294).  sl[3] carries them.
// The flow-stress part of the return (rate and thermal factors, the radial
// return, F_p, plastic heating and damage) for a particle whose trial stress
// can reach the flow stress.  Out of line and with its state passed by value,
// so that the common elastic path keeps fewer registers.
template <typename R> struct JCFlow {
    R Hp[9], sig[6], sl[3], sd[6], bs[6], e[6];
    R eps, dT, D, q, p3, Ts, edot, tt;
    int errf;
    bool yielded, to_chip;
};

template <typename R>
__device__ __noinline__ JCFlow<R> jc_flow(const Inst<R>& P, JCFlow<R> f, R* bsx, R* sres_p, int inst_tag) {
    R(&Hp)[9] = f.Hp;
    R(&sig)[6] = f.sig;
    R(&sl)[3] = f.sl;
    R(&sd)[6] = f.sd;
    R(&bs)[6] = f.bs;
    R& eps = f.eps;
    R& dT = f.dT;
    R& D = f.D;
    int& errf = f.errf;
    const R q = f.q, p3 = f.p3, Ts = f.Ts, edot = f.edot, tt = f.tt;
    const R ex = f.e[0], ey = f.e[1], ez = f.e[2], exy = f.e[3], exz = f.e[4], eyz = f.e[5];
    JCOut o{true, false, false};
    const R es = fmax(edot / P.edot0, R(1e-5));
    const R rt = R(1) + P.C * log(es);
    const R Y = (P.A + P.B * ((eps > R(0) || !(P.n > R(0))) ? pow(eps, P.n) : R(0))) * rt * tt;
    if (q > Y && q > R(1e-12)) {
        R dE, Yr = Y;
        if (P.plast == 1) {
            double dg;
            if (!newton_return((double)q, (double)P.mu, (double)eps, (double)P.A, (double)P.B, (double)P.n, (double)rt,
                               (double)tt, P.newton_tol, P.newton_maxit, &dg)) {
                // the failing instance (tag = index + 1, from the record's address) in
                // a register; a second instance failing on this thread makes it -1
                const int tag = inst_tag;
                errf = (errf == 0 || errf == tag) ? tag : -1;
            }
            dE = (R)dg;
            Yr = (R)((double)q - 3.0 * (double)P.mu * dg);
        } else {
            dE = (q - Y) / fmax(R(3) * P.mu, R(1e-12));
            if (dE > P.deps_cap) dE = P.deps_cap;
        }
        const R sc = Yr / q;
        sd[0] = bs[0] + sc * ex; sd[1] = bs[1] + sc * ey; sd[2] = bs[2] + sc * ez;
        sd[3] = bs[3] + sc * exy; sd[4] = bs[4] + sc * exz; sd[5] = bs[5] + sc * eyz;
        sig[0] = sd[0] + p3; sig[1] = sd[1] + p3; sig[2] = sd[2] + p3;
        sig[3] = sd[3]; sig[4] = sd[4]; sig[5] = sd[5];
        if (dE > R(0)) {
            o.yielded = true;
            if (bsx && P.Hkin > R(0)) {
                const R ns = P.Hkin * dE / q;
                bsx[0] += ns * ex; bsx[1] += ns * ey; bsx[2] += ns * ez;
                bsx[3] += ns * exy; bsx[4] += ns * exz; bsx[5] += ns * eyz;
            }
            eps += dE;
            // F_p <- (I + a s) F_p / cbrt(det), a = 1.5 dE/|s|, :277-302, as
            // Hp' = Hp + a (s + s Hp), then (I + Hp')/c - I = (Hp' - (c - 1) I)/c
            const R sn = sqrt(sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2] +
                              R(2) * (sd[3] * sd[3] + sd[4] * sd[4] + sd[5] * sd[5]));
            const R al = (sn > R(1e-12)) ? (R(1.5) * dE / sn) : R(0);
            const R S9[9] = {sd[0], sd[3], sd[4], sl[0], sd[1], sd[5], sl[1], sl[2], sd[2]};
            R N[9];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    N[r * 3 + c] = Hp[r * 3 + c] +
                                   al * (S9[r * 3 + c] + S9[r * 3] * Hp[c] + S9[r * 3 + 1] * Hp[3 + c] +
                                         S9[r * 3 + 2] * Hp[6 + c]);
            const R dm1 = detm1(N);
            R cb, cbm1;
            if (R(1) + dm1 > R(1e-12)) {
                cb = cbrt(R(1) + dm1);
                cbm1 = dm1 / (cb * cb + cb + R(1));
            } else {
                cb = cbrt(R(1e-12));
                cbm1 = cb - R(1);
            }
            const R ic = R(1) / cb;
#pragma unroll
            for (int q2 = 0; q2 < 9; ++q2) Hp[q2] = ((q2 % 4 == 0) ? (N[q2] - cbm1) : N[q2]) * ic;
            // plastic-work heating, :310-321 (dT is the rise above T_amb)
            R dTinc = P.heat * Yr * dE;
            if (dTinc > P.dT_cap) dTinc = P.dT_cap;
            dT += dTinc;
            if (dT > P.dTmax) dT = P.dTmax;
            // Johnson-Cook damage, :329-358
            const R tri = p3 / fmax(q, R(1e-12));
            const R ef = (P.D1 + P.D2 * exp(P.D3 * tri)) * (R(1) + P.D4c * log(fmax(es, R(1)))) * (R(1) + P.D5 * Ts);
            if (ef > R(1e-12)) {
                D += dE / ef;
                if (D > R(0.7) * P.Dth) {
                    R dg = (P.Dth - D) / (P.Dth * R(0.3));
                    dg = fmax(R(0), fmin(R(1), dg));
#pragma unroll
                    for (int q2 = 0; q2 < 6; ++q2) sig[q2] *= dg;
                    sl[0] *= dg; sl[1] *= dg; sl[2] *= dg;
                    const R rs = sqrt(R(1.5) * (sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2] +
                                                R(2) * (sd[3] * sd[3] + sd[4] * sd[4] + sd[5] * sd[5])));
                    *sres_p = fmax(*sres_p, rs);
                }
                if (D >= P.Dth) o.to_chip = true;
            }
        }
    }
    f.yielded = o.yielded;
    f.to_chip = o.to_chip;
    return f;
}

template <typename R>
__device__ __forceinline__ JCOut jc_update(const Inst<R>& P, const R H[9], R Hp[9], R& eps, R& dT, R& D, R edot,
                                           R sig[6], R sl[3], R& J, R* sres_p, R* bsx, int& errf,
                                           int inst_tag) {
    JCOut o{true, false, false};
    // inverse of G = I + Hp (identity when |det G| < 1e-12, inv3x3 :50-57);
    // a particle that never yielded has Hp = 0 exactly and F_e = F
    R E[9];
    bool hp0 = true;
#pragma unroll
    for (int q = 0; q < 9; ++q) hp0 = hp0 && (Hp[q] == R(0));
    if (hp0) {
#pragma unroll
        for (int q = 0; q < 9; ++q) E[q] = H[q];
    } else {
        const R dgm1 = detm1(Hp);
        const R det = R(1) + dgm1;
        R Gi[9];
        if (fabs(det) < R(1e-12)) {
#pragma unroll
            for (int q = 0; q < 9; ++q) Gi[q] = (q % 4 == 0) ? R(1) : R(0);
        } else {
            const R g0 = R(1) + Hp[0], g4 = R(1) + Hp[4], g8 = R(1) + Hp[8];
            const R id = R(1) / det;
            Gi[0] = (g4 * g8 - Hp[5] * Hp[7]) * id;
            Gi[1] = -(Hp[1] * g8 - Hp[2] * Hp[7]) * id;
            Gi[2] = (Hp[1] * Hp[5] - Hp[2] * g4) * id;
            Gi[3] = -(Hp[3] * g8 - Hp[5] * Hp[6]) * id;
            Gi[4] = (g0 * g8 - Hp[2] * Hp[6]) * id;
            Gi[5] = -(g0 * Hp[5] - Hp[2] * Hp[3]) * id;
            Gi[6] = (Hp[3] * Hp[7] - g4 * Hp[6]) * id;
            Gi[7] = -(g0 * Hp[7] - Hp[1] * Hp[6]) * id;
            Gi[8] = (g0 * g4 - Hp[1] * Hp[3]) * id;
        }
        // F_e - I = (I + H) G^-1 - I = (H - Hp) G^-1 when G^-1 is exact; with the
        // identity fallback F_e = F, so F_e - I = H.
        if (fabs(det) < R(1e-12)) {
#pragma unroll
            for (int q = 0; q < 9; ++q) E[q] = H[q];
        } else {
            R Dm[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) Dm[q] = H[q] - Hp[q];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    E[r * 3 + c] = Dm[r * 3] * Gi[c] + Dm[r * 3 + 1] * Gi[3 + c] + Dm[r * 3 + 2] * Gi[6 + c];
        }
    }
    R jm1 = detm1(E);
    jm1 = fmin(fmax(jm1, R(-0.1)), R(0.1));  // J clamp [0.9, 1.1], :174-175
    J = R(1) + jm1;
    // B - I (symmetric)
    R b00 = R(2) * E[0] + E[0] * E[0] + E[1] * E[1] + E[2] * E[2];
    R b11 = R(2) * E[4] + E[3] * E[3] + E[4] * E[4] + E[5] * E[5];
    R b22 = R(2) * E[8] + E[6] * E[6] + E[7] * E[7] + E[8] * E[8];
    R b01 = E[1] + E[3] + E[0] * E[3] + E[1] * E[4] + E[2] * E[5];
    R b02 = E[2] + E[6] + E[0] * E[6] + E[1] * E[7] + E[2] * E[8];
    R b12 = E[5] + E[7] + E[3] * E[6] + E[4] * E[7] + E[5] * E[8];
    const R muJ = P.mu / J, lj = P.lam * jm1;
    R s[6] = {muJ * b00 + lj, muJ * b11 + lj, muJ * b22 + lj, muJ * b01, muJ * b02, muJ * b12};
    // Johnson-Cook return, :205-360
    const R tr = s[0] + s[1] + s[2];
    const R p3 = tr / R(3);
    R sd[6] = {s[0] - p3, s[1] - p3, s[2] - p3, s[3], s[4], s[5]};
    R bs[6] = {0, 0, 0, 0, 0, 0};
    if (bsx) {
#pragma unroll
        for (int q = 0; q < 6; ++q) bs[q] = bsx[q];
    }
    const R ex = sd[0] - bs[0], ey = sd[1] - bs[1], ez = sd[2] - bs[2], exy = sd[3] - bs[3], exz = sd[4] - bs[4],
            eyz = sd[5] - bs[5];
    const R q = sqrt(R(1.5) * (ex * ex + ey * ey + ez * ez + R(2) * (exy * exy + exz * exz + eyz * eyz)));
    R Ts = dT / P.Tspan;
    Ts = fmin(fmax(Ts, R(0)), R(1));
#pragma unroll
    for (int q2 = 0; q2 < 6; ++q2) sig[q2] = s[q2];
    sl[0] = s[3]; sl[1] = s[4]; sl[2] = s[5];
    // thermal factor of the flow stress (pow(0, y) is +0 for y > 0: skipped
    // for the common unheated particle)
    const R tt = R(1) - ((Ts > R(0) || !(P.m > R(0))) ? pow(Ts, P.m) : R(0));
    // a particle with q below the smallest flow stress the step can have
    // (ylo tt, heated or not: ylo bounds (A + B eps^n)(1 + C ln es) from
    // below) cannot yield: the flow stress itself is not needed
    if (q < P.ylo * tt) return o;
    JCFlow<R> f;
#pragma unroll
    for (int k = 0; k < 9; ++k) f.Hp[k] = Hp[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) { f.sig[k] = sig[k]; f.sd[k] = sd[k]; f.bs[k] = bs[k]; }
    f.sl[0] = sl[0]; f.sl[1] = sl[1]; f.sl[2] = sl[2];
    f.e[0] = ex; f.e[1] = ey; f.e[2] = ez; f.e[3] = exy; f.e[4] = exz; f.e[5] = eyz;
    f.eps = eps; f.dT = dT; f.D = D; f.q = q; f.p3 = p3; f.Ts = Ts; f.edot = edot; f.tt = tt; f.errf = errf;
    f = jc_flow<R>(P, f, bsx, sres_p, inst_tag);
#pragma unroll
    for (int k = 0; k < 9; ++k) Hp[k] = f.Hp[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = f.sig[k];
    sl[0] = f.sl[0]; sl[1] = f.sl[1]; sl[2] = f.sl[2];
    eps = f.eps; dT = f.dT; D = f.D; errf = f.errf;
    o.yielded = f.yielded;
    o.to_chip = f.to_chip;
    return o;
}

// ------------------------------------------------------------------ adiabatic shear heating

// Heating of one ACTIVE particle that passed the temperature and strain-rate
// guards of applyAdiabaticHeatingKernel (reference src/AdiabaticShearModel.cu:
// 139-176), temperatures as rises above Tamb: base heating
// beta sigma_vM edot dt / (rho cp) from the stored stress (xx, yy, zz, xy |
// xz, yz); the counter c of consecutive heated steps (capped at 10) switches
// on the localisation factor 1 + 1.5 (edot / rate_crit - 1) <= 2.5 from the
// third step above the critical rate; the step is then capped at the base
// heating (at most 100 K), so the factor never raises it, as in the
// reference; T is capped at max_temp_ratio * Tm (which can lower it).
template <typename R>
__device__ __forceinline__ R asb_heat(const Inst<R>& P, const V4<R>& s0, const V4<R>& s1, R edot, R dT, uint8_t& c) {
    const R d1 = s0.x - s0.y, d2 = s0.y - s0.z, d3 = s0.z - s0.x;
    const R seq = sqrt(R(0.5) * (d1 * d1 + d2 * d2 + d3 * d3 + R(6) * (s0.w * s0.w + s1.x * s1.x + s1.y * s1.y)));
    const R base = P.asb_heat * seq * edot * (R)P.dt;
    R inc = base;
    c = (uint8_t)min((int)c + 1, 10);
    if (edot > P.asb_crit && c >= 3) inc *= fmin(R(1) + R(1.5) * (edot / fmax(P.asb_crit, R(1)) - R(1)), R(2.5));
    const R cap = fmin(base, R(100));
    if (cap > R(0) && inc > cap) inc = cap;
    return fmin(dT + inc, P.asb_Tcap);
}

// The adiabatic shear heating of an ACTIVE particle pi past the temperature
// and strain-rate guards of applyAdiabaticHeatingKernel (:114-136), after its
// move: asb_heat on the stored stress and the particle's counter; returns the
// new temperature rise.  Out of line: only heated particles call it.
template <typename R>
__device__ __noinline__ R asb_update(const Inst<R>& P, const PState<R>& ps, int64_t pi, R edot, R dT,
                                     unsigned long long* ctr) {
    uint8_t c = ps.asb[pi];
    dT = asb_heat<R>(P, ps.S[0][pi], ps.S[1][pi], edot, dT, c);
    ps.asb[pi] = c;
    // one counter add per warp for the lanes heated here
    const unsigned hm = __activemask();
    if ((threadIdx.x & 31) == (unsigned)(__ffs(hm) - 1)) atomicAdd(&ctr[3], (unsigned long long)__popc(hm));
    return dT;
}

// ------------------------------------------------------------------ particle contact

// Particle-side tool contact of one particle after its move, restating
// xpbdContactSDFKernel (reference src/ContactSolver.cu:797-923) on the analytic
// SDF with its exact normal: within contact_r of the surface the particle is
// pushed out to contact_r, loses an approaching normal velocity, takes Coulomb
// friction on the tangential velocity taken with the normal component before
// that removal (:870-873), and is heated by (1 - heat partition) of the
// friction work, T capped at Tm (:885-904).  The scalar chain is FP64.  The
// push-out comes back as a displacement in cells (hit = false: no contact).
struct ContactOut {
    bool hit;
    double dxi[3];
    double work, force;
};

template <typename R>
__device__ __noinline__ ContactOut particle_contact(const Inst<R>& P, double wx, double wz, double pe0, double pe2,
                                                    R& vx, R& vy, R& vz, R& dT) {
    ContactOut o{false, {0.0, 0.0, 0.0}, 0.0, 0.0};
    if (tool_far(P, wx, wz, pe0, pe2, P.contact_r)) return o;   // phi > contact radius: no contact
    double nrm[3];
    const double sdf = tool_sdf(P, wx, wz, pe0, pe2, nrm);
    if (!(sdf < P.contact_r)) return o;
    const double pen = P.contact_r - sdf;
    if (!(pen > 0.0)) return o;
    o.hit = true;
    const double idx = 1.0 / P.dx;
    for (int a = 0; a < 3; ++a) o.dxi[a] = nrm[a] * pen * idx;
    double v[3] = {(double)vx, (double)vy, (double)vz};
    const double vdn = v[0] * nrm[0] + v[1] * nrm[1] + v[2] * nrm[2];
    if (vdn < 0.0)
        for (int a = 0; a < 3; ++a) v[a] -= vdn * nrm[a];
    double tv[3];
    for (int a = 0; a < 3; ++a) tv[a] = v[a] - vdn * nrm[a];
    const double tvm = sqrt(tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2]);
    const double m = (double)P.pmass;
    const double nf = tvm > 0.0 ? fmax(m * pen / (P.dt * P.dt), 1e-15) : 1e-15;
    const double fimp = P.contact_mu * nf * P.dt;
    if (tvm > 0.0 && fimp > 0.0) {
        const double sc = fmin(1.0, (fimp / fmax(m, 1e-15)) / tvm);
        for (int a = 0; a < 3; ++a) v[a] -= tv[a] * sc;
    }
    const double slip = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    o.work = nf * slip * P.dt;
    o.force = nf;
    const double heat = o.work * (1.0 - P.contact_hp);
    if (heat > 0.0) {
        const double pm = fmax(P.rho_phys, 1.0) * fmax((double)P.pvol, 1e-24);
        dT = (R)fmin((double)dT + heat / (fmax(pm, 1e-15) * P.cp), (double)P.dTmax);
    }
    vx = (R)v[0]; vy = (R)v[1]; vz = (R)v[2];
    return o;
}

// Particle-side contact on the voxel tool SDF, restating xpbdContactSDFKernel
// (reference src/ContactSolver.cu:797-923) operation by operation in its float
// and double arithmetic: world -> tool frame about the tool's reference point
// pe (:825-829), voxel coordinates and the grid test (:832-840), the distance
// through the texture (:843-845), the normal from central differences half a
// voxel apart (:848-859), push-out to the contact radius (:863-869), removal
// of an approaching normal velocity (:872-877), Coulomb friction with the
// tangential velocity taken before that removal (:881-898), heating by
// (1 - heat partition) of the friction work with T <= Tm (:901-916).  The
// float operations are written as round-to-nearest intrinsics so that none is
// contracted into a fused multiply-add.
template <typename R>
__device__ __noinline__ ContactOut particle_contact_sdf(const Inst<R>& P, double wx, double wy, double wz, double pe0,
                                                        double pe1, double pe2, R& vx, R& vy, R& vz, R& dT) {
    ContactOut o{false, {0.0, 0.0, 0.0}, 0.0, 0.0};
    const cudaTextureObject_t tex = (cudaTextureObject_t)P.sdf_tex;
    const float dx = __fsub_rn((float)wx, (float)pe0), dy = __fsub_rn((float)wy, (float)pe1);
    const float lx = __fadd_rn(__fmul_rn(dx, P.sdf_cos), __fmul_rn(dy, P.sdf_sin));
    const float ly = __fadd_rn(__fmul_rn(-dx, P.sdf_sin), __fmul_rn(dy, P.sdf_cos));
    const float lz = __fsub_rn((float)wz, (float)pe2);
    const float tx = __fdiv_rn(__fsub_rn(lx, P.sdf_o[0]), P.sdf_vox);
    const float ty = __fdiv_rn(__fsub_rn(ly, P.sdf_o[1]), P.sdf_vox);
    const float tz = __fdiv_rn(__fsub_rn(lz, P.sdf_o[2]), P.sdf_vox);
    if (tx < 0.0f || ty < 0.0f || tz < 0.0f || tx > (float)(P.sdf_n[0] - 1) || ty > (float)(P.sdf_n[1] - 1) ||
        tz > (float)(P.sdf_n[2] - 1))
        return o;
    const float rad = (float)P.contact_r;
    const float sdf = tex3D<float>(tex, tx, ty, tz);
    if (sdf >= rad) return o;
    const float eps = 0.5f;
    const float den = __fmul_rn(__fmul_rn(eps, 2.0f), P.sdf_vox);
    const float gx = __fdiv_rn(__fsub_rn(tex3D<float>(tex, __fadd_rn(tx, eps), ty, tz),
                                         tex3D<float>(tex, __fsub_rn(tx, eps), ty, tz)), den);
    const float gy = __fdiv_rn(__fsub_rn(tex3D<float>(tex, tx, __fadd_rn(ty, eps), tz),
                                         tex3D<float>(tex, tx, __fsub_rn(ty, eps), tz)), den);
    const float gz = __fdiv_rn(__fsub_rn(tex3D<float>(tex, tx, ty, __fadd_rn(tz, eps)),
                                         tex3D<float>(tex, tx, ty, __fsub_rn(tz, eps))), den);
    const float glen = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz)));
    if (glen < 1e-10f) return o;
    const float nx = __fdiv_rn(gx, glen), ny = __fdiv_rn(gy, glen), nz = __fdiv_rn(gz, glen);
    const float pen = __fsub_rn(rad, sdf);
    if (pen <= 0.0f) return o;
    o.hit = true;
    o.dxi[0] = (double)__fmul_rn(nx, pen) / P.dx;
    o.dxi[1] = (double)__fmul_rn(ny, pen) / P.dx;
    o.dxi[2] = (double)__fmul_rn(nz, pen) / P.dx;
    double ux = (double)vx, uy = (double)vy, uz = (double)vz;
    const float vdn = (float)__dadd_rn(__dadd_rn(__dmul_rn(ux, (double)nx), __dmul_rn(uy, (double)ny)),
                                       __dmul_rn(uz, (double)nz));
    if (vdn < 0.0f) {
        ux = __dsub_rn(ux, (double)__fmul_rn(vdn, nx));
        uy = __dsub_rn(uy, (double)__fmul_rn(vdn, ny));
        uz = __dsub_rn(uz, (double)__fmul_rn(vdn, nz));
    }
    const float tvx = __fsub_rn((float)ux, __fmul_rn(vdn, nx));
    const float tvy = __fsub_rn((float)uy, __fmul_rn(vdn, ny));
    const float tvz = __fsub_rn((float)uz, __fmul_rn(vdn, nz));
    const float tvm = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(tvx, tvx), __fmul_rn(tvy, tvy)), __fmul_rn(tvz, tvz)));
    const float pm = (float)P.pmass, dt = (float)P.dt;
    const float nf = (tvm > 0.0f) ? fmaxf(__fdiv_rn(__fmul_rn(pm, pen), __fmul_rn(dt, dt)), 1e-15f) : 1e-15f;
    const float fimp = __fmul_rn(__fmul_rn((float)P.contact_mu, nf), dt);
    if (tvm > 0.0f && fimp > 0.0f) {
        const float sc = fminf(1.0f, __fdiv_rn(__fdiv_rn(fimp, fmaxf(pm, 1e-15f)), tvm));
        ux = __dsub_rn(ux, (double)__fmul_rn(tvx, sc));
        uy = __dsub_rn(uy, (double)__fmul_rn(tvy, sc));
        uz = __dsub_rn(uz, (double)__fmul_rn(tvz, sc));
    }
    const float fx = (float)ux, fy = (float)uy, fz = (float)uz;
    const float slip = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)), __fmul_rn(fz, fz)));
    o.work = (double)__fmul_rn(__fmul_rn(nf, slip), dt);
    o.force = (double)fmaxf(nf, 1e-15f);
    const double heat = o.work * (1.0 - (double)(float)P.contact_hp);
    if (heat > 0.0) {
        const double pv = (double)P.pvol;
        const double vol = pv > 1e-24 ? pv : (double)P.pmass / fmax((double)P.pmass / pv, 1.0);
        const double mass_phys = fmax(P.rho_phys, 1.0) * fmax(vol, 1e-24);
        dT = (R)fmin((double)dT + heat / (fmax(mass_phys, 1e-15) * P.cp), (double)P.dTmax);
    }
    vx = (R)ux; vy = (R)uy; vz = (R)uz;
    return o;
}

// ------------------------------------------------------------------ the step kernel

// Particles staged per pass and scatter payload per particle: xi (bin-local,
// after the move), Q = m (v - dx C d) + f_ext dt, R = m dx C and
// S = -dt V J sigma / dx (row-major), in six 4-vectors grouped by the half of
// the cell's thread pair that reads them (h = 0 takes m and p_x: groups 0-2;
// h = 1 takes p_y and p_z: groups 0 and 2-5), so each half loads whole
// 128-bit words:
//   0 (xi_x, xi_y, xi_z, Q_x)  1 (R_xx, R_xy, R_xz, S_xx)  2 (S_xy, S_xz, Q_y, Q_z)
//   3 (R_yx, R_yy, R_yz, S_yx) 4 (S_yy, S_yz, R_zx, R_zy)  5 (R_zz, S_zx, S_zy, S_zz)
// and, in the extension variant, 6 (T, -, -, -).
// FP32 passes stage CH x 128 particles, CH in {1, 2, 4} (the launch
// config's pass size, 128 by default: about 2 per cell at 8 per cell; larger
// passes halve the barriers and node-tile adds per particle but hold more
// payload and registers, and measured slower on the current kernel); FP64
// passes stage 128.
#ifndef MPMB_MIN_CTAS
#define MPMB_MIN_CTAS 4
#endif
constexpr int kDefaultChunk = 1;
template <typename R, int CH> struct StepCfg {
    static constexpr int kChunk = sizeof(R) == 4 ? CH * kNT : kNT;
    static constexpr int kPerThread = kChunk / kNT;
    static constexpr int kMaskWords = kChunk / 32;   // words of a cell's slot mask
};
constexpr int kOff = 27;  // stencil offsets, off = i + 3j + 9k

// Staged particles of a pass are recorded per base cell as bit masks, so
// that the cell's thread pair takes them in a fixed order whatever order the
// atomics set the bits in.  In the column layout the particle in slot s of a
// pass is filed under cell s mod 64 (row s / 64) unless it overflowed its
// column or has moved since the re-bin: a "home" particle (base cell = s mod
// 64) sets bit s / 64 of its cell's home mask, any other sets bit s of the
// cell's foreign mask (kMaskWords words of 32 slots) and bit 31 of the home
// mask.  The cell takes its home rows in ascending order, then its foreign
// slots in ascending order.
template <typename R, int CH> struct SlotIter {
    uint32_t hb;      // home rows left
    uint32_t fb;      // foreign slots left in word fq
    int fq;           // current foreign word
    int n;            // staged slots of the cell
    int cell;
    // home: the cell's home mask; fmask: its foreign words (read only when
    // bit 31 of home says there are any)
    template <typename Mask>
    __device__ __forceinline__ SlotIter(uint32_t home, const Mask& fmask, int c)
        : hb(home & 0x7fffffffu), fb(0u), fq(-1), n(0), cell(c) {
        n = __popc(hb);
        if (home >> 31) {
#pragma unroll
            for (int q = 0; q < StepCfg<R, CH>::kMaskWords; ++q) n += __popc(fmask[q][c]);
        }
    }
    // the next staged slot (call n times): home rows first, then foreign slots
    template <typename Mask> __device__ __forceinline__ int next(const Mask& fmask) {
        if (hb) {
            const int b = __ffs((int)hb) - 1;
            hb &= hb - 1u;
            return (b << 6) | cell;
        }
        while (fb == 0u) fb = fmask[++fq][cell];
        const int b = __ffs((int)fb) - 1;
        fb &= fb - 1u;
        return (fq << 5) | b;
    }
};

// EXT: the kernel variant with the extensions (adiabatic shear heating, heat
// conduction), which adds the payload's absolute temperature (group 6), the
// T m node sums (nacc[4]) and the node temperature tile with its m > 1e-18
// mask (ttile).
template <typename R, bool EXT, int CH> struct StepSmem {
    // The TMA tile is read only by the fill at the start of a bin and the payload
    // only inside the bin's passes, with barriers between: one buffer holds both,
    // which keeps four CTAs within the 164 KB shared-memory carveout (92 KB of L1
    // left for the register spills).  (Loading the next bin's tile during the
    // passes, into a buffer of its own, measured 3 % slower: the thread that
    // issues it stalls on the next work item's descriptor.)
    union {
        V4<R> raw[kTileNodes];                           // TMA destination (offset 0 of the 128-byte aligned block)
        V4<R> pay[EXT ? 7 : 6][StepCfg<R, CH>::kChunk];  // scatter payload of the staged particles
    };
    V4<R> vel[kVPlane];                    // node velocities after the grid update (vidx layout)
    // the bin's node sums m, p_x, p_y, p_z (, T m) (tidx layout), one copy per
    // half of the bin's cells: each warp adds only to its own copy, so the
    // adds need no atomics (the flush sums the two)
    R nacc[2][EXT ? 5 : 4][kPlane];
    R ttile[EXT ? 2 : 1][EXT ? kPlane : 1];  // node temperatures and their m > 1e-18 mask
    // staged slots of each base cell, by pass parity (see SlotIter): home rows,
    // and foreign slots with bit s of word q for slot 32 q + s (the cells of a
    // warp read consecutive words)
    uint32_t hmask[2][kCellsPerBin];
    uint32_t fmask[2][StepCfg<R, CH>::kMaskWords][kCellsPerBin];
    // the work item's tool poses at the G2P step (x, y, z) and at the P2G step:
    // read where used (volatile), so that no thread holds them in registers
    // across the particle loop
    double pose[6];
    // the work item's instance record (the particle loop reads its constants
    // from here rather than holding them in registers)
    Inst<R> inst;
    uint64_t mbar;
    int fail;
};

template <typename R, bool EXT, int CH> constexpr size_t step_smem_bytes() { return sizeof(StepSmem<R, EXT, CH>); }

// Momentum + impulse of one channel a over the 27 stencil nodes (i,j,k) of a
// particle, relative to its base node:
//   w_ijk (Q + rx i + ry j + rz k) + sx dwx_i wy_j wz_k + sy wx_i dwy_j wz_k + sz wx_i wy_j dwz_k
// = wy_j (wx_i Az_k + Bx_i wz_k) + (wx_i Cy_j) wz_k
// with Az_k = Q wz_k + rz k wz_k + sz dwz_k, Bx_i = rx i wx_i + sx dwx_i,
// Cy_j = ry j wy_j + sy dwy_j: two FMAs per node.
template <typename R>
__device__ __forceinline__ void channel_add(const R (&w)[3][3], const R (&dw)[3][3], R Q, R rx, R ry, R rz, R sx,
                                            R sy, R sz, R (&acc)[27]) {
    R Az[3], Bx[3], Cy[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        Az[t] = fma(Q, w[2][t], fma(rz * R(t), w[2][t], sz * dw[2][t]));
        Bx[t] = fma(rx * R(t), w[0][t], sx * dw[0][t]);
        Cy[t] = fma(ry * R(t), w[1][t], sy * dw[1][t]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R Pk[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) Pk[k] = fma(w[0][i], Az[k], Bx[i] * w[2][k]);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const R Qij = w[0][i] * Cy[j];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int o = i + 3 * j + 9 * k;
                acc[o] = fma(w[1][j], Pk[k], fma(Qij, w[2][k], acc[o]));
            }
        }
    }
}

// Accumulation of one cell's staged particles (thread pair per cell: h = 0
// takes m and p_x, h = 1 takes p_y and p_z) in registers, then added to the
// 27 nodes of the cell's stencil in the warp's own copy of the node tile
// (half = the warp's half of the cells).  The adds run in 27 phases, one
// stencil offset each, separated by __syncwarp: within a phase the 32 cells
// of the warp (cz in {0,1} or {2,3}) address 32 distinct nodes, and tidx's z
// stride of 68 (4 mod 32) puts them in 32 distinct banks, so plain
// load-add-stores neither collide nor conflict (a shared-memory FP32 atomic
// costs several times a plain add on this part).  Every lane takes part in
// every phase (a cell without particles adds zeros), so the warp stays
// converged at each __syncwarp.  par: parity of the staging pass.
template <typename R, bool EXT, int CH>
__device__ __forceinline__ void cell_accumulate(StepSmem<R, EXT, CH>& Sm, int cell, int h, int half, R pm, int par,
                                                bool heat) {
    R a0[kOff], a1[kOff];
#pragma unroll
    for (int o = 0; o < kOff; ++o) { a0[o] = R(0); a1[o] = R(0); }
    constexpr int kW = StepCfg<R, CH>::kMaskWords;
    // the other parity's masks were last read in the previous pass: clear
    // them for the next one
    if (h == 0) {
        const uint32_t old = Sm.hmask[par ^ 1][cell];
        Sm.hmask[par ^ 1][cell] = 0u;
        if (old >> 31) {
#pragma unroll
            for (int q = 0; q < kW; ++q) Sm.fmask[par ^ 1][q][cell] = 0u;
        }
    }
    const uint32_t home = Sm.hmask[par][cell];
    SlotIter<R, CH> it(home, Sm.fmask[par], cell);
    for (int q = 0; q < it.n; ++q) {
        const int e = it.next(Sm.fmask[par]);
        R w[3][3], dw[3][3];
        const V4<R> g0 = Sm.pay[0][e], g2 = Sm.pay[2][e];
        (void)bspline(g0.x, w[0], dw[0]);
        (void)bspline(g0.y, w[1], dw[1]);
        (void)bspline(g0.z, w[2], dw[2]);
        if (h == 0) {
            const V4<R> g1 = Sm.pay[1][e];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const R mx = pm * w[0][i];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const R mxy = mx * w[1][j];
#pragma unroll
                    for (int k = 0; k < 3; ++k) a0[i + 3 * j + 9 * k] = fma(mxy, w[2][k], a0[i + 3 * j + 9 * k]);
                }
            }
            channel_add<R>(w, dw, g0.w, g1.x, g1.y, g1.z, g1.w, g2.x, g2.y, a1);
        } else {
            const V4<R> g3 = Sm.pay[3][e], g4 = Sm.pay[4][e], g5 = Sm.pay[5][e];
            channel_add<R>(w, dw, g2.z, g3.x, g3.y, g3.z, g3.w, g4.x, g4.y, a0);
            channel_add<R>(w, dw, g2.w, g4.z, g4.w, g5.x, g5.y, g5.z, g5.w, a1);
        }
    }
    // a warp whose 32 cells staged nothing in this pass (a sparse surface
    // bin) has only zeros to add
    const bool warp_any = __any_sync(0xffffffffu, home != 0u);
    if (warp_any) {
        const int base = tidx(cell & (kBin - 1), (cell / kBin) & (kBin - 1), cell / (kBin * kBin));
        R* __restrict__ t0 = Sm.nacc[half][2 * h];
        R* __restrict__ t1 = Sm.nacc[half][2 * h + 1];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const int o = i + 3 * j + 9 * k, t = base + i + kSY * j + kSZ * k;
                    __syncwarp();
                    t0[t] += a0[o];
                    t1[t] += a1[o];
                }
        __syncwarp();
    }
    if (EXT && heat && h == 0 && warp_any) {
        // heat conduction: the T m channel, w m T over the cell's particles (the
        // lighter half of the pair takes it)
#pragma unroll
        for (int o = 0; o < kOff; ++o) a0[o] = R(0);
        SlotIter<R, CH> ih(home, Sm.fmask[par], cell);
        for (int q = 0; q < ih.n; ++q) {
            const int e = ih.next(Sm.fmask[par]);
            R w[3][3], dw[3][3];
            const V4<R> g0 = Sm.pay[0][e];
            (void)bspline(g0.x, w[0], dw[0]);
            (void)bspline(g0.y, w[1], dw[1]);
            (void)bspline(g0.z, w[2], dw[2]);
            const R mT = pm * Sm.pay[EXT ? 6 : 0][e].x;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const R mx = mT * w[0][i];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const R mxy = mx * w[1][j];
#pragma unroll
                    for (int k = 0; k < 3; ++k) a0[i + 3 * j + 9 * k] = fma(mxy, w[2][k], a0[i + 3 * j + 9 * k]);
                }
            }
        }
        const int base = tidx(cell & (kBin - 1), (cell / kBin) & (kBin - 1), cell / (kBin * kBin));
        R* __restrict__ t4 = Sm.nacc[half][EXT ? 4 : 0];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    __syncwarp();
                    t4[base + i + kSY * j + kSZ * k] += a0[i + 3 * j + 9 * k];
                }
        __syncwarp();
    }
}

template <typename R, bool G2P, bool P2G, bool EXT, int CH>
__global__ void __launch_bounds__(kNT, MPMB_MIN_CTAS) k_step(const Inst<R>* __restrict__ insts, const Work* __restrict__ work,
                                              const int* __restrict__ n_work, PState<R> ps, StepArgs sa, int rbuf,
                                              int* __restrict__ err, unsigned long long* __restrict__ ctr) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    StepSmem<R, EXT, CH>& Sm = *reinterpret_cast<StepSmem<R, EXT, CH>*>(smem_raw);
    constexpr int kChunk = StepCfg<R, CH>::kChunk;
    const int tid = threadIdx.x, lane = tid & 31;
    const int nw = *n_work;
    uint32_t phase = 0;
    unsigned int c_esc = 0, c_yield = 0, c_contact = 0;   // per thread: far below 2^32
    double f_work = 0.0, f_force = 0.0;
    int errf = 0;   // Newton failures: 0 none, k > 0 instance k - 1 only, -1 several instances
    if (G2P && tid == 0) {
        mbar_init(&Sm.mbar, 1);
        fence_async_smem();
    }
    if (tid == 0) Sm.fail = 0;
    for (int q = tid; q < 2 * kCellsPerBin; q += kNT) (&Sm.hmask[0][0])[q] = 0u;
    for (int q = tid; q < 2 * StepCfg<R, CH>::kMaskWords * kCellsPerBin; q += kNT) (&Sm.fmask[0][0][0])[q] = 0u;
    // node sums start at zero; the end-of-bin flush clears what it reads
    if (P2G)
        for (int q = tid; q < 2 * (EXT ? 5 : 4) * kPlane; q += kNT) (&Sm.nacc[0][0][0])[q] = R(0);
    __syncthreads();
    int par = 0;  // parity of the staging pass (counts double-buffered across passes)
    int last_inst = -1;
    int cur_inst = -1;

    for (int wi = blockIdx.x; wi < nw; wi += gridDim.x) {
        const Work wk = work[wi];
        if (wk.inst != cur_inst) {
            // all threads are past the previous item (the barrier that ends it)
            const uint4* __restrict__ src = reinterpret_cast<const uint4*>(&insts[wk.inst]);
            uint4* dst = reinterpret_cast<uint4*>(&Sm.inst);
            for (int q = tid; q < (int)(sizeof(Inst<R>) / 16); q += kNT) dst[q] = src[q];
            cur_inst = wk.inst;
            __syncthreads();
        }
        const Inst<R>& P = Sm.inst;
        const Inst<R>& Pg = insts[wk.inst];   // the tensor maps are read from global memory
        const int bx = wk.bin % P.nbx, by = (wk.bin / P.nbx) % P.nby, bz = wk.bin / (P.nbx * P.nby);
        const int g0x = bx * kBin, g0y = by * kBin, g0z = bz * kBin;
        // (uniform across the CTA: a skipped work item skips for every thread)
        if (!MPMB_CHECK(wk.bin >= 0 && wk.bin < P.nbins && wk.start >= 0 && wk.count >= 0 &&
                            (int64_t)wk.start + wk.count <= P.np,
                        kSiteBin, wi))
            continue;
        const double tg = da(P.t0, dm((double)sa.k, P.dt));         // time of the G2P step
        const double tp = da(P.t0, dm((double)sa.p2g_step, P.dt));  // time of the P2G step
        if (tid == 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                Sm.pose[a] = da(P.tool_p0[a], dm(P.tool_v[a], ds(tg, P.tool_t0)));
                Sm.pose[3 + a] = da(P.tool_p0[a], dm(P.tool_v[a], ds(tp, P.tool_t0)));
            }
        }
        const volatile double* pose = Sm.pose;
        const V4<R>* __restrict__ gr = P.grid[rbuf];
        V4<R>* __restrict__ gw = P.grid[rbuf ^ (G2P ? 1 : 0)];

        if (G2P) {
            if (tid == 0) {
                if (wk.inst != last_inst) tmap_acquire(&Pg.tmap[rbuf]);
                fence_async_smem();
                mbar_expect_tx(&Sm.mbar, (uint32_t)(kTileNodes * sizeof(V4<R>)));
                tma_load_4d(Sm.raw, &Pg.tmap[rbuf], &Sm.mbar, 0, g0x, g0y, g0z);
                if (!mbar_wait_bounded(&Sm.mbar, phase, 2000000000ull)) {
                    // give the copy in flight a second bounded chance, then stop
                    mbar_wait_bounded(&Sm.mbar, phase, 2000000000ull);
                    Sm.fail = 1;
                }
            }
            phase ^= 1u;
            last_inst = wk.inst;
            __syncthreads();
            if (Sm.fail) {
                // The tile copy has not landed after 4 s.  If it is only late
                // rather than lost, it can still write Sm.raw after this CTA
                // has returned, into shared memory that the SM's next CTA may
                // own.  The error word is never cleared: every later status or
                // metrics call on the handle returns MPM_TIMEOUT, and the
                // caller is expected to stop using it.
                if (tid == 0) atomicOr(err, ERR_TIMEOUT);
                return;
            }
            for (int nidx = tid; nidx < kTileNodes; nidx += kNT) {
                const int lx = nidx % kTile, ly = (nidx / kTile) % kTile, lz = nidx / (kTile * kTile);
                const NV<R> nv = node_vel_inl(P, Sm.raw[nidx], g0x + lx, g0y + ly, g0z + lz, pose[0], pose[2]);
                const int t = tidx(lx, ly, lz);
                Sm.vel[vidx(lx, ly, lz)] = mk4<R>(nv.x, nv.y, nv.z, R(0));
                if (EXT && P.heat_on) {
                    // node temperatures after the diffusion step, for the nodes the
                    // temperature gather counts (m > 1e-18, inside the domain)
                    const int gx = g0x + lx, gy = g0y + ly, gz = g0z + lz;
                    const bool use = Sm.raw[nidx].x > R(1e-18) && gx < P.nx && gy < P.ny && gz < P.nz;
                    Sm.ttile[0][t] = use ? P.tn[gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz)] : R(0);
                    Sm.ttile[1][t] = use ? R(1) : R(0);
                }
            }
        }
        __syncthreads();

        const R dtdx = (R)(P.dt / P.dx);
        const R idx_ = (R)(1.0 / P.dx);
        const bool chip_now = G2P && P.chip_every > 0 && ((P.step0 + sa.k) % P.chip_every) == 0;
        for (int base = 0; base < wk.count; base += kChunk) {
#pragma unroll 1
            for (int sidx = 0; sidx < StepCfg<R, CH>::kPerThread; ++sidx) {
                const int slot = tid + sidx * kNT;
                const int pl = base + slot;
                // the loads the G2P needs are issued here, before any branch on the
                // particle's state: one memory round trip (F_p waits for the
                // constitutive update).  Slots past the bin's end read the bin's
                // first particle (bins are never empty) and are discarded.
#ifdef MPMB_CHECKED
                bool valid = pl < wk.count;
                int64_t pi = P.pbase + wk.start + (valid ? pl : 0);
                if (!MPMB_CHECK(pi >= P.pbase && pi < P.pbase + P.pcap, kSiteParticle, pi)) {
                    valid = false;
                    pi = P.pbase;
                }
#else
                const bool valid = pl < wk.count;
                const int64_t pi = P.pbase + wk.start + (valid ? pl : 0);
#endif
                const uint8_t st_ld = ps.status[pi];
                const V4<R> a0 = ldcs4(&ps.A[0][pi]), a1 = ldcs4(&ps.A[1][pi]), a2 = ldcs4(&ps.A[2][pi]),
                            a3 = ldcs4(&ps.A[3][pi]);
                const V4<R> xl = (G2P && ps.X) ? ldcs4(&ps.X[pi]) : mk4<R>(0, 0, 0, 0);
                const V4<R> b0_ld = G2P ? mk4<R>(0, 0, 0, 0) : ldcs4(&ps.B[0][pi]);
                uint8_t st = valid ? st_ld : (uint8_t)ST_INACTIVE;
                if (st != ST_INACTIVE) {
                    const uint8_t st_in = st;
                    const bool fixed = (st == ST_FIXED);
                    R xi[3] = {a0.x, a0.y, a0.z};
                    R eps = a0.w;
                    R H[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
                    R Hp8 = a3.y, dT = a3.z, Dm = a3.w;
                    // low parts of the position (FP32 state); the move is an exact two-sum
                    R lo[3] = {R(0), R(0), R(0)};
                    const bool has_lo = G2P && !fixed && ps.X != nullptr;
                    if (has_lo) { lo[0] = xl.x; lo[1] = xl.y; lo[2] = xl.z; }
                    R v[3] = {0, 0, 0}, Cm[9], edot = R(0);
                    bool have_C = false, dirtyA = false, wrote_C = false;

                    if (G2P) {
                        if (!fixed) {
                            bool far = false;
                            if (P.lod && st == ST_ACTIVE) {
                                const double wx = P.ox + ((double)g0x + ((double)xi[0] + (double)lo[0])) * P.dx - pose[0];
                                const double wy = P.oy + ((double)g0y + ((double)xi[1] + (double)lo[1])) * P.dx - pose[1];
                                const double wz =
                                    P.oz + ((double)g0z + ((double)xi[2] + (double)lo[2])) * P.dx - (pose[2] + P.tool_tip_dz);
                                far = sqrt(wx * wx + wy * wy + wz * wz) > P.lod_r2;
                            }
                            R w[3][3], dw[3][3];
                            int b[3];
#pragma unroll
                            for (int a = 0; a < 3; ++a) b[a] = bspline(xi[a], w[a], dw[a]);
                            R M[3][3], L[3][3];
                            TSum<R> tsum{R(0), R(0)};
                            if (b[0] >= 0 && b[0] < kBin && b[1] >= 0 && b[1] < kBin && b[2] >= 0 && b[2] < kBin) {
                                gather_tile<R>(Sm.vel, vidx(b[0], b[1], b[2]), w, dw, v, M, L);
                                if (EXT && P.heat_on) {
                                    const int tb = tidx(b[0], b[1], b[2]);
#pragma unroll
                                    for (int k = 0; k < 3; ++k)
#pragma unroll
                                        for (int j = 0; j < 3; ++j) {
                                            const R wjk = w[1][j] * w[2][k];
#pragma unroll
                                            for (int i = 0; i < 3; ++i) {
                                                const int q = tb + i + kSY * j + kSZ * k;
                                                const R ww = w[0][i] * wjk;
                                                tsum.ts = fma(ww, Sm.ttile[0][q], tsum.ts);
                                                tsum.ws = fma(ww, Sm.ttile[1][q], tsum.ws);
                                            }
                                        }
                                }
                            } else {
                                const GatherOut<R> go = gather_global<R>(P, gr, g0x, g0y, g0z, xi[0], xi[1], xi[2],
                                                                         pose[0], pose[2]);
#pragma unroll
                                for (int c = 0; c < 3; ++c) {
                                    v[c] = go.v[c];
#pragma unroll
                                    for (int q = 0; q < 3; ++q) { M[c][q] = go.M[c][q]; L[c][q] = go.L[c][q]; }
                                }
                                ++c_esc;
                                if (EXT && P.heat_on) tsum = gather_T_global<R>(P, gr, g0x, g0y, g0z, xi[0], xi[1], xi[2]);
                            }
                            if (EXT && P.heat_on && tsum.ws > R(1e-8)) {
                                // heat conduction: the temperature gather of mpmG2PKernel
                                // (src/MPMWorkpieceSolver.cu:282-306), clamped to [Tamb, Tm]
                                dT = fmin(fmax(tsum.ts / tsum.ws, P.Tamb), P.Tamb + P.dTmax) - P.Tamb;
                            }
                            const R d[3] = {xi[0] - R(b[0]), xi[1] - R(b[1]), xi[2] - R(b[2])};
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                if (has_lo) {
                                    // (xi, lo) <- xi + (lo + v dt/dx), Knuth's two-sum: exact
                                    const R inc = fma(v[a], dtdx, lo[a]);
                                    const R s = xi[a] + inc;
                                    const R bv = s - xi[a];
                                    lo[a] = (xi[a] - (s - bv)) + (inc - bv);
                                    xi[a] = s;
                                } else {
                                    xi[a] = fma(v[a], dtdx, xi[a]);
                                }
                            }
                            dirtyA = true;
                            if (st == ST_CHIP) {
                                edot = R(0);
                            } else {
                                // C = factor/dx^2 * B with B = dx (M - d v), then decay (0 in the far zone)
                                const R cf = far ? R(0) : P.apic * idx_ * P.decay;
#pragma unroll
                                for (int a = 0; a < 3; ++a)
#pragma unroll
                                    for (int c = 0; c < 3; ++c) Cm[a * 3 + c] = cf * (M[a][c] - d[c] * v[a]);
                                have_C = true;
                                // F <- (I + L dt) F  as  H <- H + Ldt (I + H)
                                R Ld[9];
#pragma unroll
                                for (int a = 0; a < 3; ++a)
#pragma unroll
                                    for (int c = 0; c < 3; ++c) Ld[a * 3 + c] = L[a][c] * dtdx;
                                R Hn[9];
#pragma unroll
                                for (int a = 0; a < 3; ++a)
#pragma unroll
                                    for (int c = 0; c < 3; ++c)
                                        Hn[a * 3 + c] = H[a * 3 + c] + Ld[a * 3 + c] + Ld[a * 3] * H[c] +
                                                        Ld[a * 3 + 1] * H[3 + c] + Ld[a * 3 + 2] * H[6 + c];
#pragma unroll
                                for (int q = 0; q < 9; ++q) H[q] = Hn[q];
                                const R l00 = L[0][0] * idx_, l11 = L[1][1] * idx_, l22 = L[2][2] * idx_;
                                const R s01 = (L[0][1] + L[1][0]) * idx_, s02 = (L[0][2] + L[2][0]) * idx_,
                                        s12 = (L[1][2] + L[2][1]) * idx_;
                                edot = sqrt(R(2.0 / 3.0) * (l00 * l00 + l11 * l11 + l22 * l22 + R(0.5) * s01 * s01 +
                                                              R(0.5) * s02 * s02 + R(0.5) * s12 * s12));
                            }
                        }
                        // adiabatic shear band heating after the move and before chip separation
                        // (AdiabaticShearModel::update after g2pKernel, src/MPMSolver.cu:1130-1132;
                        // guards of src/AdiabaticShearModel.cu:114-136); the stress is the one the
                        // constitutive update of this step stored
                        if (EXT && P.asb_on) {
                            if (st == ST_CHIP) {
                                if (ps.asb[pi] != 0) ps.asb[pi] = 0;   // :114-117
                            } else if (st == ST_ACTIVE && dT > P.asb_rise) {   // :119-123
                                if (edot < P.asb_min_rate) {                    // :131-136: decay
                                    const uint8_t c = ps.asb[pi];
                                    if (c != 0) ps.asb[pi] = (uint8_t)(c - 1);
                                } else {
                                    dT = asb_update<R>(P, ps, pi, edot, dT, ctr);
                                    dirtyA = true;
                                }
                            }
                        }
                        // chip separation and fracture after the move (step counter parity)
                        if (chip_now) {
                            if (st == ST_ACTIVE) {
                                const double tipz = ds(da(pose[2], P.tool_tip_dz), dm(P.dx, 1.5));
                                const double zw = P.oz + ((double)g0z + ((double)xi[2] + (double)lo[2])) * P.dx;
                                if (zw < tipz && Dm > R(1e-6)) {
                                    st = ST_CHIP;
                                    const V4<R> s0 = ldcs4(&ps.S[0][pi]);
                                    const R rs = sqrt(s0.x * s0.x + s0.y * s0.y + s0.z * s0.z);
                                    ps.sres[pi] = fmax(ps.sres[pi], rs);
                                    stcs4(&ps.S[0][pi], mk4<R>(0, 0, 0, 0));
                                    stcs4(&ps.S[1][pi], mk4<R>(0, 0, 0, 0));
                                    Dm = fmax(Dm, P.Dth);
                                    dirtyA = true;
                                }
                            } else if (st == ST_CHIP && Dm >= P.Dth * R(1.5)) {
                                const uint32_t seed = (uint32_t)ps.id[pi] * 2654435761u;
                                const R rx = (R)((double)((seed >> 16) & 0xFF) / 255.0 - 0.5);
                                const R ry = (R)((double)((seed >> 8) & 0xFF) / 255.0 - 0.5);
                                const R rz = (R)((double)(seed & 0xFF) / 255.0 - 0.5);
                                const R sp = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                                const R pm = sp * R(0.3) + R(0.5);
                                v[0] += rx * pm; v[1] += ry * pm; v[2] += rz * pm;
                                Dm = P.Dth * R(0.5);
                                dirtyA = true;
                            }
                        }
                        // particle-side tool contact after the move, at the tool pose of the
                        // step's end (every contact_every-th step)
                        if (P.contact_every > 0 && !fixed && ((P.step0 + sa.k + 1) % P.contact_every) == 0) {
                            const double te = da(P.t0, dm((double)(sa.k + 1), P.dt));
                            const double pe0 = da(P.tool_p0[0], dm(P.tool_v[0], ds(te, P.tool_t0)));
                            const double pe2 = da(P.tool_p0[2], dm(P.tool_v[2], ds(te, P.tool_t0)));
                            const double wx = P.ox + ((double)g0x + ((double)xi[0] + (double)lo[0])) * P.dx;
                            const double wz = P.oz + ((double)g0z + ((double)xi[2] + (double)lo[2])) * P.dx;
                            ContactOut co;
                            if (EXT && P.sdf_on) {
                                // voxel tool SDF (the extension variant)
                                const double pe1 = da(P.tool_p0[1], dm(P.tool_v[1], ds(te, P.tool_t0)));
                                const double wy = P.oy + ((double)g0y + ((double)xi[1] + (double)lo[1])) * P.dx;
                                co = particle_contact_sdf<R>(P, wx, wy, wz, pe0, pe1, pe2, v[0], v[1], v[2], dT);
                            } else {
                                co = particle_contact<R>(P, wx, wz, pe0, pe2, v[0], v[1], v[2], dT);
                            }
                            if (co.hit) {
#pragma unroll
                                for (int a = 0; a < 3; ++a) {
                                    if (has_lo) {
                                        const R inc = (R)co.dxi[a] + lo[a];
                                        const R s = xi[a] + inc;
                                        const R bv = s - xi[a];
                                        lo[a] = (xi[a] - (s - bv)) + (inc - bv);
                                        xi[a] = s;
                                    } else {
                                        xi[a] = (R)((double)xi[a] + co.dxi[a]);
                                    }
                                }
                                dirtyA = true;
                                ++c_contact;
                                f_work += co.work;
                                f_force += co.force;
                            }
                        }
                    } else {
                        // P2G-only launch: velocity and strain rate come from memory
                        v[0] = b0_ld.x; v[1] = b0_ld.y; v[2] = b0_ld.z; edot = b0_ld.w;
                    }

                    bool yielded = false;
                    if (P2G) {
                        // kill zone on the cell index, :130-139.  Written on the floored
                        // bin-local position so that a NaN position fails every bound and is
                        // killed, as in the reference, whose integer cell index of a NaN
                        // position (0 from the GPU's conversion) is below 1; a non-finite
                        // position also marks the instance's error word (byte 0)
                        const R f0 = floor(xi[0]), f1 = floor(xi[1]), f2 = floor(xi[2]);
                        if (!(f0 >= R(1 - g0x) && f0 < R(P.nx - 2 - g0x) && f1 >= R(1 - g0y) &&
                              f1 < R(P.ny - 2 - g0y) && f2 >= R(1 - g0z) && f2 < R(P.nz - 2 - g0z))) {
                            if (!isfinite(f0 + f1 + f2)) reinterpret_cast<unsigned char*>(P.ierr)[0] = 1;
                            st = ST_INACTIVE;
                            if (G2P) {
                                // no later G2P writes this particle: store this step's v, strain rate and C
                                stcs4(&ps.B[0][pi], mk4<R>(v[0], v[1], v[2], edot));
                                if (have_C) {
                                    stcs4(&ps.B[1][pi], mk4<R>(Cm[0], Cm[1], Cm[2], Cm[3]));
                                    stcs4(&ps.B[2][pi], mk4<R>(Cm[4], Cm[5], Cm[6], Cm[7]));
                                    stcs4(&ps.B[3][pi], mk4<R>(Cm[8], R(0), R(0), R(0)));
                                }
                            }
                        } else {
                            // within one cell of the kill zone the stress is kept in memory, since a
                            // kill in the next launch leaves the last computed stress as the state
                            const int cx = g0x + (int)f0, cy = g0y + (int)f1, cz = g0z + (int)f2;
                            const bool near_kill = cx < 3 || cx >= P.nx - 4 || cy < 3 || cy >= P.ny - 4 ||
                                                   cz < 3 || cz >= P.nz - 4;
                            bool far = false;
                            if (P.lod && st == ST_ACTIVE) {
                                const double wx = P.ox + ((double)g0x + ((double)xi[0] + (double)lo[0])) * P.dx - pose[3];
                                const double wy = P.oy + ((double)g0y + ((double)xi[1] + (double)lo[1])) * P.dx - pose[4];
                                const double wz =
                                    P.oz + ((double)g0z + ((double)xi[2] + (double)lo[2])) * P.dx - (pose[5] + P.tool_tip_dz);
                                far = sqrt(wx * wx + wy * wy + wz * wz) > P.lod_r2;
                            }
                            bool skip = far || fixed || st == ST_CHIP;
                            R Jv = R(1);
                            R sig[6] = {0, 0, 0, 0, 0, 0};
                            R sl[3] = {0, 0, 0};
                            if (!skip && st == ST_ACTIVE) {
                                // F_p - I: loaded here, where the constitutive update needs
                                // it, rather than held in registers through the gather
                                const V4<R> a4 = ldcs4(&ps.A[4][pi]), a5 = ldcs4(&ps.A[5][pi]);
                                R Hp[9] = {a4.x, a4.y, a4.z, a4.w, a5.x, a5.y, a5.z, a5.w, Hp8};
                                R bsv[6];
                                R* bsp = nullptr;
                                if (P.Hkin > R(0)) {
                                    const V4<R> k0 = ps.K[0][pi], k1 = ps.K[1][pi];
                                    bsv[0] = k0.x; bsv[1] = k0.y; bsv[2] = k0.z; bsv[3] = k0.w;
                                    bsv[4] = k1.x; bsv[5] = k1.y;
                                    bsp = bsv;
                                }
                                JCOut jo = jc_update<R>(P, H, Hp, eps, dT, Dm, edot, sig, sl, Jv, &ps.sres[pi], bsp,
                                                        errf, wk.inst + 1);
                                if (jo.yielded) {
                                    yielded = true;
                                    dirtyA = true;
                                    Hp8 = Hp[8];
                                    stcs4(&ps.A[4][pi], mk4<R>(Hp[0], Hp[1], Hp[2], Hp[3]));
                                    stcs4(&ps.A[5][pi], mk4<R>(Hp[4], Hp[5], Hp[6], Hp[7]));
                                    if (bsp) {
                                        ps.K[0][pi] = mk4<R>(bsv[0], bsv[1], bsv[2], bsv[3]);
                                        ps.K[1][pi] = mk4<R>(bsv[4], bsv[5], R(0), R(0));
                                    }
                                }
                                if (jo.to_chip) { st = ST_CHIP; skip = true; }
                                // with the shear model on, the next step's heating reads the stress
                                // of every particle that passes its temperature guard
                                if (sa.sigma_all || Dm > R(1e-6) || P.lod || near_kill ||
                                    (P.asb_on && dT > P.asb_rise)) {
                                    stcs4(&ps.S[0][pi], mk4<R>(sig[0], sig[1], sig[2], sig[3]));
                                    stcs4(&ps.S[1][pi], mk4<R>(sig[4], sig[5], R(0), R(0)));
                                }
                            }
                            // C of the particle: from this launch's gather, or the frozen value of
                            // a CHIP particle (g2pKernel keeps it)
                            if (!have_C && !fixed) {
                                const V4<R> c1 = ldcs4(&ps.B[1][pi]), c2 = ldcs4(&ps.B[2][pi]),
                                            c3 = ldcs4(&ps.B[3][pi]);
                                Cm[0] = c1.x; Cm[1] = c1.y; Cm[2] = c1.z; Cm[3] = c1.w;
                                Cm[4] = c2.x; Cm[5] = c2.y; Cm[6] = c2.z; Cm[7] = c2.w; Cm[8] = c3.x;
                            }
                            if (!fixed && have_C && st == ST_CHIP && st_in != ST_CHIP) {
                                // turned CHIP this launch: freeze C as the reference does
                                stcs4(&ps.B[1][pi], mk4<R>(Cm[0], Cm[1], Cm[2], Cm[3]));
                                stcs4(&ps.B[2][pi], mk4<R>(Cm[4], Cm[5], Cm[6], Cm[7]));
                                stcs4(&ps.B[3][pi], mk4<R>(Cm[8], R(0), R(0), R(0)));
                                wrote_C = true;
                            }
                            // scatter payload: Q = m (v - dx C d) + f_ext dt, R = m dx C,
                            // S = -dt V J sigma / dx (sigma with the reference's trial lower triangle)
                            const int bb[3] = {(int)floor(xi[0] - R(0.5)), (int)floor(xi[1] - R(0.5)),
                                               (int)floor(xi[2] - R(0.5))};
                            const R m = P.pmass;
                            R Q[3] = {0, 0, 0}, Rm[9], S[9];
#pragma unroll
                            for (int q = 0; q < 9; ++q) { Rm[q] = R(0); S[q] = R(0); }
                            R ef[3] = {0, 0, 0};
                            if (sa.use_ext && P.pext) {
                                // an imported per-particle force (MPMParticle::ext_f) acts on every
                                // particle the step scatters, FIXED included: p2gKernel adds
                                // w * ext_f to the node force (src/MPMSolver.cu:410-417)
                                const V4<R> e = P.pext[P.pbase + ps.orig[pi]];
                                const R fdt = (R)P.dt;
                                ef[0] = e.x * fdt; ef[1] = e.y * fdt; ef[2] = e.z * fdt;
                                if (fixed) { Q[0] = ef[0]; Q[1] = ef[1]; Q[2] = ef[2]; }
                            }
                            if (!fixed) {
                                const R d[3] = {xi[0] - R(bb[0]), xi[1] - R(bb[1]), xi[2] - R(bb[2])};
                                const R mdx = m * (R)P.dx;
                                if (sa.use_ext && P.ext_r > 0.0 && (st == ST_ACTIVE || st == ST_CHIP)) {
                                    const double ex = P.ox + ((double)g0x + ((double)xi[0] + (double)lo[0])) * P.dx - P.ext_c[0];
                                    const double ey = P.oy + ((double)g0y + ((double)xi[1] + (double)lo[1])) * P.dx - P.ext_c[1];
                                    const double ez = P.oz + ((double)g0z + ((double)xi[2] + (double)lo[2])) * P.dx - P.ext_c[2];
                                    const double dist = sqrt(ex * ex + ey * ey + ez * ez);
                                    if (dist < P.ext_r) {
                                        const double fw = (1.0 - dist / P.ext_r) * P.dt;
                                        ef[0] += (R)(P.ext_f[0] * fw); ef[1] += (R)(P.ext_f[1] * fw);
                                        ef[2] += (R)(P.ext_f[2] * fw);
                                    }
                                }
#pragma unroll
                                for (int a = 0; a < 3; ++a) {
                                    Q[a] = m * v[a] -
                                           mdx * (Cm[a * 3] * d[0] + Cm[a * 3 + 1] * d[1] + Cm[a * 3 + 2] * d[2]) + ef[a];
#pragma unroll
                                    for (int c = 0; c < 3; ++c) Rm[a * 3 + c] = mdx * Cm[a * 3 + c];
                                }
                                const R sf = skip ? R(0) : -(R)P.dt * P.pvol * Jv * idx_;
                                S[0] = sf * sig[0]; S[4] = sf * sig[1]; S[8] = sf * sig[2];
                                S[1] = sf * sig[3]; S[3] = sf * sl[0];
                                S[2] = sf * sig[4]; S[6] = sf * sl[1];
                                S[5] = sf * sig[5]; S[7] = sf * sl[2];
                            }
                            if (bb[0] >= 0 && bb[0] < kBin && bb[1] >= 0 && bb[1] < kBin && bb[2] >= 0 &&
                                bb[2] < kBin) {
                                const int scell = bb[0] + kBin * (bb[1] + kBin * bb[2]);
                                if (scell == (slot & (kCellsPerBin - 1))) {
                                    atomicOr(&Sm.hmask[par][scell], 1u << (slot >> 6));
                                } else {
                                    atomicOr(&Sm.fmask[par][slot >> 5][scell], 1u << (slot & 31));
                                    atomicOr(&Sm.hmask[par][scell], 0x80000000u);
                                }
                                if (EXT)   // absolute T (heat conduction)
                                    Sm.pay[EXT ? 6 : 0][slot] = mk4<R>(P.Tamb + dT, R(0), R(0), R(0));
                                Sm.pay[0][slot] = mk4<R>(xi[0], xi[1], xi[2], Q[0]);
                                Sm.pay[1][slot] = mk4<R>(Rm[0], Rm[1], Rm[2], S[0]);
                                Sm.pay[2][slot] = mk4<R>(S[1], S[2], Q[1], Q[2]);
                                Sm.pay[3][slot] = mk4<R>(Rm[3], Rm[4], Rm[5], S[3]);
                                Sm.pay[4][slot] = mk4<R>(S[4], S[5], Rm[6], Rm[7]);
                                Sm.pay[5][slot] = mk4<R>(Rm[8], S[6], S[7], S[8]);
                            } else {
                                ScatterIn<R> si;
#pragma unroll
                                for (int a = 0; a < 3; ++a) { si.xi[a] = xi[a]; si.Q[a] = Q[a]; }
#pragma unroll
                                for (int q = 0; q < 9; ++q) { si.Rm[q] = Rm[q]; si.S[q] = S[q]; }
                                si.g0[0] = g0x; si.g0[1] = g0y; si.g0[2] = g0z;
                                scatter_global<R>(P, gw, si, m);
                                if (EXT && P.heat_on)
                                    scatter_T_global<R>(P, P.tm[rbuf ^ (G2P ? 1 : 0)], g0x, g0y, g0z, xi[0], xi[1],
                                                        xi[2], m * (P.Tamb + dT));
                                ++c_esc;
                            }
                        }
                    }

                    // write back
                    if (dirtyA) {
                        if (has_lo) stcs4(&ps.X[pi], mk4<R>(lo[0], lo[1], lo[2], R(0)));
                        stcs4(&ps.A[0][pi], mk4<R>(xi[0], xi[1], xi[2], eps));
                        stcs4(&ps.A[1][pi], mk4<R>(H[0], H[1], H[2], H[3]));
                        stcs4(&ps.A[2][pi], mk4<R>(H[4], H[5], H[6], H[7]));
                        stcs4(&ps.A[3][pi], mk4<R>(H[8], Hp8, dT, Dm));
                    }
                    if (st != st_in) ps.status[pi] = st;
                    if (G2P && sa.write_out && st != ST_INACTIVE) {
                        if (fixed) {
                            const V4<R> b0 = ldcs4(&ps.B[0][pi]);
                            stcs4(&ps.B[0][pi], mk4<R>(R(0), R(0), R(0), b0.w));
                        } else {
                            stcs4(&ps.B[0][pi], mk4<R>(v[0], v[1], v[2], edot));
                            if (have_C && !wrote_C && st_in != ST_CHIP) {
                                stcs4(&ps.B[1][pi], mk4<R>(Cm[0], Cm[1], Cm[2], Cm[3]));
                                stcs4(&ps.B[2][pi], mk4<R>(Cm[4], Cm[5], Cm[6], Cm[7]));
                                stcs4(&ps.B[3][pi], mk4<R>(Cm[8], R(0), R(0), R(0)));
                            }
                        }
                    }
                    c_yield += yielded ? 1 : 0;
                }
            }
            if (P2G) {
                __syncthreads();
                cell_accumulate<R, EXT, CH>(Sm, tid & (kCellsPerBin - 1), tid >> 6, (tid >> 5) & 1, P.pmass, par,
                                        P.heat_on != 0);
                par ^= 1;
                __syncthreads();
            }
        }

        if (P2G && sa.part) {
            // deterministic mode: the bin's node tile is stored for k_node_sum
            // (every node and channel, zeros included), clearing it for the next bin
            R* __restrict__ dst = static_cast<R*>(sa.part) + (int64_t)wi * (kPartCh * kTileNodes);
            for (int nidx = tid; nidx < kTileNodes; nidx += kNT) {
                const int X = nidx % kTile, Y = (nidx / kTile) % kTile, Z = nidx / (kTile * kTile);
                const int t = tidx(X, Y, Z);
#pragma unroll
                for (int q = 0; q < (EXT ? 5 : 4); ++q) {
                    dst[q * kTileNodes + nidx] = Sm.nacc[0][q][t] + Sm.nacc[1][q][t];
                    Sm.nacc[0][q][t] = R(0);
                    Sm.nacc[1][q][t] = R(0);
                }
            }
        } else if (P2G) {
            // flush the bin's node tile to the grid, clearing it for the next bin
            for (int nidx = tid; nidx < kTileNodes; nidx += kNT) {
                const int X = nidx % kTile, Y = (nidx / kTile) % kTile, Z = nidx / (kTile * kTile);
                const int t = tidx(X, Y, Z);
                R c[EXT ? 5 : 4];
#pragma unroll
                for (int q = 0; q < (EXT ? 5 : 4); ++q) {
                    c[q] = Sm.nacc[0][q][t] + Sm.nacc[1][q][t];
                    Sm.nacc[0][q][t] = R(0);
                    Sm.nacc[1][q][t] = R(0);
                }
                const R m = c[0], px = c[1], py = c[2], pz = c[3];
                const R mT = EXT ? c[EXT ? 4 : 0] : R(0);
                if (m == R(0)) continue;
                const int gx = g0x + X, gy = g0y + Y, gz = g0z + Z;
                if (gx >= P.nx || gy >= P.ny || gz >= P.nz) continue;
                const int64_t gi = gx + (int64_t)P.nx * (gy + (int64_t)P.ny * gz);
                if (!MPMB_CHECK(gi >= 0 && gi < P.nn, kSiteFlush, gi)) continue;
                vec_atomic_add<R>(&gw[gi], m, px, py, pz);
                if (EXT && P.heat_on) atomicAdd(&P.tm[rbuf ^ (G2P ? 1 : 0)][gi], mT);
            }
        }
        __syncthreads();
    }
    // counters: warp-reduce, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c_esc += __shfl_down_sync(0xffffffffu, c_esc, o);
        c_yield += __shfl_down_sync(0xffffffffu, c_yield, o);
        c_contact += __shfl_down_sync(0xffffffffu, c_contact, o);
        f_work += __shfl_down_sync(0xffffffffu, f_work, o);
        f_force += __shfl_down_sync(0xffffffffu, f_force, o);
    }
    if (lane == 0) {
        if (c_esc) atomicAdd(&ctr[0], (unsigned long long)c_esc);
        if (c_yield) atomicAdd(&ctr[1], (unsigned long long)c_yield);
        if (c_contact) {
            // ctr[2] counts contacts; two FP64 sums follow the four counters
            atomicAdd(&ctr[2], (unsigned long long)c_contact);
            atomicAdd(reinterpret_cast<double*>(ctr + 4), f_work);
            atomicAdd(reinterpret_cast<double*>(ctr + 4) + 1, f_force);
        }
    }
    // Newton failures to the failing instance's error word (byte 1), or to the
    // handle's word when this thread saw more than one instance fail
    if (errf > 0) reinterpret_cast<unsigned char*>(insts[errf - 1].ierr)[1] = 1;
    else if (errf < 0) atomicOr(err, ERR_NEWTON);
}

// Sets the variant's shared-memory size once and returns how many of its
// CTAs fit on one SM.  The work loop hands every CTA of the grid the same
// share of the work items, so a grid with more CTAs than fit would run its
// last CTAs as a second wave: launches clamp the grid to this.
template <typename R, bool G2P, bool P2G, bool EXT, int CH> static int set_smem_attr() {
    static bool attr = false;
    static int fit = 0;
    if (!attr) {
        cudaFuncSetAttribute(k_step<R, G2P, P2G, EXT, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)step_smem_bytes<R, EXT, CH>());
        attr = true;
    }
    if (!fit) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step<R, G2P, P2G, EXT, CH>, kNT,
                                                          step_smem_bytes<R, EXT, CH>()) == cudaSuccess &&
            n >= 1)
            fit = n;
        else
            return 8;   // not known (the query failed): no clamp this time, asked again next launch
    }
    return fit;
}

// Deterministic mode, the grid of one P2G: one thread per node of a bin's
// 4x4x4 core (a CTA of 128 threads takes two bins of the batch's bin table)
// adds, in a fixed order, the node's values in the stored tiles of the bins
// whose 6x6x6 tile holds it (per axis the bin itself and, for the first two
// layers of its core, the bin before; z, then y, then x, lower bin first),
// then the node's escaped fixed-point sums (cleared after reading), and
// writes the node -- zero where nothing reached it, so no clear of the grid
// precedes the P2G.  No float atomics anywhere: with the re-bin's order fixed,
// the grid is the same bit for bit on every run and launch shape.
template <typename R>
__global__ void __launch_bounds__(128) k_node_sum(const Inst<R>* __restrict__ insts, const int32_t* __restrict__ bin_inst,
                                                  const int32_t* __restrict__ bin_local,
                                                  const int32_t* __restrict__ flag,
                                                  const int32_t* __restrict__ flag_scan, const R* __restrict__ part,
                                                  int64_t part_items, int b, int nbins_total) {
    const int gb = blockIdx.x * 2 + (threadIdx.x >> 6);
    const int c = threadIdx.x & (kCellsPerBin - 1);
    const bool have = gb < nbins_total;
    const Inst<R>* P = have ? &insts[bin_inst[gb]] : insts;
    const int lb = have ? bin_local[gb] : 0;
    bool esc = false;
    if (have) {
        const int bx = lb % P->nbx, by = (lb / P->nbx) % P->nby, bz = lb / (P->nbx * P->nby);
        const int gx = bx * kBin + (c & 3), gy = by * kBin + ((c >> 2) & 3), gz = bz * kBin + (c >> 4);
        R acc[kPartCh] = {R(0), R(0), R(0), R(0), R(0)};
        const int nch = P->heat_on ? 5 : 4;
        for (int z = bz - 1; z <= bz; ++z) {
            const int Z = gz - z * kBin;
            if (z < 0 || Z >= kTile) continue;
            for (int y = by - 1; y <= by; ++y) {
                const int Y = gy - y * kBin;
                if (y < 0 || Y >= kTile) continue;
                for (int x = bx - 1; x <= bx; ++x) {
                    const int X = gx - x * kBin;
                    if (x < 0 || X >= kTile) continue;
                    const int g = P->bin0 + x + P->nbx * (y + P->nby * z);
                    if (!flag[g]) continue;
                    const int64_t wi = flag_scan[g];
                    if (!MPMB_CHECK(wi >= 0 && wi < part_items, kSitePart, wi)) continue;
                    const R* __restrict__ t = part + wi * (kPartCh * kTileNodes) + X + kTile * (Y + kTile * Z);
                    for (int q = 0; q < nch; ++q) acc[q] += t[q * kTileNodes];
                }
            }
        }
        if (gx < P->nx && gy < P->ny && gz < P->nz) {
            const int64_t li = gx + (int64_t)P->nx * (gy + (int64_t)P->ny * gz);
            esc = P->esc != nullptr && P->esc_flag[lb] != 0;
            if (esc) {
                for (int q = 0; q < nch; ++q) {
                    unsigned long long* e = &P->esc[q * P->esc_stride + li];
                    const long long v = (long long)*e;
                    if (v != 0) {
                        acc[q] += (R)((double)v / P->esc_scale);
                        *e = 0ull;
                    }
                }
            }
            if (MPMB_CHECK(li >= 0 && li < P->nn, kSiteNodeSum, li)) {
                P->grid[b][li] = mk4<R>(acc[0], acc[1], acc[2], acc[3]);
                if (P->heat_on) P->tm[b][li] = acc[4];
            }
        }
    }
    // every thread of the bin has read its flag before it is cleared
    __syncthreads();
    if (have && c == 0 && P->esc != nullptr && P->esc_flag[lb] != 0) P->esc_flag[lb] = 0;
    (void)esc;
}

template <typename R>
void launch_node_sum(const Inst<R>* insts, const int32_t* bin_inst, const int32_t* bin_local, const int32_t* flag,
                     const int32_t* flag_scan, const R* part, int64_t part_items, int b, int nbins_total,
                     cudaStream_t st) {
    if (nbins_total <= 0) return;
    Range nvtx_range("mpm.node_sum");
    k_node_sum<R><<<(nbins_total + 1) / 2, 128, 0, st>>>(insts, bin_inst, bin_local, flag, flag_scan, part,
                                                         part_items, b, nbins_total);
    ++launch_counter();
}

// One pass size: the G2P / P2G / extension variant of the launch.  (FP64
// instantiates only the default pass size, whose kChunk is 128 like all of
// its pass sizes.)
template <typename R, int CH>
static void launch_variant(const Inst<R>* insts, const Work* work, const int* n_work, const PState<R>& ps,
                           const StepArgs& a, int rbuf, bool g2p, bool p2g, int sms, int cps, int max_work, int* err,
                           unsigned long long* counters, cudaStream_t st) {
    // persistent CTAs: cps per SM, at most as many as fit, at most one per work item
    auto grid_of = [&](int fit) { return std::max(1, std::min(sms * std::min(cps, fit), max_work)); };
    if constexpr (sizeof(R) == 8 && CH != kDefaultChunk) {
        launch_variant<R, kDefaultChunk>(insts, work, n_work, ps, a, rbuf, g2p, p2g, sms, cps, max_work, err, counters,
                                         st);
    } else if (a.ext) {
        const size_t smem = step_smem_bytes<R, true, kDefaultChunk>();
        if (g2p && p2g) {
            const int grid = grid_of(set_smem_attr<R, true, true, true, kDefaultChunk>());
            k_step<R, true, true, true, kDefaultChunk><<<grid, kNT, smem, st>>>(insts, work, n_work, ps, a, rbuf, err,
                                                                               counters);
        } else if (g2p) {
            const int grid = grid_of(set_smem_attr<R, true, false, true, kDefaultChunk>());
            k_step<R, true, false, true, kDefaultChunk><<<grid, kNT, smem, st>>>(insts, work, n_work, ps, a, rbuf, err,
                                                                                counters);
        } else {
            const int grid = grid_of(set_smem_attr<R, false, true, true, kDefaultChunk>());
            k_step<R, false, true, true, kDefaultChunk><<<grid, kNT, smem, st>>>(insts, work, n_work, ps, a, rbuf, err,
                                                                                counters);
        }
    } else {
        const size_t smem = step_smem_bytes<R, false, CH>();
        if (g2p && p2g) {
            const int grid = grid_of(set_smem_attr<R, true, true, false, CH>());
            k_step<R, true, true, false, CH><<<grid, kNT, smem, st>>>(insts, work, n_work, ps, a, rbuf, err, counters);
        } else if (g2p) {
            const int grid = grid_of(set_smem_attr<R, true, false, false, CH>());
            k_step<R, true, false, false, CH><<<grid, kNT, smem, st>>>(insts, work, n_work, ps, a, rbuf, err, counters);
        } else {
            const int grid = grid_of(set_smem_attr<R, false, true, false, CH>());
            k_step<R, false, true, false, CH><<<grid, kNT, smem, st>>>(insts, work, n_work, ps, a, rbuf, err, counters);
        }
    }
}

template <typename R>
void launch_step(const Inst<R>* insts, const Work* work, const int* n_work, int max_work, const PState<R>& ps,
                 const StepArgs& a, int rbuf, bool g2p, bool p2g, int threads, int ctas_per_sm, int* err,
                 unsigned long long* counters, cudaStream_t st) {
    (void)threads;
    Range nvtx_range(g2p && p2g ? "mpm.launch.g2p_p2g" : (g2p ? "mpm.launch.g2p" : "mpm.launch.p2g"));
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    if (max_work <= 0) return;
    const int cps = ctas_per_sm > 0 ? ctas_per_sm : 4;
    // FP64 passes are 128 particles whatever the pass size; the extension
    // variant runs the default pass size
    const int ch = (sizeof(R) == 8 || a.ext) ? kDefaultChunk : a.chunk;
    if (ch == 1)
        launch_variant<R, 1>(insts, work, n_work, ps, a, rbuf, g2p, p2g, sms, cps, max_work, err, counters, st);
    else if (ch == 4)
        launch_variant<R, 4>(insts, work, n_work, ps, a, rbuf, g2p, p2g, sms, cps, max_work, err, counters, st);
    else
        launch_variant<R, kDefaultChunk>(insts, work, n_work, ps, a, rbuf, g2p, p2g, sms, cps, max_work, err,
                                         counters, st);
    ++launch_counter();
}

template void launch_node_sum<float>(const Inst<float>*, const int32_t*, const int32_t*, const int32_t*,
                                    const int32_t*, const float*, int64_t, int, int, cudaStream_t);
template void launch_node_sum<double>(const Inst<double>*, const int32_t*, const int32_t*, const int32_t*,
                                     const int32_t*, const double*, int64_t, int, int, cudaStream_t);
template void launch_step<float>(const Inst<float>*, const Work*, const int*, int, const PState<float>&,
                                 const StepArgs&, int, bool, bool, int, int, int*, unsigned long long*, cudaStream_t);
template void launch_step<double>(const Inst<double>*, const Work*, const int*, int, const PState<double>&,
                                  const StepArgs&, int, bool, bool, int, int, int*, unsigned long long*, cudaStream_t);

}  // namespace mpmb

extern "C" mpm_status mpm_check_report(int64_t* violations, int32_t* site, int64_t* index, int32_t reset) {
#ifdef MPMB_CHECKED
    using mpmb::CheckRecord;
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        return MPM_CUDA_ERROR;
    }
    CheckRecord r{};
    if (cudaMemcpyFromSymbol(&r, mpmb::g_check, sizeof(r)) != cudaSuccess) {
        cudaGetLastError();
        return MPM_CUDA_ERROR;
    }
    if (violations) *violations = (int64_t)r.count;
    if (site) *site = r.site;
    if (index) *index = r.index;
    if (reset) {
        const CheckRecord z{};
        if (cudaMemcpyToSymbol(mpmb::g_check, &z, sizeof(z)) != cudaSuccess) {
            cudaGetLastError();
            return MPM_CUDA_ERROR;
        }
    }
    return MPM_OK;
#else
    (void)reset;
    if (violations) *violations = 0;
    if (site) *site = 0;
    if (index) *index = 0;
    return MPM_NOT_SUPPORTED;
#endif
}
