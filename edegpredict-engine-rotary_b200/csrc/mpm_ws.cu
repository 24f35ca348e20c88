// mpm_ws.cu -- the reference's other MPM solver, MPMWorkpieceSolver
// (src/MPMWorkpieceSolver.cu), as an alternate step semantics of a handle
// (mpm_set_workpiece_semantics): trilinear PIC transfers, a hypoelastic
// stress rate with the Johnson-Cook radial return at the old plastic strain,
// and a tool boundary that projects out the approaching normal velocity at
// the nearest tool sample, heating the node.  The engine never constructs
// that solver, so this path is an option; it runs as plain per-particle and
// per-node kernels over the handle's SoA state and grid (no bins, no tile).
//
// Grid buffer 0 carries per node (m, p + f dt) before the grid kernel and
// (m, v) after it; the heat-conduction buffer tm[0] carries T m.
#include <cuda_runtime.h>

#include "mpm_device.cuh"
#include "mpm_internal.h"

namespace mpmb {
namespace {

constexpr int kWT = 256;

template <typename R> __device__ __forceinline__ void atomic_v4(V4<R>* d, R a, R b, R c, R e);
template <> __device__ __forceinline__ void atomic_v4<float>(float4* d, float a, float b, float c, float e) {
    atomicAdd(d, make_float4(a, b, c, e));
}
template <> __device__ __forceinline__ void atomic_v4<double>(D4* d, double a, double b, double c, double e) {
    atomicAdd(&d->x, a);
    atomicAdd(&d->y, b);
    atomicAdd(&d->z, c);
    atomicAdd(&d->w, e);
}

// World position of slot pi: its bin's origin + the bin-local position (+ the
// FP32 low parts).
template <typename R>
__device__ __forceinline__ void ws_world(const Inst<R>& P, const PState<R>& ps, int64_t pi, const V4<R>& a0,
                                         double w[3]) {
    const int bin = ps.bin[pi];
    const int b[3] = {bin % P.nbx, (bin / P.nbx) % P.nby, bin / (P.nbx * P.nby)};
    double lo[3] = {0.0, 0.0, 0.0};
    if (ps.X) {
        const V4<R> x = ps.X[pi];
        lo[0] = (double)x.x; lo[1] = (double)x.y; lo[2] = (double)x.z;
    }
    const double o[3] = {P.ox, P.oy, P.oz};
    const R l[3] = {a0.x, a0.y, a0.z};
    for (int a = 0; a < 3; ++a) w[a] = o[a] + ((double)(b[a] * kBin) + ((double)l[a] + lo[a])) * P.dx;
}

// computeWeights (src/MPMWorkpieceSolver.cu:52-90): the 8 trilinear nodes in
// dz, dy, dx order (index -1 outside the grid).
template <typename R>
__device__ __forceinline__ void ws_weights(const Inst<R>& P, const double x[3], int64_t id[8], R w[8], R g[8][3]) {
    const double o[3] = {P.ox, P.oy, P.oz};
    int base[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
        const double r = (x[a] - o[a]) / P.dx;
        base[a] = (int)floor(r);
        f[a] = r - base[a];
    }
    const R idx = (R)(1.0 / P.dx);
    int q = 0;
    for (int dz = 0; dz <= 1; ++dz)
        for (int dy = 0; dy <= 1; ++dy)
            for (int dx = 0; dx <= 1; ++dx, ++q) {
                const int i = base[0] + dx, j = base[1] + dy, k = base[2] + dz;
                if (i < 0 || j < 0 || k < 0 || i >= P.nx || j >= P.ny || k >= P.nz) {
                    id[q] = -1;
                    w[q] = R(0);
                    g[q][0] = g[q][1] = g[q][2] = R(0);
                    continue;
                }
                const R wx = (R)(dx ? f[0] : 1.0 - f[0]), wy = (R)(dy ? f[1] : 1.0 - f[1]),
                        wz = (R)(dz ? f[2] : 1.0 - f[2]);
                const R gx = dx ? idx : -idx, gy = dy ? idx : -idx, gz = dz ? idx : -idx;
                id[q] = ((int64_t)k * P.ny + j) * P.nx + i;
                w[q] = wx * wy * wz;
                g[q][0] = gx * wy * wz;
                g[q][1] = wx * gy * wz;
                g[q][2] = wx * wy * gz;
            }
}

template <typename R> __device__ __forceinline__ R ws_eq(R xx, R yy, R zz, R xy, R xz, R yz) {
    const R s1 = xx - yy, s2 = yy - zz, s3 = zz - xx;
    return sqrt(R(0.5) * (s1 * s1 + s2 * s2 + s3 * s3 + R(6) * (xy * xy + xz * xz + yz * yz)));
}

// mpmP2GKernel (:98-134): mass, momentum and T m of every particle that is
// not INACTIVE, the force impulse f dt added to the momentum (the grid kernel
// divides once): the stress divergence and the particle force of ACTIVE and
// FIXED particles, the particle force alone of CHIP ones.  The particle force
// (MPMParticleGPU::f) is, in the first step of a call, the pending external
// force -- applyMPMExternalForceKernel's (:402-413): the whole force on
// ACTIVE particles within the radius -- plus an imported per-particle force.
template <typename R>
__global__ void __launch_bounds__(kWT) k_ws_p2g(const Inst<R>* __restrict__ insts, int ii, PState<R> ps, int use_ext) {
    const Inst<R>& P = insts[ii];
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.np) return;
    const int64_t pi = P.pbase + s;
    const uint8_t st = ps.status[pi];
    if (st == ST_INACTIVE) return;
    const V4<R> a0 = ps.A[0][pi], a3 = ps.A[3][pi], b0 = ps.B[0][pi];
    double x[3];
    ws_world(P, ps, pi, a0, x);
    int64_t id[8];
    R w[8], g[8][3];
    ws_weights(P, x, id, w, g);
    R fp[3] = {R(0), R(0), R(0)};
    if (use_ext) {
        if (P.ext_r > 0.0 && st == ST_ACTIVE) {
            const double d[3] = {x[0] - P.ext_c[0], x[1] - P.ext_c[1], x[2] - P.ext_c[2]};
            if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] <= P.ext_r * P.ext_r)
                for (int a = 0; a < 3; ++a) fp[a] = (R)P.ext_f[a];
        }
        if (P.pext) {
            const V4<R> e = P.pext[P.pbase + ps.orig[pi]];
            fp[0] += e.x; fp[1] += e.y; fp[2] += e.z;
        }
    }
    R sg[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
    const bool stress = st == ST_ACTIVE || st == ST_FIXED;
    if (stress) {
        const V4<R> s0 = ps.S[0][pi], s1 = ps.S[1][pi];
        sg[0] = s0.x; sg[1] = s0.y; sg[2] = s0.z; sg[3] = s0.w; sg[4] = s1.x; sg[5] = s1.y;
    }
    const bool force = stress || st == ST_CHIP;
    const R m = P.pmass, V = P.pvol, dt = (R)P.dt, T = P.Tamb + a3.z;
    V4<R>* __restrict__ grid = P.grid[0];
    R* __restrict__ tm = P.tm[0];
    for (int q = 0; q < 8; ++q) {
        if (id[q] < 0 || !(w[q] > R(0))) continue;
        const R mw = m * w[q];
        R f[3] = {R(0), R(0), R(0)};
        if (force) {
            for (int a = 0; a < 3; ++a) f[a] = fp[a] * w[q];
            if (stress) {
                f[0] += -(sg[0] * g[q][0] + sg[3] * g[q][1] + sg[4] * g[q][2]) * V;
                f[1] += -(sg[3] * g[q][0] + sg[1] * g[q][1] + sg[5] * g[q][2]) * V;
                f[2] += -(sg[4] * g[q][0] + sg[5] * g[q][1] + sg[2] * g[q][2]) * V;
            }
        }
        atomic_v4<R>(&grid[id[q]], mw, b0.x * mw + f[0] * dt, b0.y * mw + f[1] * dt, b0.z * mw + f[2] * dt);
        atomicAdd(&tm[id[q]], T * mw);
    }
}

// mpmGridUpdateKernel (:136-192) per node with m > 1e-18: v = (p + f dt) / m;
// nodes at or below min z + fixture thickness + dx stop; then the nearest
// tool sample within the contact radius (samples at the pose of step k, the
// first of equal distances) gives n = (node - sample) / |.|, and v.n < 0 is
// removed, heating T m by min(0.5 m vn^2 damping / (m cp), cap) m and adding
// |m vn / dt| to the contact force (ctr[0], FP64).
template <typename R>
__global__ void __launch_bounds__(kWT) k_ws_grid(const Inst<R>* __restrict__ insts, int ii, int k,
                                                 double* __restrict__ fsum) {
    const Inst<R>& P = insts[ii];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.nn) return;
    V4<R>* __restrict__ grid = P.grid[0];
    const V4<R> gv = grid[idx];
    const R m = gv.x;
    if (!(m > R(1e-18))) return;
    R v[3] = {gv.y / m, gv.z / m, gv.w / m};
    const int i = (int)(idx % P.nx);
    const int64_t t = idx / P.nx;
    const int j = (int)(t % P.ny), kz = (int)(t / P.ny);
    const double pos[3] = {P.ox + i * P.dx, P.oy + j * P.dx, P.oz + kz * P.dx};
    if (pos[2] <= P.oz + P.fix_thick + P.dx) {
        grid[idx] = mk4<R>(m, R(0), R(0), R(0));
        return;
    }
    if (P.n_samples > 0) {
        const double tk = da(P.t0, dm((double)k, P.dt));
        const double pr[3] = {da(P.tool_p0[0], dm(P.tool_v[0], ds(tk, P.tool_t0))),
                              da(P.tool_p0[1], dm(P.tool_v[1], ds(tk, P.tool_t0))),
                              da(P.tool_p0[2], dm(P.tool_v[2], ds(tk, P.tool_t0)))};
        // nodes farther than the radius from the samples' box cannot meet one
        bool near = true;
        for (int a = 0; a < 3; ++a)
            near = near && pos[a] >= pr[a] + P.ws_sbox[a] - P.ws_contact_r &&
                   pos[a] <= pr[a] + P.ws_sbox[3 + a] + P.ws_contact_r;
        if (near) {
            double r2 = P.ws_contact_r * P.ws_contact_r, bn[3] = {0.0, 0.0, 0.0};
            bool hit = false;
            const int ns = P.n_samples;
            for (int q = 0; q < ns; ++q) {
                const double d[3] = {pos[0] - (pr[0] + P.samples[q]), pos[1] - (pr[1] + P.samples[ns + q]),
                                     pos[2] - (pr[2] + P.samples[2 * ns + q])};
                const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (d2 < r2 && d2 > 1e-20) {
                    r2 = d2;
                    const double len = sqrt(d2);
                    if (len > 1e-12) { bn[0] = d[0] / len; bn[1] = d[1] / len; bn[2] = d[2] / len; }
                    else { bn[0] = bn[1] = bn[2] = 0.0; }
                    hit = true;
                }
            }
            if (hit) {
                const R vn = v[0] * (R)bn[0] + v[1] * (R)bn[1] + v[2] * (R)bn[2];
                if (vn < R(0)) {
                    atomicAdd(fsum, fabs((double)m * (double)vn / fmax(P.dt, 1e-15)));
                    for (int a = 0; a < 3; ++a) v[a] -= vn * (R)bn[a];
                    const R heat = R(0.5) * m * vn * vn * P.ws_damping;
                    R dT = heat / fmax(m * (R)P.cp, R(1e-12));
                    if (P.ws_clamp) dT = fmin(dT, P.ws_max_rise);
                    P.tm[0][idx] += dT * m;
                }
            }
        }
    }
    grid[idx] = mk4<R>(m, v[0], v[1], v[2]);
}

// mpmG2PKernel (:264-400), then on even step counts the workpiece solver's
// chipFractureAndSeparationKernel (:667-725) on the same particle.
template <typename R>
__global__ void __launch_bounds__(kWT) k_ws_g2p(const Inst<R>* __restrict__ insts, int ii, PState<R> ps, int k,
                                                int diffused) {
    const Inst<R>& P = insts[ii];
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.np) return;
    const int64_t pi = P.pbase + s;
    uint8_t st = ps.status[pi];
    if (st == ST_INACTIVE) return;
    V4<R> a0 = ps.A[0][pi], a3 = ps.A[3][pi], b0 = ps.B[0][pi];
    double x[3];
    ws_world(P, ps, pi, a0, x);
    int64_t id[8];
    R w[8], g[8][3];
    ws_weights(P, x, id, w, g);
    const V4<R>* __restrict__ grid = P.grid[0];
    R v[3] = {R(0), R(0), R(0)}, temp = R(0), wsum = R(0), L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < 8; ++q) {
        if (id[q] < 0 || !(w[q] > R(0))) continue;
        const V4<R> nv = grid[id[q]];
        if (!(nv.x > R(1e-18))) continue;
        const R vv[3] = {nv.y, nv.z, nv.w};
        for (int a = 0; a < 3; ++a) v[a] += vv[a] * w[q];
        temp += (diffused ? P.tn[id[q]] : P.tm[0][id[q]] / nv.x) * w[q];
        wsum += w[q];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) L[a][b] += vv[a] * g[q][b];
    }
    if (st == ST_FIXED) {
        ps.B[0][pi] = mk4<R>(R(0), R(0), R(0), b0.w);
        return;
    }
    const R dt = (R)P.dt;
    // x += v dt, in the particle's bin (FP32: the exact two-sum of the step kernel)
    const R dtdx = (R)(P.dt / P.dx);
    R xi[3] = {a0.x, a0.y, a0.z};
    if (ps.X) {
        V4<R> lo = ps.X[pi];
        R l[3] = {lo.x, lo.y, lo.z};
        for (int a = 0; a < 3; ++a) {
            const R inc = fma(v[a], dtdx, l[a]);
            const R sm = xi[a] + inc;
            const R bv = sm - xi[a];
            l[a] = (xi[a] - (sm - bv)) + (inc - bv);
            xi[a] = sm;
        }
        ps.X[pi] = mk4<R>(l[0], l[1], l[2], R(0));
    } else {
        for (int a = 0; a < 3; ++a) xi[a] = (R)((double)xi[a] + (double)v[a] * P.dt / P.dx);
    }
    R eps = a0.w, D = a3.w, dT = a3.z, edot = b0.w;
    R T = P.Tamb + dT;
    if (wsum > R(1e-8)) T = fmin(fmax(temp / wsum, P.Tamb), P.Tamb + P.dTmax);
    R sg[6], bs[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
    {
        const V4<R> s0 = ps.S[0][pi], s1 = ps.S[1][pi];
        sg[0] = s0.x; sg[1] = s0.y; sg[2] = s0.z; sg[3] = s0.w; sg[4] = s1.x; sg[5] = s1.y;
    }
    if (ps.K[0]) {
        const V4<R> k0 = ps.K[0][pi], k1 = ps.K[1][pi];
        bs[0] = k0.x; bs[1] = k0.y; bs[2] = k0.z; bs[3] = k0.w; bs[4] = k1.x; bs[5] = k1.y;
    }
    R sres = ps.sres[pi];
    const R Dth = P.Dth;
    if (st == ST_ACTIVE) {
        const R Dxx = L[0][0], Dyy = L[1][1], Dzz = L[2][2];
        const R Dxy = R(0.5) * (L[0][1] + L[1][0]), Dxz = R(0.5) * (L[0][2] + L[2][0]),
                Dyz = R(0.5) * (L[1][2] + L[2][1]);
        const R tr = Dxx + Dyy + Dzz;
        const R dxx = Dxx - tr / R(3), dyy = Dyy - tr / R(3), dzz = Dzz - tr / R(3);
        const R rate = sqrt(R(2.0 / 3.0) * (dxx * dxx + dyy * dyy + dzz * dzz +
                                             R(2) * (Dxy * Dxy + Dxz * Dxz + Dyz * Dyz)));
        edot = rate;
        const R G = P.ws_shear, K = P.ws_bulk;
        const R pinc = K * tr * dt;
        sg[0] += (R(2) * G * dxx) * dt + pinc;
        sg[1] += (R(2) * G * dyy) * dt + pinc;
        sg[2] += (R(2) * G * dzz) * dt + pinc;
        sg[3] += R(2) * G * Dxy * dt;
        sg[4] += R(2) * G * Dxz * dt;
        sg[5] += R(2) * G * Dyz * dt;
        R sh[6];
        for (int q = 0; q < 6; ++q) sh[q] = sg[q] - bs[q];
        const R seq = ws_eq(sh[0], sh[1], sh[2], sh[3], sh[4], sh[5]);
        // johnsonCookStress (:43-50) at the old plastic strain, the new rate and temperature
        const R strain = P.A + P.B * pow(fmax(eps, R(0)), P.n);
        const R ratio = fmax(edot / fmax(P.edot0, R(1e-9)), R(1));
        const R rt = R(1) + P.C * log(ratio);
        const R ts = fmax(R(0), fmin(R(1), (T - P.Tamb) / P.Tspan));
        const R flow = strain * rt * fmax(R(0.01), R(1) - pow(ts, P.m));
        if (seq > flow && seq > R(1e-9)) {
            const R sc = flow / seq;
            for (int q = 0; q < 6; ++q) sg[q] = bs[q] + sc * sh[q];
            const R dp = (seq - flow) / fmax(R(3) * G, R(1));
            if (P.Hkin > R(0) && dp > R(0)) {
                const R ns = P.Hkin * dp / seq;
                for (int q = 0; q < 6; ++q) bs[q] += ns * sh[q];
            }
            eps += dp;
            R h = R(0.9) * flow * dp / fmax((R)(P.rho_phys * P.cp), R(1));
            if (P.ws_clamp) h = fmin(h, P.ws_max_rise);
            T = fmin(T + h, P.Tamb + P.dTmax);
        }
        if (rate > R(0)) D += (rate * dt) / fmax(P.ws_fail, R(1e-3));
        if (D > R(0.7) * Dth && D < Dth) {
            const R dg = fmax(R(0), (Dth - D) / (Dth * R(0.3)));
            for (int q = 0; q < 6; ++q) { sg[q] *= dg; bs[q] *= dg; }
            sres = fmax(sres, ws_eq(sg[0], sg[1], sg[2], sg[3], sg[4], sg[5]));
        }
    }
    if (st == ST_ACTIVE && (D >= Dth || eps >= P.ws_crit_eps || T >= (P.Tamb + P.dTmax) * P.ws_chip_ratio)) {
        st = ST_CHIP;
        sres = fmax(sres, ws_eq(sg[0], sg[1], sg[2], sg[3], sg[4], sg[5]));
        for (int q = 0; q < 6; ++q) { sg[q] = R(0); bs[q] = R(0); }
        D = fmax(D, Dth);
    }
    // chip separation and fracture on even step counts, after the move
    if (((P.step0 + k) % 2) == 0) {
        if (st == ST_ACTIVE) {
            const double tk = da(P.t0, dm((double)k, P.dt));
            const double tipz = da(da(P.tool_p0[2], dm(P.tool_v[2], ds(tk, P.tool_t0))), P.tool_tip_dz);
            const int bin = ps.bin[pi];
            const double lo = ps.X ? (double)ps.X[pi].z : 0.0;
            const double zw = P.oz + ((double)((bin / (P.nbx * P.nby)) * kBin) + ((double)xi[2] + lo)) * P.dx;
            if (zw < tipz - P.dx * 1.5 && eps > R(1e-6)) {
                st = ST_CHIP;
                sres = fmax(sres, sqrt(sg[0] * sg[0] + sg[1] * sg[1] + sg[2] * sg[2]));
                for (int q = 0; q < 6; ++q) { sg[q] = R(0); bs[q] = R(0); }
                D = fmax(D, Dth);
            }
        } else if (st == ST_CHIP && D >= Dth * R(1.5)) {
            const uint32_t seed = (uint32_t)ps.id[pi] * 2654435761u;
            const R rx = (R)((double)((seed >> 16) & 0xFF) / 255.0 - 0.5);
            const R ry = (R)((double)((seed >> 8) & 0xFF) / 255.0 - 0.5);
            const R rz = (R)((double)(seed & 0xFF) / 255.0 - 0.5);
            const R sp = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            const R pm = sp * R(0.3) + R(0.5);
            v[0] += rx * pm; v[1] += ry * pm; v[2] += rz * pm;
            D = Dth * R(0.5);
        }
    }
    ps.A[0][pi] = mk4<R>(xi[0], xi[1], xi[2], eps);
    a3.z = T - P.Tamb;
    a3.w = D;
    ps.A[3][pi] = a3;
    ps.B[0][pi] = mk4<R>(v[0], v[1], v[2], edot);
    ps.S[0][pi] = mk4<R>(sg[0], sg[1], sg[2], sg[3]);
    ps.S[1][pi] = mk4<R>(sg[4], sg[5], R(0), R(0));
    if (ps.K[0]) {
        ps.K[0][pi] = mk4<R>(bs[0], bs[1], bs[2], bs[3]);
        ps.K[1][pi] = mk4<R>(bs[4], bs[5], R(0), R(0));
    }
    ps.sres[pi] = sres;
    if (st != ps.status[pi]) ps.status[pi] = st;
}

}  // namespace

template <typename R>
void launch_ws_step(const Inst<R>* insts, const std::vector<int64_t>& np, const std::vector<int64_t>& nn,
                    const PState<R>& ps, int k, int use_ext, int diffuse, double* fsum, cudaStream_t st,
                    void (*diffuse_fn)(const Inst<R>*, int, int, int64_t, cudaStream_t), int64_t nn_total) {
    Range nvtx_range("mpm.ws_step");
    const int n = (int)np.size();
    for (int i = 0; i < n; ++i) {
        if (np[i] <= 0) continue;
        k_ws_p2g<R><<<(int)((np[i] + kWT - 1) / kWT), kWT, 0, st>>>(insts, i, ps, use_ext);
        ++launch_counter();
    }
    for (int i = 0; i < n; ++i) {
        if (nn[i] <= 0) continue;
        k_ws_grid<R><<<(int)((nn[i] + kWT - 1) / kWT), kWT, 0, st>>>(insts, i, k, fsum);
        ++launch_counter();
    }
    if (diffuse) diffuse_fn(insts, n, 0, nn_total, st);
    for (int i = 0; i < n; ++i) {
        if (np[i] <= 0) continue;
        k_ws_g2p<R><<<(int)((np[i] + kWT - 1) / kWT), kWT, 0, st>>>(insts, i, ps, k, diffuse);
        ++launch_counter();
    }
}

template void launch_ws_step<float>(const Inst<float>*, const std::vector<int64_t>&, const std::vector<int64_t>&,
                                    const PState<float>&, int, int, int, double*, cudaStream_t,
                                    void (*)(const Inst<float>*, int, int, int64_t, cudaStream_t), int64_t);
template void launch_ws_step<double>(const Inst<double>*, const std::vector<int64_t>&, const std::vector<int64_t>&,
                                     const PState<double>&, int, int, int, double*, cudaStream_t,
                                     void (*)(const Inst<double>*, int, int, int64_t, cudaStream_t), int64_t);

}  // namespace mpmb
