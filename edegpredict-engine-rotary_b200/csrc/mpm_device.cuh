// mpm_device.cuh -- device-side types and helpers of the B200 MPM step.
//
// Layout in HBM (per handle; a batch concatenates instances):
//   particles, SoA of 16-byte (FP32) or 32-byte (FP64) vectors, one vector
//   array per group of four scalars, so every particle load is one coalesced
//   128-bit access per group:
//     A0 = (xi_x, xi_y, xi_z, eps_p)   xi: position in cells relative to the
//                                       origin of the particle's 4^3-cell bin
//     A1 = (H0..H3) A2 = (H4..H7)      H  = F - I   (row-major)
//     A3 = (H8, Hp8, dT, D)            Hp = F_p - I, dT = T - T_amb, D damage
//     A4 = (Hp0..Hp3) A5 = (Hp4..Hp7)
//     B0 = (vx, vy, vz, edot) B1 = (C0..C3) B2 = (C4..C7) B3 = (C8, 0, 0, 0)
//     S0 = (sxx, syy, szz, sxy) S1 = (sxz, syz, 0, 0)
//     K0/K1 backstress (same packing as S; only with H_kin > 0)
//     sres (scalar), status (u8), id (i32)
//     X  = (xi_x, xi_y, xi_z, 0) low parts  (FP32 state only: xi = A0.xyz + X.xyz)
//   Storing F - I and F_p - I keeps FP32 relative precision on small strains.
//   A per-step move is ~1e-4 cell, a few hundred ulps of a bin-local FP32
//   coordinate, so its rounding would bias the trajectory by ~1e-3 of the
//   displacement; the hi + lo pair (updated by an exact two-sum) removes that.
//   grid: per node one vector (m, p_x, p_y, p_z), row-major (x fastest); p
//   already contains the internal and external force impulse f*dt.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mpmb {

constexpr int kBin = 4;          // bin edge in cells (particles binned by their stencil base node)
constexpr int kTile = 6;         // tile edge in nodes (bin + 2 for the quadratic stencil)
constexpr int kTileNodes = kTile * kTile * kTile;
// padded shared-memory plane: node (x,y,z) -> x + 8y + 68z; a warp of 32 distinct
// bin cells (4x4x2) then maps to 32 distinct banks
constexpr int kSY = 8, kSZ = 68, kPlane = 392;

enum : uint8_t { ST_ACTIVE = 0, ST_INACTIVE = 1, ST_CHIP = 2, ST_BOUNDARY = 3, ST_FIXED = 4 };
enum : int { TOOL_NONE = 0, TOOL_RASTER = 1, TOOL_SDF_STICKY = 2, TOOL_SDF_SLIP = 3 };
// Error bits.  ERR_TIMEOUT lives in the handle's word (a bounded wait gave
// up).  The instance words hold one byte per cause, each set by a plain byte
// store of 1 (no read-modify-write): byte 0 a non-finite position, byte 1 a
// Newton return that did not converge.
enum : int { ERR_NUMERIC = 1, ERR_TIMEOUT = 2, ERR_NEWTON = 1 << 8 };

struct alignas(32) D4 { double x, y, z, w; };

template <typename R> struct V4T;
template <> struct V4T<float> { using T = float4; };
template <> struct V4T<double> { using T = D4; };
template <typename R> using V4 = typename V4T<R>::T;

template <typename R> __host__ __device__ inline V4<R> mk4(R a, R b, R c, R d) {
    V4<R> v;
    v.x = a; v.y = b; v.z = c; v.w = d;
    return v;
}

// Particle state of a handle (or of a whole batch), device pointers.
template <typename R> struct PState {
    V4<R>* A[6];
    V4<R>* B[4];
    V4<R>* S[2];
    V4<R>* K[2];
    V4<R>* X;           // FP32 state: low parts of the bin-local position (x, y, z, 0); NULL for FP64
    R* sres;
    uint8_t* status;
    uint8_t* asb;       // adiabatic shear counter (MPMParticle::asbCounter), 0..10
    int32_t* id;
    int32_t* bin;       // bin (block) index the particle is filed under, written by the re-bin
    int32_t* orig;      // position of the particle in upload order
    int32_t* skey;      // the particle's key at the re-bin that placed it, relative to its
                        // instance (bin*64 + cell; nbins*64 when INACTIVE; -1 before any)
};

// Per-instance constants, built on the host.  Lives in a device array (the
// tensor maps must be 64-byte aligned in global memory).
template <typename R> struct alignas(128) Inst {
    CUtensorMap tmap[2];           // TMA descriptors of grid buffers 0 and 1
    V4<R>* grid[2];
    // raster mode, per grid node: 0 unmarked, 1 marked by a sample (the tool's
    // velocity), q + 1 marked last by tool node q (that node's velocity)
    int32_t* tool_mask;
    int nx, ny, nz;
    int nbx, nby, nbz;
    int64_t nn;
    double dx, ox, oy, oz;
    double dt, t0;                 // step size and time at the first step of the current call
    int64_t step0;                 // step counter at the first step of the current call
    // material (R copies for the hot path)
    R mu, lam, pmass, pvol;
    R A, B, n, C, m, edot0, Hkin;
    R D1, D2, D3, D4c, D5, Dth;
    R Tspan;                       // max(Tm - Tamb, 1)
    R ylo;                         // lower bound of the flow stress of an unheated particle (0: none)
    R dTmax;                       // Tm - Tamb (temperature cap as a rise)
    R heat;                        // beta / max(rho_phys cp, 1e-12)
    R apic;                        // apic_dinv_factor, applied as factor/dx
    R decay, deps_cap, dT_cap;
    double fix_thick, fix_damp, grav, mthr;
    int lod, plast;
    double lod_r1, lod_r2;
    int chip_every;
    int newton_maxit;
    double newton_tol;
    // tool
    int tool_mode, tool_shape;
    double tool_p0[3], tool_v[3], tool_t0;
    double tool_r, tool_rake, tool_clear, tool_tip_dz;
    double tool_sg, tool_cg, tool_sa, tool_ca;   // sin/cos of rake and clearance, computed on the host
    // raster samples (offsets from the tool pose: x..., y..., z...), rasterised
    // at the pose of each step; or, when tn_end is set, the FEM tool's node
    // records: node q at tn_start_q + a (tn_end_q - tn_start_q), a = tn_a0 +
    // (steps since tn_step0) tn_da (tn_end_q when tn_start is NULL)
    const double* samples;
    int n_samples;
    int tn_n, tn_stride;
    int tn_off[6];                 // byte offsets of x, y, z, vx, vy, vz
    const unsigned char* tn_start;
    const unsigned char* tn_end;
    double tn_a0, tn_da;
    int64_t tn_step0;
    // particle-side tool contact after every contact_every-th step (0: off)
    int contact_every;
    double contact_r, contact_mu, contact_hp;
    double rho_phys, cp;           // physical density and specific heat (contact heating)
    // adiabatic shear band heating after the move (asb_on = 0: off); temperatures as rises
    // above Tamb: the heated-particle guard, the cap asb_max_temp_ratio * Tm - Tamb
    int asb_on;
    R asb_rise, asb_min_rate, asb_crit, asb_heat, asb_Tcap;
    // grid heat conduction (heat_on = 0: off): T m scatter buffers (with grid[2]), the node
    // temperatures after the diffusion step, alpha dt / dx^2, and the absolute ambient (the
    // particles hold the rise above it)
    int heat_on;
    R* tm[2];
    R* tn;
    double heat_c;
    R Tamb;
    int64_t gbase;                 // first node of this instance in the batch grid arrays
    // voxel tool SDF for the contact (sdf_on = 0: the analytic SDF): texture, voxels per axis,
    // voxel (0,0,0) corner and edge in the tool frame, the frame's rotation about z
    int sdf_on;
    unsigned long long sdf_tex;
    int sdf_n[3];
    float sdf_o[3], sdf_vox, sdf_cos, sdf_sin;
    // external force for one step (radius 0: none)
    double ext_c[3], ext_r, ext_f[3];
    // per-particle external force for one step, indexed pbase + upload order
    // (written by an AoS import; NULL: none)
    const V4<R>* pext;
    // MPMWorkpieceSolver's semantics (mpm_set_workpiece_semantics): its shear
    // and bulk moduli, damage rate divisor, CHIP thresholds (plastic strain,
    // fraction of Tm), tool contact radius, contact heating damping, per-step
    // heating cap with its switch, and the tool samples' offset box (x, y, z
    // min then max) that bounds the nearest-sample search
    R ws_shear, ws_bulk, ws_fail, ws_crit_eps, ws_chip_ratio, ws_damping, ws_max_rise;
    int ws_clamp;
    double ws_contact_r;
    double ws_sbox[6];
    int64_t pbase;                 // first particle slot of this instance in the batch arrays
    int64_t np;                    // live particles of this instance, at [pbase, pbase + np)
    int64_t pcap;                  // particle slots of this instance
    int fresh;                     // positions still in the upload scratch (not yet binned)
    int nbins;                     // nbx * nby * nbz
    int* ierr;                     // this instance's error word: byte 0 NaN/Inf, byte 1 Newton
    int bin0;                      // first bin of this instance in the batch bin tables
    // re-bin phase: this instance is re-binned before the step launches of
    // points k = rebin_first, rebin_first + sort_every, ... of the current
    // call (point k: before the launch that holds G2P of step k, fused
    // schedule; before the P2G of step k, split schedule); at other re-bins
    // of the handle it keeps its layout
    int rebin_first;
    int rebin_now;                 // binned from its positions at the next re-bin whatever its phase
    // deterministic mode: the node sums of particles whose stencil left their
    // bin's tile, in fixed point (value x esc_scale rounded to an integer and
    // added with integer atomics, so that the order of the adds cannot change
    // the sum), channel c (m, p_x, p_y, p_z, T m) of node li at
    // esc[c * esc_stride + li]; esc_flag[b] is set for each bin b whose core
    // holds such a node.  NULL: the default mode's float atomics on the grid.
    unsigned long long* esc;
    int64_t esc_stride;
    int* esc_flag;
    double esc_scale;
};

// Deterministic mode: node-tile values stored per work item (channels m,
// p_x, p_y, p_z, T m; kTileNodes nodes each, in tile order x + 6y + 36z).
constexpr int kPartCh = 5;

// Threads per CTA of the step kernel (four warps, each with its own P2G tile).
constexpr int kNT = 128;
constexpr int kWarps = kNT / 32;
// Cells per bin (4x4x4): the sort key of a particle is bin*64 + cell in bin.
constexpr int kCellsPerBin = kBin * kBin * kBin;

// One unit of work: the particles of one bin of one instance.
struct Work {
    int inst;
    int bin;
    int start;     // relative to the instance's pbase
    int count;
};

struct StepArgs {
    int k;              // step index within the current call (G2P part: step k; P2G part: step k+1 when fused)
    int write_out;      // G2P: store v, C, edot (final step of a call, or split schedule)
    int sigma_all;      // P2G: store stress for every ACTIVE particle (last P2G of a call)
    int use_ext;        // P2G: apply the one-step external force
    int p2g_step;       // step index of the P2G part
    int ext;            // some instance runs the adiabatic shear model or heat conduction: launches
                        // take the kernel variant that has them (the others carry none of their code)
    int chunk = 2;         // FP32 particles per pass / 128 (1, 2 or 4): the launch config's pass size
    void* part = nullptr;  // deterministic mode: each work item's node tile is stored at
                           // part + wi * kPartCh * kTileNodes (R values) for k_node_sum to add
                           // up in a fixed order, instead of added to the grid with atomics
};

// ------------------------------------------------------------------ weights

// Quadratic B-spline weights on one axis, restating getWeightsAndGradients
// (reference src/MPMSolver.cu:20-34) in cell units: base = floor(xi - 0.5),
// d = xi - base in [0.5, 1.5); dw is d/dxi (divide by dx for a gradient).
template <typename R> __device__ __forceinline__ int bspline(R xi, R w[3], R dw[3]) {
    R fb = floor(xi - R(0.5));
    R d = xi - fb;
    R a = R(1.5) - d, b = d - R(1), c = d - R(0.5);
    w[0] = R(0.5) * a * a;
    w[1] = R(0.75) - b * b;
    w[2] = R(0.5) * c * c;
    dw[0] = -a;
    dw[1] = R(-2) * b;
    dw[2] = c;
    return (int)fb;
}

__device__ __forceinline__ int tidx(int x, int y, int z) { return x + kSY * y + kSZ * z; }

// ------------------------------------------------------------------ tool SDF

// Analytic rigid-tool SDF and outward normal (an extension of this build; the
// reference boundary is the rasterised tool, src/MPMSolver.cu:444-492).
// Cylinder with axis along y, or a rounded wedge extruded along y (sharp core
// wedge with apex at the edge-circle centre, offset by the edge radius).
// Every product and sum is rounded separately (no FMA contraction), so that
// the inside/outside decision of a node lying on the tool surface is the same
// as in a plain IEEE evaluation of the formula.
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }

template <typename I>
__device__ inline double tool_sdf(const I& P, double x, double z, double pr0, double pr2, double nrm[3]) {
    const double qx = ds(x, pr0), qz = ds(z, pr2);
    nrm[1] = 0.0;
    if (P.tool_shape == 0) {
        const double r = sqrt(da(dm(qx, qx), dm(qz, qz)));
        if (r > 0.0) { nrm[0] = qx / r; nrm[2] = qz / r; } else { nrm[0] = 0.0; nrm[2] = 1.0; }
        return ds(r, P.tool_r);
    }
    const double sg = P.tool_sg, cg = P.tool_cg, sa = P.tool_sa, ca = P.tool_ca;
    const double t1x = -sg, t1z = cg, n1x = cg, n1z = sg;
    const double t2x = -ca, t2z = sa, n2x = -sa, n2z = -ca;
    const double d1 = da(dm(n1x, qx), dm(n1z, qz)), d2 = da(dm(n2x, qx), dm(n2z, qz));
    double core;
    if (d1 <= 0.0 && d2 <= 0.0) {
        if (d1 >= d2) { core = d1; nrm[0] = n1x; nrm[2] = n1z; } else { core = d2; nrm[0] = n2x; nrm[2] = n2z; }
    } else {
        const double s1 = fmax(da(dm(qx, t1x), dm(qz, t1z)), 0.0), s2 = fmax(da(dm(qx, t2x), dm(qz, t2z)), 0.0);
        const double e1x = ds(qx, dm(s1, t1x)), e1z = ds(qz, dm(s1, t1z));
        const double e2x = ds(qx, dm(s2, t2x)), e2z = ds(qz, dm(s2, t2z));
        const double l1 = sqrt(da(dm(e1x, e1x), dm(e1z, e1z))), l2 = sqrt(da(dm(e2x, e2x), dm(e2z, e2z)));
        if (l1 <= l2) {
            core = l1;
            if (l1 > 0) { nrm[0] = e1x / l1; nrm[2] = e1z / l1; } else { nrm[0] = n1x; nrm[2] = n1z; }
        } else {
            core = l2;
            if (l2 > 0) { nrm[0] = e2x / l2; nrm[2] = e2z / l2; } else { nrm[0] = n2x; nrm[2] = n2z; }
        }
    }
    return ds(core, P.tool_r);
}

// True when the point is certainly outside the tool (phi > 0), from a bound
// that needs no square root: the cylinder's squared radius, or for the
// convex core wedge the larger face-plane distance (a lower bound of the
// distance to it).  The margin is far above the rounding of either path.
template <typename I>
__device__ __forceinline__ bool tool_far(const I& P, double x, double z, double pr0, double pr2, double extra = 0.0) {
    // phi > extra for certain (extra = 0: outside the tool)
    const double qx = ds(x, pr0), qz = ds(z, pr2);
    const double r = P.tool_r + extra;
    const double m = r + 1e-9 * (r + fabs(qx) + fabs(qz));
    if (P.tool_shape == 0) return da(dm(qx, qx), dm(qz, qz)) > m * m;
    const double d1 = da(dm(P.tool_cg, qx), dm(P.tool_sg, qz));
    const double d2 = da(dm(-P.tool_sa, qx), dm(-P.tool_ca, qz));
    return fmax(d1, d2) > m;
}

// World coordinate of grid node index g on one axis: g*dx + origin, rounded
// like the reference's (gx * config.dx + domainMin.x) (src/MPMSolver.cu:387).
__device__ __forceinline__ double node_coord(int g, double dx, double o) { return da(dm((double)g, dx), o); }

// ------------------------------------------------------------------ Philox

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), 24-bit uniforms in [0,1).
__host__ __device__ inline void philox_u4(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2,
                                          uint32_t c3, float out[4]) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = (float)(c0 >> 8) * (1.0f / 16777216.0f);
    out[1] = (float)(c1 >> 8) * (1.0f / 16777216.0f);
    out[2] = (float)(c2 >> 8) * (1.0f / 16777216.0f);
    out[3] = (float)(c3 >> 8) * (1.0f / 16777216.0f);
}

}  // namespace mpmb
