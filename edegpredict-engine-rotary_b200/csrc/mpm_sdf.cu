// mpm_sdf.cu -- mpm_tool_sdf_build: the voxel signed-distance field of a
// closed tool mesh, as the reference's ToolSDF builds it on the host
// (src/ToolSDF.cu:212-280 build, :348-377 buildFromVerts, :379-532
// computeSDFCPU), with the per-voxel work on the GPU:
//   - every triangle's squared distance to the voxel centres of its bounding
//     box (grown by one voxel below and two above), kept as a minimum with an
//     integer atomic on the float bits (non-negative floats order like their
//     bit patterns, so the result does not depend on the order);
//   - distances, and the sign of the voxels within two voxels of the surface
//     from the nearest triangle's normal (the first nearest in triangle order
//     wins, as in the reference's loop);
// and on the host the three in-place passes that reach the voxels no
// triangle box covered (sequential by definition) and the large distance for
// the rest.  The float arithmetic is the reference's host arithmetic: the
// device code uses round-to-nearest intrinsics so that nothing is contracted.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/mpm_capi.h"
#include "mpm_internal.h"

namespace mpmb {
namespace {

constexpr unsigned kFltMaxBits = 0x7f7fffffu;   // FLT_MAX

struct SdfGeom {
    float ox, oy, oz, vox, inv;
    int nx, ny, nz;
};

// Squared distance from p to triangle abc and the closest point q: the region
// tests of Ericson's closest-point-on-triangle algorithm (Real-Time Collision
// Detection, 5.1.5) with the reference's interior case a + u (b - a) +
// v (c - a), u = 1 - v - w (src/ToolSDF.cu:92-167).
__device__ float tri_dist2(const float p[3], const float a[3], const float b[3], const float c[3], float q[3]) {
    float ab[3], ac[3], ap[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = __fsub_rn(b[k], a[k]);
        ac[k] = __fsub_rn(c[k], a[k]);
        ap[k] = __fsub_rn(p[k], a[k]);
    }
    auto dot = [](const float* u, const float* v) {
        return __fadd_rn(__fadd_rn(__fmul_rn(u[0], v[0]), __fmul_rn(u[1], v[1])), __fmul_rn(u[2], v[2]));
    };
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        for (int k = 0; k < 3; ++k) q[k] = a[k];
    } else {
        float bp[3];
        for (int k = 0; k < 3; ++k) bp[k] = __fsub_rn(p[k], b[k]);
        const float d3 = dot(ab, bp), d4 = dot(ac, bp);
        const float vc = __fsub_rn(__fmul_rn(d1, d4), __fmul_rn(d3, d2));
        if (d3 >= 0.0f && d4 <= d3) {
            for (int k = 0; k < 3; ++k) q[k] = b[k];
        } else if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
            const float v = __fdiv_rn(d1, __fsub_rn(d1, d3));
            for (int k = 0; k < 3; ++k) q[k] = __fadd_rn(a[k], __fmul_rn(v, ab[k]));
        } else {
            float cp[3];
            for (int k = 0; k < 3; ++k) cp[k] = __fsub_rn(p[k], c[k]);
            const float d5 = dot(ab, cp), d6 = dot(ac, cp);
            const float vb = __fsub_rn(__fmul_rn(d5, d2), __fmul_rn(d1, d6));
            const float va = __fsub_rn(__fmul_rn(d3, d6), __fmul_rn(d5, d4));
            if (d6 >= 0.0f && d5 <= d6) {
                for (int k = 0; k < 3; ++k) q[k] = c[k];
            } else if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
                const float w = __fdiv_rn(d2, __fsub_rn(d2, d6));
                for (int k = 0; k < 3; ++k) q[k] = __fadd_rn(a[k], __fmul_rn(w, ac[k]));
            } else if (va <= 0.0f && __fsub_rn(d4, d3) >= 0.0f && __fsub_rn(d5, d6) >= 0.0f) {
                const float w = __fdiv_rn(__fsub_rn(d4, d3), __fadd_rn(__fsub_rn(d4, d3), __fsub_rn(d5, d6)));
                for (int k = 0; k < 3; ++k) q[k] = __fadd_rn(b[k], __fmul_rn(w, __fsub_rn(c[k], b[k])));
            } else {
                const float den = __fdiv_rn(1.0f, __fadd_rn(__fadd_rn(va, vb), vc));
                const float v = __fmul_rn(vb, den), w = __fmul_rn(vc, den);
                const float u = __fsub_rn(__fsub_rn(1.0f, v), w);
                for (int k = 0; k < 3; ++k)
                    q[k] = __fadd_rn(__fadd_rn(a[k], __fmul_rn(u, __fsub_rn(b[k], a[k]))),
                                     __fmul_rn(v, __fsub_rn(c[k], a[k])));
            }
        }
    }
    const float dx = __fsub_rn(p[0], q[0]), dy = __fsub_rn(p[1], q[1]), dz = __fsub_rn(p[2], q[2]);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ void voxel_centre(const SdfGeom& G, int ix, int iy, int iz, float p[3]) {
    p[0] = __fadd_rn(G.ox, __fmul_rn(__fadd_rn((float)ix, 0.5f), G.vox));
    p[1] = __fadd_rn(G.oy, __fmul_rn(__fadd_rn((float)iy, 0.5f), G.vox));
    p[2] = __fadd_rn(G.oz, __fmul_rn(__fadd_rn((float)iz, 0.5f), G.vox));
}

__device__ void tri_verts(const float* __restrict__ v, const int* __restrict__ t, int i, float a[3], float b[3],
                          float c[3]) {
    for (int k = 0; k < 3; ++k) {
        a[k] = v[3 * t[3 * i] + k];
        b[k] = v[3 * t[3 * i + 1] + k];
        c[k] = v[3 * t[3 * i + 2] + k];
    }
}

__global__ void k_sdf_fill(unsigned* g, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        g[i] = kFltMaxBits;
}

// One CTA per triangle: its squared distance to the centres of its voxel box.
__global__ void k_sdf_scatter(const float* __restrict__ verts, const int* __restrict__ tris, int nt, SdfGeom G,
                              unsigned* __restrict__ g) {
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        float a[3], b[3], c[3];
        tri_verts(verts, tris, t, a, b, c);
        const float o[3] = {G.ox, G.oy, G.oz};
        const int n[3] = {G.nx, G.ny, G.nz};
        int i0[3], i1[3];
        for (int k = 0; k < 3; ++k) {
            const float lo = fminf(a[k], fminf(b[k], c[k])), hi = fmaxf(a[k], fmaxf(b[k], c[k]));
            const int l = (int)__fmul_rn(__fsub_rn(lo, o[k]), G.inv) - 1;
            const int h = (int)__fmul_rn(__fsub_rn(hi, o[k]), G.inv) + 2;
            i0[k] = max(0, l);
            i1[k] = min(n[k] - 1, h);
        }
        const int sx = i1[0] - i0[0] + 1, sy = i1[1] - i0[1] + 1, sz = i1[2] - i0[2] + 1;
        if (sx <= 0 || sy <= 0 || sz <= 0) continue;
        const int64_t cnt = (int64_t)sx * sy * sz;
        for (int64_t q = threadIdx.x; q < cnt; q += blockDim.x) {
            const int ix = i0[0] + (int)(q % sx), iy = i0[1] + (int)((q / sx) % sy), iz = i0[2] + (int)(q / ((int64_t)sx * sy));
            float p[3], cl[3];
            voxel_centre(G, ix, iy, iz, p);
            const float d2 = tri_dist2(p, a, b, c, cl);
            atomicMin(&g[ix + (int64_t)G.nx * (iy + (int64_t)G.ny * iz)], __float_as_uint(d2));
        }
    }
}

// Per voxel: the distance, and within two voxels of the surface the sign of
// (centre - nearest point) . normal of the nearest triangle.
__global__ void k_sdf_sign(const float* __restrict__ verts, const int* __restrict__ tris,
                           const float* __restrict__ normals, int nt, SdfGeom G, float* __restrict__ g) {
    const int64_t total = (int64_t)G.nx * G.ny * G.nz;
    const float band = __fmul_rn(G.vox, 2.0f);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        float d = g[i];
        if (d < FLT_MAX) d = __fsqrt_rn(d);
        g[i] = d;
        if (d > band) continue;
        const int ix = (int)(i % G.nx), iy = (int)((i / G.nx) % G.ny), iz = (int)(i / ((int64_t)G.nx * G.ny));
        float p[3];
        voxel_centre(G, ix, iy, iz, p);
        float best = FLT_MAX, bn[3] = {0, 0, 0}, bq[3] = {0, 0, 0};
        for (int t = 0; t < nt; ++t) {
            float a[3], b[3], c[3];
            tri_verts(verts, tris, t, a, b, c);
            bool skip = false;
            for (int k = 0; k < 3; ++k) {
                const float lo = fminf(a[k], fminf(b[k], c[k])), hi = fmaxf(a[k], fmaxf(b[k], c[k]));
                if (p[k] < __fsub_rn(lo, G.vox) || p[k] > __fadd_rn(hi, G.vox)) skip = true;
            }
            if (skip) continue;
            float q[3];
            const float d2 = tri_dist2(p, a, b, c, q);
            if (d2 < best) {
                best = d2;
                for (int k = 0; k < 3; ++k) { bn[k] = normals[3 * t + k]; bq[k] = q[k]; }
            }
        }
        if (best < FLT_MAX) {
            const float dot = __fadd_rn(__fadd_rn(__fmul_rn(__fsub_rn(p[0], bq[0]), bn[0]),
                                                  __fmul_rn(__fsub_rn(p[1], bq[1]), bn[1])),
                                        __fmul_rn(__fsub_rn(p[2], bq[2]), bn[2]));
            if (dot < 0.0f) g[i] = -d;
        }
    }
}

mpm_status fail(mpm_status s, const std::string& m) {
    set_lib_error("mpm_tool_sdf_build: " + m);
    return s;
}

}  // namespace
}  // namespace mpmb

extern "C" mpm_status mpm_tool_sdf_build(const float* verts, int32_t n_verts, const int32_t* tris, int32_t n_tris,
                                         const float* normals, double padding, int32_t voxels_per_axis,
                                         mpm_tool_sdf* desc, float* values) {
    using namespace mpmb;
    if (!verts || !tris || !desc || n_verts <= 0 || n_tris <= 0 || voxels_per_axis <= 0 || !(padding >= 0.0))
        return fail(MPM_INVALID_ARG, "needs vertices, triangles, a descriptor, padding >= 0 and voxels per axis > 0");
    for (int64_t i = 0; i < 3 * (int64_t)n_tris; ++i)
        if (tris[i] < 0 || tris[i] >= n_verts) return fail(MPM_INVALID_ARG, "triangle index out of range");
    // ToolSDF::build: bounding box, padding, isotropic voxel on the longest
    // axis, dims = extent / voxel + 2 (at most 256)
    float bmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < n_verts; ++i)
        for (int k = 0; k < 3; ++k) {
            bmin[k] = std::fmin(bmin[k], verts[3 * i + k]);
            bmax[k] = std::fmax(bmax[k], verts[3 * i + k]);
        }
    const float pad = (float)padding;
    float ext[3];
    for (int k = 0; k < 3; ++k) {
        bmin[k] -= pad;
        bmax[k] += pad;
        ext[k] = bmax[k] - bmin[k];
    }
    const float vox = std::fmax(ext[0], std::fmax(ext[1], ext[2])) / (float)voxels_per_axis;
    if (!(vox > 0.0f)) return fail(MPM_INVALID_ARG, "degenerate mesh");
    int n[3];
    for (int k = 0; k < 3; ++k) n[k] = std::min((int)(ext[k] / vox) + 2, 256);
    desc->nx = n[0]; desc->ny = n[1]; desc->nz = n[2];
    for (int k = 0; k < 3; ++k) desc->origin[k] = bmin[k];
    desc->voxel = vox;
    desc->angle = 0.0f;
    desc->values = values;
    if (!values) return MPM_OK;

    // triangle normals: the mesh's, or (b - a) x (c - a) normalised
    std::vector<float> nrm(3 * (size_t)n_tris);
    for (int t = 0; t < n_tris; ++t) {
        if (normals) {
            for (int k = 0; k < 3; ++k) nrm[3 * t + k] = normals[3 * t + k];
            continue;
        }
        const float* a = verts + 3 * tris[3 * t];
        const float* b = verts + 3 * tris[3 * t + 1];
        const float* c = verts + 3 * tris[3 * t + 2];
        const float u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        const float x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
        const float l = std::sqrt(x * x + y * y + z * z);
        nrm[3 * t] = l > 0.0f ? x / l : 0.0f;
        nrm[3 * t + 1] = l > 0.0f ? y / l : 0.0f;
        nrm[3 * t + 2] = l > 0.0f ? z / l : 0.0f;
    }
    const int64_t total = (int64_t)n[0] * n[1] * n[2];
    SdfGeom G{bmin[0], bmin[1], bmin[2], vox, 1.0f / vox, n[0], n[1], n[2]};

    float *d_v = nullptr, *d_n = nullptr, *d_g = nullptr;
    int* d_t = nullptr;
    cudaError_t e = cudaMalloc(&d_v, sizeof(float) * 3 * (size_t)n_verts);
    if (e == cudaSuccess) e = cudaMalloc(&d_n, sizeof(float) * 3 * (size_t)n_tris);
    if (e == cudaSuccess) e = cudaMalloc(&d_t, sizeof(int) * 3 * (size_t)n_tris);
    if (e == cudaSuccess) e = cudaMalloc(&d_g, sizeof(float) * (size_t)total);
    if (e == cudaSuccess) e = cudaMemcpy(d_v, verts, sizeof(float) * 3 * (size_t)n_verts, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_n, nrm.data(), sizeof(float) * 3 * (size_t)n_tris, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_t, tris, sizeof(int) * 3 * (size_t)n_tris, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
        k_sdf_fill<<<blocks, 256>>>(reinterpret_cast<unsigned*>(d_g), total);
        k_sdf_scatter<<<std::min(n_tris, 148 * 32), 128>>>(d_v, d_t, n_tris, G, reinterpret_cast<unsigned*>(d_g));
        k_sdf_sign<<<blocks, 256>>>(d_v, d_t, d_n, n_tris, G, d_g);
        launch_counter() += 3;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(values, d_g, sizeof(float) * (size_t)total, cudaMemcpyDeviceToHost);
    cudaFree(d_v);
    cudaFree(d_n);
    cudaFree(d_t);
    cudaFree(d_g);
    if (e != cudaSuccess) return fail(MPM_CUDA_ERROR, cudaGetErrorString(e));

    // three in-place passes give a voxel no triangle box reached its nearest
    // known neighbour's |distance| + half a voxel (:494-524), then the rest a
    // large distance (:526-531)
    const int nx = n[0], ny = n[1], nz = n[2];
    float* g = values;
    for (int pass = 0; pass < 3; ++pass)
        for (int iz = 1; iz < nz - 1; ++iz)
            for (int iy = 1; iy < ny - 1; ++iy)
                for (int ix = 1; ix < nx - 1; ++ix) {
                    const int64_t idx = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
                    if (g[idx] < FLT_MAX) continue;
                    float nd = FLT_MAX;
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                if (!dx && !dy && !dz) continue;
                                nd = std::fmin(nd, std::fabs(g[(ix + dx) + (int64_t)nx * ((iy + dy) + (int64_t)ny * (iz + dz))]));
                            }
                    if (nd < FLT_MAX) g[idx] = nd + vox * 0.5f;
                }
    const int dmax = std::max(nx, std::max(ny, nz));
    for (int64_t i = 0; i < total; ++i)
        if (g[i] >= FLT_MAX) g[i] = vox * (float)dmax;
    return MPM_OK;
}
