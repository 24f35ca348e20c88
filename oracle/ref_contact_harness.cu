// ref_contact_harness.cu -- runs the REFERENCE's own SDF contact kernel,
// unmodified, on a voxel SDF given by the caller.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's src/ContactSolver.cu (built from its sources where they lie)
// and ref_link_stubs.cu into oracle/_ref/libmpm_ref.so.  The texture is set up
// as ToolSDF::createTexture does (src/ToolSDF.cu:534-567): float texels,
// trilinear filtering, clamp addressing, unnormalised coordinates.
#include "ContactSolver.cuh"

#include <cstdint>
#include <cstdio>
#include <vector>

#include "mpm_oracle.h"

namespace {

char g_contact_err[256] = {0};

int fail(const char* what, cudaError_t e) {
    snprintf(g_contact_err, sizeof(g_contact_err), "%s: %s", what, cudaGetErrorString(e));
    return -1;
}

// The voxel grid as a 3D texture; owns the array and the texture object.
struct SdfTexture {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    ~SdfTexture() {
        if (tex) cudaDestroyTextureObject(tex);
        if (arr) cudaFreeArray(arr);
    }
    cudaError_t create(const orc_sdf_grid* g) {
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
        cudaExtent ext = make_cudaExtent(g->nx, g->ny, g->nz);
        cudaError_t e = cudaMalloc3DArray(&arr, &ch, ext);
        if (e != cudaSuccess) return e;
        cudaMemcpy3DParms cp = {};
        cp.srcPtr = make_cudaPitchedPtr((void*)g->v, g->nx * sizeof(float), g->nx, g->ny);
        cp.dstArray = arr;
        cp.extent = ext;
        cp.kind = cudaMemcpyHostToDevice;
        e = cudaMemcpy3D(&cp);
        if (e != cudaSuccess) return e;
        cudaResourceDesc rd = {};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td = {};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        return cudaCreateTextureObject(&tex, &rd, &td, nullptr);
    }
};

__global__ void k_tex_probe(cudaTextureObject_t tex, const float* xyz, int n, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex3D<float>(tex, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}

}  // namespace

extern "C" {

const char* ref_contact_last_error(void) { return g_contact_err; }

// Texture fetches at n points (voxel coordinates, xyz interleaved).
int ref_tex_probe(const orc_sdf_grid* g, const float* xyz, int n, float* out) {
    SdfTexture t;
    cudaError_t e = t.create(g);
    if (e != cudaSuccess) return fail("texture", e);
    float *d_xyz = nullptr, *d_out = nullptr;
    e = cudaMalloc(&d_xyz, sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(float) * (size_t)(n > 0 ? n : 1));
    if (e == cudaSuccess) e = cudaMemcpy(d_xyz, xyz, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) {
        k_tex_probe<<<(n + 255) / 256, 256>>>(t.tex, d_xyz, n, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
    if (d_xyz) cudaFree(d_xyz);
    if (d_out) cudaFree(d_out);
    return e == cudaSuccess ? 0 : fail("probe", e);
}

// One launch of xpbdContactSDFKernel (src/ContactSolver.cu:797-923) over the
// particles of s (positions, velocities and temperatures updated in place).
int ref_contact_sdf(const orc_sdf_grid* g, const orc_contact_sdf_args* a, orc_state* s, int64_t* count,
                    double* heat, double* force) {
    using namespace edgepredict;
    const int n = s->n;
    std::vector<MPMParticle> h((size_t)n);
    for (int i = 0; i < n; ++i) {
        MPMParticle& q = h[i];
        q.x = s->x[i]; q.y = s->y[i]; q.z = s->z[i];
        q.vx = s->vx[i]; q.vy = s->vy[i]; q.vz = s->vz[i];
        q.mass = s->mass[i]; q.volume = s->vol[i]; q.density = s->mass[i] / s->vol[i];
        q.temperature = s->T[i];
        q.status = static_cast<ParticleStatus>(s->status[i]);
    }
    SdfTexture t;
    cudaError_t e = t.create(g);
    if (e != cudaSuccess) return fail("texture", e);
    MPMParticle* d = nullptr;
    int* d_cnt = nullptr;
    double* d_sum = nullptr;
    e = cudaMalloc(&d, sizeof(MPMParticle) * (size_t)(n > 0 ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_cnt, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_sum, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(d_cnt, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_sum, 0, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), sizeof(MPMParticle) * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) {
        xpbdContactSDFKernel<<<(n + 255) / 256, 256>>>(
            d, n, t.tex, make_float3(g->ox, g->oy, g->oz), g->voxel, make_int3(g->nx, g->ny, g->nz), a->cx, a->cy,
            a->cz, a->cos_a, a->sin_a, a->radius, a->friction, a->heat_partition, a->dt, a->cp, a->rho_phys, a->Tm,
            0.0, false, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0, d_cnt, d_sum, d_sum + 1);
        e = cudaGetLastError();
    }
    int cnt = 0;
    double sums[2] = {0.0, 0.0};
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, sizeof(MPMParticle) * (size_t)n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&cnt, d_cnt, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sums, d_sum, 2 * sizeof(double), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (d_cnt) cudaFree(d_cnt);
    if (d_sum) cudaFree(d_sum);
    if (e != cudaSuccess) return fail("contact", e);
    for (int i = 0; i < n; ++i) {
        const MPMParticle& q = h[i];
        s->x[i] = q.x; s->y[i] = q.y; s->z[i] = q.z;
        s->vx[i] = q.vx; s->vy[i] = q.vy; s->vz[i] = q.vz;
        s->T[i] = q.temperature;
    }
    *count = cnt;
    *heat = sums[0];
    *force = sums[1];
    return 0;
}

// One launch of xpbdContactSDFKernel on n MPMParticle records already in
// device memory (d_particles), updated in place: the reference's contact
// pass run on an array another solver handed out (ContactSolver::
// resolveContacts launches it on MPMSolver::getDeviceParticles(),
// src/ContactSolver.cu:1130-1147).
int ref_contact_sdf_device(const orc_sdf_grid* g, const orc_contact_sdf_args* a, void* d_particles, int n,
                           int64_t* count, double* heat, double* force) {
    using namespace edgepredict;
    SdfTexture t;
    cudaError_t e = t.create(g);
    if (e != cudaSuccess) return fail("texture", e);
    int* d_cnt = nullptr;
    double* d_sum = nullptr;
    e = cudaMalloc(&d_cnt, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_sum, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(d_cnt, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_sum, 0, 2 * sizeof(double));
    if (e == cudaSuccess && n > 0) {
        xpbdContactSDFKernel<<<(n + 255) / 256, 256>>>(
            static_cast<MPMParticle*>(d_particles), n, t.tex, make_float3(g->ox, g->oy, g->oz), g->voxel,
            make_int3(g->nx, g->ny, g->nz), a->cx, a->cy, a->cz, a->cos_a, a->sin_a, a->radius, a->friction,
            a->heat_partition, a->dt, a->cp, a->rho_phys, a->Tm, 0.0, false, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0,
            d_cnt, d_sum, d_sum + 1);
        e = cudaGetLastError();
    }
    int cnt = 0;
    double sums[2] = {0.0, 0.0};
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&cnt, d_cnt, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sums, d_sum, 2 * sizeof(double), cudaMemcpyDeviceToHost);
    if (d_cnt) cudaFree(d_cnt);
    if (d_sum) cudaFree(d_sum);
    if (e != cudaSuccess) return fail("contact (device array)", e);
    *count = cnt;
    *heat = sums[0];
    *force = sums[1];
    return 0;
}

}  // extern "C"
