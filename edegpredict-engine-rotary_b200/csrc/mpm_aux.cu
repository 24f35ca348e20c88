// mpm_aux.cu -- re-binning (counting sort by 4^3-cell bin), scans, upload and
// download conversions, the reference-layout AoS export, FP64 metric
// reductions, tool rasterisation, the seeded workpiece generator and the heat
// conduction diffusion step.
#include <cuda.h>
#include <algorithm>
#include <cuda_runtime.h>

#include "mpm_device.cuh"
#include "mpm_internal.h"

namespace mpmb {

namespace {

constexpr int kT = 256;

inline int nblk(int64_t n, int t = kT) {
    int64_t b = (n + t - 1) / t;
    if (b < 1) b = 1;
    if (b > (1 << 20)) b = (1 << 20);
    return (int)b;
}

template <typename R> __device__ __forceinline__ R ld_user(const void* p, int elem, int64_t i) {
    return elem == 8 ? (R)((const double*)p)[i] : (R)((const float*)p)[i];
}
__device__ __forceinline__ double ld_userd(const void* p, int elem, int64_t i) {
    return elem == 8 ? ((const double*)p)[i] : (double)((const float*)p)[i];
}
__device__ __forceinline__ void st_user(void* p, int elem, int64_t i, double v) {
    if (elem == 8) ((double*)p)[i] = v; else ((float*)p)[i] = (float)v;
}

template <typename R> __device__ __forceinline__ int find_inst(const Inst<R>* insts, int n_inst, int64_t pi) {
    int lo = 0, hi = n_inst - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (insts[mid].pbase <= pi) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace

// ------------------------------------------------------------------ scan

// Three-phase exclusive scan: per-CTA scan of 1024 elements with block sums,
// a single-CTA scan of the block sums, then the offsets are added.
__global__ void k_scan_local(const int32_t* in, int32_t* out, int32_t* sums, int64_t n) {
    __shared__ int32_t s[1024];
    const int64_t base = (int64_t)blockIdx.x * 1024;
    const int t = threadIdx.x;  // 512 threads, 2 elements each
    int64_t i0 = base + 2 * t, i1 = i0 + 1;
    int32_t a = i0 < n ? in[i0] : 0, b = i1 < n ? in[i1] : 0;
    s[2 * t] = a;
    s[2 * t + 1] = b;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // Hillis-Steele on the 1024 values
        int32_t x0 = 0, x1 = 0;
        int j0 = 2 * t, j1 = 2 * t + 1;
        if (j0 >= off) x0 = s[j0 - off];
        if (j1 >= off) x1 = s[j1 - off];
        __syncthreads();
        s[j0] += x0;
        s[j1] += x1;
        __syncthreads();
    }
    if (i0 < n) out[i0] = s[2 * t] - a;
    if (i1 < n) out[i1] = s[2 * t + 1] - b;
    if (t == 511) sums[blockIdx.x] = s[1023];
}

__global__ void k_scan_sums(int32_t* sums, int nb) {
    __shared__ int32_t carry;
    __shared__ int32_t s[1024];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int t = threadIdx.x;
        int32_t v = (base + t < nb) ? sums[base + t] : 0;
        s[t] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            int32_t x = t >= off ? s[t - off] : 0;
            __syncthreads();
            s[t] += x;
            __syncthreads();
        }
        if (base + t < nb) sums[base + t] = carry + s[t] - v;
        __syncthreads();
        if (t == 1023) carry += s[1023];
        __syncthreads();
    }
}

__global__ void k_scan_add(int32_t* out, const int32_t* sums, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / 1024];
}

int64_t scan_tmp_size(int64_t n) { return (n + 1023) / 1024 + 1; }

void exclusive_scan(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t st) {
    if (n <= 0) return;
    const int nb = (int)((n + 1023) / 1024);
    k_scan_local<<<nb, 512, 0, st>>>(in, out, tmp, n);
    k_scan_sums<<<1, 1024, 0, st>>>(tmp, nb);
    k_scan_add<<<(int)((n + 255) / 256), 256, 0, st>>>(out, tmp, n);
    launch_counter() += 3;
}

__global__ void k_fill_i32(int32_t* p, int32_t v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
void fill_i32(int32_t* p, int32_t v, int64_t n, cudaStream_t st) {
    if (n > 0) {
        k_fill_i32<<<nblk(n), kT, 0, st>>>(p, v, n);
        ++launch_counter();
    }
}

// ------------------------------------------------------------------ work list

// One work item per non-empty bin.  A bin's keys are contiguous (bin*64 +
// cell), so its particles are [offset[first], offset[first + 64]).
__global__ void k_work_flags(const int32_t* offset, const int32_t* bin_key, int64_t nbins_total, int32_t* flag) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbins_total) {
        const int32_t fk = bin_key[b];
        flag[b] = (offset[fk + kCellsPerBin] - offset[fk]) > 0 ? 1 : 0;
    }
}

__global__ void k_work_emit(const int32_t* offset, const int32_t* bin_key, const int32_t* bin_inst,
                            const int32_t* bin_local, const int64_t* inst_pbase, const int32_t* flag,
                            const int32_t* flag_scan, int64_t nbins_total, Work* work, int* n_work) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbins_total && flag[b]) {
        const int32_t fk = bin_key[b];
        const int i = bin_inst[b];
        Work w;
        w.inst = i;
        w.bin = bin_local[b];
        w.start = (int)(offset[fk] - inst_pbase[i]);
        w.count = offset[fk + kCellsPerBin] - offset[fk];
        work[flag_scan[b]] = w;
    }
    if (b == nbins_total - 1) *n_work = flag_scan[b] + flag[b];
}

void build_work(const int32_t* offset, const int32_t* bin_key, const int32_t* bin_inst, const int32_t* bin_local,
                const int64_t* inst_pbase, int64_t nbins_total, int32_t* flag, int32_t* flag_scan, int32_t* tmp,
                Work* work, int* n_work, cudaStream_t st) {
    k_work_flags<<<nblk(nbins_total), kT, 0, st>>>(offset, bin_key, nbins_total, flag);
    exclusive_scan(flag, flag_scan, nbins_total, tmp, st);
    k_work_emit<<<nblk(nbins_total), kT, 0, st>>>(offset, bin_key, bin_inst, bin_local, inst_pbase, flag, flag_scan,
                                                  nbins_total, work, n_work);
    launch_counter() += 2;
}

// ------------------------------------------------------------------ re-bin

// Key of every particle: instance key base + bin*64 + cell within the bin,
// where the cell is the stencil base node; INACTIVE particles take the
// instance's sentinel key (after all bins).  rank = arrival order in the key.
// An instance that keeps its layout at this re-bin (keep_all, or not due at
// point kpt of its re-bin phase) takes the keys its particles were placed
// under (skey), so that the move leaves every particle of it in its slot.
template <typename R>
__global__ void k_bin_count(const Inst<R>* insts, int n_inst, PState<R> ps, const int32_t* key_base, bool initial,
                            const double* pos_scratch, int32_t* key, int32_t* rank, int32_t* count, int32_t* newbin,
                            int64_t np, int kpt, int sort_every, bool keep_all) {
    const int64_t pi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= np) return;
    const int ii = find_inst(insts, n_inst, pi);
    const Inst<R>& P = insts[ii];
    if (pi >= P.pbase + P.np) return;  // unused slot of the instance
    const bool fresh = initial && P.fresh;
    const bool due = kpt < 0 || (kpt >= P.rebin_first && (kpt - P.rebin_first) % sort_every == 0);
    const int32_t sk = ps.skey[pi];
    if (!fresh && !P.rebin_now && (keep_all || !due) && sk >= 0) {
        const int32_t kk = key_base[ii] + sk;
        key[pi] = kk;
        newbin[pi] = sk < P.nbins * kCellsPerBin ? sk / kCellsPerBin : ps.bin[pi];
        rank[pi] = atomicAdd(&count[kk], 1);
        return;
    }
    int b[3];
    if (fresh) {
        for (int a = 0; a < 3; ++a) {
            const double f = floor(pos_scratch[3 * pi + a] - 0.5);
            b[a] = f < -1e9 ? -1000000000 : (f > 1e9 ? 1000000000 : (int)f);
        }
    } else {
        const int bn = ps.bin[pi];
        const int ob[3] = {bn % P.nbx, (bn / P.nbx) % P.nby, bn / (P.nbx * P.nby)};
        const V4<R> a0 = ps.A[0][pi];
        const R xl[3] = {a0.x, a0.y, a0.z};
        for (int a = 0; a < 3; ++a) {
            const R f = floor(xl[a] - R(0.5));
            const int fi = f < R(-1e8) ? -100000000 : (f > R(1e8) ? 100000000 : (int)f);
            b[a] = ob[a] * kBin + fi;
        }
    }
    const int nb[3] = {P.nbx, P.nby, P.nbz};
    int B[3], L[3];
    for (int a = 0; a < 3; ++a) {
        const int q = b[a] >= 0 ? b[a] / kBin : -1;
        B[a] = q < 0 ? 0 : (q >= nb[a] ? nb[a] - 1 : q);
        const int l = b[a] - B[a] * kBin;
        L[a] = l < 0 ? 0 : (l >= kBin ? kBin - 1 : l);
    }
    const int bin = B[0] + P.nbx * (B[1] + P.nby * B[2]);
    const int cell = L[0] + kBin * (L[1] + kBin * L[2]);
    const int32_t kk = key_base[ii] + ((ps.status[pi] == ST_INACTIVE) ? P.nbins * kCellsPerBin
                                                                       : bin * kCellsPerBin + cell);
    key[pi] = kk;
    newbin[pi] = bin;
    rank[pi] = atomicAdd(&count[kk], 1);
}

// Position in its bin of the particle of cell c (0..63) with rank r among
// that cell's particles; cs points at the bin's 65 cell offsets in the new
// layout (cell q holds cs[q+1] - cs[q] particles, n = cs[64] - cs[0]).
// The bin is a table of 64 columns, column c for cell c: with R = n / 64
// full rows, particle (c, r < R) sits at r*64 + c.  The particles of cells
// holding more than R (the overflow, in cell then rank order) fill first
// the holes the smaller cells leave in the full rows (row m..R-1 of a cell
// with m < R particles, in cell then row order), then the tail [64R, n).
// A warp of the step kernel takes 32 consecutive positions: mostly 32
// distinct cells of one half of the bin (x, y and two z layers), which is
// what makes its velocity-tile gathers and node-tile adds conflict-free,
// and a 256-particle pass holds at most four particles of a cell outside
// the overflow.
__device__ __forceinline__ int64_t column_slot(const int32_t* __restrict__ cs, int c, int r) {
    const int n = cs[kCellsPerBin] - cs[0];
    const int R = n / kCellsPerBin;
    if (r < R) return (int64_t)r * kCellsPerBin + c;
    int k = r - R;   // k-th overflow particle of the bin
    for (int q = 0; q < c; ++q) {
        const int m = cs[q + 1] - cs[q];
        if (m > R) k += m - R;
    }
    for (int q = 0; q < kCellsPerBin; ++q) {
        const int m = cs[q + 1] - cs[q];
        const int holes = m < R ? R - m : 0;
        if (k < holes) return (int64_t)(m + k) * kCellsPerBin + q;
        k -= holes;
    }
    return (int64_t)R * kCellsPerBin + k;
}

// Destination slot of source slot pi in the new layout (-1: an unused slot).
template <typename R>
__device__ __forceinline__ int64_t bin_dest(const Inst<R>& P, int ii, int64_t pi, const int32_t* key,
                                            const int32_t* rank, const int32_t* offset, const int32_t* key_base,
                                            const int32_t* newbin) {
    if (pi >= P.pbase + P.np) return -1;
    const int32_t kk = key[pi];
    if (kk - key_base[ii] >= P.nbins * kCellsPerBin) return offset[kk] + rank[pi];  // INACTIVE: after the bins
    const int32_t fk = key_base[ii] + newbin[pi] * kCellsPerBin;
    return offset[fk] + column_slot(offset + fk, kk - fk, rank[pi]);
}

// The re-bin's move, in two launches so that the writes are coalesced: the
// first records for every destination slot its source (perm[d] = pi), the
// second runs one thread per destination slot and copies the particle from
// its source, which lies in the same bin's window of the old layout (read
// through L2) -- a scatter by source slot wrote every 16-, 4- and 1-byte field
// to a permuted slot and moved about twice the bytes through DRAM.
template <typename R>
// perm[d] = the source slot of destination slot d, perm[np + d] = that
// source's upload position (the order k_bin_order sorts by, read here where
// it is coalesced).
__global__ void k_bin_perm(const Inst<R>* insts, int n_inst, const int32_t* key, const int32_t* rank,
                           const int32_t* offset, const int32_t* key_base, const int32_t* newbin,
                           const int32_t* orig, int32_t* perm, int64_t np) {
    const int64_t pi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= np) return;
    const int ii = find_inst(insts, n_inst, pi);
    const int64_t d = bin_dest(insts[ii], ii, pi, key, rank, offset, key_base, newbin);
    if (d >= 0) {
        perm[d] = (int32_t)pi;
        perm[np + d] = orig[pi];
    }
}

// The ranks of k_bin_count follow the atomics' arrival order.  One CTA per
// bin of the bin table puts each cell's particles in the order of their
// upload positions (orig): thread c takes the destinations of cell c (rank
// order) and hands them the cell's sources sorted by orig.  The layout -- and
// with it the order of every sum the step kernel forms -- then depends on the
// particles' positions and upload order alone, not on the thread schedule or
// the layout before (so re-binning a freshly binned state changes nothing).
// Cells of up to kOrderLocal particles sort in registers and local memory; a
// larger one (a cell packed several times over its particles per cell) takes
// a selection sort through global memory.
constexpr int kOrderLocal = 48;

__device__ __forceinline__ int64_t order_dest(const int32_t* cs, int c, int r, int64_t b0) {
    return b0 + column_slot(cs, c, r);
}

__global__ void __launch_bounds__(kCellsPerBin) k_bin_order(const int32_t* __restrict__ bin_key,
                                                            const int32_t* __restrict__ offset, int32_t* perm,
                                                            int64_t np) {
    const int32_t* __restrict__ okey = perm + np;   // upload position of each destination's source
    __shared__ int32_t cs[kCellsPerBin + 1];
    const int32_t fk = bin_key[blockIdx.x];
    const int c = threadIdx.x;
    cs[c] = offset[fk + c];
    if (c == 0) cs[kCellsPerBin] = offset[fk + kCellsPerBin];
    __syncthreads();
    const int m = cs[c + 1] - cs[c];
    if (m <= 1) return;
    const int64_t b0 = cs[0];
    if (m <= kOrderLocal) {
        int32_t src[kOrderLocal], key[kOrderLocal];
        int64_t dst[kOrderLocal];
        for (int r = 0; r < m; ++r) {
            dst[r] = order_dest(cs, c, r, b0);
            src[r] = perm[dst[r]];
            key[r] = okey[dst[r]];
        }
        // insertion sort by orig (distinct within an instance)
        for (int r = 1; r < m; ++r) {
            const int32_t v = src[r], k = key[r];
            int q = r - 1;
            while (q >= 0 && key[q] > k) {
                src[q + 1] = src[q];
                key[q + 1] = key[q];
                --q;
            }
            src[q + 1] = v;
            key[q + 1] = k;
        }
        for (int r = 0; r < m; ++r) perm[dst[r]] = src[r];
    } else {
        // selection sort in place: rank r takes the smallest orig among ranks r..m-1
        for (int r = 0; r < m - 1; ++r) {
            const int64_t dr = order_dest(cs, c, r, b0);
            int64_t best = dr;
            int32_t bv = perm[dr], bk = okey[dr];
            for (int q = r + 1; q < m; ++q) {
                const int64_t dq = order_dest(cs, c, q, b0);
                const int32_t v = perm[dq], k = okey[dq];
                if (k < bk) { bv = v; bk = k; best = dq; }
            }
            if (best != dr) {
                perm[best] = perm[dr];
                perm[np + best] = okey[dr];
                perm[dr] = bv;
                perm[np + dr] = bk;
            }
        }
    }
}

template <typename R>
__global__ void k_bin_gather(PState<R> src, PState<R> dst, const Inst<R>* insts, int n_inst, const int32_t* key,
                             const int32_t* key_base, const int32_t* newbin, const int32_t* perm, bool initial,
                             const double* pos_scratch, bool has_K, int64_t np) {
    const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= np) return;
    const int64_t pi = perm[d];
    if (pi < 0) return;
    const int ii = find_inst(insts, n_inst, pi);
    const Inst<R>& P = insts[ii];
    const bool fresh = initial && P.fresh;
    const int nbn = newbin[pi];
    const int nbv[3] = {nbn % P.nbx, (nbn / P.nbx) % P.nby, nbn / (P.nbx * P.nby)};
    V4<R> a0 = src.A[0][pi];
    if (fresh) {
        const double p[3] = {pos_scratch[3 * pi + 0] - (double)(nbv[0] * kBin),
                             pos_scratch[3 * pi + 1] - (double)(nbv[1] * kBin),
                             pos_scratch[3 * pi + 2] - (double)(nbv[2] * kBin)};
        a0.x = (R)p[0];
        a0.y = (R)p[1];
        a0.z = (R)p[2];
        if (dst.X) dst.X[d] = mk4<R>((R)(p[0] - (double)a0.x), (R)(p[1] - (double)a0.y), (R)(p[2] - (double)a0.z), R(0));
    } else {
        if (dst.X && src.X) dst.X[d] = src.X[pi];
        const int ob = src.bin[pi];
        const int obv[3] = {ob % P.nbx, (ob / P.nbx) % P.nby, ob / (P.nbx * P.nby)};
        if (ob != nbn) {
            a0.x += (R)((obv[0] - nbv[0]) * kBin);
            a0.y += (R)((obv[1] - nbv[1]) * kBin);
            a0.z += (R)((obv[2] - nbv[2]) * kBin);
        }
    }
    dst.A[0][d] = a0;
    dst.skey[d] = key[pi] - key_base[ii];
#pragma unroll
    for (int q = 1; q < 6; ++q) dst.A[q][d] = src.A[q][pi];
#pragma unroll
    for (int q = 0; q < 4; ++q) dst.B[q][d] = src.B[q][pi];
    dst.S[0][d] = src.S[0][pi];
    dst.S[1][d] = src.S[1][pi];
    if (has_K) {
        dst.K[0][d] = src.K[0][pi];
        dst.K[1][d] = src.K[1][pi];
    }
    dst.sres[d] = src.sres[pi];
    dst.status[d] = src.status[pi];
    dst.asb[d] = src.asb[pi];
    dst.id[d] = src.id[pi];
    dst.orig[d] = src.orig[pi];
    dst.bin[d] = nbn;
}

// Unused slots of each instance are counted into the instance's last key so
// that the global scan keeps every instance at its own slot range.
template <typename R>
__global__ void k_pad_counts(const Inst<R>* insts, int n_inst, const int32_t* key_base, int32_t* count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_inst) return;
    count[key_base[i] + insts[i].nbins * kCellsPerBin + 1] = (int32_t)(insts[i].pcap - insts[i].np);
}

template <typename R>
void launch_pad_counts(const Inst<R>* insts, int n_inst, const int32_t* key_base, int32_t* count, cudaStream_t st) {
    k_pad_counts<R><<<(n_inst + 127) / 128, 128, 0, st>>>(insts, n_inst, key_base, count);
    ++launch_counter();
}
template void launch_pad_counts<float>(const Inst<float>*, int, const int32_t*, int32_t*, cudaStream_t);
template void launch_pad_counts<double>(const Inst<double>*, int, const int32_t*, int32_t*, cudaStream_t);

// ------------------------------------------------------------------ raster

// rasterizeToolKernel (reference src/MPMSolver.cu:444-473): each tool sample
// marks the 2x2x2 nodes from round((x - min)/dx).
// The raster tool of instance i at step k of the current call, restating
// rasterizeToolKernel (src/MPMSolver.cu:444-473): each point marks the 2x2x2
// grid nodes from g = round((p - origin) / dx).  The pose comes from the
// instance record (time t0 + k dt, as the step kernel computes it), so the
// launch has the same arguments in every call and replays from a CUDA graph.
// Samples: p = pose + offset, mark 1.  FEM nodes: p = start + a (end -
// start) with the blend weight a of this step (fused multiply-add, as the
// reference's compiled blend kernel, src/MPMSolver.cu:494-504, rounds it), or
// end when there is no blend; the mark is the node's index + 1, the highest
// winning, so a marked grid node's velocity is one node's, whatever the
// thread order.
template <typename R>
__global__ void k_raster(const Inst<R>* __restrict__ insts, int i, int k) {
    const Inst<R>& P = insts[i];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double p[3];
    int32_t mark;
    if (P.tn_end) {
        if (t >= P.tn_n) return;
        const unsigned char* e = P.tn_end + (int64_t)t * P.tn_stride;
        for (int a = 0; a < 3; ++a) p[a] = *reinterpret_cast<const double*>(e + P.tn_off[a]);
        if (P.tn_start) {
            const unsigned char* s0 = P.tn_start + (int64_t)t * P.tn_stride;
            const double al = P.tn_a0 + (double)(P.step0 + k - P.tn_step0) * P.tn_da;
            for (int a = 0; a < 3; ++a) {
                const double q0 = *reinterpret_cast<const double*>(s0 + P.tn_off[a]);
                p[a] = fma(al, p[a] - q0, q0);
            }
        }
        mark = t + 1;
    } else {
        if (t >= P.n_samples) return;
        const double tk = da(P.t0, dm((double)k, P.dt));
        for (int a = 0; a < 3; ++a)
            p[a] = da(da(P.tool_p0[a], dm(P.tool_v[a], ds(tk, P.tool_t0))), P.samples[a * P.n_samples + t]);
        mark = 1;
    }
    const double inv_dx = 1.0 / P.dx;
    const int gx = (int)round(ds(p[0], P.ox) * inv_dx);
    const int gy = (int)round(ds(p[1], P.oy) * inv_dx);
    const int gz = (int)round(ds(p[2], P.oz) * inv_dx);
    for (int a = 0; a < 2; ++a) {
        const int cx = gx + a;
        if (cx < 0 || cx >= P.nx) continue;
        for (int b = 0; b < 2; ++b) {
            const int cy = gy + b;
            if (cy < 0 || cy >= P.ny) continue;
            for (int c = 0; c < 2; ++c) {
                const int cz = gz + c;
                if (cz < 0 || cz >= P.nz) continue;
                int32_t* m = &P.tool_mask[cx + (int64_t)P.nx * (cy + (int64_t)P.ny * cz)];
                if (mark == 1) *m = 1;
                else atomicMax(m, mark);
            }
        }
    }
}

// ------------------------------------------------------------------ upload

template <typename R>
__global__ void k_import(DevSoA in, int64_t n, double ox, double oy, double oz, double inv_dx, double Tamb, PState<R> ps,
                         int64_t pbase, double* pos_scratch) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int e = in.elem;
    const int64_t d = pbase + i;
    const double x = ld_userd(in.x, e, i), y = ld_userd(in.y, e, i), z = ld_userd(in.z, e, i);
    pos_scratch[3 * d + 0] = (x - ox) * inv_dx;
    pos_scratch[3 * d + 1] = (y - oy) * inv_dx;
    pos_scratch[3 * d + 2] = (z - oz) * inv_dx;
    const R eps = in.eps ? ld_user<R>(in.eps, e, i) : R(0);
    R H[9], Hp[9], C[9];
    for (int q = 0; q < 9; ++q) {
        const double id = (q % 4 == 0) ? 1.0 : 0.0;
        H[q] = in.F ? (R)(ld_userd(in.F, e, 9 * i + q) - id) : R(0);
        Hp[q] = in.Fp ? (R)(ld_userd(in.Fp, e, 9 * i + q) - id) : R(0);
        C[q] = in.C ? ld_user<R>(in.C, e, 9 * i + q) : R(0);
    }
    const R dT = in.T ? (R)(ld_userd(in.T, e, i) - Tamb) : R(0);
    const R D = in.D ? ld_user<R>(in.D, e, i) : R(0);
    ps.A[0][d] = mk4<R>(R(0), R(0), R(0), eps);
    ps.A[1][d] = mk4<R>(H[0], H[1], H[2], H[3]);
    ps.A[2][d] = mk4<R>(H[4], H[5], H[6], H[7]);
    ps.A[3][d] = mk4<R>(H[8], Hp[8], dT, D);
    ps.A[4][d] = mk4<R>(Hp[0], Hp[1], Hp[2], Hp[3]);
    ps.A[5][d] = mk4<R>(Hp[4], Hp[5], Hp[6], Hp[7]);
    const R vx = in.vx ? ld_user<R>(in.vx, e, i) : R(0), vy = in.vy ? ld_user<R>(in.vy, e, i) : R(0),
            vz = in.vz ? ld_user<R>(in.vz, e, i) : R(0);
    const R ed = in.edot ? ld_user<R>(in.edot, e, i) : R(0);
    ps.B[0][d] = mk4<R>(vx, vy, vz, ed);
    ps.B[1][d] = mk4<R>(C[0], C[1], C[2], C[3]);
    ps.B[2][d] = mk4<R>(C[4], C[5], C[6], C[7]);
    ps.B[3][d] = mk4<R>(C[8], R(0), R(0), R(0));
    R s[6] = {0, 0, 0, 0, 0, 0}, k[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < 6; ++q) {
        if (in.stress) s[q] = ld_user<R>(in.stress, e, 6 * i + q);
        if (in.bs) k[q] = ld_user<R>(in.bs, e, 6 * i + q);
    }
    ps.S[0][d] = mk4<R>(s[0], s[1], s[2], s[3]);
    ps.S[1][d] = mk4<R>(s[4], s[5], R(0), R(0));
    if (ps.K[0]) {
        ps.K[0][d] = mk4<R>(k[0], k[1], k[2], k[3]);
        ps.K[1][d] = mk4<R>(k[4], k[5], R(0), R(0));
    }
    ps.sres[d] = in.sres ? ld_user<R>(in.sres, e, i) : R(0);
    ps.status[d] = in.status ? (uint8_t)in.status[i] : (uint8_t)ST_ACTIVE;
    ps.asb[d] = 0;
    ps.id[d] = in.id ? in.id[i] : (int32_t)i;
    ps.orig[d] = (int32_t)i;
    ps.bin[d] = 0;
    ps.skey[d] = -1;
}

// ------------------------------------------------------------------ generator

// Seeded box workpiece: candidate (cell, k) gets Philox4x32-10 uniforms keyed
// by (seed_lo, seed_hi) with counter (cell index in the box, k, instance, 0),
// and sits at a jittered point of its own stratum of the cell (the reference
// fills the box on a regular lattice, src/MPMSolver.cu:1311-1315; the jitter
// is the seeded part).  For ppc <= 8 the strata are the cell's octants, in
// the fixed order kOctant, whose prefixes of even length take each half of
// every axis equally often; with the same octants in every cell, each
// interior cell's stencil base (the node below x - 1/2, which collects the
// upper octants of its cell and the lower ones of the next) holds exactly ppc
// particles.  For ppc > 8 the strata are sub-cells of an n^3 grid, n the
// smallest even number with n^3 >= ppc (even, so that the same holds),
// candidate k taking sub-cell s = 37 k mod n^3 (spread over the cell).
// Offsets in cells: octant o, axis a: 0.5 bit_a(o) + 0.5 u_a (exact);
// sub-cell s: (s_a + u_a) / n.
// keep = not inside the tool at t=0 (phi > 0 when a tool is given).
__constant__ int kOctant[8] = {0, 7, 3, 4, 5, 2, 6, 1};
__device__ __forceinline__ void gen_offset(int k, int ppc, const float u[4], double off[3]) {
    if (ppc <= 8) {
        const int o = kOctant[k & 7];
        for (int a = 0; a < 3; ++a) off[a] = 0.5 * (double)((o >> a) & 1) + 0.5 * (double)u[a];
    } else {
        int n = 4;
        while (n * n * n < ppc) n += 2;
        const int q = (int)((37ll * k) % (n * n * n));
        const int sa[3] = {q % n, (q / n) % n, q / (n * n)};
        for (int a = 0; a < 3; ++a) off[a] = ((double)sa[a] + (double)u[a]) / (double)n;
    }
}
template <typename R>
__global__ void k_gen_flags(Inst<R> P, int c0x, int c0y, int c0z, int wx, int wy, int wz, int ppc, uint32_t s0,
                            uint32_t s1, uint32_t inst, int tool_check, int32_t* flag, int64_t ncand) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncand) return;
    int keep = 1;
    if (tool_check) {
        const int64_t cell = c / ppc;
        const int k = (int)(c % ppc);
        const int ix = (int)(cell % wx), iy = (int)((cell / wx) % wy), iz = (int)(cell / ((int64_t)wx * wy));
        float u[4];
        philox_u4(s0, s1, (uint32_t)cell, (uint32_t)k, inst, 0u, u);
        double off[3];
        gen_offset(k, ppc, u, off);
        const double x = P.ox + ((double)(c0x + ix) + off[0]) * P.dx;
        const double z = P.oz + ((double)(c0z + iz) + off[2]) * P.dx;
        (void)iy;
        double nrm[3];
        if (tool_sdf(P, x, z, P.tool_p0[0], P.tool_p0[2], nrm) <= 0.0) keep = 0;
    }
    flag[c] = keep;
}

template <typename R>
__global__ void k_gen_write(Inst<R> P, int c0x, int c0y, int c0z, int wx, int wy, int wz, int ppc, uint32_t s0,
                            uint32_t s1, uint32_t inst, int fixed_layers, R dT0, const int32_t* flag,
                            const int32_t* idx, PState<R> ps, int64_t pbase, double* pos_scratch, int64_t ncand) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncand || !flag[c]) return;
    const int64_t cell = c / ppc;
    const int k = (int)(c % ppc);
    const int ix = (int)(cell % wx), iy = (int)((cell / wx) % wy), iz = (int)(cell / ((int64_t)wx * wy));
    float u[4];
    philox_u4(s0, s1, (uint32_t)cell, (uint32_t)k, inst, 0u, u);
    double off[3];
    gen_offset(k, ppc, u, off);
    const int64_t i = idx[c];
    const int64_t d = pbase + i;
    pos_scratch[3 * d + 0] = (double)(c0x + ix) + off[0];
    pos_scratch[3 * d + 1] = (double)(c0y + iy) + off[1];
    pos_scratch[3 * d + 2] = (double)(c0z + iz) + off[2];
    ps.A[0][d] = mk4<R>(R(0), R(0), R(0), R(0));
    ps.A[1][d] = mk4<R>(R(0), R(0), R(0), R(0));
    ps.A[2][d] = mk4<R>(R(0), R(0), R(0), R(0));
    ps.A[3][d] = mk4<R>(R(0), R(0), dT0, R(0));
    ps.A[4][d] = mk4<R>(R(0), R(0), R(0), R(0));
    ps.A[5][d] = mk4<R>(R(0), R(0), R(0), R(0));
    for (int q = 0; q < 4; ++q) ps.B[q][d] = mk4<R>(R(0), R(0), R(0), R(0));
    ps.S[0][d] = mk4<R>(R(0), R(0), R(0), R(0));
    ps.S[1][d] = mk4<R>(R(0), R(0), R(0), R(0));
    if (ps.K[0]) {
        ps.K[0][d] = mk4<R>(R(0), R(0), R(0), R(0));
        ps.K[1][d] = mk4<R>(R(0), R(0), R(0), R(0));
    }
    ps.sres[d] = R(0);
    ps.status[d] = (iz < fixed_layers) ? (uint8_t)ST_FIXED : (uint8_t)ST_ACTIVE;
    ps.asb[d] = 0;
    ps.id[d] = (int32_t)i;
    ps.orig[d] = (int32_t)i;
    ps.bin[d] = 0;
    ps.skey[d] = -1;
    (void)wz;
    (void)P;
}

// ------------------------------------------------------------------ download

// World position of slot pi: grid origin + (bin origin + xi) dx, with the
// low parts of xi where the state keeps them.
template <typename R>
__device__ __forceinline__ void world_pos(const Inst<R>& P, const PState<R>& ps, int64_t pi, const V4<R>& a0,
                                          double out[3]) {
    const int bin = ps.bin[pi];
    const int bx = bin % P.nbx, by = (bin / P.nbx) % P.nby, bz = bin / (P.nbx * P.nby);
    double lo[3] = {0.0, 0.0, 0.0};
    if (ps.X) {
        const V4<R> x = ps.X[pi];
        lo[0] = (double)x.x; lo[1] = (double)x.y; lo[2] = (double)x.z;
    }
    out[0] = P.ox + ((double)(bx * kBin) + ((double)a0.x + lo[0])) * P.dx;
    out[1] = P.oy + ((double)(by * kBin) + ((double)a0.y + lo[1])) * P.dx;
    out[2] = P.oz + ((double)(bz * kBin) + ((double)a0.z + lo[2])) * P.dx;
}

template <typename R>
__global__ void k_export(const Inst<R>* inst, PState<R> ps, int64_t pbase, int64_t n, double Tamb, DevSoAOut o) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const Inst<R>& P = *inst;
    const int64_t pi = pbase + s;
    const int64_t i = ps.orig[pi];
    const int e = o.elem;
    const V4<R> a0 = ps.A[0][pi], a1 = ps.A[1][pi], a2 = ps.A[2][pi], a3 = ps.A[3][pi], a4 = ps.A[4][pi],
                a5 = ps.A[5][pi];
    const V4<R> b0 = ps.B[0][pi], b1 = ps.B[1][pi], b2 = ps.B[2][pi], b3 = ps.B[3][pi];
    double xw[3];
    world_pos(P, ps, pi, a0, xw);
    if (o.x) st_user(o.x, e, i, xw[0]);
    if (o.y) st_user(o.y, e, i, xw[1]);
    if (o.z) st_user(o.z, e, i, xw[2]);
    if (o.vx) st_user(o.vx, e, i, (double)b0.x);
    if (o.vy) st_user(o.vy, e, i, (double)b0.y);
    if (o.vz) st_user(o.vz, e, i, (double)b0.z);
    if (o.edot) st_user(o.edot, e, i, (double)b0.w);
    const R H[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
    const R Hp[9] = {a4.x, a4.y, a4.z, a4.w, a5.x, a5.y, a5.z, a5.w, a3.y};
    const R C[9] = {b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w, b3.x};
    for (int q = 0; q < 9; ++q) {
        const double id = (q % 4 == 0) ? 1.0 : 0.0;
        if (o.F) st_user(o.F, e, 9 * i + q, (double)H[q] + id);
        if (o.Fp) st_user(o.Fp, e, 9 * i + q, (double)Hp[q] + id);
        if (o.C) st_user(o.C, e, 9 * i + q, (double)C[q]);
    }
    const V4<R> s0 = ps.S[0][pi], s1 = ps.S[1][pi];
    const R sv[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
    for (int q = 0; q < 6; ++q) {
        if (o.stress) st_user(o.stress, e, 6 * i + q, (double)sv[q]);
    }
    if (o.bs) {
        R kv[6] = {0, 0, 0, 0, 0, 0};
        if (ps.K[0]) {
            const V4<R> k0 = ps.K[0][pi], k1 = ps.K[1][pi];
            kv[0] = k0.x; kv[1] = k0.y; kv[2] = k0.z; kv[3] = k0.w; kv[4] = k1.x; kv[5] = k1.y;
        }
        for (int q = 0; q < 6; ++q) st_user(o.bs, e, 6 * i + q, (double)kv[q]);
    }
    if (o.eps) st_user(o.eps, e, i, (double)a0.w);
    if (o.T) st_user(o.T, e, i, Tamb + (double)a3.z);
    if (o.D) st_user(o.D, e, i, (double)a3.w);
    if (o.sres) st_user(o.sres, e, i, (double)ps.sres[pi]);
    if (o.status) o.status[i] = ps.status[pi];
    if (o.id) o.id[i] = ps.id[pi];
}

template <typename R>
__global__ void k_export_aos(const Inst<R>* inst, PState<R> ps, int64_t pbase, int64_t n, double Tamb, double rho,
                             AosParticle* out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const Inst<R>& P = *inst;
    const int64_t pi = pbase + s;
    AosParticle q;
    const V4<R> a0 = ps.A[0][pi], a1 = ps.A[1][pi], a2 = ps.A[2][pi], a3 = ps.A[3][pi], a4 = ps.A[4][pi],
                a5 = ps.A[5][pi];
    const V4<R> b0 = ps.B[0][pi], b1 = ps.B[1][pi], b2 = ps.B[2][pi], b3 = ps.B[3][pi];
    double xw[3];
    world_pos(P, ps, pi, a0, xw);
    q.x = xw[0]; q.y = xw[1]; q.z = xw[2];
    q.vx = b0.x; q.vy = b0.y; q.vz = b0.z;
    q.fx = q.fy = q.fz = 0.0;
    q.ext_fx = q.ext_fy = q.ext_fz = 0.0;
    q.density = rho;
    q.pressure = 0.0;
    q.volume = (double)P.pvol;
    q.mass = (double)P.pmass;
    q.temperature = Tamb + (double)a3.z;
    const R H[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
    const R Hp[9] = {a4.x, a4.y, a4.z, a4.w, a5.x, a5.y, a5.z, a5.w, a3.y};
    const R C[9] = {b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w, b3.x};
    for (int k = 0; k < 9; ++k) {
        const double id = (k % 4 == 0) ? 1.0 : 0.0;
        q.F[k] = (double)H[k] + id;
        q.F_p[k] = (double)Hp[k] + id;
        q.C[k] = (double)C[k];
    }
    const V4<R> s0 = ps.S[0][pi], s1 = ps.S[1][pi];
    q.stress_xx = s0.x; q.stress_yy = s0.y; q.stress_zz = s0.z; q.stress_xy = s0.w; q.stress_xz = s1.x; q.stress_yz = s1.y;
    q.backstress_xx = q.backstress_yy = q.backstress_zz = q.backstress_xy = q.backstress_xz = q.backstress_yz = 0.0;
    if (ps.K[0]) {
        const V4<R> k0 = ps.K[0][pi], k1 = ps.K[1][pi];
        q.backstress_xx = k0.x; q.backstress_yy = k0.y; q.backstress_zz = k0.z;
        q.backstress_xy = k0.w; q.backstress_xz = k1.x; q.backstress_yz = k1.y;
    }
    q.plasticStrain = a0.w;
    q.strainRate = b0.w;
    q.damage = a3.w;
    q.residualStress = ps.sres[pi];
    q.id = ps.id[pi];
    q.status = ps.status[pi];
    q.cellHash = 0;
    q.lodZone = 0;
    q.lastUpdateStep = 0;
    q.asbCounter = ps.asb[pi];
    out[ps.orig[pi]] = q;
}

// ------------------------------------------------------------------ metrics

// Per-CTA FP64 partials (slots below), then a single-CTA final pass:
//  0 mass 1-3 momentum 4 kinetic 5 elastic 6 thermal 7 max dT 8 max vm 9 max eps
//  10 sum eps 11 ref max stress 12 ref max T 13 ref kinetic 14 ref internal
//  15 n active 16 n chip 17 n fixed 18 n inactive 19-21 bmin 22-24 bmax
// The way back from k_export_aos for the fields the reference's consumers of
// the particle array write in place (ContactSolver: x, v, T; CFD coupling:
// ext_f, T).  Slot pi reads record orig[pi] (upload order, as exported).  A
// position or temperature equal to what the export writes now is left as it
// is, so an unmodified array imports bit for bit; a moved particle is
// re-expressed in its current bin (hi + lo in FP32 state) and flags[0] asks
// the host to re-bin.  The external force goes to pext in upload order (the
// next step's first P2G reads it there, whatever the re-bin does).  A status
// outside 0..4 is left as it was and counted in flags[1].
template <typename R>
__global__ void k_import_aos(const Inst<R>* inst, PState<R> ps, int64_t pbase, int64_t n, double Tamb, uint32_t fields,
                             const AosParticle* __restrict__ in, V4<R>* __restrict__ pext, int* __restrict__ flags) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const Inst<R>& P = *inst;
    const int64_t pi = pbase + s;
    const int32_t o = ps.orig[pi];
    const AosParticle& q = in[o];
    if (fields & MPM_AOS_POSITION) {
        const V4<R> a0 = ps.A[0][pi];
        double xw[3];
        world_pos(P, ps, pi, a0, xw);
        const double nw[3] = {q.x, q.y, q.z};
        if (nw[0] != xw[0] || nw[1] != xw[1] || nw[2] != xw[2]) {
            const int bin = ps.bin[pi];
            const int bo[3] = {(bin % P.nbx) * kBin, ((bin / P.nbx) % P.nby) * kBin, (bin / (P.nbx * P.nby)) * kBin};
            const double org[3] = {P.ox, P.oy, P.oz};
            double l[3];
            R hi[3];
            for (int a = 0; a < 3; ++a) {
                l[a] = (nw[a] - org[a]) / P.dx - (double)bo[a];
                hi[a] = (R)l[a];
            }
            ps.A[0][pi] = mk4<R>(hi[0], hi[1], hi[2], a0.w);
            if (ps.X) ps.X[pi] = mk4<R>((R)(l[0] - (double)hi[0]), (R)(l[1] - (double)hi[1]), (R)(l[2] - (double)hi[2]),
                                        R(0));
            flags[0] = 1;
        }
    }
    if (fields & MPM_AOS_VELOCITY) {
        const V4<R> b0 = ps.B[0][pi];
        ps.B[0][pi] = mk4<R>((R)q.vx, (R)q.vy, (R)q.vz, b0.w);
    }
    if (fields & MPM_AOS_TEMPERATURE) {
        V4<R> a3 = ps.A[3][pi];
        if (q.temperature != Tamb + (double)a3.z) {
            a3.z = (R)(q.temperature - Tamb);
            ps.A[3][pi] = a3;
        }
    }
    if (fields & MPM_AOS_STATUS) {
        const int32_t st = q.status;
        if (st >= (int32_t)ST_ACTIVE && st <= (int32_t)ST_FIXED) ps.status[pi] = (uint8_t)st;
        else atomicAdd(&flags[1], 1);
    }
    if (fields & MPM_AOS_EXT_FORCE) pext[pbase + o] = mk4<R>((R)q.ext_fx, (R)q.ext_fy, (R)q.ext_fz, R(0));
}

template <typename R>
__global__ void k_stats(const Inst<R>* inst, PState<R> ps, int64_t pbase, int64_t n, double mu, double K, double rho,
                        double cp, double Tamb, double* partial) {
    __shared__ double sh[kStatSlots][kT / 32];
    const Inst<R>& P = *inst;
    // the accumulators stay in registers: every loop over them is unrolled
    double acc[kStatSlots];
#pragma unroll
    for (int q = 0; q < kStatSlots; ++q) acc[q] = 0.0;
    acc[7] = -INFINITY; acc[8] = 0.0; acc[9] = -INFINITY; acc[11] = 0.0; acc[12] = 0.0;
#pragma unroll
    for (int q = 19; q < 22; ++q) acc[q] = INFINITY;
#pragma unroll
    for (int q = 22; q < 25; ++q) acc[q] = -INFINITY;
    const double m = (double)P.pmass, V = (double)P.pvol;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pi = pbase + s;
        // every load before the branch on the status (the position's bin and
        // low parts included): one memory round trip
        const int st = ps.status[pi];
        const V4<R> a0 = ps.A[0][pi], a3 = ps.A[3][pi], b0 = ps.B[0][pi], s0 = ps.S[0][pi], s1 = ps.S[1][pi];
        const int bin = ps.bin[pi];
        const V4<R> xl = ps.X ? ps.X[pi] : mk4<R>(0, 0, 0, 0);
        if (st == ST_INACTIVE) { acc[18] += 1.0; continue; }
        if (st == ST_ACTIVE) acc[15] += 1.0;
        else if (st == ST_CHIP) acc[16] += 1.0;
        else if (st == ST_FIXED) acc[17] += 1.0;
        const double sxx = s0.x, syy = s0.y, szz = s0.z, sxy = s0.w, sxz = s1.x, syz = s1.y;
        const double tr = sxx + syy + szz;
        const double dx_ = sxx - tr / 3.0, dy_ = syy - tr / 3.0, dz_ = szz - tr / 3.0;
        const double vm = sqrt(1.5 * (dx_ * dx_ + dy_ * dy_ + dz_ * dz_ + 2.0 * (sxy * sxy + sxz * sxz + syz * syz)));
        const double vx = b0.x, vy = b0.y, vz = b0.z;
        const double v2 = vx * vx + vy * vy + vz * vz;
        const double dT = a3.z, eps = a0.w;
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
            acc[11] = fmax(acc[11], vm);
            acc[12] = fmax(acc[12], Tamb + dT);
            acc[13] += 0.5 * m * v2;
            acc[14] += (vm * vm * m) / (6.0 * 80e9) + V * eps * vm;
            const int bx = bin % P.nbx, by = (bin / P.nbx) % P.nby, bz = bin / (P.nbx * P.nby);
            const double xw[3] = {P.ox + ((double)(bx * kBin) + ((double)a0.x + (double)xl.x)) * P.dx,
                                  P.oy + ((double)(by * kBin) + ((double)a0.y + (double)xl.y)) * P.dx,
                                  P.oz + ((double)(bz * kBin) + ((double)a0.z + (double)xl.z)) * P.dx};
#pragma unroll
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
        const bool isMin = (q >= 19 && q < 22);
        const bool isMax = (q == 7 || q == 8 || q == 9 || q == 11 || q == 12 || (q >= 22 && q < 25));
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, o);
            v = isMin ? fmin(v, u) : (isMax ? fmax(v, u) : v + u);
        }
        if (lane == 0) sh[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < kStatSlots) {
        const int q = threadIdx.x;
        const bool isMin = (q >= 19 && q < 22);
        const bool isMax = (q == 7 || q == 8 || q == 9 || q == 11 || q == 12 || (q >= 22 && q < 25));
        double v = sh[q][0];
        for (int w = 1; w < kT / 32; ++w) v = isMin ? fmin(v, sh[q][w]) : (isMax ? fmax(v, sh[q][w]) : v + sh[q][w]);
        partial[(int64_t)blockIdx.x * kStatSlots + q] = v;
    }
}

// One CTA per slot: thread t combines the block partials t, t + kFinalT, ...
// in order, then a fixed tree over the threads (the same order on every run).
constexpr int kFinalT = 256;
__global__ void __launch_bounds__(kFinalT) k_stats_final(const double* partial, int nb, double* out) {
    __shared__ double sh[kFinalT];
    const int q = blockIdx.x, t = threadIdx.x;
    const bool isMin = (q >= 19 && q < 22);
    const bool isMax = (q == 7 || q == 8 || q == 9 || q == 11 || q == 12 || (q >= 22 && q < 25));
    double v = isMin ? INFINITY : (isMax ? -INFINITY : 0.0);
    for (int b = t; b < nb; b += kFinalT) {
        const double u = partial[(int64_t)b * kStatSlots + q];
        v = isMin ? fmin(v, u) : (isMax ? fmax(v, u) : v + u);
    }
    sh[t] = v;
    __syncthreads();
    for (int w = kFinalT / 2; w > 0; w >>= 1) {
        if (t < w) {
            const double u = sh[t + w];
            sh[t] = isMin ? fmin(sh[t], u) : (isMax ? fmax(sh[t], u) : sh[t] + u);
        }
        __syncthreads();
    }
    if (t == 0) out[q] = sh[0];
}

template <typename R>
__global__ void k_set_temps(PState<R> ps, int64_t pbase, int64_t n, const double* T, int64_t count, double Tamb) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t pi = pbase + s;
    const int64_t o = ps.orig[pi];
    if (o < count) {
        V4<R> a3 = ps.A[3][pi];
        a3.z = (R)(T[o] - Tamb);
        ps.A[3][pi] = a3;
    }
}

// ------------------------------------------------------------------ launchers

std::atomic<int64_t>& launch_counter() {
    static std::atomic<int64_t> c{0};
    return c;
}

template <typename R>
void launch_bin_count(const Inst<R>* insts, int n_inst, const PState<R>& ps, const int32_t* key_base, bool initial,
                      const double* pos_scratch, int32_t* key, int32_t* rank, int32_t* count, int32_t* newbin,
                      int64_t np, int kpt, int sort_every, bool keep_all, cudaStream_t st) {
    if (np <= 0) return;
    k_bin_count<R><<<(int)((np + kT - 1) / kT), kT, 0, st>>>(insts, n_inst, ps, key_base, initial, pos_scratch, key,
                                                             rank, count, newbin, np, kpt, sort_every, keep_all);
    ++launch_counter();
}

template <typename R>
void launch_bin_scatter(const PState<R>& src, const PState<R>& dst, const Inst<R>* insts, int n_inst,
                        const int32_t* key, const int32_t* rank, const int32_t* offset, const int32_t* key_base,
                        const int32_t* newbin, bool initial, const double* pos_scratch, bool has_K, int64_t np,
                        int32_t* perm, const int32_t* bin_key, int nbins_total, cudaStream_t st) {
    if (np <= 0) return;
    const int blocks = (int)((np + kT - 1) / kT);
    cudaMemsetAsync(perm, 0xff, sizeof(int32_t) * np, st);
    k_bin_perm<R><<<blocks, kT, 0, st>>>(insts, n_inst, key, rank, offset, key_base, newbin, src.orig, perm, np);
    if (nbins_total > 0) k_bin_order<<<nbins_total, kCellsPerBin, 0, st>>>(bin_key, offset, perm, np);
    k_bin_gather<R><<<blocks, kT, 0, st>>>(src, dst, insts, n_inst, key, key_base, newbin, perm, initial,
                                           pos_scratch, has_K, np);
    launch_counter() += nbins_total > 0 ? 3 : 2;
}

template <typename R>
void launch_raster(const Inst<R>* insts, int i, int k, int npoints, cudaStream_t st) {
    if (npoints <= 0) return;
    k_raster<R><<<(npoints + kT - 1) / kT, kT, 0, st>>>(insts, i, k);
    ++launch_counter();
}

template <typename R>
void launch_import(const DevSoA& in, int64_t n, double ox, double oy, double oz, double dx, double Tamb,
                   const PState<R>& ps, int64_t pbase, double* pos_scratch, cudaStream_t st) {
    if (n <= 0) return;
    k_import<R><<<(int)((n + kT - 1) / kT), kT, 0, st>>>(in, n, ox, oy, oz, 1.0 / dx, Tamb, ps, pbase, pos_scratch);
    ++launch_counter();
}

template <typename R>
void launch_gen(const Inst<R>& P, const int32_t c0[3], const int32_t c1[3], int ppc, uint64_t seed, uint32_t inst,
                int fixed_layers, double dT0, int tool_check, int32_t* flag, int32_t* idx, int32_t* scan_tmp,
                const PState<R>& ps, int64_t pbase, double* pos_scratch, cudaStream_t st) {
    const int wx = c1[0] - c0[0], wy = c1[1] - c0[1], wz = c1[2] - c0[2];
    const int64_t ncand = (int64_t)wx * wy * wz * ppc;
    if (ncand <= 0) return;
    const uint32_t s0 = (uint32_t)(seed & 0xffffffffu), s1 = (uint32_t)(seed >> 32);
    const int nb = (int)((ncand + kT - 1) / kT);
    k_gen_flags<R><<<nb, kT, 0, st>>>(P, c0[0], c0[1], c0[2], wx, wy, wz, ppc, s0, s1, inst, tool_check, flag, ncand);
    exclusive_scan(flag, idx, ncand, scan_tmp, st);
    k_gen_write<R><<<nb, kT, 0, st>>>(P, c0[0], c0[1], c0[2], wx, wy, wz, ppc, s0, s1, inst, fixed_layers, (R)dT0,
                                      flag, idx, ps, pbase, pos_scratch, ncand);
    launch_counter() += 2;
}

template <typename R>
void launch_export(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double Tamb,
                   const DevSoAOut& out, cudaStream_t st) {
    if (n <= 0) return;
    k_export<R><<<(int)((n + kT - 1) / kT), kT, 0, st>>>(inst_dev, ps, pbase, n, Tamb, out);
    ++launch_counter();
}

template <typename R>
void launch_export_aos(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double Tamb,
                       double rho, void* out, cudaStream_t st) {
    if (n <= 0) return;
    k_export_aos<R><<<(int)((n + kT - 1) / kT), kT, 0, st>>>(inst_dev, ps, pbase, n, Tamb, rho, (AosParticle*)out);
    ++launch_counter();
}

template <typename R>
void launch_import_aos(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double Tamb,
                       uint32_t fields, const void* in, V4<R>* pext, int* flags, cudaStream_t st) {
    if (n <= 0) return;
    Range nvtx_range("mpm.import_aos");
    k_import_aos<R><<<(int)((n + kT - 1) / kT), kT, 0, st>>>(inst_dev, ps, pbase, n, Tamb, fields,
                                                             (const AosParticle*)in, pext, flags);
    ++launch_counter();
}

template <typename R>
void launch_stats(const Inst<R>* inst_dev, const PState<R>& ps, int64_t pbase, int64_t n, double mu, double K,
                  double rho, double cp, double Tamb, double* partial, int nblocks, double* out, cudaStream_t st) {
    k_stats<R><<<nblocks, kT, 0, st>>>(inst_dev, ps, pbase, n, mu, K, rho, cp, Tamb, partial);
    k_stats_final<<<kStatSlots, kFinalT, 0, st>>>(partial, nblocks, out);
    launch_counter() += 2;
}

template <typename R>
void launch_set_temps(const PState<R>& ps, int64_t pbase, int64_t n, const double* T, int64_t count, double Tamb,
                      cudaStream_t st) {
    if (n <= 0) return;
    k_set_temps<R><<<(int)((n + kT - 1) / kT), kT, 0, st>>>(ps, pbase, n, T, count, Tamb);
    ++launch_counter();
}

// ------------------------------------------------------------------ relayout

template <typename R>
__global__ void k_relayout(PState<R> src, PState<R> dst, const RelayoutMap* __restrict__ map, int n_inst,
                           int64_t total) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
    int lo = 0, hi = n_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (map[mid].new_pbase <= s) lo = mid; else hi = mid - 1;
    }
    const RelayoutMap m = map[lo];
    const int64_t r = s - m.new_pbase;
    if (r < 0 || r >= m.np) return;
    const int64_t o = m.old_pbase + r;
#pragma unroll
    for (int q = 0; q < 6; ++q) dst.A[q][s] = src.A[q][o];
#pragma unroll
    for (int q = 0; q < 4; ++q) dst.B[q][s] = src.B[q][o];
    dst.S[0][s] = src.S[0][o];
    dst.S[1][s] = src.S[1][o];
    if (src.K[0] && dst.K[0]) {
        dst.K[0][s] = src.K[0][o];
        dst.K[1][s] = src.K[1][o];
    }
    dst.sres[s] = src.sres[o];
    dst.status[s] = src.status[o];
    dst.asb[s] = src.asb[o];
    dst.id[s] = src.id[o];
    if (src.X && dst.X) dst.X[s] = src.X[o];
    dst.orig[s] = src.orig[o];
    dst.bin[s] = src.bin[o];
    dst.skey[s] = src.skey[o];
}

template <typename R>
void launch_relayout(const PState<R>& src, const PState<R>& dst, const RelayoutMap* map, int n_inst, int64_t total,
                     cudaStream_t st) {
    if (total <= 0 || n_inst <= 0) return;
    k_relayout<R><<<(int)((total + kT - 1) / kT), kT, 0, st>>>(src, dst, map, n_inst, total);
    ++launch_counter();
}

// ------------------------------------------------------------------ heat conduction

// mpmDiffuseTemperatureKernel (reference src/MPMWorkpieceSolver.cu:208-262) as
// the Jacobi step it describes, over the nodes of every instance that conducts
// heat: from grid buffer b (mass in .x) and its T m buffer to the node
// temperatures tn.  A node with m >= 1e-15 takes T + alpha dt lap(T) / dx^2,
// T = (T m)/m, 7-point Laplacian over the neighbours inside the domain, a
// neighbour's T = (T m) / max(m, 1e-30) (0 at an empty node), then T >= 0; a
// lighter node keeps (T m)/m.  (The reference updates in place, so there a
// node can read a neighbour already updated, depending on the schedule.)
template <typename R>
__global__ void k_heat_diffuse(const Inst<R>* __restrict__ insts, int n_inst, int b, int64_t total) {
    for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < total;
         gi += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_inst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (insts[mid].gbase <= gi) lo = mid; else hi = mid - 1;
        }
        const Inst<R>& P = insts[lo];
        if (!P.heat_on) continue;
        const int64_t li = gi - P.gbase;
        if (li < 0 || li >= P.nn) continue;
        const V4<R>* __restrict__ g = P.grid[b];
        const R* __restrict__ tm = P.tm[b];
        const R m = g[li].x;
        if (m < R(1e-15)) {
            P.tn[li] = m > R(0) ? tm[li] / m : R(0);
            continue;
        }
        const R T = tm[li] / m;
        const int nx = P.nx, ny = P.ny, nz = P.nz;
        const int64_t nxy = (int64_t)nx * ny;
        const int i = (int)(li % nx);
        const int64_t t = li / nx;
        const int j = (int)(t % ny), k = (int)(t / ny);
        R lap = R(0);
        if (i > 0) lap += tm[li - 1] / fmax(g[li - 1].x, R(1e-30)) - T;
        if (i < nx - 1) lap += tm[li + 1] / fmax(g[li + 1].x, R(1e-30)) - T;
        if (j > 0) lap += tm[li - nx] / fmax(g[li - nx].x, R(1e-30)) - T;
        if (j < ny - 1) lap += tm[li + nx] / fmax(g[li + nx].x, R(1e-30)) - T;
        if (k > 0) lap += tm[li - nxy] / fmax(g[li - nxy].x, R(1e-30)) - T;
        if (k < nz - 1) lap += tm[li + nxy] / fmax(g[li + nxy].x, R(1e-30)) - T;
        P.tn[li] = fmax(T + (R)P.heat_c * lap, R(0));
    }
}

template <typename R>
void launch_heat_diffuse(const Inst<R>* insts, int n_inst, int b, int64_t total, cudaStream_t st) {
    if (total <= 0 || n_inst <= 0) return;
    Range nvtx_range("mpm.heat_diffuse");
    const int64_t blocks = std::min<int64_t>((total + kT - 1) / kT, 148 * 16);
    k_heat_diffuse<R><<<(int)blocks, kT, 0, st>>>(insts, n_inst, b, total);
    ++launch_counter();
}

#define MPMB_INST(R)                                                                                                  \
    template void launch_bin_count<R>(const Inst<R>*, int, const PState<R>&, const int32_t*, bool, const double*,   \
                                      int32_t*, int32_t*, int32_t*, int32_t*, int64_t, int, int, bool, cudaStream_t); \
    template void launch_bin_scatter<R>(const PState<R>&, const PState<R>&, const Inst<R>*, int, const int32_t*,    \
                                        const int32_t*, const int32_t*, const int32_t*, const int32_t*, bool,       \
                                        const double*, bool, int64_t, int32_t*, const int32_t*, int, cudaStream_t);  \
    template void launch_import<R>(const DevSoA&, int64_t, double, double, double, double, double, const PState<R>&, \
                                   int64_t, double*, cudaStream_t);                                                  \
    template void launch_gen<R>(const Inst<R>&, const int32_t*, const int32_t*, int, uint64_t, uint32_t, int, double, \
                                int, int32_t*, int32_t*, int32_t*, const PState<R>&, int64_t, double*, cudaStream_t); \
    template void launch_export<R>(const Inst<R>*, const PState<R>&, int64_t, int64_t, double, const DevSoAOut&,     \
                                   cudaStream_t);                                                                    \
    template void launch_export_aos<R>(const Inst<R>*, const PState<R>&, int64_t, int64_t, double, double, void*,    \
                                       cudaStream_t);                                                                \
    template void launch_import_aos<R>(const Inst<R>*, const PState<R>&, int64_t, int64_t, double, uint32_t,         \
                                       const void*, V4<R>*, int*, cudaStream_t);                                     \
    template void launch_stats<R>(const Inst<R>*, const PState<R>&, int64_t, int64_t, double, double, double, double, \
                                  double, double*, int, double*, cudaStream_t);                                      \
    template void launch_set_temps<R>(const PState<R>&, int64_t, int64_t, const double*, int64_t, double, cudaStream_t); \
    template void launch_relayout<R>(const PState<R>&, const PState<R>&, const RelayoutMap*, int, int64_t, cudaStream_t); \
    template void launch_heat_diffuse<R>(const Inst<R>*, int, int, int64_t, cudaStream_t);                      \
    template void launch_raster<R>(const Inst<R>*, int, int, int, cudaStream_t);

MPMB_INST(float)
MPMB_INST(double)

}  // namespace mpmb
