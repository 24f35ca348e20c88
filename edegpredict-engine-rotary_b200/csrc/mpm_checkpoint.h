// mpm_checkpoint.h -- the checkpoint format of one workpiece (host code only,
// no CUDA).  The reference has no state serialisation; this is the raw dump a
// serving loop needs to preempt and resume a workpiece.
//
// Layout of a checkpoint (little-endian, this library's ABI):
//   CkptHeader
//   the instance's particle arrays in the engine's internal order, each np
//   elements: A0..A5, B0..B3, S0, S1 (vectors of 4 reals), K0, K1 (only with
//   backstress), X (FP32 state: position low parts), sres (real), status,
//   shear counter (uint8), id, bin, orig (int32)
//   the raster tool's sample offsets (3 x n_samples doubles), if any
// The payload (everything after the header) carries a 64-bit checksum.  The
// particles keep their bin-local positions and bins, so a checkpoint loads
// only into an instance with the same grid size and precision.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpm_capi.h"

namespace mpmb {

constexpr char kCkptMagic[8] = {'M', 'P', 'M', 'C', 'K', 'P', 'T', '\0'};
constexpr uint32_t kCkptVersion = 2;

struct CkptHeader {
    char magic[8];
    uint32_t version;
    uint32_t abi_version;
    int32_t precision;      // MPM_PREC_F32 or MPM_PREC_F64
    int32_t has_K;          // backstress arrays present
    int32_t n_samples;      // raster tool samples after the arrays
    int32_t since_rebin;    // steps since the instance's last re-bin (its re-bin phase)
    int64_t np;             // particles
    int64_t step;           // steps taken
    double time, tool_t0, dt;
    uint64_t payload_bytes; // bytes after the header
    uint64_t checksum;      // ckpt_checksum of the payload
    mpm_params params;      // the instance's parameters when it was saved
    mpm_tool_desc tool;     // its tool (sample pointers cleared)
};

// Bytes per particle of each array, in payload order.
inline std::vector<size_t> ckpt_array_elem(int precision, bool has_K) {
    const size_t r = precision == MPM_PREC_F64 ? 8 : 4, v4 = 4 * r;
    std::vector<size_t> e(12, v4);           // A0..A5, B0..B3, S0, S1
    if (has_K) { e.push_back(v4); e.push_back(v4); }
    if (precision == MPM_PREC_F32) e.push_back(v4);   // X
    e.push_back(r);                           // sres
    e.push_back(1); e.push_back(1);           // status, shear counter
    e.push_back(4); e.push_back(4); e.push_back(4);   // id, bin, orig
    e.push_back(4);                           // the re-bin key (layout)
    return e;
}

inline uint64_t ckpt_payload_bytes(int precision, bool has_K, int64_t np, int32_t n_samples) {
    uint64_t per = 0;
    for (size_t b : ckpt_array_elem(precision, has_K)) per += b;
    return per * (uint64_t)np + 24ull * (uint64_t)(n_samples > 0 ? n_samples : 0);
}

// 64-bit FNV-1a over 8-byte words (bytes for the tail): fast enough for
// checkpoints of tens of GB, and catches truncation and corruption.
inline uint64_t ckpt_checksum(const unsigned char* p, uint64_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    const uint64_t prime = 0x100000001b3ull;
    uint64_t k = 0;
    for (; k + 8 <= n; k += 8) {
        uint64_t w;
        std::memcpy(&w, p + k, 8);
        h = (h ^ w) * prime;
    }
    for (; k < n; ++k) h = (h ^ p[k]) * prime;
    return h;
}

// Checks a checkpoint against the instance it is to be loaded into: its
// precision, backstress arrays, grid size and particle capacity.  Returns
// MPM_OK or MPM_INVALID_ARG / MPM_NOT_SUPPORTED / MPM_CAPACITY with a message.
inline mpm_status ckpt_check(const void* buf, int64_t bytes, int precision, bool handle_has_K, int nx, int ny,
                             int nz, int64_t capacity, CkptHeader* out, std::string* err) {
    if (!buf || bytes < (int64_t)sizeof(CkptHeader)) {
        *err = "checkpoint buffer NULL or shorter than its header";
        return MPM_INVALID_ARG;
    }
    CkptHeader h;
    std::memcpy(&h, buf, sizeof(h));
    if (std::memcmp(h.magic, kCkptMagic, sizeof(kCkptMagic)) != 0) {
        *err = "not a checkpoint (magic)";
        return MPM_INVALID_ARG;
    }
    if (h.version != kCkptVersion || h.abi_version != MPM_ABI_VERSION) {
        *err = "checkpoint format version " + std::to_string(h.version) + " / ABI " + std::to_string(h.abi_version) +
               " is not this library's (" + std::to_string(kCkptVersion) + " / " + std::to_string(MPM_ABI_VERSION) +
               ")";
        return MPM_NOT_SUPPORTED;
    }
    if (h.precision != precision) {
        *err = "checkpoint precision differs from the instance's";
        return MPM_INVALID_ARG;
    }
    if (h.np < 0 || h.n_samples < 0 || h.has_K < 0 || h.has_K > 1) {
        *err = "checkpoint header is corrupt";
        return MPM_INVALID_ARG;
    }
    if (h.has_K && !handle_has_K) {
        *err = "checkpoint holds backstress state; the handle has none (create it with H_kin > 0)";
        return MPM_NOT_SUPPORTED;
    }
    if (h.params.nx != nx || h.params.ny != ny || h.params.nz != nz) {
        *err = "checkpoint grid size differs from the instance's";
        return MPM_INVALID_ARG;
    }
    if (h.np > capacity) {
        *err = "checkpoint holds more particles than the instance's capacity";
        return MPM_CAPACITY;
    }
    const uint64_t want = ckpt_payload_bytes(h.precision, h.has_K != 0, h.np, h.n_samples);
    if (h.payload_bytes != want || (uint64_t)bytes < sizeof(CkptHeader) + want) {
        *err = "checkpoint is truncated or its sizes do not agree";
        return MPM_INVALID_ARG;
    }
    if (ckpt_checksum(static_cast<const unsigned char*>(buf) + sizeof(CkptHeader), want) != h.checksum) {
        *err = "checkpoint checksum mismatch (corrupt payload)";
        return MPM_INVALID_ARG;
    }
    if (out) *out = h;
    return MPM_OK;
}

}  // namespace mpmb
