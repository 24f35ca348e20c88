"""The checkpoint format's validation (csrc/mpm_checkpoint.h) without a GPU: a
small C++ program builds a checkpoint of synthetic bytes and checks that a
good one passes and that every kind of bad one is refused with its own status:
wrong magic, another format version, another precision, backstress state for
a handle without it, another grid size, more particles than the capacity, a
truncated buffer and a flipped payload byte (checksum).  Also pins the bytes
per particle of the two precisions and the C ABI's argument checks."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess

import pytest

from conftest import ROOT
from mpm_b200 import capi as A

CORE = ROOT / "edegpredict-engine-rotary_b200" / "csrc"

PROG = r"""
#include <cassert>
#include <cstdio>
#include <string>
#include <vector>
#include "mpm_checkpoint.h"
using namespace mpmb;

static std::vector<unsigned char> make(int prec, int has_K, int64_t np, int ns) {
    const uint64_t pay = ckpt_payload_bytes(prec, has_K != 0, np, ns);
    std::vector<unsigned char> b(sizeof(CkptHeader) + pay);
    for (uint64_t k = 0; k < pay; ++k) b[sizeof(CkptHeader) + k] = (unsigned char)(k * 131 + 7);
    CkptHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = kCkptVersion;
    h.abi_version = MPM_ABI_VERSION;
    h.precision = prec;
    h.has_K = has_K;
    h.n_samples = ns;
    h.np = np;
    h.payload_bytes = pay;
    h.checksum = ckpt_checksum(b.data() + sizeof(CkptHeader), pay);
    h.params.nx = 16; h.params.ny = 12; h.params.nz = 8;
    std::memcpy(b.data(), &h, sizeof(h));
    return b;
}

static mpm_status chk(const std::vector<unsigned char>& b, int prec = MPM_PREC_F32, bool K = false,
                      int nx = 16, int64_t cap = 1000, int64_t len = -1) {
    std::string e;
    CkptHeader h;
    return ckpt_check(b.data(), len < 0 ? (int64_t)b.size() : len, prec, K, nx, 12, 8, cap, &h, &e);
}

int main() {
    // bytes per particle: FP32 13 vectors of 16 B + sres 4 + 2 x 1 + 4 x 4 (id, bin, orig, re-bin key);
    // FP64 12 x 32 + 8 + 2 + 16
    assert(ckpt_payload_bytes(MPM_PREC_F32, false, 1, 0) == 13 * 16 + 4 + 2 + 16);
    assert(ckpt_payload_bytes(MPM_PREC_F64, false, 1, 0) == 12 * 32 + 8 + 2 + 16);
    assert(ckpt_payload_bytes(MPM_PREC_F64, true, 1, 0) == 14 * 32 + 8 + 2 + 16);
    assert(ckpt_payload_bytes(MPM_PREC_F32, false, 0, 5) == 5 * 24);
    auto good = make(MPM_PREC_F32, 0, 100, 3);
    assert(chk(good) == MPM_OK);
    assert(chk(make(MPM_PREC_F64, 1, 10, 0), MPM_PREC_F64, true) == MPM_OK);
    auto b = good; b[0] = 'X';
    assert(chk(b) == MPM_INVALID_ARG);                                   // magic
    b = good; reinterpret_cast<CkptHeader*>(b.data())->version = kCkptVersion + 1;
    assert(chk(b) == MPM_NOT_SUPPORTED);                                 // format version
    assert(chk(good, MPM_PREC_F64) == MPM_INVALID_ARG);                  // precision
    assert(chk(make(MPM_PREC_F32, 1, 10, 0)) == MPM_NOT_SUPPORTED);      // backstress, handle has none
    assert(chk(make(MPM_PREC_F32, 0, 10, 0), MPM_PREC_F32, true) == MPM_OK);   // handle has it, zeroed
    assert(chk(good, MPM_PREC_F32, false, 17) == MPM_INVALID_ARG);       // grid size
    assert(chk(good, MPM_PREC_F32, false, 16, 99) == MPM_CAPACITY);      // capacity
    assert(chk(good, MPM_PREC_F32, false, 16, 1000, (int64_t)good.size() - 1) == MPM_INVALID_ARG);  // truncated
    assert(chk(good, MPM_PREC_F32, false, 16, 1000, 10) == MPM_INVALID_ARG);   // shorter than the header
    b = good; b[sizeof(CkptHeader) + 777] ^= 1;
    assert(chk(b) == MPM_INVALID_ARG);                                   // checksum
    b = good; reinterpret_cast<CkptHeader*>(b.data())->np = 101;
    assert(chk(b) == MPM_INVALID_ARG);                                   // sizes disagree
    std::printf("OK\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_checkpoint_validation(tmp_path):
    src = tmp_path / "ckpt.cpp"
    src.write_text(PROG)
    exe = tmp_path / "ckpt"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(CORE), "-I", str(ROOT / "include"),
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stderr


def test_checkpoint_entry_points_check_their_arguments():
    L = A.lib()
    n = C.c_int64()
    assert L.mpm_checkpoint_bytes(None, 0, C.byref(n)) == A.MPM_INVALID_ARG
    assert L.mpm_checkpoint_save(None, 0, None, 0) == A.MPM_INVALID_ARG
    assert L.mpm_checkpoint_load(None, 0, None, 0) == A.MPM_INVALID_ARG
