"""The serving loop's scheduler (csrc/mpm_server_core.h) without a GPU: a small
C++ program drives it with a fake engine and a fake clock and checks arrival-
order admission under the pool budget (no overtaking), the resident limit,
the chunk sizes (the fewest remaining steps, at most max_chunk), that each
request's steps follow it across instance-index changes, the time stamps and
the refusal of requests that can never fit.  Also checks that the ctypes
mirrors of the request/result/config/stats structs have the C layout."""
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
#include <vector>
#include "mpm_server_core.h"
using namespace mpmb;

struct FakeOps {
    std::vector<int64_t> caps;
    std::vector<int> steps;
    std::vector<int> chunks;
    int changes = 0;
    mpm_status change(const std::vector<mpm_params>& add, const std::vector<int64_t>& c,
                      const std::vector<int32_t>& remove, int* first) {
        for (auto it = remove.rbegin(); it != remove.rend(); ++it) {
            caps.erase(caps.begin() + *it);
            steps.erase(steps.begin() + *it);
        }
        *first = (int)caps.size();
        for (size_t k = 0; k < add.size(); ++k) { caps.push_back(c[k]); steps.push_back(0); }
        ++changes;
        return MPM_OK;
    }
    mpm_status init(int inst, const mpm_request& r, int64_t* np) {
        assert(inst >= 0 && inst < (int)caps.size());
        *np = caps[inst];
        return MPM_OK;
    }
    mpm_status step(int k, const std::vector<double>& dts) {
        assert(dts.size() == caps.size());
        for (auto& s : steps) s += k;
        chunks.push_back(k);
        return MPM_OK;
    }
    mpm_status metrics(int inst, mpm_metrics* m) {
        m->mass = steps[inst];     // steps this instance has seen
        return MPM_OK;
    }
    mpm_status health(std::vector<int32_t>& st) {
        assert(st.size() == caps.size());
        return MPM_OK;
    }
    mpm_status save(int, std::vector<unsigned char>*) { return MPM_NOT_SUPPORTED; }
    mpm_status restore(int, const std::vector<unsigned char>&, int64_t*) { return MPM_NOT_SUPPORTED; }
};

static mpm_request req(int cells_x, int nsteps) {
    mpm_request r{};
    r.params.nx = 16; r.params.ny = 16; r.params.nz = 16;
    r.c0[0] = r.c0[1] = r.c0[2] = 0;
    r.c1[0] = cells_x; r.c1[1] = 1; r.c1[2] = 1;
    r.ppc = 1; r.nsteps = nsteps; r.dt = 1e-9;
    return r;
}

int main() {
    double now = 0.0;
    FakeOps ops;
    Pools pools;
    pools.particles = 100; pools.nodes = 1 << 20; pools.keys = 1 << 20; pools.bins = 1 << 20;
    Scheduler<FakeOps> s(&ops, pools, 50, 3, [&]() { now += 1.0; return now; });
    int64_t id[6];
    // 60 + 30 fit (90 <= 100); 20 would fit after them but must not overtake the 50
    assert(s.submit(req(60, 30), &id[0]) == MPM_OK);
    assert(s.submit(req(30, 100), &id[1]) == MPM_OK);
    assert(s.submit(req(50, 10), &id[2]) == MPM_OK);
    assert(s.submit(req(5, 10), &id[3]) == MPM_OK);
    int64_t big;
    assert(s.submit(req(101, 1), &big) == MPM_CAPACITY);
    int32_t nres = 0;
    assert(s.tick(&nres) == MPM_OK);
    assert(nres == 2 && ops.chunks.back() == 30);      // fewest remaining: 30
    mpm_result r0;
    s.poll(id[0], &r0);
    assert(r0.state == MPM_REQ_DONE && r0.metrics.mass == 30 && r0.steps_done == 30);
    assert(r0.t_submit < r0.t_admit && r0.t_admit < r0.t_done);
    mpm_result r2;
    s.poll(id[2], &r2);
    assert(r2.state == MPM_REQ_QUEUED);
    // request 0 leaves, 50 and 5 come in (30 + 50 + 5 = 85 <= 100, 3 resident)
    assert(s.tick(&nres) == MPM_OK);
    assert(nres == 3 && ops.chunks.back() == 10);
    s.poll(id[2], &r2);
    mpm_result r3;
    s.poll(id[3], &r3);
    assert(r2.state == MPM_REQ_DONE && r2.metrics.mass == 10);
    assert(r3.state == MPM_REQ_DONE && r3.metrics.mass == 10);
    // request 1 runs on alone: 100 - 40 = 60 left -> 50, then 10
    assert(s.tick(&nres) == MPM_OK && ops.chunks.back() == 50);
    assert(s.tick(&nres) == MPM_OK && ops.chunks.back() == 10);
    mpm_result r1;
    s.poll(id[1], &r1);
    assert(r1.state == MPM_REQ_DONE && r1.metrics.mass == 100 && r1.steps_done == 100);
    assert(s.tick(&nres) == MPM_OK && nres == 0);
    mpm_server_stats st = s.stats();
    assert(st.offered == 4 && st.admitted == 4 && st.completed == 4 && st.failed == 0 && st.queued == 0);
    assert(st.particle_updates == 60 * 30 + 30 * 100 + 50 * 10 + 5 * 10);
    // the resident limit: 5 small requests, at most 3 at once
    FakeOps ops2;
    Scheduler<FakeOps> s2(&ops2, pools, 50, 3, [&]() { now += 1.0; return now; });
    for (int k = 0; k < 5; ++k) s2.submit(req(1, 5), &id[0]);
    s2.tick(&nres);
    assert(nres == 3);
    s2.tick(&nres);
    assert(nres == 2);
    // the resident-particle cap: 40 particles; a 60-particle request still runs when alone
    FakeOps ops3;
    Scheduler<FakeOps> s3(&ops3, pools, 50, 8, [&]() { now += 1.0; return now; }, 40);
    s3.submit(req(60, 5), &id[0]);
    s3.submit(req(10, 5), &id[1]);
    s3.tick(&nres);
    assert(nres == 1);          // 60 alone; 10 more would exceed the cap
    s3.tick(&nres);
    assert(nres == 1);          // the 60 left, the 10 came in
    s3.poll(id[1], &r1);
    assert(r1.state == MPM_REQ_DONE);
    std::printf("OK\n");
    return 0;
}
"""

SIZES = r"""
#include <stdio.h>
#include <stddef.h>
#include "mpm_capi.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(mpm_request), sizeof(mpm_result), sizeof(mpm_server_config),
           sizeof(mpm_server_stats), offsetof(mpm_request, seed), offsetof(mpm_request, dt),
           offsetof(mpm_result, metrics));
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_scheduler_with_fake_engine(tmp_path):
    src = tmp_path / "sched.cpp"
    src.write_text(PROG)
    exe = tmp_path / "sched"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(CORE), "-I", str(ROOT / "include"),
                        str(src), "-o", str(exe), "-pthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stderr


FAULTS = r"""
#include <cassert>
#include <cmath>
#include <cstdio>
#include <vector>
#include "mpm_server_core.h"
using namespace mpmb;

// A fake engine whose faults are made on the host: instance errors that the
// health read reports (as the device error words would), and an instance
// change that fails like an allocator that is out of memory.
struct FaultyOps {
    std::vector<int64_t> caps;   // particles per instance: the request's tag
    std::vector<int> steps;
    int64_t bad_tag = -1;        // the instance holding this many particles fails after a step
    int oom_changes = 0;         // the next n instance changes fail
    std::vector<int> removed_tags;
    mpm_status change(const std::vector<mpm_params>& add, const std::vector<int64_t>& c,
                      const std::vector<int32_t>& remove, int* first) {
        if (oom_changes > 0) {
            --oom_changes;
            return MPM_OOM;
        }
        for (auto it = remove.rbegin(); it != remove.rend(); ++it) {
            removed_tags.push_back((int)caps[*it]);
            caps.erase(caps.begin() + *it);
            steps.erase(steps.begin() + *it);
        }
        *first = (int)caps.size();
        for (size_t k = 0; k < add.size(); ++k) { caps.push_back(c[k]); steps.push_back(0); }
        return MPM_OK;
    }
    mpm_status init(int inst, const mpm_request&, int64_t* np) { *np = caps[inst]; return MPM_OK; }
    mpm_status step(int k, const std::vector<double>&) {
        for (auto& s : steps) s += k;
        return MPM_OK;
    }
    mpm_status metrics(int inst, mpm_metrics* m) { m->mass = steps[inst]; return MPM_OK; }
    mpm_status health(std::vector<int32_t>& st) {
        assert(st.size() == caps.size());
        for (size_t i = 0; i < caps.size(); ++i) st[i] = caps[i] == bad_tag ? MPM_NUMERIC : MPM_OK;
        return MPM_OK;
    }
    // a checkpoint of the fake: the instance's tag and step count
    mpm_status save(int inst, std::vector<unsigned char>* buf) {
        const int64_t v[2] = {caps[inst], steps[inst]};
        buf->assign((const unsigned char*)v, (const unsigned char*)v + sizeof(v));
        ++saves;
        return MPM_OK;
    }
    mpm_status restore(int inst, const std::vector<unsigned char>& buf, int64_t* np) {
        int64_t v[2];
        assert(buf.size() == sizeof(v));
        std::memcpy(v, buf.data(), sizeof(v));
        assert(v[0] == caps[inst]);
        steps[inst] = (int)v[1];
        *np = caps[inst];
        ++restores;
        return MPM_OK;
    }
    int saves = 0, restores = 0;
};

static mpm_request req(int cells_x, int nsteps) {
    mpm_request r{};
    r.params.nx = 16; r.params.ny = 16; r.params.nz = 16;
    r.c1[0] = cells_x; r.c1[1] = 1; r.c1[2] = 1;
    r.ppc = 1; r.nsteps = nsteps; r.dt = 1e-9;
    return r;
}

int main() {
    double now = 0.0;
    Pools pools;
    pools.particles = 1000; pools.nodes = 1 << 20; pools.keys = 1 << 20; pools.bins = 1 << 20;
    int32_t nres = 0;
    mpm_result r;

    // 1. a workpiece that fails is ended FAILED and dropped; the others run on
    {
        FaultyOps ops;
        ops.bad_tag = 20;
        Scheduler<FaultyOps> s(&ops, pools, 10, 8, [&]() { now += 1.0; return now; });
        int64_t a, b, c;
        s.submit(req(10, 30), &a);
        s.submit(req(20, 30), &b);   // fails at its first step
        s.submit(req(30, 30), &c);
        assert(s.tick(&nres) == MPM_OK && nres == 3);
        s.poll(b, &r);
        assert(r.state == MPM_REQ_FAILED && r.status == MPM_NUMERIC && r.steps_done == 10);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_RUNNING && r.steps_done == 10);
        assert(s.tick(&nres) == MPM_OK && nres == 2);        // evicted
        assert(ops.removed_tags.size() == 1 && ops.removed_tags[0] == 20);
        assert(s.tick(&nres) == MPM_OK);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_DONE && r.steps_done == 30 && r.metrics.mass == 30);
        s.poll(c, &r);
        assert(r.state == MPM_REQ_DONE && r.metrics.mass == 30);
        mpm_server_stats st = s.stats();
        assert(st.completed == 2 && st.failed == 1 && st.cancelled == 0);
        assert(st.particle_updates == 10 * 30 + 20 * 10 + 30 * 30);
    }
    // 2. cancel: a queued request leaves at once, a running one at the next tick
    {
        FaultyOps ops;
        Scheduler<FaultyOps> s(&ops, pools, 10, 1, [&]() { now += 1.0; return now; });
        int64_t a, b;
        s.submit(req(10, 100), &a);
        s.submit(req(20, 100), &b);
        assert(s.cancel(b) == MPM_OK);
        s.poll(b, &r);
        assert(r.state == MPM_REQ_CANCELLED && r.status == MPM_CANCELLED && r.steps_done == 0);
        assert(s.tick(&nres) == MPM_OK && nres == 1);
        assert(s.cancel(a) == MPM_OK);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_RUNNING);                  // still resident until the next tick
        assert(s.tick(&nres) == MPM_OK && nres == 0);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_CANCELLED && r.steps_done == 10);
        assert(ops.removed_tags.size() == 1 && ops.removed_tags[0] == 10);
        assert(s.cancel(a) == MPM_OK);                       // an ended request keeps its state
        s.poll(a, &r);
        assert(r.state == MPM_REQ_CANCELLED);
        assert(s.cancel(12345) == MPM_INVALID_ARG);
        mpm_request nan_t0 = req(5, 10);
        nan_t0.T0 = std::nan("");
        assert(s.submit(nan_t0, &b) == MPM_INVALID_ARG);     // refused at the door
        mpm_server_stats st = s.stats();
        assert(st.cancelled == 2 && st.completed == 0 && st.queued == 0);
    }
    // 3. an instance change that fails (out of memory) admits nothing and keeps
    //    the queue in arrival order; the next tick admits the same requests
    {
        FaultyOps ops;
        Scheduler<FaultyOps> s(&ops, pools, 10, 8, [&]() { now += 1.0; return now; });
        int64_t a, b;
        s.submit(req(10, 10), &a);
        s.submit(req(20, 10), &b);
        ops.oom_changes = 1;
        assert(s.tick(&nres) == MPM_OOM);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_QUEUED);
        assert(s.stats().queued == 2 && s.stats().resident == 0);
        assert(s.tick(&nres) == MPM_OK && nres == 2);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_DONE && r.metrics.mass == 10);
        s.poll(b, &r);
        assert(r.state == MPM_REQ_DONE && r.metrics.mass == 10);
    }
    // 4. preemption: the workpiece is saved, dropped and queued behind the
    //    others, then restored and run to its full step count
    {
        FaultyOps ops;
        pools.particles = 35;     // 20 + 10 fit; 20 + 10 + 15 do not
        Scheduler<FaultyOps> s(&ops, pools, 10, 8, [&]() { now += 1.0; return now; });
        int64_t a, b, c;
        s.submit(req(20, 30), &a);
        s.submit(req(10, 30), &b);
        assert(s.tick(&nres) == MPM_OK && nres == 2);
        s.submit(req(15, 20), &c);                      // waits: 45 > 35
        assert(s.preempt(c) == MPM_INVALID_ARG);         // not running
        assert(s.preempt(a) == MPM_OK);
        assert(s.tick(&nres) == MPM_OK);                 // a saved (10 steps) and queued behind c
        assert(ops.saves == 1);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_QUEUED && r.steps_done == 10);
        s.poll(c, &r);
        assert(r.state == MPM_REQ_RUNNING);
        for (int t = 0; t < 10; ++t) s.tick(&nres);
        s.poll(a, &r);
        assert(r.state == MPM_REQ_DONE && r.steps_done == 30 && r.metrics.mass == 30 && ops.restores == 1);
        s.poll(b, &r);
        assert(r.state == MPM_REQ_DONE && r.metrics.mass == 30);
        s.poll(c, &r);
        assert(r.state == MPM_REQ_DONE && r.metrics.mass == 20);
        assert(s.stats().preempted == 1 && s.stats().completed == 3);
    }
    std::printf("OK\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_scheduler_faults_on_the_host(tmp_path):
    """Fault injection without a GPU: a workpiece whose error word is set ends
    FAILED (MPM_NUMERIC) and is dropped while the others finish with their full
    step counts; cancel ends a queued request at once and a running one at the
    next tick; a request with a NaN initial temperature is refused; an instance
    change that fails like an out-of-memory allocator leaves the queue intact
    for the next tick; a preempted request is saved, queued behind the waiting
    ones and resumed from its checkpoint to its full step count."""
    src = tmp_path / "faults.cpp"
    src.write_text(FAULTS)
    exe = tmp_path / "faults"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(CORE), "-I", str(ROOT / "include"),
                        str(src), "-o", str(exe), "-pthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stderr


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_server_structs_match_ctypes(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(SIZES)
    exe = tmp_path / "sizes"
    r = subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    want = [C.sizeof(A.MpmRequest), C.sizeof(A.MpmResult), C.sizeof(A.MpmServerConfig), C.sizeof(A.MpmServerStats),
            A.MpmRequest.seed.offset, A.MpmRequest.dt.offset, A.MpmResult.metrics.offset]
    assert got == want


def test_footprint_is_host_arithmetic():
    """mpm_server_footprint needs no device: bytes = particles x state bytes +
    nodes x grid bytes + keys x 8 + bins x 40 (FP32 state: 13 vectors of 16 B
    per particle and buffer)."""
    from mpm_b200 import workpiece as W
    from mpm_b200.solver import make_request
    case = W.config1(cells=(16, 16, 16))
    cfg = A.MpmServerConfig(A.PREC_F32, 50, 1 << 30, 0, 0, 0, 0)
    r = make_request(case, 100)
    b = C.c_int64()
    assert A.lib().mpm_server_footprint(C.byref(cfg), C.byref(r), C.byref(b)) == A.MPM_OK
    p = case["params"]
    nodes = p["nx"] * p["ny"] * p["nz"]
    bins = ((p["nx"] + 3) // 4) * ((p["ny"] + 3) // 4) * ((p["nz"] + 3) // 4)
    particles = 16 ** 3 * 8
    per_particle = 2 * (13 * 16 + 4 + 2 + 16) + 36 + 8   # 12 state vectors + the position low parts, permutation
    # per node: two 16 B grids, an int32 tool mask, three FP32 heat-conduction arrays
    want = particles * per_particle + nodes * (36 + 12) + (bins * 64 + 2) * 8 + bins * 40
    assert abs(b.value - want) <= 1


def test_deterministic_footprint_counts_the_mode_scratch():
    """A deterministic server counts the mode's escaped fixed-point sums (5 x
    8 B per grid node) and, per bin, its stored node tile (5 x 216 FP32
    values) and escape mark (4 B)."""
    from mpm_b200 import workpiece as W
    from mpm_b200.solver import make_request
    case = W.config1(cells=(16, 16, 16))
    r = make_request(case, 100)
    got = []
    for det in (0, 1):
        cfg = A.MpmServerConfig(A.PREC_F32, 50, 1 << 30, 0, 0, 0, det, 0)
        b = C.c_int64()
        assert A.lib().mpm_server_footprint(C.byref(cfg), C.byref(r), C.byref(b)) == A.MPM_OK
        got.append(b.value)
    p = r.params
    nodes = p.nx * p.ny * p.nz
    bins = -(-p.nx // 4) * -(-p.ny // 4) * -(-p.nz // 4)
    assert abs(got[1] - got[0] - (nodes * 40 + bins * (5 * 216 * 4 + 4))) <= 1
