// mpm_server_core.h -- scheduling of the serving loop (host code only, no CUDA).
//
// Requests (a workpiece, its tool, a step count) arrive at any time through
// submit().  Every tick():
//   1. drops the requests that finished in the previous tick from the engine;
//   2. admits queued requests in arrival order while their device footprint
//      fits the pools reserved from the HBM budget (no request overtakes an
//      earlier one);
//   3. adds the admitted ones to the engine in one instance change and
//      generates their particles;
//   4. steps every resident request by k = min(max_chunk, fewest remaining
//      steps of any resident request) in one engine step call, so requests
//      admitted while others run share their launches from then on;
//   5. reads the engine's per-instance status: a request whose workpiece
//      failed (MPM_NUMERIC) ends FAILED and is dropped by the next tick's
//      step 1, while the others run on;
//   6. records the metrics of every request that reached its step count.
// cancel() ends a queued request at once and marks a running one, which the
// next tick's step 1 drops.  preempt() marks a running request: the next
// tick's step 1 saves its workpiece to host memory (a checkpoint), drops it
// from the device and queues it again at the back; when it is admitted again
// its checkpoint is loaded in place of a new workpiece, so it resumes where
// it stopped.  The engine is a template parameter: the GPU engine in the
// library, a fake in the host tests.  submit(), poll(), cancel() and
// preempt() may run on other threads than tick().
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/mpm_capi.h"

namespace mpmb {

// Pool entries one request holds while resident.
struct Footprint {
    int64_t particles = 0, nodes = 0, keys = 0, bins = 0;
};

inline Footprint request_footprint(const mpm_request& r) {
    Footprint f;
    int64_t cells = 1;
    for (int a = 0; a < 3; ++a) cells *= std::max<int64_t>(0, (int64_t)r.c1[a] - r.c0[a]);
    f.particles = cells * std::max(r.ppc, 0);
    f.nodes = (int64_t)r.params.nx * r.params.ny * r.params.nz;
    f.bins = (int64_t)((r.params.nx + 3) / 4) * ((r.params.ny + 3) / 4) * ((r.params.nz + 3) / 4);
    f.keys = f.bins * 64 + 2;
    return f;
}

// Device bytes of one pool entry (both state buffers, sort scratch).
struct PoolBytes {
    double particle, node, key, bin;
};

inline PoolBytes pool_bytes(int precision, bool backstress, bool deterministic = false) {
    const double v4 = precision == MPM_PREC_F64 ? 32.0 : 16.0, r = precision == MPM_PREC_F64 ? 8.0 : 4.0;
    PoolBytes b;
    // A0-A5, B0-B3, S0-S1 (+K0-K1), X (FP32 only), sres, status, shear
    // counter, id, bin, orig, re-bin key; two buffers; sort key, rank, new
    // bin (int32) and the FP64 position scratch
    const double nv4 = 12.0 + (backstress ? 2.0 : 0.0) + (precision == MPM_PREC_F64 ? 0.0 : 1.0);
    b.particle = 2.0 * (nv4 * v4 + r + 2.0 + 16.0) + 12.0 + 24.0 + 8.0;   // + the re-bin permutation and keys
    b.node = 2.0 * v4 + 3.0 * r + 4.0;   // two grid buffers, three heat-conduction arrays, tool mask (int32)
    b.key = 8.0;                 // count and offset
    b.bin = 40.0;                // bin tables, flags and the work item
    // deterministic mode: the escaped fixed-point sums (5 x int64 per node),
    // each work item's stored node tile (5 x 216 reals) and its escape mark
    if (deterministic) {
        b.node += 5.0 * 8.0;
        b.bin += 5.0 * 216.0 * r + 4.0;
    }
    return b;
}

// The budget split between the pools (shares of hbm_budget_bytes).
struct Pools {
    int64_t particles = 0, nodes = 0, keys = 0, bins = 0;
    bool fits(const Footprint& used, const Footprint& f) const {
        return used.particles + f.particles <= particles && used.nodes + f.nodes <= nodes &&
               used.keys + f.keys <= keys && used.bins + f.bins <= bins;
    }
};

inline Pools pools_for_budget(int64_t budget, int precision, bool backstress, bool deterministic = false) {
    const PoolBytes b = pool_bytes(precision, backstress, deterministic);
    Pools p;
    p.particles = (int64_t)(0.88 * (double)budget / b.particle);
    p.nodes = (int64_t)(0.08 * (double)budget / b.node);
    p.keys = (int64_t)(0.03 * (double)budget / b.key);
    p.bins = (int64_t)(0.005 * (double)budget / b.bin);
    return p;
}

template <class Engine>
class Scheduler {
   public:
    struct Req {
        int64_t id = 0;
        mpm_request r{};
        Footprint f;
        mpm_result res{};
        bool cancel = false;   // cancelled while resident: dropped by the next tick
        bool preempt = false;  // preempted while resident: saved and requeued by the next tick
        std::vector<unsigned char> ckpt;   // the saved workpiece of a preempted request
    };

    Scheduler(Engine* eng, Pools pools, int max_chunk, int max_resident, std::function<double()> clock,
              int64_t max_resident_particles = 0)
        : eng_(eng), pools_(pools), max_chunk_(max_chunk > 0 ? max_chunk : 50),
          max_resident_(max_resident > 0 ? max_resident : 4096), clock_(std::move(clock)),
          max_particles_(max_resident_particles) {}

    // Queues a request (stamped with the clock); MPM_CAPACITY when it could
    // never fit the pools.
    mpm_status submit(const mpm_request& r, int64_t* id) {
        const Footprint f = request_footprint(r);
        if (!pools_.fits(Footprint{}, f)) return MPM_CAPACITY;
        if (r.nsteps < 0 || !(r.dt > 0.0) || !std::isfinite(r.dt) || r.ppc <= 0 || !std::isfinite(r.T0))
            return MPM_INVALID_ARG;
        std::lock_guard<std::mutex> lock(mu_);
        Req q;
        q.id = next_id_++;
        q.r = r;
        q.f = f;
        q.res.state = MPM_REQ_QUEUED;
        q.res.t_submit = clock_();
        all_[q.id] = q;
        queue_.push_back(q.id);
        ++stats_.offered;
        if (id) *id = q.id;
        return MPM_OK;
    }

    mpm_status poll(int64_t id, mpm_result* out) {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = all_.find(id);
        if (it == all_.end()) return MPM_INVALID_ARG;
        *out = it->second.res;
        return MPM_OK;
    }

    // Cancels a request (see the file comment); MPM_INVALID_ARG for an unknown id.
    mpm_status cancel(int64_t id) {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = all_.find(id);
        if (it == all_.end()) return MPM_INVALID_ARG;
        Req& q = it->second;
        if (q.res.state == MPM_REQ_QUEUED) {
            queue_.erase(std::find(queue_.begin(), queue_.end(), id));
            end_cancelled(q);
        } else if (q.res.state == MPM_REQ_RUNNING) {
            q.cancel = true;
        }
        return MPM_OK;
    }

    // Preempts a running request (see the file comment); MPM_INVALID_ARG for
    // an unknown id or a request that is not running.
    mpm_status preempt(int64_t id) {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = all_.find(id);
        if (it == all_.end() || it->second.res.state != MPM_REQ_RUNNING) return MPM_INVALID_ARG;
        it->second.preempt = true;
        return MPM_OK;
    }

    mpm_server_stats stats() {
        std::lock_guard<std::mutex> lock(mu_);
        mpm_server_stats s = stats_;
        s.queued = (int64_t)queue_.size();
        s.resident = (int64_t)resident_.size();
        s.resident_particles = used_.particles;
        return s;
    }

    // One scheduling round (see the file comment).  Returns the engine's
    // status of a failed step (the requests stay resident and the call may
    // be repeated); per-request failures only mark that request FAILED.
    mpm_status tick(int32_t* n_resident) {
        const double t_in = clock_();
        // 1. retire finished requests
        std::vector<int32_t> remove;
        std::vector<int64_t> keep;
        Footprint used = used_;
        // preempted requests: save the workpiece while it is still resident
        for (size_t i = 0; i < resident_.size(); ++i) {
            Req& q = ref(resident_[i]);
            bool pre;
            {
                std::lock_guard<std::mutex> lock(mu_);
                pre = q.res.state == MPM_REQ_RUNNING && q.preempt && !q.cancel;
            }
            if (!pre) continue;
            std::vector<unsigned char> buf;
            const mpm_status s = eng_->save((int)i, &buf);
            std::lock_guard<std::mutex> lock(mu_);
            q.preempt = false;
            if (s != MPM_OK) continue;   // stays resident; a later preempt may retry
            q.ckpt = std::move(buf);
            q.res.state = MPM_REQ_QUEUED;
            queue_.push_back(q.id);
            ++stats_.preempted;
        }
        {
            std::lock_guard<std::mutex> lock(mu_);
            for (size_t i = 0; i < resident_.size(); ++i) {
                Req& q = all_[resident_[i]];
                if (q.res.state == MPM_REQ_RUNNING && q.cancel) end_cancelled(q);
                if (q.res.state != MPM_REQ_RUNNING) {
                    remove.push_back((int32_t)i);
                    sub(used, q.f);
                } else {
                    keep.push_back(resident_[i]);
                }
            }
        }
        // 2. admit in arrival order
        std::vector<int64_t> add;
        {
            std::lock_guard<std::mutex> lock(mu_);
            while (!queue_.empty() && keep.size() + add.size() < (size_t)max_resident_) {
                Req& q = all_[queue_.front()];
                if (!pools_.fits(used, q.f)) break;
                // the resident-particle cap never keeps the device empty
                const bool empty = keep.empty() && add.empty();
                if (max_particles_ > 0 && !empty && used.particles + q.f.particles > max_particles_) break;
                addf(used, q.f);
                add.push_back(q.id);
                queue_.pop_front();
            }
        }
        // 3. one instance change, then the new workpieces
        if (!remove.empty() || !add.empty()) {
            std::vector<mpm_params> ap;
            std::vector<int64_t> ac;
            for (int64_t id : add) {
                ap.push_back(ref(id).r.params);
                ac.push_back(ref(id).f.particles);
            }
            int first = 0;
            mpm_status s = eng_->change(ap, ac, remove, &first);
            if (s != MPM_OK) {
                // nothing changed on the device: put the admitted requests back
                std::lock_guard<std::mutex> lock(mu_);
                for (auto it = add.rbegin(); it != add.rend(); ++it) queue_.push_front(*it);
                return s;
            }
            resident_ = keep;
            used_ = used;
            for (size_t k = 0; k < add.size(); ++k) {
                Req& q = ref(add[k]);
                resident_.push_back(q.id);
                int64_t np = 0;
                const bool resume = !q.ckpt.empty();
                mpm_status si = resume ? eng_->restore(first + (int)k, q.ckpt, &np)
                                       : eng_->init(first + (int)k, q.r, &np);
                std::lock_guard<std::mutex> lock(mu_);
                if (resume) {
                    std::vector<unsigned char>().swap(q.ckpt);   // the host copy is no longer needed
                } else {
                    q.res.t_admit = clock_();
                }
                q.res.n_particles = np;
                if (si != MPM_OK) {
                    q.res.state = MPM_REQ_FAILED;
                    q.res.status = si;
                    ++stats_.failed;
                } else {
                    q.res.state = MPM_REQ_RUNNING;
                    ++stats_.admitted;
                }
            }
        }
        // 4. step every running request
        int k = max_chunk_;
        int running = 0;
        for (int64_t id : resident_) {
            const Req& q = ref(id);
            if (q.res.state != MPM_REQ_RUNNING) continue;
            ++running;
            k = std::min<int64_t>(k, q.r.nsteps - q.res.steps_done);
        }
        std::vector<int32_t> health(resident_.size(), MPM_OK);
        if (running > 0 && k > 0) {
            std::vector<double> dts;
            for (int64_t id : resident_) dts.push_back(ref(id).r.dt);
            mpm_status s = eng_->step(k, dts);
            if (s != MPM_OK) return s;
            // 5. per-workpiece failures
            s = eng_->health(health);
            if (s != MPM_OK) return s;
        }
        // 6. completions
        for (size_t i = 0; i < resident_.size(); ++i) {
            Req& q = ref(resident_[i]);
            if (q.res.state != MPM_REQ_RUNNING) continue;
            const int kk = running > 0 ? std::max(k, 0) : 0;
            if (health[i] != MPM_OK) {
                std::lock_guard<std::mutex> lock(mu_);
                q.res.steps_done += kk;
                stats_.particle_updates += q.res.n_particles * kk;
                q.res.t_done = clock_();
                q.res.state = MPM_REQ_FAILED;
                q.res.status = health[i];
                ++stats_.failed;
                continue;
            }
            mpm_metrics m{};
            mpm_status sm = MPM_OK;
            const bool done = q.res.steps_done + kk >= q.r.nsteps;
            if (done) sm = eng_->metrics((int)i, &m);
            std::lock_guard<std::mutex> lock(mu_);
            q.res.steps_done += kk;
            stats_.particle_updates += q.res.n_particles * kk;
            if (done) {
                q.res.t_done = clock_();
                q.res.metrics = m;
                q.res.state = sm == MPM_OK ? MPM_REQ_DONE : MPM_REQ_FAILED;
                q.res.status = sm;
                if (sm == MPM_OK) ++stats_.completed; else ++stats_.failed;
            }
        }
        {
            std::lock_guard<std::mutex> lock(mu_);
            ++stats_.ticks;
            stats_.busy_seconds += clock_() - t_in;
        }
        if (n_resident) *n_resident = (int32_t)resident_.size();
        return MPM_OK;
    }

   private:
    // (mu_ held)
    void end_cancelled(Req& q) {
        q.res.state = MPM_REQ_CANCELLED;
        q.res.status = MPM_CANCELLED;
        q.res.t_done = clock_();
        std::vector<unsigned char>().swap(q.ckpt);
        ++stats_.cancelled;
    }
    Req& ref(int64_t id) {
        std::lock_guard<std::mutex> lock(mu_);
        return all_[id];
    }
    static void addf(Footprint& a, const Footprint& b) {
        a.particles += b.particles; a.nodes += b.nodes; a.keys += b.keys; a.bins += b.bins;
    }
    static void sub(Footprint& a, const Footprint& b) {
        a.particles -= b.particles; a.nodes -= b.nodes; a.keys -= b.keys; a.bins -= b.bins;
    }

    Engine* eng_;
    Pools pools_;
    int max_chunk_, max_resident_;
    std::function<double()> clock_;
    int64_t max_particles_ = 0;
    std::mutex mu_;
    std::unordered_map<int64_t, Req> all_;
    std::deque<int64_t> queue_;
    std::vector<int64_t> resident_;   // request ids in engine instance order
    Footprint used_;
    int64_t next_id_ = 1;
    mpm_server_stats stats_{};
};

}  // namespace mpmb
