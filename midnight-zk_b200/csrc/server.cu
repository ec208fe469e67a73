// server.cu — a proving service over the device proof core.
//
// Requests (one proof each, any registered k) are queued by any number of
// host threads and served by `lanes` worker threads, each with its own device
// context (stream and scratch arena).  An idle lane takes a wave: queued
// requests, oldest first, while the wave holds fewer than `max_batch` proofs
// and the device scratch of every proof in flight (all lanes) stays within
// the memory budget; it runs the wave as ONE mixed-k call of the proof core,
// in which the witness commitments of all its proofs form one batched MSM and
// the quotient-limb commitments another.  Requests that arrive while a wave is
// on the GPU are taken by the next free lane at once, so their kernels run
// beside the running wave's on the device and fill what one wave leaves idle
// (the host-side tails of a wave included): continuous batching.  With
// max_batch = 1 and one lane the same service is the plain
// one-proof-at-a-time prover.  Latency is measured from submit to the moment
// the wave that holds the request has its results on the host.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mzk.h"
#include "ntt.hpp"
#include "quotient.hpp"
#include "runtime.hpp"

namespace mzk {

// access to the context internals of capi.cu
Context* context_of(mzk_ctx* ctx);
const Domain* domain_of(mzk_domain* d);

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct ServerKey {
    const Domain* dom;
    mzk_proving_key_desc pk;
    uint64_t job_bytes;  // device scratch of one proof of this k
};

struct Request {
    uint32_t k = 0;
    mzk_proof_job job;
    double t_submit = 0, t_done = 0;
    int status = OK;
    std::string error;
    bool done = false;
    uint64_t out[kProofCoreCommitments * 18];
};

}  // namespace

struct Server {
    std::vector<mzk_ctx*> lanes;  // one device context per worker
    uint32_t max_batch = 1;
    uint32_t flags = 0;       // MZK_PROVE_* flags of every wave
    uint64_t mem_budget = 0;  // 0: no limit
    std::map<uint32_t, ServerKey> keys;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_ticket = 1;
    uint64_t in_flight_bytes = 0;
    bool stop = false;
    uint64_t waves = 0, proofs = 0;
    double busy_ms = 0;
    std::vector<std::thread> workers;

    // the next wave for an idle lane; called with mu held.  Empty when the
    // head of the queue does not fit in the memory left by the waves in flight.
    std::vector<uint64_t> take_wave(uint64_t* bytes) {
        std::vector<uint64_t> batch;
        *bytes = 0;
        // one wave takes at most its lane's share of the budget, so the other
        // lanes can admit requests beside it
        const uint64_t lane_cap = mem_budget / lanes.size();
        while (!queue.empty() && batch.size() < max_batch) {
            const ServerKey& key = keys[reqs[queue.front()]->k];
            const uint64_t wave_after = *bytes + key.job_bytes;
            // the first proof of a wave is admitted when nothing else is in flight,
            // so a proof larger than the budget still runs (alone)
            const bool fits = mem_budget == 0 ||
                              (in_flight_bytes + wave_after <= mem_budget && wave_after <= lane_cap) ||
                              (in_flight_bytes == 0 && batch.empty());
            if (!fits) break;
            *bytes += key.job_bytes;
            batch.push_back(queue.front());
            queue.pop_front();
        }
        return batch;
    }

    void run(mzk_ctx* lane) {
        Context* ctx = context_of(lane);
        cudaSetDevice(ctx->device);
        for (;;) {
            std::vector<uint64_t> batch;
            std::vector<mzk_proof_job> jobs;
            std::vector<const Domain*> doms;
            std::vector<const mzk_proving_key_desc*> pks;
            uint64_t bytes = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    if (stop && queue.empty()) return true;
                    if (queue.empty()) return false;
                    batch = take_wave(&bytes);
                    return !batch.empty();
                });
                if (batch.empty()) return;  // stop requested and nothing left
                in_flight_bytes += bytes;
                for (uint64_t t : batch) {
                    const Request& r = *reqs[t];
                    const ServerKey& key = keys[r.k];
                    jobs.push_back(r.job);
                    doms.push_back(key.dom);
                    pks.push_back(&key.pk);
                }
            }
            std::vector<uint64_t> out(batch.size() * kProofCoreCommitments * 18);
            const double t0 = now_ms();
            Status st;
            std::string err;
            {
                std::lock_guard<std::recursive_mutex> g(ctx->mu);
                st = prove_core_multi(ctx, doms.data(), pks.data(), jobs.data(), jobs.size(), out.data(), flags,
                                      ctx->stream);
                if (st == OK) {
                    cudaError_t e = cudaStreamSynchronize(ctx->stream);
                    if (e != cudaSuccess) {
                        st = ERR_CUDA;
                        set_error(std::string("server wave: ") + cudaGetErrorString(e));
                    }
                }
                if (st != OK) err = mzk_last_error();
            }
            const double t1 = now_ms();
            {
                std::lock_guard<std::mutex> lk(mu);
                in_flight_bytes -= bytes;
                waves++;
                proofs += batch.size();
                busy_ms += t1 - t0;
                for (size_t i = 0; i < batch.size(); i++) {
                    Request& r = *reqs[batch[i]];
                    std::memcpy(r.out, out.data() + i * kProofCoreCommitments * 18, sizeof(r.out));
                    r.status = st;
                    r.error = err;
                    r.t_done = t1;
                    r.done = true;
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();  // memory came free: another lane may admit now
        }
    }
};

}  // namespace mzk

struct mzk_server {
    mzk::Server impl;
};

namespace {

// device scratch of one proof of size 2^k in the proof core: coefficient and
// extended forms of seven polynomials, three delta forms, four limbs, three
// device-derived columns (z, h, Z), plus the
// sorted MSM entries it contributes to the batched witness MSM (the largest
// of the two batched MSMs)
uint64_t job_scratch_bytes(const mzk::Domain* d) {
    const uint64_t n = 1ull << d->k, en = 1ull << d->ext_k;
    const uint64_t fr = 32;
    const uint64_t polys = (7 * n + 7 * en + 3 * n + 4 * n + 3 * n) * fr;
    const uint64_t msm = 7 * n * 20 * 4;  // sorted entries of 7 MSMs (<= 20 windows)
    return polys + msm;
}

}  // namespace

// these entry points are declared in include/mzk.h
extern "C" {

int mzk_server_create(mzk_ctx* ctx, uint32_t max_batch, uint32_t lanes, uint64_t mem_budget_bytes,
                      uint32_t flags, mzk_server** out);
int mzk_server_add_key(mzk_server* s, mzk_domain* d, const mzk_proving_key_desc* pk);
int mzk_server_submit(mzk_server* s, uint32_t k, const mzk_proof_job* job, uint64_t* ticket);
int mzk_server_wait(mzk_server* s, uint64_t ticket, uint64_t* out, double* latency_ms);
int mzk_server_stats(mzk_server* s, uint64_t* waves, uint64_t* proofs, double* busy_ms);
int mzk_server_destroy(mzk_server* s);

}  // extern "C"

extern "C" int mzk_server_create(mzk_ctx* ctx, uint32_t max_batch, uint32_t lanes, uint64_t mem_budget_bytes,
                                 uint32_t flags, mzk_server** out) {
    if (!ctx || !out || max_batch == 0 || lanes == 0 || lanes > 8) {
        mzk::set_error("server: need a context, max_batch >= 1 and 1..8 lanes");
        return mzk::ERR_ARG;
    }
    *out = nullptr;
    mzk_server* s = new mzk_server;
    s->impl.max_batch = max_batch;
    s->impl.mem_budget = mem_budget_bytes;
    s->impl.flags = flags;
    const int device = mzk::context_of(ctx)->device;
    for (uint32_t i = 0; i < lanes; i++) {
        mzk_ctx* lane = nullptr;
        if (int st = mzk_ctx_create(device, &lane)) {
            for (mzk_ctx* c : s->impl.lanes) mzk_ctx_destroy(c);
            delete s;
            return st;
        }
        s->impl.lanes.push_back(lane);
    }
    for (mzk_ctx* lane : s->impl.lanes) s->impl.workers.emplace_back([s, lane] { s->impl.run(lane); });
    *out = s;
    return mzk::OK;
}

extern "C" int mzk_server_add_key(mzk_server* s, mzk_domain* d, const mzk_proving_key_desc* pk) {
    if (!s || !d || !pk) return mzk::ERR_ARG;
    const mzk::Domain* dom = mzk::domain_of(d);
    if (pk->k != dom->k) {
        mzk::set_error("server: key and domain sizes differ");
        return mzk::ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(s->impl.mu);
    s->impl.keys[pk->k] = mzk::ServerKey{dom, *pk, job_scratch_bytes(dom)};
    return mzk::OK;
}

extern "C" int mzk_server_submit(mzk_server* s, uint32_t k, const mzk_proof_job* job, uint64_t* ticket) {
    if (!s || !job || !ticket) return mzk::ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(s->impl.mu);
        if (!s->impl.keys.count(k)) {
            mzk::set_error("server: no key registered for k = " + std::to_string(k));
            return mzk::ERR_ARG;
        }
        auto r = std::make_unique<mzk::Request>();
        r->k = k;
        r->job = *job;
        r->t_submit = mzk::now_ms();
        const uint64_t t = s->impl.next_ticket++;
        s->impl.reqs[t] = std::move(r);
        s->impl.queue.push_back(t);
        *ticket = t;
    }
    s->impl.cv_work.notify_one();
    return mzk::OK;
}

extern "C" int mzk_server_wait(mzk_server* s, uint64_t ticket, uint64_t* out, double* latency_ms) {
    if (!s) return mzk::ERR_ARG;
    std::unique_lock<std::mutex> lk(s->impl.mu);
    auto it = s->impl.reqs.find(ticket);
    if (it == s->impl.reqs.end()) {
        mzk::set_error("server: unknown ticket");
        return mzk::ERR_ARG;
    }
    mzk::Request* r = it->second.get();
    s->impl.cv_done.wait(lk, [&] { return r->done; });
    const int st = r->status;
    if (st != mzk::OK) mzk::set_error(r->error);
    if (out) std::memcpy(out, r->out, sizeof(r->out));
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
    s->impl.reqs.erase(it);
    return st;
}

extern "C" int mzk_server_stats(mzk_server* s, uint64_t* waves, uint64_t* proofs, double* busy_ms) {
    if (!s) return mzk::ERR_ARG;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    if (waves) *waves = s->impl.waves;
    if (proofs) *proofs = s->impl.proofs;
    if (busy_ms) *busy_ms = s->impl.busy_ms;
    return mzk::OK;
}

extern "C" int mzk_server_destroy(mzk_server* s) {
    if (!s) return mzk::OK;
    {
        std::lock_guard<std::mutex> lk(s->impl.mu);
        s->impl.stop = true;
    }
    s->impl.cv_work.notify_all();
    for (std::thread& w : s->impl.workers)
        if (w.joinable()) w.join();
    for (mzk_ctx* c : s->impl.lanes) mzk_ctx_destroy(c);
    delete s;
    return mzk::OK;
}
