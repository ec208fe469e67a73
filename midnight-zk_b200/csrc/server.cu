// server.cu — a proving service over create_proof.
//
// Requests (one proof each: a key, the witness, the blinding values and the
// output buffer of its transcript) are queued by any number of host threads
// and served by `lanes` worker threads, each with its own device context
// (stream and scratch arena).  An idle lane takes a wave: queued requests,
// oldest first, over the SRS buffer of the first, while the wave holds fewer
// than `max_batch` proofs and the device scratch of every proof in flight
// (all lanes) stays within the memory budget; it runs the wave as ONE
// create_proof call, in which every Fiat-Shamir phase runs for all proofs of
// the wave with its MSMs as one batched MSM.  A wave stops at its host-side
// steps (transcript hashing between phases, the window tails of its MSMs);
// requests that arrive meanwhile are taken by the next free lane at once, so
// their kernels fill what the first wave leaves idle: continuous batching.
// With max_batch = 1 and one lane the same service is the plain
// one-proof-at-a-time prover.  Latency is measured from submit to the moment
// the wave that holds the request has its transcript on the host.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mzk.h"
#include "quotient.hpp"
#include "runtime.hpp"

namespace mzk {

// access to the context internals of capi.cu
Context* context_of(mzk_ctx* ctx);

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    mzk_proof_request req;
    const void* srs = nullptr;  // the SRS buffer of its key (waves share one)
    uint64_t bytes = 0;         // device scratch of the proof
    uint64_t rows = 0;          // 2^k of its key
    double t_submit = 0, t_done = 0;
    int status = OK;
    std::string error;
    bool done = false;
};

}  // namespace

struct Server {
    std::vector<mzk_ctx*> lanes;  // one device context per worker
    uint32_t max_batch = 1;
    uint32_t flags = 0;       // MZK_PROVE_* flags of every wave
    uint64_t mem_budget = 0;  // 0: no limit
    uint64_t max_wave_rows = 0;  // 0: no limit on the rows (sum of 2^k) of one wave
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
        uint64_t rows = 0;
        // one wave takes at most its lane's share of the budget, so the other
        // lanes can admit requests beside it
        const uint64_t lane_cap = mem_budget / lanes.size();
        const void* srs = queue.empty() ? nullptr : reqs[queue.front()]->srs;
        for (auto it = queue.begin(); it != queue.end() && batch.size() < max_batch;) {
            const Request& r = *reqs[*it];
            if (r.srs != srs) {  // keys over another SRS buffer go in a wave of their own
                ++it;
                continue;
            }
            // a wave's duration grows with its rows: the cap keeps requests that
            // arrive meanwhile from waiting behind one long wave
            if (max_wave_rows && !batch.empty() && rows + r.rows > max_wave_rows) break;
            const uint64_t wave_after = *bytes + r.bytes;
            // the first proof of a wave is admitted when nothing else is in flight,
            // so a proof larger than the budget still runs (alone)
            const bool fits = mem_budget == 0 ||
                              (in_flight_bytes + wave_after <= mem_budget && wave_after <= lane_cap) ||
                              (in_flight_bytes == 0 && batch.empty());
            if (!fits) break;
            *bytes += r.bytes;
            rows += r.rows;
            batch.push_back(*it);
            it = queue.erase(it);
        }
        return batch;
    }

    void run(mzk_ctx* lane) {
        Context* ctx = context_of(lane);
        cudaSetDevice(ctx->device);
        for (;;) {
            std::vector<uint64_t> batch;
            std::vector<mzk_proof_request> wave;
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
                for (uint64_t t : batch) wave.push_back(reqs[t]->req);
            }
            const double t0 = now_ms();
            std::vector<Status> st(batch.size(), OK);
            std::vector<std::string> err(batch.size());
            {
                std::lock_guard<std::recursive_mutex> g(ctx->mu);
                const Status s = create_proofs(ctx, wave.data(), wave.size(), flags, ctx->stream);
                if (s != OK) {
                    cudaStreamSynchronize(ctx->stream);
                    // one bad request fails its whole call: prove the wave's
                    // requests one by one, so only the bad ones fail
                    for (size_t i = 0; i < wave.size(); i++) {
                        st[i] = wave.size() == 1 ? s : create_proofs(ctx, &wave[i], 1, flags, ctx->stream);
                        if (st[i] != OK) {
                            err[i] = mzk_last_error();
                            cudaStreamSynchronize(ctx->stream);
                        }
                    }
                }
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
                    r.status = st[i];
                    r.error = err[i];
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

extern "C" int mzk_server_set_wave_rows(mzk_server* s, uint64_t max_rows) {
    if (!s) return mzk::ERR_ARG;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    s->impl.max_wave_rows = max_rows;
    return mzk::OK;
}

extern "C" int mzk_server_submit(mzk_server* s, const mzk_proof_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket || !req->key || !req->advice || !req->blinds || !req->proof_out) {
        mzk::set_error("server: null argument");
        return mzk::ERR_ARG;
    }
    {
        std::lock_guard<std::mutex> lk(s->impl.mu);
        auto r = std::make_unique<mzk::Request>();
        r->req = *req;
        mzk_srs_desc srs;
        mzk_plonk_key_srs(req->key, &srs);
        r->srs = srs.srs;
        r->bytes = mzk::proof_device_bytes(req->key);
        r->rows = mzk::proof_rows(req->key);
        r->t_submit = mzk::now_ms();
        const uint64_t t = s->impl.next_ticket++;
        s->impl.reqs[t] = std::move(r);
        s->impl.queue.push_back(t);
        *ticket = t;
    }
    s->impl.cv_work.notify_one();
    return mzk::OK;
}

extern "C" int mzk_server_wait(mzk_server* s, uint64_t ticket, double* latency_ms) {
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
