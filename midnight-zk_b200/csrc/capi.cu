// capi.cu — the extern "C" boundary (include/mzk.h) and the device context.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/mzk.h"
#include "grand.hpp"
#include "host_ec.hpp"
#include "ntt.hpp"
#include "quotient.hpp"
#include "runtime.hpp"
#include "srs.hpp"

struct mzk_ctx {
    mzk::Context impl;
};

struct mzk_domain {
    mzk::Domain* impl = nullptr;
    mzk_ctx* ctx = nullptr;
};

namespace mzk {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

Status Context::ensure(const char* name, size_t bytes, void** out) {
    if (bytes == 0) bytes = 16;
    DevBuf& b = bufs[name];
    if (b.bytes >= bytes) {
        *out = b.p;
        return OK;
    }
    if (b.p) {
        // the old buffer may still be read by queued work on our streams
        cudaStreamSynchronize(stream);
        cudaStreamSynchronize(copy_stream);
        cudaFree(b.p);
        buf_generation++;  // captured graphs may hold the old address
        b.p = nullptr;
        b.bytes = 0;
        // a buffer that had to grow once tends to grow again (mixed sizes):
        // take 25 % headroom so repeated growth reallocates rarely
        bytes += bytes / 4;
    }
    bytes = (bytes + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        set_error(std::string("device allocation of ") + std::to_string(bytes) + " bytes for " + name + " failed: " +
                  cudaGetErrorString(e));
        return ERR_OOM;
    }
    b.bytes = bytes;
    *out = b.p;
    return OK;
}

Status Context::ensure_pinned(size_t bytes, void** out) {
    if (pinned_bytes >= bytes) {
        *out = pinned;
        return OK;
    }
    if (pinned) {
        cudaStreamSynchronize(stream);
        cudaFreeHost(pinned);
        pinned = nullptr;
        pinned_bytes = 0;
    }
    MZK_CUDA_CHECK(cudaMallocHost(&pinned, bytes));
    pinned_bytes = bytes;
    *out = pinned;
    return OK;
}

Status Context::phase_begin(int phase, cudaStream_t st) {
    if (!profiling) return OK;
    if (prof_used >= kMaxRecords) {
        set_error("profiling: too many open phases");
        return ERR_STATE;
    }
    for (int k = 0; k < 2; k++)
        if (!prof_ev[2 * prof_used + k]) MZK_CUDA_CHECK(cudaEventCreate(&prof_ev[2 * prof_used + k]));
    prof_phase[prof_used] = phase;
    MZK_CUDA_CHECK(cudaEventRecord(prof_ev[2 * prof_used], st));
    return OK;
}

Status Context::phase_end(cudaStream_t st) {
    if (!profiling) return OK;
    MZK_CUDA_CHECK(cudaEventRecord(prof_ev[2 * prof_used + 1], st));
    prof_used++;
    return OK;
}

void Context::phase_collect() {
    for (int i = 0; i < prof_used; i++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, prof_ev[2 * i], prof_ev[2 * i + 1]) == cudaSuccess) {
            phase_ms[prof_phase[i]] += ms;
            phase_count[prof_phase[i]]++;
        }
    }
    prof_used = 0;
}

Context::~Context() {
    if (stream) cudaStreamSynchronize(stream);
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
    for (auto& kv : bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    if (pinned) cudaFreeHost(pinned);
    if (gen_table) cudaFree(gen_table);
    for (cudaEvent_t ev : ev_copy)
        if (ev) cudaEventDestroy(ev);
    for (int i = 0; i < kMaxEvents; i++)
        if (prof_ev[i]) cudaEventDestroy(prof_ev[i]);
    if (stream) cudaStreamDestroy(stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
}

}  // namespace mzk

namespace mzk {
Context* context_of(mzk_ctx* ctx) { return &ctx->impl; }
const Domain* domain_of(mzk_domain* d) { return d->impl; }
}  // namespace mzk

using mzk::Status;

namespace {

struct Guard {
    mzk_ctx* c;
    explicit Guard(mzk_ctx* ctx) : c(ctx) {
        c->impl.mu.lock();
        cudaSetDevice(c->impl.device);
    }
    ~Guard() { c->impl.mu.unlock(); }
};

int check_ctx(mzk_ctx* ctx) {
    if (!ctx) {
        mzk::set_error("null context");
        return mzk::ERR_ARG;
    }
    return mzk::OK;
}

}  // namespace

extern "C" {

const char* mzk_last_error(void) { return mzk::g_last_error.c_str(); }
const char* mzk_version(void) { return "mzk-b200 0.1 (sm_100a)"; }

int mzk_ctx_create(int device, mzk_ctx** out) {
    if (!out) {
        mzk::set_error("null out pointer");
        return mzk::ERR_ARG;
    }
    *out = nullptr;
    int count = 0;
    MZK_CUDA_CHECK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) {
        mzk::set_error("no CUDA device " + std::to_string(device));
        return mzk::ERR_ARG;
    }
    MZK_CUDA_CHECK(cudaSetDevice(device));
    mzk_ctx* c = new (std::nothrow) mzk_ctx;
    if (!c) return mzk::ERR_OOM;
    c->impl.device = device;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->impl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->impl.copy_stream, cudaStreamNonBlocking);
    for (cudaEvent_t& ev : c->impl.ev_copy)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        mzk::set_error(std::string("context setup: ") + cudaGetErrorString(e));
        delete c;
        return mzk::ERR_CUDA;
    }
    if (prop.major != 10) {
        mzk::set_error("this library is built for sm_100a (B200); device " + std::to_string(device) + " is sm_" +
                       std::to_string(prop.major) + std::to_string(prop.minor));
        delete c;
        return mzk::ERR_STATE;
    }
    c->impl.num_sms = prop.multiProcessorCount;
    if (const char* tf = std::getenv("MZK_TUNE_FILE")) {
        if (*tf) {
            const mzk::Status s = mzk::tune_load(&c->impl, tf);
            if (s != mzk::OK) {
                delete c;
                return s;
            }
        }
    }
    *out = c;
    return mzk::OK;
}

int mzk_ctx_destroy(mzk_ctx* ctx) {
    if (!ctx) return mzk::OK;
    cudaSetDevice(ctx->impl.device);
    delete ctx;
    return mzk::OK;
}

uint64_t mzk_ctx_launch_count(const mzk_ctx* ctx) { return ctx ? ctx->impl.launches : 0; }

void* mzk_ctx_stream(mzk_ctx* ctx) { return ctx ? (void*)ctx->impl.stream : nullptr; }

int mzk_ctx_synchronize(mzk_ctx* ctx) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.copy_stream));
    return mzk::OK;
}

int mzk_device_alloc(mzk_ctx* ctx, size_t bytes, void** out) {
    if (int s = check_ctx(ctx)) return s;
    if (!out) return mzk::ERR_ARG;
    Guard g(ctx);
    MZK_CUDA_CHECK(cudaMalloc(out, bytes ? bytes : 16));
    return mzk::OK;
}

int mzk_device_free(mzk_ctx* ctx, void* ptr) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    MZK_CUDA_CHECK(cudaFree(ptr));
    return mzk::OK;
}

int mzk_memcpy_h2d(mzk_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    MZK_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_memcpy_d2h(mzk_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    MZK_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_msm_set_window(mzk_ctx* ctx, int c) {
    if (int s = check_ctx(ctx)) return s;
    if (c != 0 && (c < 5 || c > 24)) {
        mzk::set_error("window width must be 0 (auto) or in [5, 24]");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    ctx->impl.msm_window_override = c;
    return mzk::OK;
}

int mzk_msm_pick_window(size_t n) { return mzk::msm_pick_window(n); }

int mzk_ctx_set_profiling(mzk_ctx* ctx, int on) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    ctx->impl.profiling = on != 0;
    if (on) {
        for (int i = 0; i < mzk::Context::kPhases; i++) {
            ctx->impl.phase_ms[i] = 0.0;
            ctx->impl.phase_count[i] = 0;
        }
    }
    return mzk::OK;
}

int mzk_ctx_phase_stats(mzk_ctx* ctx, double* ms_out, uint64_t* count_out, int max_phases) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    for (int i = 0; i < max_phases && i < mzk::Context::kPhases; i++) {
        if (ms_out) ms_out[i] = ctx->impl.phase_ms[i];
        if (count_out) count_out[i] = ctx->impl.phase_count[i];
    }
    return mzk::OK;
}

int mzk_ctx_prove_phase_stats(mzk_ctx* ctx, double* ms_out, uint64_t* calls, int max_phases, int reset) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    for (int i = 0; i < max_phases && i < mzk::Context::kProvePhases; i++)
        if (ms_out) ms_out[i] = ctx->impl.prove_ms[i];
    if (calls) *calls = ctx->impl.prove_calls;
    if (reset) {
        for (int i = 0; i < mzk::Context::kProvePhases; i++) ctx->impl.prove_ms[i] = 0.0;
        ctx->impl.prove_calls = 0;
    }
    return mzk::OK;
}

int mzk_g1_sum_host(const uint64_t* points, size_t count, uint64_t out[18]) {
    if (!out || (count && !points)) {
        mzk::set_error("g1_sum: null pointer");
        return mzk::ERR_ARG;
    }
    namespace h = mzk::host;
    h::Xyzz6 acc = h::infinity();
    for (size_t i = 0; i < count; i++) {
        const uint64_t* p = points + 18 * i;
        bool zero = true, one = true;
        for (int j = 0; j < 6; j++) {
            zero = zero && p[12 + j] == 0;
            one = one && p[12 + j] == h::ONE6[j];
        }
        if (zero) continue;
        if (!one) {
            mzk::set_error("g1_sum: point " + std::to_string(i) + " is not normalised (z must be 1 or the point all zero)");
            return mzk::ERR_ARG;
        }
        h::Xyzz6 q;
        std::memcpy(q.x.l, p, 48);
        std::memcpy(q.y.l, p + 6, 48);
        q.zz = h::one();
        q.zzz = h::one();
        acc = h::add(acc, q);
    }
    h::to_jacobian_normalised(acc, out);
    return mzk::OK;
}

int mzk_msm_last_shape(mzk_ctx* ctx, int* c, int* windows, uint64_t* entries) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    if (c) *c = ctx->impl.last_c;
    if (windows) *windows = ctx->impl.last_windows;
    if (entries) *entries = ctx->impl.last_entries;
    return mzk::OK;
}

int mzk_probe_imad_peak(mzk_ctx* ctx, double* imad_per_s, double* fp_mul_per_s, double variants[4]) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    return mzk::probe_imad(&ctx->impl, imad_per_s, fp_mul_per_s, variants);
}

int mzk_ctx_graph_stats(mzk_ctx* ctx, uint64_t* captures, uint64_t* replays) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    if (captures) *captures = ctx->impl.graph_captures;
    if (replays) *replays = ctx->impl.graph_replays;
    return mzk::OK;
}

int mzk_autotune(mzk_ctx* ctx, const uint64_t* d_scalars, const uint64_t* d_bases, const uint32_t* msm_log_n,
                 size_t n_msm, const uint32_t* ntt_log_n, size_t n_ntt, int reps, double* msm_ms, double* ntt_ms) {
    if (int s = check_ctx(ctx)) return s;
    if ((n_msm && !msm_log_n) || (n_ntt && !ntt_log_n)) {
        mzk::set_error("autotune: null size list");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    return mzk::autotune(&ctx->impl, d_scalars, d_bases, msm_log_n, n_msm, ntt_log_n, n_ntt, reps, msm_ms, ntt_ms);
}

static int* tune_slot(mzk_ctx* ctx, int kind, uint32_t log_n) {
    if (log_n >= (uint32_t)mzk::kTuneSlots) return nullptr;
    if (kind == MZK_TUNE_MSM_WINDOW) return &ctx->impl.tuned_msm_c[log_n];
    if (kind == MZK_TUNE_NTT_SPLIT) return &ctx->impl.tuned_ntt_split[log_n];
    return nullptr;
}

int mzk_autotune_get(mzk_ctx* ctx, int kind, uint32_t log_n, int* value) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    int* slot = tune_slot(ctx, kind, log_n);
    if (!slot || !value) {
        mzk::set_error("autotune: unknown kind or size, or null output");
        return mzk::ERR_ARG;
    }
    *value = *slot;
    return mzk::OK;
}

int mzk_autotune_set(mzk_ctx* ctx, int kind, uint32_t log_n, int value) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    int* slot = tune_slot(ctx, kind, log_n);
    const bool ok = value == 0 || (kind == MZK_TUNE_MSM_WINDOW && value >= 5 && value <= 24) ||
                    (kind == MZK_TUNE_NTT_SPLIT && value >= mzk::kSplitEven && value <= mzk::kSplitBack);
    if (!slot || !ok) {
        mzk::set_error("autotune: unknown kind or size, or value out of range");
        return mzk::ERR_ARG;
    }
    *slot = value;
    return mzk::OK;
}

int mzk_autotune_save(mzk_ctx* ctx, const char* path) {
    if (int s = check_ctx(ctx)) return s;
    if (!path) return mzk::ERR_ARG;
    Guard g(ctx);
    return mzk::tune_save(&ctx->impl, path);
}

int mzk_autotune_load(mzk_ctx* ctx, const char* path) {
    if (int s = check_ctx(ctx)) return s;
    if (!path) return mzk::ERR_ARG;
    Guard g(ctx);
    return mzk::tune_load(&ctx->impl, path);
}

int mzk_probe_fp_sqr_check(mzk_ctx* ctx, const uint64_t* d_values, size_t n, uint64_t* mismatches) {
    if (int s = check_ctx(ctx)) return s;
    if (!mismatches || (n && !d_values)) {
        mzk::set_error("probe: null pointer");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    return mzk::check_fp_sqr(&ctx->impl, d_values, n, mismatches);
}

int mzk_probe_fp_inv_check(mzk_ctx* ctx, const uint64_t* d_values, size_t n, uint64_t* mismatches) {
    if (int s = check_ctx(ctx)) return s;
    if (!mismatches || (n && !d_values)) {
        mzk::set_error("probe: null pointer");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    return mzk::check_fp_inv(&ctx->impl, d_values, n, mismatches);
}

int mzk_probe_batch_affine(mzk_ctx* ctx, double out[8]) {
    if (int s = check_ctx(ctx)) return s;
    if (!out) {
        mzk::set_error("probe: null pointer");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    return mzk::probe_batch_affine(&ctx->impl, out);
}

int mzk_msm_g1_device(mzk_ctx* ctx, const uint64_t* d_scalars, const uint64_t* d_bases, size_t n, uint64_t out[18]) {
    if (int s = check_ctx(ctx)) return s;
    if (!out || (n && (!d_scalars || !d_bases))) {
        mzk::set_error("msm: null pointer");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    return mzk::msm_g1_device(&ctx->impl, d_scalars, d_bases, n, out, ctx->impl.stream, nullptr);
}

// host-buffer MSMs of at least this many points upload and compute in parts
constexpr size_t kPipelineMinPoints = size_t(1) << 20;
// Cumulative point fractions of the parts of a pipelined host MSM.  At 2^24
// the upload (128 bytes a point at the host link's ~55 GB/s) takes ~39 ms
// and the sort and accumulation ~84 ms, both linear in the points; every
// part after the first adds one bucket set that the reduction merges key by
// key (one full XYZZ addition per key, ~4 ms at c = 20).  Three parts
// balance the two: the compute stream waits for the first 12 % only, and
// each later part is up before the one before it has been accumulated.
constexpr int kHostParts = 3;
constexpr double kPartEnd[kHostParts] = {0.12, 0.40, 1.0};
static_assert(kHostParts <= mzk::kMaxMsmParts, "parts of a pipelined MSM");
static_assert(2 * kHostParts <= mzk::Context::kCopyEvents, "two upload events per part");

int mzk_msm_g1(mzk_ctx* ctx, const uint64_t* scalars, const uint64_t* bases, size_t n, uint64_t out[18]) {
    if (int s = check_ctx(ctx)) return s;
    if (!out || (n && (!scalars || !bases))) {
        mzk::set_error("msm: null pointer");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    if (n == 0) {
        std::memset(out, 0, 18 * 8);
        return mzk::OK;
    }
    mzk::Context* c = &ctx->impl;
    void *ds, *db;
    MZK_TRY(c->ensure("in_scalars", n * 32, &ds));
    MZK_TRY(c->ensure("in_bases", n * 96, &db));
    char* dsc = static_cast<char*>(ds);
    char* dba = static_cast<char*>(db);
    const char* hsc = reinterpret_cast<const char*>(scalars);
    const char* hba = reinterpret_cast<const char*>(bases);
    // The first part's scalars go on the compute stream (its digit passes
    // need only them), everything else on the copy stream in part order:
    // the first part's bases, then each later part's scalars and bases, each
    // marked by its own event, so part p is sorted once its scalars are up
    // and accumulated once its bases are, while later parts still upload.
    const int P = n >= kPipelineMinPoints ? kHostParts : 1;
    size_t end[kHostParts];
    for (int p = 0; p < P; p++)
        end[p] = p + 1 == P ? n : (size_t)((double)n * kPartEnd[p]) & ~(size_t)1023;
    mzk::MsmPart parts[kHostParts];
    for (int p = 0; p < P; p++) {
        const size_t b0 = p ? end[p - 1] : 0, np = end[p] - b0;
        cudaStream_t sst = p ? c->copy_stream : c->stream;
        MZK_CUDA_CHECK(cudaMemcpyAsync(dsc + b0 * 32, hsc + b0 * 32, np * 32, cudaMemcpyHostToDevice, sst));
        if (p) MZK_CUDA_CHECK(cudaEventRecord(c->ev_copy[2 * p], c->copy_stream));
        MZK_CUDA_CHECK(cudaMemcpyAsync(dba + b0 * 96, hba + b0 * 96, np * 96, cudaMemcpyHostToDevice, c->copy_stream));
        MZK_CUDA_CHECK(cudaEventRecord(c->ev_copy[2 * p + 1], c->copy_stream));
        parts[p] = {b0, end[p], p ? c->ev_copy[2 * p] : nullptr, c->ev_copy[2 * p + 1]};
    }
    if (P == 1) return mzk::msm_g1_device(c, ds, db, n, out, c->stream, c->ev_copy[1]);
    return mzk::msm_g1_parts(c, ds, db, n, out, c->stream, parts, P);
}

int mzk_gen_rand_fr_device(mzk_ctx* ctx, uint64_t seed, uint64_t first, size_t n, uint64_t* d_out) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    MZK_TRY(mzk::gen_rand_fr(&ctx->impl, seed, first, n, d_out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_gen_bases_g1_device(mzk_ctx* ctx, uint64_t seed, uint64_t first, size_t n, uint64_t* d_out) {
    if (int s = check_ctx(ctx)) return s;
    Guard g(ctx);
    MZK_TRY(mzk::gen_bases_g1(&ctx->impl, seed, first, n, d_out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_gen_config3_fixed_device(mzk_ctx* ctx, uint32_t k, uint32_t blinding_factors, uint32_t table_rows,
                                 uint64_t seed, uint64_t* d_fixed) {
    if (int s = check_ctx(ctx)) return s;
    if (!d_fixed || k < 3 || k > 26 || blinding_factors + 2 >= (1u << k) || table_rows == 0) {
        mzk::set_error("gen_config3_fixed: bad argument");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::gen_config3_fixed(&ctx->impl, k, blinding_factors, table_rows, seed, d_fixed, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_gen_config3_witness_device(mzk_ctx* ctx, uint32_t k, uint32_t blinding_factors, uint32_t table_rows,
                                   uint64_t seed, const uint64_t* d_fixed, const uint64_t* d_inv_qo,
                                   const uint32_t* d_cycle_of, uint64_t* d_advice) {
    if (int s = check_ctx(ctx)) return s;
    if (!d_fixed || !d_inv_qo || !d_cycle_of || !d_advice || k < 3 || k > 26 || blinding_factors + 2 >= (1u << k) ||
        table_rows == 0) {
        mzk::set_error("gen_config3_witness: bad argument");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::gen_config3_witness(&ctx->impl, k, blinding_factors, table_rows, seed, d_fixed, d_inv_qo, d_cycle_of,
                                     d_advice, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

// ---- EvaluationDomain -----------------------------------------------------

int mzk_domain_create(mzk_ctx* ctx, uint32_t j, uint32_t k, mzk_domain** out) {
    if (int s = check_ctx(ctx)) return s;
    if (!out) return mzk::ERR_ARG;
    *out = nullptr;
    Guard g(ctx);
    mzk::Domain* d = nullptr;
    MZK_TRY(mzk::domain_create(&ctx->impl, j, k, &d));
    mzk_domain* h = new (std::nothrow) mzk_domain;
    if (!h) {
        delete d;
        return mzk::ERR_OOM;
    }
    h->impl = d;
    h->ctx = ctx;
    *out = h;
    return mzk::OK;
}

int mzk_domain_destroy(mzk_domain* d) {
    if (!d) return mzk::OK;
    Guard g(d->ctx);
    cudaStreamSynchronize(d->ctx->impl.stream);
    d->ctx->impl.buf_generation++;  // captured graphs may hold its tables
    delete d->impl;
    delete d;
    return mzk::OK;
}

int mzk_domain_shape(const mzk_domain* d, uint32_t* k, uint32_t* extended_k) {
    if (!d) return mzk::ERR_ARG;
    if (k) *k = d->impl->k;
    if (extended_k) *extended_k = d->impl->ext_k;
    return mzk::OK;
}

int mzk_domain_constant(const mzk_domain* d, int which, int idx, uint64_t out[4]) {
    if (!d || !out) return mzk::ERR_ARG;
    const mzk::Domain* D = d->impl;
    const mzk::host::Fr4* src = nullptr;
    switch (which) {
        case 0: src = &D->omega; break;
        case 1: src = &D->omega_inv; break;
        case 2: src = &D->ext_omega; break;
        case 3: src = &D->ext_omega_inv; break;
        case 4: src = &D->zeta; break;
        case 5: src = &D->zeta2; break;
        case 6: src = &D->ifft_div; break;
        case 7: src = &D->ext_ifft_div; break;
        case 8:
            if (idx < 0 || (size_t)idx >= D->t_inv.size()) return mzk::ERR_ARG;
            src = &D->t_inv[idx];
            break;
        default:
            mzk::set_error("domain constant: unknown index");
            return mzk::ERR_ARG;
    }
    std::memcpy(out, src->l, 32);
    return mzk::OK;
}

int mzk_domain_op_device(mzk_ctx* ctx, mzk_domain* d, int op, const uint64_t* d_in, uint64_t* d_out) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !d_in || !d_out) {
        mzk::set_error("domain op: null argument");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::domain_op_device(&ctx->impl, d->impl, op, d_in, d_out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_domain_op_batch_device(mzk_ctx* ctx, mzk_domain* d, int op, const uint64_t* const* d_in,
                               uint64_t* const* d_out, size_t count) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || (count && (!d_in || !d_out))) {
        mzk::set_error("domain op batch: null argument");
        return mzk::ERR_ARG;
    }
    if (op < mzk::OP_COEFF_TO_LAGRANGE || op > mzk::OP_EXTENDED_TO_COEFF || count > 0xffffffffu) {
        mzk::set_error("domain op batch: the operation must be 0-3");
        return mzk::ERR_ARG;
    }
    for (size_t i = 0; i < count; i++)
        if (!d_in[i] || !d_out[i]) {
            mzk::set_error("domain op batch: null polynomial");
            return mzk::ERR_ARG;
        }
    Guard g(ctx);
    MZK_TRY(mzk::domain_op_batch(&ctx->impl, d->impl, op, reinterpret_cast<const void* const*>(d_in),
                                 reinterpret_cast<void* const*>(d_out), (uint32_t)count, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_domain_op(mzk_ctx* ctx, mzk_domain* d, int op, const uint64_t* in, uint64_t* out) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !in || !out) {
        mzk::set_error("domain op: null argument");
        return mzk::ERR_ARG;
    }
    if (op < 0 || op > mzk::OP_DIVIDE_BY_VANISHING) {
        mzk::set_error("domain op: unknown operation");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    mzk::Context* c = &ctx->impl;
    const size_t in_len = mzk::domain_op_in_len(d->impl, op), out_len = mzk::domain_op_out_len(d->impl, op);
    void *din, *dout;
    MZK_TRY(c->ensure("ntt_in", in_len * 32, &din));
    MZK_TRY(c->ensure("ntt_out", out_len * 32, &dout));
    MZK_CUDA_CHECK(cudaMemcpyAsync(din, in, in_len * 32, cudaMemcpyHostToDevice, c->stream));
    MZK_TRY(mzk::domain_op_device(c, d->impl, op, din, dout, c->stream));
    MZK_CUDA_CHECK(cudaMemcpyAsync(out, dout, out_len * 32, cudaMemcpyDeviceToHost, c->stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return mzk::OK;
}

int mzk_quotient_eval_device(mzk_ctx* ctx, mzk_domain* d, const mzk_quotient_desc* desc, int divide,
                             uint64_t* d_out) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !desc || !d_out) {
        mzk::set_error("quotient: null argument");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::quotient_eval_device(&ctx->impl, d->impl, desc, divide, d_out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_msm_g1_batch_device(mzk_ctx* ctx, const uint64_t* d_bases, size_t bases_len, const mzk_msm_batch_item* items,
                            size_t count, uint64_t* out) {
    if (int s = check_ctx(ctx)) return s;
    if (!out || (count && (!items || !d_bases))) {
        mzk::set_error("msm batch: null pointer");
        return mzk::ERR_ARG;
    }
    static_assert(sizeof(mzk_msm_batch_item) == sizeof(mzk::BatchItem), "batch item layout");
    Guard g(ctx);
    return mzk::msm_g1_batch_device(&ctx->impl, d_bases, bases_len, reinterpret_cast<const mzk::BatchItem*>(items),
                                    count, out, ctx->impl.stream);
}

int mzk_msm_table_rows(int c) { return (c < 5 || c > 24) ? 0 : (int)mzk::msm_table_rows(c); }

int mzk_msm_window_table(mzk_ctx* ctx, uint64_t* d_table, size_t len, int c, size_t rows) {
    if (int s = check_ctx(ctx)) return s;
    if (!d_table) {
        mzk::set_error("window table: null table");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::msm_window_table(&ctx->impl, d_table, len, c, (uint32_t)std::min<size_t>(rows, 0xffffffffu),
                                  ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_msm_g1_batch_table_device(mzk_ctx* ctx, const uint64_t* d_table, size_t len, int c, size_t rows,
                                  size_t min_n, const mzk_msm_batch_item* items, size_t count, uint64_t* out) {
    if (int s = check_ctx(ctx)) return s;
    if (!out || !d_table || (count && !items) || c < 5 || c > 24) {
        mzk::set_error("msm batch table: null pointer or width outside [5, 24]");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    std::vector<mzk::BatchItem> its(count);
    for (size_t i = 0; i < count; i++) its[i] = {items[i].d_scalars, items[i].base_offset, items[i].n};
    const mzk::MsmTable table{d_table, len, c, (uint32_t)std::min<size_t>(rows, 0xffffffffu), min_n};
    return mzk::msm_g1_batch_device(&ctx->impl, d_table, len, its.data(), count, out, ctx->impl.stream, &table);
}

int mzk_compute_h_poly_device(mzk_ctx* ctx, mzk_domain* d, const mzk_quotient_desc* desc, const uint64_t* d_srs_g,
                              size_t srs_len, const uint64_t* blinds, uint64_t* out_commitments,
                              uint64_t* d_limbs_out) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !desc || !d_srs_g || !blinds || !out_commitments) {
        mzk::set_error("compute_h_poly: null argument");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    return mzk::compute_h_poly_device(&ctx->impl, d->impl, desc, d_srs_g, srs_len, blinds, out_commitments,
                                      d_limbs_out, ctx->impl.stream);
}

int mzk_batch_invert_device(mzk_ctx* ctx, uint64_t* a, size_t n) {
    if (int s = check_ctx(ctx)) return s;
    if (n && !a) return mzk::ERR_ARG;
    Guard g(ctx);
    MZK_TRY(mzk::batch_invert_device(&ctx->impl, a, n, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_eval_polynomial_device(mzk_ctx* ctx, const uint64_t* poly, size_t n, const uint64_t point[4], uint64_t out[4]) {
    if (int s = check_ctx(ctx)) return s;
    if ((n && !poly) || !point || !out) return mzk::ERR_ARG;
    Guard g(ctx);
    return mzk::eval_polynomial_device(&ctx->impl, poly, n, point, out, ctx->impl.stream);
}

int mzk_kate_division_device(mzk_ctx* ctx, const uint64_t* a, size_t n, const uint64_t b[4], uint64_t* q) {
    if (int s = check_ctx(ctx)) return s;
    if ((n > 1 && (!a || !q)) || !b) return mzk::ERR_ARG;
    Guard g(ctx);
    MZK_TRY(mzk::kate_division_device(&ctx->impl, a, n, b, q, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_poly_inner_product_device(mzk_ctx* ctx, const uint64_t* const* polys, const size_t* lens, size_t m,
                                  const uint64_t* scalars, uint64_t* out, size_t out_len) {
    if (int s = check_ctx(ctx)) return s;
    if ((m && (!polys || !lens || !scalars)) || (out_len && !out) || m >= (1u << 20)) return mzk::ERR_ARG;
    size_t longest = 0;
    for (size_t p = 0; p < m; p++) {
        if (lens[p] && !polys[p]) return mzk::ERR_ARG;
        longest = lens[p] > longest ? lens[p] : longest;
    }
    if (longest > out_len) {
        mzk::set_error("poly_inner_product: out_len shorter than the longest polynomial");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    std::vector<uint64_t> l64(lens, lens + m);
    return mzk::poly_inner_product_device(&ctx->impl, polys, l64.data(), (uint32_t)m, scalars, out, out_len,
                                          ctx->impl.stream);
}

int mzk_srs_setup_device(mzk_ctx* ctx, mzk_domain* d, const uint64_t s[4], uint64_t* g, uint64_t* g_lagrange,
                         uint64_t* g_lagrange_delta, uint64_t* g_lagrange_double_delta) {
    if (int st = check_ctx(ctx)) return st;
    if (!d || !s) return mzk::ERR_ARG;
    Guard gd(ctx);
    MZK_TRY(mzk::srs_setup_device(&ctx->impl, d->impl, s, g, g_lagrange, g_lagrange_delta, g_lagrange_double_delta,
                                  ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_g1_to_lagrange_device(mzk_ctx* ctx, mzk_domain* d, const uint64_t* g, uint64_t* out) {
    if (int st = check_ctx(ctx)) return st;
    if (!d || !g || !out) return mzk::ERR_ARG;
    Guard gd(ctx);
    MZK_TRY(mzk::g1_to_lagrange_device(&ctx->impl, d->impl, g, out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_srs_downsize_device(mzk_ctx* ctx, mzk_domain* d, const uint64_t* g, uint64_t* g_lagrange,
                            uint64_t* g_lagrange_delta, uint64_t* g_lagrange_double_delta) {
    if (int st = check_ctx(ctx)) return st;
    if (!d || !g) return mzk::ERR_ARG;
    Guard gd(ctx);
    MZK_TRY(mzk::srs_downsize_device(&ctx->impl, d->impl, g, g_lagrange, g_lagrange_delta, g_lagrange_double_delta,
                                     ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_g1_suffix_sum_device(mzk_ctx* ctx, const uint64_t* in, size_t n, uint64_t* out) {
    if (int st = check_ctx(ctx)) return st;
    if (n && (!in || !out)) return mzk::ERR_ARG;
    Guard gd(ctx);
    MZK_TRY(mzk::g1_suffix_sum_device(&ctx->impl, in, n, out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_g1_decompress_device(mzk_ctx* ctx, const uint8_t* in, size_t n, int check_subgroup, uint64_t* out,
                             uint8_t* status, uint64_t* n_invalid) {
    if (int st = check_ctx(ctx)) return st;
    if (n && (!in || !out)) return mzk::ERR_ARG;
    Guard gd(ctx);
    MZK_TRY(mzk::g1_decompress_device(&ctx->impl, in, n, check_subgroup, out, status, n_invalid, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_g1_compress_device(mzk_ctx* ctx, const uint64_t* points, size_t n, uint8_t* out) {
    if (int s = check_ctx(ctx)) return s;
    if (n && (!points || !out)) {
        mzk::set_error("g1_compress: null pointer");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::g1_compress_device(&ctx->impl, points, n, out, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_srs_write_processed(mzk_ctx* ctx, const uint64_t* g, const uint64_t* g_lagrange, size_t n, uint8_t* out,
                            size_t out_len) {
    if (int s = check_ctx(ctx)) return s;
    if (!g || !g_lagrange || !out) {
        mzk::set_error("srs_write: null pointer");
        return mzk::ERR_ARG;
    }
    Guard gd(ctx);
    return mzk::srs_write_processed(&ctx->impl, g, g_lagrange, n, out, out_len, ctx->impl.stream);
}

int mzk_srs_read_processed(mzk_ctx* ctx, const uint8_t* bytes, size_t len, size_t capacity, uint32_t* k_out,
                           uint64_t* g, uint64_t* g_lagrange, uint64_t* g_lagrange_delta,
                           uint64_t* g_lagrange_double_delta) {
    if (int st = check_ctx(ctx)) return st;
    if (!bytes || !k_out) return mzk::ERR_ARG;
    Guard gd(ctx);
    MZK_TRY(mzk::srs_read_processed(&ctx->impl, bytes, len, capacity, k_out, g, g_lagrange, g_lagrange_delta,
                                    g_lagrange_double_delta, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_permutation_z_device(mzk_ctx* ctx, mzk_domain* d, const mzk_permutation_desc* desc) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !desc) return mzk::ERR_ARG;
    Guard g(ctx);
    MZK_TRY(mzk::permutation_z_device(&ctx->impl, d->impl, desc, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_logup_device(mzk_ctx* ctx, mzk_domain* d, const mzk_logup_desc* desc) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !desc) return mzk::ERR_ARG;
    Guard g(ctx);
    MZK_TRY(mzk::logup_device(&ctx->impl, d->impl, desc, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

int mzk_prove_core_device(mzk_ctx* ctx, mzk_domain* d, const mzk_proving_key_desc* pk, const mzk_proof_job* jobs,
                          size_t count, uint32_t flags, uint64_t* out) {
    if (int s = check_ctx(ctx)) return s;
    if (!d || !pk || !out || (count && !jobs)) {
        mzk::set_error("prove_core: null argument");
        return mzk::ERR_ARG;
    }
    Guard g(ctx);
    MZK_TRY(mzk::prove_core_device(&ctx->impl, d->impl, pk, jobs, count, out, flags, ctx->impl.stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->impl.stream));
    return mzk::OK;
}

}  // extern "C"
