// tune.cu — the autotuner: per-size choices measured on the device.
//
// Two choices are tuned, each keyed by floor(log2(size)):
//   * the MSM window width c: the cost model's width and its neighbours
//     c-2 .. c+2 are timed on the caller's device inputs (the first 2^L
//     scalars and bases), whole calls including the host tail;
//   * the NTT pass split of a transform of 2^L elements: the even split
//     (default), the largest passes first, or the largest passes last
//     (`NttSplit`, ntt.hpp), timed as a forward transform of random data.
// Every choice gives the same result (the MSM is one group element whatever
// its windows; every split computes the same transform), so tuning changes
// speed only.  The table is saved and loaded as text lines
// "msm_c <log_n> <c>" and "ntt_split <log_n> <mode>".
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

int msm_window_for(const Context* ctx, size_t n) {
    if (ctx->msm_window_override > 0) return ctx->msm_window_override;
    const int lg = n ? 63 - __builtin_clzll((unsigned long long)n) : 0;
    if (lg < kTuneSlots && ctx->tuned_msm_c[lg] > 0) return ctx->tuned_msm_c[lg];
    return msm_pick_window(n);
}

namespace {

double time_msm(Context* ctx, const void* ds, const void* db, size_t n, int c, int reps, uint64_t* out18,
                Status* st) {
    const int saved = ctx->msm_window_override;
    ctx->msm_window_override = c;
    double best = 1e300;
    *st = msm_g1_device(ctx, ds, db, n, out18, ctx->stream, nullptr);  // warm-up (buffers sized)
    for (int r = 0; r < reps && *st == OK; r++) {
        const auto t0 = std::chrono::steady_clock::now();
        *st = msm_g1_device(ctx, ds, db, n, out18, ctx->stream, nullptr);
        const auto t1 = std::chrono::steady_clock::now();
        best = std::min(best, std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    ctx->msm_window_override = saved;
    return best;
}

}  // namespace

Status autotune(Context* ctx, const void* d_scalars, const void* d_bases, const uint32_t* msm_log_n, size_t n_msm,
                const uint32_t* ntt_log_n, size_t n_ntt, int reps, double* msm_ms_out, double* ntt_ms_out) {
    if (reps < 1) reps = 1;
    // MSM window widths
    for (size_t i = 0; i < n_msm; i++) {
        const uint32_t lg = msm_log_n[i];
        if (lg >= (uint32_t)kTuneSlots || lg > 30) {
            set_error("autotune: MSM size 2^" + std::to_string(lg) + " out of range");
            return ERR_ARG;
        }
        if (!d_scalars || !d_bases) {
            set_error("autotune: MSM sizes given without device inputs");
            return ERR_ARG;
        }
        const size_t n = (size_t)1 << lg;
        const int model = msm_pick_window(n);
        int best_c = model;
        double best_ms = 1e300;
        uint64_t ref[18], out[18];
        for (int c = std::max(5, model - 2); c <= std::min(24, model + 2); c++) {
            Status st;
            const double ms = time_msm(ctx, d_scalars, d_bases, n, c, reps, out, &st);
            if (st != OK) return st;
            if (c == std::max(5, model - 2)) std::memcpy(ref, out, sizeof(ref));
            if (std::memcmp(ref, out, sizeof(ref)) != 0) {  // every width must give the same point
                set_error("autotune: MSM results differ between window widths");
                return ERR_STATE;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best_c = c;
            }
        }
        ctx->tuned_msm_c[lg] = best_c;
        if (msm_ms_out) msm_ms_out[i] = best_ms;
    }
    // NTT pass splits
    for (size_t i = 0; i < n_ntt; i++) {
        const uint32_t lg = ntt_log_n[i];
        if (lg < 1 || lg >= (uint32_t)kTuneSlots || lg > 28) {
            set_error("autotune: NTT size 2^" + std::to_string(lg) + " out of range");
            return ERR_ARG;
        }
        Domain* d = nullptr;
        MZK_TRY(domain_create(ctx, 3, lg, &d));
        std::unique_ptr<Domain> hold(d);
        void* buf;
        MZK_TRY(ctx->ensure("tune_ntt", ((size_t)1 << lg) * 32, &buf));
        MZK_TRY(gen_rand_fr(ctx, 0x7u + lg, 0, (size_t)1 << lg, buf, ctx->stream));
        cudaEvent_t e0, e1;
        MZK_CUDA_CHECK(cudaEventCreate(&e0));
        MZK_CUDA_CHECK(cudaEventCreate(&e1));
        const int saved = ctx->tuned_ntt_split[lg];
        int best_mode = kSplitEven;
        double best_ms = 1e300;
        Status st = OK;
        for (int mode = kSplitEven; mode <= kSplitBack && st == OK; mode++) {
            ctx->tuned_ntt_split[lg] = mode;
            st = domain_op_device(ctx, d, OP_COEFF_TO_LAGRANGE, buf, buf, ctx->stream);  // warm-up
            for (int r = 0; r < reps && st == OK; r++) {
                cudaEventRecord(e0, ctx->stream);
                st = domain_op_device(ctx, d, OP_COEFF_TO_LAGRANGE, buf, buf, ctx->stream);
                cudaEventRecord(e1, ctx->stream);
                if (cudaEventSynchronize(e1) != cudaSuccess) st = ERR_CUDA;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (st == OK && ms < best_ms) {
                    best_ms = ms;
                    best_mode = mode;
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ctx->buf_generation++;  // the domain goes away with `hold`
        ctx->tuned_ntt_split[lg] = st == OK ? best_mode : saved;
        if (st != OK) return st;
        if (ntt_ms_out) ntt_ms_out[i] = best_ms;
    }
    return OK;
}

Status tune_save(const Context* ctx, const char* path) {
    FILE* f = std::fopen(path, "w");
    if (!f) {
        set_error(std::string("autotune: cannot write ") + path);
        return ERR_ARG;
    }
    for (int lg = 0; lg < kTuneSlots; lg++)
        if (ctx->tuned_msm_c[lg] > 0) std::fprintf(f, "msm_c %d %d\n", lg, ctx->tuned_msm_c[lg]);
    for (int lg = 0; lg < kTuneSlots; lg++)
        if (ctx->tuned_ntt_split[lg] > 0) std::fprintf(f, "ntt_split %d %d\n", lg, ctx->tuned_ntt_split[lg]);
    const bool ok = std::fclose(f) == 0;
    if (!ok) {
        set_error(std::string("autotune: cannot write ") + path);
        return ERR_ARG;
    }
    return OK;
}

// A malformed line rejects the whole file and leaves the table unchanged.
Status tune_load(Context* ctx, const char* path) {
    FILE* f = std::fopen(path, "r");
    if (!f) {
        set_error(std::string("autotune: cannot read ") + path);
        return ERR_ARG;
    }
    int msm[kTuneSlots], ntt[kTuneSlots];
    std::memcpy(msm, ctx->tuned_msm_c, sizeof(msm));
    std::memcpy(ntt, ctx->tuned_ntt_split, sizeof(ntt));
    char line[256];
    int lineno = 0;
    Status st = OK;
    while (st == OK && std::fgets(line, sizeof(line), f)) {
        lineno++;
        char key[32];
        int lg, v;
        char extra;
        if (line[0] == '#' || line[0] == '\n') continue;
        if (std::sscanf(line, "%31s %d %d %c", key, &lg, &v, &extra) != 3 || lg < 0 || lg >= kTuneSlots) {
            st = ERR_ARG;
        } else if (!std::strcmp(key, "msm_c") && v >= 5 && v <= 24) {
            msm[lg] = v;
        } else if (!std::strcmp(key, "ntt_split") && v >= kSplitEven && v <= kSplitBack) {
            ntt[lg] = v;
        } else {
            st = ERR_ARG;
        }
        if (st != OK) set_error(std::string("autotune: ") + path + " line " + std::to_string(lineno) + " malformed");
    }
    std::fclose(f);
    if (st != OK) return st;
    std::memcpy(ctx->tuned_msm_c, msm, sizeof(msm));
    std::memcpy(ctx->tuned_ntt_split, ntt, sizeof(ntt));
    return OK;
}

}  // namespace mzk
