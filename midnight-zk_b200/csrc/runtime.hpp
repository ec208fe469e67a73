// runtime.hpp — device context of the C ABI: one per (process, GPU).
//
// Holds the CUDA streams, a grow-only set of named scratch buffers (so repeated
// calls of the same size never touch the allocator), a pinned staging buffer
// for host <-> device copies, and the mutex that makes every entry point safe
// to call from many host threads (the reference commits from rayon workers,
// proofs/src/plonk/prover.rs:619-623).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace mzk {

enum Status : int {
    OK = 0,
    ERR_ARG = 1,
    ERR_OOM = 2,
    ERR_CUDA = 3,
    ERR_TIMEOUT = 4,
    ERR_STATE = 5,
};

void set_error(const std::string& msg);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct Context {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;       // compute stream
    cudaStream_t copy_stream = nullptr;  // host->device copies overlapped with compute
    // uploads of a pipelined host MSM: per part its scalars (2p) and bases (2p + 1)
    static constexpr int kCopyEvents = 8;
    cudaEvent_t ev_copy[kCopyEvents] = {};
    std::recursive_mutex mu;
    std::map<std::string, DevBuf> bufs;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    int msm_window_override = 0;
    // autotuned choices by floor(log2 size), 0 = not tuned (tune.cu): MSM
    // window width, NTT pass split (NttSplit, ntt.hpp)
    static constexpr int kTuneSlotsN = 33;
    int tuned_msm_c[kTuneSlotsN] = {};
    int tuned_ntt_split[kTuneSlotsN] = {};
    // fixed-base table of the G1 generator for synthetic inputs (device)
    void* gen_table = nullptr;
    // kernels launched by the library since context creation (for reporting)
    uint64_t launches = 0;
    // per-phase device timing with CUDA events on the launching stream
    bool profiling = false;
    static constexpr int kPhases = 16;      // phase kinds
    static constexpr int kMaxRecords = 64;  // phases recorded between two collections
    static constexpr int kMaxEvents = 2 * kMaxRecords;
    cudaEvent_t prof_ev[kMaxEvents] = {};
    int prof_phase[kMaxRecords] = {};
    int prof_used = 0;
    double phase_ms[kPhases] = {};
    uint64_t phase_count[kPhases] = {};
    // create_proof: wall time of each Fiat-Shamir phase (every phase ends
    // with a stream sync), of the MSMs inside them, and calls made
    static constexpr int kProvePhases = 10;
    double prove_ms[kProvePhases] = {};
    uint64_t prove_calls = 0;
    // Captured CUDA graphs (a proof's NTT sequence), keyed by every pointer and
    // setting their kernels use.  buf_generation is bumped whenever ensure()
    // replaces a buffer or a domain is destroyed: graphs of an older generation
    // are dropped before any lookup, so a freed address is never replayed.
    struct GraphEntry {
        std::vector<uintptr_t> key;
        cudaGraphExec_t exec;
        uint64_t launches, generation, last_use;
    };
    static constexpr size_t kMaxGraphs = 64;
    std::vector<GraphEntry> graphs;
    uint64_t buf_generation = 0, graph_clock = 0, graph_captures = 0, graph_replays = 0;
    bool graphs_unsupported = false;  // a capture failed once: launch eagerly from then on

    // shape of the last MSM: window width, windows, bucket entries processed
    int last_c = 0, last_windows = 0;
    uint64_t last_entries = 0;

    // open/close a timed phase on `st` (no-ops unless profiling)
    Status phase_begin(int phase, cudaStream_t st);
    Status phase_end(cudaStream_t st);
    // after a stream sync: fold recorded phase times into the totals
    void phase_collect();

    // device buffer `name` of at least `bytes` bytes (contents undefined)
    Status ensure(const char* name, size_t bytes, void** out);
    Status ensure_pinned(size_t bytes, void** out);
    ~Context();
};

#define MZK_CUDA_CHECK(expr)                                                                  \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) {                                                              \
            ::mzk::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));             \
            return _e == cudaErrorMemoryAllocation ? ::mzk::ERR_OOM : ::mzk::ERR_CUDA; \
        }                                                                                     \
    } while (0)

#define MZK_LAUNCH_CHECK(ctx)                                                                 \
    do {                                                                                      \
        (ctx)->launches++;                                                                    \
        cudaError_t _e = cudaGetLastError();                                                  \
        if (_e != cudaSuccess) {                                                              \
            ::mzk::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e));        \
            return ::mzk::ERR_CUDA;                                                       \
        }                                                                                     \
    } while (0)

#define MZK_TRY(expr)                          \
    do {                                       \
        ::mzk::Status _s = (expr);             \
        if (_s != ::mzk::OK) return _s;    \
    } while (0)

// ---- MSM (msm.cu) ----
// scalars: n x 8 u32 (Fr, Montgomery), bases: n x 24 u32 (affine, Montgomery),
// both device pointers; out: 18 u64 host Jacobian with Z = 1 (identity: zeros).
// bases_ready (optional): event the compute stream waits on before the
// first kernel that reads the bases (their upload overlaps the digit sort)
Status msm_g1_device(Context* ctx, const void* d_scalars, const void* d_bases, size_t n, uint64_t* out18,
                     cudaStream_t stream, cudaEvent_t bases_ready);
// A pipelined MSM over contiguous point ranges [begin, end): the compute
// stream waits on a part's scalars_ready before sorting its digits and on its
// bases_ready before accumulating, so the upload of later parts overlaps the
// accumulation of earlier ones.  Same result as one part.
constexpr int kMaxMsmParts = 4;
struct MsmPart {
    size_t begin, end;
    cudaEvent_t scalars_ready, bases_ready;  // optional
};
Status msm_g1_parts(Context* ctx, const void* d_scalars, const void* d_bases, size_t n, uint64_t* out18,
                    cudaStream_t stream, const MsmPart* parts, int n_parts);
int msm_pick_window(size_t n);
// window width for an MSM of n points: the explicit override, else the
// autotuned width for floor(log2 n), else the cost model
constexpr int kTuneSlots = Context::kTuneSlotsN;
int msm_window_for(const Context* ctx, size_t n);
// tune.cu: time the MSM window widths and NTT pass splits of the given log2
// sizes on this device and keep the fastest; save / load the table as text
Status autotune(Context* ctx, const void* d_scalars, const void* d_bases, const uint32_t* msm_log_n, size_t n_msm,
                const uint32_t* ntt_log_n, size_t n_ntt, int reps, double* msm_ms_out, double* ntt_ms_out);
Status tune_save(const Context* ctx, const char* path);
Status tune_load(Context* ctx, const char* path);
// one MSM of a batch: scalars (device) against bases[base_offset, base_offset + n)
struct BatchItem {
    const void* d_scalars;
    uint64_t base_offset;
    uint64_t n;
};
// A window table of fixed bases: row j (j < rows) holds [2^(c j)] of every
// base, `stride` points per row, row 0 the bases themselves.  Items of at
// least min_n points use it: their windows share one bucket set of width c
// and window w reads row w (no per-window reduction, no doublings).
struct MsmTable {
    const void* d_table;
    uint64_t stride;
    int c;
    uint32_t rows;
    uint64_t min_n;
};
// rows a window table of width c needs (the windows of a width-c MSM)
uint32_t msm_table_rows(int c);
// out: count x 18 u64 (host), results in item order.  With a table, d_bases
// must be its row 0 (bases_len = its stride).
Status msm_g1_batch_device(Context* ctx, const void* d_bases, size_t bases_len, const BatchItem* items, size_t count,
                           uint64_t* out, cudaStream_t stream, const MsmTable* table = nullptr);
// rows 1 .. rows-1 of a window table whose row 0 (len points) is in place
Status msm_window_table(Context* ctx, void* d_table, uint64_t len, int c, uint32_t rows, cudaStream_t stream);
enum MsmPhase { PH_HISTOGRAM = 0, PH_SCAN, PH_SCATTER, PH_ACCUMULATE, PH_FIXUP, PH_REDUCE, PH_TAIL, PH_COPY };

// ---- microbenchmarks (probe.cu) ----
// integer multiply-add pipe rate (independent mad.lo/mad.hi, 32-bit) and the
// rate of full 12-limb Montgomery multiplications, both per second
Status probe_imad(Context* ctx, double* imad_per_s, double* fp_mul_per_s, double* variants);
Status check_fp_sqr(Context* ctx, const void* d_values, size_t n, uint64_t* mismatches);
Status check_fp_inv(Context* ctx, const void* d_values, size_t n, uint64_t* mismatches);
Status probe_batch_affine(Context* ctx, double* out);

// ---- synthetic inputs (gen.cu) ----
Status gen_rand_fr(Context* ctx, uint64_t seed, uint64_t first, size_t n, void* d_out, cudaStream_t stream);
// [s_i]G for n device scalars (Montgomery) into n device affine points
Status fixed_base_g1(Context* ctx, const void* d_scalars, size_t n, void* d_out, cudaStream_t st);
Status gen_bases_g1(Context* ctx, uint64_t seed, uint64_t first, size_t n, void* d_out, cudaStream_t stream);
// the single-proof configuration's circuit: 7 fixed columns (one device
// buffer of 7 x 2^k) and a satisfying witness a, b, c (3 x 2^k)
Status gen_config3_fixed(Context* ctx, uint32_t k, uint32_t bf, uint32_t table_rows, uint64_t seed, void* d_fixed,
                         cudaStream_t st);
Status gen_config3_witness(Context* ctx, uint32_t k, uint32_t bf, uint32_t table_rows, uint64_t seed,
                           const void* d_fixed, const void* d_inv_qo, const uint32_t* d_cycle_of, void* d_advice,
                           cudaStream_t st);

}  // namespace mzk
