// Internal declarations shared by the ExaStoLog B200 library sources.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <string>
#include <vector>

#include "esl_b200.h"

namespace esl {

// ---- errors ---------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

#define ESL_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::esl::fail(ESL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define ESL_TRY(call)                  \
    do {                               \
        int s_ = (call);               \
        if (s_ != ESL_OK) return s_;   \
    } while (0)

// ---- launch accounting: every kernel launch of the library is counted --------
void count_launch();
void count_launches(uint64_t n);  // kernels of a replayed CUDA graph
#define ESL_COUNT_LAUNCH() ::esl::count_launch()

// ---- host model -------------------------------------------------------------
struct Clause {
    uint32_t pos, neg;
};

struct Model {
    std::vector<std::string> names;
    std::vector<std::vector<Clause>> rules;
    int n() const { return (int)names.size(); }
};

int parse_bnet(const std::string& text, Model& out);

// ---- device memory cache --------------------------------------------------------
// Every device buffer of the library comes from a process-wide cache per device.  A
// released block stays mapped and is handed out again for a request of its size class:
// cudaFree / cudaMalloc of the ~25 buffers that a network's symbolic data and its
// temporaries hold took up to 0.8 s per build-and-free on the B200 (driver-side
// unmapping), against microseconds for the cache.  A release synchronises the device
// first, as cudaFree does, so a block is never handed out while work on it may still
// run (on the calling API's stream, else on the device).  A device keeps at most 8 GiB of
// cached blocks (the largest go first); when cudaMalloc fails the device's cached blocks
// are freed and the request is retried once.
void* dev_alloc(size_t bytes);  // nullptr on failure
void dev_free(void* p);
void dev_trim_all();            // frees every cached block of every device
// The stream of the API call running on this thread, or nullptr: a released block waits
// for that stream only.  A device-wide synchronisation could invalidate a CUDA-graph
// capture that another thread (another context of esl_solve_many) has in progress.
extern thread_local cudaStream_t t_api_stream;
// set while a caller that has already synchronised the device releases its blocks
extern thread_local bool t_released_synced;

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        p = static_cast<T*>(dev_alloc(count * sizeof(T)));
        if (!p) return fail(ESL_ERR_NOMEM, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
        n = count;
        return ESL_OK;
    }
    T* get() const { return p; }
};

// Grow-only device workspace kept in the context between calls.
struct Workspace {
    std::vector<std::pair<void*, size_t>> bufs;
    void* get(int slot, size_t bytes, int* status) {
        if ((int)bufs.size() <= slot) bufs.resize(slot + 1, {nullptr, 0});
        auto& b = bufs[slot];
        if (b.second < bytes) {
            if (b.first) dev_free(b.first);
            b.first = nullptr;
            b.second = 0;
            b.first = dev_alloc(bytes);
            if (!b.first) {
                *status = fail(ESL_ERR_NOMEM, "workspace allocation of " + std::to_string(bytes) + " bytes failed");
                return nullptr;
            }
            b.second = bytes;
        }
        return b.first;
    }
    void swap(int a, int b) {
        int m = std::max(a, b);
        if ((int)bufs.size() <= m) bufs.resize(m + 1, {nullptr, 0});
        std::swap(bufs[a], bufs[b]);
    }
    ~Workspace() {
        for (auto& b : bufs)
            if (b.first) dev_free(b.first);
    }
};

}  // namespace esl

// ---- public handles -------------------------------------------------------------
struct esl_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 148;
    uint32_t* h_flag = nullptr;       // pinned host scratch for fixpoint flags
    esl::DevBuf<unsigned long long> d_flag;  // device counters (8 slots)
    void* work = nullptr;             // solver workspace (grow-only), freed with the context
    void* sweep_work = nullptr;       // level-sweep workspace (grow-only), freed with the context
    cudaEvent_t poll_ev[4] = {nullptr, nullptr, nullptr, nullptr};  // convergence polls of the level sweep
    // level-sweep tiling of the last esl_net_autotune on this context (0 / -1: default),
    // used for networks that have no tuning of their own
    int tune_tile_mb = 0, tune_s2 = -1;
    // budgets of the fallback paths (esl_ctx_set_budgets; 0: the default)
    int64_t graph_sweeps = 0;   // sweeps per fixpoint loop of the graph stages
    int block_iters = 0;        // Krylov budget of the block forward solve
    int dense_max = 0;          // largest SCC block of the dense LU fallback
    // measurement hook: events around the launches of the hot kernels, each record
    // with its kernel class and algorithmic bytes
    bool prof = false;
    struct ProfRec {
        cudaEvent_t a, b;
        double bytes;
        const char* name;
    };
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> prof_pool;
    size_t prof_used = 0;
    cudaEvent_t prof_event() {
        if (prof_used == prof_pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            prof_pool.push_back(e);
        }
        return prof_pool[prof_used++];
    }
};

struct esl_model {
    esl::Model m;
};

struct esl_net {
    int n = 0;
    int64_t N = 0;
    uint32_t up_ok = 0, down_ok = 0;  // zero-rate pattern the net was built for
    int n_sccs = 0, T = 0, term_states = 0;
    esl::DevBuf<uint32_t> F, G;       // out / in flip masks
    esl::DevBuf<int32_t> labels;      // SCC label (min vertex) per state
    esl::DevBuf<int32_t> order;       // reordered vertices
    esl::DevBuf<int32_t> offsets;     // SCC offsets in order (n_sccs + 1)
    esl::DevBuf<int32_t> levels;      // level of the SCC at each offset position
    esl::DevBuf<int32_t> term_of;     // terminal SCC index per state, -1 if transient
    std::vector<int32_t> h_offsets;   // host copy of the terminal part of offsets (T + 1)
    esl::DevBuf<uint32_t> Gdom;       // in-mask restricted to same-class neighbours
    esl::DevBuf<uint32_t> Fdom;       // out-mask restricted to same-class neighbours
    int max_terminal = 0;             // largest terminal SCC
    // level-group plan of the block forward solve, built on first use
    void* plan = nullptr;
    void (*plan_free)(void*) = nullptr;
    // slot plan of the state-major level sweep, built on first use
    void* sweep = nullptr;
    // level-sweep tiling picked by esl_net_autotune: L2 slice budget in MB (0: default)
    // and two systems per thread on wide tiles (-1: default, on)
    int tune_tile_mb = 0, tune_s2 = -1;
    void (*sweep_free)(void*) = nullptr;
    ~esl_net() {
        if (plan && plan_free) plan_free(plan);
        if (sweep && sweep_free) sweep_free(sweep);
    }
};

namespace esl {

// Sets the stream of the API call on this thread for its lifetime (see t_api_stream).
struct StreamScope {
    cudaStream_t prev;
    explicit StreamScope(const esl_ctx* c) : prev(t_api_stream) {
        if (c) t_api_stream = c->stream;
    }
    ~StreamScope() { t_api_stream = prev; }
    StreamScope(const StreamScope&) = delete;
    StreamScope& operator=(const StreamScope&) = delete;
};

// Measurement hook: when profiling is on, CUDA events on the context's stream bracket
// the launches made while the scope lives; the record carries the kernel class and
// the algorithmic bytes of those launches.
struct ProfScope {
    esl_ctx* ctx;
    cudaEvent_t a = nullptr;
    const char* name;
    double bytes;
    ProfScope(esl_ctx* c, const char* nm, double b) : ctx(c && c->prof ? c : nullptr), name(nm), bytes(b) {
        if (ctx) {
            a = ctx->prof_event();
            cudaEventRecord(a, ctx->stream);
        }
    }
    ~ProfScope() {
        if (ctx) {
            cudaEvent_t e = ctx->prof_event();
            cudaEventRecord(e, ctx->stream);
            ctx->prof_recs.push_back({a, e, bytes, name});
        }
    }
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;
};

// table.cu
// States per count block of the table kernels: k_flip_masks writes one edge count per
// block, k_emit_csc starts each block's edges at the block's prefix offset.
constexpr int kTableBlockStates = 1024;
// Rule tables: node i's rule over the 32 states of a word depends only on the word's
// bits at the rule's variables of index >= 5 (at most kRuleTableMaxBits of them): a
// table of 2^k words (and a second one for the rule seen across bit i) replaces the
// clause loop.  At most kRuleTableMaxWords words in all; other nodes use the clauses.
constexpr int kRuleTableMaxBits = 8;
constexpr int kRuleTableMaxWords = 8192;
constexpr uint32_t kNoRuleTable = 0xFFFFFFFFu;
struct HostModel {
    std::vector<int32_t> off;     // clause offsets per node (n + 1)
    std::vector<uint32_t> pos, neg;
    std::vector<uint4> info;      // per node: (table offset, table bits or kNoRuleTable, bit positions 0-3, 4-7)
    std::vector<uint32_t> tab;    // the tables
    uint32_t self_dep = 0;        // nodes whose rule reads their own bit
};
void host_model(const Model& m, HostModel& hm);
struct DevModel {
    int n;
    const int32_t* off;
    const uint32_t* pos;
    const uint32_t* neg;
    const uint4* info;
    const uint32_t* tab;
    uint32_t tab_words;
    uint32_t up_ok, down_ok, self_dep;
};
struct DevModelBufs {
    DevBuf<int32_t> off;
    DevBuf<uint32_t> pos, neg, tab;
    DevBuf<uint4> info;
};
int upload_model(const Model& m, DevModelBufs& b, const double* rates, DevModel& dm, cudaStream_t s);
// zero-rate masks of a rate vector: bit i of up_ok / down_ok = rate 2i / 2i+1 nonzero
void rate_masks(int n, const double* rates, uint32_t& up_ok, uint32_t& down_ok);
int launch_flip_masks(const DevModel& dm, uint32_t* F, uint32_t* G, uint32_t* block_counts, cudaStream_t s);
int64_t flip_mask_blocks(int n);
int launch_emit_csc(int n, const uint32_t* F, const uint32_t* block_offsets_excl, int32_t* indptr, int32_t* rows,
                    int32_t* cols, int64_t nnz, cudaStream_t s);
// the same with 64-bit block offsets and column pointers (tables of >= 2^31 edges)
int launch_emit_csc64(int n, const uint32_t* F, const uint64_t* block_offsets_excl, int64_t* indptr, int32_t* rows,
                      int32_t* cols, int64_t nnz, cudaStream_t s);
int masks_from_csc(int n, const int32_t* indptr, const int32_t* rows, uint32_t* F, uint32_t* G,
                   unsigned long long* d_bad, cudaStream_t s);

// graph.cu
int build_graph(esl_ctx* ctx, esl_net* net);

// solve.cu
void free_workspace(void* w);

// Terminal SCCs of 2..kDenseTerminalMax states get their kernel from a dense FP64 LU
// (solve.cu); larger ones from the deflated Krylov solve of the level sweep (sweep.cu).
constexpr int kDenseTerminalMax = 128;

// sweep.cu: state-major level sweep of the transient forward solve.  Adds into
// y[k * T + t] the mass that terminal SCC t receives in system k (rate set k / nrhs,
// x0 row k % nrhs).  Systems that miss the tolerance are listed in `failed` (their y
// rows are left as computed) and the call returns ESL_ERR_NOT_CONVERGED.
struct SweepStats {
    int iters = 0, refinements = 0, local_groups = 0, krylov_groups = 0, compactions = 0;
    double relres = 0.0;
    std::vector<int32_t> failed;
};
bool sweep_supported(const esl_net* net);
int sweep_forward(esl_ctx* ctx, const esl_net* net, int K, int nrhs, const double* rates, const double* x0,
                  size_t x0_ld, const esl_solve_opts& o, double* y, SweepStats& st);
// Kernels of the terminal SCCs above kDenseTerminalMax states for B rate sets, FP64,
// into Rb[b][position] (positions of the reordering, B x term_states), normalised to
// sum 1 per SCC.  Systems that miss the acceptance residual are listed in `failed`
// (ESL_ERR_NOT_CONVERGED).
int sweep_terminal(esl_ctx* ctx, const esl_net* net, int B, const double* rates, const esl_solve_opts& o, double* Rb,
                   SweepStats& st);
void free_sweep_workspace(void* w);
// checksums (FNV-1a 64) of the 12 parts of a freshly built level-sweep plan: rows, desc,
// ig_ptr, ig_ent, og_ptr, og_ent, tp_ptr, tp_ent, lsc_off, lsc_ne, lsc_slots, group table;
// host != 0 builds it with the host reference builder instead of the device one
int plan_checksums_for(esl_ctx* ctx, const esl_net* net, int host, uint64_t* out, int cap);
// states whose warm start the sweep's grid-wide Krylov groups read (their odd-parity rows)
int sweep_targets(esl_ctx* ctx, const esl_net* net, std::vector<uint32_t>& states);
int solve_batch(esl_ctx* ctx, const esl_net* net, int B, const double* d_rates, int R, const double* d_x0,
                double* d_x_inf, double* d_marg, double* d_R, double* d_L, const esl_solve_opts* opts,
                esl_report* rep);

}  // namespace esl
