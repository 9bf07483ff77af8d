// SCC decomposition, terminal SCCs, levels and the vertex reordering, all on the
// device and all driven by the per-state flip masks (no adjacency arrays).
//
// Replaces transition_graph::reorganize_vertices (cuda/src/transition_graph.cu:123-202),
// its SCC solver (cuda/src/sga/two_phase.cu:12-145) and the level labelling
// (cuda/src/kernels/transition_graph.cu:3-27).
//
// Graph: edge s -> s ^ (1<<i) iff bit i of F[s]; edge s ^ (1<<i) -> s iff bit i of G[s].
// SCCs: iterated trim (a state with no live successor or no live predecessor is a
// singleton SCC), then rounds of forward max-colour propagation followed by a
// backward reach within each colour from its root (the state whose colour is its
// own id, i.e. the largest id of its SCC); every round removes at least one SCC
// per colour.  Labels are made canonical afterwards: the label of an SCC is its
// smallest state, the same label the reference gives singletons.
// Levels: level 1 = SCC without out-edges to other SCCs (terminal); otherwise
// 1 + max level of its successor SCCs (the reference's labelling fixpoint).
// Order: terminal SCCs by label ascending, then the others by decreasing level and,
// within a level, decreasing label -- the order the reference's stable sort by
// level and reversal produce (cuda/src/transition_graph.cu:151-184) -- with the
// states of an SCC ascending.
// Every fixpoint loop runs under an iteration budget and fails with ESL_ERR_TIMEOUT.
#include <chrono>
#include <cstdio>
#include <cstdlib>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(uint64_t N) { return (unsigned)((N + kThreads - 1) / kThreads); }

// flag slot 0: "changed" for the running fixpoint
__global__ void k_trim(int n, uint64_t N, const uint32_t* __restrict__ F, const uint32_t* __restrict__ G,
                       int32_t* __restrict__ lab, unsigned long long* __restrict__ flags) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N || lab[v] >= 0) return;
    uint32_t f = F[v], g = G[v];
    bool out_live = false, in_live = false;
    while (f && !out_live) {
        int i = __ffs(f) - 1;
        f &= f - 1;
        out_live = lab[v ^ (1ull << i)] < 0;
    }
    while (g && !in_live) {
        int i = __ffs(g) - 1;
        g &= g - 1;
        in_live = lab[v ^ (1ull << i)] < 0;
    }
    if (!(out_live && in_live)) {
        lab[v] = (int32_t)v;
        flags[0] = 1;
        atomicAdd(&flags[1], 1ull);
    }
}

__global__ void k_color_init(uint64_t N, const int32_t* __restrict__ lab, int32_t* __restrict__ color,
                             uint8_t* __restrict__ reached) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    color[v] = lab[v] < 0 ? (int32_t)v : -1;
    reached[v] = 0;
}

// colour(v) = max colour over live predecessors (chaotic, monotone)
__global__ void k_color_fw(uint64_t N, const uint32_t* __restrict__ G, const int32_t* __restrict__ lab,
                           int32_t* __restrict__ color, unsigned long long* __restrict__ flags) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N || lab[v] >= 0) return;
    int32_t c = color[v], m = c;
    uint32_t g = G[v];
    while (g) {
        int i = __ffs(g) - 1;
        g &= g - 1;
        uint64_t u = v ^ (1ull << i);
        if (lab[u] < 0) m = max(m, color[u]);
    }
    if (m > c) {
        color[v] = m;
        flags[0] = 1;
    }
}

__global__ void k_root_init(uint64_t N, const int32_t* __restrict__ lab, const int32_t* __restrict__ color,
                            uint8_t* __restrict__ reached) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    reached[v] = (lab[v] < 0 && color[v] == (int32_t)v) ? 1 : 0;
}

// v reaches its colour's root through live successors of the same colour
__global__ void k_reach_bw(uint64_t N, const uint32_t* __restrict__ F, const int32_t* __restrict__ lab,
                           const int32_t* __restrict__ color, uint8_t* __restrict__ reached,
                           unsigned long long* __restrict__ flags) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N || lab[v] >= 0 || reached[v]) return;
    int32_t c = color[v];
    uint32_t f = F[v];
    while (f) {
        int i = __ffs(f) - 1;
        f &= f - 1;
        uint64_t w = v ^ (1ull << i);
        if (lab[w] < 0 && color[w] == c && reached[w]) {
            reached[v] = 1;
            flags[0] = 1;
            return;
        }
    }
}

__global__ void k_assign(uint64_t N, int32_t* __restrict__ lab, const int32_t* __restrict__ color,
                         const uint8_t* __restrict__ reached, unsigned long long* __restrict__ flags) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N || lab[v] >= 0 || !reached[v]) return;
    lab[v] = color[v];
    atomicAdd(&flags[1], 1ull);
}

__global__ void k_fill(uint64_t N, int32_t* __restrict__ a, int32_t val) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N) a[v] = val;
}

__global__ void k_canon_min(uint64_t N, const int32_t* __restrict__ lab, int32_t* __restrict__ canon) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N) atomicMin(&canon[lab[v]], (int32_t)v);
}

__global__ void k_canon_apply(uint64_t N, int32_t* __restrict__ lab, const int32_t* __restrict__ canon) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N) lab[v] = canon[lab[v]];
}

// level per SCC stored at its label; 1 + max successor level
__global__ void k_level(uint64_t N, const uint32_t* __restrict__ F, const int32_t* __restrict__ lab,
                        int32_t* __restrict__ level, unsigned long long* __restrict__ flags) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    int32_t c = lab[v];
    int32_t best = 0;
    uint32_t f = F[v];
    while (f) {
        int i = __ffs(f) - 1;
        f &= f - 1;
        int32_t d = lab[v ^ (1ull << i)];
        if (d != c) best = max(best, level[d]);
    }
    best += 1;
    if (best > level[c]) {
        atomicMax(&level[c], best);
        flags[0] = 1;
    }
}

// sort key: terminal -> label; other -> (1, MAXLVL - level, MAXLBL - label)
__global__ void k_keys(uint64_t N, const int32_t* __restrict__ lab, const int32_t* __restrict__ level,
                       uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    int32_t c = lab[v];
    int32_t l = level[c];
    uint64_t k;
    if (l == 1)
        k = (uint64_t)c;
    else
        k = (1ull << 62) | ((uint64_t)(0x3FFFFFFF - l) << 31) | (uint64_t)(0x7FFFFFFF - c);
    keys[v] = k;
    vals[v] = (int32_t)v;
}

__global__ void k_heads(uint64_t N, const uint64_t* __restrict__ keys, int32_t* __restrict__ pos_out,
                        uint8_t* __restrict__ head) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    head[p] = (p == 0 || keys[p] != keys[p - 1]) ? 1 : 0;
    pos_out[p] = (int32_t)p;
}

__global__ void k_scc_levels(int n_sccs, const int32_t* __restrict__ offsets, const int32_t* __restrict__ order,
                             const int32_t* __restrict__ lab, const int32_t* __restrict__ level_by_label,
                             int32_t* __restrict__ level_at) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_sccs) return;
    level_at[k] = level_by_label[lab[order[offsets[k]]]];
}

__global__ void k_term_of(uint64_t N, int T, int term_states, const int32_t* __restrict__ offsets,
                          const int32_t* __restrict__ order, int32_t* __restrict__ term_of) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    if ((int64_t)p >= term_states) {
        term_of[order[p]] = -1;
        return;
    }
    int lo = 0, hi = T;  // offsets[lo] <= p < offsets[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (offsets[mid] <= (int32_t)p) lo = mid; else hi = mid;
    }
    term_of[order[p]] = lo;
}

// same-class masks: a neighbour counts only if both states are transient or both in
// the same terminal SCC
__global__ void k_domain_masks(int n, uint64_t N, const uint32_t* __restrict__ F, const uint32_t* __restrict__ G,
                               const int32_t* __restrict__ term_of, uint32_t* __restrict__ Fd,
                               uint32_t* __restrict__ Gd) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    int32_t c = term_of[v];
    uint32_t f = F[v], g = G[v], fd = 0, gd = 0;
    for (int i = 0; i < n; i++) {
        uint32_t b = 1u << i;
        if ((f | g) & b) {
            bool same = term_of[v ^ (1ull << i)] == c;
            if (same && (f & b)) fd |= b;
            if (same && (g & b)) gd |= b;
        }
    }
    Fd[v] = fd;
    Gd[v] = gd;
}

struct Flags {
    esl_ctx* ctx;
    int64_t reads = 0;
    int reset() {
        ESL_CUDA(cudaMemsetAsync(ctx->d_flag.get(), 0, 8 * sizeof(unsigned long long), ctx->stream));
        return ESL_OK;
    }
    int reset_changed() {
        ESL_CUDA(cudaMemsetAsync(ctx->d_flag.get(), 0, sizeof(unsigned long long), ctx->stream));
        return ESL_OK;
    }
    int read(unsigned long long* out, int count) {
        reads++;
        ESL_CUDA(cudaMemcpyAsync(ctx->h_flag, ctx->d_flag.get(), count * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
        ESL_CUDA(cudaStreamSynchronize(ctx->stream));
        std::memcpy(out, ctx->h_flag, count * sizeof(unsigned long long));
        return ESL_OK;
    }
};

// Runs `sweep` until it reports no change; `per_check` sweeps per host check.
template <class Sweep>
int fixpoint(Flags& fl, Sweep sweep, int per_check, int64_t budget, const char* what) {
    for (int64_t it = 0; it < budget; it += per_check) {
        ESL_TRY(fl.reset_changed());
        for (int k = 0; k < per_check; k++) ESL_TRY(sweep());
        unsigned long long ch = 0;
        ESL_TRY(fl.read(&ch, 1));
        if (!ch) return ESL_OK;
    }
    return fail(ESL_ERR_TIMEOUT, std::string("fixpoint budget exceeded in ") + what);
}

}  // namespace

int build_graph(esl_ctx* ctx, esl_net* net) {
    const uint64_t N = (uint64_t)net->N;
    const int n = net->n;
    cudaStream_t s = ctx->stream;
    const unsigned nb = blocks_for(N);
    const uint32_t* F = net->F.get();
    const uint32_t* G = net->G.get();
    Flags fl{ctx};
    const bool dbg = getenv("ESL_DEBUG") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    auto ms_since = [&]() {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    // budgets: a sweep can only fail to progress once per state (or the context's budget)
    const int64_t budget = ctx->graph_sweeps > 0 ? ctx->graph_sweeps : (int64_t)N + 64;
    // nominal algorithmic bytes of one fixpoint sweep (measurement hook): one pass over
    // every state's mask, label and colour / level word, 4 B each.  States already
    // assigned read only their label, so later sweeps move less than this.
    const double sweep_bytes = 12.0 * (double)N;

    ESL_TRY(net->labels.alloc(N));
    int32_t* lab = net->labels.get();
    DevBuf<int32_t> color, canon, level;
    DevBuf<uint8_t> reached;
    ESL_TRY(color.alloc(N));
    ESL_TRY(reached.alloc(N));
    ESL_COUNT_LAUNCH();
    k_fill<<<nb, kThreads, 0, s>>>(N, lab, -1);
    ESL_CUDA(cudaGetLastError());
    ESL_TRY(fl.reset());

    auto trim = [&]() -> int {
        return fixpoint(fl, [&]() -> int {
            ProfScope ps(ctx, "graph_sweep", sweep_bytes);
            ESL_COUNT_LAUNCH();
            k_trim<<<nb, kThreads, 0, s>>>(n, N, F, G, lab, ctx->d_flag.get());
            ESL_CUDA(cudaGetLastError());
            return ESL_OK;
        }, 2, budget, "trim");
    };
    ESL_TRY(trim());
    unsigned long long st[2];
    ESL_TRY(fl.read(st, 2));
    int64_t rounds = 0;
    while (st[1] < N) {
        if (++rounds > (int64_t)N) return fail(ESL_ERR_TIMEOUT, "SCC colouring rounds exceeded");
        ESL_COUNT_LAUNCH();
        k_color_init<<<nb, kThreads, 0, s>>>(N, lab, color.get(), reached.get());
        ESL_CUDA(cudaGetLastError());
        ESL_TRY(fixpoint(fl, [&]() -> int {
            ProfScope ps(ctx, "graph_sweep", sweep_bytes);
            ESL_COUNT_LAUNCH();
            k_color_fw<<<nb, kThreads, 0, s>>>(N, G, lab, color.get(), ctx->d_flag.get());
            ESL_CUDA(cudaGetLastError());
            return ESL_OK;
        }, 4, budget, "forward colouring"));
        ESL_COUNT_LAUNCH();
        k_root_init<<<nb, kThreads, 0, s>>>(N, lab, color.get(), reached.get());
        ESL_CUDA(cudaGetLastError());
        ESL_TRY(fixpoint(fl, [&]() -> int {
            ProfScope ps(ctx, "graph_sweep", sweep_bytes);
            ESL_COUNT_LAUNCH();
            k_reach_bw<<<nb, kThreads, 0, s>>>(N, F, lab, color.get(), reached.get(), ctx->d_flag.get());
            ESL_CUDA(cudaGetLastError());
            return ESL_OK;
        }, 4, budget, "backward reach"));
        ESL_COUNT_LAUNCH();
        k_assign<<<nb, kThreads, 0, s>>>(N, lab, color.get(), reached.get(), ctx->d_flag.get());
        ESL_CUDA(cudaGetLastError());
        ESL_TRY(trim());
        ESL_TRY(fl.read(st, 2));
    }
    if (dbg) fprintf(stderr, "[esl-graph] SCC: %lld rounds, %lld flag reads, %.1f ms\n", (long long)rounds,
                     (long long)fl.reads, ms_since());
    // canonical labels: smallest state of each SCC
    ESL_TRY(canon.alloc(N));
    ESL_COUNT_LAUNCH();
    k_fill<<<nb, kThreads, 0, s>>>(N, canon.get(), 0x7FFFFFFF);
    ESL_COUNT_LAUNCH();
    k_canon_min<<<nb, kThreads, 0, s>>>(N, lab, canon.get());
    ESL_COUNT_LAUNCH();
    k_canon_apply<<<nb, kThreads, 0, s>>>(N, lab, canon.get());
    ESL_CUDA(cudaGetLastError());

    // levels (indexed by label)
    ESL_TRY(level.alloc(N));
    ESL_COUNT_LAUNCH();
    k_fill<<<nb, kThreads, 0, s>>>(N, level.get(), 0);
    ESL_CUDA(cudaGetLastError());
    ESL_TRY(fixpoint(fl, [&]() -> int {
        ProfScope ps(ctx, "graph_sweep", sweep_bytes);
        ESL_COUNT_LAUNCH();
        k_level<<<nb, kThreads, 0, s>>>(N, F, lab, level.get(), ctx->d_flag.get());
        ESL_CUDA(cudaGetLastError());
        return ESL_OK;
    }, 4, budget, "levels"));

    // ordering by a stable radix sort of (class, level, label) keys
    {
        DevBuf<uint64_t> keys, keys_out;
        DevBuf<int32_t> vals, pos;
        DevBuf<uint8_t> head;
        ESL_TRY(keys.alloc(N));
        ESL_TRY(keys_out.alloc(N));
        ESL_TRY(vals.alloc(N));
        ESL_TRY(net->order.alloc(N));
        ESL_COUNT_LAUNCH();
        k_keys<<<nb, kThreads, 0, s>>>(N, lab, level.get(), keys.get(), vals.get());
        ESL_CUDA(cudaGetLastError());
        size_t tmp_bytes = 0;
        ESL_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.get(), keys_out.get(), vals.get(),
                                                 net->order.get(), (int64_t)N, 0, 64, s));
        DevBuf<uint8_t> tmp;
        ESL_TRY(tmp.alloc(tmp_bytes));
        ESL_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, keys.get(), keys_out.get(), vals.get(),
                                                 net->order.get(), (int64_t)N, 0, 64, s));
        // SCC heads
        ESL_TRY(pos.alloc(N));
        ESL_TRY(head.alloc(N));
        ESL_COUNT_LAUNCH();
        k_heads<<<nb, kThreads, 0, s>>>(N, keys_out.get(), pos.get(), head.get());
        ESL_CUDA(cudaGetLastError());
        DevBuf<int32_t> offs;
        DevBuf<int64_t> d_count;
        ESL_TRY(offs.alloc(N + 1));
        ESL_TRY(d_count.alloc(1));
        size_t sel_bytes = 0;
        ESL_CUDA(cub::DeviceSelect::Flagged(nullptr, sel_bytes, pos.get(), head.get(), offs.get(), d_count.get(),
                                            (int64_t)N, s));
        DevBuf<uint8_t> tmp2;
        ESL_TRY(tmp2.alloc(sel_bytes));
        ESL_CUDA(cub::DeviceSelect::Flagged(tmp2.get(), sel_bytes, pos.get(), head.get(), offs.get(), d_count.get(),
                                            (int64_t)N, s));
        int64_t n_sccs = 0;
        ESL_CUDA(cudaMemcpyAsync(&n_sccs, d_count.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        net->n_sccs = (int)n_sccs;
        ESL_TRY(net->offsets.alloc(n_sccs + 1));
        ESL_CUDA(cudaMemcpyAsync(net->offsets.get(), offs.get(), n_sccs * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
        int32_t Nend = (int32_t)N;
        ESL_CUDA(cudaMemcpyAsync(net->offsets.get() + n_sccs, &Nend, sizeof(int32_t), cudaMemcpyHostToDevice, s));
        ESL_TRY(net->levels.alloc(n_sccs));
        ESL_COUNT_LAUNCH();
        k_scc_levels<<<(unsigned)((n_sccs + kThreads - 1) / kThreads), kThreads, 0, s>>>(
            (int)n_sccs, net->offsets.get(), net->order.get(), lab, level.get(), net->levels.get());
        ESL_CUDA(cudaGetLastError());
        // terminal count: leading SCCs with level 1
        std::vector<int32_t> h_lv(n_sccs);
        ESL_CUDA(cudaMemcpyAsync(h_lv.data(), net->levels.get(), n_sccs * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        int T = 0;
        while (T < n_sccs && h_lv[T] == 1) T++;
        net->T = T;
        net->h_offsets.resize(T + 1);
        ESL_CUDA(cudaMemcpyAsync(net->h_offsets.data(), net->offsets.get(), (T + 1) * sizeof(int32_t),
                                 cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        net->term_states = net->h_offsets[T];
        net->max_terminal = 0;
        for (int t = 0; t < T; t++)
            net->max_terminal = std::max(net->max_terminal, net->h_offsets[t + 1] - net->h_offsets[t]);
    }
    ESL_TRY(net->term_of.alloc(N));
    ESL_COUNT_LAUNCH();
    k_term_of<<<nb, kThreads, 0, s>>>(N, net->T, net->term_states, net->offsets.get(), net->order.get(),
                                      net->term_of.get());
    ESL_CUDA(cudaGetLastError());
    ESL_TRY(net->Fdom.alloc(N));
    ESL_TRY(net->Gdom.alloc(N));
    ESL_COUNT_LAUNCH();
    k_domain_masks<<<nb, kThreads, 0, s>>>(n, N, F, G, net->term_of.get(), net->Fdom.get(), net->Gdom.get());
    ESL_CUDA(cudaGetLastError());
    ESL_CUDA(cudaStreamSynchronize(s));
    if (dbg) fprintf(stderr, "[esl-graph] done: %lld flag reads, %.1f ms\n", (long long)fl.reads, ms_since());
    return ESL_OK;
}

}  // namespace esl
