// C ABI of the library (declarations and reference citations in include/esl_b200.h).
#include <cub/device/device_scan.cuh>

#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <unordered_map>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

#include "esl_internal.h"

namespace esl {

static thread_local std::string g_error;
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ---- device memory cache (declared in esl_internal.h) ----------------------------------
namespace {
struct Block {
    size_t bytes;
    int dev;
};
std::mutex g_pool_mu;
std::unordered_map<void*, Block> g_pool_live;               // handed out
std::multimap<std::pair<int, size_t>, void*> g_pool_free;    // (device, size class) -> cached block
std::unordered_map<int, size_t> g_pool_cached;              // cached bytes per device
// cached bytes a device may keep; beyond it the largest cached blocks are freed
constexpr size_t kPoolCap = (size_t)8 << 30;

// size classes: powers of two up to 1 MiB, then multiples of 2 MiB
size_t size_class(size_t b) {
    if (b <= 256) return 256;
    if (b <= ((size_t)1 << 20)) {
        size_t c = 256;
        while (c < b) c <<= 1;
        return c;
    }
    const size_t g = (size_t)2 << 20;
    return (b + g - 1) / g * g;
}

// frees every cached block of device `dev` (the caller holds the lock)
void pool_trim(int dev) {
    for (auto it = g_pool_free.begin(); it != g_pool_free.end();) {
        if (it->first.first == dev) {
            cudaFree(it->second);
            it = g_pool_free.erase(it);
        } else {
            ++it;
        }
    }
    g_pool_cached[dev] = 0;
}
}  // namespace

void* dev_alloc(size_t bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    const size_t c = size_class(bytes);
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pool_free.find({dev, c});
    if (it != g_pool_free.end()) {
        void* p = it->second;
        g_pool_free.erase(it);
        g_pool_cached[dev] -= c;
        g_pool_live[p] = Block{c, dev};
        return p;
    }
    void* p = nullptr;
    if (cudaMalloc(&p, c) != cudaSuccess) {
        cudaGetLastError();  // clear the allocation error
        pool_trim(dev);
        p = nullptr;
        if (cudaMalloc(&p, c) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    g_pool_live[p] = Block{c, dev};
    return p;
}

thread_local cudaStream_t t_api_stream = nullptr;
thread_local bool t_released_synced = false;

void dev_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pool_live.find(p);
    if (it == g_pool_live.end()) return;
    const Block b = it->second;
    g_pool_live.erase(it);
    // as cudaFree: no work on the block may still run when it is handed out again
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b.dev) cudaSetDevice(b.dev);
    if (!t_released_synced) {
        if (t_api_stream)
            cudaStreamSynchronize(t_api_stream);
        else
            cudaDeviceSynchronize();
    }
    g_pool_free.insert({{b.dev, b.bytes}, p});
    size_t& cached = g_pool_cached[b.dev];
    cached += b.bytes;
    while (cached > kPoolCap) {
        // the device's largest cached block
        auto last = g_pool_free.upper_bound({b.dev, SIZE_MAX});
        if (last == g_pool_free.begin()) break;
        --last;
        if (last->first.first != b.dev) break;
        cudaFree(last->second);
        cached -= last->first.second;
        g_pool_free.erase(last);
    }
    if (cur != b.dev) cudaSetDevice(cur);
}

void dev_trim_all() {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& kv : g_pool_free) {
        cudaSetDevice(kv.first.first);
        cudaFree(kv.second);
    }
    g_pool_free.clear();
    g_pool_cached.clear();
    cudaSetDevice(cur);
}

void set_error(const std::string& msg) { g_error = msg; }
int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

namespace {

__global__ void k_initial_state(uint64_t N, uint32_t fixed_mask, uint32_t fixed_val, double p_fixed,
                                double p_other, double* __restrict__ x0) {
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    x0[s] = (((uint32_t)s & fixed_mask) == fixed_val) ? p_fixed : p_other;
}

int check_rates(const Model& m, const double* rates) {
    if (!rates) return fail(ESL_ERR_INVALID, "rates is NULL");
    for (int j = 0; j < 2 * m.n(); j++)
        if (!(rates[j] >= 0.0) || !std::isfinite(rates[j]))
            return fail(ESL_ERR_INVALID, "transition rate must be non-negative and finite");
    return ESL_OK;
}

int rate_map(const Model& m, int count, const char* const* names, const double* vals, std::vector<int>& idx) {
    idx.assign(m.n(), -1);
    if (count < 0 || (count > 0 && (!names || !vals))) return fail(ESL_ERR_INVALID, "bad explicit rate list");
    for (int k = 0; k < count; k++) {
        if (!names[k]) return fail(ESL_ERR_INVALID, "explicit rate without a node name");
        int found = -1;
        for (int i = 0; i < m.n(); i++)
            if (m.names[i] == names[k]) {
                found = i;
                break;
            }
        if (found < 0) return fail(ESL_ERR_INVALID, std::string("node ") + names[k] + " not found");
        if (vals[k] < 0) return fail(ESL_ERR_INVALID, "transition rate must be non-negative");
        idx[found] = k;
    }
    return ESL_OK;
}

// Table counts: masks + per-block edge counts; returns nnz.
int table_pass(esl_ctx* ctx, const Model& m, const double* rates, DevBuf<uint32_t>& F, DevBuf<uint32_t>& G,
               DevBuf<uint32_t>& counts, int64_t& nnz, bool want_G) {
    ESL_TRY(check_rates(m, rates));
    cudaStream_t s = ctx->stream;
    DevModelBufs mb;
    DevModel dm;
    ESL_TRY(upload_model(m, mb, rates, dm, s));
    const uint64_t N = 1ull << m.n();
    ESL_TRY(F.alloc(N));
    if (want_G) ESL_TRY(G.alloc(N));
    const int64_t blocks = flip_mask_blocks(m.n());
    ESL_TRY(counts.alloc(blocks + 1));
    {
        // algorithmic bytes: the masks written (4 B per state each) and the block counts
        ProfScope ps(ctx, "k_flip_masks", (double)N * (want_G ? 8.0 : 4.0) + 4.0 * blocks);
        ESL_TRY(launch_flip_masks(dm, F.get(), want_G ? G.get() : nullptr, counts.get(), s));
    }
    std::vector<uint32_t> h(blocks);
    ESL_CUDA(cudaMemcpyAsync(h.data(), counts.get(), blocks * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    nnz = 0;
    for (uint32_t c : h) nnz += c;
    return ESL_OK;
}

}  // namespace
}  // namespace esl

using namespace esl;

extern "C" {

const char* esl_last_error(void) { return g_error.c_str(); }
int esl_version(void) { return 100; }

int esl_trim_cache(void) {
    dev_trim_all();
    return ESL_OK;
}

int esl_launch_count(uint64_t* count) {
    if (!count) return fail(ESL_ERR_INVALID, "NULL argument");
    *count = g_launches.load();
    return ESL_OK;
}

int esl_ctx_create(int device, void* cuda_stream, esl_ctx** out) {
    if (!out) return fail(ESL_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int count = 0;
    ESL_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(ESL_ERR_INVALID, "no such CUDA device");
    ESL_CUDA(cudaSetDevice(device));
    auto* c = new esl_ctx();
    c->device = device;
    if (cuda_stream) {
        c->stream = (cudaStream_t)cuda_stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return fail(ESL_ERR_CUDA, "cudaStreamCreate failed");
        }
        c->own_stream = true;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaMallocHost(&c->h_flag, 64) != cudaSuccess || c->d_flag.alloc(8) != ESL_OK ||
        cudaEventCreateWithFlags(&c->poll_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->poll_ev[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->poll_ev[2], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->poll_ev[3], cudaEventDisableTiming) != cudaSuccess) {
        esl_ctx_destroy(c);
        return fail(ESL_ERR_NOMEM, "context allocation failed");
    }
    *out = c;
    return ESL_OK;
}

int esl_ctx_destroy(esl_ctx* c) {
    StreamScope stream_scope_(c);
    if (!c) return ESL_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->work) free_workspace(c->work);
    if (c->sweep_work) free_sweep_workspace(c->sweep_work);
    for (auto e : c->poll_ev)
        if (e) cudaEventDestroy(e);
    for (auto e : c->prof_pool) cudaEventDestroy(e);
    c->d_flag.release();
    if (c->h_flag) cudaFreeHost(c->h_flag);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return ESL_OK;
}

int esl_ctx_set_budgets(esl_ctx* c, int64_t graph_sweeps, int block_iters, int dense_max) {
    if (!c) return fail(ESL_ERR_INVALID, "ctx is NULL");
    c->graph_sweeps = graph_sweeps > 0 ? graph_sweeps : 0;
    c->block_iters = block_iters > 0 ? block_iters : 0;
    c->dense_max = dense_max > 0 ? dense_max : 0;
    return ESL_OK;
}

int esl_ctx_set_profiling(esl_ctx* c, int on) {
    if (!c) return fail(ESL_ERR_INVALID, "ctx is NULL");
    ESL_CUDA(cudaStreamSynchronize(c->stream));
    c->prof = on != 0;
    c->prof_recs.clear();
    c->prof_used = 0;
    return ESL_OK;
}

int esl_ctx_profile(esl_ctx* c, double* total_ms, double* total_bytes, int* launches) {
    if (!c || !total_ms || !total_bytes || !launches) return fail(ESL_ERR_INVALID, "NULL argument");
    ESL_CUDA(cudaStreamSynchronize(c->stream));
    double ms = 0.0, bytes = 0.0;
    for (auto& r : c->prof_recs) {
        float t = 0.f;
        ESL_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        ms += t;
        bytes += r.bytes;
    }
    *total_ms = ms;
    *total_bytes = bytes;
    *launches = (int)c->prof_recs.size();
    return ESL_OK;
}

int esl_ctx_profile_records(esl_ctx* c, int cap, double* ms, double* bytes, int* count) {
    if (!c || !count || cap < 0 || (cap > 0 && (!ms || !bytes))) return fail(ESL_ERR_INVALID, "bad argument");
    ESL_CUDA(cudaStreamSynchronize(c->stream));
    *count = (int)c->prof_recs.size();
    for (int i = 0; i < cap && i < *count; i++) {
        float t = 0.f;
        ESL_CUDA(cudaEventElapsedTime(&t, c->prof_recs[i].a, c->prof_recs[i].b));
        ms[i] = t;
        bytes[i] = c->prof_recs[i].bytes;
    }
    return ESL_OK;
}

int esl_ctx_profile_entry(esl_ctx* c, int i, const char** name, double* ms, double* bytes) {
    if (!c || !name || !ms || !bytes) return fail(ESL_ERR_INVALID, "NULL argument");
    if (i < 0 || i >= (int)c->prof_recs.size()) return fail(ESL_ERR_INVALID, "no such profile record");
    ESL_CUDA(cudaStreamSynchronize(c->stream));
    float t = 0.f;
    ESL_CUDA(cudaEventElapsedTime(&t, c->prof_recs[i].a, c->prof_recs[i].b));
    *name = c->prof_recs[i].name;
    *ms = t;
    *bytes = c->prof_recs[i].bytes;
    return ESL_OK;
}

int esl_net_autotune(esl_ctx* c, esl_net* net, int B, const double* d_rates, int R, const double* d_x0,
                     const esl_solve_opts* opts, int* tile_mb, int* two_per_thread, double* ms_out) {
    StreamScope stream_scope_(c);
    if (!c || !net || !d_rates || !d_x0 || B < 1 || R < 1) return fail(ESL_ERR_INVALID, "bad argument");
    const size_t N = (size_t)net->N;
    DevBuf<double> xbuf;
    ESL_TRY(xbuf.alloc((size_t)B * R * N));
    double* xi = xbuf.get();
    struct Cand {
        int mb, s2;
    };
    const Cand cands[] = {{48, 1}, {48, 0}, {16, 1}, {128, 1}};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = -1, rc = ESL_OK;
    float best_ms = 0.f;
    // one untimed solve first, so that the plan and workspaces exist
    net->tune_tile_mb = cands[0].mb;
    net->tune_s2 = cands[0].s2;
    rc = esl_solve_batch(c, net, B, d_rates, R, d_x0, xi, nullptr, opts, nullptr);
    for (int i = 0; rc == ESL_OK && i < (int)(sizeof cands / sizeof cands[0]); i++) {
        net->tune_tile_mb = cands[i].mb;
        net->tune_s2 = cands[i].s2;
        cudaEventRecord(e0, c->stream);
        rc = esl_solve_batch(c, net, B, d_rates, R, d_x0, xi, nullptr, opts, nullptr);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rc == ESL_OK && (best < 0 || ms < best_ms)) {
            best = i;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best < 0) {
        net->tune_tile_mb = 0;
        net->tune_s2 = -1;
        return rc != ESL_OK ? rc : fail(ESL_ERR_INVALID, "autotune found no configuration");
    }
    net->tune_tile_mb = c->tune_tile_mb = cands[best].mb;
    net->tune_s2 = c->tune_s2 = cands[best].s2;
    if (tile_mb) *tile_mb = cands[best].mb;
    if (two_per_thread) *two_per_thread = cands[best].s2;
    if (ms_out) *ms_out = best_ms;
    return ESL_OK;
}

int esl_ctx_synchronize(esl_ctx* c) {
    if (!c) return fail(ESL_ERR_INVALID, "ctx is NULL");
    ESL_CUDA(cudaStreamSynchronize(c->stream));
    return ESL_OK;
}

int esl_model_parse(const char* text, esl_model** out) {
    if (!text || !out) return fail(ESL_ERR_INVALID, "NULL argument");
    auto* m = new esl_model();
    int st = parse_bnet(text, m->m);
    if (st != ESL_OK) {
        delete m;
        *out = nullptr;
        return st;
    }
    *out = m;
    return ESL_OK;
}

int esl_model_load(const char* path, esl_model** out) {
    if (!path || !out) return fail(ESL_ERR_INVALID, "NULL argument");
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return fail(ESL_ERR_INVALID, "could not open model file");
    std::stringstream ss;
    ss << f.rdbuf();
    return esl_model_parse(ss.str().c_str(), out);
}

int esl_model_free(esl_model* m) {
    delete m;
    return ESL_OK;
}

int esl_model_nodes(const esl_model* m, int* n) {
    if (!m || !n) return fail(ESL_ERR_INVALID, "NULL argument");
    *n = m->m.n();
    return ESL_OK;
}

const char* esl_model_node_name(const esl_model* m, int i) {
    if (!m || i < 0 || i >= m->m.n()) return nullptr;
    return m->m.names[i].c_str();
}

int esl_model_node_index(const esl_model* m, const char* name, int* index) {
    if (!m || !name || !index) return fail(ESL_ERR_INVALID, "NULL argument");
    for (int i = 0; i < m->m.n(); i++)
        if (m->m.names[i] == name) {
            *index = i;
            return ESL_OK;
        }
    return fail(ESL_ERR_INVALID, std::string("node ") + name + " not found");
}

int esl_model_clauses(const esl_model* m, int32_t* off, uint32_t* pos, uint32_t* neg, int cap, int* total) {
    if (!m || !total) return fail(ESL_ERR_INVALID, "NULL argument");
    int t = 0;
    for (auto& r : m->m.rules) t += (int)r.size();
    *total = t;
    if (cap < t || !off || !pos || !neg) return ESL_OK;
    int k = 0;
    off[0] = 0;
    for (int i = 0; i < m->m.n(); i++) {
        for (auto& c : m->m.rules[i]) {
            pos[k] = c.pos;
            neg[k] = c.neg;
            k++;
        }
        off[i + 1] = k;
    }
    return ESL_OK;
}

int esl_rates_uniform(const esl_model* m, int n_up, const char* const* up_names, const double* up_vals, int n_down,
                      const char* const* down_names, const double* down_vals, double* rates_out) {
    if (!m || !rates_out) return fail(ESL_ERR_INVALID, "NULL argument");
    std::vector<int> ui, di;
    ESL_TRY(rate_map(m->m, n_up, up_names, up_vals, ui));
    ESL_TRY(rate_map(m->m, n_down, down_names, down_vals, di));
    for (int i = 0; i < m->m.n(); i++) {
        rates_out[2 * i] = ui[i] >= 0 ? up_vals[ui[i]] : 1.0;
        rates_out[2 * i + 1] = di[i] >= 0 ? down_vals[di[i]] : 1.0;
    }
    return ESL_OK;
}

// Same generator as transition_rates::generate_normal (cuda/src/transition_rates.cpp:75-97):
// std::default_random_engine (default-seeded when seed == 0) and a float normal
// distribution, redrawing negatives up to 1000 times, node by node, up before down.
int esl_rates_normal(const esl_model* m, double mean, double stddev, uint64_t seed, int n_up,
                     const char* const* up_names, const double* up_vals, int n_down, const char* const* down_names,
                     const double* down_vals, double* rates_out) {
    if (!m || !rates_out) return fail(ESL_ERR_INVALID, "NULL argument");
    std::vector<int> ui, di;
    ESL_TRY(rate_map(m->m, n_up, up_names, up_vals, ui));
    ESL_TRY(rate_map(m->m, n_down, down_names, down_vals, di));
    std::default_random_engine gen;
    if (seed) gen.seed((std::default_random_engine::result_type)seed);
    std::normal_distribution<float> dist((float)mean, (float)stddev);
    auto draw = [&](double& out) -> int {
        float v;
        int count = 0;
        do {
            v = dist(gen);
            count++;
        } while (v < 0 && count < 1000);
        if (v < 0) return fail(ESL_ERR_INVALID, "could not generate positive transition rates with the provided mean and std");
        out = v;
        return ESL_OK;
    };
    for (int i = 0; i < m->m.n(); i++) {
        if (ui[i] >= 0) rates_out[2 * i] = up_vals[ui[i]];
        else ESL_TRY(draw(rates_out[2 * i]));
        if (di[i] >= 0) rates_out[2 * i + 1] = down_vals[di[i]];
        else ESL_TRY(draw(rates_out[2 * i + 1]));
    }
    return ESL_OK;
}

int esl_initial_state(esl_ctx* ctx, const esl_model* m, int n_fixed, const char* const* fixed_names,
                      const int* fixed_values, double fixed_probability, double* d_x0) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !d_x0 || (n_fixed > 0 && (!fixed_names || !fixed_values)))
        return fail(ESL_ERR_INVALID, "NULL argument");
    const int n = m->m.n();
    const uint64_t N = 1ull << n;
    uint32_t mask = 0, val = 0;
    for (int k = 0; k < n_fixed; k++) {
        if (!fixed_names[k]) return fail(ESL_ERR_INVALID, "fixed node without a name");
        int idx = -1;
        for (int i = 0; i < n; i++)
            if (m->m.names[i] == fixed_names[k]) {
                idx = i;
                break;
            }
        if (idx < 0) return fail(ESL_ERR_INVALID, std::string("invalid initial node name: ") + fixed_names[k]);
        mask |= 1u << idx;
        if (fixed_values[k]) val |= 1u << idx;
    }
    double p_fixed, p_other;
    if (n_fixed == 0) {
        p_fixed = p_other = 1.0 / (double)N;
    } else {
        uint64_t match = N >> __builtin_popcount(mask);
        p_fixed = fixed_probability / (double)match;
        p_other = match == N ? 0.0 : (1.0 - fixed_probability) / (double)(N - match);
    }
    ESL_COUNT_LAUNCH();
    k_initial_state<<<(unsigned)((N + 255) / 256), 256, 0, ctx->stream>>>(N, mask, val, p_fixed, p_other, d_x0);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int esl_table_nnz(esl_ctx* ctx, const esl_model* m, const double* rates, int64_t* nnz) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !nnz) return fail(ESL_ERR_INVALID, "NULL argument");
    DevBuf<uint32_t> F, G, counts;
    ESL_TRY(table_pass(ctx, m->m, rates, F, G, counts, *nnz, false));
    return ESL_OK;
}

int esl_table_build(esl_ctx* ctx, const esl_model* m, const double* rates, int32_t* d_indptr, int32_t* d_rows,
                    int32_t* d_cols) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !d_indptr || !d_rows) return fail(ESL_ERR_INVALID, "NULL argument");
    DevBuf<uint32_t> F, G, counts;
    int64_t nnz = 0;
    ESL_TRY(table_pass(ctx, m->m, rates, F, G, counts, nnz, false));
    if (nnz >= (int64_t)INT32_MAX) return fail(ESL_ERR_TOO_LARGE, "more than 2^31-1 transitions");
    const int64_t blocks = flip_mask_blocks(m->m.n());
    DevBuf<uint32_t> offs;
    ESL_TRY(offs.alloc(blocks));
    size_t tmp = 0;
    ESL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, counts.get(), offs.get(), (int)blocks, ctx->stream));
    DevBuf<uint8_t> tbuf;
    ESL_TRY(tbuf.alloc(tmp));
    ESL_CUDA(cub::DeviceScan::ExclusiveSum(tbuf.get(), tmp, counts.get(), offs.get(), (int)blocks, ctx->stream));
    {
        // algorithmic bytes: the out-masks read and indptr written (4 B per state each),
        // destinations (and sources) written (4 B per edge each)
        const double N = (double)(1ull << m->m.n());
        ProfScope ps(ctx, "k_emit_csc", 8.0 * N + 4.0 + (d_cols ? 8.0 : 4.0) * (double)nnz);
        ESL_TRY(launch_emit_csc(m->m.n(), F.get(), offs.get(), d_indptr, d_rows, d_cols, nnz, ctx->stream));
    }
    ESL_CUDA(cudaStreamSynchronize(ctx->stream));
    return ESL_OK;
}

int esl_table_build64(esl_ctx* ctx, const esl_model* m, const double* rates, int64_t* d_indptr, int32_t* d_rows,
                      int32_t* d_cols) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !d_indptr || !d_rows) return fail(ESL_ERR_INVALID, "NULL argument");
    DevBuf<uint32_t> F, G, counts;
    int64_t nnz = 0;
    ESL_TRY(table_pass(ctx, m->m, rates, F, G, counts, nnz, false));
    const int64_t blocks = flip_mask_blocks(m->m.n());
    DevBuf<uint64_t> offs;
    ESL_TRY(offs.alloc(blocks));
    // 64-bit running sum of the 32-bit block counts (the initial value sets the sum's type)
    size_t tmp = 0;
    ESL_CUDA(cub::DeviceScan::ExclusiveScan(nullptr, tmp, counts.get(), offs.get(), cub::Sum(), (uint64_t)0,
                                            (int)blocks, ctx->stream));
    DevBuf<uint8_t> tbuf;
    ESL_TRY(tbuf.alloc(tmp));
    ESL_CUDA(cub::DeviceScan::ExclusiveScan(tbuf.get(), tmp, counts.get(), offs.get(), cub::Sum(), (uint64_t)0,
                                            (int)blocks, ctx->stream));
    {
        // algorithmic bytes: the out-masks read (4 B per state), indptr written (8 B per
        // state), destinations (and sources) written (4 B per edge each)
        const double N = (double)(1ull << m->m.n());
        ProfScope ps(ctx, "k_emit_csc64", 12.0 * N + 8.0 + (d_cols ? 8.0 : 4.0) * (double)nnz);
        ESL_TRY(launch_emit_csc64(m->m.n(), F.get(), offs.get(), d_indptr, d_rows, d_cols, nnz, ctx->stream));
    }
    ESL_CUDA(cudaStreamSynchronize(ctx->stream));
    return ESL_OK;
}

int esl_flip_masks(esl_ctx* ctx, const esl_model* m, const double* rates, uint32_t* d_out, uint32_t* d_in) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !d_out) return fail(ESL_ERR_INVALID, "NULL argument");
    ESL_TRY(check_rates(m->m, rates));
    DevModelBufs mb;
    DevModel dm;
    ESL_TRY(upload_model(m->m, mb, rates, dm, ctx->stream));
    ESL_TRY(launch_flip_masks(dm, d_out, d_in, nullptr, ctx->stream));
    ESL_CUDA(cudaStreamSynchronize(ctx->stream));
    return ESL_OK;
}

int esl_net_build(esl_ctx* ctx, const esl_model* m, const double* rates, esl_net** out) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !out) return fail(ESL_ERR_INVALID, "NULL argument");
    *out = nullptr;
    ESL_TRY(check_rates(m->m, rates));
    auto* net = new esl_net();
    net->n = m->m.n();
    net->N = 1ll << net->n;
    for (int i = 0; i < net->n; i++) {
        if (rates[2 * i] != 0.0) net->up_ok |= 1u << i;
        if (rates[2 * i + 1] != 0.0) net->down_ok |= 1u << i;
    }
    DevBuf<uint32_t> counts;
    int64_t nnz = 0;
    int st = table_pass(ctx, m->m, rates, net->F, net->G, counts, nnz, true);
    if (st == ESL_OK) st = build_graph(ctx, net);
    if (st != ESL_OK) {
        delete net;
        return st;
    }
    *out = net;
    return ESL_OK;
}

int esl_net_from_csc(esl_ctx* ctx, int n_nodes, const int32_t* d_indptr, const int32_t* d_rows, esl_net** out) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !d_indptr || !d_rows || !out) return fail(ESL_ERR_INVALID, "NULL argument");
    if (n_nodes < 1 || n_nodes > ESL_MAX_NODES) return fail(ESL_ERR_INVALID, "node count out of range");
    *out = nullptr;
    auto* net = new esl_net();
    net->n = n_nodes;
    net->N = 1ll << n_nodes;
    net->up_ok = net->down_ok = (n_nodes >= 32) ? ~0u : ((1u << n_nodes) - 1);
    int st = net->F.alloc(net->N);
    if (st == ESL_OK) st = net->G.alloc(net->N);
    if (st == ESL_OK) {
        ESL_CUDA(cudaMemsetAsync(ctx->d_flag.get(), 0, 8, ctx->stream));
        st = masks_from_csc(n_nodes, d_indptr, d_rows, net->F.get(), net->G.get(), ctx->d_flag.get(), ctx->stream);
    }
    if (st == ESL_OK) {
        unsigned long long bad = 0;
        ESL_CUDA(cudaMemcpyAsync(&bad, ctx->d_flag.get(), 8, cudaMemcpyDeviceToHost, ctx->stream));
        ESL_CUDA(cudaStreamSynchronize(ctx->stream));
        if (bad) st = fail(ESL_ERR_INVALID, "table has edges that do not flip exactly one bit");
    }
    if (st == ESL_OK) st = build_graph(ctx, net);
    if (st != ESL_OK) {
        delete net;
        return st;
    }
    *out = net;
    return ESL_OK;
}

int esl_net_free(esl_net* net) {
    if (!net) return ESL_OK;
    // a net's buffers may have been read on any context's stream: one device-wide wait,
    // then its blocks go back to the cache without further waits
    cudaDeviceSynchronize();
    t_released_synced = true;
    delete net;
    t_released_synced = false;
    return ESL_OK;
}

int esl_net_info(const esl_net* net, int* n_nodes, int* n_sccs, int* n_terminals, int* n_terminal_states) {
    if (!net) return fail(ESL_ERR_INVALID, "net is NULL");
    if (n_nodes) *n_nodes = net->n;
    if (n_sccs) *n_sccs = net->n_sccs;
    if (n_terminals) *n_terminals = net->T;
    if (n_terminal_states) *n_terminal_states = net->term_states;
    return ESL_OK;
}

int esl_net_export(esl_ctx* ctx, const esl_net* net, int32_t* d_order, int32_t* d_offsets, int32_t* d_levels,
                   int32_t* d_labels) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !net) return fail(ESL_ERR_INVALID, "NULL argument");
    cudaStream_t s = ctx->stream;
    if (d_order) ESL_CUDA(cudaMemcpyAsync(d_order, net->order.get(), net->N * 4, cudaMemcpyDeviceToDevice, s));
    if (d_offsets)
        ESL_CUDA(cudaMemcpyAsync(d_offsets, net->offsets.get(), (net->n_sccs + 1) * 4, cudaMemcpyDeviceToDevice, s));
    if (d_levels) ESL_CUDA(cudaMemcpyAsync(d_levels, net->levels.get(), net->n_sccs * 4, cudaMemcpyDeviceToDevice, s));
    if (d_labels) ESL_CUDA(cudaMemcpyAsync(d_labels, net->labels.get(), net->N * 4, cudaMemcpyDeviceToDevice, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    return ESL_OK;
}

int esl_net_plan_checksums(esl_ctx* ctx, const esl_net* net, int host_builder, uint64_t* sums, int cap) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !net || !sums || cap < 0) return fail(ESL_ERR_INVALID, "bad argument");
    return plan_checksums_for(ctx, net, host_builder, sums, cap);
}

int esl_net_compatible(const esl_net* net, const double* rates, int* compatible) {
    if (!net || !rates || !compatible) return fail(ESL_ERR_INVALID, "NULL argument");
    uint32_t up = 0, down = 0;
    for (int i = 0; i < net->n; i++) {
        if (rates[2 * i] != 0.0) up |= 1u << i;
        if (rates[2 * i + 1] != 0.0) down |= 1u << i;
    }
    *compatible = (up == net->up_ok && down == net->down_ok) ? 1 : 0;
    return ESL_OK;
}

static int check_batch_rates(esl_ctx* ctx, const esl_net* net, int B, const double* d_rates) {
    std::vector<double> h((size_t)B * 2 * net->n);
    ESL_CUDA(cudaMemcpyAsync(h.data(), d_rates, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    ESL_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int b = 0; b < B; b++) {
        const double* r = h.data() + (size_t)b * 2 * net->n;
        for (int j = 0; j < 2 * net->n; j++)
            if (!(r[j] >= 0.0) || !std::isfinite(r[j]))
                return fail(ESL_ERR_INVALID, "rate set " + std::to_string(b) + " has a negative or non-finite rate");
        int ok = 0;
        esl_net_compatible(net, r, &ok);
        if (!ok)
            return fail(ESL_ERR_INVALID,
                        "rate set " + std::to_string(b) + " has a different zero pattern than the network was built for");
    }
    return ESL_OK;
}

int esl_solve(esl_ctx* ctx, const esl_net* net, const double* d_rates, const double* d_x0, double* d_x_inf,
              double* d_marginals, double* d_R, double* d_L, const esl_solve_opts* opts, esl_report* report) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !net || !d_rates || !d_x0) return fail(ESL_ERR_INVALID, "NULL argument");
    ESL_TRY(check_batch_rates(ctx, net, 1, d_rates));
    return solve_batch(ctx, net, 1, d_rates, 1, d_x0, d_x_inf, d_marginals, d_R, d_L, opts, report);
}

int esl_solve_batch(esl_ctx* ctx, const esl_net* net, int B, const double* d_rates, int R, const double* d_x0,
                    double* d_x_inf, double* d_marginals, const esl_solve_opts* opts, esl_report* report) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !net || !d_rates || !d_x0) return fail(ESL_ERR_INVALID, "NULL argument");
    if (B < 1 || R < 1 || (int64_t)B * R > 65535) return fail(ESL_ERR_INVALID, "B*R must be in [1, 65535]");
    ESL_TRY(check_batch_rates(ctx, net, B, d_rates));
    return solve_batch(ctx, net, B, d_rates, R, d_x0, d_x_inf, d_marginals, nullptr, nullptr, opts, report);
}

int esl_solve_host(esl_ctx* ctx, const esl_model* m, int B, const double* rates, int R, const double* x0,
                   double* x_inf, double* marginals, const esl_solve_opts* opts, esl_report* report) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !m || !rates || !x0 || !x_inf) return fail(ESL_ERR_INVALID, "NULL argument");
    if (B < 1 || R < 1) return fail(ESL_ERR_INVALID, "B and R must be positive");
    const int n = m->m.n();
    const size_t N = (size_t)1 << n;
    cudaStream_t s = ctx->stream;
    esl_net* net = nullptr;
    ESL_TRY(esl_net_build(ctx, m, rates, &net));
    DevBuf<double> dr, dx0, dxi, dm;
    int st = dr.alloc((size_t)B * 2 * n);
    if (st == ESL_OK) st = dx0.alloc((size_t)R * N);
    if (st == ESL_OK) st = dxi.alloc((size_t)B * R * N);
    if (st == ESL_OK && marginals) st = dm.alloc((size_t)B * R * n);
    if (st == ESL_OK) {
        if (cudaMemcpyAsync(dr.get(), rates, (size_t)B * 2 * n * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(dx0.get(), x0, (size_t)R * N * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
            st = fail(ESL_ERR_CUDA, "copy to the device failed");
        else
            st = esl_solve_batch(ctx, net, B, dr.get(), R, dx0.get(), dxi.get(), marginals ? dm.get() : nullptr,
                                 opts, report);
    }
    if (st == ESL_OK) {
        if (cudaMemcpyAsync(x_inf, dxi.get(), (size_t)B * R * N * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            (marginals &&
             cudaMemcpyAsync(marginals, dm.get(), (size_t)B * R * n * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
            cudaStreamSynchronize(s) != cudaSuccess)
            st = fail(ESL_ERR_CUDA, "copy back failed");
    }
    esl_net_free(net);
    return st;
}

}  // extern "C"
