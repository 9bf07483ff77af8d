// Allocation-free variant of the transition-table build (esl_table_build_static).
//
// Some callers cannot allocate device memory at the point where they need the table:
//   - code running inside a framework whose caching allocator has already reserved
//     the GPU's memory for itself, so a cudaMalloc by a library would fail or
//     fragment the pool;
//   - latency-sensitive loops, because cudaFree (and often cudaMalloc) synchronises
//     the whole device and stalls every other stream of the process;
//   - services that do all their allocation once at start-up and forbid it later.
// This entry point takes no context and allocates nothing.  All of its scratch
// lives in one file-scope __device__ array, sized for networks of up to
// ESL_STATIC_TABLE_MAX_NODES nodes.  Every GPU that loads the library holds that
// array until the process exits.
//
// The scratch is shared by every call on a device and keeps the last call's
// contents.  Each call writes every scratch word it reads before reading it (the
// clause lists, the per-state out-masks, the per-block edge counts and their
// prefix sums), so nothing needs clearing between calls.  Calls whose GPU work
// overlaps (two streams, or two host threads) race on the array: serialise them.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <mutex>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kStaticMaxNodes = ESL_STATIC_TABLE_MAX_NODES;
constexpr size_t kStaticStates = (size_t)1 << kStaticMaxNodes;
constexpr size_t kStaticBlocks = kStaticStates / kTableBlockStates;  // count blocks of the table kernels
constexpr size_t kStaticClauses = ESL_STATIC_TABLE_MAX_CLAUSES;
constexpr size_t kScanTempBytes = 64 * 1024;
// The CSC offsets are int32: at most n * 2^n edges must fit below 2^31.
static_assert(((int64_t)kStaticMaxNodes << kStaticMaxNodes) < (int64_t)INT32_MAX,
              "ESL_STATIC_TABLE_MAX_NODES allows more edges than int32 CSC offsets hold");

// byte offsets of the regions inside the scratch array (each 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffClauseOff = 0;
constexpr size_t kOffPos = align256(kOffClauseOff + (ESL_MAX_NODES + 1) * sizeof(int32_t));
constexpr size_t kOffNeg = align256(kOffPos + kStaticClauses * sizeof(uint32_t));
constexpr size_t kOffInfo = align256(kOffNeg + kStaticClauses * sizeof(uint32_t));
constexpr size_t kOffTab = align256(kOffInfo + ESL_MAX_NODES * sizeof(uint4));
constexpr size_t kOffF = align256(kOffTab + kRuleTableMaxWords * sizeof(uint32_t));
constexpr size_t kOffCounts = align256(kOffF + kStaticStates * sizeof(uint32_t));
constexpr size_t kOffOffsets = align256(kOffCounts + (kStaticBlocks + 1) * sizeof(uint32_t));
constexpr size_t kOffScan = align256(kOffOffsets + (kStaticBlocks + 1) * sizeof(uint32_t));
constexpr size_t kScratchBytes = align256(kOffScan + kScanTempBytes);

__device__ __align__(256) unsigned char g_table_scratch[kScratchBytes];

// Device address of g_table_scratch per device.  In host code the symbol is a
// host-side stand-in, never a device address, so it is looked up once per device
// with that device current.  The cached address belongs to the device's primary
// context: after cudaDeviceReset it is stale, and the process must not call this
// entry point on that device again.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

int scratch_for_current_device(unsigned char** out) {
    int dev = -1;
    ESL_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(ESL_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_table_scratch);
        if (e != cudaSuccess || !p)
            return fail(ESL_ERR_CUDA, std::string("cudaGetSymbolAddress(table scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return ESL_OK;
}

}  // namespace
}  // namespace esl

using namespace esl;

extern "C" int esl_table_build_static(const esl_model* m, const double* rates, void* cuda_stream, int32_t* d_indptr,
                                      int32_t* d_rows, int32_t* d_cols, int64_t rows_capacity, int64_t* nnz_out) {
    if (!m || !rates || !d_indptr || !d_rows || !nnz_out) return fail(ESL_ERR_INVALID, "NULL argument");
    *nnz_out = 0;
    const Model& model = m->m;
    const int n = model.n();
    if (n < 1) return fail(ESL_ERR_INVALID, "model has no nodes");
    if (n > kStaticMaxNodes)
        return fail(ESL_ERR_TOO_LARGE, "esl_table_build_static handles at most " + std::to_string(kStaticMaxNodes) +
                                           " nodes; this model has " + std::to_string(n));
    for (int j = 0; j < 2 * n; j++)
        if (!(rates[j] >= 0.0) || !std::isfinite(rates[j]))
            return fail(ESL_ERR_INVALID, "transition rate must be non-negative and finite");

    // clause lists and rule tables on the host (host memory only)
    HostModel hm;
    host_model(model, hm);
    if (hm.pos.size() > kStaticClauses)
        return fail(ESL_ERR_TOO_LARGE, "esl_table_build_static handles at most " + std::to_string(kStaticClauses) +
                                           " DNF clauses; this model has " + std::to_string(hm.pos.size()));

    unsigned char* base = nullptr;
    ESL_TRY(scratch_for_current_device(&base));
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    int32_t* d_off = reinterpret_cast<int32_t*>(base + kOffClauseOff);
    uint32_t* d_pos = reinterpret_cast<uint32_t*>(base + kOffPos);
    uint32_t* d_neg = reinterpret_cast<uint32_t*>(base + kOffNeg);
    uint4* d_info = reinterpret_cast<uint4*>(base + kOffInfo);
    uint32_t* d_tab = reinterpret_cast<uint32_t*>(base + kOffTab);
    uint32_t* F = reinterpret_cast<uint32_t*>(base + kOffF);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base + kOffCounts);
    uint32_t* offs = reinterpret_cast<uint32_t*>(base + kOffOffsets);
    void* scan_tmp = base + kOffScan;

    ESL_CUDA(cudaMemcpyAsync(d_off, hm.off.data(), hm.off.size() * 4, cudaMemcpyHostToDevice, s));
    if (!hm.pos.empty()) {
        ESL_CUDA(cudaMemcpyAsync(d_pos, hm.pos.data(), hm.pos.size() * 4, cudaMemcpyHostToDevice, s));
        ESL_CUDA(cudaMemcpyAsync(d_neg, hm.neg.data(), hm.neg.size() * 4, cudaMemcpyHostToDevice, s));
    }
    ESL_CUDA(cudaMemcpyAsync(d_info, hm.info.data(), hm.info.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    if (!hm.tab.empty())
        ESL_CUDA(cudaMemcpyAsync(d_tab, hm.tab.data(), hm.tab.size() * 4, cudaMemcpyHostToDevice, s));
    DevModel dm;
    dm.n = n;
    dm.off = d_off;
    dm.pos = d_pos;
    dm.neg = d_neg;
    dm.info = d_info;
    dm.tab = d_tab;
    dm.tab_words = (uint32_t)hm.tab.size();
    rate_masks(n, rates, dm.up_ok, dm.down_ok);
    dm.self_dep = hm.self_dep;

    // out-masks and per-block edge counts, then the edge total on the host
    ESL_TRY(launch_flip_masks(dm, F, nullptr, counts, s));
    const int64_t blocks = flip_mask_blocks(n);
    std::vector<uint32_t> h_counts((size_t)blocks);
    ESL_CUDA(cudaMemcpyAsync(h_counts.data(), counts, (size_t)blocks * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    int64_t nnz = 0;
    for (uint32_t c : h_counts) nnz += c;
    *nnz_out = nnz;
    if (nnz > rows_capacity)
        return fail(ESL_ERR_TOO_LARGE, "the table has " + std::to_string(nnz) + " transitions but rows_capacity is " +
                                           std::to_string(rows_capacity));

    // block offsets with the scan's temporary storage inside the scratch array
    size_t tmp = 0;
    ESL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, counts, offs, (int)blocks, s));
    if (tmp > kScanTempBytes) return fail(ESL_ERR_TOO_LARGE, "scan scratch larger than reserved");
    ESL_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, tmp, counts, offs, (int)blocks, s));
    ESL_TRY(launch_emit_csc(n, F, offs, d_indptr, d_rows, d_cols, nnz, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    return ESL_OK;
}
