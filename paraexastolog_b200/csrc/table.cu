// Transition table on the device: bit-sliced rule evaluation -> per-state flip
// masks -> CSC (indptr over sources, rows = destinations) with coalesced writes.
//
// Semantics follow transition_table::generate_transitions
// (cuda/src/transition_table.cu:76-119): node i flips up at s when its DNF is true,
// bit i of s is 0 and rates[2i] != 0; it flips down when the DNF is false, bit i is 1
// and rates[2i+1] != 0.  The reference evaluates each clause over all 2^n states with
// one thrust pass per clause, compacts per node and sorts the COO list by column;
// here one thread evaluates every rule over 32 states at once (one bit per state in a
// 32-bit word), transposes the n x 32 bit matrix in registers and the edges of a
// state are emitted already sorted, so no sort is needed.
#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kMaskThreads = 128;                 // threads per block, one 32-state word each
constexpr int kStatesPerBlock = kMaskThreads * 32;  // 4096 states per block
constexpr int kEmitThreads = 256;

__constant__ uint32_t c_lowbit_pattern[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};

// Word of variable j over the 32 states 32*w + l (bit l = bit j of that state).
__device__ __forceinline__ uint32_t var_word(int j, uint32_t w) {
    return j < 5 ? c_lowbit_pattern[j] : (((w >> (j - 5)) & 1u) ? 0xFFFFFFFFu : 0u);
}

// DNF of node i over 32 states; `comp_self` evaluates it with bit i complemented
// (the rule seen from the neighbour across bit i).
__device__ __forceinline__ uint32_t eval_rule(const DevModel& m, int i, uint32_t w, bool comp_self) {
    uint32_t f = 0;
    for (int c = m.off[i]; c < m.off[i + 1]; c++) {
        uint32_t p = m.pos[c], q = m.neg[c];
        uint32_t t = 0xFFFFFFFFu;
        while (p) {
            int j = __ffs(p) - 1;
            p &= p - 1;
            uint32_t x = var_word(j, w);
            if (comp_self && j == i) x = ~x;
            t &= x;
        }
        while (q) {
            int j = __ffs(q) - 1;
            q &= q - 1;
            uint32_t x = var_word(j, w);
            if (comp_self && j == i) x = ~x;
            t &= ~x;
        }
        f |= t;
    }
    return f;
}

// In-register transpose of a 32x32 bit matrix (a[r] bit c -> a[c] bit r):
// at step j the bit-j halves of row and column index are exchanged.
__device__ __forceinline__ void transpose32(uint32_t (&a)[32]) {
#pragma unroll
    for (int j = 16, k = 0; j != 0; j >>= 1, k++) {
        const uint32_t m = (j == 16) ? 0x0000FFFFu : (j == 8) ? 0x00FF00FFu : (j == 4) ? 0x0F0F0F0Fu
                                                   : (j == 2) ? 0x33333333u : 0x55555555u;
#pragma unroll
        for (int r = 0; r < 32; r++) {
            if (r & j) continue;
            uint32_t t = ((a[r] >> j) ^ a[r + j]) & m;
            a[r] ^= t << j;
            a[r + j] ^= t;
        }
    }
}

// One thread per 32-state word: out-flip mask F and in-flip mask G per state, plus
// the number of out-edges of the block.
__global__ void __launch_bounds__(kMaskThreads) k_flip_masks(DevModel m, uint64_t n_words, uint64_t N,
                                                             uint32_t* __restrict__ F, uint32_t* __restrict__ G,
                                                             uint32_t* __restrict__ block_counts) {
    __shared__ uint32_t s_tile[kMaskThreads * 33];
    __shared__ uint32_t s_count;
    const uint32_t w = blockIdx.x * kMaskThreads + threadIdx.x;
    uint32_t fo[32], gi[32];
#pragma unroll
    for (int i = 0; i < 32; i++) {
        fo[i] = 0;
        gi[i] = 0;
    }
    if (threadIdx.x == 0) s_count = 0;
    if (w < n_words) {
#pragma unroll
        for (int i = 0; i < 32; i++) {
            if (i < m.n) {
                const uint32_t x = var_word(i, w);
                const uint32_t up = ((m.up_ok >> i) & 1u) ? 0xFFFFFFFFu : 0u;
                const uint32_t dn = ((m.down_ok >> i) & 1u) ? 0xFFFFFFFFu : 0u;
                const uint32_t f = eval_rule(m, i, w, false);
                fo[i] = (f & ~x & up) | (~f & x & dn);
                const uint32_t fc = ((m.self_dep >> i) & 1u) ? eval_rule(m, i, w, true) : f;
                // neighbour u = s ^ (1<<i) has bit i = ~x; it flips i towards s when
                // its rule (fc) equals s's bit, in the direction given by u's bit.
                gi[i] = (fc & x & up) | (~fc & ~x & dn);
            }
        }
    }
    transpose32(fo);
    transpose32(gi);
    uint32_t cnt = 0;
    const uint64_t base = (uint64_t)w * 32;
#pragma unroll
    for (int l = 0; l < 32; l++)
        if (base + l < N) cnt += __popc(fo[l]);
    __syncthreads();
    atomicAdd(&s_count, cnt);
    // coalesced stores through shared memory
    const uint64_t blk_base = (uint64_t)blockIdx.x * kStatesPerBlock;
#pragma unroll
    for (int l = 0; l < 32; l++) s_tile[threadIdx.x * 33 + l] = fo[l];
    __syncthreads();
    for (int k = 0; k < 32; k++) {
        int idx = k * kMaskThreads + threadIdx.x;
        uint64_t s = blk_base + idx;
        if (s < N) F[s] = s_tile[(idx >> 5) * 33 + (idx & 31)];
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < 32; l++) s_tile[threadIdx.x * 33 + l] = gi[l];
    __syncthreads();
    for (int k = 0; k < 32; k++) {
        int idx = k * kMaskThreads + threadIdx.x;
        uint64_t s = blk_base + idx;
        if (s < N && G) G[s] = s_tile[(idx >> 5) * 33 + (idx & 31)];
    }
    if (threadIdx.x == 0 && block_counts) block_counts[blockIdx.x] = s_count;
}

// CSC emission.  Block b covers the same 4096 states as block b of k_flip_masks and
// starts writing edges at block_offsets[b].  Per 256-state chunk: degrees, block
// scan, edges staged in shared memory in destination order, coalesced copy out.
template <int MAXN>
__global__ void __launch_bounds__(kEmitThreads) k_emit_csc(int n, uint64_t N, const uint32_t* __restrict__ F,
                                                           const uint32_t* __restrict__ block_offsets,
                                                           int32_t* __restrict__ indptr, int32_t* __restrict__ rows,
                                                           int32_t* __restrict__ cols, int64_t nnz) {
    using Scan = cub::BlockScan<uint32_t, kEmitThreads>;
    __shared__ typename Scan::TempStorage s_scan;
    // an edge is staged as (state within chunk, flipped bit): 2 bytes
    __shared__ uint8_t s_loc[kEmitThreads * MAXN];
    __shared__ uint8_t s_bit[kEmitThreads * MAXN];
    __shared__ uint32_t s_total;
    const uint64_t blk_base = (uint64_t)blockIdx.x * kStatesPerBlock;
    uint64_t out = block_offsets[blockIdx.x];
    for (int chunk = 0; chunk < kStatesPerBlock / kEmitThreads; chunk++) {
        const uint64_t s = blk_base + (uint64_t)chunk * kEmitThreads + threadIdx.x;
        if (blk_base + (uint64_t)chunk * kEmitThreads >= N) break;
        const uint32_t f = s < N ? F[s] : 0u;
        const uint32_t deg = __popc(f);
        uint32_t excl, total;
        Scan(s_scan).ExclusiveSum(deg, excl, total);
        if (s < N) indptr[s] = (int32_t)(out + excl);
        // destinations ascending: clear bits high -> low, then set bits low -> high
        const uint32_t sv = (uint32_t)s;
        uint32_t down = f & sv, up = f & ~sv;
        int k = (int)excl;
        while (down) {
            int i = 31 - __clz(down);
            down &= ~(1u << i);
            s_loc[k] = (uint8_t)threadIdx.x;
            s_bit[k] = (uint8_t)i;
            k++;
        }
        while (up) {
            int i = __ffs(up) - 1;
            up &= up - 1;
            s_loc[k] = (uint8_t)threadIdx.x;
            s_bit[k] = (uint8_t)i;
            k++;
        }
        if (threadIdx.x == 0) s_total = total;
        __syncthreads();
        const uint32_t tot = s_total;
        const uint32_t chunk_base = (uint32_t)(blk_base + (uint64_t)chunk * kEmitThreads);
        for (uint32_t e = threadIdx.x; e < tot; e += kEmitThreads) {
            const uint32_t src = chunk_base + s_loc[e];
            rows[out + e] = (int32_t)(src ^ (1u << s_bit[e]));
            if (cols) cols[out + e] = (int32_t)src;
        }
        out += tot;
        __syncthreads();
    }
    if (blk_base + kStatesPerBlock >= N && blk_base < N) {
        // the block holding the last state closes indptr
        if (threadIdx.x == 0) indptr[N] = (int32_t)nnz;
    }
}

// Masks from an arbitrary CSC table whose every edge flips one bit.
__global__ void k_masks_from_csc(int n, uint64_t N, const int32_t* __restrict__ indptr,
                                 const int32_t* __restrict__ rows, uint32_t* __restrict__ F,
                                 unsigned long long* __restrict__ bad) {
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    uint32_t f = 0;
    for (int32_t e = indptr[s]; e < indptr[s + 1]; e++) {
        uint32_t x = (uint32_t)rows[e] ^ (uint32_t)s;
        if (x == 0 || (x & (x - 1)) != 0 || x >= (1u << n)) {
            atomicAdd(bad, 1ull);
            continue;
        }
        f |= x;
    }
    F[s] = f;
}

__global__ void k_in_masks(int n, uint64_t N, const uint32_t* __restrict__ F, uint32_t* __restrict__ G) {
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    uint32_t g = 0;
    for (int i = 0; i < n; i++)
        if ((F[s ^ (1ull << i)] >> i) & 1u) g |= 1u << i;
    G[s] = g;
}

}  // namespace

int64_t flip_mask_blocks(int n) {
    uint64_t N = 1ull << n;
    uint64_t words = (N + 31) / 32;
    return (int64_t)((words + kMaskThreads - 1) / kMaskThreads);
}

int upload_model(const Model& m, DevBuf<int32_t>& off, DevBuf<uint32_t>& pos, DevBuf<uint32_t>& neg,
                 const double* rates, DevModel& dm, cudaStream_t s) {
    int n = m.n();
    std::vector<int32_t> h_off(n + 1, 0);
    std::vector<uint32_t> h_pos, h_neg;
    uint32_t self_dep = 0;
    for (int i = 0; i < n; i++) {
        for (const Clause& c : m.rules[i]) {
            h_pos.push_back(c.pos);
            h_neg.push_back(c.neg);
            if (((c.pos | c.neg) >> i) & 1u) self_dep |= 1u << i;
        }
        h_off[i + 1] = (int32_t)h_pos.size();
    }
    ESL_TRY(off.alloc(h_off.size()));
    ESL_TRY(pos.alloc(h_pos.size()));
    ESL_TRY(neg.alloc(h_neg.size()));
    ESL_CUDA(cudaMemcpyAsync(off.get(), h_off.data(), h_off.size() * 4, cudaMemcpyHostToDevice, s));
    if (!h_pos.empty()) {
        ESL_CUDA(cudaMemcpyAsync(pos.get(), h_pos.data(), h_pos.size() * 4, cudaMemcpyHostToDevice, s));
        ESL_CUDA(cudaMemcpyAsync(neg.get(), h_neg.data(), h_neg.size() * 4, cudaMemcpyHostToDevice, s));
    }
    dm.n = n;
    dm.off = off.get();
    dm.pos = pos.get();
    dm.neg = neg.get();
    dm.up_ok = dm.down_ok = 0;
    for (int i = 0; i < n; i++) {
        if (rates[2 * i] != 0.0) dm.up_ok |= 1u << i;
        if (rates[2 * i + 1] != 0.0) dm.down_ok |= 1u << i;
    }
    dm.self_dep = self_dep;
    return ESL_OK;
}

int launch_flip_masks(const DevModel& dm, uint32_t* F, uint32_t* G, uint32_t* block_counts, cudaStream_t s) {
    uint64_t N = 1ull << dm.n;
    uint64_t words = (N + 31) / 32;
    int64_t blocks = flip_mask_blocks(dm.n);
    ESL_COUNT_LAUNCH();
    k_flip_masks<<<(unsigned)blocks, kMaskThreads, 0, s>>>(dm, words, N, F, G, block_counts);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int launch_emit_csc(int n, const uint32_t* F, const uint32_t* block_offsets_excl, int32_t* indptr, int32_t* rows,
                    int32_t* cols, int64_t nnz, cudaStream_t s) {
    uint64_t N = 1ull << n;
    int64_t blocks = flip_mask_blocks(n);
    if (n <= 16) {
        ESL_COUNT_LAUNCH();
        k_emit_csc<16><<<(unsigned)blocks, kEmitThreads, 0, s>>>(n, N, F, block_offsets_excl, indptr, rows, cols, nnz);
    } else if (n <= 24) {
        ESL_COUNT_LAUNCH();
        k_emit_csc<24><<<(unsigned)blocks, kEmitThreads, 0, s>>>(n, N, F, block_offsets_excl, indptr, rows, cols, nnz);
    } else {
        ESL_COUNT_LAUNCH();
        k_emit_csc<30><<<(unsigned)blocks, kEmitThreads, 0, s>>>(n, N, F, block_offsets_excl, indptr, rows, cols, nnz);
    }
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int masks_from_csc(int n, const int32_t* indptr, const int32_t* rows, uint32_t* F, uint32_t* G,
                   unsigned long long* d_bad, cudaStream_t s) {
    uint64_t N = 1ull << n;
    unsigned blocks = (unsigned)((N + 255) / 256);
    ESL_COUNT_LAUNCH();
    k_masks_from_csc<<<blocks, 256, 0, s>>>(n, N, indptr, rows, F, d_bad);
    ESL_CUDA(cudaGetLastError());
    ESL_COUNT_LAUNCH();
    k_in_masks<<<blocks, 256, 0, s>>>(n, N, F, G);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

}  // namespace esl
