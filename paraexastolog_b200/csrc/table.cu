// Transition table on the device: bit-sliced rule evaluation -> per-state flip
// masks -> CSC (indptr over sources, rows = destinations) with coalesced writes.
//
// Semantics follow transition_table::generate_transitions
// (cuda/src/transition_table.cu:76-119): node i flips up at s when its DNF is true,
// bit i of s is 0 and rates[2i] != 0; it flips down when the DNF is false, bit i is 1
// and rates[2i+1] != 0.  The reference evaluates each clause over all 2^n states with
// one thrust pass per clause, compacts per node and sorts the COO list by column.
// Here one warp takes 32 states at a time (one bit per state in a 32-bit word): lane i
// evaluates node i's rule over the 32 states, mostly by one look-up in a small table
// of the rule over the state bits above 5 that it reads, a warp-wide 32 x 32 bit
// transpose turns the node words into per-state flip masks, and the edges of a state
// are emitted already sorted, so no sort is needed.
#include <cub/device/device_scan.cuh>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kMaskWarps = 8;                                           // warps per block
constexpr int kWordsPerWarp = kTableBlockStates / 32 / kMaskWarps;      // 32-state words per warp
constexpr int kEmitWarps = 8;
constexpr int kEmitGroups = kTableBlockStates / 32 / kEmitWarps;        // 32-state groups per warp

__constant__ uint32_t c_lowbit_pattern[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};

// Word of variable j over the 32 states 32*w + l (bit l = bit j of that state).
__device__ __forceinline__ uint32_t var_word(int j, uint64_t w) {
    return j < 5 ? c_lowbit_pattern[j] : (((w >> (j - 5)) & 1u) ? 0xFFFFFFFFu : 0u);
}

// DNF of node i over 32 states; `comp_self` evaluates it with bit i complemented
// (the rule seen from the neighbour across bit i).
__device__ __forceinline__ uint32_t eval_rule(const DevModel& m, int i, uint64_t w, bool comp_self) {
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

// 32x32 bit transpose across a warp: lane r holds row r (bit c = column c) and gets
// column r back (bit c = row c).  At step j the off-diagonal j x j blocks of every
// 2j x 2j block are exchanged between lanes r and r ^ j.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t a, int lane) {
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const uint32_t m = (j == 16) ? 0x0000FFFFu : (j == 8) ? 0x00FF00FFu : (j == 4) ? 0x0F0F0F0Fu
                                                     : (j == 2) ? 0x33333333u : 0x55555555u;
        const uint32_t b = __shfl_xor_sync(0xFFFFFFFFu, a, j);
        if (lane & j)
            a ^= ((b >> j) ^ a) & m;
        else
            a ^= (((a >> j) ^ b) & m) << j;
    }
    return a;
}

// One warp per 32-state word, lane i = node i: the lane evaluates node i's rule over
// the word's 32 states (from its rule table, else from the clauses), forms the words of
// the up / down flips out of and into the 32 states, and a warp transpose turns the
// n node words into the 32 per-state masks, stored coalesced.  A block covers
// kTableBlockStates states and writes their out-edge count.
__global__ void __launch_bounds__(kMaskWarps * 32) k_flip_masks(DevModel m, uint64_t n_words, uint64_t N,
                                                                uint32_t* __restrict__ F, uint32_t* __restrict__ G,
                                                                uint32_t* __restrict__ block_counts) {
    extern __shared__ uint32_t s_tab[];
    __shared__ uint4 s_info[32];
    __shared__ uint32_t s_cnt[kMaskWarps];
    for (uint32_t j = threadIdx.x; j < m.tab_words; j += blockDim.x) s_tab[j] = m.tab[j];
    if (threadIdx.x < (unsigned)m.n) s_info[threadIdx.x] = m.info[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = lane;
    const bool node = i < m.n;
    const uint4 inf = node ? s_info[i] : make_uint4(0u, kNoRuleTable, 0u, 0u);
    const uint32_t up = (node && ((m.up_ok >> i) & 1u)) ? 0xFFFFFFFFu : 0u;
    const uint32_t dn = (node && ((m.down_ok >> i) & 1u)) ? 0xFFFFFFFFu : 0u;
    const bool self = node && ((m.self_dep >> i) & 1u);
    const uint32_t xlo = (node && i < 5) ? c_lowbit_pattern[i] : 0u;
    // The warp's words w0 .. w0 + 3 differ only in their two low bits: the table index
    // is idx0 (from w0) plus the table bits at word bits 0 and 1 (lo0, lo1) as set in j.
    const uint64_t w0 = (uint64_t)blockIdx.x * (kTableBlockStates / 32) + (uint64_t)warp * kWordsPerWarp;
    static_assert(kWordsPerWarp == 4, "the index split assumes 4 words per warp");
    uint32_t idx0 = 0, lo0 = 0, lo1 = 0;
    if (node && inf.y != kNoRuleTable) {
        for (uint32_t b = 0; b < inf.y; b++) {
            const uint32_t p = ((b < 4 ? inf.z : inf.w) >> (8 * (b & 3))) & 0xFFu;
            idx0 |= (uint32_t)((w0 >> p) & 1u) << b;
            if (p == 0) lo0 = 1u << b;
            if (p == 1) lo1 = 1u << b;
        }
    }
    uint32_t cnt = 0;
    for (int j = 0; j < kWordsPerWarp; j++) {
        const uint64_t w = w0 + j;
        if (w >= n_words) break;  // uniform over the warp
        uint32_t fo = 0, gi = 0;
        if (node) {
            const uint32_t x = i < 5 ? xlo : (((w >> (i - 5)) & 1u) ? 0xFFFFFFFFu : 0u);
            uint32_t f, fc;
            if (inf.y != kNoRuleTable) {
                const uint32_t idx = idx0 | ((j & 1) ? lo0 : 0u) | ((j & 2) ? lo1 : 0u);
                f = s_tab[inf.x + idx];
                fc = self ? s_tab[inf.x + (1u << inf.y) + idx] : f;
            } else {
                f = eval_rule(m, i, w, false);
                fc = (self && G) ? eval_rule(m, i, w, true) : f;
            }
            fo = (f & ~x & up) | (~f & x & dn);
            // neighbour u = s ^ (1<<i) has bit i = ~x; it flips i towards s when its
            // rule (fc) equals s's bit, in the direction given by u's bit.
            gi = (fc & x & up) | (~fc & ~x & dn);
        }
        fo = warp_transpose32(fo, lane);
        const uint64_t s = w * 32 + lane;
        if (G) {
            gi = warp_transpose32(gi, lane);
            if (s < N) G[s] = gi;
        }
        if (s < N) {
            F[s] = fo;
            cnt += __popc(fo);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    if (lane == 0) s_cnt[warp] = cnt;
    __syncthreads();
    if (threadIdx.x == 0 && block_counts) {
        uint32_t tot = 0;
        for (int k = 0; k < kMaskWarps; k++) tot += s_cnt[k];
        block_counts[blockIdx.x] = tot;
    }
}

// CSC emission.  Block b covers the same kTableBlockStates states as block b of
// k_flip_masks and starts writing edges at block_offsets[b]; each warp takes
// kEmitGroups groups of 32 states, starts at the block offset plus the edges of the
// warps before it, and per group: warp scan of the degrees, edges staged in the warp's
// shared memory in destination order, coalesced copy out.  No block-wide barrier in the
// loop.
// TOff / TPtr: 32-bit block offsets and column pointers, or 64-bit ones for tables of
// more than 2^31 - 1 edges (destinations and sources stay 32-bit: n <= 30).
template <int MAXN, class TOff, class TPtr>
__global__ void __launch_bounds__(kEmitWarps * 32) k_emit_csc(int n, uint64_t N, const uint32_t* __restrict__ F,
                                                             const TOff* __restrict__ block_offsets,
                                                             TPtr* __restrict__ indptr, int32_t* __restrict__ rows,
                                                             int32_t* __restrict__ cols, int64_t nnz) {
    // an edge is staged as (state within the group << 5 | flipped bit)
    __shared__ uint16_t s_stage[kEmitWarps][32 * MAXN];
    __shared__ uint32_t s_wsum[kEmitWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t blk_base = (uint64_t)blockIdx.x * kTableBlockStates;
    const uint64_t wbase = blk_base + (uint64_t)warp * 32 * kEmitGroups;
    uint32_t f[kEmitGroups];
    uint32_t tot = 0;
#pragma unroll
    for (int g = 0; g < kEmitGroups; g++) {
        const uint64_t s = wbase + (uint64_t)g * 32 + lane;
        f[g] = s < N ? F[s] : 0u;
        tot += __popc(f[g]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
    if (lane == 0) s_wsum[warp] = tot;
    __syncthreads();
    uint64_t out = block_offsets[blockIdx.x];
    for (int k = 0; k < warp; k++) out += s_wsum[k];
    uint16_t* st = s_stage[warp];
#pragma unroll
    for (int g = 0; g < kEmitGroups; g++) {
        const uint64_t gb = wbase + (uint64_t)g * 32;
        if (gb >= N) break;  // uniform over the warp
        const uint32_t d = __popc(f[g]);
        uint32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t excl = incl - d;
        const uint32_t gtot = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint64_t s = gb + lane;
        if (s < N) indptr[s] = (TPtr)(out + excl);
        // destinations ascending: clear bits high -> low, then set bits low -> high
        const uint32_t sv = (uint32_t)s;
        uint32_t down = f[g] & sv, upm = f[g] & ~sv;
        uint32_t k = excl;
        while (down) {
            const int i = 31 - __clz(down);
            down &= ~(1u << i);
            st[k++] = (uint16_t)((lane << 5) | i);
        }
        while (upm) {
            const int i = __ffs(upm) - 1;
            upm &= upm - 1;
            st[k++] = (uint16_t)((lane << 5) | i);
        }
        __syncwarp();
        for (uint32_t e = lane; e < gtot; e += 32) {
            const uint32_t v = st[e];
            const uint32_t src = (uint32_t)gb + (v >> 5);
            rows[out + e] = (int32_t)(src ^ (1u << (v & 31u)));
            if (cols) cols[out + e] = (int32_t)src;
        }
        out += gtot;
        __syncwarp();
    }
    if (threadIdx.x == 0 && blk_base < N && blk_base + kTableBlockStates >= N) indptr[N] = (TPtr)nnz;
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
    const uint64_t N = 1ull << n;
    return (int64_t)((N + kTableBlockStates - 1) / kTableBlockStates);
}

namespace {
const uint32_t kLowPattern[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};

// node i's DNF over the 32 states of word w (host form of eval_rule)
uint32_t host_eval(const Model& m, int i, uint64_t w, bool comp_self) {
    uint32_t f = 0;
    for (const Clause& c : m.rules[i]) {
        uint32_t t = 0xFFFFFFFFu;
        for (int j = 0; j < 32; j++) {
            const uint32_t b = 1u << j;
            if (!((c.pos | c.neg) & b)) continue;
            uint32_t x = j < 5 ? kLowPattern[j] : (((w >> (j - 5)) & 1u) ? 0xFFFFFFFFu : 0u);
            if (comp_self && j == i) x = ~x;
            t &= (c.pos & b) ? x : ~x;
        }
        f |= t;
    }
    return f;
}
}  // namespace

void host_model(const Model& m, HostModel& hm) {
    const int n = m.n();
    hm.off.assign(n + 1, 0);
    hm.pos.clear();
    hm.neg.clear();
    hm.info.assign(n, make_uint4(0u, kNoRuleTable, 0u, 0u));
    hm.tab.clear();
    hm.self_dep = 0;
    for (int i = 0; i < n; i++) {
        uint32_t support = 0;
        for (const Clause& c : m.rules[i]) {
            hm.pos.push_back(c.pos);
            hm.neg.push_back(c.neg);
            support |= c.pos | c.neg;
        }
        hm.off[i + 1] = (int32_t)hm.pos.size();
        if ((support >> i) & 1u) hm.self_dep |= 1u << i;
        // the word bits (state bits >= 5) the rule reads
        std::vector<uint32_t> hb;
        for (int j = 5; j < 32; j++)
            if ((support >> j) & 1u) hb.push_back((uint32_t)(j - 5));
        const size_t words = (size_t)2 << hb.size();
        if ((int)hb.size() > kRuleTableMaxBits || hm.tab.size() + words > (size_t)kRuleTableMaxWords) continue;
        uint4 inf = make_uint4((uint32_t)hm.tab.size(), (uint32_t)hb.size(), 0u, 0u);
        for (size_t b = 0; b < hb.size(); b++) (b < 4 ? inf.z : inf.w) |= hb[b] << (8 * (b & 3));
        const uint32_t cnt = 1u << hb.size();
        for (int comp = 0; comp < 2; comp++)
            for (uint32_t a = 0; a < cnt; a++) {
                uint64_t w = 0;
                for (size_t b = 0; b < hb.size(); b++)
                    if ((a >> b) & 1u) w |= 1ull << hb[b];
                hm.tab.push_back(host_eval(m, i, w, comp != 0));
            }
        hm.info[i] = inf;
    }
}

void rate_masks(int n, const double* rates, uint32_t& up_ok, uint32_t& down_ok) {
    up_ok = down_ok = 0;
    for (int i = 0; i < n; i++) {
        if (rates[2 * i] != 0.0) up_ok |= 1u << i;
        if (rates[2 * i + 1] != 0.0) down_ok |= 1u << i;
    }
}

int upload_model(const Model& m, DevModelBufs& b, const double* rates, DevModel& dm, cudaStream_t s) {
    const int n = m.n();
    HostModel hm;
    host_model(m, hm);
    ESL_TRY(b.off.alloc(hm.off.size()));
    ESL_TRY(b.pos.alloc(hm.pos.size()));
    ESL_TRY(b.neg.alloc(hm.neg.size()));
    ESL_TRY(b.info.alloc(std::max<size_t>(hm.info.size(), 1)));
    ESL_TRY(b.tab.alloc(hm.tab.size()));
    ESL_CUDA(cudaMemcpyAsync(b.off.get(), hm.off.data(), hm.off.size() * 4, cudaMemcpyHostToDevice, s));
    if (!hm.pos.empty()) {
        ESL_CUDA(cudaMemcpyAsync(b.pos.get(), hm.pos.data(), hm.pos.size() * 4, cudaMemcpyHostToDevice, s));
        ESL_CUDA(cudaMemcpyAsync(b.neg.get(), hm.neg.data(), hm.neg.size() * 4, cudaMemcpyHostToDevice, s));
    }
    if (!hm.info.empty())
        ESL_CUDA(cudaMemcpyAsync(b.info.get(), hm.info.data(), hm.info.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    if (!hm.tab.empty())
        ESL_CUDA(cudaMemcpyAsync(b.tab.get(), hm.tab.data(), hm.tab.size() * 4, cudaMemcpyHostToDevice, s));
    dm.n = n;
    dm.off = b.off.get();
    dm.pos = b.pos.get();
    dm.neg = b.neg.get();
    dm.info = b.info.get();
    dm.tab = b.tab.get();
    dm.tab_words = (uint32_t)hm.tab.size();
    rate_masks(n, rates, dm.up_ok, dm.down_ok);
    dm.self_dep = hm.self_dep;
    return ESL_OK;
}

int launch_flip_masks(const DevModel& dm, uint32_t* F, uint32_t* G, uint32_t* block_counts, cudaStream_t s) {
    const uint64_t N = 1ull << dm.n;
    const uint64_t words = (N + 31) / 32;
    const int64_t blocks = flip_mask_blocks(dm.n);
    ESL_COUNT_LAUNCH();
    k_flip_masks<<<(unsigned)blocks, kMaskWarps * 32, (size_t)dm.tab_words * 4, s>>>(dm, words, N, F, G, block_counts);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

template <class TOff, class TPtr>
int launch_emit(int n, const uint32_t* F, const TOff* block_offsets_excl, TPtr* indptr, int32_t* rows, int32_t* cols,
                int64_t nnz, cudaStream_t s) {
    const uint64_t N = 1ull << n;
    const int64_t blocks = flip_mask_blocks(n);
    ESL_COUNT_LAUNCH();
    if (n <= 16)
        k_emit_csc<16, TOff, TPtr><<<(unsigned)blocks, kEmitWarps * 32, 0, s>>>(n, N, F, block_offsets_excl, indptr,
                                                                               rows, cols, nnz);
    else if (n <= 24)
        k_emit_csc<24, TOff, TPtr><<<(unsigned)blocks, kEmitWarps * 32, 0, s>>>(n, N, F, block_offsets_excl, indptr,
                                                                               rows, cols, nnz);
    else
        k_emit_csc<30, TOff, TPtr><<<(unsigned)blocks, kEmitWarps * 32, 0, s>>>(n, N, F, block_offsets_excl, indptr,
                                                                               rows, cols, nnz);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int launch_emit_csc(int n, const uint32_t* F, const uint32_t* block_offsets_excl, int32_t* indptr, int32_t* rows,
                    int32_t* cols, int64_t nnz, cudaStream_t s) {
    return launch_emit<uint32_t, int32_t>(n, F, block_offsets_excl, indptr, rows, cols, nnz, s);
}

int launch_emit_csc64(int n, const uint32_t* F, const uint64_t* block_offsets_excl, int64_t* indptr, int32_t* rows,
                      int32_t* cols, int64_t nnz, cudaStream_t s) {
    return launch_emit<uint64_t, int64_t>(n, F, block_offsets_excl, indptr, rows, cols, nnz, s);
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
