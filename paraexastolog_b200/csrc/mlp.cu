// Learned warm start of the transient solve: a small MLP over per-state features.
//
// No counterpart in the reference (asmelko/paraExaStoLog has no learned component).  The
// network predicts, for a rate set k and a transient state v, the expected time z_k(v)
// the chain spends in v before absorption (the occupation the level sweep solves for).
// Its prediction is the starting iterate of the sweep's grid-wide Krylov groups
// (esl_solve_opts.d_warm); the plain solve stays the arbiter of the result.
//
//   x(v, k) (77)  ->  h1 = relu(W1 x + b1) (128)  ->  h2 = relu(W2 h1 + b2) (128)
//                 ->  y = w3 . h2 + b3,   z = exp(mu + sigma * y)
//
// Features x(v, k): [0, 20) node bits of v as +-1 (0 past n); [20] log of v's outgoing
// rate sum under k; [21, 37) +-1 for "v reaches terminal SCC t", t < 16 (0 past T);
// [37, 77) log of the 2n rates of k (0 past 2n, 0 for a zero rate).
// Weights: an FP32 master copy trained with Adam; the forward and backward passes use
// BF16-rounded weights with FP32 activations and accumulation.  Training runs on SIMT
// tiled GEMMs; inference runs layer 2 on the tensor cores (tcgen05.mma with TMEM
// accumulators, BF16 in, FP32 accumulate; mma.sync m16n8k16 with ESL_MLP_TC=0 or a rate-set
// count that is not a multiple of 8) with layer 1 split into a per-state part, a
// per-rate-set part and the log-rate-sum column, so that the 77-wide product is never
// formed per sample.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kBits = 20, kReach = 16;
constexpr int kIn = 77, kXld = 80, kH = 128;
constexpr int kFq = 20, kFreach = 21, kFrates = 37;
// parameter layout (floats)
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH,
              kParams = oB3 + 1;
static_assert(kParams == ESL_MLP_PARAMS, "parameter count");

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ float log_rate_sum(uint32_t v, uint32_t f, const double* __restrict__ r) {
    double q = 0.0;
    while (f) {
        const int i = __ffs(f) - 1;
        f &= f - 1;
        q += r[2 * i + ((v >> i) & 1u)];
    }
    return q > 0.0 ? (float)log(q) : 0.0f;
}

// ---- features ------------------------------------------------------------------------
// full feature rows of samples (k_s, v_s)
__global__ void k_mlp_features(int S, int n, int T, const int32_t* __restrict__ ks, const int32_t* __restrict__ vs,
                               const double* __restrict__ rates, const uint32_t* __restrict__ F,
                               const uint32_t* __restrict__ reach, float* __restrict__ X) {
    const int s = blockIdx.x;
    if (s >= S) return;
    const int k = ks[s];
    const uint32_t v = (uint32_t)vs[s];
    const double* r = rates + (size_t)k * 2 * n;
    float* x = X + (size_t)s * kXld;
    for (int j = threadIdx.x; j < kXld; j += blockDim.x) {
        float f = 0.0f;
        if (j < kBits) {
            if (j < n) f = ((v >> j) & 1u) ? 1.0f : -1.0f;
        } else if (j == kFq) {
            f = log_rate_sum(v, F[v], r);
        } else if (j < kFrates) {
            const int t = j - kFreach;
            if (t < T) f = ((reach[v] >> t) & 1u) ? 1.0f : -1.0f;
        } else if (j < kIn) {
            const int q = j - kFrates;
            if (q < 2 * n && r[q] > 0.0) f = (float)log(r[q]);
        }
        x[j] = f;
    }
}

// state part of the features (bits, reachability) of every target state
__global__ void k_mlp_state_features(int nt, int n, int T, const uint32_t* __restrict__ targets,
                                     const uint32_t* __restrict__ reach, float* __restrict__ X) {
    const int i = blockIdx.x;
    if (i >= nt) return;
    const uint32_t v = targets[i];
    float* x = X + (size_t)i * kXld;
    for (int j = threadIdx.x; j < kXld; j += blockDim.x) {
        float f = 0.0f;
        if (j < kBits) {
            if (j < n) f = ((v >> j) & 1u) ? 1.0f : -1.0f;
        } else if (j >= kFreach && j < kFrates) {
            const int t = j - kFreach;
            if (t < T) f = ((reach[v] >> t) & 1u) ? 1.0f : -1.0f;
        }
        x[j] = f;
    }
}

// rate part of the features of every rate set
__global__ void k_mlp_rate_features(int B, int n, const double* __restrict__ rates, float* __restrict__ X) {
    const int k = blockIdx.x;
    if (k >= B) return;
    for (int j = threadIdx.x; j < kXld; j += blockDim.x) {
        float f = 0.0f;
        const int q = j - kFrates;
        if (j >= kFrates && j < kIn && q < 2 * n) {
            const double r = rates[(size_t)k * 2 * n + q];
            if (r > 0.0) f = (float)log(r);
        }
        X[(size_t)k * kXld + j] = f;
    }
}

// ---- SIMT tiled GEMM:  C[m][n] (op)= sum_k A(m, k) B(k, n) --------------------------------
// A(m, k) = A[m * sam + k * sak], B(k, n) = B[k * sbk + n * sbn]; 64 x 64 tiles, 256 threads
// of 4 x 4 outputs, K in chunks of 16; blockIdx.z splits K (G_ATOMIC only).
enum { G_STORE, G_BIAS, G_BIAS_RELU, G_MASK, G_ATOMIC };

template <int EPI>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float* __restrict__ A, long sam, long sak,
                                              const float* __restrict__ Bm, long sbk, long sbn, float* __restrict__ C,
                                              long ldc, const float* __restrict__ bias, const float* __restrict__ mask,
                                              int kper) {
    __shared__ float As[16][68], Bs[16][68];
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int kb = blockIdx.z * kper, ke = min(K, kb + kper);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    for (int k0 = kb; k0 < ke; k0 += 16) {
        for (int i = threadIdx.x; i < 1024; i += 256) {
            int mm, kk;
            if (sam == 1) {
                mm = i & 63;
                kk = i >> 6;
            } else {
                mm = i >> 4;
                kk = i & 15;
            }
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < ke) ? A[(long)m * sam + (long)k * sak] : 0.0f;
            int nn, kq;
            if (sbn == 1) {
                nn = i & 63;
                kq = i >> 6;
            } else {
                nn = i >> 4;
                kq = i & 15;
            }
            const int n = n0 + nn, kk2 = k0 + kq;
            Bs[kq][nn] = (n < N && kk2 < ke) ? Bm[(long)kk2 * sbk + (long)n * sbn] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float* c = C + (long)m * ldc + n;
            const float v = acc[i][j];
            if (EPI == G_STORE) *c = v;
            if (EPI == G_BIAS) *c = v + bias[n];
            if (EPI == G_BIAS_RELU) *c = fmaxf(v + bias[n], 0.0f);
            if (EPI == G_MASK) *c = mask[(long)m * ldc + n] > 0.0f ? v : 0.0f;
            if (EPI == G_ATOMIC) atomicAdd(c, v);
        }
    }
}

// ---- training pieces ------------------------------------------------------------------------
// random (rate set, target state) pairs with their standardized log-occupation labels
__global__ void k_mlp_sample(int S, uint64_t seed, uint64_t step, int B, int nt, const uint32_t* __restrict__ targets,
                             size_t N, const double* __restrict__ occ, float mu, float sigma, int32_t* __restrict__ ks,
                             int32_t* __restrict__ vs, float* __restrict__ ts, float* __restrict__ ws) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const uint64_t h = mix64(seed ^ mix64(step * 0x100000001ull + (uint64_t)s));
    const int k = (int)((h >> 32) % (uint64_t)B);
    const uint32_t v = targets[(uint32_t)(h & 0xffffffffu) % (uint32_t)nt];
    const double z = occ[(size_t)k * N + v];
    const bool ok = z > 0.0 && isfinite(z);
    ks[s] = k;
    vs[s] = (int32_t)v;
    ts[s] = ok ? (float)((log(z) - mu) / sigma) : 0.0f;
    ws[s] = ok ? 1.0f : 0.0f;
}

// per-state log occupations of a sample of pairs (for mu, sigma): sums of t, t^2, count
__global__ void k_mlp_label_stats(int S, uint64_t seed, int B, int nt, const uint32_t* __restrict__ targets, size_t N,
                                  const double* __restrict__ occ, double* __restrict__ acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0.0, b = 0.0, c = 0.0;
    if (s < S) {
        const uint64_t h = mix64(seed ^ mix64(0xFFFFFFFF00000000ull + (uint64_t)s));
        const int k = (int)((h >> 32) % (uint64_t)B);
        const uint32_t v = targets[(uint32_t)(h & 0xffffffffu) % (uint32_t)nt];
        const double z = occ[(size_t)k * N + v];
        if (z > 0.0 && isfinite(z)) {
            const double t = log(z);
            a = t;
            b = t * t;
            c = 1.0;
        }
    }
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc, a);
        atomicAdd(acc + 1, b);
        atomicAdd(acc + 2, c);
    }
}

// output layer, one warp per sample: y = H2 . w3 + b3, loss += w (y - t)^2 / S,
// dy = 2 w (y - t) / S, dZ2 = dy w3 [H2 > 0]
__global__ void k_mlp_head(int S, const float* __restrict__ H2, const float* __restrict__ Wq,
                           const float* __restrict__ ts, const float* __restrict__ ws, float* __restrict__ y,
                           float* __restrict__ dy, float* __restrict__ dZ2, float* __restrict__ loss) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= S) return;
    const float* h = H2 + (size_t)s * kH;
    const float* w3 = Wq + oW3;
    float a = 0.0f;
    for (int j = lane; j < kH; j += 32) a += h[j] * w3[j];
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    const float yy = a + Wq[oB3];
    const float r = yy - ts[s];
    const float g = 2.0f * ws[s] * r / (float)S;
    if (lane == 0) {
        if (y) y[s] = yy;
        if (dy) dy[s] = g;
        if (loss) atomicAdd(loss, ws[s] * r * r / (float)S);
    }
    if (dZ2)
        for (int j = lane; j < kH; j += 32) dZ2[(size_t)s * kH + j] = h[j] > 0.0f ? g * w3[j] : 0.0f;
}

// column sums of an S x W matrix, added into out[W]
__global__ void k_colsum(int S, int W, const float* __restrict__ X, float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= W) return;
    const int per = (S + gridDim.y - 1) / gridDim.y;
    const int s0 = blockIdx.y * per, s1 = min(S, s0 + per);
    float a = 0.0f;
    for (int s = s0; s < s1; s++) a += X[(size_t)s * W + j];
    atomicAdd(out + j, a);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// weights rounded to BF16 for the passes (biases kept), and layer 2's BF16 bits for inference
__global__ void k_mlp_quant(const float* __restrict__ P, float* __restrict__ Wq, __nv_bfloat16* __restrict__ W2h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const bool weight = (i < oB1) || (i >= oW2 && i < oB2) || (i >= oW3 && i < oB3);
    Wq[i] = weight ? bf16_round(P[i]) : P[i];
    if (i >= oW2 && i < oB2) W2h[i - oW2] = __float2bfloat16_rn(P[i]);
}

__global__ void k_mlp_adam(int cnt, float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M1,
                           float* __restrict__ M2, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const float g = G[i];
    const float m = b1 * M1[i] + (1.0f - b1) * g;
    const float v = b2 * M2[i] + (1.0f - b2) * g * g;
    M1[i] = m;
    M2[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void k_mlp_init(uint64_t seed, float* __restrict__ P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    // uniform in +-sqrt(6 / fan_in) (He-uniform) for weights, zero biases
    float bound = 0.0f;
    if (i < oB1) bound = sqrtf(6.0f / kIn);
    else if (i >= oW2 && i < oB2) bound = sqrtf(6.0f / kH);
    else if (i >= oW3 && i < oB3) bound = sqrtf(3.0f / kH);
    const uint64_t h = mix64(seed ^ mix64((uint64_t)i));
    const float u = (float)((h >> 40) * (1.0 / 16777216.0));  // [0, 1)
    P[i] = bound * (2.0f * u - 1.0f);
}

// ---- inference on tensor cores ---------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&p);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kW2ld = 68;  // 32-bit words per layer-2 row in shared memory (64 + 4: no bank conflicts)

// Samples s = i * B + k (target state i, rate set k); each warp takes 16 samples at a time.
// h1 = relu(A1[i] + C1[k] + log q(v, k) * W1[:, 20]) is built straight into the A fragments;
// layer 2 is 8 x 16 mma per 16 samples; the head is reduced across each quad of lanes.
__global__ void __launch_bounds__(128) k_mlp_predict(int nt, int B, int n, size_t N, const uint32_t* __restrict__ targets,
                                                     const uint32_t* __restrict__ F, const double* __restrict__ rates,
                                                     const float* __restrict__ A1, const float* __restrict__ C1,
                                                     const __nv_bfloat16* __restrict__ W2h,
                                                     const float* __restrict__ Wq, float mu, float sigma,
                                                     double* __restrict__ warm) {
    __shared__ uint32_t sW2[kH * kW2ld];
    __shared__ float sb2[kH], sw3[kH], swq[kH];
    const uint32_t* w2 = reinterpret_cast<const uint32_t*>(W2h);
    for (int i = threadIdx.x; i < kH * (kH / 2); i += blockDim.x) sW2[(i >> 6) * kW2ld + (i & 63)] = w2[i];
    for (int j = threadIdx.x; j < kH; j += blockDim.x) {
        sb2[j] = Wq[oB2 + j];
        sw3[j] = Wq[oW3 + j];
        swq[j] = Wq[oW1 + j * kIn + kFq];
    }
    __syncthreads();
    const float b3 = Wq[oB3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tq = lane & 3;
    const long total = (long)nt * B;
    const long tiles = (total + 15) / 16;
    for (long tile = (long)blockIdx.x * 4 + warp; tile < tiles; tile += (long)gridDim.x * 4) {
        const long s0 = tile * 16;
        bool valid[2];
        uint32_t vv[2];
        int kk[2];
        float lq[2];
        const float* a1[2];
        const float* c1[2];
#pragma unroll
        for (int rr = 0; rr < 2; rr++) {
            long s = s0 + g + 8 * rr;
            valid[rr] = s < total;
            if (!valid[rr]) s = total - 1;
            const int i = (int)(s / B);
            kk[rr] = (int)(s - (long)i * B);
            vv[rr] = targets[i];
            lq[rr] = log_rate_sum(vv[rr], F[vv[rr]], rates + (size_t)kk[rr] * 2 * n);
            a1[rr] = A1 + (size_t)i * kH;
            c1[rr] = C1 + (size_t)kk[rr] * kH;
        }
        uint32_t af[8][4];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int j0 = c * 16 + tq * 2;
            float h[2][4];
#pragma unroll
            for (int rr = 0; rr < 2; rr++) {
                const float2 p = *reinterpret_cast<const float2*>(a1[rr] + j0);
                const float2 q = *reinterpret_cast<const float2*>(c1[rr] + j0);
                const float2 p8 = *reinterpret_cast<const float2*>(a1[rr] + j0 + 8);
                const float2 q8 = *reinterpret_cast<const float2*>(c1[rr] + j0 + 8);
                h[rr][0] = fmaxf(p.x + q.x + lq[rr] * swq[j0], 0.0f);
                h[rr][1] = fmaxf(p.y + q.y + lq[rr] * swq[j0 + 1], 0.0f);
                h[rr][2] = fmaxf(p8.x + q8.x + lq[rr] * swq[j0 + 8], 0.0f);
                h[rr][3] = fmaxf(p8.y + q8.y + lq[rr] * swq[j0 + 9], 0.0f);
            }
            af[c][0] = pack_bf16(h[0][0], h[0][1]);
            af[c][1] = pack_bf16(h[1][0], h[1][1]);
            af[c][2] = pack_bf16(h[0][2], h[0][3]);
            af[c][3] = pack_bf16(h[1][2], h[1][3]);
        }
        float y0 = 0.0f, y1 = 0.0f;
#pragma unroll 4
        for (int nc = 0; nc < 16; nc++) {
            float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            const uint32_t* brow = sW2 + (nc * 8 + g) * kW2ld + tq;
#pragma unroll
            for (int kc = 0; kc < 8; kc++) mma_bf16(acc, af[kc], brow[kc * 8], brow[kc * 8 + 4]);
            const int col = nc * 8 + tq * 2;
            y0 += fmaxf(acc[0] + sb2[col], 0.0f) * sw3[col] + fmaxf(acc[1] + sb2[col + 1], 0.0f) * sw3[col + 1];
            y1 += fmaxf(acc[2] + sb2[col], 0.0f) * sw3[col] + fmaxf(acc[3] + sb2[col + 1], 0.0f) * sw3[col + 1];
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (tq == 0) {
#pragma unroll
            for (int rr = 0; rr < 2; rr++) {
                if (!valid[rr]) continue;
                // a non-finite prediction gives no warm start for that entry
                const double lz = (double)mu + (double)sigma * (double)((rr ? y1 : y0) + b3);
                warm[(size_t)kk[rr] * N + vv[rr]] = isfinite(lz) ? exp(fmin(fmax(lz, -700.0), 700.0)) : 0.0;
            }
        }
    }
}

// ---- inference with tcgen05 (the default path) -----------------------------------------------
// A persistent CTA of 128 threads keeps W2 (BF16) in shared memory in the UMMA canonical
// K-major layout without swizzle.  Per tile of 128 samples:
//  1. thread t builds its sample's h1 (BF16) into row t of the A tile, in the same layout;
//  2. one thread issues eight tcgen05.mma (M = 128, N = 128, K = 16 each, kind::f16: BF16
//     operands from shared memory, FP32 accumulation in 128 TMEM columns) and commits them
//     to an mbarrier;
//  3. after that barrier phase completes (a bounded wait), warp w reads TMEM lanes
//     32w .. 32w + 31 (the rows of its threads' samples) with tcgen05.ld, 16 columns at a
//     time, and forms y = w3 . relu(acc + b2) + b3 in registers.
// Canonical K-major layout, no swizzle: an 8-row x 16-byte core matrix is 128 contiguous
// bytes, and element (r, k) of a 128 x 128 BF16 tile sits at byte
//   (r % 8) * 16 + (r / 8) * 2048 + (k / 8) * 128 + (k % 8) * 2:
// core matrices adjacent in K are 128 bytes apart (the descriptor's leading byte offset),
// those adjacent in M or N 2,048 bytes apart (its stride byte offset), and MMA step s
// (K = 16 s .. 16 s + 15) starts 256 s bytes into the tile.
constexpr uint32_t kTcTile = 128;
constexpr int kTcI = 16, kTcK = 8;  // a tile's target states x rate sets (kTcI * kTcK = kTcTile)
constexpr uint32_t kTcLBO = 128, kTcSBO = 2048;
constexpr uint32_t kTcTileBytes = kTcTile * kH * 2;
constexpr uint32_t kTcWaitLimit = 1u << 22;  // mbarrier polls before a tile is given up
constexpr uint32_t kTcTestWaitLimit = 1u << 10;  // the same when the timeout path is tested
// instruction descriptor, kind::f16: F32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9
// and 10-12 = 1), both K-major (bits 15 and 16 = 0), N >> 3 in bits 17-22, M >> 4 in 24-28
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((kTcTile >> 3) << 17) | ((kTcTile >> 4) << 24);

__device__ __forceinline__ uint32_t tc_off(uint32_t r, uint32_t k) {
    return (r & 7) * 16 + (r >> 3) * kTcSBO + (k >> 3) * kTcLBO + (k & 7) * 2;
}
// shared-memory matrix descriptor: start address, leading and stride byte offsets (each
// >> 4), descriptor version 1 (bits 46-47), base offset 0, no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kTcLBO >> 4) << 16) | ((uint64_t)(kTcSBO >> 4) << 32) |
           (1ull << 46);
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// polls the mbarrier's phase `parity` at most `limit` times; true once it completed
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Two groups of 4 warps per CTA, each with its own A tile, mbarrier and 128 TMEM columns,
// take alternate tiles, so that one group's MMAs and epilogue overlap the other's h1
// construction.  A group synchronises on its own named barrier (ids 1 and 2).
__device__ __forceinline__ void tc_group_sync(int g) {
    if (g == 0)
        asm volatile("bar.sync 1, 128;" ::: "memory");
    else
        asm volatile("bar.sync 2, 128;" ::: "memory");
}

__global__ void __launch_bounds__(256) k_mlp_predict_tc(int nt, int B, int n, size_t N,
                                                        const uint32_t* __restrict__ targets,
                                                        const uint32_t* __restrict__ F,
                                                        const double* __restrict__ rates,
                                                        const float* __restrict__ A1, const float* __restrict__ C1,
                                                        const __nv_bfloat16* __restrict__ W2h,
                                                        const float* __restrict__ Wq, float mu, float sigma,
                                                        double* __restrict__ warm, int* __restrict__ err,
                                                        int no_mma) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char* sB = tc_smem;  // W2: row = output feature, column = input
    // read as float4: four columns per shared-memory load in the h1 loop and the head
    __shared__ __align__(16) float sb2[kH], sw3[kH], swq[kH];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int sfail[2];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = warp >> 2, gt = tid & 127, gw = warp & 3;  // group, thread and warp within it
    unsigned char* sA = tc_smem + (1 + g) * kTcTileBytes;  // this group's h1 tile
    const uint32_t* w2 = reinterpret_cast<const uint32_t*>(W2h);
    for (int i = tid; i < kH * kH / 2; i += blockDim.x) {
        const uint32_t r = (uint32_t)i / (kH / 2), k = ((uint32_t)i % (kH / 2)) * 2;
        *reinterpret_cast<uint32_t*>(sB + tc_off(r, k)) = w2[i];
    }
    for (int j = tid; j < kH; j += blockDim.x) {
        sb2[j] = Wq[oB2 + j];
        sw3[j] = Wq[oW3 + j];
        swq[j] = Wq[oW1 + j * kIn + kFq];
    }
    const uint32_t bar_a = smem_u32(&bar[g]);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(2 * kTcTile)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t tmem_g = tmem + (uint32_t)g * kTcTile;           // this group's accumulator
    const uint32_t tmem_w = tmem_g + ((uint32_t)(gw * 32) << 16);  // this warp's lanes of it
    const float b3 = Wq[oB3];
    const uint32_t sA_a = smem_u32(sA), sB_a = smem_u32(sB);
    // a tile is 16 target states x 8 rate sets (B is a multiple of 8): its 16 rows of A1
    // and 8 rows of C1 are read by 8 and 16 threads each, and consecutive tiles of a CTA's
    // sweep (rate-set blocks fastest) reuse the same A1 rows from L2
    const long kblocks = B / kTcK, tiles = (long)((nt + kTcI - 1) / kTcI) * kblocks;
    uint32_t parity = 0;
    bool ok = true;
    for (long tile = 2L * blockIdx.x + g; tile < tiles; tile += 2L * gridDim.x) {
        const long ib = tile / kblocks, kb = tile - ib * kblocks;
        int i = (int)(ib * kTcI) + gt / kTcK;
        const int k = (int)(kb * kTcK) + gt % kTcK;
        const bool valid = i < nt;
        if (!valid) i = nt - 1;
        if (gt == 0) sfail[g] = 0;
        const uint32_t v = targets[i];
        const float lq = log_rate_sum(v, F[v], rates + (size_t)k * 2 * n);
        const float* a1 = A1 + (size_t)i * kH;
        const float* c1 = C1 + (size_t)k * kH;
#pragma unroll 4
        for (int c = 0; c < kH / 8; c++) {
            const float4 p0 = *reinterpret_cast<const float4*>(a1 + 8 * c);
            const float4 p1 = *reinterpret_cast<const float4*>(a1 + 8 * c + 4);
            const float4 q0 = *reinterpret_cast<const float4*>(c1 + 8 * c);
            const float4 q1 = *reinterpret_cast<const float4*>(c1 + 8 * c + 4);
            const float4 w0 = *reinterpret_cast<const float4*>(swq + 8 * c);
            const float4 w1 = *reinterpret_cast<const float4*>(swq + 8 * c + 4);
            uint4 pk;
            pk.x = pack_bf16(fmaxf(p0.x + q0.x + lq * w0.x, 0.0f), fmaxf(p0.y + q0.y + lq * w0.y, 0.0f));
            pk.y = pack_bf16(fmaxf(p0.z + q0.z + lq * w0.z, 0.0f), fmaxf(p0.w + q0.w + lq * w0.w, 0.0f));
            pk.z = pack_bf16(fmaxf(p1.x + q1.x + lq * w1.x, 0.0f), fmaxf(p1.y + q1.y + lq * w1.y, 0.0f));
            pk.w = pack_bf16(fmaxf(p1.z + q1.z + lq * w1.z, 0.0f), fmaxf(p1.w + q1.w + lq * w1.w, 0.0f));
            *reinterpret_cast<uint4*>(sA + tc_off((uint32_t)gt, 8u * c)) = pk;
        }
        // the tile's h1 (and, at the first tile, W2) becomes visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_group_sync(g);
        // no_mma (a test of the timeout path): nothing is issued, so the wait below runs
        // out with no tensor-core work in flight
        if (gt == 0 && !no_mma) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (uint32_t st = 0; st < kH / 16; st++) {
                const uint64_t da = tc_desc(sA_a + 256u * st), db = tc_desc(sB_a + 256u * st);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(tmem_g), "l"(da), "l"(db), "r"(kTcIdesc), "r"(st), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                         : "memory");
        }
        if (!tc_wait(bar_a, parity, no_mma ? kTcTestWaitLimit : kTcWaitLimit)) sfail[g] = 1;
        parity ^= 1u;
        tc_group_sync(g);
        if (sfail[g]) {  // the same for every thread of the group
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float y = 0.0f;
#pragma unroll
        for (int c = 0; c < kH / 16; c++) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem_w + 16u * c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 16; e += 4) {
                const float4 bb = *reinterpret_cast<const float4*>(sb2 + 16 * c + e);
                const float4 ww = *reinterpret_cast<const float4*>(sw3 + 16 * c + e);
                y += fmaxf(__uint_as_float(r[e]) + bb.x, 0.0f) * ww.x;
                y += fmaxf(__uint_as_float(r[e + 1]) + bb.y, 0.0f) * ww.y;
                y += fmaxf(__uint_as_float(r[e + 2]) + bb.z, 0.0f) * ww.z;
                y += fmaxf(__uint_as_float(r[e + 3]) + bb.w, 0.0f) * ww.w;
            }
        }
        if (valid) {
            // a non-finite prediction gives no warm start for that entry
            const double lz = (double)mu + (double)sigma * (double)(y + b3);
            warm[(size_t)k * N + v] = isfinite(lz) ? exp(fmin(fmax(lz, -700.0), 700.0)) : 0.0;
        }
        // the group's TMEM reads and its MMAs' reads of the A tile are complete before the
        // next tile overwrites them
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        tc_group_sync(g);
    }
    if (!ok) {
        // the tile's MMAs did not complete within the bound: report, give them one more
        // bounded wait, then release TMEM
        if (gt == 0) atomicExch(err, 1);
        tc_wait(bar_a, parity ^ 1u, no_mma ? kTcTestWaitLimit : kTcWaitLimit);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTcTile)
                     : "memory");
}

}  // namespace
}  // namespace esl

using namespace esl;

struct esl_mlp {
    esl_ctx* ctx = nullptr;
    const esl_net* net = nullptr;
    int n = 0, T = 0, nt = 0;
    int64_t N = 0;
    uint64_t seed = 0, step = 0, version = 0, a1_version = ~0ull;
    float mu = 0.0f, sigma = 1.0f;
    bool have_norm = false;
    DevBuf<uint32_t> targets, reach;
    DevBuf<float> P, G, M1, M2, Wq, Xs, A1;
    DevBuf<__nv_bfloat16> W2h;
    // per-call scratch (grow-only)
    DevBuf<float> X, H1, H2, dZ2, dZ1, y, dy, ts, ws, C1, Xr, loss;
    DevBuf<int32_t> ks, vs;
    DevBuf<double> stats;
    DevBuf<int> tc_err;  // timeout flag of the tcgen05 inference
    int cap = 0, cap_b = 0;
};

namespace {

int grow(esl_mlp* m, int S) {
    if (S <= m->cap) return ESL_OK;
    ESL_TRY(m->X.alloc((size_t)S * kXld));
    ESL_TRY(m->H1.alloc((size_t)S * kH));
    ESL_TRY(m->H2.alloc((size_t)S * kH));
    ESL_TRY(m->dZ2.alloc((size_t)S * kH));
    ESL_TRY(m->dZ1.alloc((size_t)S * kH));
    ESL_TRY(m->y.alloc(S));
    ESL_TRY(m->dy.alloc(S));
    ESL_TRY(m->ts.alloc(S));
    ESL_TRY(m->ws.alloc(S));
    ESL_TRY(m->ks.alloc(S));
    ESL_TRY(m->vs.alloc(S));
    m->cap = S;
    return ESL_OK;
}

template <int EPI>
int gemm(cudaStream_t s, int M, int N, int K, const float* A, long sam, long sak, const float* B, long sbk, long sbn,
         float* C, long ldc, const float* bias = nullptr, const float* mask = nullptr, int split = 1) {
    const int kper = (K + split - 1) / split;
    dim3 g((N + 63) / 64, (M + 63) / 64, split);
    ESL_COUNT_LAUNCH();
    k_gemm<EPI><<<g, 256, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, bias, mask, (kper + 15) / 16 * 16);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int quantize(esl_mlp* m) {
    ESL_COUNT_LAUNCH();
    k_mlp_quant<<<(kParams + 255) / 256, 256, 0, m->ctx->stream>>>(m->P.get(), m->Wq.get(), m->W2h.get());
    ESL_CUDA(cudaGetLastError());
    m->version++;
    return ESL_OK;
}

// forward (and with grad != 0 backward) over S samples whose features are in X;
// gradients are added into G, loss into *dloss
int pass(esl_mlp* m, int S, bool grad, float* dloss) {
    cudaStream_t s = m->ctx->stream;
    const float* Wq = m->Wq.get();
    float* G = m->G.get();
    ESL_TRY(gemm<G_BIAS_RELU>(s, S, kH, kIn, m->X.get(), kXld, 1, Wq + oW1, 1, kIn, m->H1.get(), kH, Wq + oB1));
    ESL_TRY(gemm<G_BIAS_RELU>(s, S, kH, kH, m->H1.get(), kH, 1, Wq + oW2, 1, kH, m->H2.get(), kH, Wq + oB2));
    ESL_COUNT_LAUNCH();
    k_mlp_head<<<(S + 7) / 8, 256, 0, s>>>(S, m->H2.get(), Wq, m->ts.get(), m->ws.get(), m->y.get(),
                                          grad ? m->dy.get() : nullptr, grad ? m->dZ2.get() : nullptr, dloss);
    ESL_CUDA(cudaGetLastError());
    if (!grad) return ESL_OK;
    const int split = std::max(1, std::min(64, S / 1024));
    // dw3 = H2^T dy, db3 = sum dy
    ESL_TRY(gemm<G_ATOMIC>(s, kH, 1, S, m->H2.get(), 1, kH, m->dy.get(), 1, 0, G + oW3, 1, nullptr, nullptr, split));
    ESL_COUNT_LAUNCH();
    k_colsum<<<dim3(1, 64), 32, 0, s>>>(S, 1, m->dy.get(), G + oB3);
    // dW2 = dZ2^T H1, db2 = colsum dZ2
    ESL_TRY(gemm<G_ATOMIC>(s, kH, kH, S, m->dZ2.get(), 1, kH, m->H1.get(), kH, 1, G + oW2, kH, nullptr, nullptr,
                           split));
    ESL_COUNT_LAUNCH();
    k_colsum<<<dim3(1, 64), kH, 0, s>>>(S, kH, m->dZ2.get(), G + oB2);
    // dZ1 = (dZ2 W2) [H1 > 0]
    ESL_TRY(gemm<G_MASK>(s, S, kH, kH, m->dZ2.get(), kH, 1, Wq + oW2, kH, 1, m->dZ1.get(), kH, nullptr, m->H1.get()));
    // dW1 = dZ1^T X, db1 = colsum dZ1
    ESL_TRY(gemm<G_ATOMIC>(s, kH, kIn, S, m->dZ1.get(), 1, kH, m->X.get(), kXld, 1, G + oW1, kIn, nullptr, nullptr,
                           split));
    ESL_COUNT_LAUNCH();
    k_colsum<<<dim3(1, 64), kH, 0, s>>>(S, kH, m->dZ1.get(), G + oB1);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

// reachability of the first 16 terminal SCCs, from the condensation order (sinks last
// among transient SCCs reach only terminals and lower levels)
int build_reach(esl_mlp* m) {
    const esl_net* net = m->net;
    cudaStream_t s = m->ctx->stream;
    const size_t N = (size_t)net->N;
    std::vector<int32_t> order(N), offsets(net->n_sccs + 1), term_of(N), labels(N);
    std::vector<uint32_t> F(N);
    ESL_CUDA(cudaMemcpyAsync(order.data(), net->order.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(offsets.data(), net->offsets.get(), (net->n_sccs + 1) * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(term_of.data(), net->term_of.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(labels.data(), net->labels.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(F.data(), net->F.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> reach(N, 0);
    for (size_t v = 0; v < N; v++)
        if (term_of[v] >= 0 && term_of[v] < kReach) reach[v] = 1u << term_of[v];
    // transient SCCs from the last (lowest level) to the first: successors outside the
    // SCC have lower levels, so their sets are final
    for (int c = net->n_sccs - 1; c >= net->T; c--) {
        uint32_t r = 0;
        for (int p = offsets[c]; p < offsets[c + 1]; p++) {
            const uint32_t v = (uint32_t)order[p];
            uint32_t f = F[v];
            while (f) {
                const int i = __builtin_ctz(f);
                f &= f - 1;
                const uint32_t u = v ^ (1u << i);
                if (labels[u] != labels[v]) r |= reach[u];
            }
        }
        for (int p = offsets[c]; p < offsets[c + 1]; p++) reach[(uint32_t)order[p]] = r;
    }
    ESL_TRY(m->reach.alloc(N));
    ESL_CUDA(cudaMemcpyAsync(m->reach.get(), reach.data(), N * 4, cudaMemcpyHostToDevice, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    return ESL_OK;
}

}  // namespace

extern "C" {

int esl_mlp_create(esl_ctx* ctx, const esl_net* net, uint64_t seed, esl_mlp** out) {
    StreamScope stream_scope_(ctx);
    if (!ctx || !net || !out) return fail(ESL_ERR_INVALID, "NULL argument");
    if (net->n > kBits) return fail(ESL_ERR_TOO_LARGE, "the learned warm start takes networks of at most 20 nodes");
    auto* m = new esl_mlp();
    m->ctx = ctx;
    m->net = net;
    m->n = net->n;
    m->N = net->N;
    m->T = net->T;
    m->seed = seed;
    int rc = ESL_OK;
    std::vector<uint32_t> targets;
    rc = sweep_targets(ctx, net, targets);
    if (rc == ESL_OK) rc = build_reach(m);
    m->nt = (int)targets.size();
    cudaStream_t s = ctx->stream;
    if (rc == ESL_OK) rc = m->targets.alloc(std::max(1, m->nt));
    if (rc == ESL_OK && m->nt > 0 &&
        cudaMemcpyAsync(m->targets.get(), targets.data(), (size_t)m->nt * 4, cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = fail(ESL_ERR_CUDA, "target upload failed");
    for (DevBuf<float>* b : {&m->P, &m->G, &m->M1, &m->M2, &m->Wq})
        if (rc == ESL_OK) rc = b->alloc(kParams);
    if (rc == ESL_OK) rc = m->W2h.alloc(kH * kH);
    if (rc == ESL_OK) rc = m->loss.alloc(1);
    if (rc == ESL_OK) rc = m->stats.alloc(4);
    if (rc == ESL_OK) rc = m->Xs.alloc((size_t)std::max(1, m->nt) * kXld);
    if (rc == ESL_OK) rc = m->A1.alloc((size_t)std::max(1, m->nt) * kH);
    if (rc == ESL_OK) {
        ESL_COUNT_LAUNCH();
        k_mlp_init<<<(kParams + 255) / 256, 256, 0, s>>>(seed, m->P.get());
        if (m->nt > 0) {
            ESL_COUNT_LAUNCH();
            k_mlp_state_features<<<m->nt, 128, 0, s>>>(m->nt, m->n, m->T, m->targets.get(), m->reach.get(),
                                                       m->Xs.get());
        }
        if (cudaMemsetAsync(m->M1.get(), 0, kParams * 4, s) != cudaSuccess ||
            cudaMemsetAsync(m->M2.get(), 0, kParams * 4, s) != cudaSuccess || cudaGetLastError() != cudaSuccess)
            rc = fail(ESL_ERR_CUDA, "MLP initialisation failed");
    }
    if (rc == ESL_OK) rc = quantize(m);
    if (rc == ESL_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(ESL_ERR_CUDA, "MLP initialisation failed");
    if (rc != ESL_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return ESL_OK;
}

int esl_mlp_free(esl_mlp* m) {
    if (!m) return ESL_OK;
    // as esl_net_free: one device-wide wait, and the context is not touched, so that an
    // mlp may be freed after its context (a garbage collector frees them in any order)
    cudaDeviceSynchronize();
    t_released_synced = true;
    delete m;
    t_released_synced = false;
    return ESL_OK;
}

int esl_mlp_info(const esl_mlp* m, int* n_targets, float* mu, float* sigma) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m) return fail(ESL_ERR_INVALID, "mlp is NULL");
    if (n_targets) *n_targets = m->nt;
    if (mu) *mu = m->mu;
    if (sigma) *sigma = m->sigma;
    return ESL_OK;
}

int esl_mlp_targets(const esl_mlp* m, uint32_t* d_states) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || !d_states) return fail(ESL_ERR_INVALID, "NULL argument");
    if (m->nt > 0)
        ESL_CUDA(cudaMemcpyAsync(d_states, m->targets.get(), (size_t)m->nt * 4, cudaMemcpyDeviceToDevice,
                                 m->ctx->stream));
    return ESL_OK;
}

int esl_mlp_reach(const esl_mlp* m, uint32_t* d_reach) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || !d_reach) return fail(ESL_ERR_INVALID, "NULL argument");
    ESL_CUDA(cudaMemcpyAsync(d_reach, m->reach.get(), (size_t)m->N * 4, cudaMemcpyDeviceToDevice, m->ctx->stream));
    return ESL_OK;
}

int esl_mlp_get_params(const esl_mlp* m, float* params) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || !params) return fail(ESL_ERR_INVALID, "NULL argument");
    ESL_CUDA(cudaMemcpyAsync(params, m->P.get(), kParams * 4, cudaMemcpyDeviceToHost, m->ctx->stream));
    ESL_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return ESL_OK;
}

int esl_mlp_set_params(esl_mlp* m, const float* params, float mu, float sigma) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || !params) return fail(ESL_ERR_INVALID, "NULL argument");
    if (!(sigma > 0.0f) || !std::isfinite(mu)) return fail(ESL_ERR_INVALID, "sigma must be > 0 and mu finite");
    ESL_CUDA(cudaMemcpyAsync(m->P.get(), params, kParams * 4, cudaMemcpyHostToDevice, m->ctx->stream));
    m->mu = mu;
    m->sigma = sigma;
    m->have_norm = true;
    ESL_TRY(quantize(m));
    ESL_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return ESL_OK;
}

int esl_mlp_features(esl_mlp* m, int S, const double* d_rates, const int32_t* d_k, const int32_t* d_state,
                     float* d_x) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || S < 0 || (S > 0 && (!d_rates || !d_k || !d_state || !d_x))) return fail(ESL_ERR_INVALID, "bad argument");
    if (S == 0) return ESL_OK;
    ESL_COUNT_LAUNCH();
    k_mlp_features<<<S, 128, 0, m->ctx->stream>>>(S, m->n, m->T, d_k, d_state, d_rates, m->net->F.get(),
                                                  m->reach.get(), d_x);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int esl_mlp_loss_grad(esl_mlp* m, int S, const double* d_rates, const int32_t* d_k, const int32_t* d_state,
                      const float* d_target, float* loss, float* grad) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || S <= 0 || !d_rates || !d_k || !d_state || !d_target || !loss)
        return fail(ESL_ERR_INVALID, "bad argument");
    cudaStream_t s = m->ctx->stream;
    ESL_TRY(grow(m, S));
    ESL_TRY(esl_mlp_features(m, S, d_rates, d_k, d_state, m->X.get()));
    ESL_CUDA(cudaMemcpyAsync(m->ts.get(), d_target, (size_t)S * 4, cudaMemcpyDeviceToDevice, s));
    std::vector<float> ones(S, 1.0f);
    ESL_CUDA(cudaMemcpyAsync(m->ws.get(), ones.data(), (size_t)S * 4, cudaMemcpyHostToDevice, s));
    ESL_CUDA(cudaMemsetAsync(m->G.get(), 0, kParams * 4, s));
    ESL_CUDA(cudaMemsetAsync(m->loss.get(), 0, 4, s));
    ESL_TRY(pass(m, S, grad != nullptr, m->loss.get()));
    ESL_CUDA(cudaMemcpyAsync(loss, m->loss.get(), 4, cudaMemcpyDeviceToHost, s));
    if (grad) ESL_CUDA(cudaMemcpyAsync(grad, m->G.get(), kParams * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    return ESL_OK;
}

int esl_mlp_train(esl_mlp* m, int B, const double* d_rates, const double* d_occupation, int steps, int batch, float lr,
                  float* final_loss) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || B <= 0 || !d_rates || !d_occupation || steps < 0 || batch <= 0 || !(lr > 0.0f))
        return fail(ESL_ERR_INVALID, "bad argument");
    if (m->nt == 0) return fail(ESL_ERR_INVALID, "the network has no state that takes a warm start");
    cudaStream_t s = m->ctx->stream;
    ESL_TRY(grow(m, batch));
    if (!m->have_norm) {
        // label standardisation from 64K random pairs
        const int S = 65536;
        ESL_CUDA(cudaMemsetAsync(m->stats.get(), 0, 4 * 8, s));
        ESL_COUNT_LAUNCH();
        k_mlp_label_stats<<<S / 256, 256, 0, s>>>(S, m->seed, B, m->nt, m->targets.get(), (size_t)m->N, d_occupation,
                                                  m->stats.get());
        double h[4];
        ESL_CUDA(cudaMemcpyAsync(h, m->stats.get(), 4 * 8, cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        if (!(h[2] > 1.0)) return fail(ESL_ERR_INVALID, "occupation labels are all zero");
        const double mean = h[0] / h[2], var = std::max(h[1] / h[2] - mean * mean, 1e-12);
        m->mu = (float)mean;
        m->sigma = (float)std::sqrt(var);
        m->have_norm = true;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int it = 0; it < steps; it++) {
        m->step++;
        ESL_COUNT_LAUNCH();
        k_mlp_sample<<<(batch + 255) / 256, 256, 0, s>>>(batch, m->seed, m->step, B, m->nt, m->targets.get(),
                                                         (size_t)m->N, d_occupation, m->mu, m->sigma, m->ks.get(),
                                                         m->vs.get(), m->ts.get(), m->ws.get());
        ESL_TRY(esl_mlp_features(m, batch, d_rates, m->ks.get(), m->vs.get(), m->X.get()));
        ESL_CUDA(cudaMemsetAsync(m->G.get(), 0, kParams * 4, s));
        const bool last = it + 1 == steps;
        if (last) ESL_CUDA(cudaMemsetAsync(m->loss.get(), 0, 4, s));
        ESL_TRY(pass(m, batch, true, last ? m->loss.get() : nullptr));
        const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
        ESL_COUNT_LAUNCH();
        k_mlp_adam<<<(kParams + 255) / 256, 256, 0, s>>>(kParams, m->P.get(), m->G.get(), m->M1.get(), m->M2.get(), lr,
                                                         b1, b2, eps, c1, c2);
        ESL_CUDA(cudaGetLastError());
        ESL_TRY(quantize(m));
    }
    float l = 0.0f;
    if (steps > 0) ESL_CUDA(cudaMemcpyAsync(&l, m->loss.get(), 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    if (final_loss) *final_loss = l;
    return ESL_OK;
}

int esl_mlp_predict(esl_mlp* m, int B, const double* d_rates, double* d_warm) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || B <= 0 || !d_rates || !d_warm) return fail(ESL_ERR_INVALID, "bad argument");
    cudaStream_t s = m->ctx->stream;
    ESL_CUDA(cudaMemsetAsync(d_warm, 0, (size_t)B * m->N * 8, s));
    if (m->nt == 0) return ESL_OK;
    const float* Wq = m->Wq.get();
    // per-state part of layer 1 (cached until the weights change)
    if (m->a1_version != m->version) {
        ESL_TRY(gemm<G_BIAS>(s, m->nt, kH, kIn, m->Xs.get(), kXld, 1, Wq + oW1, 1, kIn, m->A1.get(), kH, Wq + oB1));
        m->a1_version = m->version;
    }
    // per-rate-set part
    if (B > m->cap_b) {
        ESL_TRY(m->Xr.alloc((size_t)B * kXld));
        ESL_TRY(m->C1.alloc((size_t)B * kH));
        m->cap_b = B;
    }
    ESL_COUNT_LAUNCH();
    k_mlp_rate_features<<<B, 128, 0, s>>>(B, m->n, d_rates, m->Xr.get());
    ESL_TRY(gemm<G_STORE>(s, B, kH, kIn, m->Xr.get(), kXld, 1, Wq + oW1, 1, kIn, m->C1.get(), kH));
    // layer 2 on the tcgen05 tensor cores; ESL_MLP_TC=0 selects the mma.sync kernel
    const char* tc_env = getenv("ESL_MLP_TC");
    if (!(tc_env && tc_env[0] == '0') && B % kTcK == 0) {
        // ESL_MLP_TC_TIMEOUT_TEST=1 issues no MMAs, so that the kernel's bounded wait runs
        // out and the call returns ESL_ERR_TIMEOUT (a test of that path; read per call)
        const char* tt_env = getenv("ESL_MLP_TC_TIMEOUT_TEST");
        const int no_mma = (tt_env && tt_env[0] == '1') ? 1 : 0;
        ESL_CUDA(cudaFuncSetAttribute(k_mlp_predict_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(3 * kTcTileBytes)));
        if (!m->tc_err.get()) ESL_TRY(m->tc_err.alloc(1));
        ESL_CUDA(cudaMemsetAsync(m->tc_err.get(), 0, sizeof(int), s));
        const long tiles = (long)((m->nt + kTcI - 1) / kTcI) * (B / kTcK);
        // at most 2 CTAs per SM fit the 98 KB of shared memory, so the 256 TMEM columns of
        // each stay within the SM's 512
        const unsigned grid = (unsigned)std::min<long>((tiles + 1) / 2, (long)m->ctx->sm_count * 2);
        ESL_COUNT_LAUNCH();
        k_mlp_predict_tc<<<grid, 256, 3 * kTcTileBytes, s>>>(m->nt, B, m->n, (size_t)m->N, m->targets.get(),
                                                             m->net->F.get(), d_rates, m->A1.get(), m->C1.get(),
                                                             m->W2h.get(), Wq, m->mu, m->sigma, d_warm,
                                                             m->tc_err.get(), no_mma);
        ESL_CUDA(cudaGetLastError());
        int h_err = 0;
        ESL_CUDA(cudaMemcpyAsync(&h_err, m->tc_err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        if (h_err) return fail(ESL_ERR_TIMEOUT, "tensor-core inference: an MMA did not complete in time");
        return ESL_OK;
    }
    const long tiles = ((long)m->nt * B + 15) / 16;
    const unsigned grid = (unsigned)std::min<long>((tiles + 3) / 4, (long)m->ctx->sm_count * 16);
    ESL_COUNT_LAUNCH();
    k_mlp_predict<<<grid, 128, 0, s>>>(m->nt, B, m->n, (size_t)m->N, m->targets.get(), m->net->F.get(), d_rates,
                                       m->A1.get(), m->C1.get(), m->W2h.get(), Wq, m->mu, m->sigma, d_warm);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

// reference forward of the training passes (FP32 SIMT, BF16-rounded weights) for samples,
// written as predicted occupations; used to check the tensor-core inference
int esl_mlp_forward(esl_mlp* m, int S, const double* d_rates, const int32_t* d_k, const int32_t* d_state,
                    float* d_y) {
    StreamScope stream_scope_(m ? m->ctx : nullptr);
    if (!m || S <= 0 || !d_rates || !d_k || !d_state || !d_y) return fail(ESL_ERR_INVALID, "bad argument");
    cudaStream_t s = m->ctx->stream;
    ESL_TRY(grow(m, S));
    ESL_TRY(esl_mlp_features(m, S, d_rates, d_k, d_state, m->X.get()));
    ESL_CUDA(cudaMemsetAsync(m->ts.get(), 0, (size_t)S * 4, s));
    ESL_CUDA(cudaMemsetAsync(m->ws.get(), 0, (size_t)S * 4, s));
    ESL_TRY(pass(m, S, false, nullptr));
    ESL_CUDA(cudaMemcpyAsync(d_y, m->y.get(), (size_t)S * 4, cudaMemcpyDeviceToDevice, s));
    return ESL_OK;
}

}  // extern "C"
