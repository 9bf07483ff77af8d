// Level sweep of the transient forward solve, in state-major layout.
//
// Replaces the transient half of solver::solve_nonterminal_part
// (cuda/src/solver.cu:205-300) and its block-triangular solve
// (cuda/src/linear_system_solve.cu:249-325, 492-626) for the forward form: the expected
// occupation z of the transient states solves (Q - A) z = x0, and terminal SCC t
// receives y_t = x0(t) + sum over edges u -> v, u transient, v in t, of rate * z_u.
// That is L x0 of the reference without forming L.
//
// The transient block is lower triangular in the topological order of the condensation:
// an SCC receives flow only from SCCs of higher level and never from another SCC of its
// own level.  Level groups are solved one after another, sources first, and inside a
// group every SCC is an independent diagonal block.  Per group:
//   - singleton SCCs only: z_v = b_v / q_v;
//   - SCCs of at most kSwDenseMax states: dense FP64 Gauss-Jordan per (SCC, system),
//     without pivoting (a transient SCC leaks, so its block is column diagonally
//     dominant);
//   - otherwise BiCGStab on the odd-parity Schur complement.  Every edge flips one bit, so
//     the graph is bipartite by popcount parity and the even rows are eliminated exactly.
//     The right preconditioner is the Schur diagonal, and inner iterations run in FP64
//     (ESL_METHOD_DIRECT) or FP32 (ESL_METHOD_MIXED) inside FP64 iterative refinement on
//     the true residual.
//
// Layout: every vector is [row][system], the Kp (K rounded up to 32) systems of a row
// contiguous.  A warp handles 32 systems of one state, so every neighbour gather reads a
// contiguous run of 32 values however scattered the group's states are among the 2^n.
// Rows are "slots": the transient states numbered group by group, even-parity states of
// a group first, then odd.  The row structure (state, out-mask, predecessor lists) is
// read once per row and shared by every system.  Rates are staged per CTA in shared
// memory as [rate index][system lane].
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kSwT = 256;            // threads per row kernel
constexpr int kSwDenseMax = 256;     // largest SCC of a group solved by dense Gauss-Jordan
constexpr int kSwDenseSmem = 160;    // dense SCCs up to this size keep their matrix in shared memory
constexpr int kSwPoll = 4;           // Krylov iterations launched between convergence polls
constexpr double kSwAcceptRel = 1e-8;  // stagnating systems are accepted at this relative residual
constexpr int kSwStall = 30;         // inner iterations without halving the residual before an inner solve stops

// per-system flags
constexpr int SW_DONE = 1;   // group solve finished for this system
constexpr int SW_FAIL = 2;   // finished without meeting the acceptance residual
constexpr int SW_RUN = 4;    // runs an inner solve in this refinement step
constexpr int SW_IDONE = 8;  // its inner solve has stopped

// per-system scalar arrays (doubles), each Kp long
enum Scal { C_BB, C_RR64, C_PREV, C_RHO, C_R0V, C_TS, C_TT, C_RR, C_RN, C_BETA, C_OMEGA, C_TARGET, C_BEST, C_NSCAL };
// per-system int arrays
enum IScal { I_FLAGS, I_ITERS, I_NOIMP, I_TOTAL, I_STALL, I_NISCAL };

struct SwGroup {
    uint32_t beg, ne, no;  // first slot, even rows, odd rows
    int kind;              // 0 singletons, 1 dense, 2 Krylov
    int max_scc;
    uint32_t scc0, nscc;   // dense groups: range in the dense SCC list
    uint64_t scr;          // dense groups: scratch doubles per system (matrices kept in global memory)
    int smax;              // dense groups: largest SCC
};

struct SweepPlan {
    uint32_t M = 0, max_rows = 0, max_even = 0, max_odd = 0;
    int TS = 0;
    std::vector<SwGroup> groups;
    DevBuf<uint2> rows;                  // per slot: (state, out-mask)
    DevBuf<uint32_t> ig_ptr, ig_ent;     // predecessors inside the group: slot << 5 | bit
    DevBuf<uint32_t> og_ptr, og_ent;     // predecessors in earlier groups
    DevBuf<uint32_t> tp_ptr, tp_ent;     // transient predecessors of terminal position p
    DevBuf<uint32_t> dscc_off;           // dense SCCs: offsets into dscc_slots
    DevBuf<uint32_t> dscc_slots;         // dense SCCs: slots, SCC by SCC
    DevBuf<uint64_t> dscc_scr;           // dense SCCs: scratch offset within the group's per-system scratch
    DevBuf<uint32_t> dloc;               // per slot of a dense group: index inside its SCC
};

void free_plan_sweep(void* p) { delete static_cast<SweepPlan*>(p); }

struct SwArgs {
    int n, K, Kp, nrhs, KT;
    const double* rateT;     // [2n][Kp], rateT[j * Kp + k] = rate j of system k (0 past K)
    const uint2* rows;
    const uint32_t* ig_ptr;
    const uint32_t* ig_ent;
    uint32_t beg, ne, no;
    const int* flags;        // per-system flags or null
};

struct Tile {
    int lane, rsub, RB, KT, k;
};

__device__ __forceinline__ Tile tile_of(int KT) {
    Tile t;
    t.KT = KT;
    t.RB = blockDim.x / KT;
    t.lane = threadIdx.x % KT;
    t.rsub = threadIdx.x / KT;
    t.k = blockIdx.y * KT + t.lane;
    return t;
}

template <class T>
__device__ __forceinline__ void sw_rates(T* s, const SwArgs& a, const Tile& t) {
    const int k0 = blockIdx.y * t.KT;
    const int tot = 2 * a.n * t.KT;
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int j = idx / t.KT, l = idx - j * t.KT;
        s[idx] = (T)a.rateT[(size_t)j * a.Kp + k0 + l];
    }
    __syncthreads();
}

// out-rate of state v (out-mask f) for this thread's system
template <class T>
__device__ __forceinline__ T sw_q(const T* s, uint32_t v, uint32_t f, const Tile& t) {
    T q = 0;
    while (f) {
        const int i = __ffs(f) - 1;
        f &= f - 1;
        q += s[(2 * i + ((v >> i) & 1u)) * t.KT + t.lane];
    }
    return q;
}

// rate of the edge into v that flips bit i (its source has bit i of v complemented)
template <class T>
__device__ __forceinline__ T sw_in(const T* s, uint32_t v, int i, const Tile& t) {
    return s[(2 * i + (((v >> i) & 1u) ^ 1u)) * t.KT + t.lane];
}

__device__ __forceinline__ bool sw_skip(const SwArgs& a, int k) {
    if (k >= a.K) return true;
    if (!a.flags) return false;
    const int f = a.flags[k];
    return !(f & SW_RUN) || (f & SW_IDONE);
}

// Block-wide sums of NV per-thread values for this thread's system, added atomically to
// dst[j][k] by the first row-lane.
template <int NV>
__device__ __forceinline__ void sw_reduce(const double (&v)[NV], double* const (&dst)[NV], const Tile& t, int K) {
    __shared__ double red[NV * kSwT];
#pragma unroll
    for (int j = 0; j < NV; j++) red[j * kSwT + threadIdx.x] = v[j];
    __syncthreads();
    if (t.rsub == 0 && t.k < K) {
#pragma unroll
        for (int j = 0; j < NV; j++) {
            double acc = 0.0;
            for (int r = 0; r < t.RB; r++) acc += red[j * kSwT + r * t.KT + t.lane];
            if (acc != 0.0) atomicAdd(dst[j] + t.k, acc);
        }
    }
}

// ---- right-hand sides -------------------------------------------------------------------
// b_v = x0(v) + inflow from transient states of earlier groups, for every row of the
// group; DIRECT groups store z_v = b_v / q_v in Z, others b into the group buffer Bv.
template <bool DIRECT>
__global__ void __launch_bounds__(kSwT) k_sw_rhs(SwArgs a, const uint32_t* __restrict__ og_ptr,
                                                 const uint32_t* __restrict__ og_ent, const double* __restrict__ x0,
                                                 size_t x0_ld, double* __restrict__ Z, double* __restrict__ Bv) {
    extern __shared__ double s_rate[];
    const Tile t = tile_of(a.KT);
    sw_rates(s_rate, a, t);
    if (t.k >= a.K) return;
    const uint32_t cnt = a.ne + a.no;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < cnt; r += gridDim.x * t.RB) {
        const uint32_t slot = a.beg + r;
        const uint2 row = a.rows[slot];
        const uint32_t v = row.x;
        double acc = x0[(size_t)(t.k % a.nrhs) * x0_ld + v];
        for (uint32_t e = og_ptr[slot]; e < og_ptr[slot + 1]; e++) {
            const uint32_t ent = og_ent[e];
            acc += sw_in(s_rate, v, (int)(ent & 31u), t) * Z[(size_t)(ent >> 5) * a.Kp + t.k];
        }
        if (DIRECT)
            Z[(size_t)slot * a.Kp + t.k] = acc / sw_q(s_rate, v, row.y, t);
        else
            Bv[(size_t)r * a.Kp + t.k] = acc;
    }
}

// Schur diagonal on the odd rows: dS_o = q_o - sum over in-group e with e -> o and o -> e
// of rate(e -> o) rate(o -> e) / q_e.
__global__ void __launch_bounds__(kSwT) k_sw_diag(SwArgs a, double* __restrict__ dS64, float* __restrict__ dS32) {
    extern __shared__ double s_rate[];
    const Tile t = tile_of(a.KT);
    sw_rates(s_rate, a, t);
    if (t.k >= a.K) return;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
        const uint32_t slot = a.beg + a.ne + r;
        const uint2 row = a.rows[slot];
        const uint32_t o = row.x;
        double d = sw_q(s_rate, o, row.y, t);
        for (uint32_t e = a.ig_ptr[slot]; e < a.ig_ptr[slot + 1]; e++) {
            const uint32_t ent = a.ig_ent[e];
            const int i = (int)(ent & 31u);
            if (!((row.y >> i) & 1u)) continue;  // no edge o -> e
            const uint2 re = a.rows[ent >> 5];
            d -= sw_in(s_rate, o, i, t) * sw_in(s_rate, re.x, i, t) / sw_q(s_rate, re.x, re.y, t);
        }
        dS64[(size_t)r * a.Kp + t.k] = d;
        if (dS32) dS32[(size_t)r * a.Kp + t.k] = (float)d;
    }
}

// Even-row elimination: W_e = (C_e + sum over in-group odd predecessors o of
// rate(o -> e) X_o) / q_e.  C (FP64, even rows of the group buffer) and X may be null.
template <class TX, class TW, class TC>
__global__ void __launch_bounds__(kSwT) k_sw_elim(SwArgs a, const double* __restrict__ C, const TX* __restrict__ X,
                                                  TW* __restrict__ W) {
    extern __shared__ unsigned char s_raw[];
    TC* s_rate = reinterpret_cast<TC*>(s_raw);
    const Tile t = tile_of(a.KT);
    sw_rates(s_rate, a, t);
    if (sw_skip(a, t.k)) return;
    const uint32_t obase = a.beg + a.ne;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.ne; r += gridDim.x * t.RB) {
        const uint32_t slot = a.beg + r;
        const uint2 row = a.rows[slot];
        const uint32_t v = row.x;
        TC acc = C ? (TC)C[(size_t)r * a.Kp + t.k] : (TC)0;
        if (X) {
            for (uint32_t e = a.ig_ptr[slot]; e < a.ig_ptr[slot + 1]; e++) {
                const uint32_t ent = a.ig_ent[e];
                acc += sw_in(s_rate, v, (int)(ent & 31u), t) * (TC)X[(size_t)((ent >> 5) - obase) * a.Kp + t.k];
            }
        }
        W[(size_t)r * a.Kp + t.k] = (TW)(acc / sw_q(s_rate, v, row.y, t));
    }
}

// Odd-row operator.  y = q X - sum over in-group even predecessors e of rate(e -> o) W_e.
//   MODE 0: Y = B + sum(rate W)          (reduced rhs, FP64), acc0 += Y^2
//   MODE 1: Y = B - y                    (true residual, FP64), acc0 += Y^2
//   MODE 2: Y = y                        acc0 += AUX . Y   (AUX = r0)
//   MODE 3: Y = y                        acc0 += Y . (AUX X), acc1 += Y . Y   (AUX = dS)
template <int MODE, class T>
__global__ void __launch_bounds__(kSwT) k_sw_apply(SwArgs a, const T* __restrict__ X, const T* __restrict__ W,
                                                   const double* __restrict__ B, const T* __restrict__ AUX,
                                                   T* __restrict__ Y, double* acc0, double* acc1) {
    extern __shared__ unsigned char s_raw[];
    T* s_rate = reinterpret_cast<T*>(s_raw);
    const Tile t = tile_of(a.KT);
    sw_rates(s_rate, a, t);
    double d0 = 0.0, d1 = 0.0;
    const bool skip = (MODE >= 2) ? sw_skip(a, t.k) : (t.k >= a.K);
    if (!skip) {
        for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
            const uint32_t slot = a.beg + a.ne + r;
            const uint2 row = a.rows[slot];
            const uint32_t o = row.x;
            const size_t idx = (size_t)r * a.Kp + t.k;
            T flow = 0;
            for (uint32_t e = a.ig_ptr[slot]; e < a.ig_ptr[slot + 1]; e++) {
                const uint32_t ent = a.ig_ent[e];
                flow += sw_in(s_rate, o, (int)(ent & 31u), t) * W[(size_t)((ent >> 5) - a.beg) * a.Kp + t.k];
            }
            if (MODE == 0) {
                const double y = B[idx] + (double)flow;
                Y[idx] = (T)y;
                d0 += y * y;
            } else {
                const T x = X[idx];
                const T y = sw_q(s_rate, o, row.y, t) * x - flow;
                if (MODE == 1) {
                    const double res = B[idx] - (double)y;
                    Y[idx] = (T)res;
                    d0 += res * res;
                } else if (MODE == 2) {
                    Y[idx] = y;
                    d0 += (double)AUX[idx] * (double)y;
                } else {
                    Y[idx] = y;
                    d0 += (double)y * ((double)AUX[idx] * (double)x);
                    d1 += (double)y * (double)y;
                }
            }
        }
    }
    if (MODE == 3) {
        double v[2] = {d0, d1};
        double* const dst[2] = {acc0, acc1};
        sw_reduce<2>(v, dst, t, a.K);
    } else {
        double v[1] = {d0};
        double* const dst[1] = {acc0};
        sw_reduce<1>(v, dst, t, a.K);
    }
}

// ---- BiCGStab vector steps (odd rows; scalars per system) --------------------------------
struct SwScalPtr {
    double* c[C_NSCAL];
    int* i[I_NISCAL];
};

template <class T>
__global__ void __launch_bounds__(kSwT) k_sw_p(SwArgs a, SwScalPtr sc, const T* __restrict__ R, const T* __restrict__ dS,
                                               const T* __restrict__ V, T* __restrict__ PH) {
    const Tile t = tile_of(a.KT);
    if (sw_skip(a, t.k)) return;
    const T beta = (T)sc.c[C_BETA][t.k], omega = (T)sc.c[C_OMEGA][t.k];
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
        const size_t idx = (size_t)r * a.Kp + t.k;
        const T d = dS[idx];
        PH[idx] = (R[idx] + beta * (d * PH[idx] - omega * V[idx])) / d;
    }
}

template <class T>
__global__ void __launch_bounds__(kSwT) k_sw_s(SwArgs a, SwScalPtr sc, const T* __restrict__ R, const T* __restrict__ V,
                                               const T* __restrict__ dS, T* __restrict__ SH) {
    const Tile t = tile_of(a.KT);
    if (sw_skip(a, t.k)) return;
    const double r0v = sc.c[C_R0V][t.k];
    const T alpha = r0v != 0.0 ? (T)(sc.c[C_RHO][t.k] / r0v) : (T)0;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
        const size_t idx = (size_t)r * a.Kp + t.k;
        SH[idx] = (R[idx] - alpha * V[idx]) / dS[idx];
    }
}

template <class T>
__global__ void __launch_bounds__(kSwT) k_sw_xr(SwArgs a, SwScalPtr sc, const T* __restrict__ PH,
                                                const T* __restrict__ SH, const T* __restrict__ dS,
                                                const T* __restrict__ TT, const T* __restrict__ R0, T* __restrict__ D,
                                                T* __restrict__ R) {
    const Tile t = tile_of(a.KT);
    double d0 = 0.0, d1 = 0.0;
    if (!sw_skip(a, t.k)) {
        const double r0v = sc.c[C_R0V][t.k], tt = sc.c[C_TT][t.k];
        const T alpha = r0v != 0.0 ? (T)(sc.c[C_RHO][t.k] / r0v) : (T)0;
        const T omega = tt > 0.0 ? (T)(sc.c[C_TS][t.k] / tt) : (T)0;
        for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
            const size_t idx = (size_t)r * a.Kp + t.k;
            const T sh = SH[idx];
            D[idx] += alpha * PH[idx] + omega * sh;
            const T rn = dS[idx] * sh - omega * TT[idx];
            R[idx] = rn;
            d0 += (double)rn * (double)rn;
            d1 += (double)R0[idx] * (double)rn;
        }
    }
    double v[2] = {d0, d1};
    double* const dst[2] = {sc.c[C_RR], sc.c[C_RN]};
    sw_reduce<2>(v, dst, t, a.K);
}

// Scalar step after each iteration; one CTA; writes the number of running systems.
__global__ void k_sw_scal(int K, SwScalPtr sc, int max_iters, int* active) {
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    int cnt = 0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        int f = sc.i[I_FLAGS][k];
        if (!(f & SW_RUN) || (f & SW_IDONE)) continue;
        const int it = ++sc.i[I_ITERS][k];
        sc.i[I_TOTAL][k]++;
        const double rho = sc.c[C_RHO][k], r0v = sc.c[C_R0V][k], ts = sc.c[C_TS][k], tt = sc.c[C_TT][k];
        const double rr = sc.c[C_RR][k], rn = sc.c[C_RN][k];
        const double alpha = r0v != 0.0 ? rho / r0v : 0.0;
        const double omega = tt > 0.0 ? ts / tt : 0.0;
        if (rr < 0.5 * sc.c[C_BEST][k]) {
            sc.c[C_BEST][k] = rr;
            sc.i[I_STALL][k] = 0;
        } else {
            sc.i[I_STALL][k]++;
        }
        const bool stop = !(rr > sc.c[C_TARGET][k]) || it >= max_iters || r0v == 0.0 || omega == 0.0 ||
                          rn == 0.0 || !isfinite(rr) || !isfinite(alpha) || sc.i[I_STALL][k] >= kSwStall;
        if (stop) {
            sc.i[I_FLAGS][k] = f | SW_IDONE;
        } else {
            sc.c[C_BETA][k] = (rn / rho) * (alpha / omega);
            sc.c[C_OMEGA][k] = omega;
            sc.c[C_RHO][k] = rn;
            cnt++;
        }
        sc.c[C_R0V][k] = sc.c[C_TS][k] = sc.c[C_TT][k] = sc.c[C_RR][k] = sc.c[C_RN][k] = 0.0;
    }
    atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0) *active = s_cnt;
}

// Decide, per system, whether another refinement step runs; writes the count.
__global__ void k_sw_outer(int K, SwScalPtr sc, double tol2, double inner_rel2, double accept2, int outer,
                           int max_refine, int* active) {
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    int cnt = 0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        int f = sc.i[I_FLAGS][k];
        if (f & SW_DONE) continue;
        const double rr = sc.c[C_RR64][k], b2 = sc.c[C_BB][k];
        if (!(b2 > 0.0) || rr <= tol2 * b2) {
            sc.i[I_FLAGS][k] = SW_DONE;
            continue;
        }
        if (outer > 0 && !(rr < 0.25 * sc.c[C_PREV][k])) sc.i[I_NOIMP][k]++;
        if (sc.i[I_NOIMP][k] >= 2 || outer >= max_refine || !isfinite(rr)) {
            sc.i[I_FLAGS][k] = (rr <= accept2 * b2) ? SW_DONE : (SW_DONE | SW_FAIL);
            continue;
        }
        sc.i[I_FLAGS][k] = SW_RUN;
        sc.i[I_ITERS][k] = 0;
        sc.c[C_PREV][k] = rr;
        sc.c[C_RHO][k] = rr;
        sc.c[C_BETA][k] = 0.0;
        sc.c[C_OMEGA][k] = 1.0;
        sc.c[C_TARGET][k] = fmax(inner_rel2 * rr, 0.01 * tol2 * b2);
        sc.c[C_BEST][k] = rr;
        sc.i[I_STALL][k] = 0;
        sc.c[C_R0V][k] = sc.c[C_TS][k] = sc.c[C_TT][k] = sc.c[C_RR][k] = sc.c[C_RN][k] = 0.0;
        cnt++;
    }
    atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0) *active = s_cnt;
}

// start of an inner solve: R = R0 = (T) R64, D = PH = V = 0
template <class T>
__global__ void __launch_bounds__(kSwT) k_sw_start(SwArgs a, const double* __restrict__ R64, T* __restrict__ R,
                                                   T* __restrict__ R0, T* __restrict__ D, T* __restrict__ PH,
                                                   T* __restrict__ V) {
    const Tile t = tile_of(a.KT);
    if (sw_skip(a, t.k)) return;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
        const size_t idx = (size_t)r * a.Kp + t.k;
        const T x = (T)R64[idx];
        R[idx] = x;
        R0[idx] = x;
        D[idx] = 0;
        PH[idx] = 0;
        V[idx] = 0;
    }
}

template <class T>
__global__ void __launch_bounds__(kSwT) k_sw_commit(SwArgs a, const T* __restrict__ D, double* __restrict__ X64) {
    const Tile t = tile_of(a.KT);
    if (t.k >= a.K || !(a.flags[t.k] & SW_RUN)) return;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
        const size_t idx = (size_t)r * a.Kp + t.k;
        X64[idx] += (double)D[idx];
    }
}

// starting iterate of the odd rows: the warm start (K x N, by state) or 0
__global__ void __launch_bounds__(kSwT) k_sw_warm(SwArgs a, const double* __restrict__ warm, size_t warm_ld,
                                                  double* __restrict__ X64) {
    const Tile t = tile_of(a.KT);
    if (t.k >= a.K) return;
    for (uint32_t r = blockIdx.x * t.RB + t.rsub; r < a.no; r += gridDim.x * t.RB) {
        const uint32_t v = a.rows[a.beg + a.ne + r].x;
        X64[(size_t)r * a.Kp + t.k] = warm ? warm[(size_t)t.k * warm_ld + v] : 0.0;
    }
}

// ---- dense Gauss-Jordan per (SCC, system) ---------------------------------------------------
// One CTA per (SCC j of the group, system k0 + blockIdx.y).  Row a is the equation of the
// SCC's a-th state: q_a z_a - sum over in-SCC predecessors b of rate(b -> a) z_b = rhs_a.
__global__ void __launch_bounds__(256) k_sw_dense(SwArgs a, const uint32_t* __restrict__ scc_off,
                                                  const uint32_t* __restrict__ scc_slots,
                                                  const uint32_t* __restrict__ dloc,
                                                  const uint64_t* __restrict__ scr_off, uint64_t scr_stride,
                                                  double* __restrict__ scratch, int smem_max,
                                                  const double* __restrict__ Bv, double* __restrict__ Z, int k0) {
    extern __shared__ double s_dyn[];
    const int j = blockIdx.x;
    const int k = k0 + blockIdx.y;
    if (k >= a.K) return;
    const uint32_t off = scc_off[j];
    const int s = (int)(scc_off[j + 1] - off);
    const int w = s + 1;
    double* s_rate = s_dyn;                       // 2n rates of system k
    double* fac = s_dyn + 2 * a.n;                // s factors
    double* A = (s <= smem_max) ? fac + s : scratch + (size_t)(k - k0) * scr_stride + scr_off[j];
    for (int idx = threadIdx.x; idx < 2 * a.n; idx += blockDim.x) s_rate[idx] = a.rateT[(size_t)idx * a.Kp + k];
    for (int idx = threadIdx.x; idx < s * w; idx += blockDim.x) A[idx] = 0.0;
    __syncthreads();
    for (int r = threadIdx.x; r < s; r += blockDim.x) {
        const uint32_t slot = scc_slots[off + r];
        const uint2 row = a.rows[slot];
        const uint32_t v = row.x;
        double q = 0.0;
        uint32_t f = row.y;
        while (f) {
            const int i = __ffs(f) - 1;
            f &= f - 1;
            q += s_rate[2 * i + ((v >> i) & 1u)];
        }
        A[(size_t)r * w + r] = q;
        for (uint32_t e = a.ig_ptr[slot]; e < a.ig_ptr[slot + 1]; e++) {
            const uint32_t ent = a.ig_ent[e];
            const int i = (int)(ent & 31u);
            A[(size_t)r * w + dloc[ent >> 5]] -= s_rate[2 * i + (((v >> i) & 1u) ^ 1u)];
        }
        A[(size_t)r * w + s] = Bv[(size_t)(slot - a.beg) * a.Kp + k];
    }
    for (int p = 0; p < s; p++) {
        __syncthreads();
        const double inv = 1.0 / A[(size_t)p * w + p];
        for (int r = threadIdx.x; r < s; r += blockDim.x) fac[r] = (r == p) ? 0.0 : A[(size_t)r * w + p] * inv;
        __syncthreads();
        const int cols = s - p;  // columns p+1 .. s
        for (int idx = threadIdx.x; idx < s * cols; idx += blockDim.x) {
            const int r = idx / cols, c = p + 1 + (idx - r * cols);
            const double fr = fac[r];
            if (fr != 0.0) A[(size_t)r * w + c] -= fr * A[(size_t)p * w + c];
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < s; r += blockDim.x)
        Z[(size_t)scc_slots[off + r] * a.Kp + k] = A[(size_t)r * w + s] / A[(size_t)r * w + r];
}

// ---- terminal masses ----------------------------------------------------------------------
// y[k][t] += x0(v) + sum over transient predecessors u of v of rate(u -> v) z_u, v in t
__global__ void __launch_bounds__(kSwT) k_sw_term(SwArgs a, int TS, const int32_t* __restrict__ order,
                                                  const int32_t* __restrict__ term_of,
                                                  const uint32_t* __restrict__ tp_ptr,
                                                  const uint32_t* __restrict__ tp_ent, const double* __restrict__ x0,
                                                  size_t x0_ld, const double* __restrict__ Z, int T,
                                                  double* __restrict__ y) {
    extern __shared__ double s_rate[];
    const Tile t = tile_of(a.KT);
    sw_rates(s_rate, a, t);
    if (t.k >= a.K) return;
    for (int p = blockIdx.x * t.RB + t.rsub; p < TS; p += gridDim.x * t.RB) {
        const uint32_t v = (uint32_t)order[p];
        double acc = x0[(size_t)(t.k % a.nrhs) * x0_ld + v];
        for (uint32_t e = tp_ptr[p]; e < tp_ptr[p + 1]; e++) {
            const uint32_t ent = tp_ent[e];
            acc += sw_in(s_rate, v, (int)(ent & 31u), t) * Z[(size_t)(ent >> 5) * a.Kp + t.k];
        }
        atomicAdd(&y[(size_t)t.k * T + term_of[v]], acc);
    }
}

__global__ void k_sw_rate_table(int n, int K, int Kp, int nrhs, const double* __restrict__ rates,
                                double* __restrict__ rateT) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= Kp) return;
    rateT[(size_t)j * Kp + k] = k < K ? rates[(size_t)(k / nrhs) * 2 * n + j] : 0.0;
}

// ---- host side ------------------------------------------------------------------------------
enum SwSlot { W_Z, W_RATET, W_BV, W_BS, W_R64, W_DS64, W_DS32, W_W64, W_WT, W_R, W_R0, W_PH, W_V, W_SH, W_TT,
              W_D, W_SCAL, W_ISCAL, W_CNT, W_DENSE, W_COUNT };

int build_plan(esl_ctx* ctx, const esl_net* net, SweepPlan*& out) {
    if (net->sweep) {
        out = static_cast<SweepPlan*>(net->sweep);
        return ESL_OK;
    }
    cudaStream_t s = ctx->stream;
    const size_t N = (size_t)net->N;
    const int n_sccs = net->n_sccs, T = net->T;
    std::vector<int32_t> order(N), offsets(n_sccs + 1), levels(std::max(n_sccs, 1)), term_of(N);
    std::vector<uint32_t> F(N), G(N);
    ESL_CUDA(cudaMemcpyAsync(order.data(), net->order.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(offsets.data(), net->offsets.get(), (n_sccs + 1) * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(levels.data(), net->levels.get(), n_sccs * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(term_of.data(), net->term_of.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(F.data(), net->F.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(G.data(), net->G.get(), N * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));

    auto* P = new SweepPlan();
    const int TS = offsets[T];
    P->TS = TS;
    const uint32_t M = (uint32_t)(N - (size_t)TS);
    P->M = M;
    std::vector<uint32_t> slot_of(N, 0xFFFFFFFFu);
    std::vector<uint2> rows;
    rows.reserve(M);
    std::vector<uint32_t> dscc_off{0}, dscc_slots, dloc(M, 0);
    std::vector<uint64_t> dscc_scr;
    for (int c = T; c < n_sccs;) {
        int c1 = c, mx = 0;
        while (c1 < n_sccs && levels[c1] == levels[c]) {
            mx = std::max(mx, offsets[c1 + 1] - offsets[c1]);
            c1++;
        }
        SwGroup g{};
        g.beg = (uint32_t)rows.size();
        g.max_scc = mx;
        g.kind = mx == 1 ? 0 : (mx <= kSwDenseMax ? 1 : 2);
        for (int par = 0; par < 2; par++) {
            for (int p = offsets[c]; p < offsets[c1]; p++) {
                const uint32_t v = (uint32_t)order[p];
                if ((uint32_t)(__builtin_popcount(v) & 1) != (uint32_t)par) continue;
                slot_of[v] = (uint32_t)rows.size();
                rows.push_back(make_uint2(v, F[v]));
            }
            (par ? g.no : g.ne) = (uint32_t)rows.size() - g.beg - (par ? g.ne : 0);
        }
        if (g.kind == 1) {
            g.scc0 = (uint32_t)dscc_off.size() - 1;
            uint64_t scr = 0;
            for (int cc = c; cc < c1; cc++) {
                const int sz = offsets[cc + 1] - offsets[cc];
                for (int p = offsets[cc]; p < offsets[cc + 1]; p++) {
                    const uint32_t sl = slot_of[(uint32_t)order[p]];
                    dloc[sl] = (uint32_t)(p - offsets[cc]);
                    dscc_slots.push_back(sl);
                }
                dscc_off.push_back((uint32_t)dscc_slots.size());
                dscc_scr.push_back(scr);
                if (sz > kSwDenseSmem) scr += (uint64_t)sz * (sz + 1);
                g.smax = std::max(g.smax, sz);
            }
            g.nscc = (uint32_t)(c1 - c);
            g.scr = scr;
        }
        P->max_rows = std::max(P->max_rows, g.ne + g.no);
        P->max_even = std::max(P->max_even, g.ne);
        P->max_odd = std::max(P->max_odd, g.no);
        P->groups.push_back(g);
        c = c1;
    }
    // predecessor lists
    std::vector<uint32_t> ig_ptr{0}, og_ptr{0}, ig, og;
    ig_ptr.reserve(M + 1);
    og_ptr.reserve(M + 1);
    for (const SwGroup& g : P->groups) {
        const uint32_t end = g.beg + g.ne + g.no;
        for (uint32_t sl = g.beg; sl < end; sl++) {
            const uint32_t v = rows[sl].x;
            uint32_t in = G[v];
            while (in) {
                const int i = __builtin_ctz(in);
                in &= in - 1;
                const uint32_t su = slot_of[v ^ (1u << i)];
                if (su == 0xFFFFFFFFu) continue;  // a terminal state has no edge out of its SCC
                ((su >= g.beg && su < end) ? ig : og).push_back((su << 5) | (uint32_t)i);
            }
            ig_ptr.push_back((uint32_t)ig.size());
            og_ptr.push_back((uint32_t)og.size());
        }
    }
    std::vector<uint32_t> tp_ptr{0}, tp;
    for (int p = 0; p < TS; p++) {
        const uint32_t v = (uint32_t)order[p];
        uint32_t in = G[v];
        while (in) {
            const int i = __builtin_ctz(in);
            in &= in - 1;
            const uint32_t su = slot_of[v ^ (1u << i)];
            if (su != 0xFFFFFFFFu) tp.push_back((su << 5) | (uint32_t)i);
        }
        tp_ptr.push_back((uint32_t)tp.size());
    }
    int rc = ESL_OK;
    auto up32 = [&](DevBuf<uint32_t>& d, const std::vector<uint32_t>& h) {
        if (rc != ESL_OK) return;
        rc = d.alloc(h.size());
        if (rc == ESL_OK && !h.empty() &&
            cudaMemcpyAsync(d.get(), h.data(), h.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = fail(ESL_ERR_CUDA, "sweep plan upload failed");
    };
    if (rc == ESL_OK) rc = P->rows.alloc(rows.size());
    if (rc == ESL_OK && !rows.empty() &&
        cudaMemcpyAsync(P->rows.get(), rows.data(), rows.size() * sizeof(uint2), cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
        rc = fail(ESL_ERR_CUDA, "sweep plan upload failed");
    up32(P->ig_ptr, ig_ptr);
    up32(P->ig_ent, ig);
    up32(P->og_ptr, og_ptr);
    up32(P->og_ent, og);
    up32(P->tp_ptr, tp_ptr);
    up32(P->tp_ent, tp);
    up32(P->dscc_off, dscc_off);
    up32(P->dscc_slots, dscc_slots);
    up32(P->dloc, dloc);
    if (rc == ESL_OK) rc = P->dscc_scr.alloc(dscc_scr.size());
    if (rc == ESL_OK && !dscc_scr.empty() &&
        cudaMemcpyAsync(P->dscc_scr.get(), dscc_scr.data(), dscc_scr.size() * 8, cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
        rc = fail(ESL_ERR_CUDA, "sweep plan upload failed");
    if (rc == ESL_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(ESL_ERR_CUDA, "sweep plan upload failed");
    if (rc != ESL_OK) {
        delete P;
        return rc;
    }
    esl_net* mnet = const_cast<esl_net*>(net);
    mnet->sweep = P;
    mnet->sweep_free = free_plan_sweep;
    out = P;
    return ESL_OK;
}

// systems per CTA tile: a divisor of Kp, at most 128, and rates of the tile within 40 KB.
// With `rows` > 0 the tile is also narrowed (down to 32) until one tile's slice of a
// vector over `rows` rows fits in kSwTileBytes, so that the neighbour gathers of a
// Krylov iteration hit L2.
constexpr size_t kSwTileBytes = 48ull << 20;
int tile_for(int Kp, int n, size_t elem, uint32_t rows = 0) {
    int kt = 128;
    while (kt > 32 && (Kp % kt != 0 || (size_t)2 * n * kt * elem > 40 * 1024 ||
                       (size_t)rows * kt * elem > kSwTileBytes))
        kt >>= 1;
    return kt;
}

// Grid of a row kernel: blockIdx.y is the system tile, blockIdx.x strides over rows.
// Each tile gets up to 8 CTAs per SM, so a large group fills the GPU with one tile at a
// time (CTAs are dispatched x-fastest) and its working set stays that tile's slice.
dim3 row_grid(uint32_t rows, int Kp, int KT, int sm_count) {
    const int RB = kSwT / KT;
    const unsigned ty = (unsigned)(Kp / KT);
    uint64_t want = ((uint64_t)rows + RB - 1) / RB;
    const uint64_t cap = std::max<uint64_t>(1, (uint64_t)sm_count * 8);
    if (want > cap) want = cap;
    if (want == 0) want = 1;
    return dim3((unsigned)want, ty);
}

bool debug_on() {
    static int on = -1;
    if (on < 0) on = getenv("ESL_DEBUG") ? 1 : 0;
    return on == 1;
}

}  // namespace

void free_sweep_workspace(void* w) { delete static_cast<Workspace*>(w); }

bool sweep_supported(const esl_net* net) { return net->n >= 1 && net->n <= 27; }

int sweep_forward(esl_ctx* ctx, const esl_net* net, int K, int nrhs, const double* rates, const double* x0,
                  size_t x0_ld, const esl_solve_opts& o, double* y, SweepStats& st) {
    if (!sweep_supported(net)) return fail(ESL_ERR_TOO_LARGE, "level sweep supports at most 27 nodes");
    SweepPlan* P = nullptr;
    ESL_TRY(build_plan(ctx, net, P));
    if (!ctx->sweep_work) ctx->sweep_work = new Workspace();
    Workspace& ws = *static_cast<Workspace*>(ctx->sweep_work);
    cudaStream_t s = ctx->stream;
    const int n = net->n, T = net->T;
    const int Kp = (K + 31) & ~31;
    const bool mixed = o.method == ESL_METHOD_MIXED;
    int st_ = ESL_OK;
    double* Z = (double*)ws.get(W_Z, (size_t)std::max<uint32_t>(P->M, 1) * Kp * 8, &st_);
    double* rateT = (double*)ws.get(W_RATET, (size_t)2 * n * Kp * 8, &st_);
    double* scal = (double*)ws.get(W_SCAL, (size_t)C_NSCAL * Kp * 8, &st_);
    int* iscal = (int*)ws.get(W_ISCAL, (size_t)I_NISCAL * Kp * 4, &st_);
    int* d_cnt = (int*)ws.get(W_CNT, 64, &st_);
    if (st_ != ESL_OK) return st_;
    SwScalPtr sc;
    for (int j = 0; j < C_NSCAL; j++) sc.c[j] = scal + (size_t)j * Kp;
    for (int j = 0; j < I_NISCAL; j++) sc.i[j] = iscal + (size_t)j * Kp;
    ESL_COUNT_LAUNCH();
    k_sw_rate_table<<<dim3((Kp + 127) / 128, 2 * n), 128, 0, s>>>(n, K, Kp, nrhs, rates, rateT);
    ESL_CUDA(cudaGetLastError());

    const int KT64 = tile_for(Kp, n, 8), KT32 = tile_for(Kp, n, 4);
    const size_t sm64 = (size_t)2 * n * KT64 * 8, sm32 = (size_t)2 * n * KT32 * 4;
    SwArgs a{};
    a.n = n;
    a.K = K;
    a.Kp = Kp;
    a.nrhs = nrhs;
    a.rateT = rateT;
    a.rows = P->rows.get();
    a.ig_ptr = P->ig_ptr.get();
    a.ig_ent = P->ig_ent.get();
    int* h_cnt = reinterpret_cast<int*>(ctx->h_flag);  // pinned, at least 8 ints

    const double tol = o.tol > 0 ? o.tol : 1e-10;
    const int max_iters = o.max_iters > 0 ? o.max_iters : 600;
    const int max_refine = o.max_refine > 0 ? o.max_refine : 6;
    std::vector<int> h_flags;
    std::vector<char> failed(K, 0);
    int total_iters = 0;

    for (const SwGroup& g : P->groups) {
        a.beg = g.beg;
        a.ne = g.ne;
        a.no = g.no;
        a.flags = nullptr;
        a.KT = KT64;
        const uint32_t rows = g.ne + g.no;
        if (g.kind == 0) {
            ESL_COUNT_LAUNCH();
            k_sw_rhs<true><<<row_grid(rows, Kp, KT64, ctx->sm_count), kSwT, sm64, s>>>(
                a, P->og_ptr.get(), P->og_ent.get(), x0, x0_ld, Z, nullptr);
            ESL_CUDA(cudaGetLastError());
            continue;
        }
        double* Bv = (double*)ws.get(W_BV, (size_t)P->max_rows * Kp * 8, &st_);
        if (st_ != ESL_OK) return st_;
        ESL_COUNT_LAUNCH();
        k_sw_rhs<false><<<row_grid(rows, Kp, KT64, ctx->sm_count), kSwT, sm64, s>>>(
            a, P->og_ptr.get(), P->og_ent.get(), x0, x0_ld, Z, Bv);
        ESL_CUDA(cudaGetLastError());
        if (g.kind == 1) {
            // dense Gauss-Jordan, systems in chunks that bound the global scratch to ~2 GB
            st.dense_groups++;
            int chunk = K;
            if (g.scr > 0) chunk = (int)std::max<uint64_t>(1, std::min<uint64_t>(K, (256ull << 20) / g.scr));
            double* scr = g.scr > 0 ? (double*)ws.get(W_DENSE, (size_t)chunk * g.scr * 8, &st_) : nullptr;
            if (st_ != ESL_OK) return st_;
            // rates, one factor per row of the largest SCC, and the largest in-smem matrix
            const int sm_s = std::min(g.smax, kSwDenseSmem);
            const size_t smem = (size_t)(2 * n + g.smax + (size_t)sm_s * (sm_s + 1)) * 8;
            ESL_CUDA(cudaFuncSetAttribute(k_sw_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            for (int k0 = 0; k0 < K; k0 += chunk) {
                const int kc = std::min(chunk, K - k0);
                ESL_COUNT_LAUNCH();
                k_sw_dense<<<dim3(g.nscc, kc), 256, smem, s>>>(a, P->dscc_off.get() + g.scc0, P->dscc_slots.get(),
                                                               P->dloc.get(), P->dscc_scr.get() + g.scc0, g.scr, scr,
                                                               kSwDenseSmem, Bv, Z, k0);
                ESL_CUDA(cudaGetLastError());
            }
            continue;
        }
        // ---- Krylov group ----
        st.krylov_groups++;
        const size_t vo = (size_t)std::max<uint32_t>(P->max_odd, 1) * Kp, ve = (size_t)std::max<uint32_t>(P->max_even, 1) * Kp;
        double* bS = (double*)ws.get(W_BS, vo * 8, &st_);
        double* R64 = (double*)ws.get(W_R64, vo * 8, &st_);
        double* dS64 = (double*)ws.get(W_DS64, vo * 8, &st_);
        float* dS32 = mixed ? (float*)ws.get(W_DS32, vo * 4, &st_) : nullptr;
        double* W64 = (double*)ws.get(W_W64, ve * 8, &st_);
        const size_t es = mixed ? 4 : 8;
        void* WT = mixed ? ws.get(W_WT, ve * es, &st_) : (void*)W64;
        void* vR = ws.get(W_R, vo * es, &st_);
        void* vR0 = ws.get(W_R0, vo * es, &st_);
        void* vPH = ws.get(W_PH, vo * es, &st_);
        void* vV = ws.get(W_V, vo * es, &st_);
        void* vSH = ws.get(W_SH, vo * es, &st_);
        void* vTT = ws.get(W_TT, vo * es, &st_);
        void* vD = ws.get(W_D, vo * es, &st_);
        if (st_ != ESL_OK) return st_;
        double* X64 = Z + (size_t)(g.beg + g.ne) * Kp;  // the odd rows of the group, in place
        // tiles narrow enough that one tile's slice of a gathered vector stays in L2
        const int gKT64 = tile_for(Kp, n, 8, std::max(g.ne, g.no)), gKT32 = tile_for(Kp, n, 4, std::max(g.ne, g.no));
        const size_t gsm64 = (size_t)2 * n * gKT64 * 8, gsm32 = (size_t)2 * n * gKT32 * 4;
        a.KT = gKT64;
        const dim3 ge = row_grid(g.ne, Kp, gKT64, ctx->sm_count), go = row_grid(g.no, Kp, gKT64, ctx->sm_count);
        ESL_CUDA(cudaMemsetAsync(scal, 0, (size_t)C_NSCAL * Kp * 8, s));
        ESL_CUDA(cudaMemsetAsync(iscal, 0, (size_t)I_NISCAL * Kp * 4, s));
        ESL_COUNT_LAUNCH();
        k_sw_diag<<<go, kSwT, gsm64, s>>>(a, dS64, dS32);
        // reduced rhs bS = b_odd + A_oe (b_even / q_e)
        ESL_COUNT_LAUNCH();
        k_sw_elim<double, double, double><<<ge, kSwT, gsm64, s>>>(a, Bv, (const double*)nullptr, W64);
        ESL_COUNT_LAUNCH();
        k_sw_apply<0, double><<<go, kSwT, gsm64, s>>>(a, nullptr, W64, Bv + (size_t)g.ne * Kp, nullptr, bS,
                                                     sc.c[C_BB], nullptr);
        ESL_COUNT_LAUNCH();
        k_sw_warm<<<go, kSwT, 0, s>>>(a, o.d_warm, (size_t)net->N, X64);
        ESL_CUDA(cudaGetLastError());
        auto true_residual = [&]() -> int {
            a.flags = nullptr;
            a.KT = gKT64;
            ESL_CUDA(cudaMemsetAsync(sc.c[C_RR64], 0, (size_t)Kp * 8, s));
            ESL_COUNT_LAUNCH();
            k_sw_elim<double, double, double><<<ge, kSwT, gsm64, s>>>(a, nullptr, X64, W64);
            ESL_COUNT_LAUNCH();
            k_sw_apply<1, double><<<go, kSwT, gsm64, s>>>(a, X64, W64, bS, nullptr, R64, sc.c[C_RR64], nullptr);
            ESL_CUDA(cudaGetLastError());
            return ESL_OK;
        };
        ESL_TRY(true_residual());
        bool inner64 = !mixed;
        int group_iters = 0;
        for (int outer = 0;; outer++) {
            const double inner_rel = inner64 ? 1e-13 : 1e-5;
            ESL_COUNT_LAUNCH();
            k_sw_outer<<<1, 1024, 0, s>>>(K, sc, tol * tol, inner_rel * inner_rel, kSwAcceptRel * kSwAcceptRel,
                                          outer, max_refine, d_cnt);
            ESL_CUDA(cudaGetLastError());
            ESL_CUDA(cudaMemcpyAsync(h_cnt, d_cnt, 4, cudaMemcpyDeviceToHost, s));
            ESL_CUDA(cudaStreamSynchronize(s));
            if (h_cnt[0] == 0) break;
            a.flags = sc.i[I_FLAGS];
            a.KT = inner64 ? gKT64 : gKT32;
            const size_t smT = inner64 ? gsm64 : gsm32;
            const dim3 gei = row_grid(g.ne, Kp, a.KT, ctx->sm_count), goi = row_grid(g.no, Kp, a.KT, ctx->sm_count);
            auto run_inner = [&](auto tag) -> int {
                using TT = decltype(tag);
                TT* R = (TT*)vR;
                TT* R0 = (TT*)vR0;
                TT* PH = (TT*)vPH;
                TT* V = (TT*)vV;
                TT* SH = (TT*)vSH;
                TT* Tt = (TT*)vTT;
                TT* D = (TT*)vD;
                TT* WW = (TT*)(sizeof(TT) == 8 ? (void*)W64 : WT);
                const TT* dS = (const TT*)(sizeof(TT) == 8 ? (void*)dS64 : (void*)dS32);
                ESL_COUNT_LAUNCH();
                k_sw_start<TT><<<goi, kSwT, 0, s>>>(a, R64, R, R0, D, PH, V);
                int it = 0, chunk = 0;
                for (; it < max_iters; it += kSwPoll, chunk++) {
                    for (int j = 0; j < kSwPoll; j++) {
                        ESL_COUNT_LAUNCH();
                        k_sw_p<TT><<<goi, kSwT, 0, s>>>(a, sc, R, dS, V, PH);
                        ESL_COUNT_LAUNCH();
                        k_sw_elim<TT, TT, TT><<<gei, kSwT, smT, s>>>(a, nullptr, PH, WW);
                        ESL_COUNT_LAUNCH();
                        k_sw_apply<2, TT><<<goi, kSwT, smT, s>>>(a, PH, WW, nullptr, R0, V, sc.c[C_R0V], nullptr);
                        ESL_COUNT_LAUNCH();
                        k_sw_s<TT><<<goi, kSwT, 0, s>>>(a, sc, R, V, dS, SH);
                        ESL_COUNT_LAUNCH();
                        k_sw_elim<TT, TT, TT><<<gei, kSwT, smT, s>>>(a, nullptr, SH, WW);
                        ESL_COUNT_LAUNCH();
                        k_sw_apply<3, TT><<<goi, kSwT, smT, s>>>(a, SH, WW, nullptr, dS, Tt, sc.c[C_TS], sc.c[C_TT]);
                        ESL_COUNT_LAUNCH();
                        k_sw_xr<TT><<<goi, kSwT, 0, s>>>(a, sc, PH, SH, dS, Tt, R0, D, R);
                        ESL_COUNT_LAUNCH();
                        k_sw_scal<<<1, 1024, 0, s>>>(K, sc, max_iters, d_cnt + 1 + (chunk & 1));
                    }
                    ESL_CUDA(cudaGetLastError());
                    ESL_CUDA(cudaMemcpyAsync(h_cnt + 1 + (chunk & 1), d_cnt + 1 + (chunk & 1), 4,
                                             cudaMemcpyDeviceToHost, s));
                    ESL_CUDA(cudaEventRecord(ctx->poll_ev[chunk & 1], s));
                    if (chunk >= 1) {
                        ESL_CUDA(cudaEventSynchronize(ctx->poll_ev[(chunk - 1) & 1]));
                        if (h_cnt[1 + ((chunk - 1) & 1)] == 0) {
                            it += kSwPoll;
                            break;
                        }
                    }
                }
                group_iters += it;
                ESL_COUNT_LAUNCH();
                k_sw_commit<TT><<<goi, kSwT, 0, s>>>(a, D, X64);
                ESL_CUDA(cudaGetLastError());
                return ESL_OK;
            };
            if (inner64) {
                ESL_TRY(run_inner(double{}));
            } else {
                ESL_TRY(run_inner(float{}));
            }
            ESL_TRY(true_residual());
            // an FP32 step that no longer halves the residual: continue in FP64
            if (!inner64 && outer >= 2) inner64 = true;
        }
        // even rows of the group from the odd solution, straight into Z
        a.flags = nullptr;
        a.KT = gKT64;
        ESL_COUNT_LAUNCH();
        k_sw_elim<double, double, double><<<ge, kSwT, gsm64, s>>>(a, Bv, X64, Z + (size_t)g.beg * Kp);
        ESL_CUDA(cudaGetLastError());
        h_flags.resize(K);
        std::vector<double> h_rr(K), h_bb(K);
        ESL_CUDA(cudaMemcpyAsync(h_flags.data(), sc.i[I_FLAGS], (size_t)K * 4, cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaMemcpyAsync(h_rr.data(), sc.c[C_RR64], (size_t)K * 8, cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaMemcpyAsync(h_bb.data(), sc.c[C_BB], (size_t)K * 8, cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        double worst = 0.0;
        for (int k = 0; k < K; k++) {
            if (h_flags[k] & SW_FAIL) failed[k] = 1;
            if (h_bb[k] > 0) worst = std::max(worst, std::sqrt(h_rr[k] / h_bb[k]));
        }
        st.relres = std::max(st.relres, worst);
        total_iters += group_iters;
        if (debug_on())
            fprintf(stderr, "[esl-sweep] group beg %u even %u odd %u max_scc %d: iters %d relres %.3e\n", g.beg, g.ne,
                    g.no, g.max_scc, group_iters, worst);
    }
    // masses into the terminal SCCs
    a.flags = nullptr;
    a.KT = KT64;
    if (P->TS > 0) {
        ESL_COUNT_LAUNCH();
        k_sw_term<<<row_grid((uint32_t)P->TS, Kp, KT64, ctx->sm_count), kSwT, sm64, s>>>(
            a, P->TS, net->order.get(), net->term_of.get(), P->tp_ptr.get(), P->tp_ent.get(), x0, x0_ld, Z, T, y);
        ESL_CUDA(cudaGetLastError());
    }
    st.iters = total_iters;
    st.failed.clear();
    for (int k = 0; k < K; k++)
        if (failed[k]) st.failed.push_back(k);
    if (!st.failed.empty()) {
        char msg[160];
        snprintf(msg, sizeof msg, "level sweep: %zu of %d systems above the acceptance residual",
                 st.failed.size(), K);
        return fail(ESL_ERR_NOT_CONVERGED, msg);
    }
    return ESL_OK;
}

}  // namespace esl
