// Numeric phase: terminal kernels R, transient absorption, x_inf = R (L x0) and
// per-node marginals, batched over rate sets and initial distributions.
//
// Replaces solver::solve (cuda/src/solver.cu:311-334): solve_terminal_part
// (:102-159, minor determinants per state), solve_nonterminal_part (:205-300,
// block LU of N^T with one triangular solve per terminal) and compute_final_states
// (:302-309).
//
// Generator convention of the reference (cuda/src/kernels/solver.cu:20-44):
// K[dst,src] = rate of src -> dst, rate index 2*i + (up ? 0 : 1) for a flip of bit i,
// diagonal = -(total out-rate).
//
// Terminal kernels: per terminal SCC C, K_C pi = 0 with the last equation replaced
// by sum(pi) = 1, dense FP64 LU with partial pivoting in shared memory (one CTA per
// SCC and rate set); larger SCCs pin their first state and solve the remaining
// (nonsingular) system with the Krylov engine below.
//
// Transient part, forward form (one system per rate set and x0): the expected
// occupation z of the transient states solves (Q - A) z = x0 with Q = diag(out-rate)
// and A the transient->transient rates; the mass entering terminal t is
// y_t = x0(t) + sum over edges u->v, u transient, v in t of rate * z_u.  Backward
// form (one system per rate set and terminal, gives the reference's L): h_t solves
// (Q - A^T) h = rate into t.
//
// Every state-transition edge flips one bit, so the graph is bipartite by the parity
// of popcount(state).  The systems are reduced to their odd-parity half (Schur
// complement after eliminating the even half, whose diagonal block is diagonal);
// half index h of state s is s >> 1.  The reduced system is solved by BiCGStab with
// the Schur diagonal as (right) Jacobi preconditioner, inside an FP64 iterative
// refinement loop: the true residual is always formed in FP64, the inner solve runs
// in FP64 (ESL_METHOD_FP64) or FP32 (ESL_METHOD_MIXED).  All operators are applied
// matrix-free from the flip masks and the rates.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "esl_internal.h"

namespace esl {
namespace {

constexpr int kT = 256;
constexpr uint32_t kDomainBit = 0x80000000u;
constexpr uint32_t kMaskBits = 0x3FFFFFFFu;

__device__ __forceinline__ uint32_t state_of(uint32_t h, int parity) {
    return (h << 1) | (uint32_t)((__popc(h) & 1) ^ parity);
}
__device__ __forceinline__ uint32_t nb_half(uint32_t h, int i) { return i == 0 ? h : (h ^ (1u << (i - 1))); }

// per-system scalar state of BiCGStab
struct KState {
    double rho, alpha, omega, beta;
    double r0v, ts, tt, r0r, rr;
    double rnorm2_true, bnorm2, target2, prev_r2, rnorm2_trial;
    int done, iters, breakdown, pad, noimp, total_iters;
    // the last inner solve's exit, kept for the debug report: breakdown code, its
    // iterations, and r0.v / r.r when it stopped
    int last_breakdown, last_iters;
    double last_r0v, last_rr;
    // inner solves restarted after a breakdown or a correction that did not lower the
    // true residual; from the first, the shadow residual r0 is no longer r itself but r
    // plus a dense positive vector (k_inner_start)
    int shadow;
};

// A system whose true FP64 residual stops improving (a refinement step no longer
// halves it) has reached the accuracy FP64 can deliver for it; it is accepted when
// that residual is within kAcceptRel of ||b||.
constexpr double kAcceptRel = 1e-8;
// iteration budget of each level-group solve of the block forward solve; systems
// that miss it have the group's SCC blocks (up to kDenseFallbackMax states) solved
// by dense LU instead
constexpr int kBlockBudget = 3000;
constexpr int kDenseFallbackMax = 4096;
// scratch of one dense-fallback launch; failed systems are taken in chunks that fit
constexpr size_t kDenseScratchBytes = (size_t)2 << 30;

int block_budget(const esl_ctx* ctx, const esl_solve_opts& o) {
    return ctx->block_iters > 0 ? ctx->block_iters : std::max(o.max_iters, kBlockBudget);
}
int dense_cap(const esl_ctx* ctx) { return ctx->dense_max > 0 ? ctx->dense_max : kDenseFallbackMax; }

template <class T>
__device__ __forceinline__ void load_rates(T* s_rate, const double* __restrict__ rates, int b, int n) {
    for (int j = threadIdx.x; j < 2 * n; j += blockDim.x) s_rate[j] = (T)rates[(size_t)b * 2 * n + j];
}

template <class T>
__device__ __forceinline__ T out_rate(const T* s_rate, uint32_t f, uint32_t v) {
    T q = 0;
    while (f) {
        int i = __ffs(f) - 1;
        f &= f - 1;
        q += s_rate[2 * i + ((v >> i) & 1u)];
    }
    return q;
}

// coupling of state v with its neighbour across bit i in v's equation
template <bool FWD, class T>
__device__ __forceinline__ T coupling(const T* s_rate, int i, uint32_t v) {
    uint32_t bit = (v >> i) & 1u;
    return FWD ? s_rate[2 * i + (bit ^ 1u)] : s_rate[2 * i + bit];
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// block-wide sum of up to 2 values, atomically added to dst0/dst1 by thread 0
__device__ __forceinline__ void block_sum2(double a, double b, double* dst0, double* dst1) {
    __shared__ double s_a[kT / 32], s_b[kT / 32];
    a = warp_sum(a);
    b = warp_sum(b);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        s_a[w] = a;
        s_b[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = l < (int)(blockDim.x >> 5) ? s_a[l] : 0.0;
        b = l < (int)(blockDim.x >> 5) ? s_b[l] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        if (l == 0) {
            if (dst0) atomicAdd(dst0, a);
            if (dst1) atomicAdd(dst1, b);
        }
    }
}

struct Layout {
    int n;
    uint32_t H;         // half length N/2
    size_t ld;          // leading dimension of per-system vectors
    int nrhs;           // systems per rate set
    // x0 row of system k: k % nrhs, or k when the caller gathered one x0 row per system
    int x0_sys = 0;
    const uint32_t* M0; // even-half coupling masks | domain bit
    const uint32_t* M1; // odd-half coupling masks | domain bit
    const uint32_t* F0; // even-half out-masks
    const uint32_t* F1; // odd-half out-masks
    // pinned terminal systems: state pins[k*T + terminal] is fixed to 1 in system k
    const int32_t* pins;
    const int32_t* term_of;
    int T;
    // when set, blockIdx.y indexes this list of running systems
    const int32_t* act;
    // when set, rows are restricted to these half indices (even / odd parity)
    const uint32_t* list0;
    const uint32_t* list1;
    uint32_t n0, n1;
};

__device__ __forceinline__ int sys_index(const Layout& L) { return L.act ? L.act[blockIdx.y] : (int)blockIdx.y; }

// half index of this thread's row of the given parity; false past the last row
__device__ __forceinline__ bool row_h(const Layout& L, int parity, uint32_t& h) {
    const uint32_t idx = blockIdx.x * kT + threadIdx.x;
    const uint32_t* list = parity ? L.list1 : L.list0;
    if (list) {
        if (idx >= (parity ? L.n1 : L.n0)) return false;
        h = list[idx];
        return true;
    }
    h = idx;
    return idx < L.H;
}

// pinned state of the row's SCC in system k, or -1
__device__ __forceinline__ int32_t row_pin(const Layout& L, int k, uint32_t v) {
    return L.pins ? L.pins[(size_t)k * L.T + L.term_of[v]] : -1;
}

// wE[h] = (bE[h] + sum_i c_i x1[nb]) / q  on the even half (bE may be null)
template <bool FWD, class T, class TX>
__global__ void __launch_bounds__(kT) k_elim(Layout L, const double* __restrict__ rates, const TX* __restrict__ x1,
                                             const double* __restrict__ bE, T* __restrict__ wE,
                                             const KState* __restrict__ st) {
    __shared__ T s_rate[64];
    const int k = sys_index(L);
    if (st && st[k].done) return;
    load_rates(s_rate, rates, k / L.nrhs, L.n);
    __syncthreads();
    uint32_t h;
    if (!row_h(L, 0, h)) return;
    const size_t o = (size_t)k * L.ld;
    uint32_t m = L.M0[h];
    if (!(m & kDomainBit)) {
        wE[o + h] = 0;
        return;
    }
    uint32_t v = state_of(h, 0);
    const int32_t pin = row_pin(L, k, v);
    if ((int32_t)v == pin) {
        wE[o + h] = 0;
        return;
    }
    T acc = bE ? (T)bE[o + h] : (T)0;
    if (x1) {
        uint32_t mm = m & kMaskBits;
        while (mm) {
            int i = __ffs(mm) - 1;
            mm &= mm - 1;
            if ((int32_t)(v ^ (1u << i)) == pin) continue;
            acc += coupling<FWD>(s_rate, i, v) * (T)x1[o + nb_half(h, i)];
        }
    }
    wE[o + h] = acc / out_rate(s_rate, L.F0[h], v);
}

// Odd-half operator.  mode 0: y = S x (and dot r0.y -> st.r0v);
// mode 2: y = S x with x = s / dS, dots (y . dS x) -> ts and (y . y) -> tt;
// mode 3: residual r = b - S x (FP64) with r.r -> rnorm2_true;
// mode 5: as mode 3 for a trial iterate, r.r -> rnorm2_trial (systems with an inner solve);
// mode 4: rhs  y = b + sum_i c_i w[nb]  (x unused).
template <bool FWD, int MODE, class T, class TX>
__global__ void __launch_bounds__(kT) k_apply(Layout L, const double* __restrict__ rates, const TX* __restrict__ x,
                                              const T* __restrict__ wE, const double* __restrict__ dS,
                                              const double* __restrict__ b, const T* __restrict__ r0,
                                              T* __restrict__ y, KState* __restrict__ st) {
    __shared__ T s_rate[64];
    const int k = sys_index(L);
    if (st && MODE != 3 && MODE != 4 && MODE != 5 && st[k].done) return;
    if (MODE == 5 && st[k].pad) return;
    load_rates(s_rate, rates, k / L.nrhs, L.n);
    __syncthreads();
    uint32_t h = 0;
    const bool valid = row_h(L, 1, h);
    const size_t o = (size_t)k * L.ld;
    double d0 = 0, d1 = 0;
    if (valid) {
        uint32_t m = L.M1[h];
        const uint32_t v = state_of(h, 1);
        const int32_t pin = (m & kDomainBit) ? row_pin(L, k, v) : -1;
        T out;
        if (!(m & kDomainBit) || (int32_t)v == pin) {
            out = MODE == 4 ? (T)0 : ((MODE == 3 || MODE == 5) ? (T)0 : (T)x[o + h]);
        } else {
            T acc = 0;
            uint32_t mm = m & kMaskBits;
            while (mm) {
                int i = __ffs(mm) - 1;
                mm &= mm - 1;
                if ((int32_t)(v ^ (1u << i)) == pin) continue;
                acc += coupling<FWD>(s_rate, i, v) * wE[o + nb_half(h, i)];
            }
            if (MODE == 4) {
                out = (T)b[o + h] + acc;
            } else {
                T q = out_rate(s_rate, L.F1[h], v);
                T sx = q * (T)x[o + h] - acc;
                out = (MODE == 3 || MODE == 5) ? (T)b[o + h] - sx : sx;
            }
        }
        y[o + h] = out;
        if (MODE == 0) d0 = (double)r0[o + h] * (double)out;
        if (MODE == 2) {
            d0 = (double)out * (double)x[o + h] * dS[o + h];
            d1 = (double)out * (double)out;
        }
        if (MODE == 3 || MODE == 5) d0 = (double)out * (double)out;
    }
    if (MODE == 0) block_sum2(d0, 0.0, &st[k].r0v, nullptr);
    if (MODE == 2) block_sum2(d0, d1, &st[k].ts, &st[k].tt);
    if (MODE == 3) block_sum2(d0, 0.0, &st[k].rnorm2_true, nullptr);
    if (MODE == 5) block_sum2(d0, 0.0, &st[k].rnorm2_trial, nullptr);
}

// Schur diagonal dS[h] = q_o - sum_i c_i(o) c_i(e)/q_e over odd states o (1 outside the domain)
template <bool FWD>
__global__ void __launch_bounds__(kT) k_schur_diag(Layout L, const double* __restrict__ rates, double* __restrict__ dS) {
    __shared__ double s_rate[64];
    const int k = blockIdx.y;
    load_rates(s_rate, rates, k / L.nrhs, L.n);
    __syncthreads();
    uint32_t h;
    if (!row_h(L, 1, h)) return;
    const size_t o = (size_t)k * L.ld;
    uint32_t m = L.M1[h];
    const uint32_t v = state_of(h, 1);
    const int32_t pin = (m & kDomainBit) ? row_pin(L, k, v) : -1;
    if (!(m & kDomainBit) || (int32_t)v == pin) {
        dS[o + h] = 1.0;
        return;
    }
    double d = out_rate(s_rate, L.F1[h], v);
    uint32_t mm = m & kMaskBits;
    while (mm) {
        int i = __ffs(mm) - 1;
        mm &= mm - 1;
        if ((int32_t)(v ^ (1u << i)) == pin) continue;
        uint32_t he = nb_half(h, i);
        uint32_t me = L.M0[he];
        if ((me >> i) & 1u) {
            uint32_t e = state_of(he, 0);
            d -= coupling<FWD>(s_rate, i, v) * coupling<FWD>(s_rate, i, e) / out_rate(s_rate, L.F0[he], e);
        }
    }
    dS[o + h] = d;
}

// ---- BiCGStab vector updates ------------------------------------------------------
// start of an inner solve: r = (T) r64, d = 0, p = v = 0, scalars reset.  The shadow
// residual is r0 = r, except in a system restarted after a breakdown or a useless
// correction (st.shadow > 0): there domain row h gets r0_h = r_h + c_h |r| / sqrt(rows),
// c_h in [0.5, 1.5) from a hash of (h, system, restart), and rho = r0.r is summed here
// (k_outer_check left it at 0).  Why: when the transient part is acyclic, the Jacobi-
// scaled Schur complement is I - N with N nilpotent, and a shadow residual with the
// support of r can be orthogonal to the whole Krylov space: in one backward system of
// the 15-node kras network with uniform rates (32,768 singleton SCCs), r0.v fell to
// 1e-16 |r0||v| at the second iteration of every refinement round, with r0 = r and with
// r0 = r scaled row by row alike; the dense shadow converges in 8 iterations.  Any r0
// with r0.r != 0 is a valid BiCGStab shadow residual.
template <class T>
__global__ void __launch_bounds__(kT) k_inner_start(Layout L, const double* __restrict__ r64, T* __restrict__ r,
                                                    T* __restrict__ r0, T* __restrict__ d, T* __restrict__ ph,
                                                    T* __restrict__ v, KState* __restrict__ st) {
    const int k = sys_index(L);
    if (st[k].done) return;
    const int shadow = st[k].shadow;
    uint32_t h = 0;
    const bool valid = row_h(L, 1, h);
    double a = 0.0;
    if (valid) {
        size_t i = (size_t)k * L.ld + h;
        T val = (T)r64[i];
        r[i] = val;
        T sv = val;
        if (shadow && (L.M1[h] & kDomainBit)) {
            uint32_t x = h * 0x9E3779B1u ^ (uint32_t)k * 0x85EBCA77u ^ (uint32_t)shadow * 0xC2B2AE3Du;
            x ^= x >> 15;
            x *= 0x2C1B3C6Du;
            x ^= x >> 12;
            const double rows = (double)(L.list1 ? L.n1 : L.H);
            const double c = 0.5 + (double)(x >> 8) * (1.0 / 16777216.0);
            sv = (T)((double)val + c * sqrt(st[k].rnorm2_true / rows));
            a = (double)sv * (double)val;
        }
        r0[i] = sv;
        d[i] = 0;
        ph[i] = 0;
        v[i] = 0;
    }
    if (shadow) block_sum2(a, 0.0, &st[k].rho, nullptr);
}

template <class T>
__global__ void k_update_p(Layout L, const double* __restrict__ dS, const T* __restrict__ r, T* __restrict__ ph,
                           const T* __restrict__ v, const KState* __restrict__ st) {
    const int k = sys_index(L);
    if (st[k].done) return;
    uint32_t h;
    if (!row_h(L, 1, h)) return;
    size_t i = (size_t)k * L.ld + h;
    T beta = (T)st[k].beta, omega = (T)st[k].omega;
    T inv = (T)(1.0 / dS[i]);
    ph[i] = r[i] * inv + beta * (ph[i] - omega * v[i] * inv);
}

template <class T>
__global__ void k_update_s(Layout L, const double* __restrict__ dS, const T* __restrict__ r, const T* __restrict__ v,
                           T* __restrict__ sh, const KState* __restrict__ st) {
    const int k = sys_index(L);
    if (st[k].done) return;
    uint32_t h;
    if (!row_h(L, 1, h)) return;
    size_t i = (size_t)k * L.ld + h;
    T alpha = (T)st[k].alpha;
    sh[i] = (r[i] - alpha * v[i]) * (T)(1.0 / dS[i]);
}

template <class T>
__global__ void __launch_bounds__(kT) k_update_xr(Layout L, const double* __restrict__ dS, T* __restrict__ d,
                                                  T* __restrict__ r, const T* __restrict__ r0,
                                                  const T* __restrict__ ph, const T* __restrict__ sh,
                                                  const T* __restrict__ t, KState* __restrict__ st) {
    const int k = sys_index(L);
    if (st[k].done) return;
    uint32_t h = 0;
    const bool valid = row_h(L, 1, h);
    double a = 0, b = 0;
    if (valid) {
        size_t i = (size_t)k * L.ld + h;
        T alpha = (T)st[k].alpha, omega = (T)st[k].omega;
        d[i] += alpha * ph[i] + omega * sh[i];
        T rn = (T)dS[i] * sh[i] - omega * t[i];
        r[i] = rn;
        a = (double)r0[i] * (double)rn;
        b = (double)rn * (double)rn;
    }
    block_sum2(a, b, &st[k].r0r, &st[k].rr);
}

// scalar steps, one thread per system
__global__ void k_scal_alpha(int K, KState* st) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K || st[k].done) return;
    KState& s = st[k];
    if (s.r0v == 0.0 || !isfinite(s.r0v)) {
        s.breakdown = 1;
        s.done = 1;
        return;
    }
    s.alpha = s.rho / s.r0v;
    s.ts = s.tt = 0.0;
}

__global__ void k_scal_omega(int K, KState* st) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K || st[k].done) return;
    KState& s = st[k];
    s.omega = s.tt > 0.0 ? s.ts / s.tt : 0.0;
    s.r0r = s.rr = 0.0;
}

__global__ void k_scal_beta(int K, KState* st, int max_iters) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K || st[k].done) return;
    KState& s = st[k];
    s.iters++;
    s.total_iters++;
    if (s.rr <= s.target2 || s.iters >= max_iters) {
        s.done = 1;
        return;
    }
    // BiCGStab residuals grow transiently (by 1e5 in squared norm on these systems);
    // only a blow-up beyond 1e20 or a NaN stops the inner solve
    if (!(s.rr <= 1e20 * s.rnorm2_true)) {
        s.breakdown = 2;
        s.done = 1;
        return;
    }
    if (s.omega == 0.0 || s.r0r == 0.0 || !isfinite(s.r0r)) {
        s.breakdown = 1;
        s.done = 1;
        return;
    }
    s.beta = (s.r0r / s.rho) * (s.alpha / s.omega);
    s.rho = s.r0r;
    s.r0v = 0.0;
}

// after the true residual: decide which systems still need an inner solve
__global__ void k_outer_check(int K, KState* st, double tol2, double inner_rel2, int outer, int budget,
                              int* n_active) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    KState& s = st[k];
    bool conv = s.rnorm2_true <= tol2 * s.bnorm2 || s.bnorm2 == 0.0;
    bool stalled = outer > 0 && (s.noimp || s.rnorm2_true > 0.25 * s.prev_r2) &&
                   s.rnorm2_true <= kAcceptRel * kAcceptRel * s.bnorm2;
    s.prev_r2 = s.rnorm2_true;
    s.last_breakdown = s.breakdown;
    s.last_iters = s.iters;
    s.last_r0v = s.r0v;
    s.last_rr = s.rr;
    s.done = (conv || stalled || s.total_iters >= budget) ? 1 : 0;
    if (!s.done) {
        atomicAdd(n_active, 1);
        if (s.breakdown || s.noimp) s.shadow++;
        s.rho = s.shadow ? 0.0 : s.rnorm2_true;  // r0 = r: rho = r0.r; else k_inner_start sums it
        s.alpha = s.omega = 1.0;
        s.beta = 0.0;
        s.r0v = 0.0;
        // inner target: reach tol in one inner solve if the inner precision allows
        s.target2 = fmax(0.25 * tol2 * s.bnorm2, inner_rel2 * s.rnorm2_true);
        s.breakdown = 0;
        s.iters = 0;
    }
}


// xt = x + d for systems that ran an inner solve
template <class T>
__global__ void k_trial(Layout L, const double* __restrict__ x64, const T* __restrict__ d, double* __restrict__ xt,
                        const KState* __restrict__ st) {
    const int k = blockIdx.y;
    if (st[k].pad) return;
    uint32_t h;
    if (!row_h(L, 1, h)) return;
    size_t i = (size_t)k * L.ld + h;
    xt[i] = x64[i] + (double)d[i];
}

// keep the trial iterate only where it lowered the true residual
__global__ void k_commit_flags(int K, KState* st, int* n_noimp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    KState& s = st[k];
    s.noimp = 0;
    if (s.pad) return;
    if (s.rnorm2_trial < s.rnorm2_true) {
        s.rnorm2_true = s.rnorm2_trial;
    } else {
        s.noimp = 1;
        atomicAdd(n_noimp, 1);
    }
}

__global__ void k_commit(Layout L, double* __restrict__ x64, double* __restrict__ r64, const double* __restrict__ xt,
                         const double* __restrict__ rt, const KState* __restrict__ st) {
    const int k = blockIdx.y;
    if (st[k].pad || st[k].noimp) return;
    uint32_t h;
    if (!row_h(L, 1, h)) return;
    size_t i = (size_t)k * L.ld + h;
    x64[i] = xt[i];
    r64[i] = rt[i];
}

__global__ void k_zero_trial(int K, KState* st) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) st[k].rnorm2_trial = 0.0;
}

__global__ void k_mark_inner(int K, KState* st) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    st[k].pad = st[k].done;  // systems already converged get no correction
}

__global__ void k_zero_r(int K, KState* st) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    st[k].rnorm2_true = 0.0;
}

// ---- right-hand sides ---------------------------------------------------------------
// forward: b = x0 on transient states; backward (system = (rate set, terminal t)):
// b_v = sum of rates of edges v -> terminal t.  Written in both halves.
template <bool FWD>
__global__ void k_rhs(Layout L, int n, const double* __restrict__ rates, const double* __restrict__ x0,
                      size_t x0_ld, const uint32_t* __restrict__ F, const int32_t* __restrict__ term_of,
                      double* __restrict__ bE, double* __restrict__ bO) {
    __shared__ double s_rate[64];
    const int k = blockIdx.y;
    load_rates(s_rate, rates, k / L.nrhs, L.n);
    __syncthreads();
    uint32_t h = blockIdx.x * kT + threadIdx.x;
    if (h >= L.H) return;
    const size_t o = (size_t)k * L.ld;
    const int r = k % L.nrhs;
#pragma unroll
    for (int par = 0; par < 2; par++) {
        uint32_t v = state_of(h, par);
        double val = 0.0;
        if (term_of[v] < 0) {
            if (FWD) {
                val = x0[(size_t)r * x0_ld + v];
            } else {
                uint32_t f = F[v];
                while (f) {
                    int i = __ffs(f) - 1;
                    f &= f - 1;
                    if (term_of[v ^ (1u << i)] == r) val += s_rate[2 * i + ((v >> i) & 1u)];
                }
            }
        }
        (par ? bO : bE)[o + h] = val;
    }
}

// ---- assembly ---------------------------------------------------------------------
// forward: y[k][t] += x0(v) + sum_{u -> v, u transient} rate * z(u) over v in t
// x0_sys: x0 row of system k is k (one gathered row per system) instead of k % nrhs.
__global__ void k_terminal_mass(int n, int T, int term_states, int nrhs, int x0_sys, size_t ld,
                                const double* __restrict__ rates,
                                const double* __restrict__ x0, size_t x0_ld, const int32_t* __restrict__ order,
                                const int32_t* __restrict__ term_of, const uint32_t* __restrict__ G,
                                const double* __restrict__ zE, const double* __restrict__ zO,
                                double* __restrict__ y) {
    const int k = blockIdx.y;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = k / nrhs, r = x0_sys ? k : k % nrhs;
    const double* rt = rates + (size_t)b * 2 * n;
    int t = -1;
    double acc = 0.0;
    if (p < term_states) {
        const uint32_t v = (uint32_t)order[p];
        t = term_of[v];
        acc = x0[(size_t)r * x0_ld + v];
        uint32_t g = G[v];
        while (g) {
            int i = __ffs(g) - 1;
            g &= g - 1;
            uint32_t u = v ^ (1u << i);
            if (term_of[u] >= 0) continue;
            uint32_t hu = u >> 1;
            double zu = (__popc(u) & 1) ? zO[(size_t)k * ld + hu] : zE[(size_t)k * ld + hu];
            acc += rt[2 * i + ((u >> i) & 1u)] * zu;
        }
    }
    // Positions are grouped by terminal SCC, so the lanes of one SCC are a contiguous
    // run of the warp: a segmented suffix sum leaves the run's total in its first lane,
    // which adds it with one atomic (fewer, larger additions round less).
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double va = __shfl_down_sync(0xFFFFFFFFu, acc, o);
        const int ta = __shfl_down_sync(0xFFFFFFFFu, t, o);
        if (lane + o < 32 && ta == t) acc += va;
    }
    const int tprev = __shfl_up_sync(0xFFFFFFFFu, t, 1);
    if (t >= 0 && (lane == 0 || tprev != t)) atomicAdd(&y[(size_t)k * T + t], acc);
}

// x_inf[k][v] = R_b[pos] * y[k][t] on terminal states; marginals accumulated
__global__ void k_scatter_xinf(int n, int T, int term_states, int nrhs, size_t N, const int32_t* __restrict__ order,
                               const int32_t* __restrict__ term_of, const double* __restrict__ Rb,
                               const double* __restrict__ y, double* __restrict__ x_inf, double* __restrict__ marg) {
    const int k = blockIdx.y;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= term_states) return;
    const int b = k / nrhs;
    uint32_t v = (uint32_t)order[p];
    int t = term_of[v];
    double val = Rb[(size_t)b * term_states + p] * y[(size_t)k * T + t];
    x_inf[(size_t)k * N + v] = val;
    if (marg && val != 0.0) {
        for (int i = 0; i < n; i++)
            if ((v >> i) & 1u) atomicAdd(&marg[(size_t)k * n + i], val);
    }
}

// ---- dense terminal kernels ----------------------------------------------------------
// One CTA per (terminal SCC of size 2..kDenseTerm, rate set).  A = K_C with the last row
// replaced by ones; solve A pi = e_last by Gaussian elimination with partial pivoting.
constexpr int kDenseTerm = kDenseTerminalMax;

__global__ void __launch_bounds__(256) k_dense_terminal(int n, const int32_t* __restrict__ sccs,
                                                        const int32_t* __restrict__ offsets,
                                                        const int32_t* __restrict__ order,
                                                        const uint32_t* __restrict__ F,
                                                        const double* __restrict__ rates, int term_states,
                                                        double* __restrict__ Rb) {
    extern __shared__ double s_mem[];
    __shared__ double s_rate[64];
    __shared__ int s_piv;
    const int t = sccs[blockIdx.x];
    const int b = blockIdx.y;
    const int beg = offsets[t];
    const int s = offsets[t + 1] - beg;
    double* A = s_mem;                         // s x (s+1), last column = rhs
    int32_t* mem = (int32_t*)(A + s * (s + 1));
    const int ld = s + 1;
    for (int j = threadIdx.x; j < 2 * n; j += blockDim.x) s_rate[j] = rates[(size_t)b * 2 * n + j];
    for (int j = threadIdx.x; j < s; j += blockDim.x) mem[j] = order[beg + j];
    for (int j = threadIdx.x; j < s * ld; j += blockDim.x) A[j] = 0.0;
    __syncthreads();
    // column c = source state mem[c]; members are ascending, so locate by binary search
    for (int c = threadIdx.x; c < s; c += blockDim.x) {
        uint32_t v = (uint32_t)mem[c];
        uint32_t f = F[v];
        double diag = 0.0;
        while (f) {
            int i = __ffs(f) - 1;
            f &= f - 1;
            int32_t w = (int32_t)(v ^ (1u << i));
            int lo = 0, hi = s - 1;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (mem[mid] < w) lo = mid + 1; else hi = mid;
            }
            double rt = s_rate[2 * i + ((v >> i) & 1u)];
            if (mem[lo] == w && lo != s - 1) A[lo * ld + c] += rt;  // row lo, written only by column c
            diag += rt;
        }
        if (c != s - 1) A[c * ld + c] -= diag;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < s; c += blockDim.x) A[(s - 1) * ld + c] = 1.0;
    for (int r = threadIdx.x; r < s; r += blockDim.x) A[r * ld + s] = (r == s - 1) ? 1.0 : 0.0;
    __syncthreads();
    for (int col = 0; col < s; col++) {
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = col;
            for (int r = col + threadIdx.x; r < s; r += 32) {
                double a = fabs(A[r * ld + col]);
                if (a > best) { best = a; bi = r; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
                int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (threadIdx.x == 0) s_piv = bi;
        }
        __syncthreads();
        const int piv = s_piv;
        if (piv != col)
            for (int j = col + threadIdx.x; j <= s; j += blockDim.x) {
                double tmp = A[col * ld + j];
                A[col * ld + j] = A[piv * ld + j];
                A[piv * ld + j] = tmp;
            }
        __syncthreads();
        const double inv = 1.0 / A[col * ld + col];
        const int rows = s - col - 1, cols = s - col;  // columns col+1 .. s
        for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
            int r = col + 1 + e / cols, j = col + 1 + e % cols;
            A[r * ld + j] -= A[r * ld + col] * inv * A[col * ld + j];
        }
        __syncthreads();
    }
    // back substitution on the rhs column (single warp, rows descending)
    if (threadIdx.x < 32) {
        for (int r = s - 1; r >= 0; r--) {
            double acc = 0.0;
            for (int j = r + 1 + threadIdx.x; j < s; j += 32) acc += A[r * ld + j] * A[j * ld + s];
            acc = warp_sum(acc);
            if (threadIdx.x == 0) A[r * ld + s] = (A[r * ld + s] - acc) / A[r * ld + r];
            __syncwarp();
        }
    }
    __syncthreads();
    // normalise |pi| (the reference normalises |minor determinants| the same way)
    if (threadIdx.x < 32) {
        double sum = 0.0;
        for (int j = threadIdx.x; j < s; j += 32) sum += fabs(A[j * ld + s]);
        sum = warp_sum(sum);
        for (int j = threadIdx.x; j < s; j += 32) Rb[(size_t)b * term_states + beg + j] = fabs(A[j * ld + s]) / sum;
    }
}

__global__ void k_unit_terminals(int T, const int32_t* __restrict__ offsets, int term_states, double* __restrict__ Rb) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    if (offsets[t + 1] - offsets[t] == 1) Rb[(size_t)blockIdx.y * term_states + offsets[t]] = 1.0;
}

// half-layout masks for one domain; domain(v) decided by `dom`:
// dom = 0: transient states; dom = 1: states of "big" terminal SCCs
__global__ void k_half_masks(int n, uint32_t H, const uint32_t* __restrict__ Md, const uint32_t* __restrict__ F,
                             const int32_t* __restrict__ term_of, const uint8_t* __restrict__ big_term, int dom,
                             uint32_t* __restrict__ M0, uint32_t* __restrict__ M1, uint32_t* __restrict__ F0,
                             uint32_t* __restrict__ F1) {
    uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    for (int par = 0; par < 2; par++) {
        uint32_t v = state_of(h, par);
        int t = term_of[v];
        bool in = dom == 0 ? t < 0 : (t >= 0 && big_term[t]);
        (par ? M1 : M0)[h] = in ? (Md[v] | kDomainBit) : 0u;
        (par ? F1 : F0)[h] = F[v];
    }
}

// Pin of each (big terminal SCC, rate set): the state with the largest ratio of
// in-rate to out-rate, a cheap proxy for the largest stationary mass; pinning a
// high-mass state keeps the remaining system well conditioned.  Ties -> smallest state.
__global__ void k_pin_score(int n, int T, int term_states, const int32_t* __restrict__ order,
                            const int32_t* __restrict__ term_of, const uint8_t* __restrict__ big_term,
                            const uint32_t* __restrict__ F, const uint32_t* __restrict__ G,
                            const double* __restrict__ rates, unsigned long long* __restrict__ best) {
    const int b = blockIdx.y;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= term_states) return;
    uint32_t v = (uint32_t)order[p];
    int t = term_of[v];
    if (!big_term[t]) return;
    const double* rt = rates + (size_t)b * 2 * n;
    double in = 0.0, out = 0.0;
    uint32_t g = G[v], f = F[v];
    while (g) {
        int i = __ffs(g) - 1;
        g &= g - 1;
        uint32_t u = v ^ (1u << i);
        in += rt[2 * i + ((u >> i) & 1u)];
    }
    while (f) {
        int i = __ffs(f) - 1;
        f &= f - 1;
        out += rt[2 * i + ((v >> i) & 1u)];
    }
    float score = (float)(in / out);  // positive: its bits order like unsigned ints
    unsigned long long key = ((unsigned long long)__float_as_uint(score) << 32) | (0xFFFFFFFFull - v);
    atomicMax(&best[(size_t)b * T + t], key);
}

__global__ void k_pin_decode(int count, const unsigned long long* __restrict__ best, int32_t* __restrict__ pins) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    unsigned long long key = best[j];
    pins[j] = key ? (int32_t)(0xFFFFFFFFull - (key & 0xFFFFFFFFull)) : -1;
}

// pinned terminal systems: rhs b_v = rate(pin -> v) for states v of a big terminal SCC
__global__ void k_rhs_pinned(Layout L, const double* __restrict__ rates, const uint32_t* __restrict__ G,
                             double* __restrict__ bE, double* __restrict__ bO) {
    __shared__ double s_rate[64];
    const int k = blockIdx.y;
    load_rates(s_rate, rates, k, L.n);
    __syncthreads();
    uint32_t h = blockIdx.x * kT + threadIdx.x;
    if (h >= L.H) return;
    for (int par = 0; par < 2; par++) {
        uint32_t v = state_of(h, par);
        uint32_t m = (par ? L.M1 : L.M0)[h];
        double val = 0.0;
        if (m & kDomainBit) {
            const int32_t pin = row_pin(L, k, v);
            if ((int32_t)v != pin) {
                uint32_t g = G[v];
                while (g) {
                    int i = __ffs(g) - 1;
                    g &= g - 1;
                    uint32_t u = v ^ (1u << i);
                    if ((int32_t)u == pin) val += s_rate[2 * i + ((u >> i) & 1u)];
                }
            }
        }
        (par ? bO : bE)[(size_t)k * L.ld + h] = val;
    }
}

// R for big terminal SCCs from the pinned solution z (pin = 1), normalised per SCC
__global__ void k_pinned_sum(int T, const int32_t* __restrict__ offsets, const int32_t* __restrict__ order,
                             const uint8_t* __restrict__ big_term, const int32_t* __restrict__ pins, size_t ld,
                             const double* __restrict__ zE, const double* __restrict__ zO, int term_states,
                             double* __restrict__ Rb, double* __restrict__ sums) {
    const int b = blockIdx.y;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= term_states) return;
    uint32_t v = (uint32_t)order[p];
    int t = 0;
    {
        int lo = 0, hi = T;
        while (hi - lo > 1) {
            int mid = (lo + hi) / 2;
            if (offsets[mid] <= p) lo = mid; else hi = mid;
        }
        t = lo;
    }
    if (!big_term[t]) return;
    double val = (int32_t)v == pins[(size_t)b * T + t] ? 1.0 : fabs((__popc(v) & 1) ? zO[(size_t)b * ld + (v >> 1)] : zE[(size_t)b * ld + (v >> 1)]);
    Rb[(size_t)b * term_states + p] = val;
    atomicAdd(&sums[(size_t)b * T + t], val);
}

__global__ void k_pinned_norm(int T, const int32_t* __restrict__ offsets, const uint8_t* __restrict__ big_term,
                              int term_states, double* __restrict__ Rb, const double* __restrict__ sums) {
    const int b = blockIdx.y;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= term_states) return;
    int lo = 0, hi = T;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (offsets[mid] <= p) lo = mid; else hi = mid;
    }
    if (!big_term[lo]) return;
    Rb[(size_t)b * term_states + p] /= sums[(size_t)b * T + lo];
}

// absorption matrix L[t][v] (backward form, one rate set): h on transient states,
// 1 on the states of t
__global__ void k_scatter_L(uint32_t H, int T, size_t N, size_t ld, const int32_t* __restrict__ term_of,
                            const double* __restrict__ zE, const double* __restrict__ zO, double* __restrict__ Lm) {
    const int t = blockIdx.y;
    uint32_t h = blockIdx.x * kT + threadIdx.x;
    if (h >= H) return;
    for (int par = 0; par < 2; par++) {
        uint32_t v = state_of(h, par);
        int c = term_of[v];
        double val = c < 0 ? (par ? zO : zE)[(size_t)t * ld + h] : (c == t ? 1.0 : 0.0);
        Lm[(size_t)t * N + v] = val;
    }
}

// ---- driver ---------------------------------------------------------------------------------

// list of running systems (order irrelevant)
__global__ void k_active_list(int K, const KState* st, int* n, int32_t* list) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K && !st[k].done) list[atomicAdd(n, 1)] = k;
}

__global__ void __launch_bounds__(kT) k_norm2(Layout L, const double* __restrict__ x, KState* st) {
    const int k = blockIdx.y;
    uint32_t h = 0;
    const bool valid = row_h(L, 1, h);
    double a = 0.0;
    if (valid) {
        double v = x[(size_t)k * L.ld + h];
        a = v * v;
    }
    block_sum2(a, 0.0, &st[k].bnorm2, nullptr);
}

__global__ void k_half_from_full(Layout L, const double* __restrict__ full, size_t full_ld, double* __restrict__ x1) {
    const int k = blockIdx.y;
    uint32_t h;
    if (!row_h(L, 1, h)) return;
    x1[(size_t)k * L.ld + h] = (L.M1[h] & kDomainBit) ? full[(size_t)k * full_ld + state_of(h, 1)] : 0.0;
}

__global__ void k_zero_rows(Layout L, int parity, double* __restrict__ x) {
    const int k = blockIdx.y;
    uint32_t h;
    if (!row_h(L, parity, h)) return;
    x[(size_t)k * L.ld + h] = 0.0;
}

bool debug_enabled() {
    static const bool on = getenv("ESL_DEBUG") != nullptr;
    return on;
}

template <class T>
struct InnerVecs {
    T *r, *r0, *ph, *v, *sh, *t, *d, *w;
};

inline dim3 grid2(uint32_t H, int K) { return dim3((H + kT - 1) / kT, (unsigned)K); }
inline dim3 grid_rows(const Layout& L, int parity, int K) {
    uint32_t rows = (parity ? L.list1 : L.list0) ? (parity ? L.n1 : L.n0) : L.H;
    return dim3((std::max(rows, 1u) + kT - 1) / kT, (unsigned)K);
}

// Algorithmic bytes of one Schur-operator application (k_elim + k_apply) over K
// systems: every array once -- elim reads x (odd) and writes w (even); apply reads
// x, w, r0 and writes y (odd); the four mask words per half index are shared by
// all systems.
double schur_bytes(const Layout& L, int K, size_t tsz) {
    const double n0 = L.list0 ? L.n0 : L.H, n1 = L.list1 ? L.n1 : L.H;
    return (double)K * tsz * (2.0 * n0 + 4.0 * n1) + 8.0 * (n0 + n1);
}

template <bool FWD, class T>
int inner_bicgstab(esl_ctx* ctx, Layout L, const double* rates, int K, const double* dS, const double* r64,
                   KState* st, int* n_active, int32_t* act, InnerVecs<T> iv, int max_iters, int* iters_out) {
    cudaStream_t s = ctx->stream;
    unsigned sb = (unsigned)((K + 127) / 128);
    L.act = nullptr;
    ESL_COUNT_LAUNCH();
    k_inner_start<T><<<grid_rows(L, 1, K), kT, 0, s>>>(L, r64, iv.r, iv.r0, iv.d, iv.ph, iv.v, st);
    int it = 0;
    const int check_every = 8;
    while (it < max_iters) {
        // launch only over the systems still running
        ESL_CUDA(cudaMemsetAsync(n_active, 0, sizeof(int), s));
        ESL_COUNT_LAUNCH();
        k_active_list<<<sb, 128, 0, s>>>(K, st, n_active, act);
        int active = 0;
        ESL_CUDA(cudaMemcpyAsync(&active, n_active, sizeof(int), cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        if (active == 0) break;
        L.act = act;
        const dim3 g0 = grid_rows(L, 0, active), g1 = grid_rows(L, 1, active);
        for (int c = 0; c < check_every; c++, it++) {
            ESL_COUNT_LAUNCH();
            k_update_p<T><<<g1, kT, 0, s>>>(L, dS, iv.r, iv.ph, iv.v, st);
            cudaEvent_t ea = nullptr, eb = nullptr;
            if (ctx->prof) {
                ea = ctx->prof_event();
                eb = ctx->prof_event();
                cudaEventRecord(ea, s);
            }
            ESL_COUNT_LAUNCH();
            k_elim<FWD, T, T><<<g0, kT, 0, s>>>(L, rates, iv.ph, nullptr, iv.w, st);
            ESL_COUNT_LAUNCH();
            k_apply<FWD, 0, T, T><<<g1, kT, 0, s>>>(L, rates, iv.ph, iv.w, dS, nullptr, iv.r0, iv.v, st);
            if (ctx->prof) {
                cudaEventRecord(eb, s);
                ctx->prof_recs.push_back({ea, eb, schur_bytes(L, active, sizeof(T)), "schur_operator_whole_system"});
            }
            ESL_COUNT_LAUNCH();
            k_scal_alpha<<<sb, 128, 0, s>>>(K, st);
            ESL_COUNT_LAUNCH();
            k_update_s<T><<<g1, kT, 0, s>>>(L, dS, iv.r, iv.v, iv.sh, st);
            ESL_COUNT_LAUNCH();
            k_elim<FWD, T, T><<<g0, kT, 0, s>>>(L, rates, iv.sh, nullptr, iv.w, st);
            ESL_COUNT_LAUNCH();
            k_apply<FWD, 2, T, T><<<g1, kT, 0, s>>>(L, rates, iv.sh, iv.w, dS, nullptr, nullptr, iv.t, st);
            ESL_COUNT_LAUNCH();
            k_scal_omega<<<sb, 128, 0, s>>>(K, st);
            ESL_COUNT_LAUNCH();
            k_update_xr<T><<<g1, kT, 0, s>>>(L, dS, iv.d, iv.r, iv.r0, iv.ph, iv.sh, iv.t, st);
            ESL_COUNT_LAUNCH();
            k_scal_beta<<<sb, 128, 0, s>>>(K, st, max_iters);
        }
        ESL_CUDA(cudaGetLastError());
    }
    *iters_out = it;
    return ESL_OK;
}

}  // namespace

void free_workspace(void* w) { delete static_cast<Workspace*>(w); }

namespace {

enum Slot {
    S_BE, S_BS, S_DS, S_X64, S_R64, S_W64, S_ZE, S_ST, S_ACT,
    S_R, S_R0, S_PH, S_V, S_SH, S_T, S_D, S_W,
    S_M0, S_M1, S_F0, S_F1, S_RB, S_Y, S_SUM, S_BIG, S_PIN, S_BO, S_LIST, S_XT, S_RT, S_ACTLIST, S_ZEF, S_ZOF, S_ZEB, S_ZOB, S_RSUB, S_XSUB, S_LUOFF, S_LUSYS, S_LU, S_COUNT
};

struct SolveOut {
    int iters = 0, refinements = 0;
    double relres = 0.0;
    bool converged = true;
    std::vector<double> sys_relres;  // per system, from the last Krylov solve
    int fallback_systems = 0;        // systems the level sweep handed to the block forward solve
    int dense_systems = 0;           // (system, level group) pairs solved by the dense LU fallback
    bool absorption_by_sweep = false;  // L came from forward sweeps after the backward solve missed
};

void fill_report(esl_report* rep, const SolveOut& agg, bool converged) {
    if (!rep) return;
    rep->iterations = agg.iters;
    rep->refinements = agg.refinements;
    rep->relres = agg.relres;
    rep->converged = converged ? 1 : 0;
    rep->fallback_systems = agg.fallback_systems;
    rep->dense_lu_systems = agg.dense_systems;
    rep->absorption_by_sweep = agg.absorption_by_sweep ? 1 : 0;
}

// Solves the K systems whose rhs halves are in (bE, bO); solution in x64 (odd) and zE (even).
template <bool FWD>
int krylov_solve(esl_ctx* ctx, Workspace& ws, const Layout& L, const double* rates, int K, double* bE, double* bO,
                 const double* warm, size_t warm_ld, const esl_solve_opts& o, double*& x64_out, double*& zE_out,
                 SolveOut& out) {
    cudaStream_t s = ctx->stream;
    int st_ = ESL_OK;
    const size_t vec = (size_t)K * L.ld;
    double* dS = (double*)ws.get(S_DS, vec * 8, &st_);
    double* bS = (double*)ws.get(S_BS, vec * 8, &st_);
    double* x64 = (double*)ws.get(S_X64, vec * 8, &st_);
    double* r64 = (double*)ws.get(S_R64, vec * 8, &st_);
    double* w64 = (double*)ws.get(S_W64, vec * 8, &st_);
    double* zE = (double*)ws.get(S_ZE, vec * 8, &st_);
    KState* st = (KState*)ws.get(S_ST, (size_t)K * sizeof(KState), &st_);
    int* n_active = (int*)ws.get(S_ACT, 2 * sizeof(int), &st_);
    int32_t* act = (int32_t*)ws.get(S_ACTLIST, (size_t)K * sizeof(int32_t), &st_);
    const bool mixed = o.method == ESL_METHOD_MIXED;
    // sized for FP64 elements even in mixed mode: a mixed solve may continue with
    // FP64 inner iterations on the same buffers
    void* iv_p[8];
    for (int j = 0; j < 8; j++) iv_p[j] = ws.get(S_R + j, vec * sizeof(double), &st_);
    if (st_ != ESL_OK) return st_;
    const dim3 g0 = grid_rows(L, 0, K), g1 = grid_rows(L, 1, K);
    unsigned sb = (unsigned)((K + 127) / 128);
    ESL_CUDA(cudaMemsetAsync(st, 0, (size_t)K * sizeof(KState), s));
    ESL_COUNT_LAUNCH();
    k_schur_diag<FWD><<<g1, kT, 0, s>>>(L, rates, dS);
    // reduced rhs: bS = bO + A_oe (bE / q_e)
    ESL_COUNT_LAUNCH();
    k_elim<FWD, double, double><<<g0, kT, 0, s>>>(L, rates, (const double*)nullptr, bE, w64, nullptr);
    ESL_COUNT_LAUNCH();
    k_apply<FWD, 4, double, double><<<g1, kT, 0, s>>>(L, rates, (const double*)nullptr, w64, dS, bO, nullptr, bS,
                                                      nullptr);
    ESL_COUNT_LAUNCH();
    k_norm2<<<g1, kT, 0, s>>>(L, bS, st);
    if (warm) {
        ESL_COUNT_LAUNCH();
        k_half_from_full<<<g1, kT, 0, s>>>(L, warm, warm_ld, x64);
    } else {
        ESL_COUNT_LAUNCH();
        k_zero_rows<<<g1, kT, 0, s>>>(L, 1, x64);
    }
    ESL_CUDA(cudaGetLastError());
    const double tol = o.tol > 0 ? o.tol : 1e-10;
    // FP32 inner solves stop at 1e-4 relative: below that the FP32 operator's
    // rounding (cancellation between the diagonal and the neighbour flow) dominates
    const double floor_rel = mixed ? 1e-4 : 1e-13;
    int total_iters = 0, outer = 0;
    int active = 0;
    bool inner64 = !mixed;
    double* xt = (double*)ws.get(S_XT, vec * 8, &st_);
    double* rt = (double*)ws.get(S_RT, vec * 8, &st_);
    if (st_ != ESL_OK) return st_;
    // true residual of the starting iterate
    ESL_COUNT_LAUNCH();
    k_zero_r<<<sb, 128, 0, s>>>(K, st);
    ESL_COUNT_LAUNCH();
    k_elim<FWD, double, double><<<g0, kT, 0, s>>>(L, rates, x64, nullptr, w64, nullptr);
    ESL_COUNT_LAUNCH();
    k_apply<FWD, 3, double, double><<<g1, kT, 0, s>>>(L, rates, x64, w64, dS, bS, nullptr, r64, st);
    for (;; outer++) {
        ESL_CUDA(cudaMemsetAsync(n_active, 0, 2 * sizeof(int), s));
        // inner target: a relative reduction that reaches tol in one inner solve,
        // but not below what the inner precision can deliver
        const double floor_now = inner64 ? 1e-13 : floor_rel;
        ESL_COUNT_LAUNCH();
        k_outer_check<<<sb, 128, 0, s>>>(K, st, tol * tol, floor_now * floor_now, outer, o.max_iters, n_active);
        ESL_CUDA(cudaGetLastError());
        ESL_CUDA(cudaMemcpyAsync(&active, n_active, sizeof(int), cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        if (debug_enabled()) {
            std::vector<KState> h_st(K);
            ESL_CUDA(cudaMemcpy(h_st.data(), st, (size_t)K * sizeof(KState), cudaMemcpyDeviceToHost));
            int shown = 0;
            for (int k = 0; k < K && shown < 6; k++) {
                double rel = h_st[k].bnorm2 > 0 ? std::sqrt(h_st[k].rnorm2_true / h_st[k].bnorm2) : 0.0;
                if (k >= 2 && rel <= tol) continue;
                shown++;
                fprintf(stderr,
                        "[esl] outer %d sys %d/%d relres %.3e b2 %.3e inner64 %d last inner: breakdown %d iters %d "
                        "r0v %.3e rr %.3e\n",
                        outer, k, K, rel, h_st[k].bnorm2, (int)inner64, h_st[k].last_breakdown, h_st[k].last_iters,
                        h_st[k].last_r0v, h_st[k].last_rr);
            }
        }
        if (active == 0 || outer >= o.max_refine) break;
        ESL_COUNT_LAUNCH();
        k_mark_inner<<<sb, 128, 0, s>>>(K, st);
        int it = 0;
        ESL_COUNT_LAUNCH();
        k_zero_trial<<<sb, 128, 0, s>>>(K, st);
        if (!inner64) {
            InnerVecs<float> iv{(float*)iv_p[0], (float*)iv_p[1], (float*)iv_p[2], (float*)iv_p[3],
                                (float*)iv_p[4], (float*)iv_p[5], (float*)iv_p[6], (float*)iv_p[7]};
            ESL_TRY((inner_bicgstab<FWD, float>(ctx, L, rates, K, dS, r64, st, n_active, act, iv, o.max_iters, &it)));
            ESL_COUNT_LAUNCH();
            k_trial<float><<<g1, kT, 0, s>>>(L, x64, iv.d, xt, st);
        } else {
            InnerVecs<double> iv{(double*)iv_p[0], (double*)iv_p[1], (double*)iv_p[2], (double*)iv_p[3],
                                 (double*)iv_p[4], (double*)iv_p[5], (double*)iv_p[6], (double*)iv_p[7]};
            ESL_TRY((inner_bicgstab<FWD, double>(ctx, L, rates, K, dS, r64, st, n_active, act, iv, o.max_iters, &it)));
            ESL_COUNT_LAUNCH();
            k_trial<double><<<g1, kT, 0, s>>>(L, x64, iv.d, xt, st);
        }
        total_iters += it;
        // true residual of the trial iterate; commit where it improved
        ESL_COUNT_LAUNCH();
        k_elim<FWD, double, double><<<g0, kT, 0, s>>>(L, rates, xt, nullptr, w64, nullptr);
        ESL_COUNT_LAUNCH();
        k_apply<FWD, 5, double, double><<<g1, kT, 0, s>>>(L, rates, xt, w64, dS, bS, nullptr, rt, st);
        ESL_CUDA(cudaMemsetAsync(n_active + 1, 0, sizeof(int), s));
        ESL_COUNT_LAUNCH();
        k_commit_flags<<<sb, 128, 0, s>>>(K, st, n_active + 1);
        ESL_COUNT_LAUNCH();
        k_commit<<<g1, kT, 0, s>>>(L, x64, r64, xt, rt, st);
        ESL_CUDA(cudaGetLastError());
        int noimp = 0;
        ESL_CUDA(cudaMemcpyAsync(&noimp, n_active + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        ESL_CUDA(cudaStreamSynchronize(s));
        // an FP32 correction that did not help: continue in FP64
        if (noimp > 0 && !inner64) inner64 = true;
    }
    // even half: zE = (bE + A_eo x) / q_e
    ESL_COUNT_LAUNCH();
    k_elim<FWD, double, double><<<g0, kT, 0, s>>>(L, rates, x64, bE, zE, nullptr);
    ESL_CUDA(cudaGetLastError());
    std::vector<KState> h_st(K);
    ESL_CUDA(cudaMemcpyAsync(h_st.data(), st, (size_t)K * sizeof(KState), cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    double worst = 0.0;
    out.sys_relres.assign(K, 0.0);
    for (int k = 0; k < K; k++)
        if (h_st[k].bnorm2 > 0) {
            out.sys_relres[k] = std::sqrt(h_st[k].rnorm2_true / h_st[k].bnorm2);
            worst = std::max(worst, out.sys_relres[k]);
        }
    if (debug_enabled()) {
        std::vector<int> its;
        long long sum = 0;
        for (auto& k : h_st) {
            its.push_back(k.total_iters);
            sum += k.total_iters;
        }
        std::sort(its.begin(), its.end());
        fprintf(stderr, "[esl] K=%d inner iterations per system: mean %.1f min %d p50 %d p90 %d p99 %d max %d\n", K,
                (double)sum / K, its.front(), its[K / 2], its[(K * 9) / 10], its[(K * 99) / 100], its.back());
        for (int k = 0; k < K; k++)
            if (h_st[k].total_iters > 1000)
                fprintf(stderr, "[esl]   hard system %d iterations %d relres %.3e\n", k, h_st[k].total_iters,
                        h_st[k].bnorm2 > 0 ? std::sqrt(h_st[k].rnorm2_true / h_st[k].bnorm2) : 0.0);
    }
    out.iters = total_iters;
    out.refinements = outer;
    out.relres = worst;
    // residual-based: a system that ran out of budget is done but not converged
    out.converged = worst <= kAcceptRel;
    x64_out = x64;
    zE_out = zE;
    if (!out.converged)
    {
        char msg[160];
        snprintf(msg, sizeof msg, "relative residual %.3e above tolerance after %d refinement steps", worst, outer);
        return fail(ESL_ERR_NOT_CONVERGED, msg);
    }
    return ESL_OK;
}


// ---- block forward solve over SCC levels --------------------------------------------------
// The transient part is block lower-triangular in topological order: the SCCs of
// one level depend only on SCCs of higher levels (sources come first), never on
// each other.  Levels are solved in order; a level of singleton SCCs is a direct
// division, any other level a Krylov solve restricted to its states (block-diagonal
// over its SCCs).  This is the reference's block-triangular structure
// (cuda/src/linear_system_solve.cu:249-325) with the per-block LU replaced by
// direct/Krylov solves, and it is exact in the inter-block coupling.
struct BlockPlan {
    std::vector<uint32_t> off0, off1;  // group offsets into list0 / list1
    std::vector<int> max_scc;          // largest SCC of each group
    DevBuf<uint32_t> list0, list1;     // half indices of each group's even / odd states
    DevBuf<uint32_t> hm;               // half-layout masks: M0, M1 (same-SCC in-edges | domain), F0, F1
    DevBuf<uint32_t> Gx;               // per state: in-edges from other transient SCCs
    // SCCs of each group up to kDenseFallbackMax states (first position in `order`, size), for the LU fallback
    std::vector<uint32_t> off_scc;
    std::vector<int64_t> lu_doubles;   // dense scratch of one system for each group
    DevBuf<int32_t> scc_beg, scc_size;
};

void free_plan(void* p) { delete static_cast<BlockPlan*>(p); }

__global__ void k_scc_masks(int n, uint64_t N, const uint32_t* __restrict__ F, const uint32_t* __restrict__ G,
                            const int32_t* __restrict__ lab, const int32_t* __restrict__ term_of,
                            uint32_t* __restrict__ Gx, uint32_t* __restrict__ hm, uint32_t H) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const bool transient = term_of[v] < 0;
    uint32_t g = G[v], same = 0, cross = 0;
    const int32_t c = lab[v];
    while (g) {
        int i = __ffs(g) - 1;
        g &= g - 1;
        uint64_t u = v ^ (1ull << i);
        if (term_of[u] >= 0) continue;
        if (lab[u] == c) same |= 1u << i;
        else cross |= 1u << i;
    }
    Gx[v] = transient ? cross : 0u;
    const uint32_t h = (uint32_t)(v >> 1);
    const int par = __popcll(v) & 1;
    hm[(size_t)par * H + h] = transient ? (same | kDomainBit) : 0u;
    hm[(size_t)(2 + par) * H + h] = F[v];
}

// Dense LU fallback for transient SCC blocks (forward form), one CTA per (SCC, system):
// rows = equations of the SCC's states, A[a][a] = out-rate, A[a][b] = -rate(b -> a) for
// edges inside the SCC, rhs = the group rhs already formed in bE / bO.  Gaussian
// elimination with partial pivoting in a global scratch matrix (s x (s+1), row-major).
__global__ void __launch_bounds__(256) k_dense_block(int n, const int32_t* __restrict__ scc_beg,
                                                     const int32_t* __restrict__ scc_size,
                                                     const int64_t* __restrict__ scc_scratch,
                                                     const int32_t* __restrict__ sys, int64_t sys_stride,
                                                     const int32_t* __restrict__ order,
                                                     const uint32_t* __restrict__ F, const uint32_t* __restrict__ G,
                                                     const double* __restrict__ rates, int nrhs, size_t ld,
                                                     const double* __restrict__ bE, const double* __restrict__ bO,
                                                     double* __restrict__ ZE, double* __restrict__ ZO,
                                                     double* __restrict__ scratch) {
    __shared__ double s_rate[64];
    __shared__ int s_piv;
    __shared__ double s_red[32];
    __shared__ int s_redi[32];
    const int j = blockIdx.x;
    const int k = sys[blockIdx.y];
    const int beg = scc_beg[j], sz = scc_size[j];
    const int ldA = sz + 1;
    double* A = scratch + (size_t)blockIdx.y * sys_stride + scc_scratch[j];
    const int32_t* mem = order + beg;
    load_rates(s_rate, rates, k / nrhs, n);
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)sz * ldA; e += blockDim.x) A[e] = 0.0;
    __syncthreads();
    for (int a = threadIdx.x; a < sz; a += blockDim.x) {
        const uint32_t v = (uint32_t)mem[a];
        A[(size_t)a * ldA + a] = out_rate(s_rate, F[v], v);
        uint32_t g = G[v];
        while (g) {
            int i = __ffs(g) - 1;
            g &= g - 1;
            const int32_t u = (int32_t)(v ^ (1u << i));
            int lo = 0, hi = sz - 1;  // members ascending
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (mem[mid] < u) lo = mid + 1; else hi = mid;
            }
            if (mem[lo] == u) A[(size_t)a * ldA + lo] -= s_rate[2 * i + (((uint32_t)u >> i) & 1u)];
        }
        const size_t o = (size_t)k * ld + (v >> 1);
        A[(size_t)a * ldA + sz] = (__popc(v) & 1) ? bO[o] : bE[o];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int col = 0; col < sz; col++) {
        double best = -1.0;
        int bi = col;
        for (int r = col + threadIdx.x; r < sz; r += blockDim.x) {
            double a = fabs(A[(size_t)r * ldA + col]);
            if (a > best) { best = a; bi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
            int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (lane == 0) { s_red[warp] = best; s_redi[warp] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double b0 = s_red[0];
            int i0 = s_redi[0];
            for (int w = 1; w < nw; w++)
                if (s_red[w] > b0 || (s_red[w] == b0 && s_redi[w] < i0)) { b0 = s_red[w]; i0 = s_redi[w]; }
            s_piv = i0;
        }
        __syncthreads();
        const int piv = s_piv;
        if (piv != col)
            for (int c = col + threadIdx.x; c <= sz; c += blockDim.x) {
                double t = A[(size_t)col * ldA + c];
                A[(size_t)col * ldA + c] = A[(size_t)piv * ldA + c];
                A[(size_t)piv * ldA + c] = t;
            }
        __syncthreads();
        const double inv = 1.0 / A[(size_t)col * ldA + col];
        const int rows = sz - col - 1, cols = sz - col;
        for (int64_t e = threadIdx.x; e < (int64_t)rows * cols; e += blockDim.x) {
            const int r = col + 1 + (int)(e / cols), c = col + 1 + (int)(e % cols);
            A[(size_t)r * ldA + c] -= A[(size_t)r * ldA + col] * inv * A[(size_t)col * ldA + c];
        }
        __syncthreads();
    }
    if (warp == 0) {
        for (int r = sz - 1; r >= 0; r--) {
            double acc = 0.0;
            for (int c = r + 1 + lane; c < sz; c += 32) acc += A[(size_t)r * ldA + c] * A[(size_t)c * ldA + sz];
            acc = warp_sum(acc);
            if (lane == 0) A[(size_t)r * ldA + sz] = (A[(size_t)r * ldA + sz] - acc) / A[(size_t)r * ldA + r];
            __syncwarp();
        }
    }
    __syncthreads();
    for (int a = threadIdx.x; a < sz; a += blockDim.x) {
        const uint32_t v = (uint32_t)mem[a];
        const size_t o = (size_t)k * ld + (v >> 1);
        ((__popc(v) & 1) ? ZO : ZE)[o] = A[(size_t)a * ldA + sz];
    }
}

int get_plan(esl_ctx* ctx, const esl_net* net, BlockPlan*& out) {
    // one builder at a time, so that threads solving the same network share one plan
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (net->plan) {
        out = static_cast<BlockPlan*>(net->plan);
        return ESL_OK;
    }
    cudaStream_t s = ctx->stream;
    const size_t N = (size_t)net->N;
    const uint32_t H = (uint32_t)(N / 2);
    auto* P = new BlockPlan();
    std::vector<int32_t> order(N), offsets(net->n_sccs + 1), levels(net->n_sccs);
    int rc = ESL_OK;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == ESL_OK) rc = fail(ESL_ERR_CUDA, cudaGetErrorString(e));
    };
    chk(cudaMemcpyAsync(order.data(), net->order.get(), N * 4, cudaMemcpyDeviceToHost, s));
    chk(cudaMemcpyAsync(offsets.data(), net->offsets.get(), offsets.size() * 4, cudaMemcpyDeviceToHost, s));
    chk(cudaMemcpyAsync(levels.data(), net->levels.get(), levels.size() * 4, cudaMemcpyDeviceToHost, s));
    chk(cudaStreamSynchronize(s));
    if (rc != ESL_OK) {
        delete P;
        return rc;
    }
    std::vector<uint32_t> l0, l1;
    std::vector<int32_t> sb, ss;
    P->off0.push_back(0);
    P->off1.push_back(0);
    P->off_scc.push_back(0);
    for (int c = net->T; c < net->n_sccs;) {
        int c1 = c, mx = 0;
        int64_t lu = 0;
        while (c1 < net->n_sccs && levels[c1] == levels[c]) {
            const int sz = offsets[c1 + 1] - offsets[c1];
            mx = std::max(mx, sz);
            if (sz <= kDenseFallbackMax) {  // singletons too: a failed Krylov iterate is redone everywhere
                sb.push_back(offsets[c1]);
                ss.push_back(sz);
                lu += (int64_t)sz * (sz + 1);
            }
            for (int p = offsets[c1]; p < offsets[c1 + 1]; p++) {
                uint32_t v = (uint32_t)order[p];
                (__builtin_popcount(v) & 1 ? l1 : l0).push_back(v >> 1);
            }
            c1++;
        }
        P->off0.push_back((uint32_t)l0.size());
        P->off1.push_back((uint32_t)l1.size());
        P->off_scc.push_back((uint32_t)sb.size());
        P->lu_doubles.push_back(lu);
        P->max_scc.push_back(mx);
        c = c1;
    }
    rc = P->list0.alloc(l0.size());
    if (rc == ESL_OK) rc = P->scc_beg.alloc(sb.size());
    if (rc == ESL_OK) rc = P->scc_size.alloc(ss.size());
    if (rc == ESL_OK && !sb.empty()) {
        chk(cudaMemcpyAsync(P->scc_beg.get(), sb.data(), sb.size() * 4, cudaMemcpyHostToDevice, s));
        chk(cudaMemcpyAsync(P->scc_size.get(), ss.data(), ss.size() * 4, cudaMemcpyHostToDevice, s));
    }
    if (rc == ESL_OK) rc = P->list1.alloc(l1.size());
    if (rc == ESL_OK) rc = P->hm.alloc((size_t)4 * H);
    if (rc == ESL_OK) rc = P->Gx.alloc(N);
    if (rc == ESL_OK) {
        if (!l0.empty()) chk(cudaMemcpyAsync(P->list0.get(), l0.data(), l0.size() * 4, cudaMemcpyHostToDevice, s));
        if (!l1.empty()) chk(cudaMemcpyAsync(P->list1.get(), l1.data(), l1.size() * 4, cudaMemcpyHostToDevice, s));
        ESL_COUNT_LAUNCH();
        k_scc_masks<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(net->n, N, net->F.get(), net->G.get(),
                                                                net->labels.get(), net->term_of.get(), P->Gx.get(),
                                                                P->hm.get(), H);
        chk(cudaGetLastError());
        chk(cudaStreamSynchronize(s));
    }
    if (rc != ESL_OK) {
        delete P;
        return rc;
    }
    esl_net* mnet = const_cast<esl_net*>(net);
    mnet->plan = P;
    mnet->plan_free = free_plan;
    out = P;
    return ESL_OK;
}

// rhs of one level group: b_v = x0(v) + inflow from already solved transient states;
// `direct` groups (singleton SCCs only) store z_v = b_v / q_v immediately.
__global__ void __launch_bounds__(kT) k_group_rhs(Layout L, int parity, const double* __restrict__ rates,
                                                  const double* __restrict__ x0, size_t x0_ld,
                                                  const uint32_t* __restrict__ Gx, const double* __restrict__ ZE,
                                                  const double* __restrict__ ZO, double* __restrict__ b, int direct,
                                                  double* __restrict__ Zout) {
    __shared__ double s_rate[64];
    const int k = blockIdx.y;
    load_rates(s_rate, rates, k / L.nrhs, L.n);
    __syncthreads();
    uint32_t h;
    if (!row_h(L, parity, h)) return;
    const uint32_t v = state_of(h, parity);
    const size_t o = (size_t)k * L.ld;
    double acc = x0[(size_t)(L.x0_sys ? k : k % L.nrhs) * x0_ld + v];
    uint32_t g = Gx[v];
    while (g) {
        int i = __ffs(g) - 1;
        g &= g - 1;
        uint32_t u = v ^ (1u << i);
        // u has the other parity; its half index is u >> 1
        const double zu = (parity ? ZE : ZO)[o + (u >> 1)];
        acc += s_rate[2 * i + ((u >> i) & 1u)] * zu;
    }
    if (direct) {
        const uint32_t* Fh = parity ? L.F1 : L.F0;
        Zout[o + h] = acc / out_rate(s_rate, Fh[h], v);
    } else {
        b[o + h] = acc;
    }
}

__global__ void k_group_store(Layout L, int parity, const double* __restrict__ src, double* __restrict__ dst) {
    const int k = blockIdx.y;
    uint32_t h;
    if (!row_h(L, parity, h)) return;
    dst[(size_t)k * L.ld + h] = src[(size_t)k * L.ld + h];
}

// dst row idx[j] = src row j (rows of `width` doubles)
__global__ void k_set_rows(int width, const int32_t* __restrict__ idx, const double* __restrict__ src,
                           double* __restrict__ dst) {
    const int j = blockIdx.y;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < width) dst[(size_t)idx[j] * width + c] = src[(size_t)j * width + c];
}

// copy system rows j -> idx[j] (K' systems) between half-layout arrays
__global__ void k_scatter_systems(size_t ld, const int32_t* __restrict__ idx, const double* __restrict__ src,
                                  double* __restrict__ dst) {
    const int j = blockIdx.y;
    size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= ld) return;
    dst[(size_t)idx[j] * ld + h] = src[(size_t)j * ld + h];
}

// Block forward solve of K systems (rate set k / nrhs, x0 row k % nrhs); results in
// the half-layout arrays ZE (even) and ZO (odd).
// x0_per_system: x0 holds one row per system (a gathered subset) instead of nrhs rows.
int block_forward_solve(esl_ctx* ctx, Workspace& ws, const esl_net* net, int K, int nrhs, const double* rates,
                        const double* x0, size_t x0_ld, double* ZE, double* ZO, const esl_solve_opts& o,
                        SolveOut& out, bool x0_per_system = false) {
    cudaStream_t s = ctx->stream;
    BlockPlan* P = nullptr;
    ESL_TRY(get_plan(ctx, net, P));
    const uint32_t H = (uint32_t)(net->N / 2);
    Layout L;
    L.n = net->n;
    L.H = H;
    L.ld = ((size_t)H + 31) & ~(size_t)31;
    L.nrhs = nrhs;
    L.x0_sys = x0_per_system ? 1 : 0;
    L.M0 = P->hm.get();
    L.M1 = P->hm.get() + H;
    L.F0 = P->hm.get() + 2 * (size_t)H;
    L.F1 = P->hm.get() + 3 * (size_t)H;
    L.pins = nullptr;
    L.term_of = nullptr;
    L.T = 0;
    L.act = nullptr;
    int st_ = ESL_OK;
    const size_t vec = (size_t)K * L.ld;
    double* bE = (double*)ws.get(S_BE, vec * 8, &st_);
    double* bO = (double*)ws.get(S_BO, vec * 8, &st_);
    if (st_ != ESL_OK) return st_;
    esl_solve_opts go = o;
    go.method = ESL_METHOD_FP64;
    go.d_warm = nullptr;
    const int G = (int)P->max_scc.size();
    for (int gi = 0; gi < G; gi++) {
        L.list0 = P->list0.get() + P->off0[gi];
        L.list1 = P->list1.get() + P->off1[gi];
        L.n0 = P->off0[gi + 1] - P->off0[gi];
        L.n1 = P->off1[gi + 1] - P->off1[gi];
        const int direct = P->max_scc[gi] == 1;
        if (L.n0) {
            ESL_COUNT_LAUNCH();
            k_group_rhs<<<grid_rows(L, 0, K), kT, 0, s>>>(L, 0, rates, x0, x0_ld, P->Gx.get(), ZE, ZO, bE, direct,
                                                          ZE);
        }
        if (L.n1) {
            ESL_COUNT_LAUNCH();
            k_group_rhs<<<grid_rows(L, 1, K), kT, 0, s>>>(L, 1, rates, x0, x0_ld, P->Gx.get(), ZE, ZO, bO, direct,
                                                          ZO);
        }
        ESL_CUDA(cudaGetLastError());
        if (direct) continue;
        double *x64 = nullptr, *zE = nullptr;
        SolveOut so;
        int rc = krylov_solve<true>(ctx, ws, L, rates, K, bE, bO, nullptr, 0, go, x64, zE, so);
        if (debug_enabled())
            fprintf(stderr, "[esl] group %d/%d even %u odd %u max_scc %d: rc %d iters %d relres %.3e\n", gi, G, L.n0,
                    L.n1, P->max_scc[gi], rc, so.iters, so.relres);
        out.iters += so.iters;
        if (rc != ESL_OK && rc != ESL_ERR_NOT_CONVERGED) return rc;
        if (L.n0) { ESL_COUNT_LAUNCH(); k_group_store<<<grid_rows(L, 0, K), kT, 0, s>>>(L, 0, zE, ZE); }
        if (L.n1) { ESL_COUNT_LAUNCH(); k_group_store<<<grid_rows(L, 1, K), kT, 0, s>>>(L, 1, x64, ZO); }
        ESL_CUDA(cudaGetLastError());
        double worst = 0.0;
        if (rc == ESL_ERR_NOT_CONVERGED) {
            // LU fallback for the systems that missed the budget
            std::vector<int32_t> failed;
            for (int k = 0; k < K; k++)
                if (so.sys_relres[k] > kAcceptRel) failed.push_back(k);
                else worst = std::max(worst, so.sys_relres[k]);
            const int nscc = (int)(P->off_scc[gi + 1] - P->off_scc[gi]);
            const bool covered = P->max_scc[gi] <= dense_cap(ctx);
            if (!covered || nscc == 0) {
                out.converged = false;
                worst = so.relres;
            } else {
                const int Kf = (int)failed.size();
                std::vector<int64_t> scr(nscc);
                int64_t acc = 0;
                for (int jj = 0; jj < nscc; jj++) {
                    scr[jj] = acc;
                    int64_t sz = 0;
                    ESL_CUDA(cudaMemcpyAsync(&sz, P->scc_size.get() + P->off_scc[gi] + jj, 4, cudaMemcpyDeviceToHost, s));
                    ESL_CUDA(cudaStreamSynchronize(s));
                    acc += sz * (sz + 1);
                }
                // systems in chunks whose matrices fit the scratch budget
                const int chunk = (int)std::max<int64_t>(
                    1, std::min<int64_t>(Kf, (int64_t)(kDenseScratchBytes / (8 * (size_t)std::max<int64_t>(acc, 1)))));
                int64_t* d_scr = (int64_t*)ws.get(S_LUOFF, (size_t)nscc * 8, &st_);
                int32_t* d_sys = (int32_t*)ws.get(S_LUSYS, (size_t)Kf * 4, &st_);
                double* scratch = (double*)ws.get(S_LU, (size_t)acc * chunk * 8, &st_);
                if (st_ != ESL_OK) return st_;
                ESL_CUDA(cudaMemcpyAsync(d_scr, scr.data(), (size_t)nscc * 8, cudaMemcpyHostToDevice, s));
                ESL_CUDA(cudaMemcpyAsync(d_sys, failed.data(), (size_t)Kf * 4, cudaMemcpyHostToDevice, s));
                out.dense_systems += Kf;
                for (int c0 = 0; c0 < Kf; c0 += chunk) {
                    const int kc = std::min(chunk, Kf - c0);
                    ESL_COUNT_LAUNCH();
                    k_dense_block<<<dim3((unsigned)nscc, (unsigned)kc), 256, 0, s>>>(
                        net->n, P->scc_beg.get() + P->off_scc[gi], P->scc_size.get() + P->off_scc[gi], d_scr,
                        d_sys + c0, acc, net->order.get(), net->F.get(), net->G.get(), rates, nrhs, L.ld, bE, bO, ZE,
                        ZO, scratch);
                    ESL_CUDA(cudaGetLastError());
                }
                ESL_CUDA(cudaStreamSynchronize(s));
                if (debug_enabled())
                    fprintf(stderr, "[esl] group %d: dense LU fallback for %d systems on %d SCC blocks\n", gi, Kf, nscc);
            }
        } else {
            worst = so.relres;
        }
        out.relres = std::max(out.relres, worst);
    }
    if (!out.converged) {
        char msg[160];
        snprintf(msg, sizeof msg, "block solve: relative residual %.3e above tolerance", out.relres);
        return fail(ESL_ERR_NOT_CONVERGED, msg);
    }
    return ESL_OK;
}

int make_layout(esl_ctx* ctx, Workspace& ws, const esl_net* net, int dom, const uint8_t* big_term, bool fwd,
                Layout& L, int nrhs) {
    int st_ = ESL_OK;
    const uint32_t H = (uint32_t)(net->N / 2);
    uint32_t* M0 = (uint32_t*)ws.get(S_M0, (size_t)H * 4 * 4, &st_);
    if (st_ != ESL_OK) return st_;
    uint32_t* M1 = M0 + H;
    uint32_t* F0 = M0 + 2 * (size_t)H;
    uint32_t* F1 = M0 + 3 * (size_t)H;
    ESL_COUNT_LAUNCH();
    k_half_masks<<<(H + kT - 1) / kT, kT, 0, ctx->stream>>>(net->n, H, fwd ? net->Gdom.get() : net->Fdom.get(),
                                                           net->F.get(), net->term_of.get(), big_term, dom, M0, M1,
                                                           F0, F1);
    ESL_CUDA(cudaGetLastError());
    L.n = net->n;
    L.H = H;
    L.ld = ((size_t)H + 31) & ~(size_t)31;
    L.nrhs = nrhs;
    L.M0 = M0;
    L.M1 = M1;
    L.F0 = F0;
    L.F1 = F1;
    L.pins = nullptr;
    L.term_of = nullptr;
    L.T = 0;
    L.act = nullptr;
    L.list0 = L.list1 = nullptr;
    L.n0 = L.n1 = 0;
    return ESL_OK;
}

}  // namespace

// L (T x N) from forward solves: column s of L is the mass that each terminal SCC receives
// from a unit initial distribution at transient state s (the level sweep's terminal
// masses), solved for chunks of transient states at a time.  Terminal columns are
// L[t][v] = [v in t].  The fallback of the backward form.
__global__ void k_unit_rows(int c, size_t N, const int32_t* __restrict__ order, int64_t first,
                            double* __restrict__ x0) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < c) x0[(size_t)j * N + order[first + j]] = 1.0;
}

__global__ void k_L_columns(int c, int T, size_t N, const int32_t* __restrict__ order, int64_t first,
                            const double* __restrict__ y, double* __restrict__ Lm) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= c) return;
    const size_t v = (size_t)order[first + j];
    for (int t = 0; t < T; t++) Lm[(size_t)t * N + v] = y[(size_t)j * T + t];
}

__global__ void k_L_terminals(size_t N, int T, const int32_t* __restrict__ term_of, double* __restrict__ Lm) {
    const size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N || term_of[v] < 0) return;
    for (int t = 0; t < T; t++) Lm[(size_t)t * N + v] = term_of[v] == t ? 1.0 : 0.0;
}

int absorption_by_sweep(esl_ctx* ctx, Workspace& ws, const esl_net* net, const double* d_rates,
                        const esl_solve_opts& o, double* d_L) {
    cudaStream_t s = ctx->stream;
    const size_t N = (size_t)net->N;
    const int T = net->T;
    const int64_t TS = net->term_states, M = (int64_t)N - TS;
    // unit initial distributions of up to ~1 GB per chunk
    const int chunk = (int)std::max<int64_t>(32, std::min<int64_t>(4096, (int64_t)((1ull << 30) / (8 * N))));
    int st_ = ESL_OK;
    double* x0 = (double*)ws.get(S_XSUB, (size_t)chunk * N * 8, &st_);
    double* y = (double*)ws.get(S_SUM, (size_t)chunk * T * 8, &st_);
    if (st_ != ESL_OK) return st_;
    esl_solve_opts so = o;
    so.method = ESL_METHOD_DIRECT;
    so.d_warm = nullptr;
    so.d_occupation = nullptr;
    ESL_CUDA(cudaMemsetAsync(d_L, 0, (size_t)T * N * 8, s));
    for (int64_t first = 0; first < M; first += chunk) {
        const int c = (int)std::min<int64_t>(chunk, M - first);
        ESL_CUDA(cudaMemsetAsync(x0, 0, (size_t)c * N * 8, s));
        ESL_COUNT_LAUNCH();
        k_unit_rows<<<(c + 127) / 128, 128, 0, s>>>(c, N, net->order.get(), TS + first, x0);
        ESL_CUDA(cudaMemsetAsync(y, 0, (size_t)c * T * 8, s));
        SweepStats sw;
        ESL_TRY(sweep_forward(ctx, net, c, c, d_rates, x0, N, so, y, sw));
        ESL_COUNT_LAUNCH();
        k_L_columns<<<(c + 127) / 128, 128, 0, s>>>(c, T, N, net->order.get(), TS + first, y, d_L);
        ESL_CUDA(cudaGetLastError());
    }
    ESL_COUNT_LAUNCH();
    k_L_terminals<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(N, T, net->term_of.get(), d_L);
    ESL_CUDA(cudaGetLastError());
    return ESL_OK;
}

int solve_batch(esl_ctx* ctx, const esl_net* net, int B, const double* d_rates, int R, const double* d_x0,
                double* d_x_inf, double* d_marg, double* d_R, double* d_L, const esl_solve_opts* opts,
                esl_report* rep) {
    if (net->n < 1) return fail(ESL_ERR_INVALID, "network has no nodes");
    esl_solve_opts o;
    if (opts) o = *opts;
    else {
        o.method = ESL_METHOD_FP64;
        o.tol = 0;
        o.max_iters = 0;
        o.max_refine = 0;
        o.d_warm = nullptr;
        o.d_occupation = nullptr;
    }
    if (o.d_occupation && !((o.method == ESL_METHOD_DIRECT || o.method == ESL_METHOD_MIXED) && sweep_supported(net)))
        return fail(ESL_ERR_INVALID, "the occupation output needs ESL_METHOD_DIRECT or ESL_METHOD_MIXED and n <= 26");
    if (o.tol <= 0) o.tol = 1e-10;
    if (o.max_iters <= 0) o.max_iters = 600;
    if (o.max_refine <= 0) o.max_refine = 6;
    if (!ctx->work) ctx->work = new Workspace();
    Workspace& ws = *static_cast<Workspace*>(ctx->work);
    cudaStream_t s = ctx->stream;
    const size_t N = (size_t)net->N;
    const int T = net->T, TS = net->term_states, n = net->n;
    int st_ = ESL_OK;
    SolveOut agg;

    // ---- terminal kernels R_b (B x TS) ----
    double* Rb = (double*)ws.get(S_RB, (size_t)B * TS * 8, &st_);
    if (st_ != ESL_OK) return st_;
    {
        std::vector<int32_t> dense_list, big_list;
        for (int t = 0; t < T; t++) {
            int sz = net->h_offsets[t + 1] - net->h_offsets[t];
            if (sz >= 2 && sz <= kDenseTerm) dense_list.push_back(t);
            if (sz > kDenseTerm) big_list.push_back(t);
        }
        ESL_COUNT_LAUNCH();
        k_unit_terminals<<<dim3((T + 127) / 128, B), 128, 0, s>>>(T, net->offsets.get(), TS, Rb);
        ESL_CUDA(cudaGetLastError());
        if (!dense_list.empty()) {
            int32_t* d_list = (int32_t*)ws.get(S_LIST, dense_list.size() * 4, &st_);
            if (st_ != ESL_OK) return st_;
            ESL_CUDA(cudaMemcpyAsync(d_list, dense_list.data(), dense_list.size() * 4, cudaMemcpyHostToDevice, s));
            int smax = 0;
            for (int t : dense_list) smax = std::max(smax, net->h_offsets[t + 1] - net->h_offsets[t]);
            size_t smem = (size_t)smax * (smax + 1) * 8 + (size_t)smax * 4 + 16;
            ESL_CUDA(cudaFuncSetAttribute(k_dense_terminal, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            ESL_COUNT_LAUNCH();
            k_dense_terminal<<<dim3((unsigned)dense_list.size(), B), 256, smem, s>>>(
                n, d_list, net->offsets.get(), net->order.get(), net->F.get(), d_rates, TS, Rb);
            ESL_CUDA(cudaGetLastError());
            ESL_CUDA(cudaStreamSynchronize(s));  // d_list is reused below
        }
        if (!big_list.empty() && sweep_supported(net)) {
            // deflated FP64 Krylov on the odd-row Schur complement of each big terminal SCC
            SweepStats sw;
            const int rc = sweep_terminal(ctx, net, B, d_rates, o, Rb, sw);
            agg.iters += sw.iters;
            agg.relres = std::max(agg.relres, sw.relres);
            if (rc != ESL_OK) {
                if (rep) {
                    fill_report(rep, agg, false);
                }
                return rc;
            }
        } else if (!big_list.empty()) {
            // networks beyond the level sweep's 26 nodes: pin one high-mass state per
            // (big terminal SCC, rate set) and solve the rest with Krylov
            std::vector<uint8_t> h_big(T, 0);
            for (int t : big_list) h_big[t] = 1;
            uint8_t* d_big = (uint8_t*)ws.get(S_BIG, T, &st_);
            unsigned long long* d_best = (unsigned long long*)ws.get(S_PIN, (size_t)B * T * 8, &st_);
            int32_t* d_pins = (int32_t*)ws.get(S_LIST, (size_t)B * T * 4, &st_);
            if (st_ != ESL_OK) return st_;
            ESL_CUDA(cudaMemcpyAsync(d_big, h_big.data(), T, cudaMemcpyHostToDevice, s));
            ESL_CUDA(cudaMemsetAsync(d_best, 0, (size_t)B * T * 8, s));
            dim3 gt((TS + kT - 1) / kT, B);
            ESL_COUNT_LAUNCH();
            k_pin_score<<<gt, kT, 0, s>>>(n, T, TS, net->order.get(), net->term_of.get(), d_big, net->F.get(),
                                          net->G.get(), d_rates, d_best);
            ESL_COUNT_LAUNCH();
            k_pin_decode<<<(unsigned)((B * T + 255) / 256), 256, 0, s>>>(B * T, d_best, d_pins);
            ESL_CUDA(cudaGetLastError());
            Layout L;
            ESL_TRY(make_layout(ctx, ws, net, 1, d_big, true, L, 1));
            L.pins = d_pins;
            L.term_of = net->term_of.get();
            L.T = T;
            const size_t vec = (size_t)B * L.ld;
            double* bE = (double*)ws.get(S_BE, vec * 8, &st_);
            double* bO = (double*)ws.get(S_BO, vec * 8, &st_);
            double* sums = (double*)ws.get(S_SUM, (size_t)B * T * 8, &st_);
            if (st_ != ESL_OK) return st_;
            dim3 g = grid2(L.H, B);
            ESL_COUNT_LAUNCH();
            k_rhs_pinned<<<g, kT, 0, s>>>(L, d_rates, net->G.get(), bE, bO);
            ESL_CUDA(cudaGetLastError());
            // terminal kernels are solved in FP64 throughout: they can be badly
            // conditioned and their cost is small next to the transient part
            esl_solve_opts to = o;
            to.method = ESL_METHOD_FP64;
            to.tol = std::min(o.tol, 1e-12);
            to.d_warm = nullptr;
            to.max_refine = std::max(o.max_refine, 8);
            to.max_iters = std::max(o.max_iters, 5000);
            double *x64 = nullptr, *zE = nullptr;
            SolveOut so;
            ESL_TRY(krylov_solve<true>(ctx, ws, L, d_rates, B, bE, bO, nullptr, 0, to, x64, zE, so));
            agg.iters += so.iters;
            ESL_CUDA(cudaMemsetAsync(sums, 0, (size_t)B * T * 8, s));
            ESL_COUNT_LAUNCH();
            k_pinned_sum<<<gt, kT, 0, s>>>(T, net->offsets.get(), net->order.get(), d_big, d_pins, L.ld, zE, x64, TS,
                                           Rb, sums);
            ESL_COUNT_LAUNCH();
            k_pinned_norm<<<gt, kT, 0, s>>>(T, net->offsets.get(), d_big, TS, Rb, sums);
            ESL_CUDA(cudaGetLastError());
            ESL_CUDA(cudaStreamSynchronize(s));
        }
    }
    if (d_R) ESL_CUDA(cudaMemcpyAsync(d_R, Rb, (size_t)TS * 8, cudaMemcpyDeviceToDevice, s));

    // ---- transient part ----
    const int K = B * R;
    double* y = (double*)ws.get(S_Y, (size_t)K * T * 8, &st_);
    if (st_ != ESL_OK) return st_;
    ESL_CUDA(cudaMemsetAsync(y, 0, (size_t)K * T * 8, s));
    if (o.d_occupation) ESL_CUDA(cudaMemsetAsync(o.d_occupation, 0, (size_t)K * N * 8, s));
    const bool has_transient = (size_t)TS < N;
    bool swept = false;
    if (has_transient && (o.method == ESL_METHOD_DIRECT || o.method == ESL_METHOD_MIXED) && sweep_supported(net)) {
        // state-major level sweep; systems it cannot bring below the acceptance
        // residual are redone by the block solve with its dense-LU fallback
        SweepStats sw;
        int rc = sweep_forward(ctx, net, K, R, d_rates, d_x0, N, o, y, sw);
        agg.iters += sw.iters;
        agg.relres = std::max(agg.relres, sw.relres);
        if (rc == ESL_ERR_NOT_CONVERGED && !sw.failed.empty()) {
            const int Kf = (int)sw.failed.size();
            if (debug_enabled()) fprintf(stderr, "[esl] sweep: block-solve fallback for %d of %d systems\n", Kf, K);
            Layout L;
            ESL_TRY(make_layout(ctx, ws, net, 0, nullptr, true, L, 1));
            double* r_sub = (double*)ws.get(S_RSUB, (size_t)Kf * 2 * n * 8, &st_);
            double* x_sub = (double*)ws.get(S_XSUB, (size_t)Kf * N * 8, &st_);
            int32_t* d_failed = (int32_t*)ws.get(S_LIST, (size_t)Kf * 4, &st_);
            double* ZEb = (double*)ws.get(S_ZEB, (size_t)Kf * L.ld * 8, &st_);
            double* ZOb = (double*)ws.get(S_ZOB, (size_t)Kf * L.ld * 8, &st_);
            double* y_sub = (double*)ws.get(S_SUM, (size_t)Kf * T * 8, &st_);
            if (st_ != ESL_OK) return st_;
            for (int j = 0; j < Kf; j++) {
                const int k = sw.failed[j];
                ESL_CUDA(cudaMemcpyAsync(r_sub + (size_t)j * 2 * n, d_rates + (size_t)(k / R) * 2 * n, 2 * n * 8,
                                         cudaMemcpyDeviceToDevice, s));
                ESL_CUDA(cudaMemcpyAsync(x_sub + (size_t)j * N, d_x0 + (size_t)(k % R) * N, N * 8,
                                         cudaMemcpyDeviceToDevice, s));
            }
            ESL_CUDA(cudaMemcpyAsync(d_failed, sw.failed.data(), (size_t)Kf * 4, cudaMemcpyHostToDevice, s));
            esl_solve_opts bo = o;
            bo.method = ESL_METHOD_DIRECT;
            bo.d_warm = nullptr;
            bo.max_iters = block_budget(ctx, o);
            bo.max_refine = std::max(o.max_refine, 6);  // the fallback refines at least as far as the default
            SolveOut sb;
            rc = block_forward_solve(ctx, ws, net, Kf, 1, r_sub, x_sub, N, ZEb, ZOb, bo, sb, true);
            if (rc != ESL_OK && rc != ESL_ERR_NOT_CONVERGED) return rc;
            agg.iters += sb.iters;
            agg.fallback_systems += Kf;
            agg.dense_systems += sb.dense_systems;
            agg.converged = sb.converged;
            agg.relres = std::max(agg.relres, sb.relres);
            ESL_CUDA(cudaMemsetAsync(y_sub, 0, (size_t)Kf * T * 8, s));
            ESL_COUNT_LAUNCH();
            k_terminal_mass<<<dim3((TS + 127) / 128, Kf), 128, 0, s>>>(n, T, TS, 1, 1, L.ld, r_sub, x_sub, N,
                                                                         net->order.get(), net->term_of.get(),
                                                                         net->G.get(), ZEb, ZOb, y_sub);
            ESL_COUNT_LAUNCH();
            k_set_rows<<<dim3((T + 127) / 128, Kf), 128, 0, s>>>(T, d_failed, y_sub, y);
            ESL_CUDA(cudaGetLastError());
            if (rc == ESL_ERR_NOT_CONVERGED) {
                if (rep) {
                    fill_report(rep, agg, false);
                }
                return rc;
            }
        } else if (rc != ESL_OK) {
            return rc;
        }
        swept = true;
    }
    if (swept) {
        // terminal masses are in y
    } else if (has_transient) {
        Layout L;
        ESL_TRY(make_layout(ctx, ws, net, 0, nullptr, true, L, R));
        const size_t vec = (size_t)K * L.ld;
        double* ZE = nullptr;
        double* ZO = nullptr;
        int rc = ESL_OK;
        SolveOut so;
        if (o.method == ESL_METHOD_DIRECT) {
            ZE = (double*)ws.get(S_ZEF, vec * 8, &st_);
            ZO = (double*)ws.get(S_ZOF, vec * 8, &st_);
            if (st_ != ESL_OK) return st_;
            esl_solve_opts bo = o;
            bo.max_iters = block_budget(ctx, o);
            rc = block_forward_solve(ctx, ws, net, K, R, d_rates, d_x0, N, ZE, ZO, bo, so);
            agg.iters += so.iters;
            agg.dense_systems += so.dense_systems;
            agg.relres = so.relres;
            agg.converged = so.converged;
        } else {
            double* bE = (double*)ws.get(S_BE, vec * 8, &st_);
            double* bO = (double*)ws.get(S_BO, vec * 8, &st_);
            if (st_ != ESL_OK) return st_;
            dim3 g = grid2(L.H, K);
            ESL_COUNT_LAUNCH();
            k_rhs<true><<<g, kT, 0, s>>>(L, n, d_rates, d_x0, N, net->F.get(), net->term_of.get(), bE, bO);
            ESL_CUDA(cudaGetLastError());
            double *x64 = nullptr, *zE = nullptr;
            rc = krylov_solve<true>(ctx, ws, L, d_rates, K, bE, bO, o.d_warm, N, o, x64, zE, so);
            agg.iters += so.iters;
            agg.refinements = so.refinements;
            agg.relres = so.relres;
            agg.converged = so.converged;
            // keep the whole-system result out of the Krylov scratch slots
            ws.swap(S_X64, S_ZOF);
            ws.swap(S_ZE, S_ZEF);
            ZO = x64;
            ZE = zE;
            if (rc == ESL_ERR_NOT_CONVERGED) {
                // fallback: systems that missed the budget go through the block solve
                std::vector<int32_t> failed;
                for (int k = 0; k < K; k++)
                    if (so.sys_relres[k] > kAcceptRel) failed.push_back(k);
                const int Kf = (int)failed.size();
                if (debug_enabled()) fprintf(stderr, "[esl] block-solve fallback for %d of %d systems\n", Kf, K);
                double* r_sub = (double*)ws.get(S_RSUB, (size_t)Kf * 2 * n * 8, &st_);
                double* x_sub = (double*)ws.get(S_XSUB, (size_t)Kf * N * 8, &st_);
                int32_t* d_failed = (int32_t*)ws.get(S_LIST, (size_t)Kf * 4, &st_);
                double* ZEb = (double*)ws.get(S_ZEB, (size_t)Kf * L.ld * 8, &st_);
                double* ZOb = (double*)ws.get(S_ZOB, (size_t)Kf * L.ld * 8, &st_);
                if (st_ != ESL_OK) return st_;
                for (int j = 0; j < Kf; j++) {
                    const int k = failed[j];
                    ESL_CUDA(cudaMemcpyAsync(r_sub + (size_t)j * 2 * n, d_rates + (size_t)(k / R) * 2 * n, 2 * n * 8,
                                             cudaMemcpyDeviceToDevice, s));
                    ESL_CUDA(cudaMemcpyAsync(x_sub + (size_t)j * N, d_x0 + (size_t)(k % R) * N, N * 8,
                                             cudaMemcpyDeviceToDevice, s));
                }
                ESL_CUDA(cudaMemcpyAsync(d_failed, failed.data(), (size_t)Kf * 4, cudaMemcpyHostToDevice, s));
                esl_solve_opts bo = o;
                bo.max_iters = block_budget(ctx, o);
                bo.max_refine = std::max(o.max_refine, 6);
                SolveOut sb;
                rc = block_forward_solve(ctx, ws, net, Kf, 1, r_sub, x_sub, N, ZEb, ZOb, bo, sb, true);
                agg.iters += sb.iters;
                agg.fallback_systems += Kf;
                agg.dense_systems += sb.dense_systems;
                agg.converged = sb.converged;
                double worst = 0.0;
                for (int k = 0; k < K; k++)
                    if (so.sys_relres[k] <= kAcceptRel) worst = std::max(worst, so.sys_relres[k]);
                agg.relres = std::max(worst, sb.relres);
                dim3 gs((unsigned)((L.ld + 255) / 256), (unsigned)Kf);
                ESL_COUNT_LAUNCH();
                k_scatter_systems<<<gs, 256, 0, s>>>(L.ld, d_failed, ZEb, ZE);
                ESL_COUNT_LAUNCH();
                k_scatter_systems<<<gs, 256, 0, s>>>(L.ld, d_failed, ZOb, ZO);
                ESL_CUDA(cudaGetLastError());
            }
        }
        if (rc != ESL_OK && rc != ESL_ERR_NOT_CONVERGED) return rc;
        ESL_COUNT_LAUNCH();
        k_terminal_mass<<<dim3((TS + 127) / 128, K), 128, 0, s>>>(n, T, TS, R, 0, L.ld, d_rates, d_x0, N,
                                                                    net->order.get(), net->term_of.get(),
                                                                    net->G.get(), ZE, ZO, y);
        ESL_CUDA(cudaGetLastError());
        if (rc == ESL_ERR_NOT_CONVERGED) {
            if (rep) {
                fill_report(rep, agg, false);
            }
            return rc;
        }
    } else {
        dim3 g((TS + 127) / 128, K);
        ESL_COUNT_LAUNCH();
        k_terminal_mass<<<g, 128, 0, s>>>(n, T, TS, R, 0, 0, d_rates, d_x0, N, net->order.get(), net->term_of.get(),
                                          net->G.get(), nullptr, nullptr, y);
        ESL_CUDA(cudaGetLastError());
    }
    // ---- x_inf and marginals ----
    if (d_x_inf) {
        ESL_CUDA(cudaMemsetAsync(d_x_inf, 0, (size_t)K * N * 8, s));
        if (d_marg) ESL_CUDA(cudaMemsetAsync(d_marg, 0, (size_t)K * n * 8, s));
        ESL_COUNT_LAUNCH();
        k_scatter_xinf<<<dim3((TS + 127) / 128, K), 128, 0, s>>>(n, T, TS, R, N, net->order.get(),
                                                                   net->term_of.get(), Rb, y, d_x_inf, d_marg);
        ESL_CUDA(cudaGetLastError());
    }
    // ---- absorption matrix L (backward form, first rate set) ----
    if (d_L) {
        if (has_transient) {
            Layout L;
            ESL_TRY(make_layout(ctx, ws, net, 0, nullptr, false, L, T));
            const size_t vec = (size_t)T * L.ld;
            double* bE = (double*)ws.get(S_BE, vec * 8, &st_);
            double* bO = (double*)ws.get(S_BO, vec * 8, &st_);
            if (st_ != ESL_OK) return st_;
            dim3 g = grid2(L.H, T);
            ESL_COUNT_LAUNCH();
            k_rhs<false><<<g, kT, 0, s>>>(L, n, d_rates, d_x0, N, net->F.get(), net->term_of.get(), bE, bO);
            ESL_CUDA(cudaGetLastError());
            double *x64 = nullptr, *zE = nullptr;
            SolveOut so;
            esl_solve_opts lo = o;
            lo.d_warm = nullptr;
            lo.d_occupation = nullptr;
            lo.max_iters = std::max(o.max_iters, 5000);
            const int rc = krylov_solve<false>(ctx, ws, L, d_rates, T, bE, bO, nullptr, 0, lo, x64, zE, so);
            if (rc == ESL_OK) {
                ESL_COUNT_LAUNCH();
                k_scatter_L<<<g, kT, 0, s>>>(L.H, T, N, L.ld, net->term_of.get(), zE, x64, d_L);
                ESL_CUDA(cudaGetLastError());
            } else if (rc == ESL_ERR_NOT_CONVERGED && sweep_supported(net)) {
                if (debug_enabled()) fprintf(stderr, "[esl] L: backward solve missed its tolerance, forward sweep\n");
                ESL_TRY(absorption_by_sweep(ctx, ws, net, d_rates, o, d_L));
                agg.absorption_by_sweep = true;
            } else {
                return rc;
            }
        } else {
            // every state terminal: L[t][v] = [v in t]
            ESL_CUDA(cudaMemsetAsync(d_L, 0, (size_t)T * N * 8, s));
            Layout L;
            ESL_TRY(make_layout(ctx, ws, net, 0, nullptr, false, L, T));
            double* z = (double*)ws.get(S_BE, (size_t)T * L.ld * 8 * 2, &st_);
            if (st_ != ESL_OK) return st_;
            ESL_COUNT_LAUNCH();
            k_scatter_L<<<grid2(L.H, T), kT, 0, s>>>(L.H, T, N, L.ld, net->term_of.get(), z, z + (size_t)T * L.ld,
                                                    d_L);
            ESL_CUDA(cudaGetLastError());
        }
    }
    ESL_CUDA(cudaStreamSynchronize(s));
    if (rep) {
        fill_report(rep, agg, agg.converged);
    }
    return ESL_OK;
}

}  // namespace esl
