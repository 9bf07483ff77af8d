/*
 * esl_b200.h -- C ABI of the B200 (sm_100a) ExaStoLog stationary-distribution path.
 *
 * The reference (asmelko/paraExaStoLog) exposes this path as C++ classes; every
 * entry point below names the reference interface it replaces.  Conventions:
 *   - every function returns an int status (ESL_OK or a negative ESL_ERR_*) and
 *     never exits the process; esl_last_error() gives the message (per thread);
 *   - pointers named d_* are device pointers owned by the caller; everything
 *     else is host memory;
 *   - work is ordered on the stream given to esl_ctx_create; functions that
 *     return host results synchronise that stream;
 *   - threads: one context per host thread at a time; a network may be solved from
 *     several threads (on their own contexts) at once, its level-sweep plan is built
 *     once under a lock and then only read;
 *   - state s is an n-bit integer, bit i is node i in bnet line order;
 *     rates are [up_0, down_0, ..., up_{n-1}, down_{n-1}] (FP64).
 */
#ifndef ESL_B200_H
#define ESL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ESL_OK 0
#define ESL_ERR_INVALID (-1)       /* bad argument or inconsistent sizes */
#define ESL_ERR_PARSE (-2)         /* bnet / expression error */
#define ESL_ERR_CUDA (-3)          /* CUDA runtime error */
#define ESL_ERR_NOMEM (-4)         /* device or host allocation failed */
#define ESL_ERR_TIMEOUT (-5)       /* a device fixpoint loop exceeded its budget */
#define ESL_ERR_NOT_CONVERGED (-6) /* iterative solve missed its tolerance */
#define ESL_ERR_TOO_LARGE (-7)     /* size beyond a documented limit */

#define ESL_MAX_NODES 30

typedef struct esl_ctx esl_ctx;     /* device + stream + scratch */
typedef struct esl_model esl_model; /* parsed bnet: node names + DNF clauses */
typedef struct esl_net esl_net;     /* device symbolic data for one (model, zero-rate pattern) */
typedef struct esl_mlp esl_mlp;     /* learned warm start of one network's transient solve */

/* Solver method for the transient absorption and large terminal kernels. */
#define ESL_METHOD_FP64 0    /* FP64 BiCGStab on the red-black reduced system of all transient states;
                                systems that miss the budget fall back to ESL_METHOD_DIRECT */
#define ESL_METHOD_MIXED 1   /* as FP64 with FP32 inner iterations and FP64 iterative refinement */
#define ESL_METHOD_DIRECT 2  /* block forward substitution over SCC levels: singleton levels exact,
                                other levels FP64 Krylov with a dense-LU fallback per SCC block */

typedef struct esl_solve_opts {
    int method;            /* ESL_METHOD_* */
    double tol;            /* relative residual target of the transient solve (default 1e-10) */
    int max_iters;         /* Krylov iteration budget per system before the fallback (default 600) */
    int max_refine;        /* FP64 refinement steps (default 6) */
    const double* d_warm;  /* optional warm start of the occupation vector, B x N (device), or NULL */
    double* d_occupation;  /* optional output (device, B x R x N): expected time spent in each transient
                              state before absorption (0 on terminal states); ESL_METHOD_DIRECT or
                              ESL_METHOD_MIXED only.  No counterpart in the reference, which never
                              forms this vector; it is the label the learned warm start trains on. */
} esl_solve_opts;

typedef struct esl_report {
    int iterations;        /* Krylov iterations (max over the batch) */
    int refinements;       /* FP64 refinement steps taken */
    double relres;         /* final relative residual (max over the batch) */
    int converged;         /* 1 if every system met tol */
    int fallback_systems;  /* systems the level sweep handed to the block forward solve */
    int dense_lu_systems;  /* (system, level group) pairs solved by the dense LU of their SCC blocks */
    int absorption_by_sweep; /* 1 if L (d_L) missed its tolerance in the backward solve and was
                                computed by forward level sweeps instead */
} esl_report;

const char* esl_last_error(void);
int esl_version(void);

/* ---- context -------------------------------------------------------- */
int esl_ctx_create(int device, void* cuda_stream, esl_ctx** out);
int esl_ctx_destroy(esl_ctx* ctx);
int esl_ctx_synchronize(esl_ctx* ctx);

/* Budgets of the fallback paths (no counterpart in the reference, whose library calls
 * std::exit on failure); a value <= 0 keeps the default.  Tests use them to drive every
 * fallback branch without a device fault:
 *   graph_sweeps: sweeps per fixpoint loop of the graph stages (default: 2^n + 64); past
 *     it esl_net_build / esl_net_from_csc return ESL_ERR_TIMEOUT;
 *   block_iters: Krylov iteration budget of the block forward solve, the fallback of
 *     the level sweep (default max(esl_solve_opts.max_iters, 3000)); systems that miss
 *     it get a dense FP64 LU of each SCC block of the level group;
 *   dense_max: largest SCC block that dense LU takes (default 4096 states); a system
 *     that misses the budget in a larger block returns ESL_ERR_NOT_CONVERGED.
 * The context stays usable after any of these errors. */
int esl_ctx_set_budgets(esl_ctx* ctx, int64_t graph_sweeps, int block_iters, int dense_max);

/* ---- model: replaces model_builder::construct_model (cuda/src/model.cpp:80-125)
 *      and clause_t::get_positive_mask/get_negative_mask (cuda/src/model.cpp:8-21) */
int esl_model_load(const char* path, esl_model** out);
int esl_model_parse(const char* bnet_text, esl_model** out);
int esl_model_free(esl_model* m);
int esl_model_nodes(const esl_model* m, int* n);
const char* esl_model_node_name(const esl_model* m, int i);
int esl_model_node_index(const esl_model* m, const char* name, int* index);
/* clause lists: off[n+1] prefixes into pos/neg; *total = clause count (arrays filled when cap >= total) */
int esl_model_clauses(const esl_model* m, int32_t* off, uint32_t* pos, uint32_t* neg, int cap, int* total);

/* ---- rates: replaces transition_rates::generate_uniform / generate_normal
 *      (cuda/src/transition_rates.cpp:24-97); names not in the model -> ESL_ERR_INVALID,
 *      negative rate -> ESL_ERR_INVALID.  rates_out has 2n entries. */
int esl_rates_uniform(const esl_model* m, int n_up, const char* const* up_names, const double* up_vals,
                      int n_down, const char* const* down_names, const double* down_vals, double* rates_out);
int esl_rates_normal(const esl_model* m, double mean, double stddev, uint64_t seed, int n_up,
                     const char* const* up_names, const double* up_vals, int n_down,
                     const char* const* down_names, const double* down_vals, double* rates_out);

/* ---- initial state: replaces initial_state::initial_state (cuda/src/initial_state.cu:7-60) */
int esl_initial_state(esl_ctx* ctx, const esl_model* m, int n_fixed, const char* const* fixed_names,
                      const int* fixed_values, double fixed_probability, double* d_x0);

/* ---- transition table: replaces transition_table::construct_table
 *      (cuda/src/transition_table.cu:121-174, sparse_utils.cu:14-32 coo2csc).
 *      CSC by source: d_indptr[N+1], d_rows[nnz] = destinations (ascending within a
 *      column), d_cols[nnz] = sources (may be NULL).  Call esl_table_nnz first. */
int esl_table_nnz(esl_ctx* ctx, const esl_model* m, const double* rates, int64_t* nnz);
int esl_table_build(esl_ctx* ctx, const esl_model* m, const double* rates, int32_t* d_indptr,
                    int32_t* d_rows, int32_t* d_cols);
/* The same CSC with 64-bit column pointers (d_indptr[N+1] int64), for tables of 2^31 or
 * more edges, which the reference's index_t = int (cuda/src/types.h:6) cannot address:
 * networks of up to ESL_MAX_NODES nodes (n = 28: about 3.8e9 edges, 17 GB). */
int esl_table_build64(esl_ctx* ctx, const esl_model* m, const double* rates, int64_t* d_indptr,
                      int32_t* d_rows, int32_t* d_cols);
/* per-state flip masks: bit i of d_out[s] = edge s -> s^(1<<i); of d_in[s] = edge s^(1<<i) -> s */
int esl_flip_masks(esl_ctx* ctx, const esl_model* m, const double* rates, uint32_t* d_out, uint32_t* d_in);

/* ---- allocation-free transition table.  No counterpart in the reference: the
 *      reference allocates its work arrays in every stage.
 *      For callers that must not allocate device memory while they run: code
 *      inside a framework whose caching allocator already holds the GPU's memory,
 *      loops that cannot afford the device-wide synchronisation of cudaFree, and
 *      services that allocate only at start-up.  Output is the same CSC as
 *      esl_table_build (d_indptr[N+1], d_rows/d_cols with rows_capacity entries,
 *      d_cols may be NULL), on the given stream of the CURRENT device.  It takes no
 *      context and calls no cudaMalloc/cudaFree: its scratch (~4.3 MB) is a static
 *      device array that every GPU loading the library keeps until exit.
 *      Limits: at most ESL_STATIC_TABLE_MAX_NODES nodes and
 *      ESL_STATIC_TABLE_MAX_CLAUSES DNF clauses, else ESL_ERR_TOO_LARGE; *nnz
 *      always receives the edge count once it is known, and a table with more than
 *      rows_capacity edges returns ESL_ERR_TOO_LARGE without writing the arrays.
 *      The first call on a device looks up the array's device address; make that
 *      first call before any stream capture.  The address is kept for the life of
 *      the process: after cudaDeviceReset on a device, do not call this entry point
 *      on that device again.  All calls on a device share the
 *      array: calls whose GPU work overlaps race, so serialise them.
 *      Synchronises the stream before returning. */
#define ESL_STATIC_TABLE_MAX_NODES 20
#define ESL_STATIC_TABLE_MAX_CLAUSES 8192
int esl_table_build_static(const esl_model* m, const double* rates, void* cuda_stream, int32_t* d_indptr,
                           int32_t* d_rows, int32_t* d_cols, int64_t rows_capacity, int64_t* nnz);

/* ---- transition graph: replaces transition_graph::reorganize_vertices
 *      (cuda/src/transition_graph.cu:39-202, kernels/transition_graph.cu:3-52).
 *      Builds table masks, SCCs, terminal SCCs, levels and the reordering on the device. */
int esl_net_build(esl_ctx* ctx, const esl_model* m, const double* rates, esl_net** out);
/* same from a CSC table (any single-bit-flip graph, e.g. one produced by esl_table_build).
 * The table is read on the device as given: d_indptr (2^n + 1 entries) must start at 0
 * and never decrease, and d_rows must hold d_indptr[2^n] entries.  Edges that do not
 * flip exactly one bit of their source are reported (ESL_ERR_INVALID); pointers are not
 * checked, so validate a table from an untrusted source before the call. */
int esl_net_from_csc(esl_ctx* ctx, int n_nodes, const int32_t* d_indptr, const int32_t* d_rows,
                     esl_net** out);
int esl_net_free(esl_net* net);
int esl_net_info(const esl_net* net, int* n_nodes, int* n_sccs, int* n_terminals, int* n_terminal_states);
/* d_order[N] reordered vertices, d_offsets[n_sccs+1] SCC offsets (terminals first),
 * d_levels[n_sccs] level of the SCC at each position (1 = terminal), d_labels[N] SCC label
 * (min vertex of the SCC).  Any pointer may be NULL. */
int esl_net_export(esl_ctx* ctx, const esl_net* net, int32_t* d_order, int32_t* d_offsets,
                   int32_t* d_levels, int32_t* d_labels);
/* Autotuner (no counterpart in the reference): times the batch solve of the level sweep
 * under a few tilings (the L2 slice budget that sets the systems per tile, and one or two
 * systems per thread in the gather kernels), keeps the fastest in `net` (and in `ctx`, for
 * networks built later on it) and returns it.  Run it outside any timed region; it solves
 * the batch five times. */
int esl_net_autotune(esl_ctx* ctx, esl_net* net, int B, const double* d_rates, int R, const double* d_x0,
                     const esl_solve_opts* opts, int* tile_mb, int* two_per_thread, double* ms);
/* Test hook (no counterpart in the reference): builds the level-sweep plan of `net` afresh,
 * on the device (host_builder = 0, the builder the solver uses) or with the host reference
 * builder (1), and writes FNV-1a 64 checksums of its parts to sums[0 .. min(cap, 12)):
 * rows, desc, in-group and earlier-group predecessor lists (pointers, entries), terminal
 * predecessor lists (pointers, entries), CTA-local SCC lists (offsets, even counts,
 * slots) and the group table.  The two builders must agree on all 12. */
int esl_net_plan_checksums(esl_ctx* ctx, const esl_net* net, int host_builder, uint64_t* sums, int cap);
/* 1 if the rate set has the zero pattern the net was built for */
int esl_net_compatible(const esl_net* net, const double* rates, int* compatible);

/* ---- solver: replaces solver::solve (cuda/src/solver.cu:311-334): terminal kernels
 *      (solve_terminal_part :102-159), absorption (solve_nonterminal_part :205-300) and
 *      x_inf = R (L x0) (compute_final_states :302-309), plus per-node marginals.
 *      d_R[n_terminal_states] aligned with d_order; d_L[T x N] by original state (optional). */
int esl_solve(esl_ctx* ctx, const esl_net* net, const double* d_rates, const double* d_x0,
              double* d_x_inf, double* d_marginals, double* d_R, double* d_L,
              const esl_solve_opts* opts, esl_report* report);

/* Batched: B rate sets (d_rates B x 2n, same zero pattern) x R initial distributions
 * (d_x0 R x N); outputs d_x_inf[B][R][N], d_marginals[B][R][n] (may be NULL). */
int esl_solve_batch(esl_ctx* ctx, const esl_net* net, int B, const double* d_rates, int R,
                    const double* d_x0, double* d_x_inf, double* d_marginals,
                    const esl_solve_opts* opts, esl_report* report);

/* ---- many networks in one call.  No counterpart in the reference, which solves one
 *      network per run (cuda/src/main.cpp:102-157).  Each job is one esl_solve_batch;
 *      the contexts of the pool (each with its own stream and workspace; create them on
 *      one device or several) run the jobs concurrently from host threads, largest
 *      first, so that small networks overlap on the GPU.  Returns the first failing
 *      job's status; every job's status and report are written back.  A context whose
 *      device cannot be selected takes no job and makes the call return ESL_ERR_CUDA;
 *      the other contexts still run the jobs. */
typedef struct esl_job {
    const esl_net* net;
    int B;                   /* rate sets (d_rates B x 2n, same zero pattern as net) */
    const double* d_rates;
    int R;                   /* initial distributions (d_x0 R x N) */
    const double* d_x0;
    double* d_x_inf;         /* B x R x N */
    double* d_marginals;     /* B x R x n, or NULL */
    esl_report report;       /* out */
    int status;              /* out */
} esl_job;
int esl_solve_many(esl_ctx* const* ctxs, int n_ctx, esl_job* jobs, int n_jobs, const esl_solve_opts* opts);

/* Host-memory end-to-end call: bnet text, rates (B x 2n) and x0 (R x N) on the host,
 * results copied back to host buffers.  Builds and frees its own net. */
int esl_solve_host(esl_ctx* ctx, const esl_model* m, int B, const double* rates, int R, const double* x0,
                   double* x_inf, double* marginals, const esl_solve_opts* opts, esl_report* report);

/* ---- learned warm start.  No counterpart in the reference, which has no learned
 *      component.  A 3-layer MLP (77 -> 128 -> 128 -> 1, BF16 weights, FP32
 *      accumulation) predicts the log occupation of a transient state under a rate set
 *      from: 20 node bits, the log outgoing rate sum, 16 terminal-reachability bits
 *      and 40 log rates.  Its prediction is the warm start (esl_solve_opts.d_warm) of
 *      the level sweep's grid-wide Krylov groups; the solve itself is unchanged and
 *      still decides convergence.  Networks of at most 20 nodes; the handle refers to
 *      `net`, which must outlive it.  Training labels come from esl_solve_batch with
 *      esl_solve_opts.d_occupation.  Parameters: W1[128][77], b1[128], W2[128][128],
 *      b2[128], w3[128], b3 (FP32 master copy). */
#define ESL_MLP_PARAMS 26625
int esl_mlp_create(esl_ctx* ctx, const esl_net* net, uint64_t seed, esl_mlp** out);
/* waits for the device, then frees; touches neither the context nor the net, so it may
 * come after either has been freed */
int esl_mlp_free(esl_mlp* mlp);
/* number of states it predicts (odd-parity rows of the grid-wide level groups) and the
 * label standardisation log z = mu + sigma * y */
int esl_mlp_info(const esl_mlp* mlp, int* n_targets, float* mu, float* sigma);
int esl_mlp_targets(const esl_mlp* mlp, uint32_t* d_states);  /* n_targets states */
int esl_mlp_reach(const esl_mlp* mlp, uint32_t* d_reach);     /* N words: bit t = reaches terminal t */
int esl_mlp_get_params(const esl_mlp* mlp, float* params);    /* host, ESL_MLP_PARAMS floats */
int esl_mlp_set_params(esl_mlp* mlp, const float* params, float mu, float sigma);
/* feature rows (S x 80 floats, device) of samples (rate set d_k[s] of d_rates, state d_state[s]).
 * Here and in esl_mlp_loss_grad / esl_mlp_forward the sample indices are read on the
 * device unchecked: 0 <= d_k[s] < the rate sets in d_rates, 0 <= d_state[s] < 2^n. */
int esl_mlp_features(esl_mlp* mlp, int S, const double* d_rates, const int32_t* d_k, const int32_t* d_state,
                     float* d_x);
/* mean squared error against standardized targets and, if grad != NULL, its gradient
 * with respect to the parameters (host, ESL_MLP_PARAMS floats) */
int esl_mlp_loss_grad(esl_mlp* mlp, int S, const double* d_rates, const int32_t* d_k, const int32_t* d_state,
                      const float* d_target, float* loss, float* grad);
/* standardized outputs y of the training forward pass (device, S floats) */
int esl_mlp_forward(esl_mlp* mlp, int S, const double* d_rates, const int32_t* d_k, const int32_t* d_state,
                    float* d_y);
/* Adam steps on random (rate set, target state) samples of B rate sets and their
 * occupations (d_occupation B x N, from esl_solve_batch) */
int esl_mlp_train(esl_mlp* mlp, int B, const double* d_rates, const double* d_occupation, int steps, int batch,
                  float lr, float* final_loss);
/* warm start d_warm (B x N, device) for B rate sets: predicted occupation on the targets, 0 elsewhere */
int esl_mlp_predict(esl_mlp* mlp, int B, const double* d_rates, double* d_warm);

/* ---- measurement hook (no counterpart in the reference): when on, the library
 *      records CUDA events around the launches of its hot kernels (table, graph sweeps,
 *      every application of the reduced (Schur) operator and the BiCGStab vector updates
 *      of the first convergence-poll window of each Krylov group).  esl_ctx_profile
 *      returns the summed device time, the algorithmic bytes (each array touched once per
 *      launch) and the record count since profiling was switched on. */
int esl_ctx_set_profiling(esl_ctx* ctx, int on);
int esl_ctx_profile(esl_ctx* ctx, double* total_ms, double* total_bytes, int* launches);
/* the same per recorded application: *count records, the first `cap` written */
int esl_ctx_profile_records(esl_ctx* ctx, int cap, double* ms, double* bytes, int* count);
/* record i (0 <= i < count): its kernel class ("k_flip_masks", "k_emit_csc", "graph_sweep",
 * "schur_operator", "bicgstab_update", "schur_operator_whole_system"), device ms and
 * algorithmic bytes.  Besides the Schur operator, profiling records the table kernels, the
 * fixpoint sweeps of the graph stages and the BiCGStab vector updates; esl_ctx_profile and
 * esl_ctx_profile_records cover every record. */
int esl_ctx_profile_entry(esl_ctx* ctx, int i, const char** name, double* ms, double* bytes);
/* number of kernels this library has launched in this process (no counterpart in the reference) */
int esl_launch_count(uint64_t* count);
/* The library keeps the device blocks it releases (up to 8 GiB per device) and hands them
 * out again, because cudaFree / cudaMalloc of a network's symbolic buffers cost up to
 * 0.8 s per build on the B200.  This returns every cached block to the driver (no
 * counterpart in the reference). */
int esl_trim_cache(void);

#ifdef __cplusplus
}
#endif
#endif /* ESL_B200_H */
