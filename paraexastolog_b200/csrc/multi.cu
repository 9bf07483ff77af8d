// Many networks in one call: a host-side scheduler over a pool of contexts.
//
// No counterpart in the reference, which solves one network per process run
// (cuda/src/main.cpp:102-157).  Each job is one esl_solve_batch (a network, B rate sets,
// R initial distributions).  Every context of the pool (its own stream and workspace)
// gets a host thread that takes jobs from a shared queue, largest first (states x
// systems), so that the level sweeps of small networks overlap on the GPU while the
// large ones run.  The symbolic sweep plans are built up front on the first context,
// so no two threads build the plan of the same network.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "esl_internal.h"

namespace esl {
int sweep_prepare(esl_ctx* ctx, const esl_net* net);
}

using namespace esl;

extern "C" int esl_solve_many(esl_ctx* const* ctxs, int n_ctx, esl_job* jobs, int n_jobs, const esl_solve_opts* opts) {
    if (!ctxs || n_ctx < 1 || (n_jobs > 0 && !jobs) || n_jobs < 0) return fail(ESL_ERR_INVALID, "bad argument");
    for (int c = 0; c < n_ctx; c++)
        if (!ctxs[c]) return fail(ESL_ERR_INVALID, "NULL context");
    for (int j = 0; j < n_jobs; j++) {
        if (!jobs[j].net) return fail(ESL_ERR_INVALID, "job without a network");
        jobs[j].status = ESL_OK;
    }
    if (n_jobs == 0) return ESL_OK;
    // symbolic plans once per distinct network, before any thread runs
    {
        StreamScope stream_scope_(ctxs[0]);
        std::vector<const esl_net*> seen;
        for (int j = 0; j < n_jobs; j++) {
            const esl_net* net = jobs[j].net;
            if (std::find(seen.begin(), seen.end(), net) != seen.end()) continue;
            seen.push_back(net);
            const int method = opts ? opts->method : ESL_METHOD_FP64;
            if ((method == ESL_METHOD_DIRECT || method == ESL_METHOD_MIXED) && sweep_supported(net))
                ESL_TRY(sweep_prepare(ctxs[0], net));
        }
    }
    std::vector<int> order(n_jobs);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (double)jobs[a].net->N * jobs[a].B * jobs[a].R > (double)jobs[b].net->N * jobs[b].B * jobs[b].R;
    });
    std::atomic<int> next{0};
    std::mutex mu;
    int first_status = ESL_OK;
    std::string first_msg;
    auto worker = [&](int c) {
        esl_ctx* ctx = ctxs[c];
        const cudaError_t e = cudaSetDevice(ctx->device);
        if (e != cudaSuccess) {
            // this worker takes no job; the others drain the queue
            std::lock_guard<std::mutex> lk(mu);
            if (first_status == ESL_OK) {
                first_status = ESL_ERR_CUDA;
                first_msg = std::string("context ") + std::to_string(c) + ": cudaSetDevice: " + cudaGetErrorString(e);
            }
            return;
        }
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n_jobs) break;
            esl_job& jb = jobs[order[i]];
            jb.status = esl_solve_batch(ctx, jb.net, jb.B, jb.d_rates, jb.R, jb.d_x0, jb.d_x_inf, jb.d_marginals, opts,
                                        &jb.report);
            if (jb.status == ESL_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                jb.status = fail(ESL_ERR_CUDA, "stream synchronisation failed");
            if (jb.status != ESL_OK) {
                std::lock_guard<std::mutex> lk(mu);
                if (first_status == ESL_OK) {
                    first_status = jb.status;
                    first_msg = std::string("job ") + std::to_string(order[i]) + ": " + esl_last_error();
                }
            }
        }
    };
    std::vector<std::thread> th;
    const int nt = std::min(n_ctx, n_jobs);
    for (int c = 0; c < nt; c++) th.emplace_back(worker, c);
    for (auto& t : th) t.join();
    // jobs that no worker took (every worker failed to select its device)
    for (int i = std::min(next.load(), n_jobs); i < n_jobs; i++) jobs[order[i]].status = first_status;
    if (first_status != ESL_OK) return fail(first_status, first_msg);
    return ESL_OK;
}
