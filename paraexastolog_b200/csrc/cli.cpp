// esl_cli: the reference's command line (cuda/src/main.cpp:159-312) over the C ABI.
//
// Same flags and the same output as the reference's executable: every state with a
// nonzero stationary probability, in state order, printed as its active node names
// joined by " --- " (or "<nil>") and the probability as an FP32 value
// (solver::print_final_state, cuda/src/solver.cu:336-372).  Differences:
//   - the stationary distribution is computed in FP64 (ESL_METHOD_DIRECT by default,
//     --method direct|mixed|fp64) and printed after conversion to FP32;
//   - --marginals also prints the per-node marginals (the reference has none);
//   - --initial-fixed-prob sets the probability of the fixed initial states; the
//     reference stores the value into the normal distribution's standard deviation
//     instead (main.cpp:256), which --compat-fixed-prob reproduces;
//   - -s/--symbolic reads and writes F.symb in the reference's layout
//     (persistent_solution.cu:31-235: 16 size_t sizes, then int32 and FP32 arrays).  A
//     stored file with a compatible zero-rate pattern replaces the table construction
//     (its CSC is reloaded); the file is rewritten when the rates change.  The matrix
//     inverse of the reference's symbolic path is never stored (its three sizes are 0),
//     as with -n/--no-symb-rates, which is accepted.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "esl_b200.h"

namespace {

struct Args {
    std::string bnet;
    bool normal = false;
    double mean = 0.0, stddev = 1.0;
    std::vector<std::string> up_names, down_names;
    std::vector<double> up_vals, down_vals;
    double fixed_prob = 1.0;
    std::vector<std::string> fixed_names;
    std::vector<int> fixed_vals;
    bool symbolic = false, no_inverse = false, marginals = false, compat_prob = false;
    int method = ESL_METHOD_DIRECT;
    uint64_t seed = 0;
};

const char* kHelp =
    "usage: esl_cli -f BNET_FILE [options]\n"
    "  -f, --bnet-file BNET_FILE          path to the bnet file\n"
    "  -t, --trans-distribution T_DISTR   NORMAL or UNIFORM (default)\n"
    "      --mean MEAN                    mean of the normal transition-rate distribution\n"
    "      --std STD                      standard deviation of the normal distribution\n"
    "      --trans-rates TRANS_RATE       explicit rates, comma separated (u|d)_NAME=VAL\n"
    "  -i, --initial-distribution D       UNIFORM (default); RANDOM is not implemented\n"
    "      --initial-fixed-prob P         probability of the fixed initial states\n"
    "      --initial-fixed-list LIST      fixed parts of the initial state, comma separated NAME=(0|1)\n"
    "  -s, --symbolic                     read/write F.symb beside F.bnet (symbolic reuse)\n"
    "  -n, --no-symb-rates                do not store the non-terminal inverse (never stored here)\n"
    "      --method M                     direct (default), mixed or fp64\n"
    "      --seed S                       seed of the normal transition-rate distribution\n"
    "      --marginals                    also print the per-node marginals\n"
    "      --compat-fixed-prob            reproduce the reference's handling of --initial-fixed-prob\n";

std::vector<std::string> split(const std::string& s, char c) {
    std::vector<std::string> out;
    size_t b = 0;
    for (;;) {
        size_t e = s.find(c, b);
        out.push_back(s.substr(b, e == std::string::npos ? std::string::npos : e - b));
        if (e == std::string::npos) break;
        b = e + 1;
    }
    return out;
}

bool parse_rates(const std::string& v, Args& a) {
    for (const std::string& e : split(v, ',')) {
        const size_t eq = e.find('=');
        if (eq == std::string::npos || e.size() < 3 || (std::toupper(e[0]) != 'U' && std::toupper(e[0]) != 'D') ||
            e[1] != '_')
            return false;
        char* end = nullptr;
        const std::string val = e.substr(eq + 1);
        const double x = std::strtod(val.c_str(), &end);
        if (val.empty() || *end) return false;
        const std::string node = e.substr(2, eq - 2);
        if (std::toupper(e[0]) == 'U') {
            a.up_names.push_back(node);
            a.up_vals.push_back(x);
        } else {
            a.down_names.push_back(node);
            a.down_vals.push_back(x);
        }
    }
    return true;
}

bool parse_fixed(const std::string& v, Args& a) {
    for (const std::string& e : split(v, ',')) {
        const size_t eq = e.find('=');
        if (eq == std::string::npos || eq + 2 != e.size() || (e[eq + 1] != '0' && e[eq + 1] != '1')) return false;
        a.fixed_names.push_back(e.substr(0, eq));
        a.fixed_vals.push_back(e[eq + 1] - '0');
    }
    return true;
}

bool number(const std::string& s, double& out) {
    char* end = nullptr;
    out = std::strtod(s.c_str(), &end);
    return !s.empty() && !*end;
}

// returns 0 on success, 1 on a usage error (usage follows), 2 on an error already reported
int parse(int argc, char** argv, Args& a) {
    bool have_file = false;
    double prob_arg = -1.0;
    for (int i = 1; i < argc; i++) {
        const std::string o = argv[i];
        auto value = [&](std::string& out) -> bool {
            if (i + 1 >= argc) return false;
            out = argv[++i];
            return true;
        };
        std::string v;
        double x;
        if (o == "-f" || o == "--bnet-file") {
            if (!value(a.bnet)) return 1;
            have_file = true;
        } else if (o == "-t" || o == "--trans-distribution") {
            if (!value(v)) return 1;
            if (v != "NORMAL" && v != "UNIFORM") {
                std::cerr << "Bad transition distribution type" << std::endl;
                return 1;
            }
            a.normal = v == "NORMAL";
        } else if (o == "--mean") {
            if (!value(v) || !number(v, a.mean)) return 1;
        } else if (o == "--std") {
            if (!value(v) || !number(v, a.stddev)) return 1;
        } else if (o == "--trans-rates") {
            if (!value(v) || !parse_rates(v, a)) return 1;
        } else if (o == "-i" || o == "--initial-distribution") {
            if (!value(v)) return 1;
            if (v == "RANDOM") {
                std::cerr << "RANDOM initial state distribution not implemented" << std::endl;
                return 2;  // the reference prints no usage here
            }
            if (v != "UNIFORM") {
                std::cerr << "Bad initial state distribution type" << std::endl;
                return 1;
            }
        } else if (o == "--initial-fixed-prob") {
            if (!value(v) || !number(v, x)) return 1;
            prob_arg = x;
        } else if (o == "--initial-fixed-list") {
            if (!value(v) || !parse_fixed(v, a)) return 1;
        } else if (o == "-s" || o == "--symbolic") {
            a.symbolic = true;
        } else if (o == "-n" || o == "--no-symb-rates") {
            a.no_inverse = true;
        } else if (o == "--marginals") {
            a.marginals = true;
        } else if (o == "--compat-fixed-prob") {
            a.compat_prob = true;
        } else if (o == "--method") {
            if (!value(v)) return 1;
            if (v == "direct") a.method = ESL_METHOD_DIRECT;
            else if (v == "mixed") a.method = ESL_METHOD_MIXED;
            else if (v == "fp64") a.method = ESL_METHOD_FP64;
            else return 1;
        } else if (o == "--seed") {
            // a whole number that a uint64_t holds (NaN and 2^64 or more are rejected)
            if (!value(v) || !number(v, x) || !(x >= 0.0 && x < 18446744073709551616.0) || x != std::floor(x))
                return 1;
            a.seed = (uint64_t)x;
        } else {
            return 1;
        }
    }
    if (!have_file) return 1;
    if (prob_arg >= 0.0) {
        if (a.compat_prob)
            a.stddev = prob_arg;  // the reference's assignment (main.cpp:256)
        else
            a.fixed_prob = prob_arg;
    }
    if (a.fixed_prob < 0.0 || a.fixed_prob > 1.0) {
        std::cerr << "Bad fixed initial states probability" << std::endl;
        return 1;
    }
    return 0;
}

// ---- .symb files (the reference's persistent_solution layout) ---------------------------
struct Symb {
    std::vector<int32_t> rows, cols, indptr, order, term_off, nonterm_off, st_indptr, st_indices, snt_indptr,
        snt_indices;
    std::vector<float> rates, st_data, snt_data;
};

bool write_symb(const std::string& path, const Symb& s) {
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    const size_t sizes[16] = {s.rows.size(),     s.cols.size(),       s.indptr.size(),     s.order.size(),
                              s.term_off.size(), s.nonterm_off.size(), s.rates.size(),      s.st_indptr.size(),
                              s.st_indices.size(), s.st_data.size(),  s.snt_indptr.size(), s.snt_indices.size(),
                              s.snt_data.size(), 0,                   0,                   0};
    f.write(reinterpret_cast<const char*>(sizes), sizeof sizes);
    auto put = [&](const auto& v) {
        f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(v[0])));
    };
    put(s.rows);
    put(s.cols);
    put(s.indptr);
    put(s.order);
    put(s.term_off);
    put(s.nonterm_off);
    put(s.rates);
    put(s.st_indptr);
    put(s.st_indices);
    put(s.st_data);
    put(s.snt_indptr);
    put(s.snt_indices);
    put(s.snt_data);
    return (bool)f;
}

// reads the arrays this program uses (table, order, rates); false if absent or corrupt
bool read_symb(const std::string& path, Symb& s) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    const std::streamsize len = f.tellg();
    if (len < (std::streamsize)(16 * sizeof(size_t))) return false;
    f.seekg(0);
    size_t sz[16];
    f.read(reinterpret_cast<char*>(sz), sizeof sz);
    size_t idx = 0, real = 0;
    for (size_t v : sz)
        if (v > (size_t)len) return false;  // keeps the sums below from wrapping
    for (int i : {0, 1, 2, 3, 4, 5, 7, 8, 10, 11, 13, 14}) idx += sz[i];
    for (int i : {6, 9, 12, 15}) real += sz[i];
    if ((size_t)len != idx * sizeof(int32_t) + real * sizeof(float) + sizeof sz) return false;
    auto get = [&](auto& v, size_t n) {
        v.resize(n);
        f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(v[0])));
    };
    get(s.rows, sz[0]);
    get(s.cols, sz[1]);
    get(s.indptr, sz[2]);
    get(s.order, sz[3]);
    get(s.term_off, sz[4]);
    get(s.nonterm_off, sz[5]);
    get(s.rates, sz[6]);
    return (bool)f;
}

// A stored table is used only if it is a well-formed CSC over the N states: the
// kernels that read it index rows[] through indptr[] without bounds checks, so a stale
// or damaged file must be turned away here.
bool valid_csc(const Symb& s, size_t N) {
    if (s.indptr.size() != N + 1 || s.indptr[0] != 0) return false;
    for (size_t v = 0; v < N; v++)
        if (s.indptr[v + 1] < s.indptr[v]) return false;
    if ((size_t)s.indptr[N] != s.rows.size()) return false;
    for (int32_t r : s.rows)
        if (r < 0 || (size_t)r >= N) return false;
    return true;
}

std::string symb_path(const std::string& bnet) {
    const size_t slash = bnet.find_last_of('/');
    const size_t dot = bnet.find_last_of('.');
    return (dot != std::string::npos && (slash == std::string::npos || dot > slash) ? bnet.substr(0, dot) : bnet) +
           ".symb";
}

#define CHECK(call)                                                           \
    do {                                                                      \
        if ((call) != ESL_OK) {                                               \
            std::cerr << "Program ended with an exception: " << esl_last_error() << std::endl; \
            return 1;                                                         \
        }                                                                     \
    } while (0)

#define CUDA_CHECK(call)                                                                          \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            std::cerr << "Program ended with an exception: " << cudaGetErrorString(e_) << std::endl; \
            return 1;                                                                             \
        }                                                                                         \
    } while (0)

template <class T>
struct Dev {
    T* p = nullptr;
    ~Dev() {
        if (p) cudaFree(p);
    }
};

int run(const Args& a) {
    esl_model* m = nullptr;
    CHECK(esl_model_load(a.bnet.c_str(), &m));
    int n = 0;
    CHECK(esl_model_nodes(m, &n));
    const size_t N = (size_t)1 << n;
    std::vector<const char*> un, dn, fn;
    for (auto& s : a.up_names) un.push_back(s.c_str());
    for (auto& s : a.down_names) dn.push_back(s.c_str());
    for (auto& s : a.fixed_names) fn.push_back(s.c_str());
    std::vector<double> rates(2 * n);
    if (a.normal)
        CHECK(esl_rates_normal(m, a.mean, a.stddev, a.seed, (int)un.size(), un.data(), a.up_vals.data(),
                               (int)dn.size(), dn.data(), a.down_vals.data(), rates.data()));
    else
        CHECK(esl_rates_uniform(m, (int)un.size(), un.data(), a.up_vals.data(), (int)dn.size(), dn.data(),
                                a.down_vals.data(), rates.data()));
    esl_ctx* ctx = nullptr;
    CHECK(esl_ctx_create(0, nullptr, &ctx));
    Dev<double> x0, xi, mg, dr, R;
    Dev<int32_t> ip, rw, cl;
    CUDA_CHECK(cudaMalloc(&x0.p, N * 8));
    CUDA_CHECK(cudaMalloc(&xi.p, N * 8));
    CUDA_CHECK(cudaMalloc(&mg.p, (size_t)n * 8));
    CUDA_CHECK(cudaMalloc(&dr.p, (size_t)2 * n * 8));
    CUDA_CHECK(cudaMemcpy(dr.p, rates.data(), (size_t)2 * n * 8, cudaMemcpyHostToDevice));
    CHECK(esl_initial_state(ctx, m, (int)fn.size(), fn.data(), a.fixed_vals.data(), a.fixed_prob, x0.p));

    // symbolic data: reuse a stored table with a compatible zero-rate pattern
    const std::string sp = symb_path(a.bnet);
    Symb stored;
    bool reuse = false, same_rates = false;
    if (a.symbolic && read_symb(sp, stored) && stored.rates.size() == rates.size() && valid_csc(stored, N)) {
        bool zeros_in_stored = false;
        reuse = true;
        same_rates = true;
        for (size_t j = 0; j < rates.size(); j++) {
            const float r = (float)rates[j];
            if ((stored.rates[j] == 0.f) != (r == 0.f)) reuse = false;
            if (stored.rates[j] != r) same_rates = false;
            zeros_in_stored |= stored.rates[j] == 0.f;
        }
        // a net rebuilt from a CSC accepts only rate sets without zeros
        if (zeros_in_stored) reuse = false;
    }
    esl_net* net = nullptr;
    int64_t nnz = 0;
    if (reuse) {
        nnz = (int64_t)stored.rows.size();
        CUDA_CHECK(cudaMalloc(&ip.p, (N + 1) * 4));
        CUDA_CHECK(cudaMalloc(&rw.p, (size_t)std::max<int64_t>(nnz, 1) * 4));
        CUDA_CHECK(cudaMemcpy(ip.p, stored.indptr.data(), (N + 1) * 4, cudaMemcpyHostToDevice));
        if (nnz) CUDA_CHECK(cudaMemcpy(rw.p, stored.rows.data(), (size_t)nnz * 4, cudaMemcpyHostToDevice));
        CHECK(esl_net_from_csc(ctx, n, ip.p, rw.p, &net));
    } else {
        CHECK(esl_net_build(ctx, m, rates.data(), &net));
    }
    int n_sccs = 0, T = 0, TS = 0, nn = 0;
    CHECK(esl_net_info(net, &nn, &n_sccs, &T, &TS));
    const bool write = a.symbolic && !(reuse && same_rates);
    Dev<double> L;
    if (write) {
        CUDA_CHECK(cudaMalloc(&R.p, (size_t)std::max(TS, 1) * 8));
        CUDA_CHECK(cudaMalloc(&L.p, (size_t)T * N * 8));
    }
    esl_solve_opts o{};
    o.method = a.method;
    o.tol = 1e-10;
    esl_report rep{};
    CHECK(esl_solve(ctx, net, dr.p, x0.p, xi.p, mg.p, R.p, L.p, &o, &rep));

    // output (solver::print_final_state)
    std::vector<double> h(N), hm(n);
    CUDA_CHECK(cudaMemcpy(h.data(), xi.p, N * 8, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(hm.data(), mg.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
    std::vector<std::string> names(n);
    for (int i = 0; i < n; i++) names[i] = esl_model_node_name(m, i);
    for (size_t s = 0; s < N; s++) {
        const float p = (float)h[s];
        if (p == 0.f) continue;
        bool printed = false;
        for (int i = 0; i < n; i++)
            if (s & ((size_t)1 << i)) {
                if (printed) std::cout << " --- ";
                std::cout << names[i];
                printed = true;
            }
        if (!printed) std::cout << "<nil>";
        std::cout << " " << p << std::endl;
    }
    if (a.marginals)
        for (int i = 0; i < n; i++) std::cout << "marginal " << names[i] << " " << hm[i] << std::endl;

    if (write) {
        Symb s;
        s.indptr.resize(N + 1);
        if (reuse) {
            s.rows = stored.rows;
            s.cols = stored.cols;
            s.indptr = stored.indptr;
        } else {
            CHECK(esl_table_nnz(ctx, m, rates.data(), &nnz));
            CUDA_CHECK(cudaMalloc(&ip.p, (N + 1) * 4));
            CUDA_CHECK(cudaMalloc(&rw.p, (size_t)std::max<int64_t>(nnz, 1) * 4));
            CUDA_CHECK(cudaMalloc(&cl.p, (size_t)std::max<int64_t>(nnz, 1) * 4));
            CHECK(esl_table_build(ctx, m, rates.data(), ip.p, rw.p, cl.p));
            s.rows.resize(nnz);
            s.cols.resize(nnz);
            CUDA_CHECK(cudaMemcpy(s.indptr.data(), ip.p, (N + 1) * 4, cudaMemcpyDeviceToHost));
            if (nnz) {
                CUDA_CHECK(cudaMemcpy(s.rows.data(), rw.p, (size_t)nnz * 4, cudaMemcpyDeviceToHost));
                CUDA_CHECK(cudaMemcpy(s.cols.data(), cl.p, (size_t)nnz * 4, cudaMemcpyDeviceToHost));
            }
        }
        Dev<int32_t> dord, doff;
        CUDA_CHECK(cudaMalloc(&dord.p, N * 4));
        CUDA_CHECK(cudaMalloc(&doff.p, ((size_t)n_sccs + 1) * 4));
        CHECK(esl_net_export(ctx, net, dord.p, doff.p, nullptr, nullptr));
        std::vector<int32_t> off(n_sccs + 1);
        s.order.resize(N);
        CUDA_CHECK(cudaMemcpy(s.order.data(), dord.p, N * 4, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(off.data(), doff.p, off.size() * 4, cudaMemcpyDeviceToHost));
        s.term_off.assign(off.begin(), off.begin() + T + 1);
        s.nonterm_off.assign(off.begin() + T, off.end());
        for (double r : rates) s.rates.push_back((float)r);
        // R: CSC N x T, column t = the states of terminal SCC t with their stationary values
        std::vector<double> hR(TS), hL((size_t)T * N);
        if (TS) CUDA_CHECK(cudaMemcpy(hR.data(), R.p, (size_t)TS * 8, cudaMemcpyDeviceToHost));
        if (T) CUDA_CHECK(cudaMemcpy(hL.data(), L.p, (size_t)T * N * 8, cudaMemcpyDeviceToHost));
        s.st_indptr = s.term_off;
        s.st_indices.assign(s.order.begin(), s.order.begin() + TS);
        for (double r : hR) s.st_data.push_back((float)r);
        // L: CSR T x N, row t = terminal t's states (1) then the transient states with a
        // nonzero absorption probability, in reordered position
        s.snt_indptr.push_back(0);
        for (int t = 0; t < T; t++) {
            for (int p = off[t]; p < off[t + 1]; p++) {
                s.snt_indices.push_back(s.order[p]);
                s.snt_data.push_back(1.f);
            }
            for (size_t p = (size_t)TS; p < N; p++) {
                const double v = hL[(size_t)t * N + s.order[p]];
                if (v != 0.0) {
                    s.snt_indices.push_back(s.order[p]);
                    s.snt_data.push_back((float)v);
                }
            }
            s.snt_indptr.push_back((int32_t)s.snt_indices.size());
        }
        if (!write_symb(sp, s)) {
            std::cerr << "Program ended with an exception: cannot write " << sp << std::endl;
            return 1;
        }
    }
    esl_net_free(net);
    esl_model_free(m);
    esl_ctx_destroy(ctx);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    Args a;
    const int pr = parse(argc, argv, a);
    if (pr != 0) {
        if (pr == 1) std::cerr << kHelp;
        return 1;
    }
    return run(a);
}
