// ExaStoLog CPU FP64 oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// This file restates, on the CPU and in FP64, the algorithm of the reference's
// stationary-distribution path (asmelko/paraExaStoLog).  It exists only to check
// the CUDA implementation: only the tests, the smoke check and the benchmark's
// CPU-baseline leg may load it.  Nothing in the product links or calls it.
//
// Parity is pinned against the reference's own known-answer tests
// (cuda/test/test.cu) by tests/test_oracle_golden.py.
//
// What each part follows:
//   bnet reading        cuda/src/model.cpp:80-125 (header skip, "name, expr" split,
//                       unterminated last line dropped by the while(!eof) loop)
//   expression grammar  cuda/src/boolstuff/BoolExprParser.cpp:65-160
//   DNF and clauses     cuda/src/boolstuff/BoolExpr.tpp:482-560 (contradictory and
//                       duplicate terms removed), cuda/src/model.cpp:35-78 (identifiers
//                       that are not nodes are dropped from a clause)
//   transitions         cuda/src/transition_table.cu:76-119 (a flip exists iff the
//                       rule disagrees with the bit and that direction's rate != 0)
//   generator           cuda/src/kernels/solver.cu:20-44 (K[dst,src] = rate,
//                       diagonal = -column sum); rate index 2*node + (up ? 0 : 1)
//   SCC levels/order    cuda/src/transition_graph.cu:76-202 and
//                       cuda/src/kernels/transition_graph.cu:3-27 (level 1 = terminal,
//                       level = 1 + max successor level; terminals first, the rest by
//                       decreasing level)
//   R, L, x_inf         cuda/src/solver.cu:102-309 (R = terminal kernels, L = [U | X]
//                       absorption probabilities, x_inf = R (L x0))
//   initial state       cuda/src/initial_state.cu:7-60
//   normal rates        cuda/src/transition_rates.cpp:24-97 (eo_rates_normal)
//
// Numerics: terminal kernels solve K_C pi = 0 with one row replaced by the
// normalisation row (dense LU with partial pivoting); the transient part is the
// block-triangular solve over SCCs in topological order with a dense LU per SCC
// block.  Blocks larger than kDenseMax states are solved by FP64 BiCGStab with a
// Jacobi preconditioner to a relative residual of 1e-14 -- not the reference's
// algorithm (its dense/host LU has no feasible fill at that size); results at that
// scale are flagged through eo_iterative_blocks() and eo_last_relres().  Terminal
// SCCs of that size solve the rank-one deflated system (-K_C + u 1^T) pi = u,
// which has the same solution as the row-replaced one (see terminal_kernel).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr int kDenseMax = 2048;

// ---------------------------------------------------------------- expression
struct Expr {
    enum Kind { VAR, NOT, AND, OR } kind;
    std::string name;
    std::unique_ptr<Expr> a, b;
};
using ExprP = std::unique_ptr<Expr>;

struct Parser {
    std::string s;
    size_t i = 0;
    void skip() { while (i < s.size() && std::isspace((unsigned char)s[i])) i++; }
    bool seen(char c) { skip(); return i < s.size() && s[i] == c; }
    ExprP expr() {
        ExprP l = term();
        if (!seen('|')) return l;
        i++;
        ExprP e(new Expr{Expr::OR, "", std::move(l), expr()});
        return e;
    }
    ExprP term() {
        ExprP l = factor();
        if (!seen('&')) return l;
        i++;
        ExprP e(new Expr{Expr::AND, "", std::move(l), term()});
        return e;
    }
    ExprP factor() {
        bool pos = true;
        while (seen('!')) { i++; pos = !pos; }
        ExprP at = atom();
        if (pos) return at;
        ExprP e(new Expr{Expr::NOT, "", nullptr, std::move(at)});
        return e;
    }
    ExprP atom() {
        skip();
        if (seen('(')) {
            i++;
            ExprP e = expr();
            if (!seen(')')) throw std::runtime_error("runaway parenthesis");
            i++;
            return e;
        }
        skip();
        size_t st = i;
        while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '_')) i++;
        if (i == st) throw std::runtime_error("identifier expected");
        ExprP e(new Expr{Expr::VAR, s.substr(st, i - st), nullptr, nullptr});
        return e;
    }
    ExprP parse(const std::string& text) {
        s = text; i = 0;
        ExprP e = expr();
        skip();
        if (i != s.size()) throw std::runtime_error("garbage at end of expression");
        return e;
    }
};

struct Term {
    std::set<std::string> pos, neg;
    bool operator<(const Term& o) const { return pos != o.pos ? pos < o.pos : neg < o.neg; }
    bool operator==(const Term& o) const { return pos == o.pos && neg == o.neg; }
};

constexpr size_t kMaxTerms = 1 << 20;

std::vector<Term> dnf(const Expr* e, bool negate) {
    if (e->kind == Expr::VAR) {
        Term t;
        (negate ? t.neg : t.pos).insert(e->name);
        return {t};
    }
    if (e->kind == Expr::NOT) return dnf(e->b.get(), !negate);
    bool is_or = (e->kind == Expr::OR) != negate;  // De Morgan
    std::vector<Term> l = dnf(e->a.get(), negate), r = dnf(e->b.get(), negate);
    if (is_or) {
        l.insert(l.end(), r.begin(), r.end());
        return l;
    }
    if (l.size() * r.size() > kMaxTerms) throw std::runtime_error("DNF too large");
    std::vector<Term> out;
    out.reserve(l.size() * r.size());
    for (auto& x : l)
        for (auto& y : r) {
            Term t = x;
            t.pos.insert(y.pos.begin(), y.pos.end());
            t.neg.insert(y.neg.begin(), y.neg.end());
            out.push_back(std::move(t));
        }
    return out;
}

bool useful(const Term& t) {
    for (auto& v : t.pos)
        if (t.neg.count(v)) return false;
    return true;
}

struct Clause { uint32_t pos, neg; };

struct Model {
    std::vector<std::string> names;
    std::vector<std::vector<Clause>> rules;
    int n() const { return (int)names.size(); }
};

Clause to_clause(const Term& t, const std::vector<std::string>& targets) {
    Clause c{0, 0};
    for (size_t i = 0; i < targets.size(); i++) {
        if (t.pos.count(targets[i])) c.pos |= 1u << i;
        if (t.neg.count(targets[i])) c.neg |= 1u << i;
    }
    return c;
}

std::vector<Clause> rule_clauses(const std::string& factor, const std::vector<std::string>& targets) {
    Parser p;
    ExprP e = p.parse(factor);
    std::vector<Term> terms = dnf(e.get(), false);
    std::vector<Clause> out;
    if (terms.size() == 1) {  // a single term is kept even when contradictory
        out.push_back(to_clause(terms[0], targets));
        return out;
    }
    std::sort(terms.begin(), terms.end());
    std::vector<Term> keep;
    for (size_t k = 0; k < terms.size(); k++) {
        if (k > 0 && terms[k] == terms[k - 1]) continue;
        if (useful(terms[k])) keep.push_back(terms[k]);
    }
    if (keep.empty()) {
        // Every term contradictory.  Unambiguous only if each contradiction
        // involves a node (the clause can never be true).
        for (auto& t : terms) {
            Clause c = to_clause(t, targets);
            if ((c.pos & c.neg) == 0)
                throw std::runtime_error("contradictory rule over identifiers that are not nodes");
        }
        out.push_back(to_clause(terms[0], targets));
        return out;
    }
    for (auto& t : keep) out.push_back(to_clause(t, targets));
    return out;
}

Model parse_bnet_stream(std::istream& f) {
    std::string line;
    std::getline(f, line);
    if (line.rfind("targets", 0) == 0) std::getline(f, line);
    std::vector<std::string> targets, factors;
    while (!f.eof()) {
        size_t te = line.find(',');
        std::string target = line.substr(0, te);
        size_t fs = line.find_first_not_of(' ', te + 1);
        std::string factor = fs == std::string::npos ? std::string() : line.substr(fs);
        targets.push_back(target);
        factors.push_back(factor);
        std::getline(f, line);
    }
    if (targets.size() > 30) throw std::runtime_error("more than 30 nodes");
    Model m;
    m.names = targets;
    for (auto& fa : factors) m.rules.push_back(rule_clauses(fa, targets));
    return m;
}

// ---------------------------------------------------------------- graph
inline bool rule_value(const std::vector<Clause>& cl, uint32_t s) {
    for (auto& c : cl)
        if ((s & c.pos) == c.pos && (s & c.neg) == 0) return true;
    return false;
}

// out-flip mask: bit i set iff the edge s -> s ^ (1 << i) exists
std::vector<uint32_t> flip_masks(const Model& m, const double* rates) {
    int n = m.n();
    uint64_t N = 1ull << n;
    std::vector<uint32_t> F(N, 0);
    for (int i = 0; i < n; i++) {
        bool up_ok = rates[2 * i] != 0.0, down_ok = rates[2 * i + 1] != 0.0;
        if (!up_ok && !down_ok) continue;
        for (uint64_t s = 0; s < N; s++) {
            bool f = rule_value(m.rules[i], (uint32_t)s);
            bool bit = (s >> i) & 1;
            if ((f && !bit && up_ok) || (!f && bit && down_ok)) F[s] |= 1u << i;
        }
    }
    return F;
}

inline double edge_rate(const double* rates, uint32_t src, int i) {
    return ((src >> i) & 1) ? rates[2 * i + 1] : rates[2 * i];
}

struct Sym {
    int n = 0;
    uint64_t N = 0;
    std::vector<uint32_t> F;          // out-flip masks
    std::vector<int32_t> scc_of;      // SCC index (in Tarjan completion order)
    std::vector<int32_t> scc_min;     // canonical label: min vertex of each SCC
    std::vector<int32_t> scc_level;
    std::vector<int32_t> order;       // reordered vertices
    std::vector<int32_t> offsets;     // SCC offsets in the order
    std::vector<int32_t> scc_at;      // SCC index at each position of offsets
    int n_sccs = 0, T = 0;
};

void tarjan(Sym& g) {
    uint64_t N = g.N;
    int n = g.n;
    std::vector<int32_t> index(N, -1), low(N, 0);
    std::vector<char> on_stack(N, 0);
    std::vector<int32_t> stack;
    struct Frame { uint32_t v; int next_bit; };
    std::vector<Frame> call;
    int32_t counter = 0;
    g.scc_of.assign(N, -1);
    for (uint64_t root = 0; root < N; root++) {
        if (index[root] >= 0) continue;
        call.push_back({(uint32_t)root, 0});
        index[root] = low[root] = counter++;
        stack.push_back((int32_t)root);
        on_stack[root] = 1;
        while (!call.empty()) {
            Frame& fr = call.back();
            uint32_t v = fr.v;
            bool descended = false;
            while (fr.next_bit < n) {
                int i = fr.next_bit++;
                if (!((g.F[v] >> i) & 1)) continue;
                uint32_t w = v ^ (1u << i);
                if (index[w] < 0) {
                    index[w] = low[w] = counter++;
                    stack.push_back((int32_t)w);
                    on_stack[w] = 1;
                    call.push_back({w, 0});
                    descended = true;
                    break;
                } else if (on_stack[w]) {
                    low[v] = std::min(low[v], index[w]);
                }
            }
            if (descended) continue;
            if (low[v] == index[v]) {
                int32_t id = g.n_sccs++;
                int32_t mn = INT32_MAX;
                while (true) {
                    int32_t w = stack.back();
                    stack.pop_back();
                    on_stack[w] = 0;
                    g.scc_of[w] = id;
                    mn = std::min(mn, w);
                    if ((uint32_t)w == v) break;
                }
                g.scc_min.push_back(mn);
            }
            call.pop_back();
            if (!call.empty()) {
                uint32_t p = call.back().v;
                low[p] = std::min(low[p], low[v]);
            }
        }
    }
}

void levels_and_order(Sym& g) {
    int C = g.n_sccs;
    // Tarjan completes every SCC after all SCCs it reaches, so completion order
    // is a reverse topological order: successors' levels are final when read.
    std::vector<std::vector<int32_t>> members(C);
    for (uint64_t v = 0; v < g.N; v++) members[g.scc_of[v]].push_back((int32_t)v);
    g.scc_level.assign(C, 1);
    for (int c = 0; c < C; c++) {
        int lvl = 0;
        for (int32_t v : members[c])
            for (int i = 0; i < g.n; i++)
                if ((g.F[v] >> i) & 1) {
                    int32_t d = g.scc_of[v ^ (1u << i)];
                    if (d != c) lvl = std::max(lvl, g.scc_level[d]);
                }
        g.scc_level[c] = lvl + 1;
    }
    std::vector<int32_t> sccs(C);
    for (int c = 0; c < C; c++) sccs[c] = c;
    std::sort(sccs.begin(), sccs.end(), [&](int32_t a, int32_t b) {
        bool ta = g.scc_level[a] == 1, tb = g.scc_level[b] == 1;
        if (ta != tb) return ta;
        if (ta) return g.scc_min[a] < g.scc_min[b];
        if (g.scc_level[a] != g.scc_level[b]) return g.scc_level[a] > g.scc_level[b];
        return g.scc_min[a] > g.scc_min[b];
    });
    g.T = 0;
    g.order.clear();
    g.offsets.assign(1, 0);
    g.scc_at.clear();
    for (int32_t c : sccs) {
        if (g.scc_level[c] == 1) g.T++;
        for (int32_t v : members[c]) g.order.push_back(v);  // members are ascending
        g.offsets.push_back((int32_t)g.order.size());
        g.scc_at.push_back(c);
    }
}

// ---------------------------------------------------------------- numerics
// Dense solve A X = B (A s x s row-major, B s x r row-major) with partial pivoting.
void dense_solve(std::vector<double>& A, std::vector<double>& B, int s, int r) {
    for (int k = 0; k < s; k++) {
        int p = k;
        double best = std::fabs(A[(size_t)k * s + k]);
        for (int i = k + 1; i < s; i++) {
            double v = std::fabs(A[(size_t)i * s + k]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0.0) throw std::runtime_error("singular block");
        if (p != k) {
            for (int j = 0; j < s; j++) std::swap(A[(size_t)k * s + j], A[(size_t)p * s + j]);
            for (int j = 0; j < r; j++) std::swap(B[(size_t)k * r + j], B[(size_t)p * r + j]);
        }
        double piv = A[(size_t)k * s + k];
        for (int i = k + 1; i < s; i++) {
            double f = A[(size_t)i * s + k] / piv;
            if (f == 0.0) continue;
            A[(size_t)i * s + k] = 0.0;
            for (int j = k + 1; j < s; j++) A[(size_t)i * s + j] -= f * A[(size_t)k * s + j];
            for (int j = 0; j < r; j++) B[(size_t)i * r + j] -= f * B[(size_t)k * r + j];
        }
    }
    for (int k = s - 1; k >= 0; k--) {
        for (int j = 0; j < r; j++) {
            double acc = B[(size_t)k * r + j];
            for (int c = k + 1; c < s; c++) acc -= A[(size_t)k * s + c] * B[(size_t)c * r + j];
            B[(size_t)k * r + j] = acc / A[(size_t)k * s + k];
        }
    }
}

// Sparse block operator over a set of states `mem` (local index by `loc`).
// transpose=false: (Q x)(a) = q_a x_a - sum_{b in block} rate(a->b) x_b   (backward/absorption)
// transpose=true : (Q^T x)(a) = q_a x_a - sum_{b in block} rate(b->a) x_b (forward/occupation)
struct BlockOp {
    const Sym* g;
    const double* rates;
    const std::vector<int32_t>* mem;
    const std::vector<int32_t>* loc;  // global -> local, -1 outside the block
    bool transpose;
    std::vector<double> diag;
    std::vector<double> u;  // optional rank-one term: y += u * (1^T x)
    void init() {
        diag.resize(mem->size());
        for (size_t a = 0; a < mem->size(); a++) {
            uint32_t v = (uint32_t)(*mem)[a];
            double q = 0;
            for (int i = 0; i < g->n; i++)
                if ((g->F[v] >> i) & 1) q += edge_rate(rates, v, i);
            diag[a] = q;
        }
    }
    void apply(const std::vector<double>& x, std::vector<double>& y) const {
        for (size_t a = 0; a < mem->size(); a++) {
            uint32_t v = (uint32_t)(*mem)[a];
            double acc = diag[a] * x[a];
            for (int i = 0; i < g->n; i++) {
                uint32_t w = v ^ (1u << i);
                int32_t b = (*loc)[w];
                if (b < 0) continue;
                if (!transpose) {
                    if ((g->F[v] >> i) & 1) acc -= edge_rate(rates, v, i) * x[b];
                } else {
                    if ((g->F[w] >> i) & 1) acc -= edge_rate(rates, w, i) * x[b];
                }
            }
            y[a] = acc;
        }
        if (!u.empty()) {
            double sx = 0;
            for (double xv : x) sx += xv;
            for (size_t a = 0; a < u.size(); a++) y[a] += u[a] * sx;
        }
    }
};

double g_last_relres = 0.0;
int g_iter_blocks = 0;

// Jacobi-preconditioned BiCGStab, FP64.  The true residual is recomputed at
// every restart; the solve stops at `tol` or when a restart no longer halves it.
void bicgstab(const BlockOp& A, const std::vector<double>& b, std::vector<double>& x, double tol, int maxit) {
    size_t m = b.size();
    auto dot = [&](const std::vector<double>& u, const std::vector<double>& v) {
        double s = 0; for (size_t i = 0; i < m; i++) s += u[i] * v[i]; return s; };
    double bn = std::sqrt(dot(b, b));
    if (bn == 0) { std::fill(x.begin(), x.end(), 0.0); return; }
    std::vector<double> r(m), r0(m), p(m), v(m), s(m), t(m), ph(m), sh(m), Ax(m);
    int it = 0;
    double rel = 1, prev_rel = 2;
    while (true) {
        A.apply(x, Ax);
        for (size_t i = 0; i < m; i++) r[i] = b[i] - Ax[i];
        rel = std::sqrt(dot(r, r)) / bn;
        if (rel <= tol || it >= maxit || rel > 0.5 * prev_rel) break;
        prev_rel = rel;
        r0 = r;
        double rho = 1, alpha = 1, omega = 1;
        std::fill(v.begin(), v.end(), 0.0);
        std::fill(p.begin(), p.end(), 0.0);
        for (; it < maxit;) {
            double rho1 = dot(r0, r);
            if (rho1 == 0 || !std::isfinite(rho1)) break;
            double beta = (rho1 / rho) * (alpha / omega);
            for (size_t i = 0; i < m; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
            for (size_t i = 0; i < m; i++) ph[i] = p[i] / A.diag[i];
            A.apply(ph, v);
            double r0v = dot(r0, v);
            if (r0v == 0 || !std::isfinite(r0v)) break;
            alpha = rho1 / r0v;
            for (size_t i = 0; i < m; i++) s[i] = r[i] - alpha * v[i];
            it++;
            if (std::sqrt(dot(s, s)) / bn <= 0.1 * tol) {
                for (size_t i = 0; i < m; i++) x[i] += alpha * ph[i];
                break;
            }
            for (size_t i = 0; i < m; i++) sh[i] = s[i] / A.diag[i];
            A.apply(sh, t);
            double tt = dot(t, t);
            omega = tt == 0 ? 0 : dot(t, s) / tt;
            for (size_t i = 0; i < m; i++) x[i] += alpha * ph[i] + omega * sh[i];
            for (size_t i = 0; i < m; i++) r[i] = s[i] - omega * t[i];
            rho = rho1;
            if (std::sqrt(dot(r, r)) / bn <= 0.1 * tol || omega == 0) break;
        }
    }
    g_last_relres = std::max(g_last_relres, rel);
}

// Solve the block system for several right-hand sides (columns of rhs, size s x r).
void block_solve(const Sym& g, const double* rates, const std::vector<int32_t>& mem,
                 std::vector<int32_t>& loc, bool transpose, std::vector<double>& rhs, int r) {
    int s = (int)mem.size();
    for (int a = 0; a < s; a++) loc[mem[a]] = a;
    BlockOp op{&g, rates, &mem, &loc, transpose, {}, {}};
    op.init();
    if (s <= kDenseMax) {
        std::vector<double> A((size_t)s * s, 0.0);
        for (int a = 0; a < s; a++) {
            uint32_t v = (uint32_t)mem[a];
            A[(size_t)a * s + a] = op.diag[a];
            for (int i = 0; i < g.n; i++) {
                uint32_t w = v ^ (1u << i);
                int32_t b = loc[w];
                if (b < 0) continue;
                if (!transpose) {
                    if ((g.F[v] >> i) & 1) A[(size_t)a * s + b] -= edge_rate(rates, v, i);
                } else {
                    if ((g.F[w] >> i) & 1) A[(size_t)a * s + b] -= edge_rate(rates, w, i);
                }
            }
        }
        dense_solve(A, rhs, s, r);
    } else {
        g_iter_blocks++;
        std::vector<double> bcol(s), xcol(s);
        for (int j = 0; j < r; j++) {
            for (int a = 0; a < s; a++) bcol[a] = rhs[(size_t)a * r + j];
            std::fill(xcol.begin(), xcol.end(), 0.0);
            bicgstab(op, bcol, xcol, 1e-14, 50000);
            for (int a = 0; a < s; a++) rhs[(size_t)a * r + j] = xcol[a];
        }
    }
    for (int a = 0; a < s; a++) loc[mem[a]] = -1;
}

// Terminal kernel of SCC `mem` (K_C pi = 0, sum pi = 1).
std::vector<double> terminal_kernel(const Sym& g, const double* rates, const std::vector<int32_t>& mem,
                                    std::vector<int32_t>& loc) {
    int s = (int)mem.size();
    if (s == 1) return {1.0};
    for (int a = 0; a < s; a++) loc[mem[a]] = a;
    std::vector<double> pi(s);
    if (s <= kDenseMax) {
        // rows = equations over destination states: sum_b K[a,b] pi_b = 0; last row -> ones
        std::vector<double> A((size_t)s * s, 0.0), B(s, 0.0);
        for (int b = 0; b < s; b++) {
            uint32_t v = (uint32_t)mem[b];
            for (int i = 0; i < g.n; i++)
                if ((g.F[v] >> i) & 1) {
                    int32_t a = loc[v ^ (1u << i)];
                    double rt = edge_rate(rates, v, i);
                    A[(size_t)a * s + b] += rt;
                    A[(size_t)b * s + b] -= rt;
                }
        }
        for (int b = 0; b < s; b++) A[(size_t)(s - 1) * s + b] = 1.0;
        B[s - 1] = 1.0;
        dense_solve(A, B, s, 1);
        pi = B;
    } else {
        // Rank-one deflation: (-K_C + u 1^T) pi = u.  Because 1^T K_C = 0, any solution
        // has 1^T pi = 1 and K_C pi = 0, the same kernel as the row-replaced system
        // above.  The simple zero eigenvalue of -K_C moves to 1^T u and every other
        // eigenvalue stays where it was (Brauer's theorem on the left eigenvector 1), so
        // the conditioning follows the chain's spectral gap.  Fixing one state to 1
        // instead makes the solution scale with 1 / pi(pinned state), which reached
        // 1e78 on a 262,144-state attractor, with a residual relative to b that says
        // nothing about the normalised kernel.  u = q / s puts 1^T u at the mean out-rate.
        g_iter_blocks++;
        BlockOp op{&g, rates, &mem, &loc, true, {}, {}};
        op.init();
        op.u.resize(s);
        for (int a = 0; a < s; a++) op.u[a] = op.diag[a] / s;
        std::vector<double> x(s, 1.0 / s);
        bicgstab(op, op.u, x, 1e-14, 50000);
        pi = x;
    }
    for (int a = 0; a < s; a++) loc[mem[a]] = -1;
    double sum = 0;
    for (double v : pi) sum += std::fabs(v);
    for (double& v : pi) v = std::fabs(v) / sum;
    return pi;
}

struct Result {
    std::vector<double> R;        // terminal kernel values, aligned with order[0:terminal states]
    std::vector<double> L;        // T x N absorption matrix by original state (optional)
    std::vector<double> y;        // per x0: T masses
    std::vector<double> x_inf;    // per x0: N
    std::vector<double> marg;     // per x0: n
};

struct Net {
    Model model;
    std::string error;
};

std::string g_error;

Sym build_sym(const Model& m, const double* rates) {
    Sym g;
    g.n = m.n();
    g.N = 1ull << g.n;
    g.F = flip_masks(m, rates);
    tarjan(g);
    levels_and_order(g);
    return g;
}

// Terminal-state bookkeeping shared by the solvers.
struct TermInfo {
    std::vector<int32_t> term_of;   // terminal index per state, -1 for transient
    int32_t term_states = 0;
};

TermInfo term_info(const Sym& g) {
    TermInfo ti;
    ti.term_of.assign(g.N, -1);
    for (int t = 0; t < g.T; t++)
        for (int32_t p = g.offsets[t]; p < g.offsets[t + 1]; p++) ti.term_of[g.order[p]] = t;
    ti.term_states = g.offsets[g.T];
    return ti;
}

std::vector<double> all_terminal_kernels(const Sym& g, const double* rates) {
    std::vector<int32_t> loc(g.N, -1);
    std::vector<double> R(g.offsets[g.T]);
    for (int t = 0; t < g.T; t++) {
        std::vector<int32_t> mem(g.order.begin() + g.offsets[t], g.order.begin() + g.offsets[t + 1]);
        std::vector<double> pi = terminal_kernel(g, rates, mem, loc);
        for (size_t a = 0; a < pi.size(); a++) R[g.offsets[t] + a] = pi[a];
    }
    return R;
}

// Backward formulation: L[t, s] = probability of absorption into terminal t from s.
std::vector<double> absorption(const Sym& g, const double* rates, const TermInfo& ti) {
    int T = g.T;
    std::vector<double> L((size_t)T * g.N, 0.0);
    for (uint64_t s = 0; s < g.N; s++)
        if (ti.term_of[s] >= 0) L[(size_t)ti.term_of[s] * g.N + s] = 1.0;
    std::vector<int32_t> loc(g.N, -1);
    int nscc = (int)g.offsets.size() - 1;
    for (int c = nscc - 1; c >= T; c--) {
        std::vector<int32_t> mem(g.order.begin() + g.offsets[c], g.order.begin() + g.offsets[c + 1]);
        int s = (int)mem.size();
        std::vector<char> inblk(0);
        std::vector<double> rhs((size_t)s * T, 0.0);
        for (int a = 0; a < s; a++) loc[mem[a]] = a;
        for (int a = 0; a < s; a++) {
            uint32_t v = (uint32_t)mem[a];
            for (int i = 0; i < g.n; i++)
                if ((g.F[v] >> i) & 1) {
                    uint32_t w = v ^ (1u << i);
                    if (loc[w] >= 0) continue;
                    double rt = edge_rate(rates, v, i);
                    for (int t = 0; t < T; t++) rhs[(size_t)a * T + t] += rt * L[(size_t)t * g.N + w];
                }
        }
        for (int a = 0; a < s; a++) loc[mem[a]] = -1;
        block_solve(g, rates, mem, loc, false, rhs, T);
        for (int a = 0; a < s; a++)
            for (int t = 0; t < T; t++) L[(size_t)t * g.N + mem[a]] = rhs[(size_t)a * T + t];
    }
    return L;
}

// Forward formulation: occupation z of the transient states, then the mass y_t
// that enters each terminal SCC.
std::vector<double> terminal_mass(const Sym& g, const double* rates, const TermInfo& ti, const double* x0) {
    int T = g.T;
    std::vector<double> z(g.N, 0.0), y(T, 0.0);
    std::vector<int32_t> loc(g.N, -1);
    int nscc = (int)g.offsets.size() - 1;
    for (uint64_t s = 0; s < g.N; s++)
        if (ti.term_of[s] >= 0) y[ti.term_of[s]] += x0[s];
    for (int c = T; c < nscc; c++) {
        std::vector<int32_t> mem(g.order.begin() + g.offsets[c], g.order.begin() + g.offsets[c + 1]);
        int s = (int)mem.size();
        std::vector<double> rhs(s, 0.0);
        for (int a = 0; a < s; a++) loc[mem[a]] = a;
        for (int a = 0; a < s; a++) {
            uint32_t v = (uint32_t)mem[a];
            double acc = x0[v];
            for (int i = 0; i < g.n; i++) {
                uint32_t w = v ^ (1u << i);
                if (loc[w] >= 0 || ti.term_of[w] >= 0) continue;
                if ((g.F[w] >> i) & 1) acc += edge_rate(rates, w, i) * z[w];
            }
            rhs[a] = acc;
        }
        for (int a = 0; a < s; a++) loc[mem[a]] = -1;
        block_solve(g, rates, mem, loc, true, rhs, 1);
        for (int a = 0; a < s; a++) z[mem[a]] = rhs[a];
    }
    for (uint64_t v = 0; v < g.N; v++) {
        if (ti.term_of[v] >= 0 || z[v] == 0.0) continue;
        for (int i = 0; i < g.n; i++)
            if ((g.F[v] >> i) & 1) {
                int32_t t = ti.term_of[v ^ (1u << i)];
                if (t >= 0) y[t] += edge_rate(rates, (uint32_t)v, i) * z[v];
            }
    }
    return y;
}

void finish(const Sym& g, const TermInfo& ti, const std::vector<double>& R, const double* y,
            double* x_inf, double* marg) {
    std::fill(x_inf, x_inf + g.N, 0.0);
    for (int t = 0; t < g.T; t++)
        for (int32_t p = g.offsets[t]; p < g.offsets[t + 1]; p++) x_inf[g.order[p]] = R[p] * y[t];
    if (marg) {
        std::fill(marg, marg + g.n, 0.0);
        for (uint64_t s = 0; s < g.N; s++)
            if (x_inf[s] != 0.0)
                for (int i = 0; i < g.n; i++)
                    if ((s >> i) & 1) marg[i] += x_inf[s];
    }
}

}  // namespace

// ============================================================== C ABI
extern "C" {

struct eo_net { Model model; };
struct eo_sym { Sym g; TermInfo ti; };

const char* eo_last_error() { return g_error.c_str(); }

// Returns the relative residual reached by the last iterative block solve
// (0 when every block was solved by dense LU) and the number of such blocks.
double eo_last_relres() { return g_last_relres; }
int eo_iterative_blocks() { return g_iter_blocks; }

eo_net* eo_parse_bnet(const char* text) {
    try {
        std::istringstream in(text);
        auto* net = new eo_net{parse_bnet_stream(in)};
        return net;
    } catch (std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

eo_net* eo_load_bnet(const char* path) {
    try {
        std::ifstream f(path);
        if (!f.is_open()) throw std::runtime_error("could not open model file");
        return new eo_net{parse_bnet_stream(f)};
    } catch (std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void eo_free_net(eo_net* net) { delete net; }
int eo_n(const eo_net* net) { return net->model.n(); }
const char* eo_node_name(const eo_net* net, int i) { return net->model.names[i].c_str(); }

// Clause lists: off[n+1] prefix offsets, pos/neg masks.  Returns total clause
// count; arrays are filled when cap is large enough.
int eo_clauses(const eo_net* net, int32_t* off, uint32_t* pos, uint32_t* neg, int cap) {
    int total = 0;
    for (auto& r : net->model.rules) total += (int)r.size();
    if (total > cap) return total;
    int k = 0;
    off[0] = 0;
    for (int i = 0; i < net->model.n(); i++) {
        for (auto& c : net->model.rules[i]) { pos[k] = c.pos; neg[k] = c.neg; k++; }
        off[i + 1] = k;
    }
    return total;
}

// Out-flip masks for a rate vector (bit i of F[s]: edge s -> s ^ (1 << i)).
void eo_flip_masks(const eo_net* net, const double* rates, uint32_t* F) {
    std::vector<uint32_t> f = flip_masks(net->model, rates);
    std::memcpy(F, f.data(), f.size() * 4);
}

// Transition table in CSC by source (rows = destinations, ascending within a column).
int64_t eo_table(const eo_net* net, const double* rates, int32_t* indptr, int32_t* rows, int32_t* cols) {
    std::vector<uint32_t> F = flip_masks(net->model, rates);
    int n = net->model.n();
    int64_t k = 0;
    uint64_t N = F.size();
    for (uint64_t s = 0; s < N; s++) {
        if (indptr) indptr[s] = (int32_t)k;
        uint32_t f = F[s];
        uint32_t down = f & (uint32_t)s, up = f & ~(uint32_t)s;
        for (int i = n - 1; i >= 0; i--)
            if ((down >> i) & 1) { if (rows) { rows[k] = (int32_t)(s ^ (1u << i)); cols[k] = (int32_t)s; } k++; }
        for (int i = 0; i < n; i++)
            if ((up >> i) & 1) { if (rows) { rows[k] = (int32_t)(s ^ (1u << i)); cols[k] = (int32_t)s; } k++; }
    }
    if (indptr) indptr[N] = (int32_t)k;
    return k;
}

eo_sym* eo_build(const eo_net* net, const double* rates) {
    try {
        auto* s = new eo_sym;
        s->g = build_sym(net->model, rates);
        s->ti = term_info(s->g);
        return s;
    } catch (std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}
void eo_free_sym(eo_sym* s) { delete s; }
int eo_n_sccs(const eo_sym* s) { return (int)s->g.offsets.size() - 1; }
int eo_n_terminals(const eo_sym* s) { return s->g.T; }

// order[N], offsets[n_sccs+1], level[n_sccs] (level of the SCC at each offset
// position), label[N] (min vertex of each state's SCC).
void eo_graph(const eo_sym* s, int32_t* order, int32_t* offsets, int32_t* level, int32_t* label) {
    const Sym& g = s->g;
    std::memcpy(order, g.order.data(), g.N * 4);
    std::memcpy(offsets, g.offsets.data(), g.offsets.size() * 4);
    if (level)
        for (size_t p = 0; p < g.scc_at.size(); p++) level[p] = g.scc_level[g.scc_at[p]];
    if (label)
        for (uint64_t v = 0; v < g.N; v++) label[v] = g.scc_min[g.scc_of[v]];
}

// Terminal kernels R (aligned with order[0 : offsets[T]]).
int eo_terminal_kernels(const eo_sym* s, const double* rates, double* R) {
    try {
        g_last_relres = 0; g_iter_blocks = 0;
        std::vector<double> r = all_terminal_kernels(s->g, rates);
        std::memcpy(R, r.data(), r.size() * 8);
        return 0;
    } catch (std::exception& e) { g_error = e.what(); return -1; }
}

// Dense absorption matrix L (T x N, by original state).
int eo_absorption(const eo_sym* s, const double* rates, double* L) {
    try {
        g_last_relres = 0; g_iter_blocks = 0;
        std::vector<double> l = absorption(s->g, rates, s->ti);
        std::memcpy(L, l.data(), l.size() * 8);
        return 0;
    } catch (std::exception& e) { g_error = e.what(); return -1; }
}

// Terminal masses y (T) for one x0 via the forward (occupation) formulation.
int eo_terminal_mass(const eo_sym* s, const double* rates, const double* x0, double* y) {
    try {
        g_last_relres = 0; g_iter_blocks = 0;
        std::vector<double> v = terminal_mass(s->g, rates, s->ti, x0);
        std::memcpy(y, v.data(), v.size() * 8);
        return 0;
    } catch (std::exception& e) { g_error = e.what(); return -1; }
}

// Full solve for one (rates, x0): x_inf (N) and marginals (n).  use_absorption
// selects the backward formulation (through L) instead of the forward one.
int eo_solve(const eo_sym* s, const double* rates, const double* x0, double* x_inf, double* marg,
             int use_absorption) {
    try {
        g_last_relres = 0; g_iter_blocks = 0;
        const Sym& g = s->g;
        std::vector<double> R = all_terminal_kernels(g, rates);
        std::vector<double> y(g.T, 0.0);
        if (use_absorption) {
            std::vector<double> L = absorption(g, rates, s->ti);
            for (int t = 0; t < g.T; t++) {
                double acc = 0;
                for (uint64_t v = 0; v < g.N; v++) acc += L[(size_t)t * g.N + v] * x0[v];
                y[t] = acc;
            }
        } else {
            y = terminal_mass(g, rates, s->ti, x0);
        }
        finish(g, s->ti, R, y.data(), x_inf, marg);
        return 0;
    } catch (std::exception& e) { g_error = e.what(); return -1; }
}

// Many solves sharing one symbolic analysis, spread over `threads` host threads.
// rates: B x 2n, x0: B x N (one x0 per rate set), outputs B x N and B x n.
int eo_solve_many(const eo_sym* s, int B, const double* rates, const double* x0, double* x_inf,
                  double* marg, int threads) {
    const Sym& g = s->g;
    int n = g.n;
    std::vector<std::thread> pool;
    std::vector<int> status(threads, 0);
    for (int w = 0; w < threads; w++) {
        pool.emplace_back([&, w]() {
            for (int b = w; b < B; b += threads) {
                try {
                    const double* rt = rates + (size_t)b * 2 * n;
                    std::vector<double> R = all_terminal_kernels(g, rt);
                    std::vector<double> y = terminal_mass(g, rt, s->ti, x0 + (size_t)b * g.N);
                    finish(g, s->ti, R, y.data(), x_inf + (size_t)b * g.N, marg ? marg + (size_t)b * n : nullptr);
                } catch (...) { status[w] = -1; }
            }
        });
    }
    for (auto& t : pool) t.join();
    for (int v : status)
        if (v) { g_error = "solve failed"; return -1; }
    return 0;
}

// Initial state as in cuda/src/initial_state.cu:7-60: uniform, or p/|F| on the
// states matching the fixed (node, value) pairs and (1-p)/(N-|F|) elsewhere.  The
// reference forms the fixed pattern as a sum of (1 << node) * value (:41-42), so a node
// listed twice with values 1 and 0 is fixed to 1; the same node listed twice with 1
// carries into the next bit there, which is not reproduced (bit set once).
int eo_initial_state(int n, int n_fixed, const int32_t* nodes, const int32_t* values, double p, double* x0) {
    uint64_t N = 1ull << n;
    if (n_fixed == 0) {
        for (uint64_t s = 0; s < N; s++) x0[s] = 1.0 / (double)N;
        return 0;
    }
    uint64_t mask = 0, val = 0;
    for (int k = 0; k < n_fixed; k++) {
        mask |= 1ull << nodes[k];
        if (values[k]) val |= 1ull << nodes[k];
    }
    uint64_t match = 0;
    std::vector<char> m(N, 1);
    for (uint64_t s = 0; s < N; s++) {
        m[s] = (s & mask) == val;
        match += m[s];
    }
    for (uint64_t s = 0; s < N; s++)
        x0[s] = m[s] ? p / (double)match : (1.0 - p) / (double)(N - match);
    return 0;
}

// Rates as in transition_rates::generate_normal (cuda/src/transition_rates.cpp:75-97)
// through transition_rates::generate (:24-55): a default-constructed
// std::default_random_engine (or one seeded with `seed` when it is not 0), a float
// normal distribution, a negative draw redrawn up to 1000 times; nodes in order, up
// before down, and a node's explicit rate (up_set / down_set >= 0: its value) takes no
// draw.  Returns -1 when 1000 draws stay negative.
int eo_rates_normal(int n, double mean, double stddev, uint64_t seed, const double* up_set, const double* down_set,
                    double* out) {
    std::default_random_engine gen;
    if (seed) gen.seed((std::default_random_engine::result_type)seed);
    std::normal_distribution<float> dist((float)mean, (float)stddev);
    auto draw = [&](double& v) {
        float x;
        int count = 0;
        do {
            x = dist(gen);
            count++;
        } while (x < 0 && count < 1000);
        v = x;
        return x >= 0;
    };
    for (int i = 0; i < n; i++) {
        if (up_set[i] >= 0) out[2 * i] = up_set[i];
        else if (!draw(out[2 * i])) { g_error = "could not generate positive transition rates"; return -1; }
        if (down_set[i] >= 0) out[2 * i + 1] = down_set[i];
        else if (!draw(out[2 * i + 1])) { g_error = "could not generate positive transition rates"; return -1; }
    }
    return 0;
}

}  // extern "C"
