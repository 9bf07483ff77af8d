// bnet front end: text -> per-node DNF clauses (host C++).
//
// Follows the reference's model_builder (cuda/src/model.cpp:80-125):
//   * the first line is skipped only when it starts with "targets";
//   * each following line is "target, expression": the target is the text before
//     the first comma (kept verbatim), the expression starts at the first
//     non-space character after it;
//   * lines are consumed while the stream is not at EOF, so an unterminated last
//     line is dropped exactly as the reference's while(!f.eof()) loop does.
// Expressions use the grammar of boolstuff::BoolExprParser
// (cuda/src/boolstuff/BoolExprParser.cpp:65-160): expr := term ['|' expr],
// term := factor ['&' term], factor := '!'* atom, atom := '(' expr ')' | identifier,
// identifiers [A-Za-z0-9_]+, whitespace skipped.
// The DNF keeps boolstuff's simplification that matters for the clauses
// (cuda/src/boolstuff/BoolExpr.tpp:482-560): duplicate literals and duplicate
// terms are removed, contradictory terms (x & !x) are dropped unless the rule has
// a single term.  Identifiers that are not node names are then dropped from each
// clause (cuda/src/model.cpp:59-67), which is why the DNF, not the truth function,
// defines the table.  A rule whose every term is contradictory is unambiguous only
// when each contradiction involves a node (the clause is never true); otherwise the
// surviving term depends on boolstuff's internal term order and the rule is rejected.
#include <algorithm>
#include <cctype>
#include <map>
#include <memory>
#include <sstream>

#include "esl_internal.h"

namespace esl {
namespace {

// Terms over identifier ids: ids < n are nodes, ids >= n are other identifiers.
struct Lits {
    uint64_t pos = 0, neg = 0;
    bool operator<(const Lits& o) const { return pos != o.pos ? pos < o.pos : neg < o.neg; }
    bool operator==(const Lits& o) const { return pos == o.pos && neg == o.neg; }
};

constexpr size_t kTermLimit = 1u << 20;

class RuleParser {
  public:
    // ids: node name -> node index; identifiers that are not nodes get ids from n up.
    RuleParser(const std::string& text, const std::map<std::string, int>& ids, int n)
        : s_(text), ids_(ids), next_id_(n) {}

    std::vector<Lits> parse() {
        auto t = texpr();
        ws();
        if (i_ != s_.size()) throw std::runtime_error("garbage at end of expression");
        return to_dnf(t.get(), false);
    }

  private:
    std::string s_;
    size_t i_ = 0;
    std::map<std::string, int> ids_;
    int next_id_;

    void ws() {
        while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
    }
    bool peek(char c) {
        ws();
        return i_ < s_.size() && s_[i_] == c;
    }
    static std::vector<Lits> disj(std::vector<Lits> a, const std::vector<Lits>& b) {
        a.insert(a.end(), b.begin(), b.end());
        return a;
    }
    static std::vector<Lits> conj(const std::vector<Lits>& a, const std::vector<Lits>& b) {
        if (a.size() * b.size() > kTermLimit) throw std::runtime_error("DNF too large");
        std::vector<Lits> r;
        r.reserve(a.size() * b.size());
        for (const Lits& x : a)
            for (const Lits& y : b) r.push_back({x.pos | y.pos, x.neg | y.neg});
        return r;
    }
    // Parse tree; the DNF is derived from it with negations pushed to the leaves.
    // '|' and '&' chains are n-ary nodes built by loops, so the depth of the parser's
    // recursion, of the tree and of to_dnf follows the parenthesis nesting, which is
    // limited, and not the length of a chain.  Folding an n-ary node left to right
    // gives the terms in the same order as the grammar's right-recursive reading
    // (concatenation for '|', the lexicographic cross product for '&').
    struct Tree {
        int kind;  // 0 var, 1 not, 2 and, 3 or
        int id;
        std::vector<std::unique_ptr<Tree>> kids;
    };
    static constexpr int kMaxNesting = 512;
    int depth_ = 0;
    std::unique_ptr<Tree> chain(int kind, char op, std::unique_ptr<Tree> (RuleParser::*next)()) {
        auto first = (this->*next)();
        if (!peek(op)) return first;
        auto t = std::make_unique<Tree>();
        t->kind = kind;
        t->kids.push_back(std::move(first));
        while (peek(op)) {
            ++i_;
            t->kids.push_back((this->*next)());
        }
        return t;
    }
    std::unique_ptr<Tree> texpr() { return chain(3, '|', &RuleParser::tterm); }
    std::unique_ptr<Tree> tterm() { return chain(2, '&', &RuleParser::tfactor); }
    std::unique_ptr<Tree> tfactor() {
        int nots = 0;
        while (peek('!')) {
            ++i_;
            ++nots;
        }
        auto a = tatom();
        if (nots % 2 == 0) return a;
        auto t = std::make_unique<Tree>();
        t->kind = 1;
        t->kids.push_back(std::move(a));
        return t;
    }
    std::unique_ptr<Tree> tatom() {
        if (peek('(')) {
            ++i_;
            if (++depth_ > kMaxNesting) throw std::runtime_error("expression nested too deeply");
            auto e = texpr();
            if (!peek(')')) throw std::runtime_error("runaway parenthesis");
            ++i_;
            --depth_;
            return e;
        }
        ws();
        size_t b = i_;
        while (i_ < s_.size() && (std::isalnum((unsigned char)s_[i_]) || s_[i_] == '_')) ++i_;
        if (i_ == b) throw std::runtime_error("identifier expected");
        std::string name = s_.substr(b, i_ - b);
        auto it = ids_.find(name);
        int id;
        if (it == ids_.end()) {
            id = next_id_++;
            if (id >= 64) throw std::runtime_error("too many distinct identifiers in one rule");
            ids_[name] = id;
        } else {
            id = it->second;
        }
        auto t = std::make_unique<Tree>();
        t->kind = 0;
        t->id = id;
        return t;
    }
    static std::vector<Lits> to_dnf(const Tree* t, bool neg) {
        switch (t->kind) {
            case 0: {
                Lits l;
                (neg ? l.neg : l.pos) = 1ull << t->id;
                return {l};
            }
            case 1:
                return to_dnf(t->kids[0].get(), !neg);
            default: {
                bool is_or = (t->kind == 3) != neg;
                auto acc = to_dnf(t->kids[0].get(), neg);
                for (size_t k = 1; k < t->kids.size(); k++) {
                    auto b = to_dnf(t->kids[k].get(), neg);
                    acc = is_or ? disj(std::move(acc), b) : conj(acc, b);
                }
                return acc;
            }
        }
    }
};

std::vector<Clause> rule_to_clauses(const std::string& rule, const std::map<std::string, int>& ids, int n) {
    RuleParser p(rule, ids, n);
    std::vector<Lits> terms = p.parse();
    const uint64_t node_mask = (n >= 64) ? ~0ull : ((1ull << n) - 1);
    auto clause = [&](const Lits& l) { return Clause{(uint32_t)(l.pos & node_mask), (uint32_t)(l.neg & node_mask)}; };
    std::vector<Clause> out;
    if (terms.size() == 1) {
        out.push_back(clause(terms[0]));
        return out;
    }
    std::sort(terms.begin(), terms.end());
    terms.erase(std::unique(terms.begin(), terms.end()), terms.end());
    bool any_useful = false;
    for (const Lits& t : terms)
        if ((t.pos & t.neg) == 0) {
            out.push_back(clause(t));
            any_useful = true;
        }
    if (any_useful) return out;
    for (const Lits& t : terms)
        if ((t.pos & t.neg & node_mask) == 0)
            throw std::runtime_error("contradictory rule over identifiers that are not nodes");
    out.push_back(clause(terms[0]));
    return out;
}

}  // namespace

int parse_bnet(const std::string& text, Model& out) {
    try {
        std::istringstream in(text);
        std::string line;
        std::getline(in, line);
        if (line.rfind("targets", 0) == 0) std::getline(in, line);
        std::vector<std::string> targets, rules;
        while (!in.eof()) {
            size_t comma = line.find(',');
            targets.push_back(line.substr(0, comma));
            size_t start = line.find_first_not_of(' ', comma + 1);
            rules.push_back(start == std::string::npos ? std::string() : line.substr(start));
            std::getline(in, line);
        }
        if (targets.empty()) return fail(ESL_ERR_PARSE, "model has no nodes");
        if ((int)targets.size() > ESL_MAX_NODES)
            return fail(ESL_ERR_TOO_LARGE, "model has more than 30 nodes");
        // a node name maps to its first line index, as the reference's lookup over
        // the target list does
        std::map<std::string, int> ids;
        for (size_t i = 0; i < targets.size(); i++)
            if (!ids.count(targets[i])) ids[targets[i]] = (int)i;
        Model m;
        m.names = targets;
        for (const std::string& r : rules) m.rules.push_back(rule_to_clauses(r, ids, (int)targets.size()));
        out = std::move(m);
        return ESL_OK;
    } catch (std::exception& e) {
        return fail(ESL_ERR_PARSE, e.what());
    }
}

}  // namespace esl
