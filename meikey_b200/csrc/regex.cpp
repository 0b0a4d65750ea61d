// Regex -> DFA over the 64 base64 values, in the GPU table layout (the host side of regex
// needles: src/model/pattern/dfa.rs:52-108 Dfa::new, 189-200 gpu_table).
//
// Table: `states` rows of 65 little-endian u16.  Row s, column v (0..63) is the next state
// after the base64 character of value v; column 64 is 1 when the state accepts at the end
// of the input.  State 0 is the absorbing accept state, state 1 the start.  Matching is an
// unanchored search over the 43 characters after the fixed key prefix: `^` anchors at the
// first of them and `$` at the last.
//
// Syntax (a subset of the regex crate's, ASCII patterns): literals, `.`, classes `[...]`
// with ranges and negation, `\d`, `\w`, escaped metacharacters, groups `(...)` and `(?:...)`,
// alternation `|`, `*`, `+`, `?`, `{m}`, `{m,}`, `{m,n}`, anchors `^` `$`, and
// case-insensitive matching (letters match both cases).
//
// Construction: a Thompson NFA (one symbol edge or epsilon edges per state, anchors as
// conditional epsilon edges), then the subset construction with the start state re-added
// after every character (unanchored search), numbering DFA states in breadth-first order of
// discovery over the values 0..63.
#include <stdio.h>
#include <string.h>

#include <map>
#include <set>
#include <string>
#include <vector>

#include "../../include/meikey_b200.h"

namespace {

const char ALPHABET[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

typedef unsigned long long u64;

// a set of base64 values as a 64-bit mask
int value_of(int c) {
    const char* p = (c > 0 && c < 128) ? strchr(ALPHABET, c) : nullptr;
    return p ? (int)(p - ALPHABET) : -1;
}

bool is_alpha(int c) { return (c >= 'A' && c <= 'Z') || (c >= 'a' && c <= 'z'); }
bool is_digit(int c) { return c >= '0' && c <= '9'; }

u64 char_set(int c, bool fold) {
    u64 m = 0;
    auto add = [&](int x) {
        int v = value_of(x);
        if (v >= 0) m |= 1ull << v;
    };
    if (fold && is_alpha(c)) {
        add(c | 0x20);
        add(c & ~0x20);
    } else {
        add(c);
    }
    return m;
}

struct Node {
    enum Kind { SET, BOL, EOL, CAT, ALT, REP } kind;
    u64 set = 0;
    std::vector<Node> kids;
    int lo = 0, hi = 0;  // REP: hi < 0 means unbounded
};

struct Error {
    std::string msg;
};

struct Parser {
    const std::string& s;
    size_t i = 0;
    bool fold;
    Parser(const std::string& str, bool f) : s(str), fold(f) {}

    int peek() const { return i < s.size() ? (unsigned char)s[i] : -1; }
    int take() {
        if (i >= s.size()) throw Error{"unexpected end of pattern"};
        return (unsigned char)s[i++];
    }

    Node parse() {
        Node n = alt();
        if (peek() != -1) throw Error{std::string("unexpected '") + (char)peek() + "'"};
        return n;
    }
    Node alt() {
        std::vector<Node> parts;
        parts.push_back(concat());
        while (peek() == '|') {
            take();
            parts.push_back(concat());
        }
        if (parts.size() == 1) return parts[0];
        Node n;
        n.kind = Node::ALT;
        n.kids = std::move(parts);
        return n;
    }
    Node concat() {
        Node n;
        n.kind = Node::CAT;
        while (peek() != -1 && peek() != '|' && peek() != ')') n.kids.push_back(repeat());
        return n;
    }
    static Node rep(Node sub, int lo, int hi) {
        Node n;
        n.kind = Node::REP;
        n.lo = lo;
        n.hi = hi;
        n.kids.push_back(std::move(sub));
        return n;
    }
    Node repeat() {
        Node a = atom();
        for (;;) {
            int c = peek();
            if (c == '*') {
                take();
                a = rep(std::move(a), 0, -1);
            } else if (c == '+') {
                take();
                a = rep(std::move(a), 1, -1);
            } else if (c == '?') {
                take();
                a = rep(std::move(a), 0, 1);
            } else if (c == '{') {
                size_t j = s.find('}', i);
                if (j == std::string::npos) throw Error{"bad repetition"};
                std::string body = s.substr(i + 1, j - i - 1);
                size_t comma = body.find(',');
                std::string a_s = comma == std::string::npos ? body : body.substr(0, comma);
                std::string b_s = comma == std::string::npos ? "" : body.substr(comma + 1);
                auto digits = [](const std::string& t) {
                    for (char ch : t)
                        if (!is_digit(ch)) return false;
                    return true;
                };
                if (a_s.empty() || !digits(a_s) || !digits(b_s) || a_s.size() > 4 || b_s.size() > 4)
                    throw Error{"bad repetition"};
                i = j + 1;
                int lo = atoi(a_s.c_str());
                int hi = comma == std::string::npos ? lo : (b_s.empty() ? -1 : atoi(b_s.c_str()));
                if (hi >= 0 && hi < lo) throw Error{"bad repetition"};
                a = rep(std::move(a), lo, hi);
            } else {
                return a;
            }
        }
    }
    u64 class_escape(int c) {
        u64 m = 0;
        if (c == 'd') {
            for (int x = '0'; x <= '9'; x++) m |= 1ull << value_of(x);
            return m;
        }
        if (c == 'w') {
            for (int v = 0; v < 64; v++)
                if (is_alpha(ALPHABET[v]) || is_digit(ALPHABET[v])) m |= 1ull << v;
            return m;
        }
        return char_set(c, fold);
    }
    static Node set_node(u64 m) {
        Node n;
        n.kind = Node::SET;
        n.set = m;
        return n;
    }
    Node atom() {
        int c = take();
        if (c == '(') {
            if (s.compare(i, 2, "?:") == 0) i += 2;
            Node n = alt();
            if (take() != ')') throw Error{"unclosed group"};
            return n;
        }
        if (c == '.') return set_node(~0ull);
        if (c == '^') {
            Node n;
            n.kind = Node::BOL;
            return n;
        }
        if (c == '$') {
            Node n;
            n.kind = Node::EOL;
            return n;
        }
        if (c == '\\') return set_node(class_escape(take()));
        if (c == '[') {
            bool neg = false;
            if (peek() == '^') {
                take();
                neg = true;
            }
            u64 m = 0;
            bool first = true;
            for (;;) {
                int ch = take();
                if (ch == ']' && !first) break;
                first = false;
                if (ch == '\\') {
                    m |= class_escape(take());
                    continue;
                }
                if (peek() == '-' && i + 1 < s.size() && s[i + 1] != ']') {
                    take();
                    int hi = take();
                    for (int x = ch; x <= hi; x++) m |= char_set(x, fold);
                } else {
                    m |= char_set(ch, fold);
                }
            }
            return set_node(neg ? ~m : m);
        }
        if (c == '*' || c == '+' || c == '?' || c == '{') throw Error{"repetition without operand"};
        return set_node(char_set(c, fold));
    }
};

int min_len(const Node& n) {
    switch (n.kind) {
        case Node::SET: return 1;
        case Node::BOL:
        case Node::EOL: return 0;
        case Node::CAT: {
            int t = 0;
            for (auto& k : n.kids) t += min_len(k);
            return t;
        }
        case Node::ALT: {
            int t = 1 << 30;
            for (auto& k : n.kids) t = std::min(t, min_len(k));
            return t;
        }
        case Node::REP: return n.lo * min_len(n.kids[0]);
    }
    return 0;
}

struct Nfa {
    enum { PLAIN = 0, BOL = 1, EOL = 2 };
    std::vector<std::vector<std::pair<int, int>>> eps;  // (kind, target)
    std::vector<u64> sym;                                // symbol set of the state's edge
    std::vector<int> sym_to;                             // its target, -1 for none
    size_t limit;

    int add() {
        if (eps.size() >= limit) throw Error{"pattern too large"};
        eps.emplace_back();
        sym.push_back(0);
        sym_to.push_back(-1);
        return (int)eps.size() - 1;
    }
    void build(const Node& n, int a, int b) {
        switch (n.kind) {
            case Node::SET:
                sym[a] = n.set;
                sym_to[a] = b;
                break;
            case Node::BOL: eps[a].push_back({BOL, b}); break;
            case Node::EOL: eps[a].push_back({EOL, b}); break;
            case Node::CAT: {
                int cur = a;
                for (auto& k : n.kids) {
                    int nxt = add();
                    build(k, cur, nxt);
                    cur = nxt;
                }
                eps[cur].push_back({PLAIN, b});
                break;
            }
            case Node::ALT:
                for (auto& k : n.kids) {
                    int x = add(), y = add();
                    eps[a].push_back({PLAIN, x});
                    build(k, x, y);
                    eps[y].push_back({PLAIN, b});
                }
                break;
            case Node::REP: {
                const Node& sub = n.kids[0];
                int cur = a;
                for (int k = 0; k < n.lo; k++) {
                    int nxt = add();
                    build(sub, cur, nxt);
                    cur = nxt;
                }
                if (n.hi < 0) {
                    int x = add(), y = add();
                    eps[cur].push_back({PLAIN, x});
                    build(sub, x, y);
                    eps[y].push_back({PLAIN, x});
                    eps[x].push_back({PLAIN, b});
                    eps[cur].push_back({PLAIN, b});
                } else {
                    eps[cur].push_back({PLAIN, b});
                    for (int k = 0; k < n.hi - n.lo; k++) {
                        int nxt = add();
                        build(sub, cur, nxt);
                        eps[nxt].push_back({PLAIN, b});
                        cur = nxt;
                    }
                }
                break;
            }
        }
    }
    std::set<int> closure(const std::set<int>& states, bool at_start, bool at_end) const {
        std::set<int> out(states);
        std::vector<int> stack(states.begin(), states.end());
        while (!stack.empty()) {
            int s = stack.back();
            stack.pop_back();
            for (auto& e : eps[s]) {
                if (e.first == BOL && !at_start) continue;
                if (e.first == EOL && !at_end) continue;
                if (out.insert(e.second).second) stack.push_back(e.second);
            }
        }
        return out;
    }
};

}  // namespace

extern "C" int mk_regex_compile(const char* pattern, int case_sensitive, uint32_t max_states, uint8_t* table,
                                uint32_t* states, char* err, size_t err_size) {
    auto error = [&](const std::string& m, int code) {
        if (err && err_size) snprintf(err, err_size, "%s", m.c_str());
        return code;
    };
    if (err && err_size) err[0] = 0;
    if (!pattern || !table || !states || max_states < 2 || max_states > 65535) return error("bad argument", MK_ERR_BAD_ARG);
    *states = 0;
    try {
        std::string s(pattern);
        Parser p(s, case_sensitive == 0);
        Node ast = p.parse();
        if (min_len(ast) == 0) return error("the pattern matches the empty string", MK_ERR_PATTERN);
        Nfa nfa;
        nfa.limit = 1u << 20;
        int start = nfa.add(), match = nfa.add();
        nfa.build(ast, start, match);
        std::map<std::set<int>, uint32_t> ids;
        std::vector<std::set<int>> order;
        std::vector<std::vector<uint32_t>> trans(1, std::vector<uint32_t>(64, 0));  // state 0: accept
        std::vector<bool> eoi(1, true);
        std::set<int> s0 = nfa.closure({start}, true, false);
        ids[s0] = 1;
        order.push_back(s0);
        for (size_t k = 0; k < order.size(); k++) {
            const std::set<int> S = order[k];
            std::vector<uint32_t> row(64);
            for (int v = 0; v < 64; v++) {
                std::set<int> nxt;
                for (int st : S)
                    if (nfa.sym_to[st] >= 0 && ((nfa.sym[st] >> v) & 1)) nxt.insert(nfa.sym_to[st]);
                nxt.insert(start);  // unanchored: a match may start after this character
                std::set<int> T = nfa.closure(nxt, false, false);
                if (T.count(match)) {
                    row[v] = 0;
                    continue;
                }
                auto it = ids.find(T);
                if (it == ids.end()) {
                    uint32_t id = (uint32_t)order.size() + 1;
                    ids[T] = id;
                    order.push_back(T);
                    if (order.size() + 1 > max_states) return error("the DFA has too many states", MK_ERR_PATTERN);
                    row[v] = id;
                } else {
                    row[v] = it->second;
                }
            }
            trans.push_back(row);
            eoi.push_back(S.count(match) || nfa.closure(S, false, true).count(match));
        }
        const size_t n = trans.size();
        for (size_t st = 0; st < n; st++) {
            for (int v = 0; v < 65; v++) {
                uint32_t x = v < 64 ? trans[st][v] : (eoi[st] ? 1u : 0u);
                table[(st * 65 + v) * 2] = (uint8_t)x;
                table[(st * 65 + v) * 2 + 1] = (uint8_t)(x >> 8);
            }
        }
        *states = (uint32_t)n;
        return MK_OK;
    } catch (const Error& e) {
        return error(e.msg, MK_ERR_PATTERN);
    } catch (...) {
        return error("out of memory", MK_ERR_OUT_OF_MEMORY);
    }
}
