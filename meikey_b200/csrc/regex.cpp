// Regex -> DFA over the 64 base64 values, in the GPU table layout (the host side of regex
// needles: src/model/pattern/dfa.rs:52-108 Dfa::new, 189-200 gpu_table, and the checks of
// Pattern::regex, src/model/pattern.rs:135-165).
//
// Table: `states` rows of 65 little-endian u16.  Row s, column v (0..63) is the next state
// after the base64 character of value v; column 64 is 1 when the state accepts at the end
// of the input.  State 0 is the absorbing accept state, state 1 the start.  Matching is an
// unanchored search over the 43 characters after the fixed key prefix, which form the whole
// haystack: `^` and `\A` anchor at the first of them, `$` and `\z` at the last, and a word
// boundary at either end sees no word character beyond it.
//
// Dialect: the reference parses with regex-syntax in ASCII mode (unicode(false), utf8(false),
// case_insensitive(!case_sensitive)), so this compiler follows that grammar:
//   literals; `.`; classes `[...]` with ranges, negation, nested classes, POSIX classes
//   `[[:alpha:]]` (and `[[:^alpha:]]`) and the set operations `&&`, `--`, `~~`;
//   Perl classes \d \D \w \W \s \S (ASCII: \w is [0-9A-Za-z_]);
//   assertions ^ $ \A \z \b \B \< \> \b{start} \b{end} \b{start-half} \b{end-half};
//   escapes of ASCII punctuation, \a \f \t \n \r \v, \x7F \x{...} \u.... \u{...} \U........;
//   groups (...), (?:...), (?P<name>...), (?<name>...), flag groups (?flags) and
//   (?flags:...) with the flags i m s U u x R (and `-` to clear); alternation;
//   repetition * + ? {m} {m,} {m,n}, each optionally lazy (a trailing ?).
// A character outside the base64 alphabet matches nothing.  Everything else the reference's
// grammar rejects is rejected here too; what it accepts but this compiler does not implement
// (Unicode classes \p / \P, a Unicode word boundary under the `u` flag) is rejected with an
// error, never compiled into something else.
//
// Construction: a Thompson NFA (one symbol edge or epsilon edges per state; assertions are
// conditional epsilon edges), then the subset construction with the start state re-added
// after every character (unanchored search), numbering DFA states in breadth-first order of
// discovery over the values 0..63.  An assertion about the next character (a word boundary,
// or the end of the haystack) is decided when that character is read: a DFA state also
// records whether the previous character was a word character, and a match that ends on such
// an assertion is reported one character later, or by the end-of-input flag.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/meikey_b200.h"
#include "regex.h"

namespace {

const char ALPHABET[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

typedef unsigned long long u64;

int value_of(int c) {
    const char* p = (c > 0 && c < 128) ? strchr(ALPHABET, c) : nullptr;
    return p ? (int)(p - ALPHABET) : -1;
}

bool is_alpha(int c) { return (c >= 'A' && c <= 'Z') || (c >= 'a' && c <= 'z'); }
bool is_digit(int c) { return c >= '0' && c <= '9'; }
bool is_alnum(int c) { return is_alpha(c) || is_digit(c); }

// base64 values that are ASCII word characters ([0-9A-Za-z_]; '+' and '/' are not)
const u64 WORD_VALUES = (1ull << 62) - 1;

bool value_is_word(int v) { return v < 62; }

// the base64 values among the ASCII characters lo..hi (one case each)
u64 range_set(int lo, int hi) {
    u64 m = 0;
    for (int c = std::max(lo, 1); c <= std::min(hi, 127); c++) {
        int v = value_of(c);
        if (v >= 0) m |= 1ull << v;
    }
    return m;
}

// simple case folding of a set of values: every letter brings its other case
u64 fold_set(u64 m) {
    u64 r = m;
    for (int v = 0; v < 52; v++)
        if ((m >> v) & 1) r |= 1ull << (v < 26 ? v + 26 : v - 26);
    return r;
}

struct Node {
    enum Kind { SET, LOOK, CAT, ALT, REP } kind = CAT;
    u64 set = 0;
    int look = 0;  // LOOK: one of the Look kinds
    std::vector<Node> kids;
    int lo = 0, hi = 0;  // REP: hi < 0 means unbounded
};

// zero-width assertions (conditional epsilon edges of the NFA)
enum Look {
    L_START = 1,       // ^ \A: at the first character of the haystack
    L_END,             // $ \z: after its last character
    L_WORD,            // \b: word character on exactly one side
    L_NOT_WORD,        // \B: word characters on both sides or on neither
    L_WORD_START,      // \< \b{start}: no word character before, one after
    L_WORD_END,        // \> \b{end}: a word character before, none after
    L_WORD_START_HALF, // \b{start-half}: no word character before
    L_WORD_END_HALF,   // \b{end-half}: no word character after
};

bool is_word_look(int k) { return k >= L_WORD; }

struct Error {
    std::string msg;
};

struct Flags {
    bool i = false, m = false, s = false, U = false, u = false, x = false, R = false;
};

struct Parser {
    const std::string& s;
    size_t i = 0;
    Flags f;
    int depth = 0;
    Parser(const std::string& str, bool fold) : s(str) { f.i = fold; }

    [[noreturn]] void error(const std::string& m) { throw Error{m}; }
    bool eof() const { return i >= s.size(); }
    int peek() const { return i < s.size() ? (unsigned char)s[i] : -1; }
    int peek_at(size_t k) const { return i + k < s.size() ? (unsigned char)s[i + k] : -1; }
    int take() {
        if (i >= s.size()) error("unexpected end of pattern");
        return (unsigned char)s[i++];
    }
    // verbose mode (x): whitespace and #-comments between tokens are ignored
    void skip_space() {
        if (!f.x) return;
        for (;;) {
            int c = peek();
            if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v') {
                i++;
            } else if (c == '#') {
                while (!eof() && s[i] != '\n') i++;
            } else {
                return;
            }
        }
    }

    Node parse() {
        Node n = alt();
        if (!eof()) {
            if (peek() == ')') error("unopened group");
            error(std::string("unexpected '") + (char)peek() + "'");
        }
        return n;
    }
    void enter() {
        if (++depth > 250) error("nest limit exceeded");
    }
    Node alt() {
        enter();
        std::vector<Node> parts;
        Flags saved = f;  // flags set inside a group end with it
        parts.push_back(concat());
        while (peek() == '|') {
            take();
            parts.push_back(concat());
        }
        f = saved;
        depth--;
        if (parts.size() == 1) return parts[0];
        Node n;
        n.kind = Node::ALT;
        n.kids = std::move(parts);
        return n;
    }
    Node concat() {
        Node n;
        n.kind = Node::CAT;
        for (;;) {
            skip_space();
            if (eof() || peek() == '|' || peek() == ')') break;
            if (peek() == '(' && peek_at(1) == '?' && flag_group_ahead()) {
                // (?flags): applies to the rest of the enclosing group
                i += 2;
                parse_flags(')');
                continue;
            }
            n.kids.push_back(repeat());
        }
        return n;
    }
    // "(?" starts a flag group without a body: flags then ')'
    bool flag_group_ahead() const {
        size_t j = i + 2;
        while (j < s.size() && strchr("imsUuxR-", s[j])) j++;
        return j < s.size() && s[j] == ')';
    }
    // flags up to `end` (':' or ')'), which is consumed
    void parse_flags(int end) {
        bool neg = false, any = false, after_neg = false;
        for (;;) {
            int c = take();
            if (c == end) break;
            if (c == ':' || c == ')') error("bad flag group");
            if (c == '-') {
                if (neg) error("repeated negation in a flag group");
                neg = true;
                after_neg = false;
                continue;
            }
            bool* fl = c == 'i' ? &f.i : c == 'm' ? &f.m : c == 's' ? &f.s : c == 'U' ? &f.U
                     : c == 'u' ? &f.u : c == 'x' ? &f.x : c == 'R' ? &f.R : nullptr;
            if (!fl) error(std::string("unrecognized flag '") + (char)c + "'");
            *fl = !neg;
            any = true;
            after_neg = neg;
        }
        if (!any && end == ')') error("empty flag group");
        if (neg && !after_neg) error("dangling flag negation");
    }
    static Node rep(Node sub, int lo, int hi) {
        Node n;
        n.kind = Node::REP;
        n.lo = lo;
        n.hi = hi;
        n.kids.push_back(std::move(sub));
        return n;
    }
    int decimal() {
        size_t st = i;
        long v = 0;
        while (is_digit(peek())) {
            v = v * 10 + (take() - '0');
            if (v > 100000) error("repetition quantifier is too large");
        }
        if (i == st) error("bad repetition: a count is missing");
        return (int)v;
    }
    Node repeat() {
        Node a = atom();
        for (;;) {
            skip_space();
            int c = peek();
            int lo, hi;
            if (c == '*') {
                take();
                lo = 0, hi = -1;
            } else if (c == '+') {
                take();
                lo = 1, hi = -1;
            } else if (c == '?') {
                take();
                lo = 0, hi = 1;
            } else if (c == '{') {
                take();
                skip_space();
                lo = decimal();
                skip_space();
                hi = lo;
                if (peek() == ',') {
                    take();
                    skip_space();
                    hi = peek() == '}' ? -1 : decimal();
                    skip_space();
                }
                if (take() != '}') error("unclosed counted repetition");
                if (hi >= 0 && hi < lo) error("invalid repetition range (min > max)");
            } else {
                return a;
            }
            skip_space();
            if (peek() == '?') take();  // lazy: the same set of matches
            a = rep(std::move(a), lo, hi);
        }
    }
    Node set_node(u64 m) {
        Node n;
        n.kind = Node::SET;
        n.set = f.i ? fold_set(m) : m;
        return n;
    }
    static Node look_node(int k) {
        Node n;
        n.kind = Node::LOOK;
        n.look = k;
        return n;
    }
    Node word_look(int k) {
        // the reference's DFA has no Unicode word boundary (regex-automata refuses it)
        if (f.u) error("a Unicode word boundary is not supported (clear the u flag)");
        return look_node(k);
    }
    // the value set of a Perl class letter (d D w W s S), or -1 when it is none
    bool perl_class(int c, u64& m) {
        switch (c) {
            case 'd': m = range_set('0', '9'); return true;
            case 'D': m = ~range_set('0', '9'); return true;
            case 'w': m = WORD_VALUES; return true;  // [0-9A-Za-z_]: '_' is not base64
            case 'W': m = ~WORD_VALUES; return true;
            case 's': m = 0; return true;            // [\t\n\v\f\r ]: no base64 character
            case 'S': m = ~0ull; return true;
        }
        return false;
    }
    int hex_digits(int n, bool braces) {
        long v = 0;
        int got = 0;
        for (;;) {
            int c = peek();
            int d = is_digit(c) ? c - '0' : (c >= 'a' && c <= 'f') ? c - 'a' + 10 : (c >= 'A' && c <= 'F') ? c - 'A' + 10 : -1;
            if (braces && c == '}') break;
            if (d < 0) {
                if (braces) error("invalid hexadecimal digit");
                break;
            }
            take();
            v = v * 16 + d;
            if (v > 0x10ffff) error("hexadecimal escape out of range");
            if (++got == n && !braces) break;
        }
        if (braces) {
            if (take() != '}' || got == 0) error("invalid hexadecimal escape");
        } else if (got != n) {
            error("invalid hexadecimal escape");
        }
        return (int)v;
    }
    // a codepoint escape after the backslash (x, u, U, control letters or punctuation);
    // -1 when `c` is not one
    int literal_escape(int c) {
        switch (c) {
            case 'a': return 7;
            case 'f': return 12;
            case 't': return 9;
            case 'n': return 10;
            case 'r': return 13;
            case 'v': return 11;
            case 'x':
                if (peek() == '{') { take(); return hex_digits(8, true); }
                return hex_digits(2, false);
            case 'u':
                if (peek() == '{') { take(); return hex_digits(8, true); }
                return hex_digits(4, false);
            case 'U':
                if (peek() == '{') { take(); return hex_digits(8, true); }
                return hex_digits(8, false);
        }
        // superfluous escapes of ASCII punctuation (and of space) stand for the character
        if (c >= 32 && c < 127 && !is_alnum(c) && c != '<' && c != '>') return c;
        return -1;
    }
    [[noreturn]] void bad_escape(int c) {
        if (c == 'p' || c == 'P') error("Unicode classes (\\p, \\P) are not supported");
        if (is_digit(c)) error("backreferences are not supported");
        error(std::string("unrecognized escape sequence '\\") + (char)c + "'");
    }
    u64 char_set(int c) { return value_of(c) >= 0 ? 1ull << value_of(c) : 0; }

    Node escape() {
        int c = take();
        u64 m;
        if (perl_class(c, m)) return set_node(m);
        switch (c) {
            case 'A': return look_node(L_START);
            case 'z': return look_node(L_END);
            case 'B': return word_look(L_NOT_WORD);
            case '<': return word_look(L_WORD_START);
            case '>': return word_look(L_WORD_END);
            case 'b': {
                if (peek() != '{') return word_look(L_WORD);
                size_t j = s.find('}', i);
                std::string name = j == std::string::npos ? "" : s.substr(i + 1, j - i - 1);
                int k = name == "start" ? L_WORD_START : name == "end" ? L_WORD_END
                      : name == "start-half" ? L_WORD_START_HALF : name == "end-half" ? L_WORD_END_HALF : 0;
                if (!k) error("unrecognized special word boundary");
                i = j + 1;
                return word_look(k);
            }
        }
        int cp = literal_escape(c);
        if (cp < 0) bad_escape(c);
        return set_node(char_set(cp));
    }

    // ---- bracketed classes ----
    // one class item: a character (returned in *single when it may start a range) or a set
    u64 class_atom(int* single) {
        *single = -1;
        int c = take();
        if (c == '[') {
            if (peek() == ':') {
                size_t j = s.find(":]", i + 1);
                if (j != std::string::npos) {
                    std::string name = s.substr(i + 1, j - i - 1);
                    bool neg = !name.empty() && name[0] == '^';
                    if (neg) name.erase(0, 1);
                    u64 m;
                    if (posix_class(name, m)) {
                        i = j + 2;
                        return neg ? ~m : m;
                    }
                }
            }
            return bracket_body();  // nested class
        }
        if (c == '\\') {
            int e = take();
            u64 m;
            if (perl_class(e, m)) return m;
            int cp = literal_escape(e);
            if (cp < 0) {
                if (strchr("AzbB<>", e)) error("an assertion is not allowed in a character class");
                bad_escape(e);
            }
            *single = cp;
            return char_set(cp);
        }
        *single = c;
        return char_set(c);
    }
    static bool posix_class(const std::string& n, u64& m) {
        if (n == "alnum") m = range_set('0', '9') | range_set('A', 'Z') | range_set('a', 'z');
        else if (n == "alpha") m = range_set('A', 'Z') | range_set('a', 'z');
        else if (n == "ascii") m = ~0ull;
        else if (n == "blank" || n == "cntrl" || n == "space") m = 0;
        else if (n == "digit") m = range_set('0', '9');
        else if (n == "graph" || n == "print") m = ~0ull;
        else if (n == "lower") m = range_set('a', 'z');
        else if (n == "punct") m = range_set('+', '+') | range_set('/', '/');
        else if (n == "upper") m = range_set('A', 'Z');
        else if (n == "word") m = WORD_VALUES;
        else if (n == "xdigit") m = range_set('0', '9') | range_set('A', 'F') | range_set('a', 'f');
        else return false;
        return true;
    }
    // union of items up to ']' or a set operator (a range is x-y of two single characters)
    u64 class_union(bool first) {
        u64 m = 0;
        bool any = false;
        for (;;) {
            skip_space();
            int c = peek();
            if (c < 0) error("unclosed character class");
            if (c == ']' && !(first && !any)) break;
            if ((c == '&' && peek_at(1) == '&') || (c == '-' && peek_at(1) == '-') || (c == '~' && peek_at(1) == '~'))
                break;
            int lo;
            u64 item = class_atom(&lo);
            any = true;
            skip_space();
            if (lo >= 0 && peek() == '-' && peek_at(1) != ']' && peek_at(1) != '-' && peek_at(1) >= 0) {
                take();
                skip_space();
                int hi;
                class_atom(&hi);
                if (hi < 0) error("invalid range: the end is not a single character");
                if (hi < lo) error("invalid range (start > end)");
                item = range_set(lo, hi);
            }
            m |= f.i ? fold_set(item) : item;
        }
        if (!any && !first) error("empty operand of a class set operation");
        return m;
    }
    // after '[': [^] items (op items)* ']'
    u64 bracket_body() {
        enter();
        bool neg = false;
        if (peek() == '^') {
            take();
            neg = true;
        }
        u64 m = class_union(true);
        for (;;) {
            int c = peek();
            if (c == ']') {
                take();
                break;
            }
            int op = take();
            take();  // the second character of &&, --, ~~
            u64 r = class_union(false);
            m = op == '&' ? (m & r) : op == '-' ? (m & ~r) : (m ^ r);
        }
        depth--;
        return neg ? ~m : m;
    }

    Node atom() {
        int c = take();
        if (c == '(') {
            Flags saved = f;
            if (peek() == '?') {
                take();
                if (peek() == 'P' && peek_at(1) == '<') {
                    i += 2;
                    group_name();
                } else if (peek() == '<') {
                    take();
                    group_name();
                } else {
                    parse_flags(':');
                }
            }
            Node n = alt();
            f = saved;
            if (eof() || take() != ')') error("unclosed group");
            return n;
        }
        if (c == '.') return set_node(~0ull);
        if (c == '^') return look_node(L_START);
        if (c == '$') return look_node(L_END);
        if (c == '\\') return escape();
        if (c == '[') {
            u64 m = bracket_body();
            Node n;
            n.kind = Node::SET;
            n.set = m;  // folding was applied item by item, before any negation
            return n;
        }
        if (c == '*' || c == '+' || c == '?' || c == '{') error("repetition operator missing expression");
        if (c == ')') error("unopened group");
        return set_node(char_set(c));
    }
    void group_name() {
        size_t j = s.find('>', i);
        if (j == std::string::npos || j == i) error("invalid capture group name");
        for (size_t k = i; k < j; k++) {
            int ch = (unsigned char)s[k];
            bool ok = is_alnum(ch) || ch == '_' || ((ch == '.' || ch == '[' || ch == ']') && k > i);
            if (!ok || (k == i && is_digit(ch))) error("invalid capture group name");
        }
        i = j + 1;
    }
};

int min_len(const Node& n) {
    switch (n.kind) {
        case Node::SET: return 1;
        case Node::LOOK: return 0;
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

// Where an assertion is evaluated: the haystack position and its neighbours.
struct At {
    bool start, end, prev_word, next_word;
};

bool look_holds(int k, const At& a) {
    switch (k) {
        case L_START: return a.start;
        case L_END: return a.end;
        case L_WORD: return a.prev_word != a.next_word;
        case L_NOT_WORD: return a.prev_word == a.next_word;
        case L_WORD_START: return !a.prev_word && a.next_word;
        case L_WORD_END: return a.prev_word && !a.next_word;
        case L_WORD_START_HALF: return !a.prev_word;
        case L_WORD_END_HALF: return !a.next_word;
    }
    return false;
}

struct Nfa {
    std::vector<std::vector<std::pair<int, int>>> eps;  // (0 plain or a Look kind, target)
    std::vector<u64> sym;                                // symbol set of the state's edge
    std::vector<int> sym_to;                             // its target, -1 for none
    size_t limit = 1u << 20;
    bool has_start = false, has_word = false;

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
            case Node::LOOK:
                eps[a].push_back({n.look, b});
                if (n.look == L_START) has_start = true;
                if (is_word_look(n.look)) has_word = true;
                break;
            case Node::CAT: {
                int cur = a;
                for (auto& k : n.kids) {
                    int nxt = add();
                    build(k, cur, nxt);
                    cur = nxt;
                }
                eps[cur].push_back({0, b});
                break;
            }
            case Node::ALT:
                for (auto& k : n.kids) {
                    int x = add(), y = add();
                    eps[a].push_back({0, x});
                    build(k, x, y);
                    eps[y].push_back({0, b});
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
                    eps[cur].push_back({0, x});
                    build(sub, x, y);
                    eps[y].push_back({0, x});
                    eps[x].push_back({0, b});
                    eps[cur].push_back({0, b});
                } else {
                    eps[cur].push_back({0, b});
                    for (int k = 0; k < n.hi - n.lo; k++) {
                        int nxt = add();
                        build(sub, cur, nxt);
                        eps[nxt].push_back({0, b});
                        cur = nxt;
                    }
                }
                break;
            }
        }
    }
    // Closure of `states` (sorted, unique) over plain edges and the assertions that hold at
    // `at`; `decided` = false leaves the word assertions and the end assertion unfollowed
    // (their next character is not known yet).
    std::vector<int> closure(const std::vector<int>& states, const At& at, bool decided, std::vector<int>& mark,
                             int& stamp) const {
        stamp++;
        std::vector<int> out, stack;
        for (int s : states)
            if (mark[s] != stamp) {
                mark[s] = stamp;
                stack.push_back(s);
            }
        while (!stack.empty()) {
            int s = stack.back();
            stack.pop_back();
            out.push_back(s);
            for (auto& e : eps[s]) {
                if (e.first != 0) {
                    const bool known = e.first == L_START || decided;
                    if (!known || !look_holds(e.first, at)) continue;
                }
                if (mark[e.second] != stamp) {
                    mark[e.second] = stamp;
                    stack.push_back(e.second);
                }
            }
        }
        std::sort(out.begin(), out.end());
        return out;
    }
};

// Probability that a uniformly random key matches the table (the first searched character
// takes 16 values, the others 64), propagated character by character.
double table_probability(const std::vector<std::vector<uint32_t>>& trans, const std::vector<bool>& eoi) {
    const size_t n = trans.size();
    std::vector<double> d(n, 0.0), nd(n);
    d[1] = 1.0;
    for (int pos = 0; pos < 43; pos++) {
        std::fill(nd.begin(), nd.end(), 0.0);
        const int values = pos == 0 ? 16 : 64;
        for (size_t s = 0; s < n; s++) {
            if (d[s] == 0.0) continue;
            const double w = d[s] / values;
            for (int v = 0; v < values; v++) nd[trans[s][v]] += w;
        }
        d.swap(nd);
    }
    double p = 0;
    for (size_t s = 0; s < n; s++)
        if (s == 0 || eoi[s]) p += d[s];
    return p;
}

const char NO_MATCH[] =
    "no public key matches this regular expression (the characters are A-Z a-z 0-9 + /, and the one right "
    "after the fixed part is A-P)";

// Parses `pattern`, applies the pattern checks and builds its NFA; throws Error.
void build_nfa(const std::string& pattern, bool fold, Nfa& nfa, int& start, int& match) {
    if (pattern.empty()) throw Error{"the pattern is empty"};
    Parser p(pattern, fold);
    Node ast = p.parse();
    if (min_len(ast) == 0) throw Error{"the pattern matches the empty string"};
    start = nfa.add();
    match = nfa.add();
    nfa.build(ast, start, match);
}

}  // namespace

namespace mkre {

std::string too_complex(uint32_t max_states) {
    return "the regular expression is too complex (the DFA has more than " + std::to_string(max_states) +
           " states)";
}

int check_table(const uint8_t* table, uint32_t states, std::string* err) {
    std::vector<std::vector<uint32_t>> trans(states, std::vector<uint32_t>(64));
    std::vector<bool> eoi(states);
    for (uint32_t st = 0; st < states; st++) {
        for (int v = 0; v < 65; v++) {
            const uint32_t x = table[(st * 65 + v) * 2] | (uint32_t)table[(st * 65 + v) * 2 + 1] << 8;
            if (v < 64) trans[st][v] = x < states ? x : 0;
            else eoi[st] = x != 0;
        }
    }
    if (states >= 2 && table_probability(trans, eoi) != 0.0) return MK_OK;
    *err = NO_MATCH;
    return MK_ERR_PATTERN;
}

int nfa_tables(const char* pattern, int case_sensitive, uint32_t max_words, NfaTables* out, std::string* err) try {
    Nfa nfa;
    int start = 0, match = 0;
    build_nfa(pattern, case_sensitive == 0, nfa, start, match);
    const uint32_t n = (uint32_t)nfa.eps.size(), words = (n + 31) / 32;
    if (words > max_words) {
        *err = "the pattern is too large for the device DFA builder (" + std::to_string(n) + " NFA states, at most " +
               std::to_string(32 * max_words) + ")";
        return MK_ERR_PATTERN;
    }
    NfaTables& t = *out;
    t = NfaTables();
    t.n = n;
    t.words = words;
    t.start = start;
    t.match = match;
    t.track_word = nfa.has_word;
    t.track_start = nfa.has_word && nfa.has_start;
    std::vector<int> mark(n, 0);
    int stamp = 0;
    auto put = [&](const std::vector<int>& set, uint32_t* bits) {
        for (int x : set) bits[x >> 5] |= 1u << (x & 31);
    };
    auto holds_match = [&](const std::vector<int>& set) { return std::binary_search(set.begin(), set.end(), match); };
    t.k0.assign(words, 0);
    put(nfa.closure({start}, At{true, false, false, false}, false, mark, stamp), t.k0.data());
    t.sym_to.assign(nfa.sym_to.begin(), nfa.sym_to.end());
    t.sym.assign(nfa.sym.begin(), nfa.sym.end());
    t.plain.assign((size_t)n * words, 0);
    t.plainm.assign(words, 0);
    t.decm.assign(8 * (size_t)words, 0);
    t.endm.assign(4 * (size_t)words, 0);
    if (t.track_word) t.dec.assign(8 * (size_t)n * words, 0);
    for (uint32_t x = 0; x < n; x++) {
        const uint32_t bit = 1u << (x & 31), w = x >> 5;
        const std::vector<int> pc = nfa.closure({(int)x}, At{false, false, false, false}, false, mark, stamp);
        put(pc, &t.plain[(size_t)x * words]);
        if (holds_match(pc)) t.plainm[w] |= bit;
        for (int c = 0; c < 4; c++) {
            const At at{(c & 2) != 0, true, (c & 1) != 0, false};
            if (holds_match(nfa.closure({(int)x}, at, true, mark, stamp))) t.endm[(size_t)c * words + w] |= bit;
        }
        if (!t.track_word) continue;
        for (int c = 0; c < 8; c++) {
            const At at{(c & 4) != 0, false, (c & 2) != 0, (c & 1) != 0};
            const std::vector<int> dc = nfa.closure({(int)x}, at, true, mark, stamp);
            put(dc, &t.dec[((size_t)c * n + x) * words]);
            if (holds_match(dc)) t.decm[(size_t)c * words + w] |= bit;
        }
    }
    return MK_OK;
} catch (const Error& e) {
    *err = e.msg;
    return MK_ERR_PATTERN;
}

}  // namespace mkre

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
        Nfa nfa;
        int start = 0, match = 0;
        build_nfa(pattern, case_sensitive == 0, nfa, start, match);
        std::vector<int> mark(nfa.eps.size(), 0);
        int stamp = 0;
        // a DFA state: NFA states (closed over plain edges and the start assertion where it
        // holds), whether the previous character was a word character (kept only when the
        // pattern has word assertions), and whether nothing has been read yet (kept only when
        // start assertions can be reached through word assertions)
        typedef std::tuple<std::vector<int>, int, int> Key;
        const bool track_word = nfa.has_word, track_start = nfa.has_word && nfa.has_start;
        std::map<Key, uint32_t> ids;
        std::vector<Key> order;
        std::vector<std::vector<uint32_t>> trans(1, std::vector<uint32_t>(64, 0));  // state 0: accept
        std::vector<bool> eoi(1, true);
        const At at0{true, false, false, false};
        Key k0{nfa.closure({start}, at0, false, mark, stamp), 0, track_start ? 1 : 0};
        ids[k0] = 1;
        order.push_back(k0);
        for (size_t k = 0; k < order.size(); k++) {
            const std::vector<int> S = std::get<0>(order[k]);
            const bool prev_word = std::get<1>(order[k]) != 0;
            const bool first = k == 0;  // only the start state has read nothing
            std::vector<uint32_t> row(64);
            for (int v = 0; v < 64; v++) {
                const bool w = value_is_word(v);
                // assertions between the previous character and this one
                const std::vector<int> C = track_word ? nfa.closure(S, At{first, false, prev_word, w}, true, mark, stamp) : S;
                if (std::binary_search(C.begin(), C.end(), match)) {
                    row[v] = 0;
                    continue;
                }
                std::vector<int> nxt;
                for (int st : C)
                    if (nfa.sym_to[st] >= 0 && ((nfa.sym[st] >> v) & 1)) nxt.push_back(nfa.sym_to[st]);
                nxt.push_back(start);  // unanchored: a match may start after this character
                std::sort(nxt.begin(), nxt.end());
                nxt.erase(std::unique(nxt.begin(), nxt.end()), nxt.end());
                std::vector<int> T = nfa.closure(nxt, At{false, false, w, false}, false, mark, stamp);
                if (std::binary_search(T.begin(), T.end(), match)) {
                    row[v] = 0;
                    continue;
                }
                Key key{std::move(T), track_word && w ? 1 : 0, 0};
                auto it = ids.find(key);
                if (it == ids.end()) {
                    uint32_t id = (uint32_t)order.size() + 1;
                    if (order.size() + 2 > max_states) return error(mkre::too_complex(max_states), MK_ERR_PATTERN);
                    ids[key] = id;
                    order.push_back(key);
                    row[v] = id;
                } else {
                    row[v] = it->second;
                }
            }
            trans.push_back(row);
            // end of input: no character follows
            const std::vector<int> E = nfa.closure(S, At{first, true, prev_word, false}, true, mark, stamp);
            eoi.push_back(std::binary_search(E.begin(), E.end(), match));
        }
        if (table_probability(trans, eoi) == 0.0) return error(NO_MATCH, MK_ERR_PATTERN);
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
