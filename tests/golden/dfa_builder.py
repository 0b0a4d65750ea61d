"""Regex -> DFA over the 64 base64 values, in the reference's GPU table layout.

Test infrastructure: builds DFA tables for golden fixtures and parity tests.  The
layout follows src/model/pattern/dfa.rs:52-108 and 189-200: state 0 is the absorbing
accept state, state 1 is the start (before the first searched character), and each
state has 64 next-state entries plus a 65th flag "accepts at end of input"; entries are
little-endian u16.  Matching is an unanchored search over the 43 characters after the
fixed key prefix; `^` anchors at the first of them and `$` at the last.

Supported syntax (a subset of the regex crate's): literals, `.`, classes `[...]` with
ranges and negation, `\\d`, `\\w`, `\\s`-free escapes of metacharacters, groups `(...)`
and `(?:...)`, alternation `|`, `*`, `+`, `?`, `{m}`, `{m,}`, `{m,n}`, anchors `^` `$`,
and case-insensitive matching.
"""
import re as _re

ALPHABET = b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/"
VALUE = {c: i for i, c in enumerate(ALPHABET)}
ALL = frozenset(range(64))


class RegexError(ValueError):
    pass


def _char_set(ch: int, fold: bool):
    out = set()
    cands = {ch}
    if fold and chr(ch).isalpha():
        cands = {ord(chr(ch).lower()), ord(chr(ch).upper())}
    for c in cands:
        if c in VALUE:
            out.add(VALUE[c])
    return out


class _Parser:
    def __init__(self, s: str, fold: bool):
        self.s, self.i, self.fold = s, 0, fold

    def peek(self):
        return self.s[self.i] if self.i < len(self.s) else None

    def take(self):
        c = self.peek()
        if c is None:
            raise RegexError("unexpected end")
        self.i += 1
        return c

    def parse(self):
        node = self.alt()
        if self.peek() is not None:
            raise RegexError(f"unexpected {self.peek()!r} at {self.i}")
        return node

    def alt(self):
        parts = [self.concat()]
        while self.peek() == "|":
            self.take()
            parts.append(self.concat())
        return ("alt", parts) if len(parts) > 1 else parts[0]

    def concat(self):
        items = []
        while self.peek() not in (None, "|", ")"):
            items.append(self.repeat())
        return ("cat", items)

    def repeat(self):
        atom = self.atom()
        while True:
            c = self.peek()
            if c == "*":
                self.take(); atom = ("rep", atom, 0, None)
            elif c == "+":
                self.take(); atom = ("rep", atom, 1, None)
            elif c == "?":
                self.take(); atom = ("rep", atom, 0, 1)
            elif c == "{":
                j = self.s.find("}", self.i)
                body = self.s[self.i + 1:j] if j > 0 else ""
                m = _re.fullmatch(r"(\d+)(,(\d*))?", body)
                if not m:
                    raise RegexError("bad repetition")
                self.i = j + 1
                lo = int(m.group(1))
                hi = lo if m.group(2) is None else (int(m.group(3)) if m.group(3) else None)
                atom = ("rep", atom, lo, hi)
            else:
                return atom

    def cls_escape(self, c):
        if c == "d":
            return {VALUE[ord(x)] for x in "0123456789"}
        if c == "w":
            return {VALUE[x] for x in ALPHABET if chr(x).isalnum()}
        return _char_set(ord(c), self.fold)

    def atom(self):
        c = self.take()
        if c == "(":
            if self.s.startswith("?:", self.i):
                self.i += 2
            node = self.alt()
            if self.take() != ")":
                raise RegexError("unclosed group")
            return node
        if c == ".":
            return ("set", ALL)
        if c == "^":
            return ("bol",)
        if c == "$":
            return ("eol",)
        if c == "\\":
            return ("set", frozenset(self.cls_escape(self.take())))
        if c == "[":
            neg = False
            if self.peek() == "^":
                self.take(); neg = True
            s = set()
            first = True
            while True:
                ch = self.take()
                if ch == "]" and not first:
                    break
                first = False
                if ch == "\\":
                    s |= self.cls_escape(self.take())
                    continue
                if self.peek() == "-" and self.s[self.i + 1:self.i + 2] not in ("]", ""):
                    self.take()
                    hi = self.take()
                    for x in range(ord(ch), ord(hi) + 1):
                        s |= _char_set(x, self.fold)
                else:
                    s |= _char_set(ord(ch), self.fold)
            return ("set", frozenset(ALL - s if neg else s))
        if c in "*+?{":
            raise RegexError("repetition without operand")
        return ("set", frozenset(_char_set(ord(c), self.fold)))


class _NFA:
    def __init__(self):
        self.eps = []   # eps[s] = list of (kind, t): kind None (plain), 'bol', 'eol'
        self.sym = []   # sym[s] = (set, t) or None

    def new(self):
        self.eps.append([])
        self.sym.append(None)
        return len(self.eps) - 1

    def build(self, node, a, b):
        k = node[0]
        if k == "set":
            self.sym[a] = (node[1], b)
        elif k == "bol":
            self.eps[a].append(("bol", b))
        elif k == "eol":
            self.eps[a].append(("eol", b))
        elif k == "cat":
            cur = a
            for item in node[1]:
                nxt = self.new()
                self.build(item, cur, nxt)
                cur = nxt
            self.eps[cur].append((None, b))
        elif k == "alt":
            for p in node[1]:
                x, y = self.new(), self.new()
                self.eps[a].append((None, x))
                self.build(p, x, y)
                self.eps[y].append((None, b))
        elif k == "rep":
            _, sub, lo, hi = node
            cur = a
            for _ in range(lo):
                nxt = self.new()
                self.build(sub, cur, nxt)
                cur = nxt
            if hi is None:
                x, y = self.new(), self.new()
                self.eps[cur].append((None, x))
                self.build(sub, x, y)
                self.eps[y].append((None, x))
                self.eps[x].append((None, b))
                self.eps[cur].append((None, b))
            else:
                self.eps[cur].append((None, b))
                for _ in range(hi - lo):
                    nxt = self.new()
                    self.build(sub, cur, nxt)
                    self.eps[nxt].append((None, b))
                    cur = nxt
        else:
            raise RegexError(k)

    def closure(self, states, at_start, at_end):
        out, stack = set(states), list(states)
        while stack:
            s = stack.pop()
            for kind, t in self.eps[s]:
                if kind == "bol" and not at_start:
                    continue
                if kind == "eol" and not at_end:
                    continue
                if t not in out:
                    out.add(t)
                    stack.append(t)
        return out


def min_len(node):
    k = node[0]
    if k == "set":
        return 1
    if k in ("bol", "eol"):
        return 0
    if k == "cat":
        return sum(min_len(x) for x in node[1])
    if k == "alt":
        return min(min_len(x) for x in node[1])
    if k == "rep":
        return node[2] * min_len(node[1])
    return 0


def build(regex: str, case_sensitive: bool = True, max_states: int = 1 << 14):
    """(table bytes, number of states) for `regex`."""
    ast = _Parser(regex, not case_sensitive).parse()
    if min_len(ast) == 0:
        raise RegexError("matches the empty string")
    nfa = _NFA()
    start, match = nfa.new(), nfa.new()
    nfa.build(ast, start, match)

    def key_of(states):
        return frozenset(states)

    s0 = key_of(nfa.closure({start}, True, False))
    ids = {s0: 1}
    order = [s0]
    trans = [[0] * 64]  # state 0: accept
    eoi = [True]
    i = 0
    while i < len(order):
        S = order[i]
        i += 1
        row = []
        for v in range(64):
            nxt = set()
            for s in S:
                sy = nfa.sym[s]
                if sy and v in sy[0]:
                    nxt.add(sy[1])
            nxt.add(start)  # unanchored: a match may start after this character
            T = key_of(nfa.closure(nxt, False, False))
            if match in T:
                row.append(0)
                continue
            if T not in ids:
                ids[T] = len(order) + 1
                order.append(T)
                if len(order) + 1 > max_states:
                    raise RegexError("too many states")
            row.append(ids[T])
        trans.append(row)
        eoi.append(match in nfa.closure(S, False, True) or (match in S))
    # the start state may accept at the very beginning via ^...$ only when the hay is empty: not reachable
    n = len(trans)
    out = bytearray()
    for s in range(n):
        for v in range(64):
            out += trans[s][v].to_bytes(2, "little")
        out += int(eoi[s]).to_bytes(2, "little")
    return bytes(out), n


def run(table: bytes, states: int, values) -> bool:
    """Whether the 43 six-bit `values` match (the GPU walk without the sign fork)."""
    def nxt(s, i):
        at = (s * 65 + i) * 2
        return table[at] | table[at + 1] << 8
    s = 1
    for v in values:
        s = nxt(s, v)
    return s == 0 or nxt(s, 64) != 0


def python_regex(regex: str, case_sensitive: bool):
    return _re.compile(regex, _re.ASCII | (0 if case_sensitive else _re.IGNORECASE))
