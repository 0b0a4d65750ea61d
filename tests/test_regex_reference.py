"""The regex compiler (mk_regex_compile) on the reference's own regex test cases and dialect.

The reference compiles patterns with regex-syntax / regex-automata in ASCII mode
(src/model/pattern/dfa.rs:52-108, src/model/pattern.rs:135-165); those crates are not here,
so these tests pin the compiler to:
  - the reference's test cases, copied as data: the SAMPLE cases (dfa.rs:225-240), the
    matches_regex_crate patterns (dfa.rs:254-281; the regex crate's answer is Python `re`
    in ASCII mode, which has the same semantics for these patterns, including \\b), the
    probability cases (dfa.rs:283-295), the error cases (dfa.rs:243-251) and the regex cases
    of pattern.rs (find_with_mode 330-352, invalid_with_mode 357-449, expected_tries_with_mode
    466-484);
  - the rest of the dialect (word-boundary forms, inline flags, class set operations, POSIX
    classes, escapes) against an equivalent Python pattern on random searched ranges;
  - every construct outside the dialect being rejected, never compiled into something else.
No device needed."""
import random
import re

import pytest

import dfa_builder
import meikey_b200 as mk

ALPHABET = dfa_builder.ALPHABET
# a real key's base64 (src/model/pattern.rs:303-304); its searched range starts after the
# 25-character fixed prefix
SAMPLE = b"AAAAC3NzaC1lZDI1NTE5AAAAIIQK2/0eXLDku+cWkIDsqHQOwFFTEDDoWaKofXuV/Gy9"
SEARCH_START = 25
MAX_STATES = 1 << 14  # src/model/pattern/dfa.rs:20


def values(b64: bytes):
    return [ALPHABET.index(c) for c in b64]


def walk(n: mk.Needle, vals) -> bool:
    return dfa_builder.run(n.text, n.states, vals)


def walk_either(n: mk.Needle, vals, pos, alt) -> bool:
    """The GPU's walk with the character at `pos` tried as itself and as `alt` (the reference's
    is_match_either, dfa.rs:139-157)."""
    other = list(vals)
    other[pos] = alt
    return walk(n, vals) or walk(n, other)


def python_re(pattern: str, cs: bool):
    return re.compile(pattern, re.ASCII | (0 if cs else re.IGNORECASE))


def random_range(rng):
    """43 searched characters: the first is A-P (16 values), the others any of the 64."""
    return [rng.randrange(16)] + [rng.randrange(64) for _ in range(42)]


# dfa.rs:225-240 (pattern, case_sensitive, matches SAMPLE)
SAMPLE_CASES = [("WaKo", True, True), ("wako", True, False), ("wako", False, True), ("^IQK2", True, True),
                ("^QK2", True, False), ("Gy9$", True, True), ("Gy$", True, False), ("[0-9]{2}[a-z]", True, False),
                ("zzzz|ofX", True, True), ("NTE5", True, False)]


@pytest.mark.parametrize("pattern,cs,want", SAMPLE_CASES)
def test_sample_cases(pattern, cs, want):
    vals = values(SAMPLE[SEARCH_START:])
    assert bool(python_re(pattern, cs).search(SAMPLE[SEARCH_START:].decode())) == want
    if pattern == "^QK2":
        # no key can start its searched range with Q: Dfa::new builds it, Pattern::regex then
        # refuses it (NeverMatches, pattern.rs:152-155); the compiler refuses it at once
        with pytest.raises(mk.GpuError):
            mk.Needle.regex(pattern, case_sensitive=cs)
        return
    assert walk(mk.Needle.regex(pattern, case_sensitive=cs), vals) == want


# dfa.rs:254-281: the DFA agrees with the regex crate on random keys, also when the character
# that depends on the x sign (position 41 of the searched range, 66 of the key) is replaced
@pytest.mark.parametrize("pattern", ["ab+c", "[0-9][A-F]x", "^[A-P]a|z$", "(ab){2,}", "\\b9", "a.b"])
@pytest.mark.parametrize("cs", [False, True])
def test_matches_regex_crate(pattern, cs):
    n = mk.Needle.regex(pattern, case_sensitive=cs)
    pyre = python_re(pattern, cs)
    rng = random.Random(hash((pattern, cs)) & 0xFFFF)
    for _ in range(1024):
        vals = random_range(rng)
        text = bytes(ALPHABET[v] for v in vals).decode()
        assert walk(n, vals) == bool(pyre.search(text)), text
        alt = rng.randrange(64)
        other = list(vals)
        other[41] = alt
        assert walk_either(n, vals, 41, alt) == (walk(n, vals) or walk(n, other))


# dfa.rs:283-295: probability that a key matches (first searched character A-P, the rest of
# the 64 uniformly); mk_expected_tries is its reciprocal
@pytest.mark.parametrize("pattern,want", [("z", 1.0 - (63 / 64) ** 42), ("z$", 1 / 64), ("^A", 1 / 16),
                                          ("ab$", 1 / 4096), ("(?i)ab$", 4 / 4096)])
def test_probability(pattern, want):
    got = 1.0 / mk.Needle.regex(pattern, case_sensitive=True).expected_tries()
    assert abs(got - want) < 1e-12, (got, want)


def test_probability_zero_is_refused():
    """^Q has probability 0 (dfa.rs:291); Pattern::regex turns that into NeverMatches."""
    with pytest.raises(mk.GpuError) as e:
        mk.Needle.regex("^Q")
    assert "no public key matches" in str(e.value)


# dfa.rs:243-251 and the regex cases of pattern.rs:357-449 (invalid_with_mode)
@pytest.mark.parametrize("pattern,why", [
    ("(", "unclosed group"), ("a(", "unclosed group"),
    ("a*|b", "matches the empty string"), ("^", "matches the empty string"),
    ("a=b", "no public key matches"), ("^Q", "no public key matches"), ("[a-z]{44}", "no public key matches"),
    ("a[A-Za-z0-9+/]{20}", "too complex"), ("", "empty"),
])
def test_reference_errors(pattern, why):
    with pytest.raises(mk.GpuError) as e:
        mk.Needle.regex(pattern, case_sensitive=True, max_states=MAX_STATES)
    assert e.value.status == mk._lib.ERR_PATTERN
    assert why in str(e.value), str(e.value)


# pattern.rs:330-352 (find_with_mode, regex cases): does the regex match SAMPLE
@pytest.mark.parametrize("pattern,cs,want", [("^IQK2", True, True), ("^AQK2", True, False), ("Wa.o", True, True),
                                             ("wa.o", False, True), ("[0-9]$", True, True), ("[0-9]", True, True),
                                             ("NzaC1l", True, False)])
def test_find_with_mode_cases(pattern, cs, want):
    assert walk(mk.Needle.regex(pattern, case_sensitive=cs), values(SAMPLE[SEARCH_START:])) == want


# pattern.rs:466-484 (expected_tries_with_mode, regex cases)
@pytest.mark.parametrize("pattern,want", [("ab$", 4096.0), ("[ab]$", 32.0)])
def test_expected_tries_of_regex(pattern, want):
    assert abs(mk.Needle.regex(pattern).expected_tries() / want - 1) < 1e-9


# the dialect beyond Python's: each pattern against a Python pattern with the same meaning on
# the searched range (\< = \b(?=\w), \> = \b(?<=\w), half boundaries as look-arounds, class
# set operations and POSIX classes spelled out over the base64 alphabet)
EQUIVALENT = [
    (r"\b9", r"\b9"), (r"\B9", r"\B9"), (r"9\b", r"9\b"), (r"\b[a-z]+\b", r"\b[a-z]+\b"), (r"\bx\b", r"\bx\b"),
    (r"x\B", r"x\B"), (r"\Bq\B", r"\Bq\B"), (r"\<a", r"\b(?=\w)a"), (r"a\>", r"a\b(?<=\w)"),
    (r"\b{start}[0-9]", r"\b(?=\w)[0-9]"), (r"[a-z]\b{end}", r"[a-z]\b(?<=\w)"),
    (r"\b{start-half}x", r"(?<!\w)x"), (r"x\b{end-half}", r"x(?!\w)"), (r"\W\w", r"\W\w"),
    (r"[^\W\d]9", r"[^\W\d]9"), (r"[\d+]/", r"[\d+]/"), (r"\AKb", r"\AKb"), (r"ab\z", r"ab\Z"),
    (r"(?i)ab$", r"(?i)ab$"), (r"(?i:ab)c", r"(?i:ab)c"), (r"a{2,3}?b", r"a{2,3}?b"),
    (r"(?x) a b  # comment", r"ab"), (r"(?P<n>ab)c", r"(?P<n>ab)c"), (r"(?<n>ab)c", r"(?P<n>ab)c"),
    (r"[a-z&&[^aeiou]]{3}", r"[b-df-hj-np-tv-z]{3}"), (r"[0-9--4]{3}", r"[0-35-9]{3}"),
    (r"[a-g~~b-h]{2}", r"[ah]{2}"), (r"[[:alpha:]][[:digit:]]{2}", r"[A-Za-z][0-9]{2}"),
    (r"[[:^alnum:]]{2}", r"[+/]{2}"), (r"[[:punct:]]a", r"[+/]a"), (r"\x41\x{62}c", r"Abc"),
    (r"[\w&&\D]{4}", r"[A-Za-z]{4}"), (r"(?s).a.", r".a."), (r"(?m)ab$", r"ab$"), (r"(?U)a+b", r"a+b"),
    (r"a\-?b", r"a-?b"), (r"[a\]]x", r"[a\]]x"), (r"[]a]b", r"[\]a]b"), (r"(a|)b", r"(a|)b"), (r"x{0}y", r"y"),
]


@pytest.mark.parametrize("ours,theirs", EQUIVALENT)
@pytest.mark.parametrize("cs", [True, False])
def test_dialect(ours, theirs, cs):
    n = mk.Needle.regex(ours, case_sensitive=cs)
    pyre = python_re(theirs, cs)
    rng = random.Random(hash((ours, cs)) & 0xFFFF)
    for _ in range(1500):
        vals = random_range(rng)
        text = bytes(ALPHABET[v] for v in vals).decode()
        assert walk(n, vals) == bool(pyre.search(text)), (ours, text)


def test_scoped_flags():
    """(?-i:...) and (?-i) clear the flag inside a case-insensitive pattern."""
    n = mk.Needle.regex("(?-i:a)b", case_sensitive=False)
    m = mk.Needle.regex("(?i)a(?-i)b", case_sensitive=True)
    for text, want_n, want_m in [("Aab", True, True), ("AAB", False, False), ("AaB", True, False),
                                 ("AAb", False, True)]:
        vals = values(text.encode()) + [63] * (43 - len(text))
        assert walk(n, vals) == want_n, text
        assert walk(m, vals) == want_m, text


def test_word_boundary_at_the_ends():
    """The searched range is the whole haystack: a word boundary before its first character
    and after its last sees no word character beyond (the reference runs the DFA from the
    start of the range, dfa.rs:117-127), although the key's fixed prefix ends in 'I'."""
    a_first = [0] + [62] * 42   # 'A' then '+' x 42
    nine_last = [62] * 42 + [61]  # '+' x 42 then '9'
    assert walk(mk.Needle.regex(r"\bA"), a_first)
    assert not walk(mk.Needle.regex(r"\BA"), a_first)
    assert walk(mk.Needle.regex(r"9\b"), nine_last)
    assert not walk(mk.Needle.regex(r"9\B"), nine_last)


@pytest.mark.parametrize("bad", [r"\pL", r"\PL", r"(?u)\b9", r"\1", r"a\e", r"\Q", r"\Z", r"[\b]", r"a{", r"a{2",
                                 r"a{3,1}", r"(?)a", r"(?z)a", r"[z-a]", r"a)", r"[a", r"(?P<1x>a)", r"\b{foo}",
                                 r"*a", r"(?i-)a", r"\x", r"\x{zz}", r"a||"])
def test_outside_the_dialect_is_rejected(bad):
    with pytest.raises(mk.GpuError) as e:
        mk.Needle.regex(bad)
    assert e.value.status == mk._lib.ERR_PATTERN
