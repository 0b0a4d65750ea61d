"""The library's regex -> DFA compiler (mk_regex_compile) against the test-side builder
(tests/golden/dfa_builder.py, itself checked against Python `re`) and against Python `re`
directly: tables are byte-identical, and the DFA walk agrees with re.search on random keys.
No device needed."""
import random
import re

import pytest

import dfa_builder
import meikey_b200 as mk

PATTERNS = [
    ("ab", True), ("[0-9]$", True), ("^[A-P]a", True), ("wa.o", False), ("(ab){2,}", True),
    ("zzzz|ofX", True), ("[0-9][A-F]x", False), ("a+b/c?", True), ("^[^A]", True), ("9$", True),
    ("\\d\\w{2}", True), ("(?:xy|z+)[+/]{1,3}$", False), ("^A.{3}b", True), ("[]a]", True), ("[a-]", True),
    ("q{2}", True), ("(a|b|c)(d|e)", False), ("[^0-9a-z]{4}", True), ("K\\+", True), ("(x(y(z)?)?)w", True),
]


@pytest.mark.parametrize("pattern,cs", PATTERNS)
def test_table_identical_to_builder(pattern, cs):
    want, states = dfa_builder.build(pattern, cs)
    got = mk.Needle.regex(pattern, case_sensitive=cs)
    assert got.states == states
    assert got.text == want


@pytest.mark.parametrize("pattern,cs", PATTERNS[:12])
def test_walk_agrees_with_python_re(pattern, cs):
    n = mk.Needle.regex(pattern, case_sensitive=cs)
    pyre = dfa_builder.python_regex(pattern, cs)
    rng = random.Random(hash(pattern) & 0xFFFF)
    for _ in range(2000):
        vals = [rng.randrange(16)] + [rng.randrange(64) for _ in range(42)]
        text = bytes(dfa_builder.ALPHABET[v] for v in vals).decode()
        assert dfa_builder.run(n.text, n.states, vals) == bool(pyre.search(text)), text


@pytest.mark.parametrize("bad", ["", "a*", "^$", "(ab", "a{2", "*a", "[ab", "a{3,1}"])
def test_rejects_bad_patterns(bad):
    with pytest.raises(mk.GpuError) as e:
        mk.Needle.regex(bad)
    assert e.value.status == mk._lib.ERR_PATTERN


def test_state_limit():
    with pytest.raises(mk.GpuError):
        mk.Needle.regex("[ab].{12}[cd]", max_states=64)
    assert mk.Needle.regex("[ab].{3}[cd]", max_states=64).states <= 64


def test_expected_tries_exact():
    """mk_expected_tries is 1/P(match) for a uniformly random key, by exact propagation through
    the needle's DFA: checked against closed forms where they exist."""
    # suffix of length L: the last L characters are uniform and independent
    for text in ("Ab", "xyz1", "Q+/9z"):
        e = mk.Needle.suffix(text).expected_tries()
        assert abs(e - 64 ** len(text)) / 64 ** len(text) < 1e-9
    # case-insensitive doubles the chance of each letter
    e_ci = mk.Needle.suffix("ab", case_sensitive=False).expected_tries()
    assert abs(e_ci - 64 ** 2 / 4) < 1e-6
    # contains of a 1-character needle: 1 - P(no occurrence in 42 uniform characters and a
    # first character from 16 values that cannot be 'z')
    e1 = mk.Needle.contains("z").expected_tries()
    assert abs(1 / e1 - (1 - (63 / 64) ** 42)) < 1e-12
    # a regex that no key can match ('a' is not among the 16 values of the first position) is
    # refused at compile time, as the reference's Pattern::regex refuses it (NeverMatches)
    with pytest.raises(mk.GpuError) as e:
        mk.Needle.regex("^a")
    assert e.value.status == mk._lib.ERR_PATTERN and "no public key matches" in str(e.value)
