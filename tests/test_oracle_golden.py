"""The CPU oracle against the reference's own known answers (CPU only)."""
import numpy as np
import pytest

import oracle
from conftest import case_input


def test_literal_overlapping_known_answers(golden):
    for case in golden["literal_overlapping"]:
        lits = [p.encode() for p in case["patterns"]]
        got = oracle.sort_matches(oracle.literal_scan(lits, list(range(len(lits))), case_input(case)))
        exp = oracle.sort_matches(np.array(case["expected"], dtype=np.uint32).reshape(-1, 3))
        assert got.tolist() == exp.tolist(), case["src"]


def test_regex_find_iter_known_answers(golden):
    for case in golden["regex_find_iter"]:
        r = oracle.Regex(case["pattern"])
        got = r.find_iter(case_input(case))
        assert [list(x) for x in got] == case["expected"], (case["src"], case["pattern"], got)


def test_regex_bitmap_known_answer():
    # core/src/gpu/ensemble.rs:375-410
    data = bytearray(b"x" * (1 << 20))
    for i in range(100):
        if i % 3 == 0:
            needle = f"R{i:03}Z42".encode()
            data[i * 7919:i * 7919 + len(needle)] = needle
    rxs = [oracle.Regex(f"R{i:03}Z[0-9]{{2}}") for i in range(100)]
    got = oracle.regex_scan(rxs, list(range(100)), bytes(data))
    hit = sorted(set(got[:, 0].tolist()))
    assert hit == [i for i in range(100) if i % 3 == 0]
    for p, s, e in got.tolist():
        assert (s, e) == (p * 7919, p * 7919 + 7)


def test_fnv_known_answers(golden):
    for case in golden["fnv"]:
        a = oracle.fnv1a(case["a"][0].encode(), case["a"][1])
        b = oracle.fnv1a(case["b"][0].encode(), case["b"][1])
        assert (a == b) == case["equal"], case["src"]
    # FNV-1a reference values (basis 2166136261, prime 16777619)
    assert oracle.fnv1a(b"a", 8) == 0xE40C292C
    assert oracle.fnv1a(b"foobar", 8) == 0xBF9CF968


def test_demotion_and_pathological():
    assert oracle.regex_literal("needle") == b"needle"
    assert oracle.regex_literal("(needle)") == b"needle"
    assert oracle.regex_literal("foo\\.bar") == b"foo.bar"
    assert oracle.regex_literal("(?i:hello)") is None
    assert oracle.regex_literal("[a]b") == b"ab"
    assert oracle.regex_literal("a|b") is None
    assert oracle.regex_pathological("(a+)+")
    assert oracle.regex_pathological("(a*)*")
    assert oracle.regex_pathological("([0-9]+)+")
    assert not oracle.regex_pathological("a+")
    assert not oracle.regex_pathological("(a+)?")


def test_regex_set_scan_equals_per_regex_find_iter():
    import workloads as w
    specs = w.gen_regexes(40, 99)
    data = w.fill_markov(1 << 18, w.PRINTABLE, 5, 6)
    r = w.Rng(7)
    w.plant(data, [specs[r.below(40)].sample(r) for _ in range(64)], 2048, 8)
    rxs = [oracle.Regex(s.source) for s in specs]
    got = oracle.sort_matches(oracle.regex_scan(rxs, list(range(40)), data))
    exp = []
    for i, rx in enumerate(rxs):
        exp += [[i, s, e] for s, e in rx.find_iter(data)]
    exp = oracle.sort_matches(np.array(exp, dtype=np.uint32).reshape(-1, 3))
    assert len(exp) > 20
    assert got.tolist() == exp.tolist()


def test_literal_scan_matches_naive_search():
    rng = np.random.default_rng(3)
    data = rng.integers(ord("a"), ord("e"), size=20000, dtype=np.uint8)
    lits = [bytes(rng.integers(ord("a"), ord("e"), size=int(rng.integers(1, 12)), dtype=np.uint8)) for _ in range(60)]
    got = oracle.sort_matches(oracle.literal_scan(lits, list(range(len(lits))), data))
    text = data.tobytes()
    exp = []
    for i, l in enumerate(lits):
        start = text.find(l)
        while start >= 0:
            exp.append([i, start, start + len(l)])
            start = text.find(l, start + 1)
    exp = oracle.sort_matches(np.array(exp, dtype=np.uint32).reshape(-1, 3))
    assert got.tolist() == exp.tolist()
