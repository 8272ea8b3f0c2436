"""Regex DFA path on the GPU against the oracle (contract R), bit-exact.

Both candidate paths are checked: the plain thread-per-start kernel and the
speculative chunked walk (proposer, fix-up, reverse walk); their K candidate
sets (every (pattern, start, end) of an anchored match) must be identical, and
the resolved find_iter spans must equal the oracle's.
"""
import numpy as np
import pytest

import oracle
import workloads as w
from conftest import case_input

pytestmark = pytest.mark.gpu

PLAIN, SPEC = 1, 0


def _ws():
    import warpstate_b200 as ws
    return ws


def matcher(patterns, mode=SPEC, proposer=None, **cfg):
    ws = _ws()
    b = ws.PatternSet.builder()
    for kind, p in patterns:
        b = b.literal_bytes(p) if kind == 0 else b.regex(p.decode() if isinstance(p, bytes) else p)
    c = ws.AutoMatcherConfig().regex_mode(mode)
    if proposer is not None:
        c.proposer(proposer)
    for k, v in cfg.items():
        getattr(c, k)(v)
    return ws.GpuMatcher.with_config(b.build(), c)


def _outside_classes(pattern: str) -> str:
    """The pattern with bracket expressions removed (a ^ there negates a class)."""
    out, i = [], 0
    while i < len(pattern):
        c = pattern[i]
        if c == "\\":
            out.append(pattern[i:i + 2])
            i += 2
        elif c == "[":
            j = i + 1
            if j < len(pattern) and pattern[j] == "^":
                j += 1
            if j < len(pattern) and pattern[j] == "]":
                j += 1
            while j < len(pattern) and pattern[j] != "]":
                j += 2 if pattern[j] == "\\" else 1
            i = j + 1
        else:
            out.append(c)
            i += 1
    return "".join(out)


def supported(pattern: str) -> bool:
    """Every regex except those that can match the empty string."""
    return not oracle.Regex(pattern).nullable


def test_goldens_with_assertions_and_negated_classes_are_run(golden):
    pats = [c["pattern"] for c in golden["regex_find_iter"]]
    assert any("[^" in p for p in pats if supported(p))
    assert any(a in _outside_classes(p) for p in pats if supported(p) for a in ("^", "$", "\\b"))


def test_golden_regex_cases(golden):
    for case in golden["regex_find_iter"]:
        if not supported(case["pattern"]):
            continue
        data = case_input(case)
        for mode in (PLAIN, SPEC):
            m = matcher([(1, case["pattern"].encode())], mode=mode)
            got = m.scan_array(data)
            assert [[s, e] for _, s, e in got.tolist()] == case["expected"], (case["src"], case["pattern"], mode)


def test_regex_bitmap_known_answer():
    # core/src/gpu/ensemble.rs:375-410 -- here with spans, not just a bitmap
    data = bytearray(b"x" * (1 << 20))
    for i in range(100):
        if i % 3 == 0:
            needle = f"R{i:03}Z42".encode()
            data[i * 7919:i * 7919 + len(needle)] = needle
    pats = [(1, f"R{i:03}Z[0-9]{{2}}".encode()) for i in range(100)]
    for mode in (PLAIN, SPEC):
        got = matcher(pats, mode=mode).scan_array(bytes(data))
        assert sorted(set(got[:, 0].tolist())) == [i for i in range(100) if i % 3 == 0]
        for p, s, e in got.tolist():
            assert (s, e) == (p * 7919, p * 7919 + 7)


def _regex_workload(size, n, seed):
    wl = w.regex(size=size, n=n, seed=seed)
    return wl.patterns, wl.data


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_regex_config_scaled_vs_oracle(mode):
    pats, data = _regex_workload(4 << 20, 500, 3)
    got = matcher(pats, mode=mode).scan_array(data)
    exp = oracle.scan_patterns(pats, data)
    assert len(exp) > 100
    assert got.shape == exp.shape and np.array_equal(got, exp)


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
@pytest.mark.parametrize("wide", [False, True])
def test_walk_image_layouts_vs_oracle(mode, wide):
    # the walk's image is indexed by class when every speculative group has at
    # most 32 byte classes, else by byte: a set over a few letters and one over
    # digits, letters and punctuation (more than 32 classes) take the two
    # layouts; both against the oracle, with small chunks so that the fix-up
    # re-walks many chunks over the same image (one unbounded regex keeps the
    # walk from deriving the chunk starts exactly)
    rng = np.random.default_rng(91 if wide else 92)
    alpha = (b"0123456789abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ_:=@!%,;/" if wide
             else b"abcdefghijkl")
    pats = []
    for k in range(120):
        lits = [rng.choice(list(alpha), size=int(rng.integers(4, 9))).astype(np.uint8).tobytes() for _ in range(3)]
        cls = b"[" + bytes(sorted(set(rng.choice(list(alpha), size=4).tolist()))) + b"]"
        src = b"(?:" + b"|".join(lits) + b")" + cls + b"{1,4}"
        pats.append((1, src))
        if k == 0:
            unbounded = (1, b"(?:" + b"|".join(lits) + b")" + cls + b"+")
    text = np.frombuffer(alpha, dtype=np.uint8)[rng.integers(0, len(alpha), 3 << 20)].copy()
    for k in range(400):  # plant matches: a pattern's first literal and one byte of its class
        src = pats[k % len(pats)][1].decode()
        lit = src[3:src.index("|")] + src[src.index("[") + 1]
        at = int(rng.integers(0, text.size - 16))
        text[at:at + len(lit)] = np.frombuffer(lit.encode(), dtype=np.uint8)
    pats.append(unbounded)
    m = matcher(pats, mode=mode, walk_chunk=256)
    info = m.info()
    assert (info["max_classes"] > 32) == wide
    assert info["exact_groups"] < info["n_groups"] - info["n_context_groups"]
    got = m.scan_array(text.tobytes())
    exp = oracle.scan_patterns(pats, text.tobytes())
    assert len(exp) > 100
    assert got.shape == exp.shape and np.array_equal(got, exp)


def test_candidate_sets_plain_equals_speculative():
    pats, data = _regex_workload(2 << 20, 200, 5)
    m = matcher(pats)
    a = oracle.sort_matches(m.regex_candidates(data, PLAIN))
    b = oracle.sort_matches(m.regex_candidates(data, SPEC))
    assert len(a) > 50
    assert np.array_equal(a, b)


@pytest.mark.parametrize("chunk", [256, 512, 4096])
def test_chunk_boundaries_without_proposer(chunk):
    # small chunks put many matches across chunk boundaries; the walk derives
    # each chunk's start from the 32 bytes before it (every regex here matches
    # at most 32 bytes, and 4 x 32 <= 256)
    pats, data = _regex_workload(1 << 20, 60, 7)
    m = matcher(pats, mode=SPEC, proposer=1, walk_chunk=chunk)
    got = m.scan_array(data)
    exp = oracle.scan_patterns(pats, data)
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("chunk", [4096, 8192])
def test_exact_chunk_starts_need_no_fixup(chunk):
    # every regex of the 500-regex configuration matches at most 32 bytes: the
    # walk of each chunk starts from the state reached over the 32 bytes before
    # it, which is the state of a walk from the input's start there, so every
    # boundary holds and the fix-up re-walks nothing
    pats, data = _regex_workload(8 << 20, 500, 3)
    m = matcher(pats, mode=SPEC, proposer=1, walk_chunk=chunk, profile=True)
    info = m.info()
    spec = info["n_groups"] - info["n_context_groups"]
    assert spec > 0 and info["exact_groups"] == spec
    got = m.scan_array(data)
    info = m.info()
    assert info["last_fixup_chunks"] == 0 and info["last_rewalk_bytes"] == 0
    assert info["last_guesses"] > 0 and info["last_guess_hits"] == info["last_guesses"]
    exp = oracle.scan_patterns(pats, data)
    assert len(exp) > 100 and np.array_equal(got, exp)


def test_unbounded_and_long_regexes_keep_guessing():
    # a group with an unbounded regex, or with one longer than 512 bytes, has
    # no exact chunk starts: its boundaries are guessed and fixed up
    rng = np.random.default_rng(17)
    data = bytearray(rng.integers(ord("a"), ord("e"), size=1 << 20, dtype=np.uint8).tobytes())
    for k in range(0, len(data) - 1200, 3000):
        data[k:k + 1] = b"X"
        data[k + 700:k + 701] = b"Y"
    for pats in ([(1, b"X[a-d]+Y"), (1, b"(?:abc|dcb)[a-d]{2}")], [(1, b"X[a-d]{600,800}Y")]):
        m = matcher(pats, mode=SPEC, proposer=1, walk_chunk=4096, profile=True)
        assert m.info()["exact_groups"] == 0
        got = m.scan_array(bytes(data))
        exp = oracle.scan_patterns(pats, bytes(data))
        assert len(exp) > 100 and np.array_equal(got, exp), pats
    # several groups, the last one holding an unbounded regex: the others
    # still start their chunks exactly
    pats, text = _regex_workload(4 << 20, 500, 3)
    pats = pats + [(1, b"~[0-9]+~")]
    m = matcher(pats, mode=SPEC, proposer=1, dfa_max_states=16384, profile=True)
    info = m.info()
    spec = info["n_groups"] - info["n_context_groups"]
    assert spec >= 2 and 0 < info["exact_groups"] < spec
    got = m.scan_array(text)
    exp = oracle.scan_patterns(pats, text)
    assert len(exp) > 100 and np.array_equal(got, exp)


def test_long_partial_matches_across_chunks():
    # a regex whose partial matches run for hundreds of bytes keeps the walk
    # away from its start state across many chunk boundaries
    rng = np.random.default_rng(1)
    data = bytearray(rng.integers(ord("a"), ord("c"), size=1 << 18, dtype=np.uint8).tobytes())
    for k in range(0, len(data) - 3000, 5000):
        data[k:k + 1] = b"X"
        data[k + 2000:k + 2001] = b"Y"
    pats = [(1, b"X[ab]{1,2500}Y"), (1, b"(?:ab|ba)[ab]{3}X"), (1, b"b[ab]{0,3}Y")]
    for mode in (PLAIN, SPEC):
        m = matcher(pats, mode=mode, proposer=1, walk_chunk=256, max_matches=1 << 22)
        got = m.scan_array(bytes(data))
        exp = oracle.scan_patterns(pats, bytes(data))
        assert np.array_equal(got, exp), mode


def test_mixed_literals_and_regexes():
    wl = w.batch(n_items=200, n_lit=300, n_rx=100, seed=9)
    data = wl.data
    got = matcher(wl.patterns).scan_array(data)
    exp = oracle.scan_patterns(wl.patterns, data)
    assert np.array_equal(got, exp)


def test_leftmost_first_semantics_on_gpu():
    cases = [
        ("a|ab", b"ab ab", [[0, 1], [3, 4]]),
        ("ab|a", b"ab ab", [[0, 2], [3, 5]]),
        ("a+?", b"aaa", [[0, 1], [1, 2], [2, 3]]),
        ("(?:ab|abcd)x", b"abx abcdx", [[0, 3], [4, 9]]),
        ("a{2,3}", b"aaaaaaa", [[0, 3], [3, 6]]),
        ("[a-c]+d", b"abcabcd xd cd", [[0, 7], [11, 13]]),
    ]
    for pat, data, exp in cases:
        for mode in (PLAIN, SPEC):
            got = matcher([(1, pat.encode())], mode=mode).scan_array(data)
            assert [[s, e] for _, s, e in got.tolist()] == exp, (pat, mode)
            assert [list(x) for x in oracle.Regex(pat).find_iter(data)] == exp


def test_unsupported_regexes_fail_loudly():
    # patterns that can match the empty string (the rest of the syntax runs)
    ws = _ws()
    for pat in ["a*", "a|", "^", "\\b", "(?:ab)?"]:
        with pytest.raises(ws.PatternCompilationFailed):
            matcher([(1, pat.encode())])


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_long_runs_of_match_ends_are_exact(mode):
    # a+ over long runs of a's: every position ends one match and starts
    # another.  The speculative path shares reverse-walk marks, cuts the
    # parallel leftmost-first walks at 1 KiB (the chain finishes the ones it
    # picks: x[a-z]*y spans 5 KB here) and merge-sorts per-regex start lists
    # of more than 4096 entries
    pats = [(1, b"a+"), (1, b"(ab)+c?"), (1, b"x[a-z]*y"), (0, b"aa"), (1, b"a{3}")]
    n = 150_000 if mode == SPEC else 30_000
    data = (b"a" * n + b"\n" + b"ab" * (n // 2) + b"c" + b"x" + b"q" * 5000 + b"y" + b"zz"
            + b"a" * (n // 3))
    m = matcher(pats, mode=mode, max_matches=1 << 21)
    got = m.scan_array(data)
    exp = oracle.scan_patterns(pats, data)
    assert len(exp) > n and np.array_equal(got, exp)


def test_distinct_candidates_hold_the_starts_of_full_k():
    # the candidates a scan works from hold exactly the distinct
    # (pattern_id, start) pairs of K, in both modes, with far fewer entries
    pats = [(1, b"a+"), (1, b"(ab)+"), (1, b"b[ab]*")]
    data = (b"a" * 1500 + b"b" + b"ab" * 700 + b"\n") * 2
    m = matcher(pats, max_matches=1 << 21)
    full = {md: m.regex_candidates(data, md) for md in (PLAIN, SPEC)}
    assert np.array_equal(oracle.sort_matches(full[PLAIN]), oracle.sort_matches(full[SPEC]))
    starts = set(map(tuple, full[PLAIN][:, :2].tolist()))
    for md in (PLAIN, SPEC):
        d = m.regex_candidates(data, md, distinct=True)
        assert set(map(tuple, d[:, :2].tolist())) == starts, md
        assert len(d) * 20 < len(full[md]), (md, len(d), len(full[md]))


def test_candidate_overflow_is_retried_exactly():
    # [a-z]{1,8}q over lowercase text: every q ends a match from up to 8
    # starts, so the candidates far exceed a small max_matches while the
    # leftmost-first result still fits.  The candidate buffers overflow on the
    # first scan; the synchronous scan repeats it with the capacity the first
    # one needed and returns the exact result.
    rng = np.random.default_rng(5)
    data = rng.integers(ord("a"), ord("z") + 1, size=6 << 20, dtype=np.uint8).tobytes()
    pats = [(1, b"[a-z]{1,8}q"), (1, b"[a-m]{2,6}[xyz]")]
    exp = oracle.scan_patterns(pats, data)
    cap = len(exp) + 10
    for mode in (PLAIN, SPEC):
        m = matcher(pats, mode=mode, max_matches=cap)
        got = m.scan_array(data)
        assert np.array_equal(got, exp), mode
        got2 = m.scan_array(data)  # the recorded capacity is kept
        assert np.array_equal(got2, exp), mode


def test_candidate_overflow_device_reports_unknown_then_succeeds():
    import torch
    rng = np.random.default_rng(6)
    data = rng.integers(ord("a"), ord("z") + 1, size=6 << 20, dtype=np.uint8)
    pats = [(1, b"[a-z]{1,8}q")]
    exp = oracle.scan_patterns(pats, data.tobytes())
    cap = len(exp) + 10
    m = matcher(pats, mode=SPEC, max_matches=cap)
    d = torch.from_numpy(data).cuda()
    out = torch.zeros((cap, 3), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    counts = []
    for _ in range(2):
        m.scan_device(d.data_ptr(), d.numel(), out.data_ptr(), cap, cnt.data_ptr())
        torch.cuda.synchronize()
        counts.append(int(cnt.item()) & 0xFFFFFFFFFFFFFFFF)
    assert counts[0] == 0xFFFFFFFFFFFFFFFF  # WS_COUNT_UNKNOWN: the candidates overflowed
    assert counts[1] == len(exp)
    got = oracle.sort_matches(out[:counts[1]].cpu().numpy().astype(np.uint32))
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_nucleotide_config_scaled_vs_oracle(mode):
    # the nucleotide configuration (k-mer literals plus IUPAC-degenerate
    # regexes over ACGT with N runs) at 64 MiB, both regex paths
    wl = w.dna(size=64 << 20)
    # more IUPAC regex samples than the configuration's one plant per MiB
    rng = np.random.default_rng(17)
    r = w.Rng(77)
    rx = w.gen_iupac(200, 5 * 1000 + 2)
    for k in range(600):
        src, pos = rx[k % len(rx)]
        s = bytes(r.choice(w.IUPAC.get(c, c)).encode()[0] for c in pos)
        at = int(rng.integers(0, wl.data.size - 64))
        wl.data[at:at + len(s)] = np.frombuffer(s, dtype=np.uint8)
    m = matcher(wl.patterns, mode=mode, max_matches=1 << 20)
    got = m.scan_array(wl.data)
    exp = oracle.scan_patterns(wl.patterns, wl.data)
    rx_ids = {i for i, (k, _) in enumerate(wl.patterns) if k == 1}
    assert sum(1 for p in exp[:, 0].tolist() if p in rx_ids) >= 100  # regex matches are part of the check
    assert got.shape == exp.shape and np.array_equal(got, exp)


# ------------------------------------------------------------ look-around
LOOK_PATTERNS = [r"^abc", r"abc$", r"\bfoo\b", r"\Bx", r"^\w+$", r"\Aab", r"ab\z", r"a\b.", r"\b[0-9]+\b",
                 r"(?:^|,)ab", r"ab(?:$|,)", r"x\B", r"\w+\b!", r"\Bab\B", r"^[a-z]+ [a-z]+$"]


def _look_data(n, seed):
    rng = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ab cx,fo\n_!y0123", dtype=np.uint8)
    return alpha[rng.integers(0, alpha.size, n)].tobytes()


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_look_around_vs_oracle(mode):
    # ^ $ (multi-line), \b \B (ASCII), \A \z: context groups walked per start
    data = _look_data(1 << 18, 8)
    pats = [(1, p.encode()) for p in LOOK_PATTERNS] + [(1, b"fo[a-z]+"), (0, b"abc")]
    m = matcher(pats, mode=mode, max_matches=1 << 20)
    assert m.info()["regex_context"] == 1
    got = m.scan_array(data)
    exp = oracle.scan_patterns(pats, data)
    assert len(exp) > 1000
    assert np.array_equal(got, exp)


def test_look_around_candidates_and_anchors_at_ends():
    data = b"abc\nabc abc\n foo foo\nab"
    pats = [(1, b"^abc"), (1, b"abc$"), (1, b"\\bfoo\\b"), (1, b"ab\\z"), (1, b"\\Aab")]
    m = matcher(pats)
    exp = oracle.scan_patterns(pats, data)
    assert np.array_equal(m.scan_array(data), exp)
    a = oracle.sort_matches(m.regex_candidates(data, PLAIN))
    b = oracle.sort_matches(m.regex_candidates(data, SPEC))
    assert np.array_equal(a, b)
