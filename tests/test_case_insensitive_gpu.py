"""ASCII case-insensitive literals on the GPU against the oracle, bit-exact.

PatternSetBuilder::case_insensitive(true) (core/src/pattern/compiler.rs:66-76)
builds the literal automata with ascii_case_insensitive (compiler.rs:247-281):
a literal matches wherever the input equals it with A-Z and a-z identified;
regexes are unaffected.  The oracle restates that as contract L over
case-folded bytes.  Covered: the compacting filter (short and long literals),
the large-set lean filter, batch items, stream pieces, and an index loaded
from the reference's on-disk format with its case flag set.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
import workloads as w

pytestmark = pytest.mark.gpu


def _ws():
    import warpstate_b200 as ws
    return ws


def matcher(patterns, ci=True, **cfg):
    ws = _ws()
    b = ws.PatternSet.builder().case_insensitive(ci)
    for kind, p in patterns:
        b = b.literal_bytes(p) if kind == 0 else b.regex(p.decode())
    c = ws.AutoMatcherConfig()
    for k, v in cfg.items():
        getattr(c, k)(v)
    return ws.GpuMatcher.with_config(b.build(), c)


def flip_case(data: np.ndarray, seed: int, frac: float = 0.5) -> np.ndarray:
    """Upper-cases a random fraction of the letters."""
    rng = np.random.default_rng(seed)
    d = data.copy()
    letters = (d >= ord("a")) & (d <= ord("z"))
    d[letters & (rng.random(d.size) < frac)] -= 32
    return d


def test_golden_case_insensitive():
    got = matcher([(0, b"Needle")]).scan_array(b"xxneedlexx NEEDLE nEeDlE")
    assert got.tolist() == [[0, 2, 8], [0, 11, 17], [0, 18, 24]]
    # the flag changes nothing for a case-sensitive set
    assert matcher([(0, b"Needle")], ci=False).scan_array(b"xxneedlexx Needle").tolist() == [[0, 11, 17]]


def test_mixed_lengths_and_regexes_vs_oracle():
    wl = w.literals_small(size=4 << 20, n=100, seed=31)
    rng = np.random.default_rng(3)
    lits = [bytes(flip_case(np.frombuffer(p, dtype=np.uint8), 7 + i)) for i, (_, p) in enumerate(wl.patterns)]
    lits += [b"Q", b"zX", b"AbC", b"\x00\xff", b"abc"]  # short ones, a non-letter pair, a duplicate up to case
    pats = [(0, p) for p in lits] + [(1, b"[a-c]{3}z[0-9]")]
    data = flip_case(wl.data, 11)
    data[rng.integers(0, data.size, 2000)] = rng.integers(0, 256, 2000, dtype=np.uint8)
    got = matcher(pats).scan_array(data)
    exp = oracle.scan_patterns(pats, data, case_insensitive=True)
    assert len(exp) > 1000
    assert np.array_equal(got, exp)


def test_large_set_lean_kernel_vs_oracle():
    wl = w.literals_large(size=32 << 20, n=10_000, seed=32)
    pats = [(0, bytes(flip_case(np.frombuffer(p, dtype=np.uint8), i, 0.3))) for i, (_, p) in enumerate(wl.patterns)]
    data = flip_case(wl.data, 12, 0.3)
    got = matcher(pats).scan_array(data)
    exp = oracle.scan_patterns(pats, data, case_insensitive=True)
    assert len(exp) > 1000
    assert np.array_equal(got, exp)


def test_batch_and_stream_vs_oracle():
    ws = _ws()
    wl = w.batch(n_items=500, n_lit=200, n_rx=20, seed=33, median=2048.0, hi=32 * 1024)
    data = flip_case(wl.data, 13)
    m = matcher(wl.patterns)
    lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
    got = ws.scan_batch_packed(m, data, lens)
    exp = oracle.batch_scan(wl.patterns, data, wl.items, case_insensitive=True)
    assert len(exp) > 50 and np.array_equal(got, exp)
    total = int(lens.sum())
    whole = oracle.scan_patterns(wl.patterns, data[:total], case_insensitive=True)
    sp = ws.StreamPipeline(m).scan_array(data[:total], block=(1 << 16) + 7)
    assert np.array_equal(sp.astype(np.uint32), whole)


def test_index_with_case_flag():
    ws = _ws()
    golden = Path(__file__).resolve().parent / "golden"
    desc = json.loads((golden / "index_fixtures.json").read_text())["case_insensitive"]
    idx = ws.CompiledPatternIndex.load((golden / desc["file"]).read_bytes())
    data = b"xx needle NEEDLE hAyStAcK haystac"
    pats = [(k, t.encode()) for k, t, _ in desc["patterns"]]
    exp = oracle.scan_patterns(pats, data, case_insensitive=True)
    assert [list(m) for m in idx.scan(data)] == exp.tolist()
    assert len(exp) == 3


@pytest.mark.parametrize("name", ["literals", "mixed", "with_dfa_sections"])
def test_index_fixtures_scan_vs_oracle(name):
    # an index in the reference's on-disk layout, loaded into device tables
    ws = _ws()
    golden = Path(__file__).resolve().parent / "golden"
    desc = json.loads((golden / "index_fixtures.json").read_text())[name]
    idx = ws.CompiledPatternIndex.load((golden / desc["file"]).read_bytes())
    pats = [(k, t.encode()) for k, t, _ in desc["patterns"]]
    rng = np.random.default_rng(5)
    pieces = [t.encode() for _, t, _ in desc["patterns"]]
    data = bytearray(rng.integers(0x20, 0x7F, 1 << 16, dtype=np.uint8).tobytes())
    for k in range(0, len(data) - 64, 977):
        p = pieces[k % len(pieces)].replace(b"[0-9]+", b"42").replace(b"[A-Z]{3}-[0-9]+", b"ABC-12") \
            .replace(b"lo[a-d]+", b"load")
        data[k:k + len(p)] = p
    exp = oracle.scan_patterns(pats, bytes(data))
    assert len(exp) > 50
    got = idx.scan(bytes(data))
    assert [list(m) for m in got] == exp.tolist()
