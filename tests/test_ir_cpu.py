"""The product's pattern-IR builder against the oracle's restatement (CPU only)."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import warpstate_b200 as ws
from conftest import ROOT


def build(pairs):
    b = ws.PatternSet.builder()
    for kind, p in pairs:
        b = b.literal(p) if kind == "literal" else b.regex(p)
    return b.build()


def test_build_errors(golden):
    names = {"EmptyPatternSet": ws.EmptyPatternSet, "EmptyPattern": ws.EmptyPattern,
             "PathologicalRegex": ws.PathologicalRegex}
    for case in golden["build_errors"]:
        if case["error"] is None:
            build(case["patterns"])
            continue
        with pytest.raises(names[case["error"]]) as ei:
            build(case["patterns"])
        if "index" in case:
            assert ei.value.index == case["index"], case["src"]


def test_literal_demotion_counts(golden):
    for case in golden["demotion"]:
        ps = build(case["patterns"])
        ir = ps.ir()
        assert len(ir["offsets"]) == case["literals"], case["src"]
        assert len(ir["regex_patterns"]) == case["regexes"], case["src"]
        assert len(ps) == len(case["patterns"])


def test_demotion_agrees_with_oracle():
    pats = ["needle", "(needle)", "(?:abc)", "foo\\.bar", "(?i:hello)", "(?i)123", "[a]b", "a{1}",
            "ab|cd", "\\x41\\x42", "()", "a()", "café", "[0-9]"]
    for p in pats:
        ps = build([["regex", p]])
        ir = ps.ir()
        lit = oracle.regex_literal(p)
        if lit:
            assert ir["packed_bytes"] == lit, p
        else:
            assert len(ir["regex_patterns"]) == 1, p


def test_prefilter_table_matches_oracle():
    import workloads as w
    alpha, wts = w.zipf_alphabet(11)
    lits = w.gen_literals(3000, 1, 20, alpha, wts, 12)
    ps = ws.PatternSet.builder()
    for l in lits:
        ps = ps.literal_bytes(l)
    ir = ps.build().ir()
    hashes = [oracle.fnv1a(l, 8) for l in lits]
    offs = np.array(ir["offsets"]).reshape(-1)
    meta, ranges, ents = oracle.prefilter_table(offs, hashes, 8)
    assert np.array_equal(ir["prefix_meta"], meta)
    assert np.array_equal(ir["bucket_ranges"], ranges)
    assert np.array_equal(ir["entries"], ents)
    # entries carry the FNV-1a hash of each literal
    assert np.array_equal(ir["entries"][:, 0][np.argsort(ir["entries"][:, 1], kind="stable")], np.array(hashes, dtype=np.uint32))


def test_invalid_regex_reports_index():
    with pytest.raises(ws.PatternCompilationFailed) as ei:
        build([["literal", "ok"], ["regex", "(unclosed"]])
    assert "index 1" in str(ei.value)


def test_header_symbols_exported():
    hdr = (ROOT / "include" / "warpstate.h").read_text()
    decls = set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(ws_\w+)\s*\(", hdr, flags=re.M))
    assert len(decls) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "warpstate_b200" / "libwarpstate_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = sorted(d for d in decls if d not in exported)
    assert not missing, missing
    from warpstate_b200 import _native
    assert set(_native.SIGNATURES) == decls
