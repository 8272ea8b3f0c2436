"""CompiledPatternIndex load / save on the CPU (no device calls).

The fixtures under tests/golden/ are written field by field in the
reference's on-disk layout by tests/golden/make_index_fixtures.py
(core/src/compiled_index/builder.rs:8-64).  The library must load each of
them with the stored tables intact, write the same bytes back for the same
pattern set, and reject the corruptions the reference's own tests reject
(core/src/compiled_index/tests.rs and adversarial_tests/) with
PatternCompilationFailed.
"""
import json
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
FIX = json.loads((GOLDEN / "index_fixtures.json").read_text())


def _ws():
    import warpstate_b200 as ws
    return ws


def _builder(desc):
    ws = _ws()
    b = ws.PatternSetBuilder().case_insensitive(desc["case_insensitive"])
    for k, t, n in desc["patterns"]:
        if k == 0:
            b = b.named_literal(n, t) if n else b.literal(t)
        else:
            b = b.named_regex(n, t) if n else b.regex(t)
    return b


@pytest.mark.parametrize("name", sorted(FIX))
def test_fixture_loads_with_stored_tables(name):
    ws = _ws()
    desc = FIX[name]
    blob = (GOLDEN / desc["file"]).read_bytes()
    idx = ws.CompiledPatternIndex.load(blob)
    assert idx.names() == [n for _, _, n in desc["patterns"]]
    ir = idx.to_pattern_set().ir()
    assert ir["literal_pattern_ids"].tolist() == desc["literal_pattern_ids"]
    assert [i for i, _ in ir["regex_patterns"]] == desc["regex_pattern_ids"]
    # the literal tables are the reference's LiteralPrefilterTable (oracle restatement)
    offs = ir["offsets"].reshape(-1)
    lits = [ir["packed_bytes"][s:s + n] for s, n in ir["offsets"].tolist()]
    meta, ranges, entries = oracle.prefilter_table(offs, [oracle.fnv1a(l) for l in lits])
    assert np.array_equal(ir["prefix_meta"], meta)
    assert np.array_equal(ir["bucket_ranges"], ranges)
    assert np.array_equal(ir["entries"], entries)


@pytest.mark.parametrize("name", sorted(FIX))
def test_writer_reproduces_fixture(name):
    ws = _ws()
    desc = FIX[name]
    blob = (GOLDEN / desc["file"]).read_bytes()
    mine = ws.CompiledPatternIndex.build(_builder(desc).build())
    if desc["dfa_sections"] == 0:
        assert mine == blob
    # either way the written index loads back to the same pattern set
    a = ws.CompiledPatternIndex.load(mine).to_pattern_set().ir()
    b = ws.CompiledPatternIndex.load(blob).to_pattern_set().ir()
    for key in ("packed_bytes", "regex_patterns"):
        assert a[key] == b[key]
    for key in ("offsets", "literal_pattern_ids", "prefix_meta", "bucket_ranges", "entries"):
        assert np.array_equal(a[key], b[key])


def _reseal(body: bytes) -> bytes:
    """A version 3 image with its CRC recomputed after an edit."""
    return body + struct.pack("<I", zlib.crc32(body) & 0xFFFFFFFF)


def _rejects(blob):
    ws = _ws()
    with pytest.raises(ws.PatternCompilationFailed):
        ws.CompiledPatternIndex.load(blob)


def test_corrupt_images_are_rejected():
    blob = (GOLDEN / FIX["mixed"]["file"]).read_bytes()
    body = blob[:-4]
    _rejects(b"not-an-index")                                       # tests.rs:34-38
    _rejects(blob[: len(blob) // 2])                                # truncated_index_rejected
    _rejects(blob[:-1] + bytes([blob[-1] ^ 0x01]))                  # CRC mismatch
    _rejects(body[:20] + bytes([body[20] ^ 0x10]) + body[21:] + blob[-4:])  # a flipped bit
    _rejects(_reseal(b"WPSIDX02" + body[8:]))                        # wrong magic
    _rejects(_reseal(body[:8] + struct.pack("<I", 4) + body[12:])[:-4] + b"\0\0\0\0")  # future version
    _rejects(_reseal(body + b"x"))                                   # trailing bytes
    # header counts that disagree with the tables
    for field in (2, 3, 4):  # pattern, literal and regex-DFA counts (after version, case flag)
        off = 8 + 4 * field
        v = struct.unpack_from("<I", body, off)[0]
        _rejects(_reseal(body[:off] + struct.pack("<I", v + 1) + body[off + 4:]))
    # packed length past the end of the image
    off = 8 + 4 * 6
    _rejects(_reseal(body[:off] + struct.pack("<I", 0x7FFFFFFF) + body[off + 4:]))


def test_every_truncation_is_rejected():
    # adversarial_tests/load_truncated_at_various_boundaries.rs
    blob = (GOLDEN / FIX["literals"]["file"]).read_bytes()
    for n in range(len(blob)):
        _rejects(blob[:n])


def test_offset_past_packed_bytes_and_bad_name():
    ws = _ws()
    ps = ws.PatternSet.builder().literal("abcd").named_literal("nm", "efgh").build()
    body = ws.CompiledPatternIndex.build(ps)[:-4]
    # the first offset pair follows the packed bytes: (start, len) of "abcd"
    packed_len = struct.unpack_from("<I", body, 32)[0]
    off = 36 + packed_len + 4
    _rejects(_reseal(body[:off] + struct.pack("<II", packed_len - 2, 4) + body[off + 8:]))
    _rejects(_reseal(body[:off] + struct.pack("<II", 0xFFFFFFFF, 4) + body[off + 8:]))
    name_at = body.index(b"nm")
    _rejects(_reseal(body[:name_at] + b"\xff\xfe" + body[name_at + 2:]))  # not UTF-8


def test_older_versions():
    ws = _ws()
    # version 2: no CRC trailer, regex sources present
    blob = (GOLDEN / FIX["mixed"]["file"]).read_bytes()[:-4]
    v2 = blob[:8] + struct.pack("<I", 2) + blob[12:]
    idx = ws.CompiledPatternIndex.load(v2)
    assert [i for i, _ in idx.to_pattern_set().ir()["regex_patterns"]] == FIX["mixed"]["regex_pattern_ids"]
    # version 1: no regex-source section; fine for literals only
    lit = (GOLDEN / FIX["literals"]["file"]).read_bytes()[:-4]
    names_end = _names_end(lit)
    v1 = lit[:8] + struct.pack("<I", 1) + lit[12:names_end] + lit[names_end + 4:]  # drop the empty regex table
    assert ws.CompiledPatternIndex.load(v1).literal_count() == 6
    _rejects(b"WPSIDX01" + struct.pack("<I", 0) + lit[12:])  # version 0


def _names_end(body: bytes) -> int:
    """Offset of the regex-source table of a version >= 2 image."""
    off = 8 + 4 * 6
    packed_len = struct.unpack_from("<I", body, off)[0]
    off += 4 + packed_len
    n = struct.unpack_from("<I", body, off)[0]
    off += 4 + 8 * n
    n = struct.unpack_from("<I", body, off)[0]
    off += 4
    for _ in range(n):
        ln = struct.unpack_from("<I", body, off)[0]
        off += 4 + (0 if ln == 0xFFFFFFFF else ln)
    return off


def test_oversized_file_is_input_too_large(tmp_path):
    ws = _ws()
    p = tmp_path / "big.idx"
    with open(p, "wb") as f:
        f.truncate(ws.CompiledPatternIndex.MAX_BYTES + 1)  # sparse
    with pytest.raises(ws.InputTooLarge):
        ws.CompiledPatternIndex.load_from_file(p)


def test_save_and_load_from_file(tmp_path):
    ws = _ws()
    ps = ws.PatternSet.builder().literal("disk").regex("lo[a-d]+").build()
    idx = ws.CompiledPatternIndex.load(ws.CompiledPatternIndex.build(ps))
    idx.save_to_file(tmp_path / "x.idx")
    again = ws.CompiledPatternIndex.load_from_file(tmp_path / "x.idx")
    assert again.to_bytes() == idx.to_bytes()
