"""Writes the CompiledPatternIndex fixtures under tests/golden/.

Each fixture is a byte image in the reference's on-disk layout, written here
field by field from core/src/compiled_index/builder.rs:8-64 (magic, version,
header counts, packed bytes, offsets, names, regex sources, literal ids, the
LiteralPrefilterTable, per-DFA sections, CRC-32), independently of the
library's own writer.  The literal tables come from the oracle's restatement
of LiteralPrefilterTable::build and the FNV-1a prefix hash; regex literal
demotion follows the oracle too.  The regex DFA sections cannot hold real
regex-automata serializations here, so the ``with_dfa_sections`` fixture
carries sections of valid shape with opaque payloads: a loader has to walk
them and take the regexes from their sources.  Run from the repository root:

    python tests/golden/make_index_fixtures.py
"""
from __future__ import annotations

import json
import struct
import sys
import zlib
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, case_insensitive, patterns as (kind, text, name or None), extra DFA sections)
SETS = [
    ("literals", False, [(0, "alpha", None), (0, "beta", "greek"), (0, "pattern_042", None), (0, "ab", None),
                         (0, "a", None), (0, "a much longer literal, over eight bytes", "long")], 0),
    ("mixed", False, [(0, "alpha", None), (1, "b[0-9]+", None), (0, "beta", None), (1, "[A-Z]{3}-[0-9]+", "key"),
                      (1, "needle", None)], 0),
    ("with_dfa_sections", False, [(0, "disk", None), (1, "lo[a-d]+", None), (0, "x\x00y", "nul")], 2),
    ("case_insensitive", True, [(0, "Needle", None), (0, "HAYstack", None)], 0),
]


def u32(v: int) -> bytes:
    return struct.pack("<I", v)


def fixture(ci: bool, pats, n_dfa_sections: int) -> tuple[bytes, dict]:
    lits, lit_ids, regexes = [], [], []
    for i, (kind, text, _) in enumerate(pats):
        b = text.encode("utf-8")
        if kind == 0:
            lits.append(b)
            lit_ids.append(i)
        else:
            demoted = oracle.regex_literal(text)
            if demoted:
                lits.append(demoted)
                lit_ids.append(i)
            else:
                regexes.append((i, b))
    packed = b"".join(lits)
    offsets, o = [], 0
    for l in lits:
        offsets.append((o, len(l)))
        o += len(l)
    hashes = [oracle.fnv1a(l, 8) for l in lits]
    meta, ranges, entries = oracle.prefilter_table([x for p in offsets for x in p], hashes, 8)
    out = bytearray(b"WPSIDX01")
    out += u32(3) + u32(1 if ci else 0) + u32(len(pats)) + u32(len(lits)) + u32(n_dfa_sections) + u32(8)
    out += u32(len(packed)) + packed
    out += u32(len(offsets)) + b"".join(u32(s) + u32(n) for s, n in offsets)
    out += u32(len(pats))
    for _, _, name in pats:
        if name is None:
            out += u32(0xFFFFFFFF)
        else:
            nb = name.encode("utf-8")
            out += u32(len(nb)) + nb
    out += u32(len(regexes)) + b"".join(u32(i) + u32(len(b)) + b for i, b in regexes)
    out += u32(len(lit_ids)) + b"".join(u32(i) for i in lit_ids)
    out += u32(len(meta)) + b"".join(u32(int(x)) for row in meta for x in row)
    out += u32(len(ranges)) + b"".join(u32(int(x)) for row in ranges for x in row)
    out += u32(len(entries)) + b"".join(u32(int(x)) for row in entries for x in row)
    for k in range(n_dfa_sections):
        classes = 3
        out += u32(2 * classes) + b"".join(u32(x) for x in (1, 0x40000000, 1, 0x80000001, 0, 0))  # transitions
        out += u32(3) + u32(0) + u32(0) + u32(1)  # match-list pointers
        out += u32(1) + u32(0)                    # match lists
        out += u32(1) + u32(0)                    # pattern lengths
        out += u32(0) + u32(classes) + u32(classes - 1)  # start state, class count, eoi class
        out += b"".join(u32(b % (classes - 1)) for b in range(256))  # byte classes
        blob = bytes((7 * j + k) & 0xFF for j in range(40))
        out += u32(len(blob)) + blob              # serialized DFA (opaque here)
        out += u32(1) + u32(regexes[k % len(regexes)][0] if regexes else 0)  # original ids
    out += u32(zlib.crc32(bytes(out)) & 0xFFFFFFFF)
    desc = {"case_insensitive": ci, "patterns": [[k, t, n] for k, t, n in pats], "dfa_sections": n_dfa_sections,
            "literal_pattern_ids": lit_ids, "regex_pattern_ids": [i for i, _ in regexes]}
    return bytes(out), desc


def main():
    index = {}
    for name, ci, pats, ndfa in SETS:
        blob, desc = fixture(ci, pats, ndfa)
        (OUT / f"index_{name}.bin").write_bytes(blob)
        desc["file"] = f"index_{name}.bin"
        index[name] = desc
    (OUT / "index_fixtures.json").write_text(json.dumps(index, indent=1) + "\n")
    print(f"wrote {len(index)} fixtures")


if __name__ == "__main__":
    main()
