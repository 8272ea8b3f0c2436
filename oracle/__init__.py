"""Python binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py as the checker.  The product
(warpstate_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
_L = None


class OrMatch(ctypes.Structure):
    _fields_ = [("pattern_id", ctypes.c_uint32), ("start", ctypes.c_uint32), ("end", ctypes.c_uint32)]


def lib():
    global _L
    if _L is None:
        so = _DIR / "liboracle.so"
        if not so.exists():
            subprocess.run(["make", "-s", "-C", str(_DIR)], check=True)
        L = ctypes.CDLL(str(so))
        u8p, u32p = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint32)
        L.or_fnv1a.restype = ctypes.c_uint32
        L.or_fnv1a.argtypes = [u8p, ctypes.c_size_t, ctypes.c_size_t]
        L.or_prefilter_build.restype = ctypes.c_int
        L.or_prefilter_build.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_uint32, u32p, u32p, u32p, u32p]
        L.or_literal_scan.restype = ctypes.c_uint64
        L.or_literal_scan.argtypes = [u8p, u32p, u32p, ctypes.c_uint32, ctypes.c_uint32, u8p, ctypes.c_uint64,
                                      ctypes.POINTER(OrMatch), ctypes.c_uint64, ctypes.c_int]
        L.or_regex_new.restype = ctypes.c_void_p
        L.or_regex_new.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
        L.or_regex_free.argtypes = [ctypes.c_void_p]
        L.or_regex_nullable.restype = ctypes.c_int
        L.or_regex_nullable.argtypes = [ctypes.c_void_p]
        L.or_regex_maxlen.restype = ctypes.c_longlong
        L.or_regex_maxlen.argtypes = [ctypes.c_void_p]
        L.or_regex_literal.restype = ctypes.c_int
        L.or_regex_literal.argtypes = [ctypes.c_char_p, u8p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.or_regex_pathological.restype = ctypes.c_int
        L.or_regex_pathological.argtypes = [ctypes.c_char_p]
        L.or_regex_find_iter.restype = ctypes.c_uint64
        L.or_regex_find_iter.argtypes = [ctypes.c_void_p, u8p, ctypes.c_uint64, u32p, u32p, ctypes.c_uint64]
        L.or_regex_set_scan.restype = ctypes.c_uint64
        L.or_regex_set_scan.argtypes = [ctypes.POINTER(ctypes.c_void_p), u32p, ctypes.c_uint32, u8p,
                                        ctypes.c_uint64, ctypes.POINTER(OrMatch), ctypes.c_uint64, ctypes.c_int]
        L.or_batch_scan.restype = ctypes.c_uint64
        L.or_batch_scan.argtypes = [u8p, u32p, u32p, ctypes.c_uint32, ctypes.c_uint32,
                                    ctypes.POINTER(ctypes.c_void_p), u32p, ctypes.c_uint32, u8p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                    ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int]
        L.or_sort_matches.argtypes = [ctypes.POINTER(OrMatch), ctypes.c_uint64]
        L.or_hw_threads.restype = ctypes.c_int
        _L = L
    return _L


def _u8(a):
    a = np.ascontiguousarray(np.frombuffer(a, dtype=np.uint8) if isinstance(a, (bytes, bytearray)) else a,
                             dtype=np.uint8)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def fnv1a(b: bytes, window: int = 8) -> int:
    a, p = _u8(b if b else b"\0")
    return lib().or_fnv1a(p, len(b), window)


def prefilter_table(offsets, hashes, window=8):
    offs, po = _u32(np.asarray(offsets, dtype=np.uint32).reshape(-1))
    hs, ph = _u32(hashes)
    n = len(hs)
    nb = ctypes.c_uint32()
    lib().or_prefilter_build(po, ph, n, window, None, None, ctypes.byref(nb), None)
    meta = np.zeros(4 * window, dtype=np.uint32)
    ranges = np.zeros(2 * max(nb.value, 1), dtype=np.uint32)
    ents = np.zeros(2 * max(n, 1), dtype=np.uint32)
    lib().or_prefilter_build(po, ph, n, window, _u32(meta)[1] if False else meta.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                             ranges.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.byref(nb),
                             ents.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return meta.reshape(-1, 4), ranges[: 2 * nb.value].reshape(-1, 2), ents[: 2 * n].reshape(-1, 2)


def _to_array(buf, n) -> np.ndarray:
    if n == 0:
        return np.zeros((0, 3), dtype=np.uint32)
    return np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_uint32)), shape=(n * 3,)).reshape(n, 3).copy()


def literal_scan(literals: list[bytes], pattern_ids, data, threads: int = 0) -> np.ndarray:
    """Contract L: (pattern_id, start, end) of every occurrence, unsorted."""
    if not literals:
        return np.zeros((0, 3), dtype=np.uint32)
    packed = b"".join(literals)
    offs = []
    o = 0
    for l in literals:
        offs += [o, len(l)]
        o += len(l)
    pk, ppk = _u8(packed)
    of, pof = _u32(offs)
    ids, pids = _u32(pattern_ids)
    d, pd = _u8(data)
    cap = 1 << 16
    while True:
        out = (OrMatch * cap)()
        n = lib().or_literal_scan(ppk, pof, pids, len(literals), 8, pd, len(d), out, cap, threads)
        if n <= cap:
            return _to_array(out, n)
        cap = int(n)


class Regex:
    def __init__(self, pattern: str | bytes):
        src = pattern.encode() if isinstance(pattern, str) else pattern
        err = ctypes.create_string_buffer(256)
        h = lib().or_regex_new(src, err, 256)
        if not h:
            raise ValueError(err.value.decode())
        self.h = h
        self.source = src

    @property
    def nullable(self) -> bool:
        return bool(lib().or_regex_nullable(self.h))

    @property
    def maxlen(self) -> int:
        """Longest match in bytes, -1 when unbounded."""
        return int(lib().or_regex_maxlen(self.h))

    def find_iter(self, data) -> list[tuple[int, int]]:
        d, pd = _u8(data)
        cap = 1 << 12
        while True:
            s = np.zeros(cap, dtype=np.uint32)
            e = np.zeros(cap, dtype=np.uint32)
            n = lib().or_regex_find_iter(self.h, pd, len(d), s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                         e.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), cap)
            if n <= cap:
                return list(zip(s[:n].tolist(), e[:n].tolist()))
            cap = int(n)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_regex_free(self.h)
            self.h = None


def regex_literal(pattern: str) -> bytes | None:
    buf = (ctypes.c_uint8 * 4096)()
    n = ctypes.c_size_t()
    r = lib().or_regex_literal(pattern.encode(), buf, 4096, ctypes.byref(n))
    if r != 1:
        return None
    return bytes(buf[: n.value])


def regex_pathological(pattern: str) -> bool:
    return lib().or_regex_pathological(pattern.encode()) == 1


def regex_scan(regexes: list["Regex"], pattern_ids, data, threads: int = 0) -> np.ndarray:
    """Contract R for many regexes: (pattern_id, start, end), unsorted."""
    if not regexes:
        return np.zeros((0, 3), dtype=np.uint32)
    hs = (ctypes.c_void_p * len(regexes))(*[r.h for r in regexes])
    ids, pids = _u32(pattern_ids)
    d, pd = _u8(data)
    cap = 1 << 16
    while True:
        out = (OrMatch * cap)()
        n = lib().or_regex_set_scan(hs, pids, len(regexes), pd, len(d), out, cap, threads)
        if n <= cap:
            return _to_array(out, n)
        cap = int(n)


def sort_matches(a: np.ndarray) -> np.ndarray:
    """Canonical order (start, pattern_id, end)."""
    if len(a) == 0:
        return a.reshape(0, 3)
    idx = np.lexsort((a[:, 2], a[:, 0], a[:, 1]))
    return a[idx]


_FOLD = np.arange(256, dtype=np.uint8)
_FOLD[ord("A"):ord("Z") + 1] |= 0x20


def ascii_fold(data) -> np.ndarray:
    """A-Z mapped to a-z, every other byte unchanged: the byte equivalence of
    an Aho-Corasick automaton built with ascii_case_insensitive(true), which
    PatternSetBuilder::case_insensitive selects for the literal patterns
    (core/src/pattern/compiler.rs:66-76,247-281)."""
    a = np.frombuffer(data, dtype=np.uint8) if isinstance(data, (bytes, bytearray)) else np.asarray(data)
    return _FOLD[a.view(np.uint8).reshape(-1)]


def scan_patterns(patterns: list[tuple[int, bytes]], data, threads: int = 0,
                  case_insensitive: bool = False) -> np.ndarray:
    """The full parity contract of a pattern list: literal patterns (and regexes
    the reference demotes to literals) under L, the other regexes under R,
    sorted by (start, pattern_id, end).  With ``case_insensitive`` the
    literals match ASCII case-insensitively (L over case-folded bytes);
    regexes are unaffected."""
    lits, lit_ids, rxs, rx_ids = split_patterns(patterns)
    if case_insensitive:
        lit_part = literal_scan([bytes(ascii_fold(l)) for l in lits], lit_ids, ascii_fold(data), threads)
    else:
        lit_part = literal_scan(lits, lit_ids, data, threads)
    parts = [lit_part, regex_scan(rxs, rx_ids, data, threads)]
    return sort_matches(np.concatenate(parts, axis=0))


def split_patterns(patterns: list[tuple[int, bytes]]):
    """(literals, literal ids, Regex handles, regex ids), with the reference's
    regex -> literal demotion applied."""
    lits, lit_ids, rxs, rx_ids = [], [], [], []
    for i, (kind, b) in enumerate(patterns):
        if kind == 0:
            lits.append(bytes(b))
            lit_ids.append(i)
        else:
            src = b.decode() if isinstance(b, (bytes, bytearray)) else b
            lit = regex_literal(src)
            if lit:
                lits.append(lit)
                lit_ids.append(i)
            else:
                rxs.append(Regex(src))
                rx_ids.append(i)
    return lits, lit_ids, rxs, rx_ids


TAGGED = np.dtype([("sid", "<u8"), ("pid", "<u4"), ("start", "<u4"), ("end", "<u4"), ("res", "<u4")])


def batch_scan(patterns: list[tuple[int, bytes]], data, items, ids=None, threads: int = 0,
               case_insensitive: bool = False) -> np.ndarray:
    """Batch contract (scan_batch_cpu, core/src/batch.rs:170-195): items are
    (offset, length) slices of ``data``, each scanned on its own; returns an
    (n, 4) uint64 array (source_id, pattern_id, start, end) sorted by
    (source_id, start, pattern_id, end).  ``case_insensitive`` as in
    scan_patterns."""
    if case_insensitive:
        # literal part on folded bytes, regex part on the bytes as they are
        lits, lit_ids, rxs, rx_ids = split_patterns(patterns)
        a = _batch_scan_split([bytes(ascii_fold(l)) for l in lits], lit_ids, [], [], ascii_fold(data), items, ids,
                              threads)
        b = _batch_scan_split([], [], rxs, rx_ids, data, items, ids, threads)
        r = np.concatenate([a, b], axis=0)
        return r[np.lexsort((r[:, 3], r[:, 1], r[:, 2], r[:, 0]))]
    lits, lit_ids, rxs, rx_ids = split_patterns(patterns)
    return _batch_scan_split(lits, lit_ids, rxs, rx_ids, data, items, ids, threads)


def _batch_scan_split(lits, lit_ids, rxs, rx_ids, data, items, ids, threads) -> np.ndarray:
    packed = b"".join(lits)
    offs, o = [], 0
    for l in lits:
        offs += [o, len(l)]
        o += len(l)
    pk, ppk = _u8(packed if packed else b"\0")
    of, pof = _u32(offs if offs else [0, 0])
    li, pli = _u32(lit_ids if lit_ids else [0])
    ri, pri = _u32(rx_ids if rx_ids else [0])
    hs = (ctypes.c_void_p * max(len(rxs), 1))(*[r.h for r in rxs])
    d, pd = _u8(data)
    it = np.asarray(items, dtype=np.uint64).reshape(-1, 2)
    off = np.ascontiguousarray(it[:, 0])
    ln = np.ascontiguousarray(it[:, 1])
    sid = np.arange(len(it), dtype=np.uint64) if ids is None else np.ascontiguousarray(ids, dtype=np.uint64)
    cap = 1 << 16
    while True:
        out = np.empty(cap, dtype=TAGGED)
        n = lib().or_batch_scan(ppk, pof, pli, len(lits), 8, hs, pri, len(rxs), pd, off.ctypes.data,
                                ln.ctypes.data, sid.ctypes.data, len(it), out.ctypes.data, cap, threads)
        if n <= cap:
            o = out[:n]
            res = np.empty((n, 4), dtype=np.uint64)
            res[:, 0], res[:, 1], res[:, 2], res[:, 3] = o["sid"], o["pid"], o["start"], o["end"]
            return res
        cap = int(n)


def hw_threads() -> int:
    return lib().or_hw_threads()
