"""warpstate_b200 -- B200-native (sm_100a) GPU scan path of warpstate.

Python mirror of the reference's Rust API for the scan path, over the C ABI in
include/warpstate.h:

* ``PatternSet.builder() ... .build()``  (core/src/pattern/compiler.rs:97)
* ``GpuMatcher`` / ``WarpStateer``: ``new``, ``with_config``, ``scan``,
  ``scan_blocking``, ``scan_block``, ``max_block_size`` (core/src/gpu/mod.rs:95-445)
* ``GpuScanner`` (core/src/gpu/scanner.rs:14-120)
* ``AutoMatcher``: always routes to the GPU (core/src/router.rs:59-305)
* ``ScanItem``, ``TaggedMatch``, ``scan_batch``, ``scan_batch_gpu``,
  ``scan_batch_auto``, ``BatchConfig`` (core/src/batch.rs)
* ``StreamPipeline`` (core/src/pipeline.rs:87-153)
* ``AutoMatcherConfig`` (core/src/config.rs:39-173) and the ``Error`` family
  (core/src/error.rs:6-91).

Scan semantics: literal patterns report every (overlapping) occurrence;
regex patterns report regex::bytes ``find_iter`` matches (leftmost-first,
non-overlapping, multi_line on, Unicode off); results are sorted by
``(start, pattern_id, end)``.  Everything runs on the GPU; there is no CPU
fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Iterable, NamedTuple, Sequence

import numpy as np

from . import _native as N

__all__ = [
    "Match", "Error", "EmptyPatternSet", "EmptyPattern", "NoGpuAdapter", "GpuDeviceError", "BufferMapFailed",
    "PatternCompilationFailed", "DfaOutOfBounds", "PatternTooLarge", "PatternSetTooLarge", "InputTooLarge",
    "MatchBufferOverflow", "PathologicalRegex", "PatternSet", "PatternSetBuilder", "AutoMatcherConfig",
    "GpuMatcher", "WarpStateer", "GpuScanner", "AutoMatcher", "ScanItem", "TaggedMatch", "BatchConfig",
    "scan_batch", "scan_batch_gpu", "scan_batch_auto", "StreamPipeline", "REGEX_SPECULATIVE", "REGEX_PLAIN",
    "CompiledPatternIndex", "HotSwapPatternSet", "ZeroCopyScan",
]

REGEX_SPECULATIVE = 0
REGEX_PLAIN = 1
PROPOSER_MLP = 0
PROPOSER_NONE = 1
CAND_DISTINCT = 0x100  # ws_regex_candidates: the candidates a scan works from


class Match(NamedTuple):
    """``Match { pattern_id, start, end }`` (three u32)."""
    pattern_id: int
    start: int
    end: int


# ------------------------------------------------------------------ errors
class Error(Exception):
    """Base of the error family of core/src/error.rs:6-91."""


class EmptyPatternSet(Error):
    pass


class EmptyPattern(Error):
    def __init__(self, index, msg=""):
        super().__init__(msg or f"pattern {index} is empty")
        self.index = index


class NoGpuAdapter(Error):
    pass


class GpuDeviceError(Error):
    def __init__(self, reason):
        super().__init__(reason)
        self.reason = reason


class BufferMapFailed(Error):
    pass


class PatternCompilationFailed(Error):
    def __init__(self, reason):
        super().__init__(reason)
        self.reason = reason


class DfaOutOfBounds(Error):
    pass


class PatternTooLarge(Error):
    def __init__(self, index, nbytes, maximum):
        super().__init__(f"pattern {index} has {nbytes} bytes (max {maximum})")
        self.index, self.bytes, self.max = index, nbytes, maximum


class PatternSetTooLarge(Error):
    pass


class InputTooLarge(Error):
    def __init__(self, nbytes, max_bytes):
        super().__init__(f"scan input is too large ({nbytes} bytes, max {max_bytes})")
        self.bytes, self.max_bytes = nbytes, max_bytes


class MatchBufferOverflow(Error):
    def __init__(self, count, maximum):
        super().__init__(f"too many matches ({count} exceeds {maximum})")
        self.count, self.max = count, maximum


class PathologicalRegex(Error):
    def __init__(self, index):
        super().__init__(f"regex pattern {index} contains nested repetitions (pathological)")
        self.index = index


def _raise(status: int, err: N.WsErrorInfo):
    msg = err.message.decode(errors="replace")
    if status == 1:
        raise EmptyPatternSet(msg)
    if status == 2:
        raise EmptyPattern(err.index, msg)
    if status == 3:
        raise NoGpuAdapter(msg)
    if status == 4:
        raise GpuDeviceError(msg)
    if status == 5:
        raise BufferMapFailed(msg)
    if status == 6:
        raise PatternCompilationFailed(msg)
    if status == 7:
        raise DfaOutOfBounds(msg)
    if status == 8:
        raise PatternTooLarge(err.index, err.count, err.max)
    if status == 9:
        raise PatternSetTooLarge(msg)
    if status == 10:
        raise InputTooLarge(err.count, err.max)
    if status == 11:
        raise MatchBufferOverflow(err.count, err.max)
    if status == 12:
        raise PathologicalRegex(err.index)
    if status == 13:
        raise GpuDeviceError(msg or "GPU operation timed out")
    raise ValueError(msg or f"invalid argument (status {status})")


def _call(fn, *args):
    err = N.WsErrorInfo()
    st = fn(*args, ctypes.byref(err))
    if st != 0:
        _raise(st, err)


# ------------------------------------------------------------ input views
def _buffer(data):
    """(pointer, length, keepalive) for bytes-like or numpy input, zero-copy."""
    if isinstance(data, np.ndarray):
        a = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
        return a.ctypes.data, a.nbytes, a
    if isinstance(data, (bytes,)):
        p = ctypes.c_char_p(data)
        return ctypes.cast(p, ctypes.c_void_p).value, len(data), (data, p)
    if isinstance(data, (bytearray, memoryview)):
        mv = memoryview(data).cast("B")
        if mv.readonly:
            b = bytes(mv)
            return _buffer(b)
        arr = (ctypes.c_char * mv.nbytes).from_buffer(mv) if mv.nbytes else None
        return (ctypes.addressof(arr) if arr is not None else 0), mv.nbytes, (mv, arr)
    if hasattr(data, "data_ptr") and hasattr(data, "numel"):  # a CPU torch tensor (e.g. pinned)
        return data.data_ptr(), data.numel() * data.element_size(), data
    raise TypeError(f"unsupported input type {type(data)!r}")


# ---------------------------------------------------------- pattern set
class PatternSetBuilder:
    """Builder for PatternSet (core/src/pattern/compiler.rs:13-93)."""

    def __init__(self):
        self._patterns: list[tuple[int, bytes, str | None]] = []
        self._ci = False
        self._dfa_size_limit = 50_000_000

    def literal(self, pattern: str):
        self._patterns.append((0, pattern.encode("utf-8"), None))
        return self

    def literal_bytes(self, pattern: bytes):
        self._patterns.append((0, bytes(pattern), None))
        return self

    def named_literal(self, name: str, pattern: str):
        self._patterns.append((0, pattern.encode("utf-8"), name))
        return self

    def regex(self, pattern: str):
        self._patterns.append((1, pattern.encode("utf-8"), None))
        return self

    def named_regex(self, name: str, pattern: str):
        self._patterns.append((1, pattern.encode("utf-8"), name))
        return self

    def case_insensitive(self, yes: bool):
        self._ci = bool(yes)
        return self

    def dfa_size_limit(self, limit: int):
        self._dfa_size_limit = int(limit)
        return self

    def build(self) -> "PatternSet":
        L = N.lib()
        n = len(self._patterns)
        specs = (N.WsPatternSpec * max(n, 1))()
        keep = []
        for i, (k, b, _) in enumerate(self._patterns):
            buf = ctypes.create_string_buffer(b, len(b)) if b else None
            keep.append(buf)
            specs[i].kind = k
            specs[i].bytes = ctypes.cast(buf, ctypes.c_void_p).value if buf is not None else None
            specs[i].len = len(b)
        h = ctypes.c_void_p()
        _call(L.ws_ir_build, specs, n, 1 if self._ci else 0, ctypes.byref(h))
        for i, (_, _, name) in enumerate(self._patterns):
            if name is not None:
                nb = name.encode("utf-8")
                _call_noerr(L.ws_ir_set_name, h, i, nb, len(nb))
        return PatternSet(h, [p[2] for p in self._patterns], self._dfa_size_limit)


class PatternSet:
    """A compiled pattern set (core/src/pattern/mod.rs:74-279), host side."""

    def __init__(self, handle, names, dfa_size_limit):
        self._h = handle
        self.dfa_size_limit = dfa_size_limit
        t = N.WsPatternTables()
        _call_noerr(N.lib().ws_ir_tables, self._h, ctypes.byref(t))
        self._tables = t
        if names is None:  # names stored with the IR (a loaded index)
            names = []
            n = ctypes.c_uint64()
            buf = ctypes.create_string_buffer(4096)
            for i in range(t.n_patterns):
                st = N.lib().ws_ir_name(self._h, i, buf, 4096, ctypes.byref(n))
                if st == 11:
                    buf = ctypes.create_string_buffer(n.value)
                    st = N.lib().ws_ir_name(self._h, i, buf, n.value, ctypes.byref(n))
                names.append(None if st != 0 or n.value == 0xFFFFFFFFFFFFFFFF else buf.raw[: n.value].decode())
        self.names = names

    @staticmethod
    def builder() -> PatternSetBuilder:
        return PatternSetBuilder()

    def __len__(self):
        return self._tables.n_patterns

    def len(self):
        return self._tables.n_patterns

    def is_empty(self):
        return self._tables.n_patterns == 0

    def tables(self) -> N.WsPatternTables:
        return self._tables

    def ir(self) -> dict:
        """The PatternIR tables (core/src/pattern/ir.rs:6-34) as numpy arrays."""
        t = self._tables

        def arr(p, n, dt=np.uint32):
            if n == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True)

        return {
            "packed_bytes": bytes(arr(t.packed_bytes, t.packed_len, np.uint8)),
            "offsets": arr(t.offsets, 2 * t.n_literals).reshape(-1, 2),
            "literal_pattern_ids": arr(t.literal_pattern_ids, t.n_literals),
            "hash_window_len": t.hash_window_len,
            "prefix_meta": arr(t.prefix_meta, 4 * t.hash_window_len).reshape(-1, 4),
            "bucket_ranges": arr(t.bucket_ranges, 2 * t.n_buckets).reshape(-1, 2),
            "entries": arr(t.entries, 2 * t.n_literals).reshape(-1, 2),
            "regex_patterns": [(int(t.regex_pattern_ids[i]), t.regex_sources[i].decode())
                               for i in range(t.n_regex)],
            "max_pattern_len": int(max([int(t.offsets[2 * i + 1]) for i in range(t.n_literals)], default=0)),
        }

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().ws_ir_destroy(h)
            except Exception:
                pass
            self._h = None


class CompiledPatternIndex:
    """CompiledPatternIndex (core/src/compiled_index/mod.rs:22-260): the
    reference's on-disk pattern index.  ``load`` parses and validates it
    (magic, version, CRC-32, consistency) into a pattern set whose literal
    tables are the stored ones; ``scan`` runs it on the GPU."""

    MAX_BYTES = 512 * 1024 * 1024  # mod.rs:19

    def __init__(self, serialized: bytes):
        self._bytes = bytes(serialized)
        self._ps = self._parse()
        self._matcher = None

    def _parse(self) -> "PatternSet":
        buf = ctypes.create_string_buffer(self._bytes, len(self._bytes)) if self._bytes else None
        h = ctypes.c_void_p()
        _call(N.lib().ws_index_load, ctypes.cast(buf, ctypes.c_void_p).value if buf is not None else None,
              len(self._bytes), ctypes.byref(h))
        return PatternSet(h, None, 50_000_000)

    @staticmethod
    def build(patterns: "PatternSet") -> bytes:
        """Serialized index image of a pattern set (builder.rs:8-64)."""
        n = ctypes.c_uint64()
        err = N.WsErrorInfo()
        st = N.lib().ws_index_save(patterns._h, None, 0, ctypes.byref(n), ctypes.byref(err))
        if st not in (0, 11):
            _raise(st, err)
        out = ctypes.create_string_buffer(max(n.value, 1))
        _call(N.lib().ws_index_save, patterns._h, out, n.value, ctypes.byref(n))
        return out.raw[: n.value]

    @classmethod
    def load(cls, data: bytes) -> "CompiledPatternIndex":
        return cls(data)

    @classmethod
    def load_from_file(cls, path) -> "CompiledPatternIndex":
        import os
        size = os.path.getsize(path)
        if size > cls.MAX_BYTES:
            raise InputTooLarge(size, cls.MAX_BYTES)
        with open(path, "rb") as f:
            return cls(f.read())

    def save_to_file(self, path) -> None:
        with open(path, "wb") as f:
            f.write(self._bytes)

    def to_bytes(self) -> bytes:
        return self._bytes

    def names(self) -> list:
        return self._ps.names

    def literal_count(self) -> int:
        return int(self._ps.tables().n_literals)

    def to_pattern_set(self) -> "PatternSet":
        """A pattern set equal to the one the index was built from."""
        return self._parse()

    def scan(self, data) -> list[Match]:
        """Scan on the GPU with the index's pattern set (sorted matches)."""
        if self._matcher is None:
            self._matcher = GpuMatcher(self._ps)
        return self._matcher.scan(data)


def _call_noerr(fn, *args):
    st = fn(*args)
    if st != 0:
        raise ValueError(f"status {st}")


# ---------------------------------------------------------------- config
class AutoMatcherConfig:
    """AutoMatcherConfig (core/src/config.rs:39-173) plus the B200 plan knobs."""

    def __init__(self):
        self.c = N.WsConfig()
        N.lib().ws_config_default(ctypes.byref(self.c))
        self._gpu_max_regex_input_size = 16 << 20
        self._max_scan_depth = None

    @staticmethod
    def new():
        return AutoMatcherConfig()

    def gpu_threshold(self, n):
        self.c.gpu_threshold = max(int(n), 1)
        return self

    def gpu_max_input_size(self, n):
        self.c.gpu_max_input_size = max(int(n), 1)
        return self

    def gpu_max_regex_input_size(self, n):
        # Kept for API compatibility: the DFA kernels have no input-size cap.
        self._gpu_max_regex_input_size = int(n)
        return self

    def max_matches(self, n):
        self.c.max_matches = int(n)
        return self

    def chunk_size(self, n):
        self.c.chunk_size = max(int(n), 1)
        if self.c.chunk_overlap >= self.c.chunk_size:
            self.c.chunk_overlap = self.c.chunk_size - 1
        return self

    def chunk_overlap(self, n):
        self.c.chunk_overlap = min(int(n), max(self.c.chunk_size - 1, 0))
        return self

    def max_scan_depth(self, depth):
        self._max_scan_depth = depth
        return self

    # B200 knobs
    def regex_mode(self, mode: int):
        self.c.regex_mode = int(mode)
        return self

    def dfa_max_states(self, n: int):
        self.c.dfa_max_states = int(n)
        return self

    def walk_chunk(self, n: int):
        self.c.walk_chunk = int(n)
        return self

    def proposer(self, kind: int, train_bytes: int | None = None, seed: int | None = None):
        self.c.proposer = int(kind)
        if train_bytes is not None:
            self.c.proposer_train_bytes = int(train_bytes)
        if seed is not None:
            self.c.proposer_seed = int(seed)
        return self

    def batch_mib(self, n: int):
        """Bytes per batch launch sequence, in MiB (0: 1024)."""
        self.c.batch_mib = int(n)
        return self

    def window_mib(self, n: int):
        """New bytes per window of a stream or a 64-bit device scan, in MiB (0: 1024)."""
        self.c.window_mib = int(n)
        return self

    def profile(self, yes: bool = True):
        """Record CUDA events around each kernel phase (GpuMatcher.info())."""
        self.c.flags = (self.c.flags | 1) if yes else (self.c.flags & ~1)
        return self

    def configured_gpu_threshold(self):
        return self.c.gpu_threshold

    def configured_gpu_max_input_size(self):
        return self.c.gpu_max_input_size

    def configured_gpu_max_regex_input_size(self):
        return self._gpu_max_regex_input_size

    def configured_max_matches(self):
        return self.c.max_matches

    def configured_chunk_size(self):
        return self.c.chunk_size

    def configured_chunk_overlap(self):
        return self.c.chunk_overlap

    def configured_max_scan_depth(self):
        return self._max_scan_depth


# --------------------------------------------------------------- matcher
_CTX = {}


def _context(device: int = 0):
    if device not in _CTX:
        h = ctypes.c_void_p()
        _call(N.lib().ws_ctx_create, device, ctypes.byref(h))
        _CTX[device] = h
    return _CTX[device]


def _matches_from(buf, n) -> list[Match]:
    if n == 0:
        return []
    a = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_uint32)), shape=(n * 3,)).reshape(n, 3)
    return [Match(int(p), int(s), int(e)) for p, s, e in a.tolist()]


class GpuMatcher:
    """GPU matcher over the sm_100a kernels (core/src/gpu/mod.rs:77-445)."""

    def __init__(self, patterns: PatternSet, config: AutoMatcherConfig | None = None, device: int = 0):
        self.patterns = patterns
        self.config = config or AutoMatcherConfig()
        ctx = _context(device)
        h = ctypes.c_void_p()
        _call(N.lib().ws_matcher_create, ctx, ctypes.byref(patterns.tables()), ctypes.byref(self.config.c),
              ctypes.byref(h))
        self._h = h
        ir = patterns.ir()
        self._chunk_overlap = max(self.config.c.chunk_overlap, ir["max_pattern_len"])

    @classmethod
    def new(cls, patterns: PatternSet) -> "GpuMatcher":
        return cls(patterns)

    @classmethod
    def with_config(cls, patterns: PatternSet, config: AutoMatcherConfig) -> "GpuMatcher":
        return cls(patterns, config)

    def scan_array(self, data) -> np.ndarray:
        """Scan and return an (n, 3) uint32 array of (pattern_id, start, end)."""
        ptr, n, keep = _buffer(data)
        cap = max(int(self.config.c.max_matches), 1)
        out = np.empty((cap, 3), dtype=np.uint32)
        cnt = ctypes.c_uint64()
        _call(N.lib().ws_scan, self._h, ptr, n, out.ctypes.data_as(ctypes.POINTER(N.WsMatch)), cap, ctypes.byref(cnt))
        del keep
        return out[: cnt.value].copy()

    def scan(self, data) -> list[Match]:
        a = self.scan_array(data)
        return [Match(int(p), int(s), int(e)) for p, s, e in a.tolist()]

    scan_blocking = scan

    def scan_block(self, data) -> list[Match]:
        return self.scan(data)

    def max_block_size(self) -> int:
        return int(self.config.c.chunk_size)

    def chunk_overlap(self) -> int:
        return self._chunk_overlap

    def scan_device(self, d_data: int, length: int, d_out: int, cap: int, d_count: int, stream: int = 0):
        """Device-resident scan (pointers are CUDA device addresses)."""
        _call(N.lib().ws_scan_device, self._h, d_data, length, d_out, cap, d_count, stream)

    def scan_device64(self, d_data: int, length: int, d_out: int, cap: int, d_count: int, stream: int = 0):
        """Device-resident scan of any size; ws_match64 output (unsorted)."""
        _call(N.lib().ws_scan_device64, self._h, d_data, length, d_out, cap, d_count, stream)

    def scan_batch_device(self, d_data: int, length: int, d_item_end: int, d_ids: int, n_items: int, d_out: int,
                          cap: int, d_count: int, stream: int = 0):
        """Device-resident batch scan of items coalesced in d_data (u32 item
        ends, u64 ids); ws_tagged_match output (unsorted)."""
        _call(N.lib().ws_scan_batch_device, self._h, d_data, length, d_item_end, d_ids, n_items, d_out, cap, d_count,
              stream)

    def train_proposer(self, corpus, seed: int = 0x5EED) -> dict:
        """Trains the learned boundary-state proposer of the speculative regex
        walk on `corpus` (same distribution as the inputs to be scanned)."""
        ptr, n, keep = _buffer(corpus)
        _call(N.lib().ws_matcher_train_proposer, self._h, ptr, n, seed)
        del keep
        i = self.info()
        return {"top1": i["proposer_top1"], "top4": i["proposer_top4"]}

    TUNE_GROUPS = 1
    TUNE_CHUNK = 2

    def tune(self, corpus, seed: int = 0x5EED, flags: int = 3) -> dict:
        """Autotunes the regex walk on `corpus` (same distribution as the
        inputs): group DFA size, hot-row placement, proposer and walk chunk,
        each chosen by timing scans on the device.  Matches never change."""
        ptr, n, keep = _buffer(corpus)
        rep = N.WsTuneReport()
        _call(N.lib().ws_matcher_tune, self._h, ptr, n, seed, flags, ctypes.byref(rep))
        del keep
        return {"dfa_max_states": rep.dfa_max_states, "n_groups": rep.n_groups, "walk_chunk": rep.walk_chunk,
                "proposer_used": bool(rep.proposer_used),
                "groups_tried": {int(c): round(m, 4) for c, m in zip(rep.group_candidates, rep.group_ms) if c},
                "chunks_tried": {int(c): [round(x, 4) for x in rep.chunk_ms[k]]
                                 for k, c in enumerate(rep.chunk_candidates) if c},
                "proposer_top1": rep.proposer_top1, "proposer_top4": rep.proposer_top4,
                "tune_seconds": round(rep.tune_seconds, 2)}

    def set_walk(self, walk_chunk: int = 0, proposer: int = PROPOSER_MLP):
        """Pins the speculative walk's chunk (0 keeps it) and its boundary
        guess: the trained proposer (PROPOSER_MLP) or the unanchored start
        (PROPOSER_NONE), overriding the autotuner.  Matches never change."""
        _call(N.lib().ws_matcher_set_walk, self._h, int(walk_chunk), int(proposer))

    def regex_candidates(self, data, mode: int, distinct: bool = False) -> np.ndarray:
        """K candidates (pattern_id, start, end), unsorted: every anchored match
        end, or with ``distinct`` the candidates a scan works from (the same
        distinct (pattern_id, start) pairs, repeats pruned)."""
        ptr, n, keep = _buffer(data)
        mode = int(mode) | (CAND_DISTINCT if distinct else 0)
        cap = max(int(self.config.c.max_matches), 1) * 4
        out = np.empty((cap, 3), dtype=np.uint32)
        cnt = ctypes.c_uint64()
        _call(N.lib().ws_regex_candidates, self._h, ptr, n, mode, out.ctypes.data_as(ctypes.POINTER(N.WsMatch)),
              cap, ctypes.byref(cnt))
        del keep
        return out[: cnt.value].copy()

    def info(self) -> dict:
        i = N.WsMatcherInfo()
        N.lib().ws_matcher_get_info(self._h, ctypes.byref(i))
        d = {f: getattr(i, f) for f, _ in N.WsMatcherInfo._fields_}
        d["last_kernel_ms"] = list(i.last_kernel_ms)
        return d

    def close(self):
        if getattr(self, "_h", None):
            N.lib().ws_matcher_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


WarpStateer = GpuMatcher  # the name used in the reference's README


class GpuScanner:
    """Synchronous shareable scanner (core/src/gpu/scanner.rs:14-120)."""

    def __init__(self, patterns: PatternSet, config: AutoMatcherConfig | None = None):
        self._m = GpuMatcher(patterns, config)

    @classmethod
    def new(cls, patterns: PatternSet):
        return cls(patterns)

    def scan(self, data) -> list[Match]:
        return self._m.scan(data)


class AutoMatcher:
    """Router that always sends input to the GPU (core/src/router.rs:59-305).

    The reference returns NoGpuAdapter for inputs below ``gpu_threshold``; this
    implementation scans every input on the GPU (the threshold is kept as a
    configuration value only)."""

    def __init__(self, patterns: PatternSet, config: AutoMatcherConfig | None = None):
        self.patterns = patterns
        self.config = config or AutoMatcherConfig()
        self._gpu: GpuMatcher | None = None

    @classmethod
    def new(cls, patterns: PatternSet):
        return cls(patterns)

    @classmethod
    def with_config(cls, patterns: PatternSet, config: AutoMatcherConfig):
        return cls(patterns, config)

    new_blocking = new

    def gpu_threshold(self) -> int:
        return int(self.config.c.gpu_threshold)

    def gpu_max_input_size(self) -> int:
        return int(self.config.c.gpu_max_input_size)

    def _backend(self) -> GpuMatcher:
        if self._gpu is None:
            self._gpu = GpuMatcher(self.patterns, self.config)
        return self._gpu

    def has_gpu(self) -> bool:
        try:
            self._backend()
            return True
        except NoGpuAdapter:
            return False

    def scan(self, data) -> list[Match]:
        return self._backend().scan(data)

    scan_blocking = scan
    scan_gpu = scan

    def matcher(self) -> GpuMatcher:
        return self._backend()


# ----------------------------------------------------------------- batch
@dataclass
class ScanItem:
    """batch::ScanItem (core/src/batch.rs:13-18)."""
    id: int
    data: object


@dataclass(frozen=True)
class TaggedMatch:
    """batch::TaggedMatch (core/src/batch.rs:22-27): offsets relative to the item."""
    source_id: int
    matched: Match


@dataclass
class BatchConfig:
    """batch::BatchConfig (core/src/batch.rs:31-48)."""
    max_inputs: int = 4096
    max_bytes: int = 256 * 1024 * 1024
    sort_by_size: bool = True


@dataclass
class CoalesceMap:
    """batch::CoalesceMap (core/src/batch.rs:51-57): ``entries`` holds
    ``(source_id, start_offset_in_buffer, length)``."""
    entries: list
    buffer: bytes


_U32_MAX = 0xFFFFFFFF


def _tagged_key(t: TaggedMatch):
    return (t.source_id, t.matched.start, t.matched.pattern_id, t.matched.end)


def coalesce(items: Sequence[ScanItem]) -> CoalesceMap:
    """batch::coalesce (core/src/batch.rs:65-98): one contiguous buffer and the
    item map; InputTooLarge beyond 32-bit offsets."""
    total = 0
    for it in items:
        n = it.data.nbytes if isinstance(it.data, np.ndarray) else len(it.data)
        if n > _U32_MAX:
            raise InputTooLarge(n, _U32_MAX)
        total += n
    if total > _U32_MAX:
        raise InputTooLarge(total, _U32_MAX)
    parts, entries, off = [], [], 0
    for it in items:
        b = bytes(memoryview(it.data).cast("B")) if not isinstance(it.data, np.ndarray) else it.data.tobytes()
        entries.append((int(it.id), off, len(b)))
        parts.append(b)
        off += len(b)
    return CoalesceMap(entries, b"".join(parts))


def decoalesce(cmap: CoalesceMap, global_matches: Sequence[Match]) -> list[TaggedMatch]:
    """batch::decoalesce (core/src/batch.rs:106-167): attribute position-sorted
    matches of a coalesced buffer to their items, dropping matches that cross
    an item boundary; sorted by (source_id, start, pattern_id, end)."""
    tagged, cursor, entries = [], 0, cmap.entries
    for m in global_matches:
        while cursor < len(entries) and not m.start < entries[cursor][1] + entries[cursor][2]:
            cursor += 1
        if cursor >= len(entries):
            break
        sid, off, ln = entries[cursor]
        if m.start < off or m.end > off + ln:
            continue
        tagged.append(TaggedMatch(sid, Match(m.pattern_id, m.start - off, m.end - off)))
    tagged.sort(key=_tagged_key)
    return tagged


def planned_batches(inputs: Sequence, config: BatchConfig) -> list[list[int]]:
    """The batch planner of core/src/batch.rs:197-236: largest inputs first
    (when ``sort_by_size``), closing a batch at ``max_inputs`` items or
    ``max_bytes`` bytes."""
    if not inputs:
        return []
    max_inputs, max_bytes = max(config.max_inputs, 1), max(config.max_bytes, 1)
    lens = [len(x) if not isinstance(x, np.ndarray) else x.nbytes for x in inputs]
    order = list(range(len(inputs)))
    if config.sort_by_size:
        order.sort(key=lambda i: -lens[i])  # stable: equal sizes keep input order
    batches, cur, cur_bytes = [], [], 0
    for idx in order:
        ln = lens[idx]
        if cur and (len(cur) >= max_inputs or cur_bytes + ln > max_bytes):
            batches.append(cur)
            cur, cur_bytes = [], 0
        cur.append(idx)
        cur_bytes += ln
        if len(cur) >= max_inputs or cur_bytes >= max_bytes:
            batches.append(cur)
            cur, cur_bytes = [], 0
    if cur:
        batches.append(cur)
    return batches


def tagged_to_nested(tagged: Iterable[TaggedMatch], input_count: int) -> list[list[Match]]:
    """core/src/batch.rs:238-250: group tagged matches by input index."""
    grouped: list[list[Match]] = [[] for _ in range(input_count)]
    for t in tagged:
        if 0 <= t.source_id < input_count:
            grouped[t.source_id].append(t.matched)
    return grouped


def _batch_array(matcher: "GpuMatcher", arr, n: int) -> np.ndarray:
    """ws_scan_batch over a prepared WsItem array; (k, 4) uint64 rows
    (source_id, pattern_id, start, end), sorted."""
    cap = max(int(matcher.config.c.max_matches), 1)
    out = np.empty(cap, dtype=np.dtype([("sid", "<u8"), ("pid", "<u4"), ("start", "<u4"), ("end", "<u4"),
                                         ("res", "<u4")]))
    cnt = ctypes.c_uint64()
    _call(N.lib().ws_scan_batch, matcher._h, arr, n, out.ctypes.data_as(ctypes.POINTER(N.WsTaggedMatch)), cap,
          ctypes.byref(cnt))
    o = out[: cnt.value]
    res = np.empty((cnt.value, 4), dtype=np.uint64)
    res[:, 0] = o["sid"]
    res[:, 1] = o["pid"]
    res[:, 2] = o["start"]
    res[:, 3] = o["end"]
    return res


def _batch_raw(matcher: "GpuMatcher", items: Sequence[ScanItem]) -> list[TaggedMatch]:
    n = len(items)
    if n == 0:
        return []
    arr = (N.WsItem * n)()
    keep = []
    for i, it in enumerate(items):
        ptr, ln, k = _buffer(it.data)
        keep.append(k)
        arr[i].id = int(it.id)
        arr[i].data = ptr
        arr[i].len = ln
    rows = _batch_array(matcher, arr, n)
    del keep
    return [TaggedMatch(int(a), Match(int(b), int(c), int(d))) for a, b, c, d in rows.tolist()]


def scan_batch_packed(matcher: "GpuMatcher | AutoMatcher", arena, lengths, ids=None) -> np.ndarray:
    """Batch scan of items stored back to back in one host buffer (``arena``;
    a pinned tensor avoids the staging copy).  ``lengths[i]`` bytes belong to
    item ``ids[i]`` (default ``i``).  Returns an (n, 4) uint64 array of
    (source_id, pattern_id, start, end), item-relative offsets, sorted by
    (source_id, start, pattern_id, end) -- the result of ``scan_batch_gpu``."""
    m = matcher.matcher() if isinstance(matcher, AutoMatcher) else matcher
    ptr, total, keep = _buffer(arena)
    lengths = np.asarray(lengths, dtype=np.uint64)
    n = int(lengths.size)
    if int(lengths.sum()) > total:
        raise ValueError("item lengths exceed the arena")
    if n == 0:
        return np.empty((0, 4), dtype=np.uint64)
    starts = np.zeros(n, dtype=np.uint64)
    np.cumsum(lengths[:-1], out=starts[1:])
    rec = np.empty(n, dtype=np.dtype([("id", "<u8"), ("data", "<u8"), ("len", "<u8")]))
    rec["id"] = np.arange(n, dtype=np.uint64) if ids is None else np.asarray(ids, dtype=np.uint64)
    rec["data"] = np.uint64(ptr) + starts
    rec["len"] = lengths
    arr = ctypes.cast(rec.ctypes.data, ctypes.POINTER(N.WsItem))
    res = _batch_array(m, arr, n)
    del keep
    return res


def scan_batch(matcher: "GpuMatcher", inputs: Sequence, config: BatchConfig | None = None) -> list[list[Match]]:
    """batch::scan_batch (core/src/batch.rs:312-319): per-input match lists.
    Inputs are grouped as the reference's planner groups them; each group is
    one device launch sequence scanning every item on its own."""
    config = config or BatchConfig()
    grouped: list[list[Match]] = [[] for _ in inputs]
    for batch in planned_batches(inputs, config):
        for t in _batch_raw(matcher, [ScanItem(i, inputs[i]) for i in batch]):
            grouped[t.source_id].append(t.matched)
    return grouped


def scan_batch_auto(matcher: "AutoMatcher", inputs: Sequence, config: BatchConfig | None = None) -> list[list[Match]]:
    """batch::scan_batch_auto (core/src/batch.rs:321-328), always on the GPU."""
    return scan_batch(matcher.matcher(), inputs, config)


def scan_batch_gpu(matcher: "AutoMatcher | GpuMatcher", items: Iterable[ScanItem]) -> list[TaggedMatch]:
    """batch::scan_batch_gpu (core/src/batch.rs:336-363): tagged matches sorted
    by (source_id, start, pattern_id, end); no match crosses an item.  All
    items go to the device planner (1 GiB per launch sequence by default)."""
    m = matcher.matcher() if isinstance(matcher, AutoMatcher) else matcher
    return _batch_raw(m, list(items))


def _pattern_set_scan_batch(self, items: Iterable[ScanItem], matcher: "GpuMatcher | None" = None):
    """``patterns.scan_batch(items)`` as README.md shows it: routes to the GPU."""
    if matcher is None:
        matcher = self.__dict__.get("_batch_matcher")
        if matcher is None:
            matcher = GpuMatcher(self)
            self.__dict__["_batch_matcher"] = matcher
    return scan_batch_gpu(matcher, items)


PatternSet.scan_batch = _pattern_set_scan_batch


# ---------------------------------------------------------------- stream
_WS_ERR_OVERFLOW = 11


class StreamPipeline:
    """StreamPipeline (core/src/pipeline.rs:15-153) with exact state carry.

    ``scan(data)`` pushes the data through the device stream API
    (``ws_stream_*``), which decides every match exactly once; the result
    equals a whole-input scan, with no overlap heuristic.  ``overlap_window``
    is accepted for API compatibility and not needed."""

    def __init__(self, backend: "GpuMatcher | AutoMatcher", overlap_window: int = 0):
        self.backend = backend.matcher() if isinstance(backend, AutoMatcher) else backend
        self.overlap_window = overlap_window

    @staticmethod
    def new(backend, overlap_window: int = 0) -> "StreamPipeline":
        return StreamPipeline(backend, overlap_window)

    def scan_array(self, data, block: int | None = None) -> np.ndarray:
        """(n, 3) uint64 array of (pattern_id, start, end) sorted by (start, pattern_id, end)."""
        ptr, n, keep = _buffer(data)
        parts = []
        with Stream(self.backend) as s:
            step = n if not block else max(int(block), 1)
            for off in range(0, n, max(step, 1)):
                parts.append(s.feed_ptr_array(ptr + off, min(step, n - off)))
            parts.append(s.end_array())
        del keep
        a = np.concatenate(parts) if parts else np.empty((0, 3), dtype=np.uint64)
        order = np.lexsort((a[:, 2], a[:, 0], a[:, 1])) if len(a) else np.empty(0, dtype=np.int64)
        return a[order]

    def scan(self, data) -> list[Match]:
        return [Match(int(p), int(s), int(e)) for p, s, e in self.scan_array(data).tolist()]


class ZeroCopyScan:
    """Two-phase zero-copy scan session (core/src/pipeline.rs:48-83): fill
    ``mapped_mut()`` (pinned, device-mapped memory the library owns), then
    ``finish()`` scans it in place."""

    def __init__(self, matcher: "GpuMatcher", input_len: int):
        self._m = matcher
        self._len = int(input_len)
        h, p = ctypes.c_void_p(), ctypes.c_void_p()
        _call(N.lib().ws_zero_copy_begin, matcher._h, self._len, ctypes.byref(h), ctypes.byref(p))
        self._h = h
        self._view = (np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), shape=(self._len,))
                      if self._len else np.empty(0, dtype=np.uint8))

    def mapped_mut(self) -> np.ndarray:
        """The writable input region (a uint8 view; valid until finish())."""
        if self._h is None:
            raise ValueError("session already finished")
        return self._view

    def finish_array(self) -> np.ndarray:
        if self._h is None:
            raise ValueError("session already finished")
        cap = max(int(self._m.config.c.max_matches), 1)
        out = np.empty((cap, 3), dtype=np.uint32)
        cnt = ctypes.c_uint64()
        h, self._h = self._h, None
        self._view = None
        _call(N.lib().ws_zero_copy_finish, h, out.ctypes.data_as(ctypes.POINTER(N.WsMatch)), cap, ctypes.byref(cnt))
        return out[: cnt.value].copy()

    def finish(self) -> list[Match]:
        return [Match(int(p), int(s), int(e)) for p, s, e in self.finish_array().tolist()]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().ws_zero_copy_abort(h)
            except Exception:
                pass


def _stream_pipeline_scan_zero_copy(self, input_len: int) -> ZeroCopyScan:
    """StreamPipeline::scan_zero_copy (core/src/pipeline.rs:31-46)."""
    return ZeroCopyScan(self.backend, input_len)


StreamPipeline.scan_zero_copy = _stream_pipeline_scan_zero_copy


class HotSwapPatternSet:
    """HotSwapPatternSet (core/src/pattern/mod.rs:17-70) on the GPU: the
    active pattern set's device tables are replaced atomically by ``swap``
    while other threads scan; each scan uses the set active when it began."""

    def __init__(self, pattern_set: PatternSet, config: AutoMatcherConfig | None = None, device: int = 0):
        self.config = config or AutoMatcherConfig()
        self._device = device
        m = GpuMatcher(pattern_set, self.config, device)
        h = ctypes.c_void_p()
        _call(N.lib().ws_hotswap_create, m._h, ctypes.byref(h))
        m._h = None  # the handle owns the matcher now
        self._h = h
        self._active = pattern_set

    @classmethod
    def new(cls, pattern_set: PatternSet) -> "HotSwapPatternSet":
        return cls(pattern_set)

    def swap(self, next_set: PatternSet) -> bool:
        """Makes ``next_set`` active; False when it already is."""
        if next_set is self._active:
            return False
        m = GpuMatcher(next_set, self.config, self._device)
        r = N.lib().ws_hotswap_swap(self._h, m._h)
        m._h = None
        if r < 0:
            raise ValueError("hot swap failed")
        self._active = next_set
        return r == 1

    def scan_array(self, data) -> np.ndarray:
        ptr, n, keep = _buffer(data)
        cap = max(int(self.config.c.max_matches), 1)
        out = np.empty((cap, 3), dtype=np.uint32)
        cnt = ctypes.c_uint64()
        _call(N.lib().ws_hotswap_scan, self._h, ptr, n, out.ctypes.data_as(ctypes.POINTER(N.WsMatch)), cap,
              ctypes.byref(cnt))
        del keep
        return out[: cnt.value].copy()

    def scan(self, data) -> list[Match]:
        return [Match(int(p), int(s), int(e)) for p, s, e in self.scan_array(data).tolist()]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().ws_hotswap_destroy(h)
            except Exception:
                pass
            self._h = None


class Stream:
    """Incremental scan with 64-bit offsets (ws_stream_*): every match is
    returned by exactly one ``feed`` or by ``end``."""

    def __init__(self, matcher: "GpuMatcher | AutoMatcher"):
        matcher = matcher.matcher() if isinstance(matcher, AutoMatcher) else matcher
        self.m = matcher
        h = ctypes.c_void_p()
        _call(N.lib().ws_stream_begin, matcher._h, ctypes.byref(h))
        self._h = h
        self._cap = max(int(matcher.config.c.max_matches), 1)
        self._out = np.empty(self._cap, dtype=np.dtype([("pid", "<u4"), ("res", "<u4"), ("start", "<u8"),
                                                        ("end", "<u8")]))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _rows(self, n: int) -> np.ndarray:
        o = self._out[:n]
        a = np.empty((n, 3), dtype=np.uint64)
        a[:, 0], a[:, 1], a[:, 2] = o["pid"], o["start"], o["end"]
        return a

    def _collect(self, call) -> np.ndarray:
        """Runs ``call(out, cap, n_out, err)``; while it reports overflow with
        some matches delivered, drains the rest with more calls."""
        parts = []
        while True:
            cnt = ctypes.c_uint64()
            err = N.WsErrorInfo()
            st = call(self._out.ctypes.data_as(ctypes.POINTER(N.WsMatch64)), self._cap, ctypes.byref(cnt),
                      ctypes.byref(err))
            parts.append(self._rows(cnt.value))
            if st == _WS_ERR_OVERFLOW and cnt.value > 0:
                continue
            if st != 0:
                _raise(st, err)
            return np.concatenate(parts)

    def feed_ptr_array(self, ptr: int, n: int) -> np.ndarray:
        lib, h = N.lib(), self._h
        first = [True]

        def call(out, cap, cnt, err):
            if first[0]:
                first[0] = False
                return lib.ws_stream_feed(h, ptr, n, out, cap, cnt, err)
            return lib.ws_stream_feed(h, None, 0, out, cap, cnt, err)
        return self._collect(call)

    def end_array(self) -> np.ndarray:
        lib, h = N.lib(), self._h
        return self._collect(lambda out, cap, cnt, err: lib.ws_stream_end(h, out, cap, cnt, err))

    @staticmethod
    def _to_matches(a: np.ndarray) -> list[Match]:
        return [Match(int(p), int(s), int(e)) for p, s, e in a.tolist()]

    def feed_ptr(self, ptr: int, n: int) -> list[Match]:
        return self._to_matches(self.feed_ptr_array(ptr, n))

    def feed(self, data) -> list[Match]:
        ptr, n, keep = _buffer(data)
        r = self.feed_ptr(ptr, n)
        del keep
        return r

    def end(self) -> list[Match]:
        return self._to_matches(self.end_array())

    def close(self):
        if getattr(self, "_h", None):
            N.lib().ws_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
