"""Multi-GPU scans: one input split across GPUs, and batch items spread over GPUs.

Replaces MultiGpuMatcher (core/src/multi_gpu.rs), which scans the shards one
after another and merges them; its regex results near shard boundaries are
those of an overlapped rescan (the shard's own find_iter chain starts afresh at
the shard start).  Here each process drives one GPU (torch.distributed), all
shards scan at once, and regex chains are exact across shards:

* ``build_scan_shards`` splits the input into equal byte ranges with a halo
  after each range (``multi_gpu.rs:170-200``); the halo is the longest reach
  of a match starting inside the range (``shard_halo``).
* Each rank scans its shard with ``ws_scan_shard``: literal matches starting in
  its own range, and every regex's find_iter chain resumed from a cursor.
* ``resolve_chains`` is the one exchange step: every rank all-gathers the
  per-regex cursors its chains leave at its range end (8 bytes per regex); a
  rank whose incoming cursors differ from the ones it assumed (a match of the
  previous shard runs into its range) rescans with the true ones.  Chains
  resynchronise within a shard, so one extra round is the rule; ``world``
  rounds bound it.
* ``partition_items`` spreads batch items over ranks by bytes, largest first
  onto the least loaded rank; items are independent, so a batch needs no
  exchange at all.

The protocol functions take the per-shard scan and the exchange as callables,
so the same code runs over NCCL, over gloo on CPU (tests use an oracle-backed
shard scan), or with every shard on one GPU (``sharded_scan_local``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from . import _native as N


@dataclass(frozen=True)
class ScanShard:
    """A shard of ``build_scan_shards``: own range [start, nominal_end),
    bytes scanned [start, scan_end)."""
    device_index: int
    start: int
    nominal_end: int
    scan_end: int


def shard_halo(max_literal_len: int, max_regex_len: int, input_len: int) -> int:
    """Bytes after a shard's own range that a match starting inside it can
    reach: the longest literal or regex match minus one; the whole remaining
    input when some regex has unbounded matches."""
    if max_regex_len < 0:
        return input_len
    return max(int(max_literal_len), int(max_regex_len), 1) - 1


def build_scan_shards(input_len: int, device_count: int, halo: int) -> list[ScanShard]:
    """Equal byte ranges, each scanned with ``halo`` extra bytes (none after
    the last), as build_scan_shards (core/src/multi_gpu.rs:170-200)."""
    if input_len <= 0 or device_count <= 0:
        return []
    active = min(device_count, input_len)
    shards = []
    for d in range(active):
        start = input_len * d // active
        nominal_end = input_len * (d + 1) // active
        if nominal_end <= start:
            continue
        scan_end = nominal_end if d + 1 == active else min(nominal_end + halo, input_len)
        shards.append(ScanShard(d, start, nominal_end, scan_end))
    return shards


def partition_items(lengths: Sequence[int], world: int) -> list[list[int]]:
    """Item indices per rank: largest item first onto the least loaded rank
    (ties to the lower rank), each rank's list in input order."""
    loads = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(lengths)), key=lambda k: (-int(lengths[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += int(lengths[i])
    for p in parts:
        p.sort()
    return parts


ScanFn = Callable[[np.ndarray], "tuple[np.ndarray, np.ndarray]"]
ExchangeFn = Callable[[np.ndarray], "list[np.ndarray]"]


def resolve_chains(rank: int, world: int, shard: ScanShard | None, n_regex: int, scan: ScanFn,
                   exchange: ExchangeFn) -> np.ndarray:
    """Runs this rank's shard scan until its incoming regex cursors agree with
    the cursors the previous rank's chains leave behind.

    ``scan(cursor_in)`` scans the shard with the given per-regex cursors and
    returns ``(matches, cursor_out)``; ``exchange(vec)`` all-gathers one
    uint64 vector per rank.  Every rank makes the same sequence of exchange
    calls.  Returns this rank's matches as an (n, 3) uint64 array
    (pattern_id, start, end)."""
    base = shard.start if shard is not None else 0
    cur_in = np.full(n_regex, base, dtype=np.uint64)
    if shard is not None:
        matches, cur_out = scan(cur_in)
    else:
        matches, cur_out = np.zeros((0, 3), dtype=np.uint64), np.zeros(n_regex, dtype=np.uint64)
    for _ in range(world):
        outs = exchange(np.concatenate([cur_out, np.array([1 if shard is not None else 0], dtype=np.uint64)]))
        redo = False
        if shard is not None and rank > 0 and n_regex:
            prev = next((o for o in reversed(outs[:rank]) if o[-1] == 1), None)
            incoming = prev[:-1] if prev is not None else np.zeros(n_regex, dtype=np.uint64)
            want = np.maximum(incoming, np.uint64(base))
            if not np.array_equal(want, cur_in):
                cur_in = want
                redo = True
        flags = exchange(np.array([1 if redo else 0], dtype=np.uint64))
        if redo:
            matches, cur_out = scan(cur_in)
        if not any(int(f[0]) for f in flags):
            break
    return matches


def shard_lead(shard: ScanShard, context: bool) -> int:
    """Bytes before a shard's own range that its buffer holds: one when the
    pattern set has look-behind assertions (^ \\b \\B \\A read the byte before a
    start) and the shard is not the first, else none."""
    return 1 if context and shard.start > 0 else 0


class ShardScanner:
    """``ws_scan_shard`` on this process's GPU for one matcher."""

    def __init__(self, matcher, cap: int | None = None):
        import torch
        self.m = matcher
        self.torch = torch
        info = matcher.info()
        self.context = bool(info["regex_context"])
        self.n_regex = int(info["n_regex"])
        self.max_literal_len = int(info["max_literal_len"])
        self.max_regex_len = int(info["max_regex_len"])
        self.cap = int(cap or matcher.config.c.max_matches)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        self.d_out = torch.empty(self.cap * 3, dtype=torch.int64, device=dev)
        self.d_cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        self.d_cursor = torch.zeros(max(self.n_regex, 1), dtype=torch.int64, device=dev)

    def halo(self, input_len: int) -> int:
        return shard_halo(self.max_literal_len, self.max_regex_len, input_len)

    def lead(self, shard: ScanShard) -> int:
        return shard_lead(shard, self.context)

    def buffer(self, host: np.ndarray, shard: ScanShard):
        """The device copy of a shard's bytes, its lead byte included."""
        a = shard.start - self.lead(shard)
        return self.torch.from_numpy(np.ascontiguousarray(host[a:shard.scan_end])).to(self.dev)

    def scan(self, d_buf, shard: ScanShard, cursor_in: np.ndarray):
        """d_buf: device tensor holding bytes [shard.start - lead, shard.scan_end)."""
        torch = self.torch
        from . import _call
        if self.n_regex:
            self.d_cursor[: self.n_regex].copy_(torch.from_numpy(cursor_in.astype(np.int64)))
        s = torch.cuda.current_stream()
        base = shard.start - self.lead(shard)
        _call(N.lib().ws_scan_shard, self.m._h, d_buf.data_ptr(), shard.scan_end - base, base,
              shard.nominal_end, self.d_cursor.data_ptr(), self.d_out.data_ptr(), self.cap, self.d_cnt.data_ptr(),
              s.cuda_stream)
        n = int(self.d_cnt.item())
        if n > self.cap:
            from . import MatchBufferOverflow
            raise MatchBufferOverflow(n, self.cap)
        a = self.d_out[: 3 * n].view(n, 3).cpu().numpy().view(np.uint64)
        out = np.stack([a[:, 0] & np.uint64(0xFFFFFFFF), a[:, 1], a[:, 2]], axis=1)
        if base < shard.start:  # literal matches at the lead byte belong to the previous shard
            out = out[out[:, 1] >= np.uint64(shard.start)]
        cur = self.d_cursor[: self.n_regex].cpu().numpy().view(np.uint64).copy()
        return out, cur


def _sort(a: np.ndarray) -> np.ndarray:
    if len(a) == 0:
        return a.reshape(0, 3)
    return a[np.lexsort((a[:, 2], a[:, 0], a[:, 1]))]


def sharded_scan(matcher, data, group=None, gather: bool = True) -> np.ndarray:
    """Scans ``data`` (host bytes, the same on every rank) split across the
    ranks of ``group`` (torch.distributed, one GPU per rank).  Returns the
    (n, 3) uint64 matches (pattern_id, start, end) of the whole input on every
    rank when ``gather``, else this rank's, sorted by (start, pattern_id, end);
    equal to one scan of the whole input."""
    import torch
    import torch.distributed as dist
    from . import _buffer
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    ptr, n, keep = _buffer(data)
    host = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)), shape=(n,)) if n else \
        np.zeros(0, np.uint8)
    sc = ShardScanner(matcher)
    shards = build_scan_shards(n, world, sc.halo(n))
    shard = shards[rank] if rank < len(shards) else None
    d_buf = None
    if shard is not None:
        d_buf = sc.buffer(host, shard)
    backend = dist.get_backend(group)
    tdev = sc.dev if backend == "nccl" else torch.device("cpu")

    def exchange(vec: np.ndarray) -> list[np.ndarray]:
        t = torch.from_numpy(vec.astype(np.int64)).to(tdev)
        outs = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(outs, t, group=group)
        return [o.cpu().numpy().view(np.uint64) for o in outs]

    mine = resolve_chains(rank, world, shard, sc.n_regex, lambda c: sc.scan(d_buf, shard, c), exchange)
    del keep
    if not gather:
        return _sort(mine)
    parts = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    return _sort(np.concatenate(parts)) if parts else mine


def sharded_scan_local(matcher, data, n_shards: int) -> np.ndarray:
    """The protocol of ``sharded_scan`` with every shard on this process's
    GPU, one after another (for checking shard scans against a whole scan)."""
    import torch
    from . import _buffer
    ptr, n, keep = _buffer(data)
    host = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)), shape=(n,)) if n else \
        np.zeros(0, np.uint8)
    sc = ShardScanner(matcher)
    shards = build_scan_shards(n, n_shards, sc.halo(n))
    bufs = [sc.buffer(host, s) for s in shards]
    results = run_local_protocol(len(shards), sc.n_regex, shards,
                                 lambda r, c: sc.scan(bufs[r], shards[r], c))
    del keep
    return _sort(np.concatenate(results)) if results else np.zeros((0, 3), np.uint64)


def run_local_protocol(world: int, n_regex: int, shards: list[ScanShard],
                       scan: Callable[[int, np.ndarray], "tuple[np.ndarray, np.ndarray]"]) -> list[np.ndarray]:
    """Runs ``resolve_chains`` for ``world`` simulated ranks in one process
    (round-robin over ranks, the exchange served from shared lists)."""
    # rank state machines: the same steps as resolve_chains, interleaved
    base = [s.start for s in shards]
    cur_in = [np.full(n_regex, b, dtype=np.uint64) for b in base]
    res = [scan(r, cur_in[r]) for r in range(world)]
    for _ in range(world):
        outs = [res[r][1] for r in range(world)]
        redo = [False] * world
        for r in range(1, world):
            if not n_regex:
                break
            want = np.maximum(outs[r - 1], np.uint64(base[r]))
            if not np.array_equal(want, cur_in[r]):
                cur_in[r] = want
                redo[r] = True
        for r in range(world):
            if redo[r]:
                res[r] = scan(r, cur_in[r])
        if not any(redo):
            break
    return [m for m, _ in res]


class MultiGpuMatcher:
    """MultiGpuMatcher (core/src/multi_gpu.rs:33-160) in one process: one
    matcher per device, the shards of an input scanned at the same time (one
    host thread per shard, each on its device's own stream), then the cursor
    exchange of ``resolve_chains`` with the rescans of a round run at once
    too.  The reference awaits its shards one after another
    (multi_gpu.rs:142-156) and leaves regex chains near shard boundaries to an
    overlapped rescan; here the result equals one scan of the whole input.
    ``devices`` may repeat an index (several shards on one GPU)."""

    def __init__(self, patterns, devices: Sequence[int] | None = None, config=None):
        import torch
        from . import GpuMatcher
        if devices is None:
            devices = list(range(torch.cuda.device_count()))
        if not devices:
            from . import NoGpuAdapter
            raise NoGpuAdapter("no CUDA device")
        self.devices = list(devices)
        self.matchers = {}
        for d in sorted(set(self.devices)):
            with torch.cuda.device(d):
                self.matchers[d] = GpuMatcher(patterns, config, device=d)
        self._scanners = {}

    def device_count(self) -> int:
        return len(self.devices)

    def _scanner(self, k: int) -> ShardScanner:
        import torch
        if k not in self._scanners:
            d = self.devices[k]
            with torch.cuda.device(d):
                self._scanners[k] = ShardScanner(self.matchers[d])
        return self._scanners[k]

    def scan_array(self, data) -> np.ndarray:
        """(n, 3) uint64 (pattern_id, start, end), sorted by (start, pattern_id, end)."""
        import torch
        from concurrent.futures import ThreadPoolExecutor
        from . import _buffer
        ptr, n, keep = _buffer(data)
        host = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)), shape=(n,)) if n else \
            np.zeros(0, np.uint8)
        world = len(self.devices)
        scanners = [self._scanner(k) for k in range(world)]
        shards = build_scan_shards(n, world, scanners[0].halo(n))
        bufs = {}

        def upload(r):
            with torch.cuda.device(self.devices[r]):
                bufs[r] = scanners[r].buffer(host, shards[r])

        def scan(r, cursor):
            with torch.cuda.device(self.devices[r]):
                return scanners[r].scan(bufs[r], shards[r], cursor)

        with ThreadPoolExecutor(max_workers=max(len(shards), 1)) as ex:
            list(ex.map(upload, range(len(shards))))
            results = run_parallel_protocol(len(shards), scanners[0].n_regex if shards else 0, shards, scan, ex)
        del keep
        return _sort(np.concatenate(results)) if results else np.zeros((0, 3), np.uint64)

    def scan(self, data):
        from . import Match
        return [Match(int(p), int(s), int(e)) for p, s, e in self.scan_array(data).tolist()]


def run_parallel_protocol(world: int, n_regex: int, shards: list[ScanShard],
                          scan: Callable[[int, np.ndarray], "tuple[np.ndarray, np.ndarray]"], executor) -> list[np.ndarray]:
    """``run_local_protocol`` with the scans of each round submitted to
    ``executor`` together (they touch disjoint shards and devices' streams)."""
    base = [s.start for s in shards]
    cur_in = [np.full(n_regex, b, dtype=np.uint64) for b in base]
    res = list(executor.map(lambda r: scan(r, cur_in[r]), range(world)))
    for _ in range(world):
        outs = [res[r][1] for r in range(world)]
        redo = []
        for r in range(1, world):
            if not n_regex:
                break
            want = np.maximum(outs[r - 1], np.uint64(base[r]))
            if not np.array_equal(want, cur_in[r]):
                cur_in[r] = want
                redo.append(r)
        if not redo:
            break
        for r, out in zip(redo, executor.map(lambda r: scan(r, cur_in[r]), redo)):
            res[r] = out
    return [m for m, _ in res]
