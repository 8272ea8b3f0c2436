"""Multi-GPU host logic on CPU: shard layout, item partition, and the chain
cursor exchange over gloo with world_size 2 (oracle-backed shard scans).

The shard scan stand-in follows ws_scan_shard's contract exactly: literal
occurrences starting in the shard's own range, and each regex's find_iter
chain resumed at its incoming cursor, deciding matches that start before the
shard's own end.  The union over ranks must equal one oracle scan of the whole
input, including regex chains that run across a shard boundary.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from warpstate_b200 import multi_gpu as mg


def test_build_scan_shards_layout():
    # core/src/multi_gpu.rs:170-200: equal ranges, halo after all but the last
    s = mg.build_scan_shards(100, 3, 7)
    assert [(x.start, x.nominal_end, x.scan_end) for x in s] == [(0, 33, 40), (33, 66, 73), (66, 100, 100)]
    assert mg.build_scan_shards(0, 4, 7) == []
    assert len(mg.build_scan_shards(2, 8, 7)) == 2  # never more shards than bytes
    assert mg.shard_halo(32, 40, 10**9) == 39
    assert mg.shard_halo(32, -1, 12345) == 12345


def test_partition_items_longest_first():
    lens = [5, 100, 7, 60, 50, 1, 40]
    parts = mg.partition_items(lens, 2)
    assert sorted(i for p in parts for i in p) == list(range(len(lens)))
    loads = [sum(lens[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(lens)
    # 100 -> r0, 60 -> r1, 50 -> r1, 40 -> r0, 7, 5, 1 -> r1 (loads 140 / 123)
    assert parts == [[1, 6], [0, 2, 3, 4, 5]]


PATTERNS = [(1, b"(?:ab|ba){1,4}"), (1, b"a[ab]{0,6}b"), (1, b"x[yz]{1,3}"), (0, b"ab"), (0, b"aab"),
            (1, b"zz+")]


def _data(n=200_000, seed=3):
    r = np.random.default_rng(seed)
    d = r.choice(np.frombuffer(b"abxyz", np.uint8), size=n).astype(np.uint8)
    # chains that cross the 2-way and 3-way boundaries
    for b in (n // 2, n // 3, 2 * n // 3):
        d[b - 3:b + 5] = np.frombuffer(b"abababab", np.uint8)
    return d


def oracle_shard_scan(data, patterns, shard, cursor_in):
    """ws_scan_shard's contract on the CPU oracle."""
    lits, lit_ids, rxs, rx_ids = oracle.split_patterns(patterns)
    seg = data[shard.start:shard.scan_end]
    out = []
    for p, s, e in oracle.literal_scan(lits, lit_ids, seg).tolist():
        if shard.start + s < shard.nominal_end:
            out.append((p, shard.start + s, shard.start + e))
    cur_out = np.zeros(len(rxs), dtype=np.uint64)
    for k, (rx, pid) in enumerate(zip(rxs, rx_ids)):
        c = int(cursor_in[k])
        last = c
        if c < shard.nominal_end:
            for s, e in rx.find_iter(data[c:shard.scan_end]):
                if c + s >= shard.nominal_end:
                    break
                out.append((pid, c + s, c + e))
                last = c + e
        cur_out[k] = max(last, shard.nominal_end)
    return np.array(out, dtype=np.uint64).reshape(-1, 3), cur_out


def _halo(patterns, n):
    lits, _, rxs, _ = oracle.split_patterns(patterns)
    lit_max = max((len(x) for x in lits), default=0)
    rx_max = -1 if any(r.maxlen < 0 for r in rxs) else max((r.maxlen for r in rxs), default=0)
    return mg.shard_halo(lit_max, rx_max, n)


def test_local_protocol_equals_whole_scan():
    data = _data()
    whole = oracle.scan_patterns(PATTERNS, data).astype(np.uint64)
    _, _, rxs, _ = oracle.split_patterns(PATTERNS)
    for world in (2, 3, 5):
        shards = mg.build_scan_shards(len(data), world, _halo(PATTERNS, len(data)))
        res = mg.run_local_protocol(world, len(rxs), shards,
                                    lambda r, c: oracle_shard_scan(data, PATTERNS, shards[r], c))
        got = np.concatenate(res)
        got = got[np.lexsort((got[:, 2], got[:, 0], got[:, 1]))]
        assert np.array_equal(got, whole), world


def test_without_exchange_chains_differ():
    # the exchange matters: starting every shard's chains afresh (the
    # reference's overlapped rescan) gives a different regex result here
    data = _data()
    whole = oracle.scan_patterns(PATTERNS, data).astype(np.uint64)
    _, _, rxs, _ = oracle.split_patterns(PATTERNS)
    shards = mg.build_scan_shards(len(data), 2, _halo(PATTERNS, len(data)))
    naive = [oracle_shard_scan(data, PATTERNS, s, np.full(len(rxs), s.start, np.uint64))[0] for s in shards]
    got = np.concatenate(naive)
    got = got[np.lexsort((got[:, 2], got[:, 0], got[:, 1]))]
    assert not np.array_equal(got, whole)


def _gloo_rank(rank, world, port, out_dir):
    import torch.distributed as dist
    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        data = _data()
        _, _, rxs, _ = oracle.split_patterns(PATTERNS)
        shards = mg.build_scan_shards(len(data), world, _halo(PATTERNS, len(data)))
        shard = shards[rank] if rank < len(shards) else None

        def exchange(vec):
            t = torch.from_numpy(vec.astype(np.int64))
            outs = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(outs, t)
            return [o.numpy().view(np.uint64) for o in outs]

        mine = mg.resolve_chains(rank, world, shard, len(rxs),
                                 lambda c: oracle_shard_scan(data, PATTERNS, shard, c), exchange)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), mine)
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_exact_chains():
    import torch.multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_rank, args=(2, port, d), nprocs=2, join=True, start_method="spawn")
        got = np.concatenate([np.load(os.path.join(d, f"rank{r}.npy")) for r in range(2)])
    got = got[np.lexsort((got[:, 2], got[:, 0], got[:, 1]))]
    whole = oracle.scan_patterns(PATTERNS, _data()).astype(np.uint64)
    assert np.array_equal(got, whole)
