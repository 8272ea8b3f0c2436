"""Seeded synthetic workloads for the five scan configurations.

Each configuration is generated from fixed seeds with xoshiro256** streams
seeded through SplitMix64: input bytes by ``libworkloads.so`` (C++, threaded,
bit-identical for any thread count), pattern sets here.  The configurations
follow the benchmark definitions of the scan path:

1. ``literals_small``  100 literals, lowercase, lengths 4-16; 16 MiB iid
   lowercase input with one planted occurrence per 64 KiB.
2. ``literals_large``  10,000 literals, lengths 8-32, printable ASCII with
   Zipf(s=1.1) character frequencies over a seeded permutation; 1 GiB order-1
   Markov input over printable ASCII; one plant per 16 KiB.
3. ``regex``  500 regexes, each ``(?:A1|..|Ak)[C]{1,8}(?:B1|..|Bj)`` with 2-4
   literals per alternation (lengths 4-12) and a narrow joining class; 1 GiB
   Markov input; one planted match per 16 KiB.
4. ``batch``  200,000 items with lognormal sizes (median 4 KiB, sigma 1.5,
   clipped to 64 B - 1 MiB) of Markov bytes; 1,500 literals (6-24) plus the
   500 regexes of configuration 3.
5. ``dna``  4 GiB iid ACGT with N runs (~1% of bytes); 50,000 k-mers (20-32)
   and 200 IUPAC-degenerate regexes (20-40); one plant per MiB.

Every size can be scaled down for parity tests; the structure stays the same.
"""
from __future__ import annotations

import ctypes
import math
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
_LIB = None

MiB = 1 << 20
GiB = 1 << 30


def _lib():
    global _LIB
    if _LIB is None:
        so = _DIR / "libworkloads.so"
        if not so.exists():
            subprocess.run(["make", "-s", "-C", str(_DIR)], check=True)
        lib = ctypes.CDLL(str(so))
        u8p = ctypes.POINTER(ctypes.c_uint8)
        lib.wl_fill_uniform.argtypes = [u8p, ctypes.c_uint64, u8p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int]
        lib.wl_fill_markov.argtypes = [u8p, ctypes.c_uint64, u8p, ctypes.c_uint32, ctypes.c_uint64,
                                       ctypes.c_uint64, ctypes.c_int]
        lib.wl_fill_acgt.argtypes = [u8p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double,
                                     ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
        lib.wl_gen_literals.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u8p,
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_uint32, ctypes.c_uint64,
                                        u8p, ctypes.POINTER(ctypes.c_uint32)]
        _LIB = lib
    return _LIB


def _u8p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


class Rng:
    """xoshiro256** seeded by SplitMix64 (pattern-structure decisions)."""

    M = (1 << 64) - 1

    def __init__(self, seed: int):
        x = seed & self.M
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & self.M
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
            s.append(z ^ (z >> 31))
        self.s = s

    def next(self) -> int:
        s = self.s
        M = self.M
        r = (((((s[1] * 5) & M) << 7 | ((s[1] * 5) & M) >> 57) & M) * 9) & M
        t = (s[1] << 17) & M
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = ((s[3] << 45) | (s[3] >> 19)) & M
        return r

    def below(self, n: int) -> int:
        return ((self.next() >> 32) * n) >> 32

    def uniform(self, lo: int, hi: int) -> int:
        return lo + self.below(hi - lo + 1)

    def unit(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def choice(self, seq):
        return seq[self.below(len(seq))]


PRINTABLE = bytes(range(0x20, 0x7F))
LOWER = b"abcdefghijklmnopqrstuvwxyz"


def fill_uniform(n: int, alphabet: bytes, seed: int) -> np.ndarray:
    out = np.empty(n + 64, dtype=np.uint8)[:n]
    al = np.frombuffer(alphabet, dtype=np.uint8).copy()
    _lib().wl_fill_uniform(_u8p(out), n, _u8p(al), len(alphabet), seed, 0)
    return out


def fill_markov(n: int, alphabet: bytes, seed: int, matrix_seed: int) -> np.ndarray:
    out = np.empty(n + 64, dtype=np.uint8)[:n]
    al = np.frombuffer(alphabet, dtype=np.uint8).copy()
    _lib().wl_fill_markov(_u8p(out), n, _u8p(al), len(alphabet), seed, matrix_seed, 0)
    return out


def fill_acgt(n: int, seed: int, p_run: float = 0.01 / 25.5, run_lo: int = 1, run_hi: int = 50) -> np.ndarray:
    out = np.empty(n + 64, dtype=np.uint8)[:n]
    _lib().wl_fill_acgt(_u8p(out), n, seed, p_run, run_lo, run_hi, 0)
    return out


def gen_literals(n: int, lmin: int, lmax: int, alphabet: bytes, weights, seed: int) -> list[bytes]:
    al = np.frombuffer(alphabet, dtype=np.uint8).copy()
    w = np.asarray(weights, dtype=np.float64)
    buf = np.zeros(n * lmax, dtype=np.uint8)
    lens = np.zeros(n, dtype=np.uint32)
    _lib().wl_gen_literals(n, lmin, lmax, _u8p(al), w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           len(alphabet), seed, _u8p(buf), lens.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    out, o = [], 0
    for L in lens.tolist():
        out.append(bytes(buf[o:o + L]))
        o += L
    return out


def zipf_alphabet(seed: int, s: float = 1.1) -> tuple[bytes, list[float]]:
    """Printable ASCII with Zipf(s) rank weights over a seeded permutation."""
    r = Rng(seed)
    perm = list(PRINTABLE)
    for i in range(len(perm) - 1, 0, -1):
        j = r.below(i + 1)
        perm[i], perm[j] = perm[j], perm[i]
    weights = [1.0 / (k + 1) ** s for k in range(len(perm))]
    return bytes(perm), weights


def plant(data: np.ndarray, items: list[bytes], slot: int, seed: int) -> list[tuple[int, int]]:
    """Writes items[i] into slot i (one per `slot` bytes) at a seeded offset
    inside the slot, so plants never overlap.  Returns (offset, item index)."""
    r = Rng(seed)
    n_slots = len(data) // slot
    placed = []
    for k in range(n_slots):
        it = r.below(len(items))
        b = items[it]
        if len(b) >= slot:
            continue
        off = k * slot + r.below(slot - len(b))
        data[off:off + len(b)] = np.frombuffer(b, dtype=np.uint8)
        placed.append((off, it))
    return placed


# ---------------------------------------------------------------- regexes
JOIN_CLASSES = ["[0-9]", "[A-F]", "[G-M]", "[N-T]", "[U-Z]", "[_.-]", "[ ]", "[#$%&]", "[0-4]", "[5-9]"]
REGEX_LIT_ALPHABET = b"abcdefghijklmnop"


def _class_members(cls: str) -> bytes:
    body = cls[1:-1]
    out = bytearray()
    i = 0
    while i < len(body):
        if i + 2 < len(body) and body[i + 1] == "-":
            out.extend(range(ord(body[i]), ord(body[i + 2]) + 1))
            i += 3
        else:
            out.append(ord(body[i]))
            i += 1
    return bytes(out)


@dataclass
class RegexSpec:
    source: str
    alts_a: list[bytes]
    join: str
    rep: tuple[int, int]
    alts_b: list[bytes]

    def sample(self, r: Rng) -> bytes:
        a = r.choice(self.alts_a)
        members = _class_members(self.join)
        k = r.uniform(*self.rep)
        mid = bytes(r.choice(members) for _ in range(k))
        return a + mid + r.choice(self.alts_b)


def gen_regexes(n: int, seed: int, alphabet: bytes = REGEX_LIT_ALPHABET, lmin: int = 4, lmax: int = 12) -> list[RegexSpec]:
    r = Rng(seed)

    def lit() -> bytes:
        L = r.uniform(lmin, lmax)
        return bytes(r.choice(alphabet) for _ in range(L))

    out = []
    for _ in range(n):
        a = [lit() for _ in range(r.uniform(2, 4))]
        b = [lit() for _ in range(r.uniform(2, 4))]
        join = r.choice(JOIN_CLASSES)
        src = "(?:" + "|".join(x.decode() for x in a) + ")" + join + "{1,8}" + \
              "(?:" + "|".join(x.decode() for x in b) + ")"
        out.append(RegexSpec(src, a, join, (1, 8), b))
    return out


IUPAC = {"R": "AG", "Y": "CT", "S": "CG", "W": "AT", "K": "GT", "M": "AC",
         "B": "CGT", "D": "AGT", "H": "ACT", "V": "ACG", "N": "ACGT"}


def gen_iupac(n: int, seed: int, lmin: int = 20, lmax: int = 40) -> list[tuple[str, list[str]]]:
    r = Rng(seed)
    codes = list(IUPAC)
    out = []
    for _ in range(n):
        L = r.uniform(lmin, lmax)
        pos = []
        for _ in range(L):
            if r.below(100) < 85:
                pos.append(r.choice("ACGT"))
            else:
                pos.append(r.choice(codes))
        src = "".join(c if c in "ACGT" else "[" + IUPAC[c] + "]" for c in pos)
        out.append((src, pos))
    return out


# ---------------------------------------------------------------- workloads
@dataclass
class Workload:
    name: str
    patterns: list[tuple[int, bytes]]          # (kind, bytes): 0 literal, 1 regex
    data: np.ndarray | None = None
    items: list[tuple[int, int]] | None = None   # (offset, length) into data
    meta: dict = field(default_factory=dict)


LIT, REGEX = 0, 1


def literals_small(size: int = 16 * MiB, n: int = 100, seed: int = 1) -> Workload:
    lits = gen_literals(n, 4, 16, LOWER, [1.0] * 26, seed * 1000 + 1)
    data = fill_uniform(size, LOWER, seed * 1000 + 2)
    plant(data, lits, 64 * 1024 if size >= 256 * 1024 else max(64, size // 16), seed * 1000 + 3)
    return Workload("literals_small", [(LIT, l) for l in lits], data,
                    meta={"literals": n, "bytes": size, "lengths": "4-16", "alphabet": "a-z"})


def literals_large(size: int = GiB, n: int = 10_000, seed: int = 2) -> Workload:
    alpha, w = zipf_alphabet(seed * 1000 + 1)
    lits = gen_literals(n, 8, 32, alpha, w, seed * 1000 + 2)
    data = fill_markov(size, PRINTABLE, seed * 1000 + 3, seed * 1000 + 4)
    plant(data, lits, 16 * 1024 if size >= 1 * MiB else max(64, size // 64), seed * 1000 + 5)
    return Workload("literals_large", [(LIT, l) for l in lits], data,
                    meta={"literals": n, "bytes": size, "lengths": "8-32", "alphabet": "printable zipf(1.1)"})


def regex(size: int = GiB, n: int = 500, seed: int = 3) -> Workload:
    specs = gen_regexes(n, seed * 1000 + 1)
    data = fill_markov(size, PRINTABLE, seed * 1000 + 3, seed * 1000 + 4)
    r = Rng(seed * 1000 + 5)
    samples = [specs[r.below(n)].sample(r) for _ in range(4096)]
    plant(data, samples, 16 * 1024 if size >= 1 * MiB else max(128, size // 64), seed * 1000 + 6)
    return Workload("regex", [(REGEX, s.source.encode()) for s in specs], data,
                    meta={"regexes": n, "bytes": size})


def regex_training_corpus(size: int = 256 * MiB, seed: int = 3) -> np.ndarray:
    """Separately seeded corpus of the regex configuration's distribution."""
    return fill_markov(size, PRINTABLE, seed * 1000 + 77, seed * 1000 + 4)


def dna_training_corpus(size: int = 256 * MiB, seed: int = 5) -> np.ndarray:
    """Separately seeded corpus of the nucleotide configuration's distribution."""
    return fill_acgt(size, seed * 1000 + 77)


def batch(n_items: int = 200_000, n_lit: int = 1500, n_rx: int = 500, seed: int = 4,
          median: float = 4096.0, sigma: float = 1.5, lo: int = 64, hi: int = MiB) -> Workload:
    r = Rng(seed * 1000 + 1)
    sizes = []
    for _ in range(n_items):
        # Box-Muller normal from two uniforms
        u1 = max(r.unit(), 1e-300)
        u2 = r.unit()
        z = math.sqrt(-2.0 * math.log(u1)) * math.cos(2 * math.pi * u2)
        sizes.append(int(min(hi, max(lo, round(math.exp(math.log(median) + sigma * z))))))
    total = sum(sizes)
    data = fill_markov(total, PRINTABLE, seed * 1000 + 3, 3 * 1000 + 4)
    alpha, w = zipf_alphabet(seed * 1000 + 2)
    lits = gen_literals(n_lit, 6, 24, alpha, w, seed * 1000 + 5)
    specs = gen_regexes(n_rx, 3 * 1000 + 1)
    items, off = [], 0
    for s in sizes:
        items.append((off, s))
        off += s
    samples = lits[:] + [specs[r.below(len(specs))].sample(r) for _ in range(len(lits))]
    plant(data, samples, 16 * 1024 if total >= MiB else max(128, total // 64), seed * 1000 + 6)
    pats = [(LIT, l) for l in lits] + [(REGEX, s.source.encode()) for s in specs]
    return Workload("batch", pats, data, items=items,
                    meta={"items": n_items, "bytes": total, "literals": n_lit, "regexes": n_rx})


def dna(size: int = 4 * GiB, n_kmer: int = 50_000, n_rx: int = 200, seed: int = 5) -> Workload:
    kmers = gen_literals(n_kmer, 20, 32, b"ACGT", [1.0] * 4, seed * 1000 + 1)
    rx = gen_iupac(n_rx, seed * 1000 + 2)
    data = fill_acgt(size, seed * 1000 + 3)
    r = Rng(seed * 1000 + 4)
    samples = kmers[:2048] + [bytes(r.choice(IUPAC.get(c, c)).encode()[0] for c in pos) for _, pos in rx]
    plant(data, samples, MiB if size >= 64 * MiB else max(256, size // 64), seed * 1000 + 5)
    pats = [(LIT, k) for k in kmers] + [(REGEX, s.encode()) for s, _ in rx]
    return Workload("dna", pats, data, meta={"kmers": n_kmer, "regexes": n_rx, "bytes": size})
