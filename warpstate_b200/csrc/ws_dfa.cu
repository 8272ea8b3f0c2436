// Regex DFA path for sm_100a (see ws_dfa.h for the pipeline).
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <numeric>

#include "ws_dfa.h"
#include "ws_async.h"
#include "ws_proposer.h"

namespace cg = cooperative_groups;

namespace ws {

namespace {

constexpr uint32_t F_MATCH = 0x80000000u;
constexpr uint32_t F_DEAD = 0x40000000u;
constexpr uint32_t F_MASK = 0x3FFFFFFFu;
constexpr uint32_t kCkpt = 256;       // bytes between recorded walk states
constexpr int kFixRounds = 3;         // parallel fix-up rounds before the serial sweep
constexpr int kWalkThreads = 1024;    // threads (= chunks) per walk block
// Reverse walks share a lossy table of visited (position, group, state)
// triples: a walk that reaches a triple another walk has passed stops there,
// since the rest of its walk -- and every start it would report -- is the
// other walk's.  This keeps a long run of match ends (a+ over a run of a's)
// linear instead of quadratic.  2^kRmarkBits slots of 8 bytes, cleared per scan.
constexpr uint32_t kRmarkBits = 20;
constexpr uint32_t kRmarkStateBits = 20;  // states below 2^20, groups below 2^12
// Leftmost-first walks in the parallel pass stop after kLfCap bytes; the
// chain kernel finishes such a walk only if it picks that start (picked
// matches do not overlap, so that work is bounded by the input).
constexpr uint64_t kLfCap = 1024;
constexpr uint32_t kLfNone = 0xFFFFFFFFu;  // no match from this start (or a duplicate start)
constexpr uint32_t kLfLong = 0xFFFFFFFEu;  // the walk reached kLfCap bytes

// ------------------------------------------------------------ scratch layout
struct RxLayout {
  uint64_t n_chunks = 0, chunk = 0, nck = 0, n_q = 0;
  uint64_t k_cap = 0, ev_cap = 0;
  size_t off_ctr, off_k, off_ev, off_guess, off_used, off_end, off_spec, off_conv, off_round, off_ckpt,
      off_count, off_offs, off_cursor, off_starts, off_lfend, off_rmark, total;
};

struct KCand { uint32_t r, s, e; };
struct Event { uint32_t e, state, q, tag; };

// counters block (unsigned long long[16]):
//  [0] K count  [1] event count  [2] error flags  [3..3+kFixRounds] round-changed flags
//  [8] chunk re-walks of the fix-up  [9] bytes those re-walks stepped
//  [10] boundary guesses that were the true state  [11] boundary guesses
enum { C_K = 0, C_EV = 1, C_ERR = 2, C_ROUND = 3, C_FIX = 8, C_REWALK = 9, C_HITS = 10, C_GUESSES = 11 };
// error bits in ctr[C_ERR]: 1 candidate overflow, 2 event overflow, 4 a
// bounded device-side wait ran out
constexpr unsigned long long kErrTimeout = 4;
static_assert(C_ROUND + kFixRounds < C_FIX, "counter slots overlap");

// Candidate and event buffers hold at most this many entries (the per-regex
// offsets of the resolution are 32-bit).
constexpr uint64_t kMaxCandidates = 0x7FFFFFFFull;

// k_min / ev_min: capacities an earlier scan of this matcher found it needed.
RxLayout layout(const RegexPlan& p, uint64_t len, uint32_t chunk, uint64_t max_matches, uint64_t k_min = 0,
                uint64_t ev_min = 0) {
  RxLayout L;
  L.chunk = chunk;
  L.n_chunks = (len + chunk - 1) / chunk;
  L.nck = chunk / kCkpt;
  L.n_q = L.n_chunks * p.n_spec;
  const uint64_t base = std::max<uint64_t>(2 * max_matches, len / 256 + 65536);
  L.k_cap = std::min(kMaxCandidates, std::max(base, k_min));
  L.ev_cap = std::min(kMaxCandidates, std::max(base, ev_min));
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = (o + bytes + 255) & ~(size_t)255; return r; };
  L.off_ctr = take(16 * 8);
  L.off_k = take(L.k_cap * sizeof(KCand));
  L.off_ev = take(L.ev_cap * sizeof(Event));
  L.off_guess = take(L.n_q * 4);
  L.off_used = take(L.n_q * 4);
  L.off_end = take(L.n_q * 4);
  L.off_spec = take(L.n_q * 4);
  L.off_conv = take(L.n_q * 4);
  L.off_round = take(L.n_q * 4);
  L.off_ckpt = take(L.n_q * L.nck * 4);
  L.off_count = take((size_t)p.n_regex * 4);
  L.off_offs = take(((size_t)p.n_regex + 1) * 4);
  L.off_cursor = take((size_t)p.n_regex * 4);
  L.off_starts = take(L.k_cap * 4);
  L.off_lfend = take(L.k_cap * 4);
  L.off_rmark = take(((size_t)1 << kRmarkBits) * 8);
  L.total = o;
  return L;
}

struct DevTables {
  const GroupDev* groups;
  const uint32_t* fwd;
  const uint32_t* hot;
  const uint32_t* rev;
  const uint32_t* lf;
  const uint8_t* cls;
  const uint32_t* mptr;
  const uint32_t* mlist;
  const uint32_t* rmptr;
  const uint32_t* rmlist;
  const uint4* lfinfo;   // per regex: {lf_off, lf_start row, group, classes}
  const uint32_t* lfx;   // per regex: context DFA starts and end-step flags (8 words)
  const uint32_t* pid;
  uint32_t n_groups, n_regex, n_spec;
};

struct ScanPtrs {
  const uint8_t* data;
  uint64_t len;
  unsigned long long* ctr;
  KCand* k;
  uint64_t k_cap;
  Event* ev;
  uint64_t ev_cap;
  uint32_t* guess;
  uint32_t* used;
  uint32_t* end;
  uint32_t* spec;
  uint32_t* conv;
  uint32_t* round;
  uint32_t* ckpt;
  uint32_t* count;
  uint32_t* offs;
  uint32_t* cursor;
  uint32_t* starts;
  uint32_t* lfend;
  unsigned long long* rmark;    // visited reverse-walk triples, or null (state numbers too large, or full K)
  uint32_t full_k;              // report every (start, end) of K, not only distinct starts (diagnostics)
  uint32_t count_guesses;       // profiled speculative scans: the speculative groups whose guesses are counted
  uint64_t n_chunks, chunk, nck;
  ws_match* out;
  uint64_t out_cap;
  unsigned long long* out_counter;
  const uint32_t* item_end;     // batch item ends (n_items), else null
  uint32_t n_items;
  unsigned long long* cursor64;  // stream: per-regex find_iter position, else null
  uint64_t base, frontier;
};

ScanPtrs make_ptrs(const RxLayout& L, void* base, const RegexLaunch& l) {
  uint8_t* b = static_cast<uint8_t*>(base);
  ScanPtrs p;
  p.data = l.data;
  p.len = l.len;
  p.ctr = reinterpret_cast<unsigned long long*>(b + L.off_ctr);
  p.k = reinterpret_cast<KCand*>(b + L.off_k);
  p.k_cap = L.k_cap;
  p.ev = reinterpret_cast<Event*>(b + L.off_ev);
  p.ev_cap = L.ev_cap;
  p.guess = reinterpret_cast<uint32_t*>(b + L.off_guess);
  p.used = reinterpret_cast<uint32_t*>(b + L.off_used);
  p.end = reinterpret_cast<uint32_t*>(b + L.off_end);
  p.spec = reinterpret_cast<uint32_t*>(b + L.off_spec);
  p.conv = reinterpret_cast<uint32_t*>(b + L.off_conv);
  p.round = reinterpret_cast<uint32_t*>(b + L.off_round);
  p.ckpt = reinterpret_cast<uint32_t*>(b + L.off_ckpt);
  p.count = reinterpret_cast<uint32_t*>(b + L.off_count);
  p.offs = reinterpret_cast<uint32_t*>(b + L.off_offs);
  p.cursor = reinterpret_cast<uint32_t*>(b + L.off_cursor);
  p.starts = reinterpret_cast<uint32_t*>(b + L.off_starts);
  p.lfend = reinterpret_cast<uint32_t*>(b + L.off_lfend);
  p.rmark = reinterpret_cast<unsigned long long*>(b + L.off_rmark);
  p.full_k = 0;
  p.count_guesses = 0;
  p.n_chunks = L.n_chunks;
  p.chunk = L.chunk;
  p.nck = L.nck;
  p.out = l.out;
  p.out_cap = l.cap;
  p.out_counter = l.counter;
  p.item_end = l.item_end;
  p.n_items = l.n_items;
  p.cursor64 = l.cursor;
  p.base = l.base;
  p.frontier = l.frontier;
  return p;
}

// One slot of an append buffer, one atomic per group of converged lanes.
__device__ __forceinline__ unsigned long long warp_append(unsigned long long* counter) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, (unsigned long long)g.size());
  base = g.shfl(base, 0);
  return base + g.thread_rank();
}

// Appends a candidate and counts it for its regex (the per-regex counts size
// the resolution's start lists).
__device__ __forceinline__ void emit_k(const ScanPtrs& p, uint32_t r, uint32_t s, uint32_t e) {
  unsigned long long i = warp_append(&p.ctr[C_K]);
  if (i < p.k_cap) {
    p.k[i] = KCand{r, s, e};
    atomicAdd(&p.count[r], 1u);
  } else {
    atomicOr(&p.ctr[C_ERR], 1ull);
  }
}

__device__ __forceinline__ void emit_event(const ScanPtrs& p, uint32_t e, uint32_t st, uint32_t q, uint32_t tag) {
  unsigned long long i = warp_append(&p.ctr[C_EV]);
  if (i < p.ev_cap) p.ev[i] = Event{e, st, q, tag};
  else atomicOr(&p.ctr[C_ERR], 2ull);
}

// Shared-memory image of a group's hot rows (32-bit words, 7 blocks of 8192):
//   block 0     the first hot row, replicated per lane: word b * 32 + lane;
//   blocks 1..6 hot rows 1..191 column-interleaved: row r, byte b at word
//               (1 + r / 32) * 8192 + b * 32 + r % 32 (column 0 of block 1 is
//               the trap column, see below).
// A thread's state is the byte offset of its row's column (lane * 4 for the
// first row), so the entry for byte b is at state + b * 128 and every row sits
// in one bank: lanes in the first row never conflict, lanes in other rows only
// when their rows share a column.  An entry is either the next row's byte
// offset (0 for the first row, made lane-specific by max(entry, lane * 4)), or
// a slow word (bit 31) for transitions into match, cold or dead states.  Cold
// states run through the trap column, whose entries are all slow, and take
// their transitions from the class-indexed table through L2.
constexpr uint32_t kImgBlock = 8192;
constexpr uint32_t kImgWords = 7 * kImgBlock;
constexpr uint32_t kTrapByte = kImgBlock * 4;
constexpr uint32_t S_SLOW = 0x80000000u, S_MATCH = 0x40000000u, S_COLD = 0x20000000u, S_TRAP = 0x10000000u,
                   S_DEAD = 0x08000000u, S_ROW = 0x07FFFFFFu;

// Shared memory of a walk block: [hot image][byte classes, 256 B][mbarrier, 16 B].
__host__ __device__ constexpr size_t hot_smem_bytes(uint32_t rows) {
  return (rows ? (size_t)kImgWords * 4 : 0) + 256 + 16;
}
__host__ __device__ constexpr size_t cls_offset(uint32_t rows) { return rows ? (size_t)kImgWords * 4 : 0; }

// The speculative walk and the fix-up stage the first kWalkImgBlocks blocks
// of the unanchored image (its hot rows are at most kHotRowsWalk, all in those
// blocks); the walk block's shared memory is
//   [image, 192 KiB][input stages: per warp 2 x 512 B][classes, 256 B]
//   [image mbarrier, 16 B][stage mbarriers: per warp 2 x 8 B].
constexpr uint32_t kWalkImgBlocks = 6;
constexpr uint32_t kWalkImgBytes = kWalkImgBlocks * kImgBlock * 4;
constexpr uint32_t kWalkWarps = kWalkThreads / 32;
constexpr uint32_t kWalkStage = 512;  // one warp's 16 bytes per lane (a 16 x 32 box of the chunk rows)
constexpr uint32_t kWalkStageBytes = kWalkWarps * 2 * kWalkStage;
constexpr size_t kWalkSmem = kWalkImgBytes + kWalkStageBytes + 256 + 16 + kWalkWarps * 2 * 8;
constexpr size_t kFixSmem = kWalkImgBytes + 256 + 16;
static_assert(kWalkSmem <= 232448, "walk block shared memory");

__host__ __device__ __forceinline__ uint32_t slot_word(uint32_t r) { return (1 + (r >> 5)) * kImgBlock + (r & 31); }

__device__ __forceinline__ uint32_t slot_byte(uint32_t r, uint32_t lane4) { return r == 0 ? lane4 : slot_word(r) * 4; }

// Global row of a walk state (rows of this image start at `first`).
__device__ __forceinline__ uint32_t row_of(uint32_t st, uint32_t cold_row, uint32_t first) {
  if (st < 128) return first;
  if (st == kTrapByte) return cold_row;
  uint32_t w = st >> 2;
  return first + ((w >> 13) - 1) * 32 + (w & 31);
}

// Walk state of a global row.
__device__ __forceinline__ uint32_t state_of(uint32_t row, uint32_t first, uint32_t rows, uint32_t lane4,
                                             uint32_t* cold_row) {
  uint32_t r = row - first;
  if (r < rows) return slot_byte(r, lane4);
  *cold_row = row;
  return kTrapByte;
}

// Stages a group's hot-row image (224 KiB) and byte-class map into shared
// memory with two bulk (TMA) copies completing on one mbarrier.  The wait is
// bounded: when it runs out (it should not), the block records a timeout in
// `err`, waits once more (again bounded) for the copies it issued, and the
// caller returns without walking (false); the scan then reports the timeout.
__device__ __forceinline__ bool stage_hot(const DevTables& t, uint32_t g, uint32_t off, uint32_t rows,
                                          uint32_t* img, uint8_t* cls_s, unsigned long long* err,
                                          uint32_t img_bytes = kImgWords * 4) {
  uint64_t* bar = reinterpret_cast<uint64_t*>(cls_s + 256);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar, (rows ? img_bytes : 0) + 256);
    if (rows) bulk_copy_g2s(img, t.hot + off, img_bytes, bar);
    bulk_copy_g2s(cls_s, t.cls + g * 256, 256, bar);
  }
  bool ok = false;
  for (uint32_t it = 0; it < (1u << 22) && !ok; ++it) ok = mbar_try(bar, 0);
  if (__syncthreads_and(ok)) return true;
  if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
  ok = false;
  for (uint32_t it = 0; it < (1u << 22) && !ok; ++it) ok = mbar_try(bar, 0);
  __syncthreads();
  return false;
}

// Slow path of one transition: handles match / cold / dead and returns false
// when the walk reached the dead state.  `m_row` receives the row of a match
// state (0xFFFFFFFF when none).
__device__ __forceinline__ bool slow_step(uint32_t w, uint32_t b, uint32_t& st, uint32_t& cold_row, uint32_t first,
                                          uint32_t rows, uint32_t lane4, const uint8_t* cls_s, const uint32_t* tab,
                                          uint32_t C, uint32_t& m_row) {
  uint32_t n;
  bool match, cold, dead;
  if (w & S_TRAP) {
    uint32_t t = __ldg(tab + cold_row * C + cls_s[b]);
    n = t & F_MASK;
    match = t & F_MATCH;
    dead = t & F_DEAD;
    cold = (n - first) >= rows;
  } else {
    n = w & S_ROW;
    match = w & S_MATCH;
    dead = w & S_DEAD;
    cold = w & S_COLD;
  }
  m_row = match ? n : 0xFFFFFFFFu;
  if (dead) return false;
  if (cold) { st = kTrapByte; cold_row = n; }
  else st = slot_byte(n - first, lane4);
  return true;
}

#define WS_STEP_FAST(img, st, b) (*reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(img) + (st) + ((b) << 7)))

// Geometry of the walk's unanchored image: 32-row blocks of `img_cols`
// entries per row (256: indexed by byte; or the group's class count: indexed
// by class), block 0 the first row once per lane, the trap column at block 1,
// column 0.  A walk state is the byte offset of its row's column.
struct WalkImg {
  uint32_t blk_words;  // words per block: 32 x img_cols
  uint32_t trap;       // byte offset of the trap column
};
__device__ __forceinline__ WalkImg walk_img(const GroupDev& gd) { return {gd.img_cols * 32, gd.img_cols * 128}; }
__device__ __forceinline__ uint32_t wslot(const WalkImg& g, uint32_t r, uint32_t lane4) {
  return r == 0 ? lane4 : ((1 + (r >> 5)) * g.blk_words + (r & 31)) * 4;
}
__device__ __forceinline__ uint32_t wrow(const WalkImg& g, uint32_t st, uint32_t cold_row) {
  if (st < 128) return 0;
  if (st == g.trap) return cold_row;
  const uint32_t w = st >> 2;
  return (w / g.blk_words - 1) * 32 + (w & 31);
}
__device__ __forceinline__ uint32_t wstate(const WalkImg& g, uint32_t row, uint32_t rows, uint32_t lane4,
                                           uint32_t* cold_row) {
  if (row < rows) return wslot(g, row, lane4);
  *cold_row = row;
  return g.trap;
}
// The image column of input byte b: the byte itself, or its class.
template <bool kCls>
__device__ __forceinline__ uint32_t wcol(const uint8_t* cls_s, uint32_t b) {
  return kCls ? (uint32_t)cls_s[b] : b;
}

// One transition of the walk's image: an entry other than the trap column's
// offset is the next hot row's column; the trap offset sends the transition
// to the class-indexed table, from the hot row or the cold row the walk is in.
// Returns the row of a match state (0xFFFFFFFF when none).
template <bool kCls>
__device__ __forceinline__ uint32_t trap_step(const uint32_t* img, const WalkImg& gi, uint32_t b, uint32_t& st,
                                              uint32_t& cold_row, uint32_t H, uint32_t lane4, const uint8_t* cls_s,
                                              const uint32_t* tab, uint32_t C) {
  const uint32_t c = cls_s[b];
  const uint32_t w = WS_STEP_FAST(img, st, kCls ? c : b);
  if (w != gi.trap) {
    st = max(w, lane4);
    return 0xFFFFFFFFu;
  }
  const uint32_t t = __ldg(tab + wrow(gi, st, cold_row) * C + c);
  const uint32_t n = t & F_MASK;
  if (n < H && !(t & F_DEAD)) {
    st = wslot(gi, n, lane4);
  } else {
    st = gi.trap;
    cold_row = n;
  }
  return (t & F_MATCH) ? n : 0xFFFFFFFFu;
}

// One transition through L2 only (fix-up walks, which are short and rare).
__device__ __forceinline__ uint32_t step_l2(uint32_t st, uint32_t b, const uint8_t* cls_g, const uint32_t* tab,
                                            uint32_t C) {
  return __ldg(tab + st * C + __ldg(cls_g + b));
}

// ------------------------------------------------------------- plain kernel
// One thread per start position; an anchored walk of the group's DFA until the
// dead state, every match state reached yields K candidates (the reference's
// per-start walk, core/src/gpu/ensemble_shader.wgsl:92-124, over the merged
// group DFA, reporting every match instead of stopping at the first).
// blockIdx.y = group; the group's hottest anchored rows sit in shared memory.
__global__ void __launch_bounds__(kWalkThreads, 1) dfa_plain_kernel(DevTables t, ScanPtrs p) {
  extern __shared__ __align__(16) uint32_t smem[];
  const uint32_t g = blockIdx.y;
  const GroupDev gd = t.groups[g];
  uint32_t* img = smem;
  uint8_t* cls_s = reinterpret_cast<uint8_t*>(smem) + cls_offset(gd.ahot_rows);
  if (!stage_hot(t, g, gd.ahot_off, gd.ahot_rows, img, cls_s, &p.ctr[C_ERR])) return;
  const uint32_t* tab = t.fwd + gd.fwd_off;
  const uint32_t* mp = t.mptr + gd.mptr_off;
  const uint32_t C = gd.n_classes, first = gd.ahot_base, rows = gd.ahot_rows;
  const uint32_t lane4 = (threadIdx.x & 31) * 4;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < p.len; s += stride) {
    uint32_t cold_row = 0;
    uint32_t st = state_of(gd.start_anchored, first, rows, lane4, &cold_row);
    const uint64_t stop = p.n_items ? min(p.len, (uint64_t)item_end_of(p.item_end, p.n_items, (uint32_t)s)) : p.len;
    // a candidate is (regex, start): the end is recomputed leftmost-first
    // later, so a match row reported earlier on this walk (a self-loop such
    // as a+, a short cycle such as (ab)+) adds nothing; the last four are kept
    uint32_t seen0 = 0xFFFFFFFFu, seen1 = 0xFFFFFFFFu, seen2 = 0xFFFFFFFFu, seen3 = 0xFFFFFFFFu;
    for (uint64_t e = s; e < stop; ++e) {
      uint32_t b = __ldg(p.data + e);
      uint32_t w = WS_STEP_FAST(img, st, b);
      if ((int32_t)w >= 0) {
        st = max(w, lane4);
        continue;
      }
      uint32_t m_row;
      bool alive = slow_step(w, b, st, cold_row, first, rows, lane4, cls_s, tab, C, m_row);
      if (m_row != 0xFFFFFFFFu &&
          (p.full_k || (m_row != seen0 && m_row != seen1 && m_row != seen2 && m_row != seen3))) {
        for (uint32_t j = __ldg(mp + m_row); j < __ldg(mp + m_row + 1); ++j)
          emit_k(p, __ldg(t.mlist + j), (uint32_t)s, (uint32_t)(e + 1));
        seen3 = seen2;
        seen2 = seen1;
        seen1 = seen0;
        seen0 = m_row;
      }
      if (!alive) break;
    }
  }
}

// --------------------------------------------------------- context groups
// Context of a byte for the assertions (byte_context in ws_regex.h).
__device__ __forceinline__ uint32_t ctx_of(uint32_t b) {
  if (b == '\n') return CTX_NL;
  const bool w = (b - '0' < 10u) || ((b | 0x20u) - 'a' < 26u) || b == '_';
  return w ? CTX_WORD : CTX_OTHER;
}

// Context groups: one thread per start position, the anchored walk of the
// group's context DFA (build_context_all_dfa): the start row chosen by the
// byte before the start (CTX_BEGIN at the start of the input or item), the
// transition on the byte at e reporting the patterns whose match ends at e,
// and after the last byte the end step (right context CTX_BEGIN) at the end
// of the input or item.  Walks of starts whose match cannot end by then stop
// at the buffer's end like the others; a caller decides only starts whose
// walks die before it (streams, shards).  blockIdx.y = context group.  The
// tables are read through L1/L2: these groups hold the patterns with
// assertions, whose anchored walks mostly die within a few bytes.
__global__ void __launch_bounds__(256) dfa_context_kernel(DevTables t, ScanPtrs p) {
  __shared__ uint8_t cls_s[256];
  const uint32_t g = t.n_spec + blockIdx.y;
  const GroupDev gd = t.groups[g];
  for (uint32_t k = threadIdx.x; k < 256; k += blockDim.x) cls_s[k] = t.cls[g * 256 + k];
  __syncthreads();
  const uint32_t* tab = t.fwd + gd.fwd_off;
  const uint32_t* mp = t.mptr + gd.mptr_off;
  const uint32_t C = gd.n_classes;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < p.len; s += stride) {
    const uint64_t lo = p.n_items ? item_start_of(p.item_end, p.n_items, (uint32_t)s) : 0;
    const uint64_t stop = p.n_items ? min(p.len, (uint64_t)item_end_of(p.item_end, p.n_items, (uint32_t)s)) : p.len;
    uint32_t st = gd.cstart[s == lo ? CTX_BEGIN : ctx_of(__ldg(p.data + s - 1))];
    // a candidate is (regex, start); a list reported earlier on this walk
    // adds nothing (the last four are kept)
    uint32_t seen0 = 0xFFFFFFFFu, seen1 = 0xFFFFFFFFu, seen2 = 0xFFFFFFFFu, seen3 = 0xFFFFFFFFu;
    auto report = [&](uint32_t slot, uint64_t e) {
      const uint32_t a = __ldg(mp + slot), b = __ldg(mp + slot + 1);
      if (a == b) return;
      if (!p.full_k && (a == seen0 || a == seen1 || a == seen2 || a == seen3)) return;
      for (uint32_t j = a; j < b; ++j) emit_k(p, __ldg(t.mlist + j), (uint32_t)s, (uint32_t)e);
      seen3 = seen2;
      seen2 = seen1;
      seen1 = seen0;
      seen0 = a;
    };
    bool alive = true;
    for (uint64_t e = s; e < stop; ++e) {
      const uint32_t b = __ldg(p.data + e);
      const uint32_t w = __ldg(tab + st * C + cls_s[b]);
      if (w & F_MATCH) report(st * 4 + ctx_of(b), e);
      if (w & F_DEAD) {
        alive = false;
        break;
      }
      st = w & F_MASK;
    }
    if (alive) report(st * 4 + CTX_BEGIN, stop);
  }
}

// ------------------------------------------------------- speculative walk
// Thread per (group, chunk): unanchored walk from the proposed start state,
// recording the state every kCkpt bytes, the end state and every match event.
// blockIdx.x = group; the group's hottest rows sit in shared memory.
//
// Input staging: the 32 lanes of a warp walk 32 adjacent chunks, so a warp's
// next 16 bytes per lane are a 16 x 32 box of the input seen as a 2-D tensor
// of full chunks (rows of `chunk` bytes).  Lane 0 brings each box into one of
// the warp's two shared-memory stages with a tensor copy (TMA) on the stage's
// mbarrier, two steps ahead, and every lane reads its 16 bytes from there.
// The input never passes through the load/store pipe, whose wavefronts the
// hot-row lookups need; one 16-byte load per lane and step from 32 different
// chunks would each take a wavefront and an L2 sector.  A lane whose chunk
// is not a full one (the last, partial chunk) loads its bytes itself.
// Whether a group's chunks start from their exact state: a bounded-length
// group (GroupDev::warm) whose warm-up is at most a quarter of the chunk.
__host__ __device__ __forceinline__ bool warm_exact(const GroupDev& gd, uint64_t chunk) {
  return gd.warm != 0 && 4 * (uint64_t)gd.warm <= chunk;
}

template <bool kCls>
__global__ void __launch_bounds__(kWalkThreads, 1)
    dfa_walk_kernel(DevTables t, ScanPtrs p, const __grid_constant__ CUtensorMap rows, uint64_t n_full) {
  extern __shared__ __align__(128) uint32_t smem[];
  // blockIdx.x = group (fastest), so the groups' blocks over the same chunks
  // run together and the input is read from HBM once, then from L2
  const uint32_t g = blockIdx.x;
  const GroupDev gd = t.groups[g];
  uint32_t* img = smem;
  uint8_t* stages = reinterpret_cast<uint8_t*>(smem) + kWalkImgBytes;
  uint8_t* cls_s = stages + kWalkStageBytes;
  uint64_t* sbar = reinterpret_cast<uint64_t*>(cls_s + 256 + 16);
  if (!stage_hot(t, g, gd.hot_off, gd.hot_rows, img, cls_s, &p.ctr[C_ERR], gd.img_bytes)) return;
  const WalkImg gi = walk_img(gd);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t wfirst = (uint64_t)blockIdx.y * blockDim.x + warp * 32;  // lane 0's chunk
  if (wfirst >= p.n_chunks) return;  // the whole warp
  const bool wtma = wfirst < n_full;  // the warp's boxes come by TMA
  uint64_t* bar = sbar + warp * 2;
  uint8_t* stg = stages + warp * 2 * kWalkStage;
  const uint64_t K = p.chunk / 16;  // 16-byte steps of a full chunk
  // the input is read once: its lines go first when L2 needs room, which
  // keeps the tables of the later kernels (reverse, resolution) resident
  const uint64_t in_policy = l2_evict_first_policy();
  if (wtma && lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
    for (uint32_t s = 0; s < 2 && s < K; ++s) {
      mbar_expect_tx(&bar[s], kWalkStage);
      tma_load_2d_hint(stg + s * kWalkStage, &rows, (int32_t)(s * 16), (int32_t)wfirst, &bar[s], in_policy);
    }
  }
  __syncwarp();
  const uint64_t i = wfirst + lane;
  const bool active = i < p.n_chunks;
  const bool own = i >= n_full;  // loads its own bytes (partial chunk) or, out of range, none
  const uint32_t* tab = t.fwd + gd.fwd_off;
  const uint32_t C = gd.n_classes, H = gd.hot_rows;
  const int32_t lane4 = (int32_t)(lane * 4);
  const uint64_t q = (uint64_t)g * p.n_chunks + i;
  const uint64_t c0 = i * p.chunk;
  const uint64_t c1 = active ? min(p.len, c0 + p.chunk) : c0;
  // a bounded-length group derives each chunk's start state from the bytes
  // before the chunk (exact); other groups start from the boundary guess
  const bool exact = warm_exact(gd, p.chunk);
  uint32_t start = gd.start_unanchored;
  if (active && i != 0 && !exact) start = p.guess[q];
  if (start >= gd.n_states) start = gd.start_unanchored;  // a guess never written
  uint32_t* ck = p.ckpt + q * p.nck;
  uint32_t cold_row = 0;
  uint32_t st = wstate(gi, start, H, (uint32_t)lane4, &cold_row);
  if (exact && active && i != 0) {
    // c0 >= chunk >= 4 * warm: the bytes [c0 - warm, c0) exist, 16-aligned
    for (uint32_t k = 0; k < gd.warm; k += 16) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(p.data + c0 - gd.warm + k));
      const uint32_t words[4] = {v.x, v.y, v.z, v.w};
      const uint32_t st0 = st;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const uint32_t b = __byte_perm(words[j >> 2], 0, 0x4440 + (j & 3));
        st = max(WS_STEP_FAST(img, st, wcol<kCls>(cls_s, b)), (uint32_t)lane4);
      }
      if (st == gi.trap) {  // careful pass; matches before the chunk are not its own
        st = st0;
        for (int j = 0; j < 16; ++j)
          trap_step<kCls>(img, gi, (words[j >> 2] >> (8 * (j & 3))) & 0xFFu, st, cold_row, H, (uint32_t)lane4,
                          cls_s, tab, C);
      }
    }
    start = wrow(gi, st, cold_row);
  }
  if (active) {
    p.used[q] = start;
    p.conv[q] = (uint32_t)c0;
    p.round[q] = 0;
  }
  // One 16-byte block: an optimistic pass over the image alone (a transition
  // that is not a plain hot one lands in the absorbing trap column, so the
  // block ends there), then, for a block that ended in the trap, a careful
  // pass from its start for match events and cold rows.
  auto block16 = [&](const uint32_t* words, uint64_t at) {
    const uint32_t st0 = st;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t b = __byte_perm(words[k >> 2], 0, 0x4440 + (k & 3));
      st = max(WS_STEP_FAST(img, st, wcol<kCls>(cls_s, b)), (uint32_t)lane4);
    }
    if (st == gi.trap) {
      st = st0;
      for (int k = 0; k < 16; ++k) {
        const uint32_t b = (words[k >> 2] >> (8 * (k & 3))) & 0xFFu;
        const uint32_t m_row = trap_step<kCls>(img, gi, b, st, cold_row, H, (uint32_t)lane4, cls_s, tab, C);
        if (m_row != 0xFFFFFFFFu) emit_event(p, (uint32_t)(at + k + 1), m_row, (uint32_t)q, 0);
      }
    }
  };
  const uint64_t nvec = (c1 - c0) / 16;
  // K steps for every lane of the warp (the stage protocol is warp-wide); a
  // lane walks its own steps [0, nvec)
  for (uint64_t k = 0; k < K; ++k) {
    uint4 cur = make_uint4(0, 0, 0, 0);
    if (wtma) {
      const uint32_t s = (uint32_t)(k & 1);
      bool ok = false;
      for (uint32_t it = 0; it < (1u << 22) && !ok; ++it) ok = mbar_try(&bar[s], (uint32_t)(k >> 1) & 1u);
      if (!__all_sync(0xFFFFFFFFu, ok)) {
        // (should not happen) record the time-out, let the copies this warp
        // issued land, and stop
        if (lane == 0) {
          atomicOr(&p.ctr[C_ERR], kErrTimeout);
          for (uint64_t j = k; j < K && j < k + 2; ++j)
            for (uint32_t it = 0; it < (1u << 22) && !mbar_try(&bar[j & 1], (uint32_t)(j >> 1) & 1u); ++it) {
            }
        }
        __syncwarp();
        return;
      }
      if (!own) cur = *reinterpret_cast<const uint4*>(stg + s * kWalkStage + lane * 16);
      __syncwarp();  // every lane has read stage s
      if (lane == 0 && k + 2 < K) {
        fence_proxy_async_smem();
        mbar_expect_tx(&bar[s], kWalkStage);
        tma_load_2d_hint(stg + s * kWalkStage, &rows, (int32_t)((k + 2) * 16), (int32_t)wfirst, &bar[s], in_policy);
      }
    }
    if (k >= nvec) continue;
    if (own) cur = __ldg(reinterpret_cast<const uint4*>(p.data + c0 + k * 16));
    const uint32_t words[4] = {cur.x, cur.y, cur.z, cur.w};
    block16(words, c0 + k * 16);
    const uint64_t done = (k + 1) * 16;
    if ((done % kCkpt) == 0) ck[done / kCkpt - 1] = wrow(gi, st, cold_row);
  }
  if (!active) return;
  for (uint64_t pos = c0 + nvec * 16; pos < c1; ++pos) {
    const uint32_t m_row =
        trap_step<kCls>(img, gi, __ldg(p.data + pos), st, cold_row, H, (uint32_t)lane4, cls_s, tab, C);
    if (m_row != 0xFFFFFFFFu) emit_event(p, (uint32_t)(pos + 1), m_row, (uint32_t)q, 0);
  }
  const uint32_t end_row = wrow(gi, st, cold_row);
  p.end[q] = end_row;
  p.spec[q] = end_row;
}

// One chunk of a fix-up round: re-walk from the predecessor's end state until
// the walk meets a recorded state of the speculative walk (from there on the
// two walks are identical), or to the end of the chunk.
__device__ void fix_chunk(const DevTables& t, const ScanPtrs& p, uint32_t g, uint64_t i, uint32_t tag,
                          unsigned long long* changed) {
  const uint64_t q = (uint64_t)g * p.n_chunks + i;
  volatile uint32_t* endv = p.end;
  const uint32_t S = endv[q - 1];
  if (S == p.used[q]) return;
  const GroupDev gd = t.groups[g];
  const uint32_t* tab = t.fwd + gd.fwd_off;
  const uint8_t* cls_g = t.cls + g * 256;
  const uint64_t c0 = i * p.chunk;
  const uint64_t c1 = min(p.len, c0 + p.chunk);
  const uint32_t* ck = p.ckpt + q * p.nck;
  uint32_t st = S;
  uint64_t pos = c0;
  bool converged = false;
  uint64_t conv = c1;
  for (uint64_t k = 0; pos < c1; ++k) {
    uint64_t stop = min(c1, c0 + (k + 1) * kCkpt);
    for (; pos < stop; ++pos) {
      uint32_t w = step_l2(st, __ldg(p.data + pos), cls_g, tab, gd.n_classes);
      st = w & F_MASK;
      if (w & F_MATCH) emit_event(p, (uint32_t)(pos + 1), st, (uint32_t)q, tag);
    }
    if (stop == c0 + (k + 1) * kCkpt && k < p.nck && st == ck[k]) {
      converged = true;
      conv = stop;
      break;
    }
  }
  p.used[q] = S;
  p.round[q] = tag;
  p.conv[q] = (uint32_t)conv;
  atomicAdd(&p.ctr[C_FIX], 1ull);
  atomicAdd(&p.ctr[C_REWALK], (unsigned long long)(conv - c0));
  uint32_t new_end = converged ? p.spec[q] : st;
  if (new_end != endv[q]) {
    endv[q] = new_end;
    atomicOr(changed, 1ull);
  }
}

// fix_chunk over the group's hot-row image in shared memory (the walk's own
// steps: a shared-memory lookup per byte, the class-indexed table in L2 only
// for cold rows), so that a re-walk is not a chain of L2 round trips.  The
// input is 16-byte aligned and chunks start at multiples of kCkpt.
template <bool kCls>
__device__ void fix_chunk_img(const DevTables& t, const ScanPtrs& p, const GroupDev& gd, const uint32_t* img,
                              const uint8_t* cls_s, uint32_t g, uint64_t i, uint32_t tag,
                              unsigned long long* changed, uint32_t lane4) {
  const uint64_t q = (uint64_t)g * p.n_chunks + i;
  volatile uint32_t* endv = p.end;
  const uint32_t S = endv[q - 1];
  if (S == p.used[q]) return;
  const uint32_t* tab = t.fwd + gd.fwd_off;
  const uint32_t C = gd.n_classes, H = gd.hot_rows;
  const uint64_t c0 = i * p.chunk;
  const uint64_t c1 = min(p.len, c0 + p.chunk);
  const uint32_t* ck = p.ckpt + q * p.nck;
  const WalkImg gi = walk_img(gd);
  uint32_t cold_row = 0;
  uint32_t st = wstate(gi, S, H, lane4, &cold_row);
  auto step = [&](uint32_t b, uint64_t at) {
    const uint32_t m_row = trap_step<kCls>(img, gi, b, st, cold_row, H, lane4, cls_s, tab, C);
    if (m_row != 0xFFFFFFFFu) emit_event(p, (uint32_t)(at + 1), m_row, (uint32_t)q, tag);
  };
  // 16-byte vectors, four in flight ahead of the walk; the state is compared
  // with the speculative walk's at every checkpoint
  const uint64_t nvec = (c1 - c0) / 16;
  auto load16 = [&](uint64_t k) -> uint4 {
    return k < nvec ? __ldg(reinterpret_cast<const uint4*>(p.data + c0 + k * 16)) : make_uint4(0, 0, 0, 0);
  };
  uint4 ring[4] = {load16(0), load16(1), load16(2), load16(3)};
  bool converged = false;
  uint64_t conv = c1;
  uint64_t k = 0;
  for (; k < nvec; ++k) {
    const uint32_t wd[4] = {ring[0].x, ring[0].y, ring[0].z, ring[0].w};
    ring[0] = ring[1];
    ring[1] = ring[2];
    ring[2] = ring[3];
    ring[3] = load16(k + 4);
#pragma unroll
    for (int j = 0; j < 16; ++j) step((wd[j >> 2] >> (8 * (j & 3))) & 0xFFu, c0 + k * 16 + j);
    const uint64_t done = (k + 1) * 16;
    if (done % kCkpt == 0 && done / kCkpt <= p.nck && wrow(gi, st, cold_row) == ck[done / kCkpt - 1]) {
      converged = true;
      conv = c0 + done;
      break;
    }
  }
  if (!converged)
    for (uint64_t pos = c0 + nvec * 16; pos < c1; ++pos) step(__ldg(p.data + pos), pos);
  p.used[q] = S;
  p.round[q] = tag;
  p.conv[q] = (uint32_t)conv;
  atomicAdd(&p.ctr[C_FIX], 1ull);
  atomicAdd(&p.ctr[C_REWALK], (unsigned long long)(conv - c0));
  const uint32_t new_end = converged ? p.spec[q] : wrow(gi, st, cold_row);
  if (new_end != endv[q]) {
    endv[q] = new_end;
    atomicOr(changed, 1ull);
  }
}

// One parallel fix-up round: blocks per group (blockIdx.x = group, as in the
// walk), each over a strided share of the group's chunks.  A block stages the
// hot-row image only when one of its chunks was walked from a start that
// differs from its predecessor's end.
template <bool kCls>
__global__ void __launch_bounds__(kWalkThreads, 1) dfa_fixup_kernel(DevTables t, ScanPtrs p, int round) {
  if (round > 0 && p.ctr[C_ROUND + round - 1] == 0) return;  // nothing changed last round
  extern __shared__ __align__(16) uint32_t smem[];
  const uint32_t g = blockIdx.x;
  const uint64_t first = 1 + (uint64_t)blockIdx.y * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.y * blockDim.x;
  bool need = false;
  for (uint64_t i = first; i < p.n_chunks && !need; i += stride) {
    const uint64_t q = (uint64_t)g * p.n_chunks + i;
    need = p.end[q - 1] != p.used[q];
  }
  if (!__syncthreads_or(need)) return;
  const GroupDev gd = t.groups[g];
  uint32_t* img = smem;
  uint8_t* cls_s = reinterpret_cast<uint8_t*>(smem) + kWalkImgBytes;
  if (!stage_hot(t, g, gd.hot_off, gd.hot_rows, img, cls_s, &p.ctr[C_ERR], gd.img_bytes)) return;
  const uint32_t lane4 = (threadIdx.x & 31) * 4;
  for (uint64_t i = first; i < p.n_chunks; i += stride)
    fix_chunk_img<kCls>(t, p, gd, img, cls_s, g, i, (uint32_t)round + 1, &p.ctr[C_ROUND + round], lane4);
}

// Final sweep, one thread per group, in chunk order: exact whatever happened
// in the parallel rounds (runs only if the last round still changed something).
__global__ void dfa_fixup_serial_kernel(DevTables t, ScanPtrs p) {
  if (p.ctr[C_ROUND + kFixRounds - 1] == 0) return;
  const uint32_t g = blockIdx.x;
  for (uint64_t i = 1; i < p.n_chunks; ++i)
    fix_chunk(t, p, g, i, (uint32_t)kFixRounds + 1, &p.ctr[C_ROUND + kFixRounds]);
}

// Profiled scans: how many chunk boundaries the guess the walk started from
// was the predecessor's true end state (the fix-up has run).
__device__ void count_guess_hits(const DevTables& t, const ScanPtrs& p) {
  const uint64_t per = p.n_chunks - 1, total = (uint64_t)p.count_guesses * per;
  unsigned long long hits = 0, seen = 0;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = (uint32_t)(x / per);
    const uint64_t q = (uint64_t)g * p.n_chunks + x % per + 1;
    // the start the walk took: the derived state of an exact group (the
    // fix-up leaves it untouched when it held), else the boundary guess
    const GroupDev& gd = t.groups[g];
    uint32_t guess = warm_exact(gd, p.chunk) ? p.used[q] : p.guess[q];
    if (guess >= gd.n_states) guess = gd.start_unanchored;
    hits += guess == p.end[q - 1];
    seen += 1;
  }
  for (int o = 16; o > 0; o >>= 1) {
    hits += __shfl_down_sync(0xFFFFFFFFu, hits, o);
    seen += __shfl_down_sync(0xFFFFFFFFu, seen, o);
  }
  if ((threadIdx.x & 31) == 0 && seen) {
    atomicAdd(&p.ctr[C_HITS], hits);
    atomicAdd(&p.ctr[C_GUESSES], seen);
  }
}

// Valid match events -> reverse walk -> K candidates (and, in profiled
// speculative scans, the guess count).
__global__ void __launch_bounds__(256) dfa_reverse_kernel(DevTables t, ScanPtrs p) {
  if (p.count_guesses && p.n_chunks > 1) count_guess_hits(t, p);
  unsigned long long n = p.ctr[C_EV];
  if (n > p.ev_cap) n = p.ev_cap;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    Event ev = p.ev[k];
    uint32_t conv = p.conv[ev.q];
    bool valid = (ev.tag == 0) ? (ev.e > conv) : (ev.tag == p.round[ev.q] && ev.e <= conv);
    if (!valid) continue;
    const uint32_t g = (uint32_t)(ev.q / p.n_chunks);
    const GroupDev gd = t.groups[g];
    const uint8_t* cm = t.cls + g * 256;
    const uint32_t* tab = t.rev + gd.rev_off;
    const uint32_t* rmp = t.rmptr + gd.rmptr_off;
    const uint32_t C = gd.n_classes;
    uint32_t st = gd.rev_start;
    const uint64_t lo = p.n_items ? item_start_of(p.item_end, p.n_items, ev.e - 1) : 0;
    for (uint64_t pos = ev.e; pos > lo; --pos) {
      uint32_t w = __ldg(tab + st * C + __ldg(cm + __ldg(p.data + pos - 1)));
      if (w & F_DEAD) break;
      st = w & F_MASK;
      // (pos - 1, g, st) fixes the rest of the walk: stop where another walk
      // has been (it reports these starts), else leave a mark first; marks
      // are kept at every eighth position only (the same positions for every
      // walk), which keeps a long run of match ends linear at an eighth of
      // the mark traffic
      if (p.rmark && ((pos - 1) & 7) == 0) {
        const uint32_t at = (uint32_t)(pos - 1);
        const unsigned long long key =
            ((unsigned long long)at << 32) | ((unsigned long long)g << kRmarkStateBits) | st;
        // the state is hashed too: walks in different states at the same
        // position (the two parities of (ab)+) must not evict each other
        unsigned long long* slot =
            p.rmark + ((at * 0x9E3779B1u ^ g * 0x7FEB352Du ^ st * 0x2C1B3C6Du) >> (32 - kRmarkBits));
        if (*(volatile unsigned long long*)slot == key) break;
        *slot = key;
      }
      if (w & F_MATCH) {
        for (uint32_t j = __ldg(rmp + st); j < __ldg(rmp + st + 1); ++j)
          emit_k(p, __ldg(t.rmlist + j), (uint32_t)(pos - 1), ev.e);
      }
    }
  }
}

// ---------------------------------------------------------------- resolution
__global__ void k_scan_kernel(ScanPtrs p, uint32_t n_regex) {
  // single-block exclusive scan (blockDim.x a multiple of 32, at most 1024):
  // each thread sums a run of regexes, the runs are scanned across the block
  // with warp shuffles, then each thread writes its run's offsets
  __shared__ uint32_t wsum[32];
  const uint32_t per = (n_regex + blockDim.x - 1) / blockDim.x;
  const uint32_t a = threadIdx.x * per, b = min(n_regex, a + per);
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t sum = 0;
  for (uint32_t r = a; r < b; ++r) sum += p.count[r];
  uint32_t incl = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t v = lane < nw ? wsum[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, d);
      if (lane >= (uint32_t)d) v += y;
    }
    wsum[lane] = v;  // inclusive sums of the warps' runs
  }
  __syncthreads();
  if (threadIdx.x == 0) p.offs[n_regex] = wsum[nw - 1];
  uint32_t acc = incl - sum + (warp ? wsum[warp - 1] : 0u);
  for (uint32_t r = a; r < b; ++r) { p.offs[r] = acc; p.cursor[r] = acc; acc += p.count[r]; }
}

__global__ void k_scatter_kernel(ScanPtrs p) {
  unsigned long long n = min(p.ctr[C_K], (unsigned long long)p.k_cap);
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    KCand c = p.k[k];
    uint32_t slot = atomicAdd(&p.cursor[c.r], 1u);
    p.starts[slot] = c.s;
  }
}

// Block-wide bitonic sort of buf[0, m) in shared memory (m a power of two).
__device__ void bitonic_smem(uint32_t* buf, uint32_t m) {
  for (uint32_t size = 2; size <= m; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) {
        uint32_t j = k ^ stride;
        if (j > k) {
          bool up = (k & size) == 0;
          uint32_t x = buf[k], y = buf[j];
          if ((x > y) == up) { buf[k] = y; buf[j] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// Sorts src[0, n), n <= 4096, in place through shared memory.
__device__ void sort_tile(uint32_t* buf, uint32_t* src, uint32_t n) {
  uint32_t m = 1;
  while (m < n) m <<= 1;
  for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) buf[k] = (k < n) ? src[k] : 0xFFFFFFFFu;
  __syncthreads();
  bitonic_smem(buf, m);
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) src[k] = buf[k];
  __syncthreads();
}

// Number of elements taken from A among the first `diag` of the merge of
// sorted A and B (ties from A first).
__device__ uint32_t merge_path(const uint32_t* A, uint32_t na, const uint32_t* B, uint32_t nb, uint32_t diag) {
  uint32_t lo = diag > nb ? diag - nb : 0, hi = min(diag, na);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (A[mid] <= B[diag - 1 - mid]) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Sorts each regex's starts ascending: a bitonic sort in shared memory for
// segments of up to 4096; beyond that, sorted 4096-tiles merged pairwise in
// global memory (merge-path split of each merge across the block), with the
// lfend array -- written only after this kernel -- as the other buffer.
__global__ void __launch_bounds__(512) k_sort_kernel(ScanPtrs p, uint32_t n_regex) {
  __shared__ uint32_t buf[4096];
  for (uint32_t r = blockIdx.x; r < n_regex; r += gridDim.x) {
    const uint32_t a = p.offs[r], n = p.offs[r + 1] - a;
    if (n <= 1) continue;
    uint32_t* src = p.starts + a;
    if (n <= 4096) {
      sort_tile(buf, src, n);
      continue;
    }
    for (uint32_t t0 = 0; t0 < n; t0 += 4096) sort_tile(buf, src + t0, min(4096u, n - t0));
    uint32_t* dst = p.lfend + a;
    for (uint32_t w = 4096; w < n; w <<= 1) {
      for (uint32_t lo = 0; lo < n; lo += 2 * w) {
        const uint32_t mid = min(lo + w, n), hi = min(lo + 2 * w, n);
        const uint32_t* A = src + lo;
        const uint32_t* B = src + mid;
        const uint32_t na = mid - lo, nb = hi - mid, total = hi - lo;
        const uint32_t per = (total + blockDim.x - 1) / blockDim.x;
        const uint32_t d0 = min(total, threadIdx.x * per), d1 = min(total, d0 + per);
        uint32_t i = merge_path(A, na, B, nb, d0), j = d0 - i;
        for (uint32_t d = d0; d < d1; ++d) dst[lo + d] = (j >= nb || (i < na && A[i] <= B[j])) ? A[i++] : B[j++];
      }
      __syncthreads();
      uint32_t* t = src;
      src = dst;
      dst = t;
    }
    if (src != p.starts + a) {
      for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) p.starts[a + k] = src[k];
      __syncthreads();
    }
  }
}

// Leftmost-first end of a match of regex r from start s: the walk of the
// regex's priority DFA from s, remembering the last match position, until the
// DFA dies or the item or input ends.  kLfNone when no match starts at s;
// kLfLong when the walk was cut off after `cap` bytes.
__device__ uint32_t lf_walk(const DevTables& t, const ScanPtrs& p, uint32_t r, uint32_t s, uint64_t cap) {
  const uint4 info = t.lfinfo[r];
  const uint8_t* cm = t.cls + info.z * 256;
  const uint32_t* tab = t.lf + info.x;
  uint32_t st = info.y;
  int64_t last = -1;
  const uint64_t stop = p.n_items ? min(p.len, (uint64_t)item_end_of(p.item_end, p.n_items, s)) : p.len;
  const uint32_t* x = t.lfx + 8 * (size_t)r;
  if (__ldg(x)) {
    // context DFA (build_context_lf_dfa): start row by the byte before s, a
    // match flag on the byte at pos ends a match at pos, the end step after
    // the last byte of the input or item
    const uint64_t lo = p.n_items ? item_start_of(p.item_end, p.n_items, s) : 0;
    st = __ldg(x + 1 + (s == lo ? CTX_BEGIN : ctx_of(__ldg(p.data + s - 1))));
    for (uint64_t pos = s; pos < stop; ++pos) {
      if (pos - s == cap) return kLfLong;
      const uint32_t w = __ldg(tab + st * info.w + __ldg(cm + __ldg(p.data + pos)));
      if (w & F_MATCH) last = (int64_t)pos;
      if (w & F_DEAD) return last < 0 ? kLfNone : (uint32_t)last;
      st = w & F_MASK;
    }
    if (__ldg(t.lf + __ldg(x + 5) + st)) last = (int64_t)stop;
    return last < 0 ? kLfNone : (uint32_t)last;
  }
  for (uint64_t pos = s; pos < stop; ++pos) {
    if (pos - s == cap) return kLfLong;
    uint32_t w = __ldg(tab + st * info.w + __ldg(cm + __ldg(p.data + pos)));
    if (w & F_DEAD) break;
    st = w & F_MASK;
    if (w & F_MATCH) last = (int64_t)pos + 1;
  }
  return last < 0 ? kLfNone : (uint32_t)last;
}

// Leftmost-first end of every distinct candidate start (in parallel), each
// walk cut off after kLfCap bytes.
// The regexes' candidate offsets are staged in shared memory when they fit
// (kLfOffsShared regexes), so that finding a candidate's regex is a binary
// search in shared memory rather than a chain of dependent global loads.
constexpr uint32_t kLfOffsShared = 8192;

__global__ void k_lf_kernel(DevTables t, ScanPtrs p, uint32_t n_regex) {
  extern __shared__ uint32_t offs_s[];
  const bool staged = n_regex < kLfOffsShared;
  if (staged) {
    for (uint32_t r = threadIdx.x; r <= n_regex; r += blockDim.x) offs_s[r] = p.offs[r];
    __syncthreads();
  }
  const uint32_t* offs = staged ? offs_s : p.offs;
  const uint32_t total = offs[n_regex];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
    // owning regex: binary search in offs
    uint32_t lo = 0, hi = n_regex;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (offs[mid] <= j) lo = mid; else hi = mid;
    }
    const uint32_t r = lo;
    const uint32_t s = p.starts[j];
    if (j > offs[r] && p.starts[j - 1] == s) { p.lfend[j] = kLfNone; continue; }  // duplicate
    p.lfend[j] = lf_walk(t, p, r, s, kLfCap);
  }
}

// find_iter chain per regex: leftmost candidate start with its leftmost-first
// end, then the next candidate at or after that end.
// One warp per regex: the warp loads 32 sorted candidates at a time and picks
// the chain's next match among them with a ballot (the first candidate whose
// start is at or after the current end), so the serial part is one ballot per
// reported match.
__global__ void k_chain_kernel(DevTables t, ScanPtrs p) {
  const uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (r >= t.n_regex) return;  // whole warps exit together
  const uint32_t a = p.offs[r], b = p.offs[r + 1];
  const uint32_t pid = t.pid[r];
  // stream scans: resume at the regex's cursor, decide only starts before the
  // frontier (both in stream offsets; the buffer starts at p.base <= cursor)
  uint64_t last_end = (p.cursor64 && p.cursor64[r] > p.base) ? p.cursor64[r] - p.base : 0;
  const uint64_t limit = p.cursor64 ? p.frontier - p.base : ~0ull;
  // each window's candidates are loaded while the previous window is decided
  uint32_t e_nx = a + lane < b ? p.lfend[a + lane] : kLfNone;
  uint32_t s_nx = a + lane < b ? p.starts[a + lane] : 0xFFFFFFFFu;
  for (uint32_t j0 = a; j0 < b; j0 += 32) {
    const uint32_t j = j0 + lane;
    const bool in = j < b;
    uint32_t e = e_nx;
    const uint32_t s = s_nx;
    e_nx = j + 32 < b ? p.lfend[j + 32] : kLfNone;
    s_nx = j + 32 < b ? p.starts[j + 32] : 0xFFFFFFFFu;
    const bool past = in && (uint64_t)s >= limit;
    bool picked = false;
    while (true) {
      const bool ok = in && e != kLfNone && (uint64_t)s >= last_end && !past;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, ok);
      if (!m) break;
      const int k = __ffs(m) - 1;
      uint32_t ek = __shfl_sync(0xFFFFFFFFu, e, k);
      if (ek == kLfLong) {  // the parallel walk was cut off: finish it here
        if ((int)lane == k) e = lf_walk(t, p, r, s, ~0ull);
        ek = __shfl_sync(0xFFFFFFFFu, e, k);
        if (ek == kLfNone) continue;  // no match from that start after all
      }
      picked |= (int)lane == k;
      last_end = ek;
    }
    // one output reservation per window of 32 candidates
    const unsigned pm = __ballot_sync(0xFFFFFFFFu, picked);
    if (pm) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(p.out_counter, (unsigned long long)__popc(pm));
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (picked) {
        const unsigned long long idx = base + __popc(pm & ((1u << lane) - 1u));
        if (idx < p.out_cap) p.out[idx] = ws_match{pid, s, e};
      }
    }
    if (__any_sync(0xFFFFFFFFu, past)) break;  // sorted: every later start is past too
  }
  if (p.cursor64 && lane == 0) p.cursor64[r] = max(p.base + last_end, p.frontier);
}

// Copies K candidates into a ws_match buffer (diagnostics).
__global__ void k_export_kernel(DevTables t, ScanPtrs p, ws_match* out, uint64_t cap) {
  unsigned long long n = min(p.ctr[C_K], (unsigned long long)p.k_cap);
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n && k < cap;
       k += (uint64_t)gridDim.x * blockDim.x) {
    KCand c = p.k[k];
    out[k] = ws_match{t.pid[c.r], c.s, c.e};
  }
}

// After a candidate or event buffer overflow the scan's match count is not
// known: the count becomes kCountUnknown (larger than any capacity), and the
// capacities the scan would have needed are recorded in `need` (host-mapped
// memory of the matcher, read by the next launch), so the same scan run again
// fits.  One thread, after every other kernel of the scan.
__global__ void finalize_kernel(ScanPtrs p, unsigned long long* need) {
  if (p.ctr[C_ERR] & kErrTimeout) {
    *p.out_counter = kCountTimeout;
  } else if (p.ctr[C_ERR]) {
    *p.out_counter = kCountUnknown;
    if (need) {
      volatile unsigned long long* v = need;
      if (p.ctr[C_K] > v[0]) v[0] = p.ctr[C_K];
      if (p.ctr[C_EV] > v[1]) v[1] = p.ctr[C_EV];
    }
  }
}

// Counts the chunk boundaries whose guess (the proposer's, or the unanchored
// start) was the true state: the predecessor's end state after the fix-up.
__global__ void fill_guess_kernel(DevTables t, ScanPtrs p) {
  const uint32_t g = blockIdx.y;
  const uint32_t st = t.groups[g].start_unanchored;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n_chunks; i += (uint64_t)gridDim.x * blockDim.x)
    p.guess[(uint64_t)g * p.n_chunks + i] = st;
}

DevTables dev_tables(const RegexPlan& P) {
  DevTables t;
  t.groups = P.d_groups.as<GroupDev>();
  t.fwd = P.d_fwd.as<uint32_t>();
  t.hot = P.d_hot.as<uint32_t>();
  t.rev = P.d_rev.as<uint32_t>();
  t.lf = P.d_lf.as<uint32_t>();
  t.cls = P.d_cls.as<uint8_t>();
  t.mptr = P.d_mptr.as<uint32_t>();
  t.mlist = P.d_mlist.as<uint32_t>();
  t.rmptr = P.d_rmptr.as<uint32_t>();
  t.rmlist = P.d_rmlist.as<uint32_t>();
  t.lfinfo = P.d_lfinfo.as<uint4>();
  t.lfx = P.d_lfx.as<uint32_t>();
  t.pid = P.d_pid.as<uint32_t>();
  t.n_groups = P.n_groups;
  t.n_regex = P.n_regex;
  t.n_spec = P.n_spec;
  return t;
}


uint32_t max_rows(const RegexPlan& P, bool anchored) {
  uint32_t m = 0;
  for (const auto& g : P.groups) m = std::max(m, anchored ? g.ahot_rows : g.hot_rows);
  return m;
}

template <class K>
void set_smem(K kernel, size_t bytes, const char* what) {
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), what);
}

// cuTensorMapEncodeTiled, from the driver through the runtime (no link
// dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// The walk's view of the input: n_full rows of `chunk` bytes (16-byte
// aligned base, chunk a multiple of 256), boxes of 16 bytes x 32 rows.
void encode_chunk_rows(CUtensorMap* map, const uint8_t* data, uint64_t chunk, uint64_t n_full) {
  auto fn = tensor_map_encoder();
  if (!fn) raise(WS_ERR_DEVICE, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[2] = {chunk, n_full};
  const cuuint64_t strides[1] = {chunk};
  const cuuint32_t box[2] = {16, 32};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(data), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) raise(WS_ERR_DEVICE, "cuTensorMapEncodeTiled failed for the walk's input view");
}

}  // namespace

bool regex_all_exact(const RegexPlan& P, uint64_t chunk) {
  return P.n_spec > 0 && P.n_warm == P.n_spec && 4 * (uint64_t)P.max_warm <= chunk;
}

namespace {

// Runs the candidate phase (plain or speculative) and leaves K in scratch.
uint32_t candidates_phase(RegexPlan& P, const DevTables& t, const ScanPtrs& p, uint32_t mode, cudaStream_t st,
                          int sm_count, cudaEvent_t* ev) {
  uint32_t launches = 0;
  auto mark = [&](int k) { if (ev) check_cuda(cudaEventRecord(ev[k], st), "event"); };
  // context groups: one anchored walk per start in either mode
  auto context_groups = [&]() {
    const uint32_t nc = P.n_groups - P.n_spec;
    if (!nc) return;
    const uint64_t want = (p.len + 255) / 256;
    const uint64_t per_group = std::max<uint64_t>(1, (uint64_t)sm_count * 8 / nc);
    dim3 grid((unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, per_group)), nc);
    dfa_context_kernel<<<grid, 256, 0, st>>>(t, p);
    check_cuda(cudaGetLastError(), "dfa_context_kernel");
    launches++;
  };
  if (mode == WS_REGEX_PLAIN) {
    mark(1);
    if (P.n_spec) {
      size_t smem = hot_smem_bytes(max_rows(P, true));
      set_smem(dfa_plain_kernel, smem, "smem(plain)");
      uint64_t per_group = std::max<uint64_t>(1, (uint64_t)sm_count / P.n_spec);
      uint64_t want = (p.len + kWalkThreads - 1) / kWalkThreads;
      dim3 grid((unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, per_group * 2)), P.n_spec);
      dfa_plain_kernel<<<grid, kWalkThreads, smem, st>>>(t, p);
      check_cuda(cudaGetLastError(), "dfa_plain_kernel");
      launches++;
    }
    context_groups();
    mark(2);
    mark(3);
    mark(4);
    return launches;
  }
  if (!P.n_spec) {
    mark(1);
    context_groups();
    mark(2);
    mark(3);
    mark(4);
    return launches;
  }
  dim3 cgrid(P.n_spec, (unsigned)((p.n_chunks + kWalkThreads - 1) / kWalkThreads));
  // the walk ignores the guesses of groups with exact chunk starts
  if (P.proposer && P.use_proposer && !regex_all_exact(P, p.chunk)) {
    launches += proposer_predict(*P.proposer, p.data, p.len, p.chunk, p.n_chunks, p.guess, st);
  } else {
    fill_guess_kernel<<<dim3(std::min<unsigned>((unsigned)((p.n_chunks + 255) / 256), 1024), P.n_spec), 256, 0, st>>>(t, p);
    check_cuda(cudaGetLastError(), "fill_guess_kernel");
    launches++;
  }
  mark(1);
  // the input as a 2-D tensor of its full chunks (rows of p.chunk bytes)
  const uint64_t n_full = p.len / p.chunk;
  CUtensorMap rows;
  std::memset(&rows, 0, sizeof(rows));
  if (n_full) encode_chunk_rows(&rows, p.data, p.chunk, n_full);
  if (P.class_image) {
    set_smem(dfa_walk_kernel<true>, kWalkSmem, "smem(walk)");
    dfa_walk_kernel<true><<<cgrid, kWalkThreads, kWalkSmem, st>>>(t, p, rows, n_full);
  } else {
    set_smem(dfa_walk_kernel<false>, kWalkSmem, "smem(walk)");
    dfa_walk_kernel<false><<<cgrid, kWalkThreads, kWalkSmem, st>>>(t, p, rows, n_full);
  }
  check_cuda(cudaGetLastError(), "dfa_walk_kernel");
  launches++;
  mark(2);
  // one wave of fix-up blocks (one per SM, the walk's shared memory)
  const uint64_t fper = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count / P.n_spec,
                                                                  (p.n_chunks + kWalkThreads - 1) / kWalkThreads));
  dim3 fgrid(P.n_spec, (unsigned)fper);
  auto fixup = P.class_image ? dfa_fixup_kernel<true> : dfa_fixup_kernel<false>;
  set_smem(fixup, kFixSmem, "smem(fixup)");
  for (int r = 0; r < kFixRounds; ++r) {
    fixup<<<fgrid, kWalkThreads, kFixSmem, st>>>(t, p, r);
    check_cuda(cudaGetLastError(), "dfa_fixup_kernel");
    launches++;
  }
  dfa_fixup_serial_kernel<<<P.n_spec, 1, 0, st>>>(t, p);
  check_cuda(cudaGetLastError(), "dfa_fixup_serial_kernel");
  launches++;
  mark(3);
  dfa_reverse_kernel<<<sm_count * 8, 256, 0, st>>>(t, p);
  check_cuda(cudaGetLastError(), "dfa_reverse_kernel");
  launches++;
  context_groups();
  mark(4);
  return launches;
}

}  // namespace

// ------------------------------------------------------------------- host plan
void ProposerDeleter::operator()(Proposer* p) const { proposer_destroy(p); }

namespace {

struct GroupBuild {
  std::vector<uint32_t> regexes;
  ByteClasses cls;
  Dfa fwd, rev;
  std::vector<Dfa> lf;
  uint32_t n_hot_u = 0, n_hot_a = 0;
  bool context = false;  // a context group (patterns with look-around assertions)
};

// Byte distribution assumed when ranking states: text-like input (printable
// ASCII and common whitespace most likely, every byte possible).
std::vector<double> class_probabilities(const ByteClasses& bc) {
  std::vector<double> pb(256, 0.02 / 156);
  for (int b = 0x20; b < 0x7F; ++b) pb[b] = 0.97 / 95;
  pb['\n'] = pb['\t'] = pb['\r'] = 0.01 / 3;
  std::vector<double> pc((size_t)bc.count, 0);
  for (int b = 0; b < 256; ++b) pc[bc.map[b]] += pb[b];
  return pc;
}

// Ranks states by estimated visit frequency: the unanchored part by the
// average of the first 64 iterates of the walk's state distribution from the
// unanchored start, the anchored part by the expected number of visits of a
// walk from the anchored start.  New order: hot unanchored rows, hot anchored
// rows, the remaining unanchored rows, the remaining anchored rows, dead.
void rank_states(GroupBuild& gb) {
  Dfa& d = gb.fwd;
  const int n = d.n_states, C = d.n_classes;
  auto pc = class_probabilities(gb.cls);
  auto propagate = [&](const std::vector<double>& cur, std::vector<double>& nxt) {
    std::fill(nxt.begin(), nxt.end(), 0.0);
    for (int s = 0; s < n; ++s) {
      if (cur[(size_t)s] == 0) continue;
      for (int c = 0; c < C; ++c) {
        uint32_t w = d.trans[(size_t)s * C + c];
        if (w & DFA_FLAG_DEAD) continue;
        nxt[w & DFA_MASK_STATE] += cur[(size_t)s] * pc[(size_t)c];
      }
    }
  };
  std::vector<double> pu((size_t)n, 0), pa((size_t)n, 0), cur((size_t)n, 0), nxt((size_t)n, 0);
  cur[d.start_unanchored] = 1;
  for (int it = 0; it < 64; ++it) {
    for (int s = 0; s < n; ++s) pu[(size_t)s] += cur[(size_t)s];
    propagate(cur, nxt);
    cur.swap(nxt);
  }
  std::fill(cur.begin(), cur.end(), 0.0);
  cur[d.start_anchored] = 1;
  for (int it = 0; it < 64; ++it) {
    for (int s = 0; s < n; ++s) pa[(size_t)s] += cur[(size_t)s];
    propagate(cur, nxt);
    cur.swap(nxt);
  }
  // which part each state belongs to: reachable from the unanchored start?
  std::vector<uint8_t> in_u((size_t)n, 0);
  std::deque<uint32_t> dq{d.start_unanchored};
  in_u[d.start_unanchored] = 1;
  while (!dq.empty()) {
    uint32_t s = dq.front();
    dq.pop_front();
    for (int c = 0; c < C; ++c) {
      uint32_t t = d.trans[(size_t)s * C + c] & DFA_MASK_STATE;
      if (!in_u[t]) { in_u[t] = 1; dq.push_back(t); }
    }
  }
  std::vector<uint32_t> us, as;
  for (int s = 1; s < n; ++s) (in_u[(size_t)s] ? us : as).push_back((uint32_t)s);
  std::stable_sort(us.begin(), us.end(), [&](uint32_t a, uint32_t b) { return pu[a] > pu[b]; });
  std::stable_sort(as.begin(), as.end(), [&](uint32_t a, uint32_t b) { return pa[a] > pa[b]; });
  gb.n_hot_u = (uint32_t)std::min<size_t>(us.size(), std::max(kHotRows, walk_hot_rows((uint32_t)C)));
  gb.n_hot_a = (uint32_t)std::min<size_t>(as.size(), kHotRows);
  std::vector<uint32_t> order;
  order.insert(order.end(), us.begin(), us.begin() + gb.n_hot_u);
  order.insert(order.end(), as.begin(), as.begin() + gb.n_hot_a);
  order.insert(order.end(), us.begin() + gb.n_hot_u, us.end());
  order.insert(order.end(), as.begin() + gb.n_hot_a, as.end());
  order.push_back(0);  // dead
  renumber_dfa(d, order);
}

bool try_group(const std::vector<ReTree>& trees, const std::vector<uint32_t>& members, int max_states,
               GroupBuild& out) {
  std::vector<const ReTree*> tp;
  for (uint32_t r : members) tp.push_back(&trees[r]);
  Nfa fn = build_nfa(tp, false);
  ByteClasses bc = compute_classes({&fn});
  Dfa fwd = build_all_dfa(fn, bc, true, max_states);
  if (fwd.too_big) return false;
  Nfa rn = build_nfa(tp, true);
  Dfa rev = build_all_dfa(rn, bc, false, 1 << 22);
  if (rev.too_big) return false;
  out.regexes = members;
  out.cls = bc;
  out.fwd = std::move(fwd);
  out.rev = std::move(rev);
  rank_states(out);
  out.lf.clear();
  for (uint32_t r : members) {
    Nfa one = build_nfa({&trees[r]}, false);
    Dfa lf = build_leftmost_first_dfa(one, bc, 1 << 20);
    if (lf.too_big) throw CompileError("leftmost-first DFA too large for regex " + std::to_string(r));
    out.lf.push_back(std::move(lf));
  }
  return true;
}

// A group of patterns with look-around assertions: the context DFA of the
// group and a context leftmost-first DFA per pattern; no unanchored walk, no
// reverse DFA, no hot rows.
bool try_context_group(const std::vector<ReTree>& trees, const std::vector<uint32_t>& members, int max_states,
                       GroupBuild& out) {
  std::vector<const ReTree*> tp;
  for (uint32_t r : members) tp.push_back(&trees[r]);
  Nfa fn = build_nfa(tp, false);
  ByteClasses bc = compute_classes({&fn});
  Dfa fwd = build_context_all_dfa(fn, bc, max_states);
  if (fwd.too_big) return false;
  out.regexes = members;
  out.cls = bc;
  out.fwd = std::move(fwd);
  out.rev = Dfa();
  out.context = true;
  out.n_hot_u = out.n_hot_a = 0;
  out.lf.clear();
  for (uint32_t r : members) {
    Nfa one = build_nfa({&trees[r]}, false);
    Dfa lf = build_context_lf_dfa(one, bc, 1 << 20);
    if (lf.too_big) throw CompileError("leftmost-first DFA too large for regex " + std::to_string(r));
    out.lf.push_back(std::move(lf));
  }
  return true;
}

uint32_t append_trans(const Dfa& d, std::vector<uint32_t>& dst) {
  size_t base = dst.size();
  dst.insert(dst.end(), d.trans.begin(), d.trans.end());
  return (uint32_t)base;
}

// Builds the forward tables of every group from P.fdfa (class-indexed words,
// 16-bit byte-indexed hot rows, match lists) and uploads them.
void layout_forward(RegexPlan& P) {
  P.fwd.clear(); P.hot.clear(); P.mptr.clear(); P.mlist.clear();
  P.total_states = 0;
  P.max_classes = 0;
  // small alphabets (every speculative group with at most
  // kClassImageMaxClasses classes) index the walk's image by class
  P.class_image = P.n_spec > 0;
  for (uint32_t g = 0; g < P.n_spec; ++g) P.class_image &= (uint32_t)P.fcls[g].count <= kClassImageMaxClasses;
  for (uint32_t g = 0; g < P.n_groups; ++g) {
    const Dfa& d = P.fdfa[g];
    const ByteClasses& bc = P.fcls[g];
    GroupDev& gd = P.groups[g];
    const uint32_t C = (uint32_t)bc.count;
    gd.n_states = (uint32_t)d.n_states;
    gd.n_classes = C;
    gd.fwd_off = append_trans(d, P.fwd);
    gd.start_anchored = d.start_anchored;
    gd.start_unanchored = d.start_unanchored;
    // slow words carry the next row in 27 bits; larger DFAs walk through L2 only
    const bool fits = d.n_states < (1 << 27);
    // The anchored image of the plain kernel: byte-indexed, slow words for
    // transitions that are not into a hot row without a match.
    auto image = [&](uint32_t first, uint32_t rows) {
      uint32_t off = (uint32_t)P.hot.size();
      if (!rows) return off;
      P.hot.resize(P.hot.size() + kImgWords, S_SLOW | S_TRAP);
      uint32_t* img = P.hot.data() + off;
      auto entry = [&](uint32_t w) -> uint32_t {
        uint32_t n = w & DFA_MASK_STATE, nl = n - first;
        bool match = w & DFA_FLAG_MATCH, dead = w & DFA_FLAG_DEAD, hot = nl < rows;
        if (!match && !dead && hot) return nl == 0 ? 0u : slot_word(nl) * 4;
        return S_SLOW | (match ? S_MATCH : 0u) | (hot ? 0u : S_COLD) | (dead ? S_DEAD : 0u) | n;
      };
      for (uint32_t r = 0; r < rows; ++r)
        for (int b = 0; b < 256; ++b) {
          uint32_t e = entry(d.trans[(size_t)(first + r) * C + bc.map[b]]);
          if (r == 0) for (int l = 0; l < 32; ++l) img[b * 32 + l] = e;
          else img[slot_word(r) + b * 32] = e;
        }
      return off;
    };
    // The walk's image of the unanchored hot rows (the walk and the fix-up):
    // 32-row blocks of `cols` entries per row (256 by byte, or C by class),
    // as many blocks as fit in kWalkImgBytes; every transition that is not
    // into a hot row without a match is the trap column's offset (an
    // absorbing column: its entries are its own offset).
    auto walk_image = [&](uint32_t rows, uint32_t cols) {
      const uint32_t blk = cols * 32, nblk = (kWalkImgBytes / 4) / blk, trap = blk * 4;
      uint32_t off = (uint32_t)P.hot.size();
      gd.img_cols = cols;
      gd.img_bytes = nblk * blk * 4;
      if (!rows) return off;
      P.hot.resize(P.hot.size() + (size_t)nblk * blk, trap);
      uint32_t* img = P.hot.data() + off;
      auto slot = [&](uint32_t r) { return (1 + r / 32) * blk + r % 32; };
      for (uint32_t r = 0; r < rows; ++r)
        for (uint32_t c = 0; c < cols; ++c) {
          const uint32_t w = d.trans[(size_t)r * C + (cols == 256 ? bc.map[c] : c)];
          const uint32_t n = w & DFA_MASK_STATE;
          const bool fast = !(w & (DFA_FLAG_MATCH | DFA_FLAG_DEAD)) && n < rows;
          const uint32_t e = fast ? (n == 0 ? 0u : slot(n) * 4) : trap;
          if (r == 0) for (uint32_t l = 0; l < 32; ++l) img[c * 32 + l] = e;
          else img[slot(r) + c * 32] = e;
        }
      return off;
    };
    const bool spec = g < P.n_spec;
    const uint32_t cols = P.class_image ? C : 256;
    const uint32_t walk_rows = 32 * ((kWalkImgBytes / 4) / (cols * 32) - 1);
    gd.hot_rows = fits && spec ? std::min(P.nhot_u[g], walk_rows) : 0;
    gd.hot_off = walk_image(gd.hot_rows, cols);
    gd.ahot_base = P.nhot_u[g];
    gd.ahot_rows = fits && spec ? std::min(P.nhot_a[g], kHotRows) : 0;
    gd.ahot_off = image(P.nhot_u[g], gd.ahot_rows);
    gd.mptr_off = (uint32_t)P.mptr.size();
    // one list per state, or per (state, right context) in a context group
    const size_t n_lists = d.match_ptr.size() - 1;
    for (size_t s = 0; s < n_lists; ++s) {
      P.mptr.push_back((uint32_t)P.mlist.size());
      for (uint32_t j = d.match_ptr[s]; j < d.match_ptr[s + 1]; ++j) P.mlist.push_back(P.gregex[g][d.match_list[j]]);
    }
    P.mptr.push_back((uint32_t)P.mlist.size());
    gd.context = g >= P.n_spec ? 1u : 0u;
    for (int k = 0; k < 4; ++k) gd.cstart[k] = d.ctx_start[k];
    P.total_states += gd.n_states;
    P.max_classes = std::max(P.max_classes, C);
  }
  if (P.fwd.size() > DFA_MASK_STATE) raise(WS_ERR_COMPILE, "regex tables exceed 2^30 words");
  P.d_groups.upload(P.groups.data(), P.groups.size() * sizeof(GroupDev));
  P.d_fwd.upload(P.fwd.data(), P.fwd.size() * 4);
  // sets whose groups all carry context have no hot image: the buffers still exist
  if (P.hot.size() < 4) P.hot.resize(4, 0);
  if (P.mlist.empty()) P.mlist.push_back(0);
  P.d_hot.upload(P.hot.data(), P.hot.size() * 4);
  P.d_mptr.upload(P.mptr.data(), P.mptr.size() * 4);
  P.d_mlist.upload(P.mlist.data(), P.mlist.size() * 4);
}

void build_groups(const std::vector<ReTree>& trees, const std::vector<uint32_t>& members, int max_states,
                  std::vector<GroupBuild>& out, bool context) {
  GroupBuild gb;
  if (context ? try_context_group(trees, members, max_states, gb) : try_group(trees, members, max_states, gb)) {
    out.push_back(std::move(gb));
    return;
  }
  if (members.size() == 1)
    raise(WS_ERR_COMPILE, "regex " + std::to_string(members[0]) + " needs more than " +
                              std::to_string(max_states) + " DFA states (raise dfa_max_states)");
  size_t h = members.size() / 2;
  build_groups(trees, std::vector<uint32_t>(members.begin(), members.begin() + h), max_states, out, context);
  build_groups(trees, std::vector<uint32_t>(members.begin() + h, members.end()), max_states, out, context);
}

}  // namespace

void plan_regex(const ws_pattern_tables& t, const ws_config& cfg, int sm_count, RegexPlan& P) {
  (void)sm_count;
  P.n_regex = t.n_regex;
  if (!t.n_regex) return;
  std::vector<ReTree> trees(t.n_regex);
  P.max_len = 0;
  for (uint32_t r = 0; r < t.n_regex; ++r) {
    std::string src(t.regex_sources[r]);
    try {
      trees[r] = parse_regex(src);
    } catch (const CompileError& e) {
      raise(WS_ERR_COMPILE, "invalid regex at index " + std::to_string(t.regex_pattern_ids[r]) + ": " + e.what(),
            t.regex_pattern_ids[r]);
    }
    if (tree_nullable(trees[r]))
      raise(WS_ERR_COMPILE, "regex " + std::to_string(t.regex_pattern_ids[r]) +
                                " can match the empty string, which the GPU DFA path does not support",
            t.regex_pattern_ids[r]);
    // a look-ahead assertion reads the byte after the match: one more byte
    // of reach for the stream and shard bookkeeping
    int64_t ml = tree_max_len(trees[r]);
    if (ml >= 0 && tree_has_look(trees[r])) ml += 1;
    if (ml < 0 || P.max_len < 0) P.max_len = -1;
    else P.max_len = std::max(P.max_len, ml);
  }
  const int max_states = (int)std::max<uint32_t>(cfg.dfa_max_states, 16);
  P.walk_chunk = std::max<uint32_t>(256, cfg.walk_chunk / 256 * 256);
  // Greedy packing by the size of each regex's own unanchored DFA, then exact
  // verification of every group (halved while it exceeds the budget).
  std::vector<int> est(t.n_regex);
  std::vector<uint8_t> ctx(t.n_regex, 0);
  for (uint32_t r = 0; r < t.n_regex; ++r) {
    ctx[r] = tree_has_look(trees[r]) ? 1 : 0;
    Nfa n = build_nfa({&trees[r]}, false);
    ByteClasses bc = compute_classes({&n});
    Dfa d = ctx[r] ? build_context_all_dfa(n, bc, max_states) : build_all_dfa(n, bc, true, max_states);
    if (d.too_big)
      raise(WS_ERR_COMPILE, "regex " + std::to_string(t.regex_pattern_ids[r]) + " needs more than " +
                                std::to_string(max_states) + " DFA states (raise dfa_max_states)",
            t.regex_pattern_ids[r]);
    est[r] = d.n_states;
  }
  // speculative groups first, then the context groups
  std::vector<GroupBuild> gbs;
  for (int want_ctx = 0; want_ctx < 2; ++want_ctx) {
    std::vector<std::vector<uint32_t>> packs(1);
    int sum = 0;
    for (uint32_t r = 0; r < t.n_regex; ++r) {
      if (ctx[r] != want_ctx) continue;
      if (!packs.back().empty() && 4 * (sum + est[r]) > 3 * max_states) { packs.emplace_back(); sum = 0; }
      packs.back().push_back(r);
      sum += est[r];
    }
    for (auto& pk : packs)
      if (!pk.empty()) build_groups(trees, pk, max_states, gbs, want_ctx != 0);
    if (!want_ctx) P.n_spec = (uint32_t)gbs.size();
  }
  P.has_context = P.n_spec < gbs.size();

  // device layout: reverse and leftmost-first tables, then the forward layout
  P.n_groups = (uint32_t)gbs.size();
  P.rev_marks = P.n_groups < (1u << (32 - kRmarkStateBits));
  P.groups.assign(P.n_groups, GroupDev{});
  P.rev.clear(); P.lf.clear(); P.rmptr.clear(); P.rmlist.clear(); P.cls.clear();
  P.fdfa.clear(); P.fcls.clear(); P.gregex.clear(); P.nhot_u.clear(); P.nhot_a.clear();
  P.lfinfo.assign(4 * (size_t)t.n_regex, 0);
  P.lfx.assign(8 * (size_t)t.n_regex, 0);
  P.pid.assign(t.regex_pattern_ids, t.regex_pattern_ids + t.n_regex);
  P.regex_group.assign(t.n_regex, 0);
  P.n_warm = P.max_warm = 0;
  for (uint32_t g = 0; g < P.n_groups; ++g) {
    GroupBuild& gb = gbs[g];
    GroupDev& gd = P.groups[g];
    const uint32_t C = (uint32_t)gb.cls.count;
    // exact chunk starts when every regex of a speculative group is bounded
    int64_t gl = 0;
    for (uint32_t r : gb.regexes) {
      const int64_t ml = tree_max_len(trees[r]);
      gl = (ml < 0 || gl < 0) ? -1 : std::max(gl, ml);
    }
    gd.warm = (g < P.n_spec && gl > 0 && gl <= (int64_t)kWarmMax) ? (uint32_t)((gl + 15) / 16 * 16) : 0u;
    if (gd.warm) {
      ++P.n_warm;
      P.max_warm = std::max(P.max_warm, gd.warm);
    }
    gd.rev_off = append_trans(gb.rev, P.rev);
    gd.rev_start = gb.rev.start_anchored;
    if ((uint64_t)gb.rev.n_states >= (1ull << kRmarkStateBits)) P.rev_marks = false;
    gd.cls_off = g * 256;
    gd.rmptr_off = (uint32_t)P.rmptr.size();
    for (int s = 0; s < gb.rev.n_states; ++s) {
      P.rmptr.push_back((uint32_t)P.rmlist.size());
      for (uint32_t j = gb.rev.match_ptr[(size_t)s]; j < gb.rev.match_ptr[(size_t)s + 1]; ++j)
        P.rmlist.push_back(gb.regexes[gb.rev.match_list[j]]);
    }
    P.rmptr.push_back((uint32_t)P.rmlist.size());
    for (int b = 0; b < 256; ++b) P.cls.push_back(gb.cls.map[b]);
    for (size_t k = 0; k < gb.regexes.size(); ++k) {
      uint32_t r = gb.regexes[k];
      const Dfa& lf = gb.lf[k];
      P.lfinfo[4 * r + 0] = append_trans(lf, P.lf);
      P.lfinfo[4 * r + 1] = lf.start_anchored;
      P.lfinfo[4 * r + 2] = g;
      P.lfinfo[4 * r + 3] = C;
      P.regex_group[r] = g;
      if (gb.context) {  // start rows per left context, end-step flags after the table
        P.lfx[8 * r + 0] = 1;
        for (int k = 0; k < 4; ++k) P.lfx[8 * r + 1 + k] = lf.ctx_start[k];
        P.lfx[8 * r + 5] = (uint32_t)P.lf.size();
        for (int s = 0; s < lf.n_states; ++s) P.lf.push_back(lf.is_match[(size_t)s]);
      }
    }
    P.fdfa.push_back(std::move(gb.fwd));
    P.fcls.push_back(gb.cls);
    P.gregex.push_back(gb.regexes);
    P.nhot_u.push_back(gb.n_hot_u);
    P.nhot_a.push_back(gb.n_hot_a);
  }
  layout_forward(P);
  P.d_rev.upload(P.rev.data(), P.rev.size() * 4);
  P.d_lf.upload(P.lf.data(), P.lf.size() * 4);
  P.d_cls.upload(P.cls.data(), P.cls.size());
  P.d_rmptr.upload(P.rmptr.data(), P.rmptr.size() * 4);
  if (P.rmlist.empty()) P.rmlist.push_back(0);
  P.d_rmlist.upload(P.rmlist.data(), P.rmlist.size() * 4);
  P.d_lfinfo.upload(P.lfinfo.data(), P.lfinfo.size() * 4);
  P.d_lfx.upload(P.lfx.data(), P.lfx.size() * 4);
  P.d_pid.upload(P.pid.data(), P.pid.size() * 4);
  P.use_proposer = cfg.proposer == WS_PROPOSER_MLP;
}

namespace {

// Visit counts of the forward states of one group over a corpus: thread per
// 4 KiB chunk walking from the unanchored start, shared-memory histogram.
__global__ void visit_hist_kernel(const uint32_t* tab, uint32_t C, uint32_t start, const uint8_t* cls,
                                  const uint8_t* data, uint64_t len, uint32_t n_states, unsigned int* hist) {
  extern __shared__ unsigned int h[];
  for (uint32_t k = threadIdx.x; k < n_states; k += blockDim.x) h[k] = 0;
  __syncthreads();
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t c0 = i * 4096;
  if (c0 < len) {
    const uint64_t c1 = min(len, c0 + 4096);
    uint32_t st = start;
    for (uint64_t pos = c0; pos < c1; ++pos) {
      st = __ldg(tab + st * C + cls[data[pos]]) & F_MASK;
      atomicAdd(&h[st], 1u);
    }
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < n_states; k += blockDim.x)
    if (h[k]) atomicAdd(&hist[k], h[k]);
}

}  // namespace

void regex_rerank_from_corpus(RegexPlan& P, const uint8_t* d_corpus, uint64_t len) {
  if (!P.n_regex) return;
  const uint64_t use = std::min<uint64_t>(len, 64ull << 20);
  for (uint32_t g = 0; g < P.n_spec; ++g) {
    Dfa& d = P.fdfa[g];
    const uint32_t n = (uint32_t)d.n_states, C = (uint32_t)d.n_classes;
    if (n > (1u << 14)) continue;  // L2-only group: nothing to place
    DeviceBuffer hist;
    hist.alloc((size_t)n * 4);
    check_cuda(cudaMemset(hist.ptr, 0, (size_t)n * 4), "memset");
    size_t smem = (size_t)n * 4;
    check_cuda(cudaFuncSetAttribute(visit_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "smem(visit)");
    uint64_t chunks = (use + 4095) / 4096;
    visit_hist_kernel<<<(unsigned)((chunks + 255) / 256), 256, smem>>>(
        P.d_fwd.as<uint32_t>() + P.groups[g].fwd_off, C, d.start_unanchored, P.d_cls.as<uint8_t>() + g * 256,
        d_corpus, use, n, hist.as<unsigned int>());
    check_cuda(cudaGetLastError(), "visit_hist_kernel");
    std::vector<unsigned int> cnt(n);
    check_cuda(cudaMemcpy(cnt.data(), hist.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost), "D2H hist");
    // current layout: [hot u][hot a][rest u][rest a][dead]; keep the anchored
    // part's order, sort the unanchored part by visits
    const uint32_t hu = P.nhot_u[g], ha = P.nhot_a[g];
    std::vector<uint8_t> in_u(n, 0);
    std::deque<uint32_t> dq{d.start_unanchored};
    in_u[d.start_unanchored] = 1;
    while (!dq.empty()) {
      uint32_t s = dq.front();
      dq.pop_front();
      for (uint32_t c = 0; c < C; ++c) {
        uint32_t t2 = d.trans[(size_t)s * C + c] & DFA_MASK_STATE;
        if (!in_u[t2]) { in_u[t2] = 1; dq.push_back(t2); }
      }
    }
    std::vector<uint32_t> us, as;
    uint32_t dead = n - 1;
    for (uint32_t s = 0; s < n; ++s) {
      if (s == dead) continue;
      (in_u[s] ? us : as).push_back(s);
    }
    std::stable_sort(us.begin(), us.end(), [&](uint32_t a, uint32_t b) { return cnt[a] > cnt[b]; });
    (void)hu;
    std::vector<uint32_t> order;
    uint32_t nu = (uint32_t)std::min<size_t>(us.size(), std::max(kHotRows, walk_hot_rows(P.groups[g].n_classes)));
    order.insert(order.end(), us.begin(), us.begin() + nu);
    order.insert(order.end(), as.begin(), as.begin() + std::min<size_t>(as.size(), ha));
    order.insert(order.end(), us.begin() + nu, us.end());
    if (as.size() > ha) order.insert(order.end(), as.begin() + ha, as.end());
    order.push_back(dead);
    renumber_dfa(d, order);
    P.nhot_u[g] = nu;
  }
  layout_forward(P);
}

void regex_fill_info(const RegexPlan& P, ws_matcher_info& info) {
  info.n_groups = P.n_groups;
  info.regex_context = P.has_context ? 1 : 0;
  info.n_context_groups = P.n_groups - P.n_spec;
  info.total_states = P.total_states;
  info.max_classes = P.max_classes;
  info.proposer_top1 = P.top1;
  info.proposer_top4 = P.top4;
  info.max_regex_len = P.n_regex ? P.max_len : 0;
  info.exact_groups = P.n_warm;
}

namespace {

// Reverse-walk marks start empty in every scan (a stale mark would stop a
// walk that no other walk continues); plans whose state numbers do not fit
// the mark key run without them.
void clear_marks(const RegexPlan& P, ScanPtrs& p, cudaStream_t st) {
  if (!P.rev_marks || p.full_k) {
    p.rmark = nullptr;
    return;
  }
  check_cuda(cudaMemsetAsync(p.rmark, 0xFF, ((size_t)1 << kRmarkBits) * 8, st), "memset marks");
}

void ensure_scratch(DeviceBuffer& scratch, size_t need) {
  if (scratch.bytes >= need) return;
  size_t n = 1;
  while (n < need) n <<= 1;
  scratch.alloc(n);
}

}  // namespace

namespace {

// The walk chunk of one scan: the plan's chunk, made smaller (to at least half
// of it, in steps of kCkpt) when that fills the last wave of walk blocks --
// one 1,024-chunk block per SM and group -- so that no SM sits idle while the
// others walk (one group over 1 GiB in 8 KiB chunks is 128 blocks on 148 SMs;
// 7 KiB chunks make it 147).
uint32_t effective_chunk(const RegexPlan& P, uint64_t len, int sm_count) {
  const uint64_t c0 = P.walk_chunk, G = std::max<uint32_t>(P.n_spec, 1), sm = (uint64_t)std::max(sm_count, 1);
  auto blocks = [&](uint64_t c) { return G * (((len + c - 1) / c + kWalkThreads - 1) / kWalkThreads); };
  const uint64_t waves = (blocks(c0) + sm - 1) / sm;
  const uint64_t per_group = waves * sm / G;  // blocks per group that fill `waves` waves
  if (per_group == 0) return (uint32_t)c0;
  uint64_t c = (len + per_group * kWalkThreads - 1) / (per_group * kWalkThreads);
  c = (c + kCkpt - 1) / kCkpt * kCkpt;
  c = std::max<uint64_t>(c, std::max<uint64_t>(kCkpt, c0 / 2 / kCkpt * kCkpt));
  return (uint32_t)std::min<uint64_t>(c, c0);
}

}  // namespace

uint32_t run_regex_scan(RegexPlan& P, const RegexLaunch& l, cudaStream_t st, DeviceBuffer& scratch, int sm_count,
                        cudaEvent_t* ev) {
  if (!P.n_regex || l.len == 0) return 0;
  RxLayout L = layout(P, l.len, effective_chunk(P, l.len, sm_count), l.cap, l.k_min, l.ev_min);
  ensure_scratch(scratch, L.total);
  ScanPtrs p = make_ptrs(L, scratch.ptr, l);
  // profiled speculative scans count the boundary guesses that held
  if (ev && l.mode != WS_REGEX_PLAIN) p.count_guesses = P.n_spec;
  DevTables t = dev_tables(P);
  uint32_t launches = 0;
  clear_marks(P, p, st);
  check_cuda(cudaMemsetAsync(p.ctr, 0, 16 * 8, st), "memset");
  check_cuda(cudaMemsetAsync(p.count, 0, (size_t)P.n_regex * 4, st), "memset");
  if (ev) check_cuda(cudaEventRecord(ev[0], st), "event");
  launches += candidates_phase(P, t, p, l.mode, st, sm_count, ev);
  int hg = (int)std::min<uint64_t>((uint64_t)sm_count * 8, (L.k_cap + 255) / 256);
  k_scan_kernel<<<1, 1024, 0, st>>>(p, P.n_regex);
  k_scatter_kernel<<<hg, 256, 0, st>>>(p);
  k_sort_kernel<<<(unsigned)std::min<uint32_t>(P.n_regex, 4096), 512, 0, st>>>(p, P.n_regex);
  k_lf_kernel<<<sm_count * 8, 128, P.n_regex < kLfOffsShared ? (P.n_regex + 1) * 4 : 0, st>>>(t, p, P.n_regex);
  k_chain_kernel<<<(P.n_regex + 3) / 4, 128, 0, st>>>(t, p);  // a warp per regex
  check_cuda(cudaGetLastError(), "resolution kernels");
  launches += 5;
  finalize_kernel<<<1, 1, 0, st>>>(p, l.need);
  check_cuda(cudaGetLastError(), "finalize_kernel");
  launches += 1;
  if (ev) {
    // profiled scans read the counters back for ws_matcher_get_info
    if (!P.prof_ctr) {
      unsigned long long* h = nullptr;
      check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&h), 16 * 8, cudaHostAllocDefault), "cudaHostAlloc");
      std::memset(h, 0, 16 * 8);
      P.prof_ctr.reset(h);
    }
    check_cuda(cudaMemcpyAsync(P.prof_ctr.get(), p.ctr, 16 * 8, cudaMemcpyDeviceToHost, st), "D2H counters");
    check_cuda(cudaEventRecord(ev[5], st), "event");
  }
  P.last_chunks = L.n_q;
  P.last_launches = launches;
  return launches;
}

void regex_collect_timing(const RegexPlan& P, cudaEvent_t* ev, ws_matcher_info& info) {
  float ms = 0;
  // [2] proposer, [1] walk or plain, [3] fix-up, [4] reverse, [5] resolution, [6] regex total
  if (cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) info.last_kernel_ms[2] = ms;
  if (cudaEventElapsedTime(&ms, ev[1], ev[2]) == cudaSuccess) info.last_kernel_ms[1] = ms;
  if (cudaEventElapsedTime(&ms, ev[2], ev[3]) == cudaSuccess) info.last_kernel_ms[3] = ms;
  if (cudaEventElapsedTime(&ms, ev[3], ev[4]) == cudaSuccess) info.last_kernel_ms[4] = ms;
  if (cudaEventElapsedTime(&ms, ev[4], ev[5]) == cudaSuccess) info.last_kernel_ms[5] = ms;
  if (cudaEventElapsedTime(&ms, ev[0], ev[5]) == cudaSuccess) info.last_kernel_ms[6] = ms;
  if (P.prof_ctr) {
    const unsigned long long* c = P.prof_ctr.get();
    info.last_kcandidates = c[C_K];
    info.last_events = c[C_EV];
    info.last_fixup_chunks = c[C_FIX];
    info.last_rewalk_bytes = c[C_REWALK];
    info.last_guess_hits = c[C_HITS];
    info.last_guesses = c[C_GUESSES];
  }
}

uint64_t regex_candidates(RegexPlan& P, const uint8_t* d_data, uint64_t len, uint32_t mode, cudaStream_t st,
                          DeviceBuffer& scratch, int sm_count, ws_match* host_out, uint64_t cap) {
  if (!P.n_regex || len == 0) return 0;
  const bool full = (mode & WS_CAND_DISTINCT) == 0;
  mode &= ~(uint32_t)WS_CAND_DISTINCT;
  RegexLaunch l{d_data, len, nullptr, cap, nullptr, mode};
  // every candidate must fit: the buffers are sized for the caller's capacity
  RxLayout L = layout(P, len, effective_chunk(P, len, sm_count), std::max<uint64_t>(cap, 1), cap, cap);
  ensure_scratch(scratch, L.total);
  ScanPtrs p = make_ptrs(L, scratch.ptr, l);
  p.full_k = full ? 1 : 0;
  DevTables t = dev_tables(P);
  clear_marks(P, p, st);
  check_cuda(cudaMemsetAsync(p.ctr, 0, 16 * 8, st), "memset");
  candidates_phase(P, t, p, mode, st, sm_count, nullptr);
  unsigned long long ctr[16];
  check_cuda(cudaMemcpyAsync(ctr, p.ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st), "D2H");
  check_cuda(cudaStreamSynchronize(st), "sync");
  if (ctr[C_ERR] & kErrTimeout) raise(WS_ERR_TIMEOUT, "a device-side wait of the regex walk ran out");
  if (ctr[C_ERR])  // at least cap + 1 candidates (an event overflow leaves the count short)
    raise(WS_ERR_OVERFLOW, "too many regex candidates", 0, std::max<uint64_t>(ctr[C_K], cap + 1), cap);
  uint64_t n = std::min<uint64_t>(ctr[C_K], L.k_cap);
  if (n > cap) raise(WS_ERR_OVERFLOW, "too many regex candidates", 0, n, cap);
  if (n) {
    DeviceBuffer tmp;
    tmp.alloc(n * sizeof(ws_match));
    k_export_kernel<<<sm_count * 4, 256, 0, st>>>(t, p, tmp.as<ws_match>(), n);
    check_cuda(cudaMemcpyAsync(host_out, tmp.ptr, n * sizeof(ws_match), cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "sync");
  }
  return n;
}

}  // namespace ws
