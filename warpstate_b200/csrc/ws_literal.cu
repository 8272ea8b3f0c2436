// Literal prefilter + verify for sm_100a.
//
// Replaces the reference's two WGSL passes, literal_prefilter
// (core/src/gpu/shader.rs:18-101) and literal_verify (core/src/gpu/shader.rs:106-236).
//
// Kernel 1, literal_filter_kernel (streams the input once, HBM-bound):
//   stage 1   every thread owns 16 input bytes per step (one 16-byte coalesced
//             load, issued one step ahead).  It looks up the 4-byte grams at the
//             P-aligned positions in a nibble table staged in shared memory and
//             forms a 16-bit mask of positions that may start a literal (see
//             LiteralPlan); the warp's 512-byte block is copied to shared memory.
//   compact   popc prefix sums put the flagged positions of the warp into a
//             shared-memory queue, so stage 1.5 runs with all 32 lanes busy.
//   stage 1.5 each queued position reads its 8-byte window from shared memory
//             and checks, at every prefix length that has literals, a
//             multiply-shift key of the first min(len, 8) bytes against a Bloom
//             bitmap of the literals' prefixes in shared memory.
//   survivors are appended to a compact position list with one atomic per warp
//             (ballot + popc).  If the list is full, the position is verified in
//             place instead, so results never depend on the list's capacity.
// Kernel 1 for large sets, literal_lean_kernel (see its comment): stages 1 and
//             1b only, no compaction; stage 1.5 moves to kernel 2.
// Kernel 2, literal_verify_kernel: the reference's per-position algorithm on the
//             surviving positions only: FNV-1a probe of the LiteralPrefilterTable
//             partition at each non-empty prefix length (shader.rs:59-98) and an
//             exact compare of every entry whose hash is equal (shader.rs:174-227).
//
// The output is contract L: every overlapping occurrence of every literal.
#include <cuda_runtime.h>


#include "ws_internal.h"

namespace ws {

namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kBloomBits = 18;  // 2^18-bit Bloom bitmap (32 KiB)

struct LitArgs {
  const uint8_t* data;
  uint64_t len;
  const uint32_t* filter;
  uint32_t filter_words;
  uint32_t bits;
  uint32_t period;
  uint32_t has_long;
  uint32_t has_short;
  uint32_t parts;            // bit i: prefix length i+1 has literals
  const uint32_t* short_bits;
  const uint32_t* bloom;
  const uint4* info;
  const uint8_t* lit_bytes;
  const uint4* meta;
  const uint2* ranges;
  const uint2* entries;
  uint32_t window;
  ws_match* out;
  uint64_t cap;
  unsigned long long* counter;
  uint32_t* survivors;       // candidate start positions (low 32 bits)
  uint32_t* survivor_hi;     // unused for inputs < 4 GiB
  unsigned long long* survivor_count;
  uint64_t survivor_cap;
  const uint32_t* item_end;  // batch: ascending item ends (n_items), else null
  uint32_t n_items;
  uint64_t min_end;          // stream: matches ending at or before it were reported
  uint64_t max_start;        // shard: matches starting at or after it belong to the next shard
  uint32_t gram_len;        // stage-1 gram bytes: 4, 8 or 16 (8 and 16 with P = 4)
  uint32_t parts16;          // stage-1.5b key lengths (bit i: i+1 bytes)
  const uint32_t* bloom2;    // stage-1.5b bitmap (2^kBloom2Bits bits, L2), or null
  const uint8_t* big;        // stage-1b gram table (2^kBigBits bytes, L2), or null
  const uint32_t* lean_bits; // stage 1 with the stage-1b table (2^kLeanBits bits), or null
  uint32_t verify_bloom;     // the verify kernel runs stage 1.5 first
  uint32_t fold;             // ASCII case-insensitive: input bytes A-Z read as a-z
};

__device__ __forceinline__ uint4 fold16(uint4 v) {
  return make_uint4(ascii_fold4(v.x), ascii_fold4(v.y), ascii_fold4(v.z), ascii_fold4(v.w));
}

__device__ __forceinline__ uint32_t nib(const uint32_t* tab, uint32_t gram, uint32_t bits) {
  uint32_t h = (gram * 0x9E3779B1u) >> (32 - bits);
  return (tab[h >> 3] >> ((h & 7) << 2)) & 0xFu;
}

// Loads the 16 bytes of vector v, zero-filling past the end of the input.
__device__ __forceinline__ uint4 load_vec(const uint8_t* data, uint64_t len, uint64_t v) {
  uint64_t off = v * 16;
  if (off + 16 <= len) return __ldg(reinterpret_cast<const uint4*>(data + off));
  uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    uint64_t p = off + k;
    if (p < len) w[k >> 2] |= (uint32_t)__ldg(data + p) << ((k & 3) * 8);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// Bytes [a, a + 4) of the input for a 4-aligned a, zero past its end.
__device__ __forceinline__ uint32_t word_at(const uint8_t* d, uint32_t len, uint32_t a) {
  if (a + 4 <= len) return __ldg(reinterpret_cast<const uint32_t*>(d + a));
  uint32_t x = 0;
  for (uint32_t k = 0; k < 4; ++k)
    if (a + k < len) x |= (uint32_t)__ldg(d + a + k) << (8 * k);
  return x;
}

// word_at for the scan's input, case-folded for case-insensitive sets.
__device__ __forceinline__ uint32_t input_word(const LitArgs& a, uint32_t len, uint32_t at) {
  const uint32_t w = word_at(a.data, len, at);
  return a.fold ? ascii_fold4(w) : w;
}

// The reference's per-position probe and exact verify (stage 2).  Inputs of
// one launch are below 4 GiB.  The hashed bytes come from two words read
// once, and a candidate literal is compared a word at a time (literal bytes
// start 4-aligned in a buffer padded to 16 bytes).
__device__ void verify_position(const LitArgs& a, uint64_t s64) {
  if (s64 >= a.max_start) return;
  const uint32_t s = (uint32_t)s64, len = (uint32_t)a.len;
  const uint32_t w0 = s & ~3u, sh = (s & 3) * 8;
  const uint32_t x0 = input_word(a, len, w0), x1 = input_word(a, len, w0 + 4), x2 = input_word(a, len, w0 + 8);
  const uint32_t lo = __funnelshift_r(x0, x1, sh), hi = __funnelshift_r(x1, x2, sh);
  uint32_t h = 2166136261u;
  const uint32_t rem = len - s;
  const uint32_t maxp = rem < a.window ? rem : a.window;
  for (uint32_t i = 0; i < maxp; ++i) {
    h = (h ^ (((i < 4 ? lo : hi) >> (8 * (i & 3))) & 0xFFu)) * 16777619u;
    if (!((a.parts >> i) & 1u)) continue;
    uint4 m = __ldg(a.meta + i);
    uint2 r = __ldg(a.ranges + m.x + (h & m.y));
    for (uint32_t e = 0; e < r.y; ++e) {
      uint2 ent = __ldg(a.entries + r.x + e);
      if (ent.x != h) continue;
      uint4 info = __ldg(a.info + ent.y);  // {offset, len, pattern id, 0}
      if (info.y > rem) continue;
      const uint32_t* lit = reinterpret_cast<const uint32_t*>(a.lit_bytes + info.x);
      bool eq = true;
      uint32_t cur = x0;
      for (uint32_t k = 0; k < info.y; k += 4) {
        const uint32_t nxt = input_word(a, len, w0 + k + 4);
        const uint32_t dw = __funnelshift_r(cur, nxt, sh);
        const uint32_t left = info.y - k;
        const uint32_t m = left >= 4 ? 0xFFFFFFFFu : ((1u << (8 * left)) - 1u);
        if ((__ldg(lit + (k >> 2)) ^ dw) & m) { eq = false; break; }
        cur = nxt;
      }
      if (!eq) continue;
      if (s + info.y <= a.min_end) continue;
      if (a.n_items && s + info.y > item_end_of(a.item_end, a.n_items, (uint32_t)s)) continue;  // crosses items
      unsigned long long idx = atomicAdd(a.counter, 1ull);
      if (idx < a.cap) {
        ws_match mm;
        mm.pattern_id = info.z;
        mm.start = (uint32_t)s;
        mm.end = (uint32_t)(s + info.y);
        a.out[idx] = mm;
      }
    }
  }
}

// 16-bit mask of owned positions that may start a literal (stage 1).  w[0..3]
// are the thread's own words; w[4..7] are the next thread's words (w[4] is
// needed by the P = 1 and P = 2 layouts and by lane 31, w[5..7] by grams
// longer than 4 bytes).  The layout is a compile-time choice (P = period,
// G = gram bytes, LONG / SHORT = literals of >= 4 / < 4 bytes present).
template <int P, int G, bool LONG, bool SHORT>
__device__ __forceinline__ uint32_t stage1(const uint32_t* filt, const uint32_t* shortb, const uint32_t (&w)[8],
                                           uint32_t lane, uint32_t bits, const uint8_t* big) {
  uint32_t mask = 0;
  if (LONG) {
    if (G > 4 || P == 4) {
      // P = 4: grams of G bytes starting at the four aligned words; full
      // 32-bit hashes, the shared-memory table indexed by their top `bits`
      // bits, the L2 table (when present) by their top kBigBits bits
      uint32_t h[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        if (j == 4 && lane != 31) { h[4] = 0; break; }
        if (G == 4) h[j] = w[j] * 0x9E3779B1u;
        else if (G == 8) h[j] = mix_words(w[j], w[j + 1], 0, 0, 8);
        else h[j] = mix_words(w[j], w[j + 1], w[j + 2], w[j + 3], 16);
      }
      // with the stage-1b table, shared memory holds its stage 1 (the
      // two-bit blocked Bloom filter of long grams, or the bitmap derived
      // from the table) and the phase bits come from stage 1b alone
      auto phases = [&](uint32_t hf) -> uint32_t {
        if (big && G > 4) {
          const uint32_t m = lean2_mask(hf);
          return (filt[lean2_word(hf)] & m) == m ? (uint32_t)__ldg(big + (hf >> (32 - kBigBits))) : 0u;
        }
        if (big) {
          const uint32_t b = hf >> (32 - kLeanBits);
          return ((filt[b >> 5] >> (b & 31)) & 1u) ? (uint32_t)__ldg(big + (hf >> (32 - kBigBits))) : 0u;
        }
        const uint32_t hs = hf >> (32 - bits);
        return (filt[hs >> 3] >> ((hs & 7) << 2)) & 0xFu;
      };
      uint32_t n[5];
#pragma unroll
      for (int j = 0; j < 4; ++j) n[j] = phases(h[j]);
      n[4] = __shfl_down_sync(0xFFFFFFFFu, n[0], 1);
      if (lane == 31) n[4] = phases(h[4]);
      const uint32_t m = n[0] | (n[1] << 4) | (n[2] << 8) | (n[3] << 12) | (n[4] << 16);
      mask |= (m >> 3) & 0xFFFFu;
    } else if (P == 2) {
      uint32_t m = 0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        uint32_t g = (j & 1) ? __funnelshift_r(w[j >> 1], w[(j >> 1) + 1], 16) : w[j >> 1];
        uint32_t n;
        if (big) {  // the bitmap of the stage-1b table, then its phase bits
          const uint32_t hf = g * 0x9E3779B1u, b = hf >> (32 - kLeanBits);
          n = ((filt[b >> 5] >> (b & 31)) & 1u) ? (uint32_t)__ldg(big + (hf >> (32 - kBigBits))) : 0u;
        } else {
          n = nib(filt, g, bits);
        }
        m |= n << (2 * j);
      }
      mask |= (m >> 1) & 0xFFFFu;
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        uint32_t g = __funnelshift_r(w[j >> 2], w[(j >> 2) + 1], 8 * (j & 3));
        mask |= (nib(filt, g, bits) & 1u) << j;
      }
    }
  }
  if (SHORT) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      uint32_t g = __funnelshift_r(w[j >> 2], w[(j >> 2) + 1], 8 * (j & 3)) & 0xFFFFu;
      mask |= ((shortb[g >> 5] >> (g & 31)) & 1u) << j;
    }
  }
  return mask;
}

// Stage 1.5 key of the first pl bytes of a window (the host builds the Bloom
// bitmap with the same function over each literal's first min(len, 8) bytes).
__device__ __forceinline__ uint32_t prefix_key(uint32_t lo, uint32_t hi, uint32_t pl) {
  uint32_t ml = pl >= 4 ? 0xFFFFFFFFu : ((1u << (8 * pl)) - 1u);
  uint32_t mh = pl >= 8 ? 0xFFFFFFFFu : pl <= 4 ? 0u : ((1u << (8 * (pl - 4))) - 1u);
  uint32_t h = (lo & ml) * 0x9E3779B1u + (hi & mh) * 0x85EBCA77u + pl * 0xC2B2AE3Du;
  return h >> (32 - kBloomBits);
}

constexpr int kBlockWords = 136;  // 512 B warp block + 16 B of the next block + slack
constexpr int kQueue = 512;       // u16 offsets: at most 16 per lane

// A warp block with at least one stage-1 candidate: the block is copied to
// shared memory, the candidates are compacted into the queue (popc prefix
// sums), stage 1.5 runs with all lanes busy, survivors are appended with one
// atomic per warp.
template <int G>
__device__ __forceinline__ void process_block(const LitArgs& a, uint32_t* blk, uint16_t* queue, const uint32_t* bloom,
                                              uint32_t lane, const uint4& cur, const uint4& tail, uint32_t mask,
                                              uint32_t blk_base) {
  reinterpret_cast<uint4*>(blk)[lane] = cur;
  if (lane == 31) {
    reinterpret_cast<uint4*>(blk)[32] = tail;
    blk[132] = 0;
    blk[133] = 0;
  }
  __syncwarp();
  // compact the candidates of the warp into the queue
  const uint32_t cnt = __popc(mask);
  uint32_t incl = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  uint32_t pos = incl - cnt;
  while (mask) {
    uint32_t i = __ffs(mask) - 1;
    mask &= mask - 1;
    queue[pos++] = (uint16_t)(lane * 16 + i);
  }
  __syncwarp();
  // stage 1.5 with all lanes busy, then a warp-aggregated append of survivors
  for (uint32_t k0 = 0; k0 < total; k0 += 32) {
    const uint32_t k = k0 + lane;
    bool keep = false;
    uint32_t off = 0;
    if (k < total) {
      off = queue[k];
      const uint32_t wi = off >> 2, sh = (off & 3) * 8;
      const uint32_t x0 = blk[wi], x1 = blk[wi + 1], x2 = blk[wi + 2];
      const uint32_t lo = __funnelshift_r(x0, x1, sh), hi = __funnelshift_r(x1, x2, sh);
      for (uint32_t m = a.parts; m; m &= m - 1) {  // prefix lengths that have literals
        const uint32_t key = prefix_key(lo, hi, __ffs(m));
        keep |= (bloom[key >> 5] >> (key & 31)) & 1u;
      }
      if (G > 4 && keep) {
        // stage 1.5b: the first min(len, 16) bytes against the L2 bitmap
        const uint32_t x3 = blk[wi + 3], x4 = blk[wi + 4];
        const uint32_t y2 = __funnelshift_r(x2, x3, sh), y3 = __funnelshift_r(x3, x4, sh);
        bool k2 = false;
        for (uint32_t m = a.parts16; m; m &= m - 1) {
          const uint32_t key = prefix16_key(lo, hi, y2, y3, __ffs(m));
          k2 |= (__ldg(a.bloom2 + (key >> 5)) >> (key & 31)) & 1u;
        }
        keep = k2;
      }
    }
    const uint32_t ball = __ballot_sync(0xFFFFFFFFu, keep);
    if (ball) {
      unsigned long long wbase = 0;
      if (lane == 0) wbase = atomicAdd(a.survivor_count, (unsigned long long)__popc(ball));
      wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
      if (keep) {
        const unsigned long long slot = wbase + __popc(ball & ((1u << lane) - 1u));
        const uint32_t s = blk_base + off;
        if (slot < a.survivor_cap) a.survivors[slot] = s;
        else verify_position(a, s);  // list full: verify in place
      }
    }
  }
  __syncwarp();
}

// Inputs of one launch are below 4 GiB, so block, vector and byte indices are
// 32-bit.
template <int P, int G, bool LONG, bool SHORT>
__global__ void __launch_bounds__(kThreads, 1) literal_filter_kernel(LitArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* filt = smem;                                 // filter_words
  uint32_t* bloom = filt + a.filter_words;               // 2^kBloomBits / 32 words
  uint32_t* shortb = bloom + (1u << (kBloomBits - 5));   // 2048 words when SHORT
  uint32_t* warpmem = shortb + (SHORT ? 2048 : 0);

  {
    const uint4* src = reinterpret_cast<const uint4*>(a.filter);
    uint4* dst = reinterpret_cast<uint4*>(filt);
    const uint32_t n4 = LONG ? a.filter_words / 4 : 0;
    for (uint32_t k = threadIdx.x; k < n4; k += kThreads) dst[k] = __ldg(src + k);
    const uint4* bs = reinterpret_cast<const uint4*>(a.bloom);
    uint4* bd = reinterpret_cast<uint4*>(bloom);
    for (uint32_t k = threadIdx.x; k < (1u << (kBloomBits - 7)); k += kThreads) bd[k] = __ldg(bs + k);
    if (SHORT) {
      const uint4* s2 = reinterpret_cast<const uint4*>(a.short_bits);
      uint4* d2 = reinterpret_cast<uint4*>(shortb);
      for (uint32_t k = threadIdx.x; k < 512; k += kThreads) d2[k] = __ldg(s2 + k);
    }
  }
  __syncthreads();

  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = threadIdx.x >> 5;
  uint32_t* blk = warpmem + warp * (kBlockWords + kQueue / 2);
  uint16_t* queue = reinterpret_cast<uint16_t*>(blk + kBlockWords);
  const uint32_t len = (uint32_t)a.len;
  const uint32_t nvec = (uint32_t)((a.len + 15) >> 4);
  const uint32_t full_vecs = len >> 4;                 // vectors entirely inside the input
  const uint32_t nblk = (nvec + 31) >> 5;              // 512-byte warp blocks
  const uint32_t nwarps = gridDim.x * kWarps;
  const uint32_t bits = a.bits;
  auto load = [&](uint32_t v) -> uint4 {
    const uint4 x = v < full_vecs ? __ldg(reinterpret_cast<const uint4*>(a.data) + v)
                    : v < nvec ? load_vec(a.data, a.len, v) : make_uint4(0, 0, 0, 0);
    return a.fold ? fold16(x) : x;
  };

  uint32_t b = blockIdx.x * kWarps + warp;
  uint4 cur = make_uint4(0, 0, 0, 0);
  if (b < nblk) cur = load(b * 32 + lane);
  for (; b < nblk; b += nwarps) {
    // software pipeline: the next block's load is in flight during this one
    const uint32_t bn = b + nwarps;
    const uint4 nxt = bn < nblk ? load(bn * 32 + lane) : make_uint4(0, 0, 0, 0);
    const uint32_t v = b * 32 + lane;
    const uint4 tail = lane == 31 ? load(v + 1) : make_uint4(0, 0, 0, 0);
    uint32_t w[8] = {cur.x, cur.y, cur.z, cur.w, __shfl_down_sync(0xFFFFFFFFu, cur.x, 1), 0, 0, 0};
    if (G > 4) {
      w[5] = __shfl_down_sync(0xFFFFFFFFu, cur.y, 1);
      w[6] = __shfl_down_sync(0xFFFFFFFFu, cur.z, 1);
      w[7] = __shfl_down_sync(0xFFFFFFFFu, cur.w, 1);
    }
    if (lane == 31) {
      w[4] = tail.x;
      w[5] = tail.y;
      w[6] = tail.z;
      w[7] = tail.w;
    }
    uint32_t mask = stage1<P, G, LONG, SHORT>(filt, shortb, w, lane, bits, a.big);
    const uint32_t blk_base = b * 512;
    if (v >= full_vecs) {  // the input's last, partial vector (or past the end)
      const uint32_t base = v * 16;
      const uint32_t valid = len > base ? len - base : 0;
      mask &= (valid >= 16) ? 0xFFFFu : ((1u << valid) - 1u);
    }
    // most warp blocks have no candidate at all once stage 1b is in place
    if (__ballot_sync(0xFFFFFFFFu, mask != 0) == 0) {
      cur = nxt;
      continue;
    }
    process_block<G>(a, blk, queue, bloom, lane, cur, tail, mask, blk_base);
    __syncwarp();
    cur = nxt;
  }
}

// Stage 1 of the P = 4 layouts with the stage-1b table, split in two so that
// the L2 loads of a block are in flight while the previous block finishes:
// grams_issue hashes the five aligned grams of a lane (the fifth only on lane
// 31), looks them up in shared memory and starts the L2 loads of the passing
// ones; grams_finish combines them into the 16-bit candidate mask.
struct Grams {
  uint32_t h[5], n[5], bw[5];
};

template <int G>
__device__ __forceinline__ void grams_issue(const uint32_t* filt, const uint8_t* big, const uint32_t (&w)[8],
                                            uint32_t lane, uint32_t bits, Grams& s) {
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    if (j == 4 && lane != 31) {
      s.h[4] = 0;
      s.n[4] = 0;
      s.bw[4] = 0;
      break;
    }
    uint32_t hf;
    if (G == 4) hf = w[j] * 0x9E3779B1u;
    else if (G == 8) hf = mix_words(w[j], w[j + 1], 0, 0, 8);
    else hf = mix_words(w[j], w[j + 1], w[j + 2], w[j + 3], 16);
    // stage 1: the 2^kLeanBits-bit bitmap derived from the stage-1b table
    const uint32_t b = hf >> (32 - kLeanBits);
    s.h[j] = hf;
    s.n[j] = ((filt[b >> 5] >> (b & 31)) & 1u) ? 0xFu : 0u;
    s.bw[j] = s.n[j] ? __ldg(big + (hf >> (32 - kBigBits))) : 0u;
  }
}

__device__ __forceinline__ uint32_t grams_finish(const Grams& s, uint32_t lane) {
  uint32_t n[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) n[j] = s.n[j] & s.bw[j];
  const uint32_t n4 = __shfl_down_sync(0xFFFFFFFFu, n[0], 1);
  const uint32_t m = n[0] | (n[1] << 4) | (n[2] << 8) | (n[3] << 12) | ((lane == 31 ? n[4] : n4) << 16);
  return (m >> 3) & 0xFFFFu;
}

// The words a lane needs: its own four and the next lane's four (the tail
// vector on lane 31).
template <int G>
__device__ __forceinline__ void lane_words(const uint4& cur, const uint4& tail, uint32_t lane, uint32_t (&w)[8]) {
  w[0] = cur.x;
  w[1] = cur.y;
  w[2] = cur.z;
  w[3] = cur.w;
  w[4] = __shfl_down_sync(0xFFFFFFFFu, cur.x, 1);
  w[5] = w[6] = w[7] = 0;
  if (G > 4) {
    w[5] = __shfl_down_sync(0xFFFFFFFFu, cur.y, 1);
    w[6] = __shfl_down_sync(0xFFFFFFFFu, cur.z, 1);
    w[7] = __shfl_down_sync(0xFFFFFFFFu, cur.w, 1);
  }
  if (lane == 31) {
    w[4] = tail.x;
    w[5] = tail.y;
    w[6] = tail.z;
    w[7] = tail.w;
  }
}

constexpr int kBigThreads = 512;
constexpr int kBigWarps = kBigThreads / 32;

// P = 4 with the stage-1b table in L2: the same work as literal_filter_kernel
// in a three-block software pipeline per warp -- the input of block i+2 is
// loaded, the grams of block i+1 are hashed and their L2 checks issued, then
// block i is finished -- so that the L2 latency overlaps useful work.
// 16 warps per CTA leave room for the pipeline's registers.
template <int G, bool SHORT>
__global__ void __launch_bounds__(kBigThreads, 1) literal_filter_big_kernel(LitArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* filt = smem;
  uint32_t* bloom = filt + a.filter_words;
  uint32_t* shortb = bloom + (1u << (kBloomBits - 5));
  uint32_t* warpmem = shortb + (SHORT ? 2048 : 0);
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.filter);
    uint4* dst = reinterpret_cast<uint4*>(filt);
    for (uint32_t k = threadIdx.x; k < a.filter_words / 4; k += kBigThreads) dst[k] = __ldg(src + k);
    const uint4* bs = reinterpret_cast<const uint4*>(a.bloom);
    uint4* bd = reinterpret_cast<uint4*>(bloom);
    for (uint32_t k = threadIdx.x; k < (1u << (kBloomBits - 7)); k += kBigThreads) bd[k] = __ldg(bs + k);
    if (SHORT) {
      const uint4* s2 = reinterpret_cast<const uint4*>(a.short_bits);
      uint4* d2 = reinterpret_cast<uint4*>(shortb);
      for (uint32_t k = threadIdx.x; k < 512; k += kBigThreads) d2[k] = __ldg(s2 + k);
    }
  }
  __syncthreads();

  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = threadIdx.x >> 5;
  uint32_t* blk = warpmem + warp * (kBlockWords + kQueue / 2);
  uint16_t* queue = reinterpret_cast<uint16_t*>(blk + kBlockWords);
  const uint32_t len = (uint32_t)a.len;
  const uint32_t nvec = (uint32_t)((a.len + 15) >> 4);
  const uint32_t full_vecs = len >> 4;
  const uint32_t nblk = (nvec + 31) >> 5;
  const uint32_t nwarps = gridDim.x * kBigWarps;
  const uint32_t bits = a.bits;
  auto load = [&](uint32_t v) -> uint4 {
    const uint4 x = v < full_vecs ? __ldg(reinterpret_cast<const uint4*>(a.data) + v)
                    : v < nvec ? load_vec(a.data, a.len, v) : make_uint4(0, 0, 0, 0);
    return a.fold ? fold16(x) : x;
  };
  const uint4 zero = make_uint4(0, 0, 0, 0);

  uint32_t b = blockIdx.x * kBigWarps + warp;
  // pipeline registers: block b (cur, grams in flight), block b + nwarps (nxt)
  uint4 cur = zero, tail_c = zero, nxt = zero, tail_n = zero;
  Grams gc;
  if (b < nblk) {
    cur = load(b * 32 + lane);
    tail_c = lane == 31 ? load(b * 32 + 32) : zero;
    uint32_t w[8];
    lane_words<G>(cur, tail_c, lane, w);
    grams_issue<G>(filt, a.big, w, lane, bits, gc);
  }
  if (b + nwarps < nblk) {
    nxt = load((b + nwarps) * 32 + lane);
    tail_n = lane == 31 ? load((b + nwarps) * 32 + 32) : zero;
  }
  for (; b < nblk; b += nwarps) {
    const uint32_t bn = b + nwarps, bn2 = bn + nwarps;
    // input of block b + 2 nwarps
    uint4 nxt2 = zero, tail2 = zero;
    if (bn2 < nblk) {
      nxt2 = load(bn2 * 32 + lane);
      tail2 = lane == 31 ? load(bn2 * 32 + 32) : zero;
    }
    // grams of block b + nwarps, L2 checks issued
    Grams gn;
    if (bn < nblk) {
      uint32_t w[8];
      lane_words<G>(nxt, tail_n, lane, w);
      grams_issue<G>(filt, a.big, w, lane, bits, gn);
    }
    // finish block b
    uint32_t mask = grams_finish(gc, lane);
    if (SHORT) {
      uint32_t w[8];
      lane_words<G>(cur, tail_c, lane, w);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const uint32_t g = __funnelshift_r(w[j >> 2], w[(j >> 2) + 1], 8 * (j & 3)) & 0xFFFFu;
        mask |= ((shortb[g >> 5] >> (g & 31)) & 1u) << j;
      }
    }
    const uint32_t v = b * 32 + lane;
    if (v >= full_vecs) {
      const uint32_t base = v * 16;
      const uint32_t valid = len > base ? len - base : 0;
      mask &= (valid >= 16) ? 0xFFFFu : ((1u << valid) - 1u);
    }
    if (__ballot_sync(0xFFFFFFFFu, mask != 0) != 0)
      process_block<G>(a, blk, queue, bloom, lane, cur, tail_c, mask, b * 512);
    cur = nxt;
    tail_c = tail_n;
    gc = gn;
    nxt = nxt2;
    tail_n = tail2;
  }
}

// ------------------------------------------------------------- lean kernel
// P = 4, 4-byte grams, stage-1b table present, no literals shorter than 4
// bytes (the large-set layout).  Stage 1.5 moves to the verify kernel, so the
// filter only hashes, looks up and appends:
//   - ownership is shifted by 3: the lane with the 16 bytes at `base` owns the
//     start positions base-3 .. base+12, whose first 4-aligned position is one
//     of its own four words, so its own four grams decide all of them (bit t of
//     n0 | n1 << 4 | n2 << 8 | n3 << 12 is position base - 3 + t) and no lane
//     needs its neighbour's bytes.  The last three positions of the input start
//     no literal of 4 or more bytes;
//   - a warp step covers kLeanVecs coalesced 512-byte halves (32 bytes per
//     lane), so the per-step overhead is paid once per kLeanVecs x 512 bytes;
//   - stage 1 and the stage-1b loads run one warp step ahead of the step
//     being finished, the input two steps ahead;
//   - the stage-1b survivors of a warp step (about 0.15 per 512 bytes on
//     10,000 literals) are appended into the warp's reserved slots of the
//     list, one atomic per kLeanChunk slots (see lean_append).
constexpr int kLeanThreads = 1024;
constexpr int kLeanVecs = 2;  // 16-byte vectors per lane per warp step (a step covers kLeanVecs x 512 bytes)

struct LeanGrams {
  uint32_t bw[4];  // the stage-1b phase bits of the four grams (0: rejected by stage 1)
};

// Stage 1 of a lane's four aligned grams from the bitmap in shared memory
// (top kLeanBits bits of the hash); the stage-1b loads from the byte table in
// L2 (top kBigBits bits, the P phase bits) are issued for the grams that pass.
__device__ __forceinline__ void lean_issue(const uint32_t* filt, const uint8_t* big, const uint4& v, LeanGrams& g) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t hf = w[q] * 0x9E3779B1u;
    const uint32_t b = hf >> (32 - kLeanBits);
    const bool pass = (filt[b >> 5] >> (b & 31)) & 1u;
    g.bw[q] = pass ? (uint32_t)__ldg(big + (hf >> (32 - kBigBits))) : 0u;
  }
}

// Candidate mask of positions base-3 .. base+12 inside [0, len).
__device__ __forceinline__ uint32_t lean_finish(const LeanGrams& g, uint32_t base, uint32_t len) {
  uint32_t mask = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) mask |= g.bw[q] << (4 * q);
  if (base == 0) mask &= ~7u;  // positions -3 .. -1
  if (base + 13 > len) {
    const uint32_t valid = len + 3 > base ? len + 3 - base : 0;
    mask &= valid >= 16 ? 0xFFFFu : ((1u << valid) - 1u);
  }
  return mask;
}

// Survivor slots are reserved per warp, kLeanChunk at a time, so that the
// single global counter sees one atomic per chunk rather than one per warp
// block; slots a warp reserved but did not fill hold kNoSurvivor.
constexpr uint32_t kLeanChunk = 32;
constexpr uint32_t kNoSurvivor = 0xFFFFFFFFu;  // no position: inputs end below 2^32 - 64

struct LeanSlots {
  unsigned long long next = 0, end = 0;  // the warp's reserved range [next, end)
};

// Marks the warp's unfilled reserved slots as holes.
__device__ __forceinline__ void lean_holes(const LitArgs& a, const LeanSlots& r, uint32_t lane) {
  for (unsigned long long k = r.next + lane; k < r.end && k < a.survivor_cap; k += 32) a.survivors[k] = kNoSurvivor;
}

template <int V>
__device__ __forceinline__ void lean_append(const LitArgs& a, LeanSlots& r, const uint32_t (&mask)[V],
                                            const uint32_t (&base)[V], uint32_t lane) {
  uint32_t any = 0, cnt = 0;
#pragma unroll
  for (int h = 0; h < V; ++h) {
    any |= mask[h];
    cnt += __popc(mask[h]);
  }
  if (__ballot_sync(0xFFFFFFFFu, any != 0) == 0) return;
  uint32_t incl = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  if (r.next + total > r.end) {  // warp-uniform: reserve a new chunk
    lean_holes(a, r, lane);
    const unsigned long long want = total > kLeanChunk ? total : kLeanChunk;
    unsigned long long wb = 0;
    if (lane == 0) wb = atomicAdd(a.survivor_count, want);
    wb = __shfl_sync(0xFFFFFFFFu, wb, 0);
    r.next = wb;
    r.end = wb + want;
  }
  unsigned long long slot = r.next + incl - cnt;
  r.next += total;
#pragma unroll
  for (int h = 0; h < V; ++h) {
    for (uint32_t m = mask[h]; m; m &= m - 1) {
      const uint32_t s = base[h] - 3 + (__ffs(m) - 1);
      if (slot < a.survivor_cap) a.survivors[slot] = s;
      else verify_position(a, s);  // list full: verify in place
      ++slot;
    }
  }
}

__global__ void __launch_bounds__(kLeanThreads, 1) literal_lean_kernel(LitArgs a) {
  constexpr uint32_t W = kLeanThreads / 32, V = kLeanVecs;
  extern __shared__ __align__(16) uint32_t filt[];
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.lean_bits);
    uint4* dst = reinterpret_cast<uint4*>(filt);
    for (uint32_t k = threadIdx.x; k < (1u << (kLeanBits - 7)); k += kLeanThreads) dst[k] = __ldg(src + k);
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t len = (uint32_t)a.len;
  const uint32_t nvec = (uint32_t)((a.len + 15) >> 4);
  const uint32_t full_vecs = len >> 4;
  const uint32_t nblk = (nvec + 32 * V - 1) / (32 * V);  // warp steps of V * 512 bytes
  const uint32_t nw = gridDim.x * W;
  const uint8_t* big = a.big;
  const uint4 zero = make_uint4(0, 0, 0, 0);
  // half h of warp step blk: the 512 coalesced bytes at (blk * V + h) * 512
  auto load = [&](uint32_t blk, uint32_t h) -> uint4 {
    const uint32_t v = (blk * V + h) * 32 + lane;
    const uint4 x = v < full_vecs ? __ldg(reinterpret_cast<const uint4*>(a.data) + v)
                    : v < nvec ? load_vec(a.data, a.len, v) : zero;
    return a.fold ? fold16(x) : x;
  };
  uint32_t b = blockIdx.x * W + warp;
  LeanSlots slots;
  // stage 1 and the stage-1b loads of step b + nw run while step b finishes;
  // the input is loaded two steps ahead
  uint4 vn[V];
  LeanGrams gc[V];
#pragma unroll
  for (uint32_t h = 0; h < V; ++h) {
    vn[h] = b + nw < nblk ? load(b + nw, h) : zero;
    if (b < nblk) lean_issue(filt, big, load(b, h), gc[h]);
  }
  for (; b < nblk; b += nw) {
    const uint32_t b1 = b + nw, b2 = b1 + nw;
    uint4 vn2[V];
    LeanGrams gn[V];
    uint32_t mask[V], base[V];
#pragma unroll
    for (uint32_t h = 0; h < V; ++h) {
      vn2[h] = b2 < nblk ? load(b2, h) : zero;
      if (b1 < nblk) lean_issue(filt, big, vn[h], gn[h]);
      base[h] = (b * V + h) * 512 + lane * 16;
      mask[h] = lean_finish(gc[h], base[h], len);
    }
    lean_append<V>(a, slots, mask, base, lane);
#pragma unroll
    for (uint32_t h = 0; h < V; ++h) {
      gc[h] = gn[h];
      vn[h] = vn2[h];
    }
  }
  lean_holes(a, slots, lane);
}

__global__ void __launch_bounds__(256) literal_verify_kernel(LitArgs a) {
  unsigned long long n = *a.survivor_count;
  if (n > a.survivor_cap) n = a.survivor_cap;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t s = a.survivors[k];
    if (s == kNoSurvivor) continue;  // a slot the lean kernel reserved but did not fill
    if (a.verify_bloom) {  // stage 1.5 for survivors of the lean kernel
      const uint32_t len = (uint32_t)a.len, w0 = s & ~3u, sh = (s & 3) * 8;
      const uint32_t x0 = input_word(a, len, w0), x1 = input_word(a, len, w0 + 4), x2 = input_word(a, len, w0 + 8);
      const uint32_t lo = __funnelshift_r(x0, x1, sh), hi = __funnelshift_r(x1, x2, sh);
      bool keep = false;
      for (uint32_t m = a.parts; m; m &= m - 1) {
        const uint32_t key = prefix_key(lo, hi, __ffs(m));
        keep |= (__ldg(a.bloom + (key >> 5)) >> (key & 31)) & 1u;
      }
      if (!keep) continue;
    }
    verify_position(a, s);
  }
}

}  // namespace

size_t literal_smem_bytes(const LiteralPlan& plan) {
  const size_t filter_words = plan.has_big ? ((size_t)1 << (kLeanBits - 5)) : plan.filter.size();
  return (filter_words + (1u << (kBloomBits - 5)) + (plan.has_short ? 2048 : 0) +
          (size_t)kWarps * (kBlockWords + kQueue / 2)) * 4;
}

size_t literal_scratch_bytes(uint64_t survivor_cap) { return 64 + survivor_cap * 4; }

void launch_literal_scan(const LiteralPlan& plan, const LiteralLaunch& l, cudaStream_t st, int sm_count) {
  if (plan.n_literals == 0 || l.len == 0) return;
  LitArgs a;
  a.data = l.data;
  a.len = l.len;
  // with a stage-1b table, stage 1 in shared memory is its bitmap
  a.filter = plan.has_big ? plan.d_lean_bits.as<uint32_t>() : plan.d_filter.as<uint32_t>();
  a.filter_words = plan.has_big ? (1u << (kLeanBits - 5)) : (uint32_t)plan.filter.size();
  a.bits = plan.table_bits;
  a.period = plan.period;
  a.has_long = plan.has_long;
  a.has_short = plan.has_short;
  a.parts = plan.parts;
  a.short_bits = plan.d_short.as<uint32_t>();
  a.bloom = plan.d_bloom.as<uint32_t>();
  a.info = plan.d_info.as<uint4>();
  a.lit_bytes = plan.d_bytes.as<uint8_t>();
  a.meta = plan.d_meta.as<uint4>();
  a.ranges = plan.d_ranges.as<uint2>();
  a.entries = plan.d_entries.as<uint2>();
  a.window = HASH_WINDOW;
  a.out = l.out;
  a.cap = l.cap;
  a.counter = l.counter;
  a.survivor_count = reinterpret_cast<unsigned long long*>(l.scratch);
  a.survivors = reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(l.scratch) + 64);
  a.survivor_hi = nullptr;
  a.survivor_cap = l.survivor_cap;
  a.item_end = l.item_end;
  a.n_items = l.n_items;
  a.min_end = l.min_end;
  a.max_start = l.max_start;
  a.gram_len = plan.gram_len;
  a.parts16 = plan.parts16;
  a.bloom2 = plan.gram_len > 4 ? plan.d_bloom2.as<uint32_t>() : nullptr;
  a.big = plan.has_big ? plan.d_big.as<uint8_t>() : nullptr;
  a.lean_bits = plan.has_big ? plan.d_lean_bits.as<uint32_t>() : nullptr;
  a.verify_bloom = 0;
  a.fold = plan.fold ? 1 : 0;
  check_cuda(cudaMemsetAsync(a.survivor_count, 0, 8, st), "memset survivors");
  if (l.len > 0xFFFFFFFFull) raise(WS_ERR_INPUT_TOO_LARGE, "literal scan launch beyond 32-bit offsets", 0, l.len,
                                   0xFFFFFFFFull);
  const size_t smem = literal_smem_bytes(plan);
  uint64_t nblk = ((l.len + 15) / 16 + 31) / 32;
  uint64_t want = (nblk + kWarps - 1) / kWarps;
  int grid = (int)std::min<uint64_t>((uint64_t)sm_count, std::max<uint64_t>(want, 1));
  // the filter layout is a compile-time choice of the kernel
  auto run = [&](auto kernel) {
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "cudaFuncSetAttribute(literal)");
    kernel<<<grid, kThreads, smem, st>>>(a);
    check_cuda(cudaGetLastError(), "literal_filter_kernel launch");
  };
  const bool lg = plan.has_long != 0, sh = plan.has_short != 0;
  auto run_big = [&](auto kernel) {
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "cudaFuncSetAttribute(literal)");
    kernel<<<grid, kBigThreads, smem, st>>>(a);
    check_cuda(cudaGetLastError(), "literal_filter_big_kernel launch");
  };
  // large sets with 4-byte grams: the lean kernel, or with literals shorter
  // than 4 bytes the pipelined compacting kernel; long grams, whose hashing
  // dominates, keep 32 warps per SM
  if (lg && !sh && a.big && a.lean_bits && plan.period == 4 && plan.gram_len == 4) {
    a.verify_bloom = 1;
    const size_t lsmem = (size_t)1 << (kLeanBits - 3);
    check_cuda(cudaFuncSetAttribute(literal_lean_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem),
               "cudaFuncSetAttribute(literal lean)");
    literal_lean_kernel<<<sm_count, kLeanThreads, lsmem, st>>>(a);
    check_cuda(cudaGetLastError(), "literal_lean_kernel launch");
  } else if (lg && sh && a.big && plan.period == 4 && plan.gram_len == 4) {
    run_big(literal_filter_big_kernel<4, true>);
  } else if (!lg) {
    run(literal_filter_kernel<4, 4, false, true>);
  } else if (plan.gram_len == 16) {
    sh ? run(literal_filter_kernel<4, 16, true, true>) : run(literal_filter_kernel<4, 16, true, false>);
  } else if (plan.gram_len == 8) {
    sh ? run(literal_filter_kernel<4, 8, true, true>) : run(literal_filter_kernel<4, 8, true, false>);
  } else if (plan.period == 4) {
    sh ? run(literal_filter_kernel<4, 4, true, true>) : run(literal_filter_kernel<4, 4, true, false>);
  } else if (plan.period == 2) {
    sh ? run(literal_filter_kernel<2, 4, true, true>) : run(literal_filter_kernel<2, 4, true, false>);
  } else {
    sh ? run(literal_filter_kernel<1, 4, true, true>) : run(literal_filter_kernel<1, 4, true, false>);
  }
  // the verify pass is a chain of dependent loads per survivor: the lean
  // path's longer survivor list (stage 1.5 runs here) gets more threads
  literal_verify_kernel<<<sm_count * (a.verify_bloom ? 16 : 4), 256, 0, st>>>(a);
  check_cuda(cudaGetLastError(), "literal_verify_kernel launch");
}

}  // namespace ws
