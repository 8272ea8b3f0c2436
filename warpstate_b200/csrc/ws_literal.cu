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
};

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

// The reference's per-position probe and exact verify (stage 2).
__device__ void verify_position(const LitArgs& a, uint64_t s) {
  if (s >= a.max_start) return;
  uint32_t h = 2166136261u;
  uint64_t rem = a.len - s;
  uint32_t maxp = (uint32_t)(rem < a.window ? rem : a.window);
  for (uint32_t i = 0; i < maxp; ++i) {
    h = (h ^ (uint32_t)__ldg(a.data + s + i)) * 16777619u;
    if (!((a.parts >> i) & 1u)) continue;
    uint4 m = __ldg(a.meta + i);
    uint2 r = __ldg(a.ranges + m.x + (h & m.y));
    for (uint32_t e = 0; e < r.y; ++e) {
      uint2 ent = __ldg(a.entries + r.x + e);
      if (ent.x != h) continue;
      uint4 info = __ldg(a.info + ent.y);  // {offset, len, pattern id, 0}
      if (info.y > rem) continue;
      const uint8_t* lit = a.lit_bytes + info.x;
      bool eq = true;
      for (uint32_t k = 0; k < info.y; ++k) {
        if (__ldg(lit + k) != __ldg(a.data + s + k)) { eq = false; break; }
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

__device__ __forceinline__ uint32_t nib_long(const uint32_t* tab, uint32_t g0, uint32_t g1, uint32_t g2, uint32_t g3,
                                             uint32_t gram_len, uint32_t bits) {
  uint32_t h = long_gram_hash(g0, g1, g2, g3, gram_len, bits);
  return (tab[h >> 3] >> ((h & 7) << 2)) & 0xFu;
}

// 16-bit mask of owned positions that may start a literal (stage 1).  w[0..3]
// are the thread's own words; w[4..7] are the next thread's words (w[4] is
// needed by the P = 1 and P = 2 layouts and by lane 31, w[5..7] by grams
// longer than 4 bytes).
__device__ __forceinline__ uint32_t stage1(const LitArgs& a, const uint32_t* filt, const uint32_t* shortb,
                                           const uint32_t (&w)[8], uint32_t lane) {
  uint32_t mask = 0;
  if (a.has_long) {
    if (a.gram_len > 4) {
      // P = 4, grams of 8 or 16 bytes starting at the four aligned words
      uint32_t n0 = nib_long(filt, w[0], w[1], w[2], w[3], a.gram_len, a.bits);
      uint32_t n1 = nib_long(filt, w[1], w[2], w[3], w[4], a.gram_len, a.bits);
      uint32_t n2 = nib_long(filt, w[2], w[3], w[4], w[5], a.gram_len, a.bits);
      uint32_t n3 = nib_long(filt, w[3], w[4], w[5], w[6], a.gram_len, a.bits);
      uint32_t n4 = __shfl_down_sync(0xFFFFFFFFu, n0, 1);
      if (lane == 31) n4 = nib_long(filt, w[4], w[5], w[6], w[7], a.gram_len, a.bits);
      uint32_t m = n0 | (n1 << 4) | (n2 << 8) | (n3 << 12) | (n4 << 16);
      mask |= (m >> 3) & 0xFFFFu;
    } else if (a.period == 4) {
      uint32_t n0 = nib(filt, w[0], a.bits);
      uint32_t n1 = nib(filt, w[1], a.bits);
      uint32_t n2 = nib(filt, w[2], a.bits);
      uint32_t n3 = nib(filt, w[3], a.bits);
      uint32_t n4 = __shfl_down_sync(0xFFFFFFFFu, n0, 1);
      if (lane == 31) n4 = nib(filt, w[4], a.bits);
      uint32_t m = n0 | (n1 << 4) | (n2 << 8) | (n3 << 12) | (n4 << 16);
      mask |= (m >> 3) & 0xFFFFu;
    } else if (a.period == 2) {
      uint32_t m = 0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        uint32_t g = (j & 1) ? __funnelshift_r(w[j >> 1], w[(j >> 1) + 1], 16) : w[j >> 1];
        m |= nib(filt, g, a.bits) << (2 * j);
      }
      mask |= (m >> 1) & 0xFFFFu;
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        uint32_t g = __funnelshift_r(w[j >> 2], w[(j >> 2) + 1], 8 * (j & 3));
        mask |= (nib(filt, g, a.bits) & 1u) << j;
      }
    }
  }
  if (a.has_short) {
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

__global__ void __launch_bounds__(kThreads, 1) literal_filter_kernel(LitArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* filt = smem;                                 // filter_words
  uint32_t* bloom = filt + a.filter_words;               // 2^kBloomBits / 32 words
  uint32_t* shortb = bloom + (1u << (kBloomBits - 5));   // 2048 words when has_short
  uint32_t* warpmem = shortb + (a.has_short ? 2048 : 0);

  {
    const uint4* src = reinterpret_cast<const uint4*>(a.filter);
    uint4* dst = reinterpret_cast<uint4*>(filt);
    uint32_t n4 = a.has_long ? a.filter_words / 4 : 0;
    for (uint32_t k = threadIdx.x; k < n4; k += kThreads) dst[k] = __ldg(src + k);
    const uint4* bs = reinterpret_cast<const uint4*>(a.bloom);
    uint4* bd = reinterpret_cast<uint4*>(bloom);
    for (uint32_t k = threadIdx.x; k < (1u << (kBloomBits - 7)); k += kThreads) bd[k] = __ldg(bs + k);
    if (a.has_short) {
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
  const uint64_t nvec = (a.len + 15) / 16;
  const uint64_t nblk = (nvec + 31) / 32;  // 512-byte warp blocks
  const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + warp;
  const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;

  uint64_t b = gwarp;
  uint4 cur = make_uint4(0, 0, 0, 0);
  if (b < nblk) {
    uint64_t v = b * 32 + lane;
    cur = (v < nvec) ? load_vec(a.data, a.len, v) : make_uint4(0, 0, 0, 0);
  }
  for (; b < nblk; b += nwarps) {
    // software pipeline: the next block's load is in flight during this one
    uint64_t bn = b + nwarps;
    uint4 nxt = make_uint4(0, 0, 0, 0);
    if (bn < nblk) {
      uint64_t vn = bn * 32 + lane;
      nxt = (vn < nvec) ? load_vec(a.data, a.len, vn) : make_uint4(0, 0, 0, 0);
    }
    const uint64_t v = b * 32 + lane;
    uint4 tail = make_uint4(0, 0, 0, 0);
    if (lane == 31 && v + 1 < nvec) tail = load_vec(a.data, a.len, v + 1);
    reinterpret_cast<uint4*>(blk)[lane] = cur;
    if (lane == 31) {
      reinterpret_cast<uint4*>(blk)[32] = tail;
      blk[132] = 0;
      blk[133] = 0;
    }
    uint32_t w[8] = {cur.x, cur.y, cur.z, cur.w, __shfl_down_sync(0xFFFFFFFFu, cur.x, 1), 0, 0, 0};
    if (a.gram_len > 4) {
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
    uint32_t mask = stage1(a, filt, shortb, w, lane);
    const uint64_t blk_base = b * 512;
    const uint64_t base = v * 16;
    if (base + 16 > a.len) {
      uint64_t valid = a.len > base ? a.len - base : 0;
      mask &= (valid >= 16) ? 0xFFFFu : ((1u << valid) - 1u);
    }
    // compact the candidates of the warp into the queue
    uint32_t cnt = __popc(mask);
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
      uint32_t k = k0 + lane;
      bool keep = false;
      uint32_t off = 0;
      if (k < total) {
        off = queue[k];
        uint32_t wi = off >> 2, sh = (off & 3) * 8;
        uint32_t x0 = blk[wi], x1 = blk[wi + 1], x2 = blk[wi + 2];
        uint32_t lo = __funnelshift_r(x0, x1, sh), hi = __funnelshift_r(x1, x2, sh);
#pragma unroll
        for (uint32_t pl = 1; pl <= 8; ++pl) {
          if ((a.parts >> (pl - 1)) & 1u) {
            uint32_t key = prefix_key(lo, hi, pl);
            keep |= (bloom[key >> 5] >> (key & 31)) & 1u;
          }
        }
        if (keep && a.bloom2) {
          // stage 1.5b: the first min(len, 16) bytes against the L2 bitmap
          uint32_t x3 = blk[wi + 3], x4 = blk[wi + 4];
          uint32_t y2 = __funnelshift_r(x2, x3, sh), y3 = __funnelshift_r(x3, x4, sh);
          bool k2 = false;
          for (uint32_t pl = 1; pl <= 16; ++pl) {
            if ((a.parts16 >> (pl - 1)) & 1u) {
              uint32_t key = prefix16_key(lo, hi, y2, y3, pl);
              k2 |= (__ldg(a.bloom2 + (key >> 5)) >> (key & 31)) & 1u;
            }
          }
          keep = k2;
        }
      }
      uint32_t ball = __ballot_sync(0xFFFFFFFFu, keep);
      if (ball) {
        unsigned long long wbase = 0;
        if (lane == 0) wbase = atomicAdd(a.survivor_count, (unsigned long long)__popc(ball));
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
        if (keep) {
          unsigned long long slot = wbase + __popc(ball & ((1u << lane) - 1u));
          uint64_t s = blk_base + off;
          if (slot < a.survivor_cap) a.survivors[slot] = (uint32_t)s;
          else verify_position(a, s);  // list full: verify in place
        }
      }
    }
    __syncwarp();
    cur = nxt;
  }
}

__global__ void __launch_bounds__(256) literal_verify_kernel(LitArgs a) {
  unsigned long long n = *a.survivor_count;
  if (n > a.survivor_cap) n = a.survivor_cap;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x)
    verify_position(a, a.survivors[k]);
}

}  // namespace

size_t literal_smem_bytes(const LiteralPlan& plan) {
  return (plan.filter.size() + (1u << (kBloomBits - 5)) + (plan.has_short ? 2048 : 0) +
          (size_t)kWarps * (kBlockWords + kQueue / 2)) * 4;
}

size_t literal_scratch_bytes(uint64_t survivor_cap) { return 64 + survivor_cap * 4; }

void launch_literal_scan(const LiteralPlan& plan, const LiteralLaunch& l, cudaStream_t st, int sm_count) {
  if (plan.n_literals == 0 || l.len == 0) return;
  LitArgs a;
  a.data = l.data;
  a.len = l.len;
  a.filter = plan.d_filter.as<uint32_t>();
  a.filter_words = (uint32_t)plan.filter.size();
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
  check_cuda(cudaMemsetAsync(a.survivor_count, 0, 8, st), "memset survivors");
  size_t smem = literal_smem_bytes(plan);
  check_cuda(cudaFuncSetAttribute(literal_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute(literal)");
  uint64_t nblk = ((l.len + 15) / 16 + 31) / 32;
  uint64_t want = (nblk + kWarps - 1) / kWarps;
  int grid = (int)std::min<uint64_t>((uint64_t)sm_count, std::max<uint64_t>(want, 1));
  literal_filter_kernel<<<grid, kThreads, smem, st>>>(a);
  check_cuda(cudaGetLastError(), "literal_filter_kernel launch");
  literal_verify_kernel<<<sm_count * 4, 256, 0, st>>>(a);
  check_cuda(cudaGetLastError(), "literal_verify_kernel launch");
}

}  // namespace ws
