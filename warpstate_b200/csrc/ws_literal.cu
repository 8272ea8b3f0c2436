// Fused literal prefilter + verify for sm_100a.
//
// Replaces the reference's two WGSL passes, literal_prefilter
// (core/src/gpu/shader.rs:18-101) and literal_verify (core/src/gpu/shader.rs:106-236),
// with one persistent kernel:
//
//   stage 1  every thread owns 16 input bytes per step, read with one 16-byte
//            coalesced load (the next thread's first word comes by shuffle).
//            It looks up the 4-byte grams at the P-aligned positions in a
//            nibble table staged in shared memory and forms a 16-bit mask of the
//            positions that may start a literal (see LiteralPlan).
//   compact  ballot/popc prefix sums place the surviving positions of the warp
//            in a shared-memory queue, so stage 2 runs with all 32 lanes busy.
//   stage 2  the reference's per-position algorithm on the queued positions:
//            FNV-1a over up to hash_window_len bytes, a probe of the
//            LiteralPrefilterTable partition at every non-empty prefix length
//            (shader.rs:59-98), and an exact compare of every entry whose hash
//            is equal (shader.rs:174-227).  Matches are appended with one
//            atomic per match (true count kept for overflow reporting).
//
// The output is contract L: every overlapping occurrence of every literal, the
// same set the reference's GPU literal path returns.
#include <cuda_runtime.h>

#include "ws_internal.h"

namespace ws {

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kUnroll = 4;          // 16-byte vectors in flight per thread
constexpr int kQueue = 32 * 16;     // worst case of one vector step of a warp

struct LitArgs {
  const uint8_t* data;
  uint64_t len;
  const uint32_t* filter;
  uint32_t filter_words;
  uint32_t bits;
  uint32_t period;
  uint32_t has_long;
  uint32_t has_short;
  const uint32_t* short_bits;
  const uint4* info;
  const uint8_t* lit_bytes;
  const uint4* meta;
  const uint2* ranges;
  const uint2* entries;
  uint32_t window;
  ws_match* out;
  uint64_t cap;
  unsigned long long* counter;
};

__device__ __forceinline__ uint32_t nib(const uint32_t* tab, uint32_t gram, uint32_t bits) {
  uint32_t h = (gram * 0x9E3779B1u) >> (32 - bits);
  return (tab[h >> 3] >> ((h & 7) * 4)) & 0xFu;
}

// Loads the 16 bytes of vector v, zero-filling past the end of the input.
__device__ __forceinline__ uint4 load_vec(const uint8_t* data, uint64_t len, uint64_t v) {
  uint64_t off = v * 16;
  if (off + 16 <= len) return __ldg(reinterpret_cast<const uint4*>(data + off));
  uint32_t w[4] = {0, 0, 0, 0};
  for (int k = 0; k < 16; ++k) {
    uint64_t p = off + k;
    if (p < len) w[k >> 2] |= (uint32_t)__ldg(data + p) << ((k & 3) * 8);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ uint32_t load_word(const uint8_t* data, uint64_t len, uint64_t off) {
  if (off + 4 <= len) {
    if ((off & 3) == 0) return __ldg(reinterpret_cast<const uint32_t*>(data + off));
  }
  uint32_t w = 0;
  for (int k = 0; k < 4; ++k)
    if (off + k < len) w |= (uint32_t)__ldg(data + off + k) << (k * 8);
  return w;
}

// Stage 2 for one position: the reference's FNV probe and exact verify.
__device__ void verify_position(const LitArgs& a, const uint4* meta_s, uint64_t s) {
  uint32_t h = 2166136261u;
  uint64_t rem = a.len - s;
  uint32_t maxp = (uint32_t)(rem < a.window ? rem : a.window);
  for (uint32_t i = 0; i < maxp; ++i) {
    h = (h ^ (uint32_t)__ldg(a.data + s + i)) * 16777619u;
    uint4 m = meta_s[i];
    if (m.z == 0) continue;
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

// 16-bit mask of the owned positions (bit i = byte 16v+i) that may start a literal.
__device__ __forceinline__ uint32_t candidate_mask(const LitArgs& a, const uint32_t* filt,
                                                   const uint32_t* shortb, uint4 w, uint32_t w4,
                                                   uint64_t v) {
  uint32_t words[5] = {w.x, w.y, w.z, w.w, w4};
  uint32_t mask = 0;
  if (a.has_long) {
    if (a.period == 4) {
      uint32_t m = 0;
#pragma unroll
      for (int j = 0; j < 5; ++j) m |= nib(filt, words[j], a.bits) << (4 * j);
      mask |= (m >> 3) & 0xFFFFu;
    } else if (a.period == 2) {
      uint32_t m = 0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        uint32_t g = (j & 1) ? __funnelshift_r(words[j >> 1], words[(j >> 1) + 1], 16) : words[j >> 1];
        m |= nib(filt, g, a.bits) << (2 * j);
      }
      mask |= (m >> 1) & 0xFFFFu;
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        uint32_t g = __funnelshift_r(words[j >> 2], words[(j >> 2) + 1], 8 * (j & 3));
        mask |= (nib(filt, g, a.bits) & 1u) << j;
      }
    }
  }
  if (a.has_short) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      uint32_t g = __funnelshift_r(words[j >> 2], words[(j >> 2) + 1], 8 * (j & 3)) & 0xFFFFu;
      mask |= ((shortb[g >> 5] >> (g & 31)) & 1u) << j;
    }
  }
  uint64_t base = v * 16;
  if (base + 16 > a.len) {
    uint64_t valid = a.len > base ? a.len - base : 0;
    mask &= (valid >= 16) ? 0xFFFFu : ((1u << valid) - 1u);
  }
  return mask;
}

__global__ void __launch_bounds__(kThreads, 1) literal_scan_kernel(LitArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* filt = smem;                                   // filter_words
  uint32_t* shortb = filt + a.filter_words;                // 2048 words
  uint4* meta_s = reinterpret_cast<uint4*>(shortb + 2048);  // window entries
  uint32_t* queues = reinterpret_cast<uint32_t*>(meta_s + 8);

  // Stage the tables (128-bit copies).
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.filter);
    uint4* dst = reinterpret_cast<uint4*>(filt);
    uint32_t n4 = a.has_long ? a.filter_words / 4 : 0;
    for (uint32_t k = threadIdx.x; k < n4; k += kThreads) dst[k] = __ldg(src + k);
    if (a.has_short) {
      const uint4* s2 = reinterpret_cast<const uint4*>(a.short_bits);
      uint4* d2 = reinterpret_cast<uint4*>(shortb);
      for (uint32_t k = threadIdx.x; k < 512; k += kThreads) d2[k] = __ldg(s2 + k);
    }
    if (threadIdx.x < 8) meta_s[threadIdx.x] = threadIdx.x < a.window ? __ldg(a.meta + threadIdx.x) : make_uint4(0, 0, 0, 0);
  }
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  uint32_t* q = queues + warp * kQueue;
  const uint64_t nvec = (a.len + 15) / 16;
  const uint64_t nblk = (nvec + 31) / 32;  // 512-byte warp blocks
  const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + warp;
  const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;

  for (uint64_t b0 = gwarp * kUnroll; b0 < nblk; b0 += nwarps * kUnroll) {
    uint4 w[kUnroll];
    uint32_t w4[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      uint64_t v = (b0 + u) * 32 + lane;
      w[u] = (v < nvec) ? load_vec(a.data, a.len, v) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      uint64_t v = (b0 + u) * 32 + lane;
      uint32_t nx = __shfl_down_sync(0xFFFFFFFFu, w[u].x, 1);
      if (lane == 31) nx = ((v + 1) * 16 < a.len) ? load_word(a.data, a.len, (v + 1) * 16) : 0u;
      w4[u] = nx;
    }
#pragma unroll 1
    for (int u = 0; u < kUnroll; ++u) {
      uint64_t v = (b0 + u) * 32 + lane;
      uint32_t mask = (v < nvec) ? candidate_mask(a, filt, shortb, w[u], w4[u], v) : 0u;
      uint32_t cnt = __popc(mask);
      // warp exclusive prefix sum of cnt
      uint32_t incl = cnt;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += y;
      }
      uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
      if (total == 0) continue;
      uint32_t pos = incl - cnt;
      uint32_t base = (uint32_t)(v * 16 - ((b0 + u) * 32) * 16);  // = lane*16
      while (mask) {
        int bit = __ffs(mask) - 1;
        mask &= mask - 1;
        q[pos++] = base + (uint32_t)bit;
      }
      __syncwarp();
      const uint64_t blk_base = (b0 + u) * 512;
      for (uint32_t k = lane; k < total; k += 32) verify_position(a, meta_s, blk_base + q[k]);
      __syncwarp();
    }
  }
}

}  // namespace

size_t literal_smem_bytes(const LiteralPlan& plan) {
  return (plan.filter.size() + 2048) * 4 + 8 * 16 + (size_t)kWarps * kQueue * 4;
}

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
  a.short_bits = plan.d_short.as<uint32_t>();
  a.info = plan.d_info.as<uint4>();
  a.lit_bytes = plan.d_bytes.as<uint8_t>();
  a.meta = plan.d_meta.as<uint4>();
  a.ranges = plan.d_ranges.as<uint2>();
  a.entries = plan.d_entries.as<uint2>();
  a.window = HASH_WINDOW;
  a.out = l.out;
  a.cap = l.cap;
  a.counter = l.counter;
  size_t smem = literal_smem_bytes(plan);
  static bool attr_set = false;
  if (!attr_set) {
    check_cuda(cudaFuncSetAttribute(literal_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "cudaFuncSetAttribute(literal)");
    attr_set = true;
  }
  uint64_t nblk = ((l.len + 15) / 16 + 31) / 32;
  uint64_t want = (nblk + (uint64_t)kWarps * kUnroll - 1) / ((uint64_t)kWarps * kUnroll);
  int grid = (int)std::min<uint64_t>((uint64_t)sm_count, std::max<uint64_t>(want, 1));
  literal_scan_kernel<<<grid, kThreads, smem, st>>>(a);
  check_cuda(cudaGetLastError(), "literal_scan_kernel launch");
}

}  // namespace ws
