// Proposer inference on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One persistent CTA per SM (512 threads) runs tiles of 256 chunk boundaries:
//   1. the 16 context bytes of every boundary are mapped to joint class ids
//      and their 16-wide BF16 embeddings are written into shared memory as the
//      A operand (256 rows x 256 K, K-major, no swizzle: 8-row x 16-byte core
//      matrices, 128 B apart along K, 4 KiB apart along rows);
//   2. every GEMM of the MLP -- hidden layer 1 (N = 256), hidden layer 2
//      (N = 256) and the heads (all groups' 64 outputs, in chunks of up to 256
//      columns) -- runs as K slices of 64: a bulk async copy (cp.async.bulk,
//      completion on an mbarrier) brings the slice's pre-packed weights into
//      one of two shared-memory slots while the tensor cores work on the other;
//      one thread issues 2 x 4 tcgen05.mma (M = 128, K = 16 each: two 128-row
//      halves into two FP32 accumulators of 256 TMEM columns each) and commits
//      them to the slot's mbarrier, which frees the slot for the next copy;
//   3. after a GEMM's last commit, all 16 warps read the accumulators back
//      with tcgen05.ld (warp w reads TMEM lanes 32*(w%4).., one row per
//      thread, 128 columns per warp group) and apply bias + GELU (tanh form)
//      into the next A operand, or, for the heads, take each group's arg-max
//      and write the guessed state.
// Every mbarrier wait is bounded; on a time-out the CTA records an error,
// drains what it issued and frees its TMEM.  Results stay exact whatever the
// guesses hold: the walk treats an out-of-range guess as the unanchored start
// and the fix-up re-walks every chunk whose guess was wrong.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "ws_async.h"
#include "ws_proposer.h"

namespace ws {

namespace {

constexpr int kTcRows = 256;           // boundaries per tile
constexpr int kTcThreads = 512;
constexpr uint32_t kAStride = 4096;    // bytes between 8-row groups of A (32 k8 blocks x 128 B)
constexpr uint32_t kABytes = kTcRows * kPropHid * 2;   // 128 KiB
constexpr uint32_t kSlotBytes = 256 * 64 * 2;          // 32 KiB: one K slice of a 256-column GEMM
constexpr uint32_t kSlots = 2;                         // weight slots: one copy in flight ahead of the MMAs
constexpr uint32_t kBarBytes = 64;                     // mbarriers, TMEM address, abort flag
// per-CTA constants staged once: b1, b2 (FP32), the joint-class map and the
// embedding table (at most 64 classes x 16 BF16); then the head biases and
// guessed states of the head GEMM in flight (256 columns each), staged per
// head GEMM
constexpr uint32_t kConstBytes = 2 * 256 * 4 + 256 + 64 * kPropEmb * 2 + 2 * 256 * 4;
constexpr uint32_t kTcSmem = kABytes + kSlots * kSlotBytes + kBarBytes + kConstBytes;
constexpr uint32_t kWaitSpins = 1u << 24;

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1 (sm_100): start >> 4 in bits 0-13, leading byte offset
// (between the two 8-element K halves of an instruction) >> 4 in 16-29,
// stride byte offset (between 8-row groups) >> 4 in 32-45.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t idesc_bf16(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// Bounded wait; false (and the abort flag set) after kWaitSpins polls, or
// when another thread has aborted.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t it = 0; it < kWaitSpins; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255u) == 255u && *abort) return false;
  }
  *abort = 1;
  return false;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  mbar_expect_tx(bar, bytes);
  bulk_copy_g2s(dst, src, bytes, bar);
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive accumulator columns of this thread's TMEM lane, without
// waiting (tmem_wait() before the registers are used).
__device__ __forceinline__ void tmem_ld32_nw(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// GELU in the tanh form of Hendrycks and Gimpel (the form training uses), with
// the hardware tanh approximation (tanh.approx.f32).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanh_hw(u));
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16(a)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16(b)) << 16);
}

// Byte offset of A element (row, col) in the K-major core-matrix layout.
__device__ __forceinline__ uint32_t a_off(uint32_t row, uint32_t col) {
  return (row >> 3) * kAStride + (col >> 3) * 128 + (row & 7) * 16 + (col & 7) * 2;
}

struct TcArgs {
  const uint8_t* data;
  uint64_t chunk, n_chunks;
  const uint8_t* jmap;
  const __nv_bfloat16* E;       // [classes][16]
  uint32_t n_emb;               // classes (rows of E), at most 64
  const float* b1;
  const float* b2;
  const float* b3;              // [G * 64]
  const uint32_t* vocab;        // [G][64] guessed state per head output
  uint32_t G;
  uint32_t* guess;              // [G][n_chunks]
  const uint8_t* blob;          // packed weight slices of every GEMM
  uint32_t n_gemm;              // 2 hidden layers + head chunks
  uint16_t gemm_n[kTcMaxGemms];
  uint32_t gemm_off[kTcMaxGemms];  // byte offset of the GEMM's first slice in blob
  int* err;                     // set to 1 when a wait timed out
  // testing: one tile, A given row-major in global memory, one GEMM, raw
  // accumulators to d_test [256][N]
  const __nv_bfloat16* a_test;
  float* d_test;
};

__global__ void __launch_bounds__(kTcThreads, 1) proposer_tc_kernel(TcArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* A = sm;
  uint8_t* const slots = sm + kABytes;
  // bars[0..2]: slot filled, bars[3..5]: slot's MMAs done, bars[6]: GEMM done
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kABytes + kSlots * kSlotBytes);
  uint64_t* const full = bars;
  uint64_t* const done = bars + kSlots;
  uint64_t* const layer_bar = bars + 2 * kSlots;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * kSlots + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
  float* const b1s = reinterpret_cast<float*>(sm + kABytes + kSlots * kSlotBytes + kBarBytes);
  float* const b2s = b1s + 256;
  uint8_t* const jmap_s = reinterpret_cast<uint8_t*>(b2s + 256);
  uint8_t* const emb_s = jmap_s + 256;
  float* const b3s = reinterpret_cast<float*>(emb_s + 64 * kPropEmb * 2);
  uint32_t* const vocab_s = reinterpret_cast<uint32_t*>(b3s + 256);
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (a.a_test == nullptr) {
    for (uint32_t k = tid; k < 256; k += kTcThreads) {
      b1s[k] = a.b1[k];
      b2s[k] = a.b2[k];
      jmap_s[k] = a.jmap[k];
    }
    const uint32_t emb_words = min(a.n_emb, 64u) * kPropEmb / 8;  // uint4 words
    for (uint32_t k = tid; k < emb_words; k += kTcThreads)
      reinterpret_cast<uint4*>(emb_s)[k] = reinterpret_cast<const uint4*>(a.E)[k];
  }

  if (tid == 0) {
    for (uint32_t k = 0; k < 2 * kSlots + 1; ++k) mbar_init(&bars[k], 1);
    *abort = 0;
    mbar_init_fence();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = *tslot;

  const bool testing = a.a_test != nullptr;
  const uint64_t n_rows = testing ? kTcRows : (a.n_chunks > 1 ? a.n_chunks - 1 : 0);  // boundaries 1..n-1
  const uint32_t n_tiles = (uint32_t)((n_rows + kTcRows - 1) / kTcRows);
  const uint32_t my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t jobs_per_tile = 4 * a.n_gemm;
  const uint32_t total_jobs = my_tiles * jobs_per_tile;

  // job j (one K slice of one GEMM of one tile) uses slot j % kSlots; it is
  // that slot's (j / kSlots)-th fill and (j / kSlots)-th MMA batch
  auto issue_load = [&](uint32_t j) {
    const uint32_t g = (j % jobs_per_tile) >> 2, s = j & 3;
    const uint32_t bytes = (uint32_t)a.gemm_n[g] * 128;  // N rows x 64 K x 2 B
    bulk_load(slots + (j % kSlots) * kSlotBytes, a.blob + a.gemm_off[g] + s * bytes, bytes, &full[j % kSlots]);
  };

  uint32_t job = 0, issued = 0, layers = 0;
  if (tid == 0)
    for (; issued < kSlots - 1 && issued < total_jobs; ++issued) issue_load(issued);

  // the 8 context bytes of this thread's (row, half) of tile t: loaded one
  // tile ahead, so that the load overlaps the previous tile's GEMMs
  auto load_ctx = [&](uint32_t t) -> uint2 {
    const uint64_t i = (uint64_t)(blockIdx.x + t * gridDim.x) * kTcRows + 1 + (tid & (kTcRows - 1));
    if (testing || t >= my_tiles || i >= a.n_chunks) return make_uint2(0, 0);
    return *reinterpret_cast<const uint2*>(a.data + i * a.chunk - kPropCtx + (tid >> 8) * 8);
  };
  uint2 ctx_next = load_ctx(0);
  for (uint32_t t = 0; t < my_tiles && !*abort; ++t) {
    const uint64_t i0 = (uint64_t)(blockIdx.x + t * gridDim.x) * kTcRows + 1;  // first boundary of the tile
    // 1. A = embeddings of the context bytes (or the test operand): thread t
    //    takes row t % 256, context bytes 8 * (t / 256) .. +7 (one 8-byte load)
    {
      const uint32_t r = tid & (kTcRows - 1), kh = tid >> 8;
      if (testing) {
        for (uint32_t k = kh * 8; k < kh * 8 + 8; ++k) {
          const uint4* src = reinterpret_cast<const uint4*>(a.a_test + (size_t)r * kPropHid + k * 16);
          *reinterpret_cast<uint4*>(A + a_off(r, k * 16)) = src[0];
          *reinterpret_cast<uint4*>(A + a_off(r, k * 16 + 8)) = src[1];
        }
      } else {
        const uint64_t i = i0 + r;
        const uint2 ctx = ctx_next;  // class 0 pads the rows past the last boundary
        ctx_next = load_ctx(t + 1);
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
          const uint32_t byte = ((k < 4 ? ctx.x : ctx.y) >> (8 * (k & 3))) & 0xFFu;
          const uint32_t cid = i < a.n_chunks ? jmap_s[byte] : 0u;
          const uint4* src = reinterpret_cast<const uint4*>(emb_s + cid * kPropEmb * 2);
          const uint32_t col = (kh * 8 + k) * 16;
          *reinterpret_cast<uint4*>(A + a_off(r, col)) = src[0];
          *reinterpret_cast<uint4*>(A + a_off(r, col + 8)) = src[1];
        }
      }
    }
    fence_async_smem();
    fence_before();
    __syncthreads();

    for (uint32_t g = 0; g < a.n_gemm && !*abort; ++g) {
      const uint32_t N = a.gemm_n[g];
      // 2. the GEMM: four K slices, weights streamed through the slot ring
      if (tid == 0) {
        fence_after();
        const uint32_t idesc = idesc_bf16(N);
        for (uint32_t s = 0; s < 4; ++s) {
          const uint32_t j = job;
          if (!mbar_wait(&full[j % kSlots], (j / kSlots) & 1, abort)) break;
          fence_after();
          const uint32_t sb = smem_u32(slots + (j % kSlots) * kSlotBytes);
          const uint32_t sa = smem_u32(A);
#pragma unroll
          for (uint32_t kk = 0; kk < 4; ++kk) {
            const uint32_t koff = (s * 8 + kk * 2) * 128;
            const uint64_t bd = smem_desc(sb + kk * 2 * 128, 128, 1024);
            mma_bf16_ss(tbase, smem_desc(sa + koff, 128, kAStride), bd, idesc, (s | kk) != 0);
            mma_bf16_ss(tbase + 256, smem_desc(sa + 16 * kAStride + koff, 128, kAStride), bd, idesc, (s | kk) != 0);
          }
          mma_commit(&done[j % kSlots]);
          ++job;
          // keep kSlots - 1 copies ahead: a slot is refilled once the MMAs of
          // its previous job (kSlots jobs back) are done
          if (issued < total_jobs && issued < job + kSlots - 1) {
            const uint32_t L = issued;
            if (L >= kSlots && !mbar_wait(&done[L % kSlots], ((L - kSlots) / kSlots) & 1, abort)) break;
            issue_load(L);
            ++issued;
          }
        }
        if (!*abort) mma_commit(layer_bar);
      }
      if (g >= 2 && !testing) {
        // the head biases and guessed states of this GEMM's (up to) four groups
        const uint32_t c = tid & 255, grp = (g - 2) * 4 + c / kPropVocab;
        if (c < N && grp < a.G) {
          if (tid < 256) b3s[c] = __ldg(a.b3 + grp * kPropVocab + c % kPropVocab);
          else vocab_s[c] = __ldg(a.vocab + grp * kPropVocab + c % kPropVocab);
        }
        __syncthreads();
      }
      // 3. epilogue, all threads
      // warp-uniform: the tcgen05.ld below are warp-collective
      const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait(layer_bar, layers & 1, abort));
      ++layers;
      fence_after();
      if (ok) {
        const uint32_t q = warp & 3, wg = warp >> 2;
        const uint32_t half = wg >> 1, cpart = wg & 1;
        const uint32_t row = half * 128 + q * 32 + lane;
        const uint32_t tcol = tbase + ((q * 32) << 16) + half * 256 + cpart * 128;
        if (testing) {
          for (uint32_t c0 = 0; c0 < 128; c0 += 32) {
            float v[32];
            tmem_ld32(tcol + c0, v);
            for (int k = 0; k < 32; ++k) {
              const uint32_t col = cpart * 128 + c0 + k;
              if (col < N) a.d_test[(size_t)row * N + col] = v[k];
            }
          }
        } else if (g < 2) {
          const float* bias = g == 0 ? b1s : b2s;
          for (uint32_t c0 = 0; c0 < 128; c0 += 64) {
            uint32_t r0[32], r1[32];  // two loads in flight, one wait
            tmem_ld32_nw(tcol + c0, r0);
            tmem_ld32_nw(tcol + c0 + 32, r1);
            tmem_wait();
#pragma unroll
            for (int k8 = 0; k8 < 8; ++k8) {
              const uint32_t col = cpart * 128 + c0 + k8 * 8;
              const uint32_t* r = k8 < 4 ? r0 + k8 * 8 : r1 + (k8 - 4) * 8;
              const float4 bl = *reinterpret_cast<const float4*>(bias + col);
              const float4 bh = *reinterpret_cast<const float4*>(bias + col + 4);
              uint4 w;
              w.x = pack2(gelu_f(__uint_as_float(r[0]) + bl.x), gelu_f(__uint_as_float(r[1]) + bl.y));
              w.y = pack2(gelu_f(__uint_as_float(r[2]) + bl.z), gelu_f(__uint_as_float(r[3]) + bl.w));
              w.z = pack2(gelu_f(__uint_as_float(r[4]) + bh.x), gelu_f(__uint_as_float(r[5]) + bh.y));
              w.w = pack2(gelu_f(__uint_as_float(r[6]) + bh.z), gelu_f(__uint_as_float(r[7]) + bh.w));
              *reinterpret_cast<uint4*>(A + a_off(row, col)) = w;
            }
          }
          fence_async_smem();
        } else {
          // heads: this thread's 128 columns hold two groups' 64 outputs
          const uint64_t i = i0 + row;
          for (uint32_t h2 = 0; h2 < 2; ++h2) {
            const uint32_t c_start = cpart * 128 + h2 * 64;
            const uint32_t grp = (g - 2) * 4 + cpart * 2 + h2;
            if (c_start + 64 > N || grp >= a.G) continue;
            float best = -3.0e38f;
            uint32_t bi = 0;
            const float* bias = b3s + c_start;
            for (uint32_t c0 = 0; c0 < 64; c0 += 32) {
              float v[32];
              tmem_ld32(tcol + h2 * 64 + c0, v);
#pragma unroll
              for (int k = 0; k < 32; ++k) {
                const float x = v[k] + bias[c0 + k];
                if (x > best) { best = x; bi = c0 + k; }  // first maximum: lowest index on ties
              }
            }
            if (i < a.n_chunks) a.guess[(uint64_t)grp * a.n_chunks + i] = vocab_s[c_start + bi];
          }
        }
      }
      fence_before();
      __syncthreads();
    }
  }

  // teardown: on an abort, let everything this CTA issued finish (bounded)
  if (tid == 0 && *abort) {
    *a.err = 1;
    mma_commit(layer_bar);  // arrives once every MMA issued so far is done
    for (uint32_t it = 0; it < kWaitSpins && !mbar_try(layer_bar, layers & 1); ++it) {
    }
    for (uint32_t j = job; j < issued; ++j)  // copies still in flight
      for (uint32_t it = 0; it < kWaitSpins && !mbar_try(&full[j % kSlots], (j / kSlots) & 1); ++it) {
      }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(512u) : "memory");
}

// W^T [N][256] (row n = output n) -> four K slices of N x 64 in the B layout
// (K-major core matrices: 128 B apart along K, 1 KiB apart along N).
__global__ void tc_pack_kernel(const __nv_bfloat16* WT, uint32_t N, __nv_bfloat16* out) {
  const uint32_t total = N * kPropHid;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const uint32_t n = idx / kPropHid, k = idx % kPropHid;
    const uint32_t s = k >> 6, kk = k & 63;
    const uint32_t o = s * N * 64 + ((n >> 3) * 8 + (kk >> 3)) * 64 + (n & 7) * 8 + (kk & 7);
    out[o] = WT[idx];
  }
}

}  // namespace

void tc_prepare(TcPlan& tp, const void* W1T, const void* W2T, const void* W3T, uint32_t n_out) {
  tp.ready = false;
  const uint32_t n_head = (n_out + 255) / 256;
  if (2 + n_head > (uint32_t)kTcMaxGemms || n_out % 64 != 0) return;  // too many groups: mma.sync path
  tp.n_gemm = 2 + n_head;
  uint64_t off = 0;
  for (uint32_t g = 0; g < tp.n_gemm; ++g) {
    const uint32_t N = g < 2 ? 256 : std::min<uint32_t>(256, n_out - (g - 2) * 256);
    tp.gemm_n[g] = (uint16_t)N;
    tp.gemm_off[g] = (uint32_t)off;
    off += (uint64_t)N * kPropHid * 2;
  }
  tp.blob.alloc(off);
  auto* out = tp.blob.as<__nv_bfloat16>();
  tc_pack_kernel<<<256, 256>>>(static_cast<const __nv_bfloat16*>(W1T), 256, out);
  tc_pack_kernel<<<256, 256>>>(static_cast<const __nv_bfloat16*>(W2T), 256, out + tp.gemm_off[1] / 2);
  for (uint32_t g = 2; g < tp.n_gemm; ++g)
    tc_pack_kernel<<<256, 256>>>(static_cast<const __nv_bfloat16*>(W3T) + (size_t)(g - 2) * 256 * kPropHid,
                                 tp.gemm_n[g], out + tp.gemm_off[g] / 2);
  check_cuda(cudaGetLastError(), "tc_pack_kernel");
  tp.err.alloc(64);
  check_cuda(cudaMemset(tp.err.ptr, 0, 64), "memset");
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  check_cuda(cudaDeviceGetAttribute(&tp.sm_count, cudaDevAttrMultiProcessorCount, dev), "sm count");
  check_cuda(cudaFuncSetAttribute(proposer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem),
             "cudaFuncSetAttribute(proposer_tc)");
  check_cuda(cudaDeviceSynchronize(), "tc_prepare");
  tp.ready = true;
}

uint32_t tc_predict(const TcPlan& tp, const TcInputs& in, cudaStream_t st) {
  const uint64_t rows = in.n_chunks > 1 ? in.n_chunks - 1 : 0;
  if (!rows) return 0;
  TcArgs a;
  std::memset(&a, 0, sizeof(a));
  a.data = in.data;
  a.chunk = in.chunk;
  a.n_chunks = in.n_chunks;
  a.jmap = in.jmap;
  a.E = static_cast<const __nv_bfloat16*>(in.E);
  a.n_emb = in.n_emb;
  a.b1 = in.b1;
  a.b2 = in.b2;
  a.b3 = in.b3;
  a.vocab = in.vocab;
  a.G = in.G;
  a.guess = in.guess;
  a.blob = tp.blob.as<uint8_t>();
  a.n_gemm = tp.n_gemm;
  for (uint32_t g = 0; g < tp.n_gemm; ++g) {
    a.gemm_n[g] = tp.gemm_n[g];
    a.gemm_off[g] = tp.gemm_off[g];
  }
  a.err = tp.err.as<int>();
  const uint64_t tiles = (rows + kTcRows - 1) / kTcRows;
  const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)tp.sm_count);
  proposer_tc_kernel<<<grid, kTcThreads, kTcSmem, st>>>(a);
  check_cuda(cudaGetLastError(), "proposer_tc_kernel");
  return 1;
}

}  // namespace ws

// Testing hook (not part of the public header): one 256 x 256 x N BF16 GEMM
// through the tcgen05 path of the proposer kernel.  A [256][256] row-major,
// WT [N][256] (row n holds output n's weights), D [256][N] FP32; device
// pointers.  Returns 0 on success.
extern "C" int ws_testing_tc_gemm(const void* A, const void* WT, int N, float* D) {
  using namespace ws;
  try {
    if (N <= 0 || N > 256 || N % 16 != 0) return 2;
    TcPlan tp;
    tp.n_gemm = 1;
    tp.gemm_n[0] = (uint16_t)N;
    tp.gemm_off[0] = 0;
    tp.blob.alloc((size_t)N * kPropHid * 2);
    tc_pack_kernel<<<64, 256>>>(static_cast<const __nv_bfloat16*>(WT), (uint32_t)N, tp.blob.as<__nv_bfloat16>());
    tp.err.alloc(64);
    check_cuda(cudaMemset(tp.err.ptr, 0, 64), "memset");
    check_cuda(cudaFuncSetAttribute(proposer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem),
               "cudaFuncSetAttribute(proposer_tc)");
    TcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n_gemm = 1;
    a.gemm_n[0] = (uint16_t)N;
    a.gemm_off[0] = 0;
    a.blob = tp.blob.as<uint8_t>();
    a.err = tp.err.as<int>();
    a.a_test = static_cast<const __nv_bfloat16*>(A);
    a.d_test = D;
    proposer_tc_kernel<<<1, kTcThreads, kTcSmem>>>(a);
    check_cuda(cudaGetLastError(), "proposer_tc_kernel(test)");
    check_cuda(cudaDeviceSynchronize(), "tc test");
    int e = 0;
    check_cuda(cudaMemcpy(&e, tp.err.ptr, 4, cudaMemcpyDeviceToHost), "D2H");
    return e ? 3 : 0;
  } catch (...) {
    return 1;
  }
}
