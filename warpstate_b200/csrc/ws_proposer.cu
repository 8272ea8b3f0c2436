// Learned boundary-state proposer: training and inference kernels (sm_100a).
//
// All matrix products use mma.sync.m16n8k16 with BF16 operands and FP32
// accumulation.  Training: Adam on FP32 master weights with BF16 copies for
// the products.  Inference: one fused kernel per 64-boundary tile (embedding
// gather, two GELU layers and the per-group heads with arg-max, activations in
// shared memory).  GELU calls CUDA's erff (exact form x * Phi(x)).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>

#include "ws_dfa.h"
#include "ws_proposer.h"

namespace ws {

namespace {

constexpr uint32_t F_MASK = 0x3FFFFFFFu;

// ---------------------------------------------------------- mma helpers
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// GELU in the tanh form of Hendrycks and Gimpel (2016):
// 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), through CUDA's tanhf; the
// tensor-core inference kernel evaluates the same form with the hardware
// tanh approximation.
constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + tanhf(kGeluC * (x + kGeluA * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float t = tanhf(kGeluC * (x + kGeluA * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * x * x);
}

// ------------------------------------------------------ generic GEMM
// C[m][n] = alpha * sum_k A(m,k) * B(k,n) + beta * C[m][n]; A(m,k) =
// A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn] (BF16), C row-major FP32 with
// leading dimension ldc.  64x64 tiles, K steps of 32, 4 warps of 32x32.
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __nv_bfloat16* A, int64_t sam, int64_t sak,
                                                        const __nv_bfloat16* B, int64_t sbk, int64_t sbn, float* C,
                                                        int64_t ldc, int M, int N, int K, float alpha, float beta) {
  __shared__ __nv_bfloat16 As[64][40];
  __shared__ __nv_bfloat16 Bs[64][40];  // [n][k]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < K; k0 += 32) {
    for (int idx = tid; idx < 64 * 32; idx += 128) {
      int r = idx / 32, c = idx % 32;
      int m = m0 + r, k = k0 + c;
      As[r][c] = (m < M && k < K) ? A[(int64_t)m * sam + (int64_t)k * sak] : zero;
      int n = n0 + r;
      Bs[r][c] = (n < N && k < K) ? B[(int64_t)k * sbk + (int64_t)n * sbn] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 32; kk += 16) {
      uint32_t a[2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        int r = wm + i * 16;
        a[i][0] = *reinterpret_cast<const uint32_t*>(&As[r + g][kk + 2 * t]);
        a[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + g + 8][kk + 2 * t]);
        a[i][2] = *reinterpret_cast<const uint32_t*>(&As[r + g][kk + 2 * t + 8]);
        a[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + g + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int n = wn + j * 8 + g;
        uint32_t b0 = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * t]);
        uint32_t b1 = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * t + 8]);
#pragma unroll
        for (int i = 0; i < 2; ++i) mma_bf16(acc[i][j], a[i], b0, b1);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int m = m0 + wm + i * 16 + g + h * 8;
        int n = n0 + wn + j * 8 + 2 * t;
        if (m >= M) continue;
        for (int q = 0; q < 2; ++q) {
          if (n + q >= N) continue;
          float v = alpha * acc[i][j][h * 2 + q];
          float* dst = C + (int64_t)m * ldc + n + q;
          *dst = (beta != 0.f) ? v + beta * *dst : v;
        }
      }
}

void gemm(const __nv_bfloat16* A, int64_t sam, int64_t sak, const __nv_bfloat16* B, int64_t sbk, int64_t sbn,
          float* C, int64_t ldc, int M, int N, int K, float alpha, float beta, cudaStream_t st) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  gemm_bf16_kernel<<<grid, 128, 0, st>>>(A, sam, sak, B, sbk, sbn, C, ldc, M, N, K, alpha, beta);
  check_cuda(cudaGetLastError(), "gemm_bf16_kernel");
}

// ------------------------------------------------------ training kernels
struct GroupWalk {
  const GroupDev* groups;
  const uint32_t* fwd;
  const uint8_t* cls;
  uint32_t G;
};

// Exact DFA state at each sampled position: the unanchored walk of the
// `lookback` bytes before it (exact once every thread older than the longest
// match has died) plus the joint-class context.
__global__ void sample_kernel(GroupWalk gw, const uint8_t* data, uint64_t len, const uint64_t* pos, uint32_t n,
                              const uint8_t* jmap, uint32_t lookback, uint8_t* ctx, uint32_t* state) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint64_t p = pos[j];
  for (int k = 0; k < kPropCtx; ++k) ctx[(uint64_t)j * kPropCtx + k] = jmap[data[p - kPropCtx + k]];
  uint64_t a = p > lookback ? p - lookback : 0;
  for (uint32_t g = 0; g < gw.G; ++g) {
    const GroupDev gd = gw.groups[g];
    const uint32_t* tab = gw.fwd + gd.fwd_off;
    const uint8_t* cm = gw.cls + g * 256;
    uint32_t st = gd.start_unanchored;
    for (uint64_t q = a; q < p; ++q) st = __ldg(tab + st * gd.n_classes + cm[data[q]]) & F_MASK;
    state[(uint64_t)j * gw.G + g] = st;
  }
}

__global__ void embed_kernel(const uint8_t* ctx, const __nv_bfloat16* E, __nv_bfloat16* X, uint32_t B) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * kPropHid) return;
  uint32_t b = idx / kPropHid, c = idx % kPropHid;
  uint32_t k = c / kPropEmb, d = c % kPropEmb;
  X[idx] = E[ctx[b * kPropCtx + k] * kPropEmb + d];
}

// Z += bias; H = bf16(GELU(Z)) (Z keeps the pre-activation for backward)
__global__ void bias_gelu_kernel(float* Z, const float* bias, __nv_bfloat16* H, uint32_t B, uint32_t N) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * N) return;
  float z = Z[idx] + bias[idx % N];
  Z[idx] = z;
  H[idx] = __float2bfloat16(gelu(z));
}

// softmax cross-entropy per (row, group) over kPropVocab logits; writes
// dlogits (bf16) = (softmax - onehot) / B and accumulates the loss.
__global__ void ce_kernel(const float* logits, const float* bias, const uint8_t* labels, uint32_t B, uint32_t G,
                          __nv_bfloat16* dlog, float* dbias_acc, float* loss) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;  // (row, group)
  if (idx >= B * G) return;
  uint32_t b = idx / G, g = idx % G;
  const float* l = logits + (uint64_t)b * G * kPropVocab + g * kPropVocab;
  const float* bb = bias + g * kPropVocab;
  float mx = -1e30f;
  for (int v = 0; v < kPropVocab; ++v) mx = fmaxf(mx, l[v] + bb[v]);
  float sum = 0.f;
  for (int v = 0; v < kPropVocab; ++v) sum += expf(l[v] + bb[v] - mx);
  uint32_t y = labels[b * G + g];
  atomicAdd(loss, (logf(sum) + mx - (l[y] + bb[y])) / (float)B);
  __nv_bfloat16* d = dlog + (uint64_t)b * G * kPropVocab + g * kPropVocab;
  for (int v = 0; v < kPropVocab; ++v) {
    float p = expf(l[v] + bb[v] - mx) / sum;
    float gr = (p - (v == (int)y ? 1.f : 0.f)) / (float)B;
    d[v] = __float2bfloat16(gr);
    atomicAdd(&dbias_acc[g * kPropVocab + v], gr);
  }
}

// dZ = dH * GELU'(Z) (bf16 for the next products) and the bias gradient
__global__ void gelu_back_kernel(const float* dH, const float* Z, __nv_bfloat16* dZ, float* dbias, uint32_t B,
                                 uint32_t N) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * N) return;
  float d = dH[idx] * gelu_grad(Z[idx]);
  dZ[idx] = __float2bfloat16(d);
  atomicAdd(&dbias[idx % N], d);
}

__global__ void embed_back_kernel(const uint8_t* ctx, const float* dX, float* dE, uint32_t B) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * kPropHid) return;
  uint32_t b = idx / kPropHid, c = idx % kPropHid;
  uint32_t k = c / kPropEmb, d = c % kPropEmb;
  atomicAdd(&dE[ctx[b * kPropCtx + k] * kPropEmb + d], dX[idx]);
}

__global__ void adam_kernel(float* w, const float* gr, float* m, float* v, __nv_bfloat16* w16, uint32_t n, float lr,
                            float b1, float b2, float c1, float c2) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float g = gr[i];
  float mi = b1 * m[i] + (1.f - b1) * g;
  float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
  w[i] = wi;
  if (w16) w16[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float* a, __nv_bfloat16* b, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16(a[i]);
}

// W[K][N] (fp32) -> WT[N][K] (bf16) for the inference kernel
__global__ void transpose_bf16_kernel(const float* W, __nv_bfloat16* WT, uint32_t K, uint32_t N) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K * N) return;
  uint32_t k = i / N, n = i % N;
  WT[(uint64_t)n * K + k] = __float2bfloat16(W[i]);
}

// top-4 hit counting on held-out rows (logits + bias)
__global__ void eval_kernel(const float* logits, const float* bias, const uint8_t* labels, const uint8_t* is_start,
                            uint32_t B, uint32_t G, unsigned long long* hits) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * G) return;
  uint32_t b = idx / G, g = idx % G;
  const float* l = logits + (uint64_t)b * G * kPropVocab + g * kPropVocab;
  const float* bb = bias + g * kPropVocab;
  uint32_t y = labels[b * G + g];
  float ly = l[y] + bb[y];
  int rank = 0;
  for (int v = 0; v < kPropVocab; ++v) {
    float x = l[v] + bb[v];
    if (x > ly || (x == ly && v < (int)y)) ++rank;
  }
  // label kPropVocab-1 ("other") hits only when the true state is the start
  bool other = (y == kPropVocab - 1);
  bool ok = !other || is_start[b * G + g];
  if (ok && rank == 0) atomicAdd(&hits[0], 1ull);
  if (ok && rank < 4) atomicAdd(&hits[1], 1ull);
}

// ------------------------------------------------------ fused inference
constexpr int kTileRows = 64;
constexpr int kLd = kPropHid + 8;  // padded row (bf16 elements)
constexpr int kWk = 64;            // k columns of a staged weight slice
constexpr int kWld = kWk + 8;

struct InferArgs {
  const uint8_t* data;
  uint64_t chunk;
  uint64_t n_chunks;
  const uint8_t* jmap;
  const __nv_bfloat16* E;    // [n_jcls+1][16]
  const __nv_bfloat16* W1T;  // [256 out][256 in]
  const float* b1;
  const __nv_bfloat16* W2T;
  const float* b2;
  const __nv_bfloat16* W3T;  // [G*64 out][256 in]
  const float* b3;
  const uint32_t* vocab;     // [G][64] premultiplied states
  uint32_t G;
  uint32_t* guess;           // [G][n_chunks]
};

// One hidden layer: out = GELU(in . W + b), in/out [64][kLd] bf16 in shared
// memory, W^T streamed through `ws` in slices of kWk input columns.
__device__ void mlp_layer(const __nv_bfloat16* in, __nv_bfloat16* out, __nv_bfloat16* wsm,
                          const __nv_bfloat16* WT, const float* bias) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int rb = (warp & 3) * 16, cb = (warp >> 2) * 128;
  float acc[16][4];
#pragma unroll
  for (int j = 0; j < 16; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
  for (int k0 = 0; k0 < kPropHid; k0 += kWk) {
    // stage W^T[:, k0:k0+kWk] -> wsm[n][k]
    for (int idx = tid; idx < kPropHid * (kWk / 8); idx += blockDim.x) {
      int n = idx / (kWk / 8), c8 = idx % (kWk / 8);
      *reinterpret_cast<uint4*>(wsm + n * kWld + c8 * 8) =
          __ldg(reinterpret_cast<const uint4*>(WT + (size_t)n * kPropHid + k0 + c8 * 8));
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kWk; kk += 16) {
      uint32_t a[4];
      a[0] = *reinterpret_cast<const uint32_t*>(in + (rb + g) * kLd + k0 + kk + 2 * t);
      a[1] = *reinterpret_cast<const uint32_t*>(in + (rb + g + 8) * kLd + k0 + kk + 2 * t);
      a[2] = *reinterpret_cast<const uint32_t*>(in + (rb + g) * kLd + k0 + kk + 2 * t + 8);
      a[3] = *reinterpret_cast<const uint32_t*>(in + (rb + g + 8) * kLd + k0 + kk + 2 * t + 8);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const __nv_bfloat16* wr = wsm + (cb + j * 8 + g) * kWld + kk + 2 * t;
        uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr);
        uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + 8);
        mma_bf16(acc[j], a, b0, b1);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    int c = cb + j * 8 + 2 * t;
    float bz0 = bias[c], bz1 = bias[c + 1];
    *reinterpret_cast<uint32_t*>(out + (rb + g) * kLd + c) =
        pack_bf16(__float2bfloat16(gelu(acc[j][0] + bz0)), __float2bfloat16(gelu(acc[j][1] + bz1)));
    *reinterpret_cast<uint32_t*>(out + (rb + g + 8) * kLd + c) =
        pack_bf16(__float2bfloat16(gelu(acc[j][2] + bz0)), __float2bfloat16(gelu(acc[j][3] + bz1)));
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) proposer_infer_kernel(InferArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  __nv_bfloat16* X = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  __nv_bfloat16* H = X + kTileRows * kLd;
  __nv_bfloat16* Wsm = H + kTileRows * kLd;
  float* best_v = reinterpret_cast<float*>(Wsm + kPropHid * kWld);
  int* best_i = reinterpret_cast<int*>(best_v + 2 * kTileRows);
  const int tid = threadIdx.x;
  const uint64_t i0 = (uint64_t)blockIdx.x * kTileRows + 1;  // first boundary of the tile
  // embeddings of the 16 context bytes of every boundary
  for (int idx = tid; idx < kTileRows * kPropCtx; idx += blockDim.x) {
    int r = idx / kPropCtx, k = idx % kPropCtx;
    uint64_t i = i0 + r;
    uint32_t cid = 0;
    if (i < a.n_chunks) cid = a.jmap[a.data[i * a.chunk - kPropCtx + k]];
    const uint4* e = reinterpret_cast<const uint4*>(a.E + cid * kPropEmb);
    uint4* dst = reinterpret_cast<uint4*>(X + r * kLd + k * kPropEmb);
    dst[0] = __ldg(e);
    dst[1] = __ldg(e + 1);
  }
  __syncthreads();
  mlp_layer(X, H, Wsm, a.W1T, a.b1);
  mlp_layer(H, X, Wsm, a.W2T, a.b2);
  // heads: per group, 64 logits per row, arg-max -> guessed state
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int rb = (warp & 3) * 16, cb = (warp >> 2) * 32;
  for (uint32_t grp = 0; grp < a.G; ++grp) {
    const __nv_bfloat16* WT = a.W3T + (size_t)grp * kPropVocab * kPropHid;
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    for (int k0 = 0; k0 < kPropHid; k0 += kWk) {
      for (int idx = tid; idx < kPropVocab * (kWk / 8); idx += blockDim.x) {
        int n = idx / (kWk / 8), c8 = idx % (kWk / 8);
        *reinterpret_cast<uint4*>(Wsm + n * kWld + c8 * 8) =
            __ldg(reinterpret_cast<const uint4*>(WT + (size_t)n * kPropHid + k0 + c8 * 8));
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kWk; kk += 16) {
        uint32_t av[4];
        av[0] = *reinterpret_cast<const uint32_t*>(X + (rb + g) * kLd + k0 + kk + 2 * t);
        av[1] = *reinterpret_cast<const uint32_t*>(X + (rb + g + 8) * kLd + k0 + kk + 2 * t);
        av[2] = *reinterpret_cast<const uint32_t*>(X + (rb + g) * kLd + k0 + kk + 2 * t + 8);
        av[3] = *reinterpret_cast<const uint32_t*>(X + (rb + g + 8) * kLd + k0 + kk + 2 * t + 8);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const __nv_bfloat16* wr = Wsm + (cb + j * 8 + g) * kWld + kk + 2 * t;
          mma_bf16(acc[j], av, *reinterpret_cast<const uint32_t*>(wr), *reinterpret_cast<const uint32_t*>(wr + 8));
        }
      }
      __syncthreads();
    }
    const float* bias = a.b3 + grp * kPropVocab;
    // per-lane best over its columns for rows rb+g and rb+g+8
    float bv[2] = {-1e30f, -1e30f};
    int bi[2] = {0, 0};
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int c = cb + j * 8 + 2 * t + (q & 1);
        float v = acc[j][q] + bias[c];
        int h = q >> 1;
        if (v > bv[h] || (v == bv[h] && c < bi[h])) { bv[h] = v; bi[h] = c; }
      }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int off = 1; off < 4; off <<= 1) {
        float ov = __shfl_xor_sync(0xFFFFFFFFu, bv[h], off);
        int oi = __shfl_xor_sync(0xFFFFFFFFu, bi[h], off);
        if (ov > bv[h] || (ov == bv[h] && oi < bi[h])) { bv[h] = ov; bi[h] = oi; }
      }
    }
    if (t == 0) {
      int half = warp >> 2;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        best_v[half * kTileRows + rb + g + h * 8] = bv[h];
        best_i[half * kTileRows + rb + g + h * 8] = bi[h];
      }
    }
    __syncthreads();
    if (tid < kTileRows) {
      float v0 = best_v[tid], v1 = best_v[kTileRows + tid];
      int c = (v1 > v0 || (v1 == v0 && best_i[kTileRows + tid] < best_i[tid])) ? best_i[kTileRows + tid] : best_i[tid];
      uint64_t i = i0 + tid;
      if (i < a.n_chunks) a.guess[(uint64_t)grp * a.n_chunks + i] = a.vocab[grp * kPropVocab + c];
    }
    __syncthreads();
  }
}

constexpr size_t kInferSmem = (size_t)2 * kTileRows * kLd * 2 + (size_t)kPropHid * kWld * 2 + 2 * kTileRows * 8;

}  // namespace

struct Proposer {
  uint32_t G = 0;
  uint32_t n_jcls = 0;
  std::vector<uint8_t> jmap;
  DeviceBuffer d_jmap, d_vocab;
  // fp32 masters, Adam moments, bf16 copies
  DeviceBuffer E, W1, b1, W2, b2, W3, b3;
  DeviceBuffer mE, vE, mW1, vW1, mb1, vb1, mW2, vW2, mb2, vb2, mW3, vW3, mb3, vb3;
  DeviceBuffer E16, W1_16, W2_16, W3_16;
  DeviceBuffer W1T, W2T, W3T;  // inference copies [out][in]
  TcPlan tc;                   // the same weights packed for the tcgen05 kernel
  bool trained = false;
};

namespace {
// Inference path: the tcgen05 kernel when its weights are packed (default), or
// the mma.sync kernel (the testing hook below selects it, for comparisons).
bool g_use_tc = true;
}  // namespace

void proposer_destroy(Proposer* p) { delete p; }

namespace {

uint64_t splitmix(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void init_uniform(DeviceBuffer& b, size_t n, float scale, uint64_t& seed) {
  std::vector<float> h(n);
  for (auto& x : h) x = (float)(((double)(splitmix(seed) >> 11) / 9007199254740992.0) * 2.0 - 1.0) * scale;
  b.upload(h.data(), n * 4);
}

void zeros(DeviceBuffer& b, size_t n) {
  std::vector<float> h(n, 0.f);
  b.upload(h.data(), n * 4);
}

unsigned blocks(uint64_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void proposer_train(RegexPlan& P, const uint8_t* d_corpus, uint64_t len, uint64_t seed, int sm_count,
                    ProposerStats* stats) {
  (void)sm_count;
  if (!P.n_regex || P.n_spec == 0) return;  // context groups take no boundary guesses
  if (len < 65536) raise(WS_ERR_INVALID_ARGUMENT, "proposer training corpus must hold at least 64 KiB");
  const uint32_t G = P.n_spec;
  auto* pr = new Proposer();
  std::unique_ptr<Proposer> guard(pr);
  pr->G = G;
  // joint byte classes of all groups (ids >= 63 share id 62)
  {
    std::unordered_map<std::string, uint32_t> ids;
    pr->jmap.assign(256, 0);
    for (int b = 0; b < 256; ++b) {
      std::string key;
      for (uint32_t g = 0; g < G; ++g) key.push_back((char)P.cls[g * 256 + b]);
      auto it = ids.find(key);
      if (it == ids.end()) it = ids.emplace(key, (uint32_t)ids.size()).first;
      pr->jmap[b] = (uint8_t)std::min<uint32_t>(it->second, 62);
    }
    pr->n_jcls = std::min<uint32_t>((uint32_t)ids.size(), 63);
    pr->d_jmap.upload(pr->jmap.data(), 256);
  }
  const uint32_t n_emb = 64;  // embedding rows (joint classes)

  // ---- training pairs: exact states at random positions of the corpus
  const uint32_t n_samples = (uint32_t)std::min<uint64_t>(1u << 19, std::max<uint64_t>(4096, len / 512));
  std::vector<uint64_t> pos(n_samples);
  uint64_t s = seed ^ 0x243F6A8885A308D3ull;
  for (auto& p : pos) p = kPropCtx + splitmix(s) % (len - kPropCtx);
  DeviceBuffer d_pos, d_ctx, d_state;
  d_pos.upload(pos.data(), pos.size() * 8);
  d_ctx.alloc((size_t)n_samples * kPropCtx);
  d_state.alloc((size_t)n_samples * G * 4);
  GroupWalk gw{P.d_groups.as<GroupDev>(), P.d_fwd.as<uint32_t>(), P.d_cls.as<uint8_t>(), G};
  sample_kernel<<<blocks(n_samples, 128), 128>>>(gw, d_corpus, len, d_pos.as<uint64_t>(), n_samples,
                                                   pr->d_jmap.as<uint8_t>(), 1024, d_ctx.as<uint8_t>(),
                                                   d_state.as<uint32_t>());
  check_cuda(cudaGetLastError(), "sample_kernel");
  std::vector<uint32_t> state((size_t)n_samples * G);
  check_cuda(cudaMemcpy(state.data(), d_state.ptr, state.size() * 4, cudaMemcpyDeviceToHost), "D2H states");

  // ---- vocabulary: the 63 most frequent states per group + other (= start)
  std::vector<uint32_t> vocab((size_t)G * kPropVocab);
  std::vector<uint8_t> labels((size_t)n_samples * G), is_start((size_t)n_samples * G);
  double start_hits = 0;
  for (uint32_t g = 0; g < G; ++g) {
    std::unordered_map<uint32_t, uint64_t> freq;
    for (uint32_t j = 0; j < n_samples; ++j) freq[state[(size_t)j * G + g]]++;
    std::vector<std::pair<uint64_t, uint32_t>> v;
    for (auto& kv : freq) v.push_back({kv.second, kv.first});
    std::sort(v.begin(), v.end(), [](auto& x, auto& y) { return x.first != y.first ? x.first > y.first : x.second < y.second; });
    std::unordered_map<uint32_t, uint32_t> index;
    for (uint32_t k = 0; k < (uint32_t)kPropVocab - 1; ++k) {
      uint32_t stv = k < v.size() ? v[k].second : P.groups[g].start_unanchored;
      vocab[(size_t)g * kPropVocab + k] = stv;
      if (k < v.size()) index.emplace(stv, k);
    }
    vocab[(size_t)g * kPropVocab + kPropVocab - 1] = P.groups[g].start_unanchored;
    for (uint32_t j = 0; j < n_samples; ++j) {
      uint32_t stv = state[(size_t)j * G + g];
      auto it = index.find(stv);
      labels[(size_t)j * G + g] = (uint8_t)(it == index.end() ? kPropVocab - 1 : it->second);
      is_start[(size_t)j * G + g] = stv == P.groups[g].start_unanchored;
      start_hits += is_start[(size_t)j * G + g];
    }
  }
  pr->d_vocab.upload(vocab.data(), vocab.size() * 4);
  DeviceBuffer d_labels, d_is_start;
  d_labels.upload(labels.data(), labels.size());
  d_is_start.upload(is_start.data(), is_start.size());

  // ---- parameters
  uint64_t ws = seed * 0x9E3779B97F4A7C15ull + 1;
  const uint32_t NO = G * kPropVocab;
  init_uniform(pr->E, (size_t)n_emb * kPropEmb, 0.5f, ws);
  init_uniform(pr->W1, (size_t)kPropHid * kPropHid, std::sqrt(6.f / (2 * kPropHid)), ws);
  init_uniform(pr->W2, (size_t)kPropHid * kPropHid, std::sqrt(6.f / (2 * kPropHid)), ws);
  init_uniform(pr->W3, (size_t)kPropHid * NO, std::sqrt(6.f / (kPropHid + NO)), ws);
  zeros(pr->b1, kPropHid);
  zeros(pr->b2, kPropHid);
  zeros(pr->b3, NO);
  DeviceBuffer* moments[] = {&pr->mE, &pr->vE, &pr->mW1, &pr->vW1, &pr->mb1, &pr->vb1, &pr->mW2,
                             &pr->vW2, &pr->mb2, &pr->vb2, &pr->mW3, &pr->vW3, &pr->mb3, &pr->vb3};
  size_t msz[] = {(size_t)n_emb * kPropEmb, (size_t)n_emb * kPropEmb, (size_t)kPropHid * kPropHid,
                  (size_t)kPropHid * kPropHid, kPropHid, kPropHid, (size_t)kPropHid * kPropHid,
                  (size_t)kPropHid * kPropHid, kPropHid, kPropHid, (size_t)kPropHid * NO, (size_t)kPropHid * NO,
                  NO, NO};
  for (int k = 0; k < 14; ++k) zeros(*moments[k], msz[k]);
  pr->E16.alloc((size_t)n_emb * kPropEmb * 2);
  pr->W1_16.alloc((size_t)kPropHid * kPropHid * 2);
  pr->W2_16.alloc((size_t)kPropHid * kPropHid * 2);
  pr->W3_16.alloc((size_t)kPropHid * NO * 2);
  to_bf16_kernel<<<blocks(n_emb * kPropEmb), 256>>>(pr->E.as<float>(), pr->E16.as<__nv_bfloat16>(), n_emb * kPropEmb);
  to_bf16_kernel<<<blocks(kPropHid * kPropHid), 256>>>(pr->W1.as<float>(), pr->W1_16.as<__nv_bfloat16>(), kPropHid * kPropHid);
  to_bf16_kernel<<<blocks(kPropHid * kPropHid), 256>>>(pr->W2.as<float>(), pr->W2_16.as<__nv_bfloat16>(), kPropHid * kPropHid);
  to_bf16_kernel<<<blocks(kPropHid * NO), 256>>>(pr->W3.as<float>(), pr->W3_16.as<__nv_bfloat16>(), kPropHid * NO);

  // ---- activations for a batch
  const uint32_t B = 512;
  DeviceBuffer X0, Z1, H1, Z2, H2, LG, DL, DH2, DZ2, DH1, DZ1, DX0, dE, dW1, db1, dW2, db2, dW3, db3, loss, hits;
  X0.alloc((size_t)B * kPropHid * 2);
  Z1.alloc((size_t)B * kPropHid * 4);
  H1.alloc((size_t)B * kPropHid * 2);
  Z2.alloc((size_t)B * kPropHid * 4);
  H2.alloc((size_t)B * kPropHid * 2);
  LG.alloc((size_t)B * NO * 4);
  DL.alloc((size_t)B * NO * 2);
  DH2.alloc((size_t)B * kPropHid * 4);
  DZ2.alloc((size_t)B * kPropHid * 2);
  DH1.alloc((size_t)B * kPropHid * 4);
  DZ1.alloc((size_t)B * kPropHid * 2);
  DX0.alloc((size_t)B * kPropHid * 4);
  dE.alloc((size_t)n_emb * kPropEmb * 4);
  dW1.alloc((size_t)kPropHid * kPropHid * 4);
  db1.alloc(kPropHid * 4);
  dW2.alloc((size_t)kPropHid * kPropHid * 4);
  db2.alloc(kPropHid * 4);
  dW3.alloc((size_t)kPropHid * NO * 4);
  db3.alloc(NO * 4);
  loss.alloc(4);
  hits.alloc(16);
  using bf = __nv_bfloat16;
  const uint32_t n_train = n_samples - n_samples / 10;
  const uint8_t* ctx = d_ctx.as<uint8_t>();
  const uint8_t* lab = d_labels.as<uint8_t>();

  auto forward = [&](uint32_t row0, uint32_t rows) {
    embed_kernel<<<blocks(rows * kPropHid), 256>>>(ctx + (size_t)row0 * kPropCtx, pr->E16.as<bf>(), X0.as<bf>(), rows);
    gemm(X0.as<bf>(), kPropHid, 1, pr->W1_16.as<bf>(), kPropHid, 1, Z1.as<float>(), kPropHid, rows, kPropHid, kPropHid, 1.f, 0.f, 0);
    bias_gelu_kernel<<<blocks(rows * kPropHid), 256>>>(Z1.as<float>(), pr->b1.as<float>(), H1.as<bf>(), rows, kPropHid);
    gemm(H1.as<bf>(), kPropHid, 1, pr->W2_16.as<bf>(), kPropHid, 1, Z2.as<float>(), kPropHid, rows, kPropHid, kPropHid, 1.f, 0.f, 0);
    bias_gelu_kernel<<<blocks(rows * kPropHid), 256>>>(Z2.as<float>(), pr->b2.as<float>(), H2.as<bf>(), rows, kPropHid);
    gemm(H2.as<bf>(), kPropHid, 1, pr->W3_16.as<bf>(), NO, 1, LG.as<float>(), NO, rows, NO, kPropHid, 1.f, 0.f, 0);
  };

  const uint32_t steps = 1200;
  const float lr = 2e-3f, be1 = 0.9f, be2 = 0.999f;
  float last_loss = 0;
  for (uint32_t it = 1; it <= steps; ++it) {
    uint32_t row0 = (uint32_t)(((uint64_t)(it - 1) * B) % (n_train - B));
    forward(row0, B);
    check_cuda(cudaMemsetAsync(db3.ptr, 0, NO * 4, 0), "memset");
    check_cuda(cudaMemsetAsync(db2.ptr, 0, kPropHid * 4, 0), "memset");
    check_cuda(cudaMemsetAsync(db1.ptr, 0, kPropHid * 4, 0), "memset");
    check_cuda(cudaMemsetAsync(dE.ptr, 0, (size_t)n_emb * kPropEmb * 4, 0), "memset");
    check_cuda(cudaMemsetAsync(loss.ptr, 0, 4, 0), "memset");
    ce_kernel<<<blocks(B * G), 256>>>(LG.as<float>(), pr->b3.as<float>(), lab + (size_t)row0 * G, B, G, DL.as<bf>(),
                                      db3.as<float>(), loss.as<float>());
    // dW3 = H2^T . DL ; dH2 = DL . W3^T
    gemm(H2.as<bf>(), 1, kPropHid, DL.as<bf>(), NO, 1, dW3.as<float>(), NO, kPropHid, NO, B, 1.f, 0.f, 0);
    gemm(DL.as<bf>(), NO, 1, pr->W3_16.as<bf>(), 1, NO, DH2.as<float>(), kPropHid, B, kPropHid, NO, 1.f, 0.f, 0);
    gelu_back_kernel<<<blocks(B * kPropHid), 256>>>(DH2.as<float>(), Z2.as<float>(), DZ2.as<bf>(), db2.as<float>(), B, kPropHid);
    gemm(H1.as<bf>(), 1, kPropHid, DZ2.as<bf>(), kPropHid, 1, dW2.as<float>(), kPropHid, kPropHid, kPropHid, B, 1.f, 0.f, 0);
    gemm(DZ2.as<bf>(), kPropHid, 1, pr->W2_16.as<bf>(), 1, kPropHid, DH1.as<float>(), kPropHid, B, kPropHid, kPropHid, 1.f, 0.f, 0);
    gelu_back_kernel<<<blocks(B * kPropHid), 256>>>(DH1.as<float>(), Z1.as<float>(), DZ1.as<bf>(), db1.as<float>(), B, kPropHid);
    gemm(X0.as<bf>(), 1, kPropHid, DZ1.as<bf>(), kPropHid, 1, dW1.as<float>(), kPropHid, kPropHid, kPropHid, B, 1.f, 0.f, 0);
    gemm(DZ1.as<bf>(), kPropHid, 1, pr->W1_16.as<bf>(), 1, kPropHid, DX0.as<float>(), kPropHid, B, kPropHid, kPropHid, 1.f, 0.f, 0);
    embed_back_kernel<<<blocks(B * kPropHid), 256>>>(ctx + (size_t)row0 * kPropCtx, DX0.as<float>(), dE.as<float>(), B);
    float c1 = 1.f - std::pow(be1, (float)it), c2 = 1.f - std::pow(be2, (float)it);
    float lr_t = lr * (it > steps * 3 / 4 ? 0.25f : 1.f);
    auto adam = [&](DeviceBuffer& w, DeviceBuffer& g, DeviceBuffer& m, DeviceBuffer& v, DeviceBuffer* w16, size_t n) {
      adam_kernel<<<blocks(n), 256>>>(w.as<float>(), g.as<float>(), m.as<float>(), v.as<float>(),
                                      w16 ? w16->as<bf>() : nullptr, (uint32_t)n, lr_t, be1, be2, c1, c2);
    };
    adam(pr->E, dE, pr->mE, pr->vE, &pr->E16, (size_t)n_emb * kPropEmb);
    adam(pr->W1, dW1, pr->mW1, pr->vW1, &pr->W1_16, (size_t)kPropHid * kPropHid);
    adam(pr->b1, db1, pr->mb1, pr->vb1, nullptr, kPropHid);
    adam(pr->W2, dW2, pr->mW2, pr->vW2, &pr->W2_16, (size_t)kPropHid * kPropHid);
    adam(pr->b2, db2, pr->mb2, pr->vb2, nullptr, kPropHid);
    adam(pr->W3, dW3, pr->mW3, pr->vW3, &pr->W3_16, (size_t)kPropHid * NO);
    adam(pr->b3, db3, pr->mb3, pr->vb3, nullptr, NO);
    check_cuda(cudaGetLastError(), "proposer training step");
    if (it == steps) check_cuda(cudaMemcpy(&last_loss, loss.ptr, 4, cudaMemcpyDeviceToHost), "D2H loss");
  }
  // ---- held-out hit rates
  check_cuda(cudaMemset(hits.ptr, 0, 16), "memset");
  uint64_t n_eval = 0;
  for (uint32_t row0 = n_train; row0 + B <= n_samples; row0 += B) {
    forward(row0, B);
    eval_kernel<<<blocks(B * G), 256>>>(LG.as<float>(), pr->b3.as<float>(), lab + (size_t)row0 * G,
                                        d_is_start.as<uint8_t>() + (size_t)row0 * G, B, G,
                                        hits.as<unsigned long long>());
    n_eval += (uint64_t)B * G;
  }
  unsigned long long h[2] = {0, 0};
  check_cuda(cudaMemcpy(h, hits.ptr, 16, cudaMemcpyDeviceToHost), "D2H hits");
  // ---- inference copies
  pr->W1T.alloc((size_t)kPropHid * kPropHid * 2);
  pr->W2T.alloc((size_t)kPropHid * kPropHid * 2);
  pr->W3T.alloc((size_t)kPropHid * NO * 2);
  transpose_bf16_kernel<<<blocks(kPropHid * kPropHid), 256>>>(pr->W1.as<float>(), pr->W1T.as<bf>(), kPropHid, kPropHid);
  transpose_bf16_kernel<<<blocks(kPropHid * kPropHid), 256>>>(pr->W2.as<float>(), pr->W2T.as<bf>(), kPropHid, kPropHid);
  transpose_bf16_kernel<<<blocks(kPropHid * NO), 256>>>(pr->W3.as<float>(), pr->W3T.as<bf>(), kPropHid, NO);
  check_cuda(cudaDeviceSynchronize(), "proposer training");
  tc_prepare(pr->tc, pr->W1T.ptr, pr->W2T.ptr, pr->W3T.ptr, NO);
  pr->trained = true;
  P.top1 = n_eval ? (double)h[0] / n_eval : 0;
  P.top4 = n_eval ? (double)h[1] / n_eval : 0;
  if (stats) {
    stats->top1 = P.top1;
    stats->top4 = P.top4;
    stats->start_rate = start_hits / ((double)n_samples * G);
    stats->samples = n_samples;
    stats->steps = steps;
    stats->final_loss = last_loss;
  }
  P.proposer.reset(guard.release());
}

uint32_t proposer_predict(Proposer& p, const uint8_t* data, uint64_t len, uint64_t chunk, uint64_t n_chunks,
                          uint32_t* guess, cudaStream_t st) {
  (void)len;
  if (n_chunks <= 1) return 0;
  if (g_use_tc && p.tc.ready) {
    TcInputs in{data, chunk, n_chunks, p.d_jmap.as<uint8_t>(), p.E16.ptr, 64u, p.b1.as<float>(), p.b2.as<float>(),
                p.b3.as<float>(), p.d_vocab.as<uint32_t>(), p.G, guess};
    return tc_predict(p.tc, in, st);
  }
  InferArgs a;
  a.data = data;
  a.chunk = chunk;
  a.n_chunks = n_chunks;
  a.jmap = p.d_jmap.as<uint8_t>();
  a.E = p.E16.as<__nv_bfloat16>();
  a.W1T = p.W1T.as<__nv_bfloat16>();
  a.b1 = p.b1.as<float>();
  a.W2T = p.W2T.as<__nv_bfloat16>();
  a.b2 = p.b2.as<float>();
  a.W3T = p.W3T.as<__nv_bfloat16>();
  a.b3 = p.b3.as<float>();
  a.vocab = p.d_vocab.as<uint32_t>();
  a.G = p.G;
  a.guess = guess;
  check_cuda(cudaFuncSetAttribute(proposer_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem),
             "cudaFuncSetAttribute(proposer)");
  unsigned grid = (unsigned)((n_chunks - 1 + kTileRows - 1) / kTileRows);
  proposer_infer_kernel<<<grid, 256, kInferSmem, st>>>(a);
  check_cuda(cudaGetLastError(), "proposer_infer_kernel");
  return 1;
}

}  // namespace ws

// Numerics hook for the tests: C = A . B with BF16 inputs and FP32 output.
extern "C" int ws_testing_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K) {
  try {
    ws::gemm(static_cast<const __nv_bfloat16*>(A), K, 1, static_cast<const __nv_bfloat16*>(B), N, 1, C, N, M, N, K,
             1.f, 0.f, 0);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
  } catch (...) {
    return 1;
  }
}

// Testing hook (not part of the public header): 1 selects the tcgen05
// inference kernel (the default), 0 the mma.sync kernel, for every matcher in
// the process.
extern "C" void ws_testing_proposer_path(int tcgen05) { ws::g_use_tc = tcgen05 != 0; }
