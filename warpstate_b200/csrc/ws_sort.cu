// Device ordering of scan results.
//
// The public calls return matches sorted by (start, pattern_id, end)
// (GpuMatcher::scan, core/src/gpu/mod.rs:380-386) and tagged matches by
// (source_id, start, pattern_id, end) (core/src/batch.rs:157-163).  The order
// is made on the device by a least-significant-key-first sequence of stable
// radix sorts over an index permutation (CUB's DeviceRadixSort, with its
// temporary storage taken from the scratch so that no call allocates):
//   pass 1  end
//   pass 2  start << 32 | pattern_id
//   pass 3  source_id                  (tagged matches only)
// Stability makes the result the lexicographic order of the full key, ties
// included.  Records are gathered once, through the final permutation.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include "ws_matcher.h"

namespace ws {
namespace {

template <class R>
__global__ void k_keys_end(const R* rec, uint32_t n, uint64_t* key, uint32_t* idx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    key[i] = rec[i].end;
    idx[i] = i;
  }
}

template <class R>
__global__ void k_keys_start_pid(const R* rec, const uint32_t* idx, uint32_t n, uint64_t* key) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const R& r = rec[idx[i]];
    key[i] = ((uint64_t)r.start << 32) | r.pattern_id;
  }
}

__global__ void k_keys_source(const ws_tagged_match* rec, const uint32_t* idx, uint32_t n, uint64_t* key) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    key[i] = rec[idx[i]].source_id;
}

template <class R>
__global__ void k_gather(const R* rec, const uint32_t* idx, uint32_t n, R* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = rec[idx[i]];
}

__global__ void k_narrow(const ws_match64* in, uint32_t n, ws_match* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const ws_match64 w = in[i];
    out[i] = ws_match{w.pattern_id, (uint32_t)w.start, (uint32_t)w.end};
  }
}

// Key and index double buffers plus CUB's temporary storage, in the scratch.
struct Bufs {
  uint64_t* key[2];
  uint32_t* idx[2];
  void* temp;
  size_t temp_bytes;
  int cur = 0;  // which of the double buffers holds the current keys / indices
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

Bufs bufs(Scratch& s, uint32_t n) {
  Bufs b{};
  cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
  cub::DoubleBuffer<uint32_t> v(nullptr, nullptr);
  check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, b.temp_bytes, k, v, (int)n, 0, 64), "radix sort size");
  const size_t kb = align256((size_t)n * 8), vb = align256((size_t)n * 4);
  ensure(s.sortbuf, 2 * kb + 2 * vb + align256(b.temp_bytes));
  uint8_t* p = s.sortbuf.as<uint8_t>();
  b.key[0] = reinterpret_cast<uint64_t*>(p);
  b.key[1] = reinterpret_cast<uint64_t*>(p + kb);
  b.idx[0] = reinterpret_cast<uint32_t*>(p + 2 * kb);
  b.idx[1] = reinterpret_cast<uint32_t*>(p + 2 * kb + vb);
  b.temp = p + 2 * kb + 2 * vb;
  return b;
}

// One stable pass over key bits [0, bits): the indices follow their keys.
void pass(Bufs& b, uint32_t n, int bits, cudaStream_t st) {
  cub::DoubleBuffer<uint64_t> k(b.key[b.cur], b.key[b.cur ^ 1]);
  cub::DoubleBuffer<uint32_t> v(b.idx[b.cur], b.idx[b.cur ^ 1]);
  check_cuda(cub::DeviceRadixSort::SortPairs(b.temp, b.temp_bytes, k, v, (int)n, 0, bits, st), "radix sort");
  if (k.selector) b.cur ^= 1;
}

unsigned grid(uint32_t n) { return (unsigned)std::min<uint32_t>((n + 255) / 256, 148u * 8); }

template <class R>
void sort_records(Scratch& s, const R* d_in, R* d_out, uint64_t n, cudaStream_t st, bool tagged) {
  if (n > kMaxDeviceSorted)
    raise(WS_ERR_OVERFLOW, "too many matches to order on the device", 0, n, kMaxDeviceSorted);
  if (n == 0) return;
  const uint32_t m = (uint32_t)n;
  Bufs b = bufs(s, m);
  k_keys_end<R><<<grid(m), 256, 0, st>>>(d_in, m, b.key[0], b.idx[0]);
  check_cuda(cudaGetLastError(), "k_keys_end");
  pass(b, m, 32, st);
  k_keys_start_pid<R><<<grid(m), 256, 0, st>>>(d_in, b.idx[b.cur], m, b.key[b.cur]);
  check_cuda(cudaGetLastError(), "k_keys_start_pid");
  pass(b, m, 64, st);
  if (tagged) {
    k_keys_source<<<grid(m), 256, 0, st>>>(reinterpret_cast<const ws_tagged_match*>(d_in), b.idx[b.cur], m,
                                           b.key[b.cur]);
    check_cuda(cudaGetLastError(), "k_keys_source");
    pass(b, m, 64, st);
  }
  k_gather<R><<<grid(m), 256, 0, st>>>(d_in, b.idx[b.cur], m, d_out);
  check_cuda(cudaGetLastError(), "k_gather");
}

}  // namespace

void sort_matches_device(Scratch& s, const ws_match* d_in, ws_match* d_out, uint64_t n, cudaStream_t st) {
  sort_records(s, d_in, d_out, n, st, false);
}

void sort_tagged_device(Scratch& s, const ws_tagged_match* d_in, ws_tagged_match* d_out, uint64_t n,
                        cudaStream_t st) {
  sort_records(s, d_in, d_out, n, st, true);
}

void narrow_matches_device(const ws_match64* d_in, ws_match* d_out, uint64_t n, cudaStream_t st) {
  if (n > kMaxDeviceSorted)
    raise(WS_ERR_OVERFLOW, "too many matches to order on the device", 0, n, kMaxDeviceSorted);
  if (n == 0) return;
  k_narrow<<<grid((uint32_t)n), 256, 0, st>>>(d_in, (uint32_t)n, d_out);
  check_cuda(cudaGetLastError(), "k_narrow");
}

}  // namespace ws
