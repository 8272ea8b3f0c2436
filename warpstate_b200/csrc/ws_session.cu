// Zero-copy scan sessions and hot-swappable matchers.
//
// Zero copy replaces StreamPipeline::scan_zero_copy / ZeroCopyScan
// (core/src/pipeline.rs:31-83) and the DmaStagingBuffer they fill
// (core/src/dma.rs:17-141): the caller writes the input straight into pinned,
// device-mapped host memory that the library owns, so the scan's host-to-device
// DMA reads the caller's bytes where they were written, with no intermediate
// copy.  The staged input is scanned like a pinned ws_scan input: copied in
// windows on a second stream while earlier windows are scanned.  Staging
// buffers are pooled per matcher and freed with it.
//
// Hot swap replaces HotSwapPatternSet (core/src/pattern/mod.rs:17-70): a
// handle whose active matcher (its device tables) can be replaced while other
// threads scan.  A scan holds a reference to the matcher it started with; a
// replaced matcher is destroyed when its last scan ends.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <mutex>

#include "ws_matcher.h"

using namespace ws;

struct ws_zero_copy {
  ws_matcher* m = nullptr;
  uint8_t* mapped = nullptr;  // pinned, device-mapped host memory (capacity `cap`)
  size_t cap = 0;
  uint64_t len = 0;
};

struct ws_hotswap {
  std::mutex mu;
  std::shared_ptr<ws_matcher> current;
};

namespace {

// Staging buffers of finished sessions, per matcher, reused by later sessions.
struct StagingPool {
  std::mutex mu;
  std::vector<std::pair<uint8_t*, size_t>> free;
  ~StagingPool() {
    for (auto& b : free) cudaFreeHost(b.first);
  }
};

std::mutex g_pools_mu;
std::vector<std::pair<const ws_matcher*, std::unique_ptr<StagingPool>>> g_pools;

StagingPool& pool_of(const ws_matcher* m) {
  std::lock_guard<std::mutex> g(g_pools_mu);
  for (auto& p : g_pools)
    if (p.first == m) return *p.second;
  g_pools.emplace_back(m, std::make_unique<StagingPool>());
  return *g_pools.back().second;
}

}  // namespace

namespace ws {
// Frees the staging buffers pooled for a matcher (called when it is destroyed).
void release_staging(const ws_matcher* m) {
  std::lock_guard<std::mutex> g(g_pools_mu);
  for (size_t k = 0; k < g_pools.size(); ++k)
    if (g_pools[k].first == m) {
      g_pools.erase(g_pools.begin() + (long)k);
      return;
    }
}
}  // namespace ws

extern "C" {

ws_status ws_zero_copy_begin(ws_matcher* m, uint64_t input_len, ws_zero_copy** out, uint8_t** mapped,
                             ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !out || !mapped) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    *mapped = nullptr;
    if (input_len > 0xFFFFFFFFull)
      raise(WS_ERR_INPUT_TOO_LARGE, "scan input is too large for 32-bit match offsets", 0, input_len, 0xFFFFFFFFull);
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    auto z = std::make_unique<ws_zero_copy>();
    z->m = m;
    z->len = input_len;
    StagingPool& pool = pool_of(m);
    {
      std::lock_guard<std::mutex> g(pool.mu);
      for (size_t k = 0; k < pool.free.size(); ++k)
        if (pool.free[k].second >= input_len) {
          z->mapped = pool.free[k].first;
          z->cap = pool.free[k].second;
          pool.free.erase(pool.free.begin() + (long)k);
          break;
        }
    }
    if (!z->mapped) {
      const size_t cap = std::max<size_t>((size_t)input_len, 4096);
      check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&z->mapped), cap, cudaHostAllocMapped | cudaHostAllocPortable),
                 "cudaHostAlloc(staging)");
      z->cap = cap;
    }
    *mapped = z->mapped;
    *out = z.release();
  });
}

void ws_zero_copy_abort(ws_zero_copy* z) {
  if (!z) return;
  StagingPool& pool = pool_of(z->m);
  {
    std::lock_guard<std::mutex> g(pool.mu);
    pool.free.emplace_back(z->mapped, z->cap);
  }
  delete z;
}

ws_status ws_zero_copy_finish(ws_zero_copy* z, ws_match* out, uint64_t cap, uint64_t* n_out, ws_error_info* err) {
  if (!z) {
    if (err) {
      std::memset(err, 0, sizeof(*err));
      std::snprintf(err->message, sizeof(err->message), "null argument");
    }
    return WS_ERR_INVALID_ARGUMENT;
  }
  const ws_status st = ws_scan(z->m, z->mapped, z->len, out, cap, n_out, err);
  ws_zero_copy_abort(z);  // the staging buffer goes back to the pool either way
  return st;
}

ws_status ws_hotswap_create(ws_matcher* initial, ws_hotswap** out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!initial || !out) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    auto h = std::make_unique<ws_hotswap>();
    h->current = std::shared_ptr<ws_matcher>(initial, [](ws_matcher* m) { ws_matcher_destroy(m); });
    *out = h.release();
  });
}

int ws_hotswap_swap(ws_hotswap* h, ws_matcher* next) {
  if (!h || !next) return -1;
  std::shared_ptr<ws_matcher> old;
  {
    std::lock_guard<std::mutex> g(h->mu);
    if (h->current.get() == next) return 0;
    old = std::move(h->current);
    h->current = std::shared_ptr<ws_matcher>(next, [](ws_matcher* m) { ws_matcher_destroy(m); });
  }
  return 1;  // `old` is destroyed here unless a scan still holds it
}

ws_status ws_hotswap_scan(ws_hotswap* h, const uint8_t* data, uint64_t len, ws_match* out, uint64_t cap,
                          uint64_t* n_out, ws_error_info* err) {
  if (!h) {
    if (err) {
      std::memset(err, 0, sizeof(*err));
      std::snprintf(err->message, sizeof(err->message), "null argument");
    }
    return WS_ERR_INVALID_ARGUMENT;
  }
  std::shared_ptr<ws_matcher> m;
  {
    std::lock_guard<std::mutex> g(h->mu);
    m = h->current;
  }
  return ws_scan(m.get(), data, len, out, cap, n_out, err);
}

void ws_hotswap_destroy(ws_hotswap* h) { delete h; }

}  // extern "C"
