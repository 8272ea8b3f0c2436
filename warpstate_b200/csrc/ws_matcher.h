// Matcher object of the C ABI and the helpers that the single-buffer scan
// (ws_api.cu), the batch scan (ws_batch.cu) and the stream scan
// (ws_stream.cu) share: per-call scratch from a pool, input staging, the
// enqueue of the literal and regex pipelines, error plumbing.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <functional>
#include <atomic>
#include <memory>
#include <mutex>
#include <vector>

#include "ws_internal.h"
#include "ws_dfa.h"

struct ws_ctx {
  int device = 0;
  int sm_count = 0;
};

namespace ws {

// The arguments of a device batch scan whose launch sequence a CUDA graph
// holds (ws_scan_batch_device): a later call with the same arguments and the
// same matcher plan replays the graph.
struct BatchGraphKey {
  const void* data = nullptr;
  uint64_t len = 0;
  const void* item_end = nullptr;
  const void* ids = nullptr;
  uint64_t n_items = 0;
  const void* out = nullptr;
  uint64_t cap = 0;
  const void* count = nullptr;
  const void* stream = nullptr;
  uint64_t plan_gen = 0;
  uint64_t need[2] = {0, 0};
  uint64_t profile = 0;
};

struct BatchGraph {
  BatchGraphKey key;
  uint32_t seen = 0;            // eager runs with this key (the first sizes every buffer)
  uint32_t launches = 0;        // kernel launches the graph holds
  bool broken = false;          // capture or instantiation failed: stay eager
  cudaGraphExec_t exec = nullptr;
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    seen = 0;
    broken = false;
  }
  ~BatchGraph() { reset(); }
};

// Per-call scratch: a stream, the device input copy, the output and counters.
struct Scratch {
  cudaStream_t stream = nullptr;
  DeviceBuffer input;        // padded device copy of the input
  DeviceBuffer input_alt;    // second input buffer: the next batch launch group is copied while one scans
  DeviceBuffer out;          // ws_match[capacity]
  DeviceBuffer counters;     // unsigned long long[8]
  DeviceBuffer rx;           // regex scratch (ws_dfa.cu manages the layout)
  DeviceBuffer lit;          // literal survivor list
  DeviceBuffer aux;          // batch item ends / tagged output
  DeviceBuffer out64;        // ws_match64 output of windowed scans
  DeviceBuffer sorted;       // matches in their final order, read back from here
  DeviceBuffer sortbuf;      // radix-sort keys, indices and temporary storage
  void* pinned = nullptr;    // pinned staging for pageable host input
  size_t pinned_bytes = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // [0], [1]: window copies; [2], [3]: staging slots drained
  bool pin_busy[2] = {false, false};                         // a DMA may still read the slot
  cudaEvent_t busy = nullptr;  // recorded after the last use
  cudaStream_t copy = nullptr;  // host-to-device copies overlapped with scans (created on first use)
  BatchGraph batch_graph;       // the last device batch scan's launch sequence
  ~Scratch() {
    if (busy) cudaEventDestroy(busy);
    if (copy) cudaStreamDestroy(copy);
    if (stream) cudaStreamDestroy(stream);
    if (pinned) cudaFreeHost(pinned);
    for (auto e : ev) if (e) cudaEventDestroy(e);
  }
};

// Extra bounds of a scan over coalesced batch items or a stream window.
struct ScanExtras {
  const uint32_t* item_end = nullptr;  // batch: ascending item ends (device)
  uint32_t n_items = 0;
  bool literals = true;                // run the literal pipeline
  uint64_t lit_min_end = 0;            // stream: literal matches ending later are new
  uint64_t lit_max_start = ~0ull;      // shard: literal matches starting earlier are this shard's
  unsigned long long* cursor = nullptr;  // stream: per-regex find_iter positions (device)
  uint64_t base = 0, frontier = 0;     // stream: window offset and decision frontier
};

// Pinned staging of `piece` bytes per slot (two slots), allocated on demand.
uint8_t* staging(Scratch& s, size_t piece);
// Host pointer of staging slot k, after any DMA still reading it has finished.
uint8_t* staging_slot(Scratch& s, int k, size_t piece);
// Marks slot k as read by the DMA just enqueued on `st` (default: the
// scratch's stream).
void staging_issued(Scratch& s, int k, cudaStream_t st = nullptr);
void ensure(DeviceBuffer& b, size_t need);
void fill_err(ws_error_info* err, const Failure& f);
bool is_pinned(const void* p);
void sort_matches(ws_match* p, uint64_t n);

// Device ordering of results (ws_sort.cu), for counts up to kMaxDeviceSorted;
// larger counts are ordered on the host.  Input and output must not alias.
constexpr uint64_t kMaxDeviceSorted = 0x7FFFFFFFull;
// By (start, pattern_id, end).
void sort_matches_device(Scratch& s, const ws_match* d_in, ws_match* d_out, uint64_t n, cudaStream_t st);
// By (source_id, start, pattern_id, end).
void sort_tagged_device(Scratch& s, const ws_tagged_match* d_in, ws_tagged_match* d_out, uint64_t n,
                        cudaStream_t st);
// 64-bit offsets to 32-bit ones (inputs below 4 GiB).
void narrow_matches_device(const ws_match64* d_in, ws_match* d_out, uint64_t n, cudaStream_t st);
// Frees the zero-copy staging buffers pooled for a matcher (ws_session.cu).
void release_staging(const ws_matcher* m);
// Reads `count` device results into host `out` in (start, pattern_id, end)
// order, through the scratch's stream; returns when they have arrived.
void read_sorted(Scratch& s, const ws_match* d_res, uint64_t count, ws_match* out);

}  // namespace ws

struct ws_matcher {
  ws_ctx* ctx = nullptr;
  ws_config cfg;
  ws::LiteralPlan lit;
  ws::RegexPlan rx;
  uint32_t n_patterns = 0;
  uint32_t max_literal_len = 0;
  std::vector<uint8_t> is_regex;  // per pattern id
  // regex sources and ids, kept so that the autotuner can re-plan the groups
  std::vector<std::string> rx_src;
  std::vector<uint32_t> rx_ids;
  std::mutex pool_mu;
  std::vector<std::unique_ptr<ws::Scratch>> pool;
  std::mutex info_mu;
  ws_matcher_info info;
  bool profile = false;          // record phase events (single caller at a time)
  // Bumped whenever the launch sequence of a scan may change (walk chunk,
  // proposer on or off, re-planned groups or hot rows): captured graphs of
  // earlier plans are not replayed.
  std::atomic<uint64_t> plan_gen{0};
  cudaEvent_t pev[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t rx_events[8] = {};
  // phase times summed over the windows of the last multi-window scan
  bool use_summed = false;
  double summed_ms[8] = {};
  // Two host-mapped words (regex candidates, match events) where a scan whose
  // candidate buffers overflowed records how many it needed; later scans
  // reserve that much (need_dev is their device address).
  unsigned long long* need_host = nullptr;
  unsigned long long* need_dev = nullptr;
  ~ws_matcher() {
    for (auto e : pev) if (e) cudaEventDestroy(e);
    for (auto e : rx_events) if (e) cudaEventDestroy(e);
    if (need_host) cudaFreeHost(need_host);
  }

  std::unique_ptr<ws::Scratch> take();
  void give(std::unique_ptr<ws::Scratch> s);
};

namespace ws {

// Returns a pooled scratch to its matcher when the scope ends.
struct ScratchLease {
  ws_matcher* m;
  std::unique_ptr<Scratch> s;
  explicit ScratchLease(ws_matcher* mm) : m(mm), s(mm->take()) {}
  ~ScratchLease() { if (s) m->give(std::move(s)); }
  Scratch* operator->() { return s.get(); }
  Scratch& operator*() { return *s; }
};

template <class F>
ws_status guarded(ws_error_info* err, F&& fn) {
  if (err) std::memset(err, 0, sizeof(*err));
  try {
    fn();
    return WS_OK;
  } catch (const WsError& e) {
    fill_err(err, e.f);
    return e.f.status;
  } catch (const CompileError& e) {
    if (err) std::snprintf(err->message, sizeof(err->message), "%s", e.what());
    return WS_ERR_COMPILE;
  } catch (const std::bad_alloc&) {
    if (err) std::snprintf(err->message, sizeof(err->message), "host allocation failed");
    return WS_ERR_DEVICE;
  } catch (const std::exception& e) {
    if (err) std::snprintf(err->message, sizeof(err->message), "%s", e.what());
    return WS_ERR_DEVICE;
  }
}

// Host -> device copy on the scratch's stream; pageable sources go through
// double-buffered pinned staging.
void stage_copy(Scratch& s, uint8_t* d_dst, const uint8_t* src, uint64_t len);
// Copies host input into the scratch's device buffer (zero padding after it).
void stage_input(ws_matcher* m, Scratch& s, const uint8_t* data, uint64_t len);
uint64_t device_capacity(const ws_matcher* m);
// Enqueues the full scan of a device-resident input on `st`; nothing is read
// back.  With profiling enabled, phase events are recorded on `st` as well.
// Returns the number of kernel launches enqueued.
uint32_t enqueue_scan(ws_matcher* m, Scratch& s, cudaStream_t st, const uint8_t* d_data, uint64_t len,
                      ws_match* d_out, uint64_t cap, unsigned long long* d_counter,
                      const ScanExtras& x = ScanExtras());
// Waits for the last profiled scan and reads its phase times (ms[8], the
// layout of ws_matcher_info.last_kernel_ms).
void read_phases(ws_matcher* m, double* ms);
// Scans whose regex candidate buffers overflow report kCountUnknown; the
// synchronous entry points repeat them (sized by what they needed) up to this
// many times before giving up with MatchBufferOverflow.
constexpr int kCandidateRetries = 4;
// Raises MatchBufferOverflow for a count that stayed unknown.
[[noreturn]] void raise_candidates_unknown(ws_matcher* m);
// After a synchronous scan: true when it must be repeated (its regex
// candidates overflowed; attempt counts from 0), false when `count` is a match
// count; raises Timeout for a scan whose device-side wait ran out and
// MatchBufferOverflow once the retries are used up.
bool repeat_scan(ws_matcher* m, unsigned long long count, int attempt);

// One window of a scan in steps (stream feeds, ws_scan_device64): the bytes
// seen so far are [0, seen), the previous window started at win_base, regex
// starts below `frontier` are decided.  The new window is [keep, seen); after
// the step every start below the returned frontier is decided (all of them
// when `last`).
struct StepPlan {
  uint64_t keep, frontier;
};
StepPlan plan_step(const ws_matcher* m, uint64_t win_base, uint64_t old_seen, uint64_t seen, uint64_t frontier,
                   bool last);

// Enqueues the scan of d_data[0, len) on `cs` as windows of `window` new
// bytes (slices of d_data with exact carry), appending ws_match64 results to
// d_out (capacity cap) and the true count to *total (zeroed here).
// `before_window(end)` runs on the host before each window is enqueued, with
// the end offset of the bytes it reads (a caller copying the input in pieces
// makes `cs` wait for them there).  Returns the number of kernel launches.
uint32_t enqueue_windows(ws_matcher* m, Scratch& s, cudaStream_t cs, const uint8_t* d_data, uint64_t len,
                         uint64_t window, ws_match64* d_out, uint64_t cap, unsigned long long* total,
                         const std::function<void(uint64_t)>& before_window);

// ws_scan of a large pinned host input copies it in windows of this size on a
// second stream, each window scanned as soon as it has arrived.
constexpr uint64_t kOverlapWindow = 128ull << 20;
void scan_overlapped(ws_matcher* m, Scratch& s, const uint8_t* data, uint64_t len, ws_match* out, uint64_t cap,
                     uint64_t* n_out);

}  // namespace ws
