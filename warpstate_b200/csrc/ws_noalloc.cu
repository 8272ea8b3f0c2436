// Allocation-free literal scan.
//
// Some callers cannot call cudaMalloc while they scan: a host framework whose
// memory manager owns every device byte (so a library allocation would be
// invisible to its accounting and could fail under its budget), or a
// latency-bound loop where cudaMalloc's implicit device synchronisation and
// cost are unacceptable.  For them this file provides ws_scan_literals_noalloc:
// the literal scan with its scratch memory (the survivor list of the filter
// kernel and its counter) in the file-scope array below instead of a pool
// allocation.  The caller still passes the input and the output buffers.
//
// The array is part of the module image: every GPU that loads this library
// holds kNoAllocScratchBytes of device memory for it until the process exits.
#include <cuda_runtime.h>

#include <cstring>

#include "ws_internal.h"

namespace ws {

// Largest input the allocation-free scan accepts: 128 MiB, the reference's
// default chunk size (core/src/config.rs:4).
constexpr uint64_t kNoAllocMaxInput = 128ull << 20;
// Survivor list for kNoAllocMaxInput bytes plus its counter header.
constexpr size_t kNoAllocScratchBytes =
    ((64 + (kNoAllocMaxInput / 64 + 4096) * 4) + 255) / 256 * 256;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, with the scan's device current.  It is looked up on
// every call (a table lookup once the module is loaded) rather than cached:
// after cudaDeviceReset the module, and with it the array, is loaded again at
// another address.  The first lookup on a device loads the module.
void* scratch_address() {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    raise(WS_ERR_DEVICE, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
  return p;
}

}  // namespace

// Accessors the C ABI file uses (defined there: the matcher is opaque here).
const LiteralPlan* matcher_literal_plan(const ws_matcher* m, uint32_t* n_regex, int* device, int* sm_count);

}  // namespace ws

using namespace ws;

extern "C" ws_status ws_scan_literals_noalloc(ws_matcher* m, const uint8_t* d_data, uint64_t len,
                                              ws_match* d_out, uint64_t cap, uint64_t* d_count, void* stream,
                                              ws_error_info* err) {
  if (err) std::memset(err, 0, sizeof(*err));
  try {
    if (!m || !d_count || (len && !d_data) || (cap && !d_out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_data & 15) != 0) raise(WS_ERR_INVALID_ARGUMENT, "device input must be 16-byte aligned");
    if (len > kNoAllocMaxInput)
      raise(WS_ERR_INPUT_TOO_LARGE,
            "the allocation-free scan accepts at most 128 MiB per call; split the input or use ws_scan_device", 0, len,
            kNoAllocMaxInput);
    uint32_t n_regex = 0;
    int device = 0, sm_count = 0;
    const LiteralPlan* plan = matcher_literal_plan(m, &n_regex, &device, &sm_count);
    if (n_regex)
      raise(WS_ERR_INVALID_ARGUMENT, "the allocation-free scan covers literal-only pattern sets; this matcher has regexes");
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(d_count);
    check_cuda(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st), "memset count");
    if (len == 0 || plan->n_literals == 0) return WS_OK;
    void* scratch = scratch_address();
    uint64_t scap = literal_survivor_cap(len);  // <= the array's capacity for len <= kNoAllocMaxInput
    LiteralLaunch ll{d_data, len, d_out, cap, counter, scratch, scap};
    launch_literal_scan(*plan, ll, st, sm_count);  // clears the survivor counter first
    return WS_OK;
  } catch (const WsError& e) {
    if (err) {
      err->index = e.f.index;
      err->count = e.f.count;
      err->max = e.f.max;
      std::snprintf(err->message, sizeof(err->message), "%s", e.f.message.c_str());
    }
    return e.f.status;
  } catch (const std::exception& e) {
    if (err) std::snprintf(err->message, sizeof(err->message), "%s", e.what());
    return WS_ERR_DEVICE;
  }
}
