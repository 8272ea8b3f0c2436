// Internal structures shared by the host compiler, the C ABI and the kernels.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/warpstate.h"
#include "ws_regex.h"

namespace ws {

constexpr uint32_t FNV_BASIS = 2166136261u;
constexpr uint32_t FNV_PRIME = 16777619u;
constexpr uint32_t HASH_WINDOW = 8;  // hash_window_len, core/src/pattern/compiler.rs:118

// Status carrier for the C ABI.
struct Failure {
  ws_status status;
  std::string message;
  uint64_t index = 0, count = 0, max = 0;
};

struct WsError : std::exception {
  Failure f;
  explicit WsError(Failure x) : f(std::move(x)) {}
  const char* what() const noexcept override { return f.message.c_str(); }
};

[[noreturn]] void raise(ws_status s, const std::string& msg, uint64_t index = 0, uint64_t count = 0,
                        uint64_t max = 0);
void check_cuda(cudaError_t e, const char* what);

uint32_t fnv1a(const uint8_t* p, size_t len, size_t window);

// ------------------------------------------------------------------ IR (host)
struct IrData {
  std::vector<uint8_t> packed_bytes;
  std::vector<uint32_t> offsets;              // (start, len) pairs
  std::vector<uint32_t> literal_pattern_ids;
  std::vector<uint32_t> literal_hashes;
  std::vector<uint32_t> prefix_meta;          // 4 * HASH_WINDOW
  std::vector<uint32_t> bucket_ranges;        // 2 per bucket
  std::vector<uint32_t> entries;              // 2 per literal
  std::vector<std::string> regex_sources;
  std::vector<uint32_t> regex_pattern_ids;
  std::vector<const char*> regex_ptrs;        // views for ws_pattern_tables
  uint32_t n_patterns = 0;
  bool case_insensitive = false;
  // optional pattern names (a CompiledPatternIndex carries them)
  std::vector<std::string> names;
  std::vector<uint8_t> named;
};

}  // namespace ws

// The handle behind ws_ir (a built pattern set or a loaded compiled index).
struct ws_ir {
  ws::IrData d;
};

namespace ws {

// LiteralPrefilterTable::build (core/src/literal_prefilter.rs:23-88).
void build_prefilter_table(const std::vector<uint32_t>& offsets, const std::vector<uint32_t>& hashes,
                           uint32_t window, std::vector<uint32_t>& meta,
                           std::vector<uint32_t>& ranges, std::vector<uint32_t>& entries);

// ------------------------------------------------------------ device memory
// A device allocation that frees itself.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    std::swap(ptr, o.ptr);
    std::swap(bytes, o.bytes);
    return *this;
  }
  ~DeviceBuffer();
  void alloc(size_t n);
  void upload(const void* src, size_t n);
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// ------------------------------------------------------- literal device plan
// Stage 1 of the literal scan: a sampled q-gram filter.  Every long literal
// (length >= 4) registers its 4-byte grams at offsets k = 0..P-1 in a table of
// 2^bits nibbles; bit (P-1-k) of entry hash(gram) records offset k.  A scan
// position s can start a long literal only if the entry of the gram at the
// first P-aligned position a >= s has bit (P-1-(a-s)) set.  Short literals
// (length 1..3) register their first two bytes in a 64 Ki-bit table checked at
// every position.  Stage 2 runs the reference's own FNV-1a probe of the
// LiteralPrefilterTable at each surviving position and verifies exactly.
struct LiteralPlan {
  uint32_t n_literals = 0;
  uint32_t period = 4;       // P: 1, 2 or 4
  uint32_t table_bits = 18;  // 2^bits nibble entries
  uint32_t has_long = 0, has_short = 0;
  uint32_t max_len = 0;
  uint32_t parts = 0;                 // bit i: some literal has prefix length i+1
  std::vector<uint32_t> filter;       // 2^bits nibbles packed 8 per word
  std::vector<uint32_t> bloom;        // 2^18-bit Bloom bitmap of prefix hashes
  std::vector<uint32_t> short_bits;   // 65536 bits
  std::vector<uint32_t> lit_info;     // 4 per literal: offset (in lit_bytes), len, pattern id, 0
  std::vector<uint8_t> lit_bytes;     // literals, each 4-byte aligned
  // Low-entropy pattern sets (e.g. nucleotide k-mers) saturate 4-byte grams:
  // stage 1 then hashes longer grams (gram_len 8 or 16 bytes) and stage 1.5
  // adds a second, L2-resident Bloom bitmap of the first min(len, 16) bytes.
  uint32_t gram_len = 4;
  uint32_t parts16 = 0;               // bit i: some literal has a key of i+1 bytes (<= 16)
  std::vector<uint32_t> bloom2;       // 2^kBloom2Bits bits, only when gram_len > 4
  // Large pattern sets fill the shared-memory gram table: a second table of
  // 2^kBigBits bytes in L2 (same hashes, more bits; each byte holds the P
  // phase bits of its hash, so a lookup is one byte load) re-checks every
  // gram that passes it (stage 1b).  Not built when the shared table is
  // sparse enough; the host copy is released once uploaded (has_big).
  std::vector<uint8_t> big;
  bool has_big = false;
  // With the stage-1b table: stage 1 in shared memory, 2^kLeanBits bits.
  // For 4-byte grams a bitmap indexed by the top kLeanBits bits of the same
  // hashes (a bit is set when any of the 2^(kBigBits - kLeanBits) stage-1b
  // bytes below it is non-zero), so that only about 3% of the grams of
  // text-like input go on to a stage-1b load.  For long grams (dense k-mer
  // sets) a blocked Bloom filter with two bits per gram (lean2_word,
  // lean2_mask), which passes 11% instead of 17% of the grams of a
  // 200,000-gram set.
  std::vector<uint8_t> lean_bits;
  DeviceBuffer d_filter, d_bloom, d_short, d_info, d_bytes, d_meta, d_ranges, d_entries, d_bloom2, d_big,
      d_lean_bits;
  uint32_t n_buckets = 0;
  // ASCII case-insensitive: the tables hold folded literals and the kernels
  // fold the input (A-Z to a-z) before hashing and comparing.
  bool fold = false;
};

// ASCII case folding of the case-insensitive literal scan: A-Z to a-z.
__host__ __device__ inline uint8_t ascii_fold(uint8_t c) { return (c >= 'A' && c <= 'Z') ? (uint8_t)(c | 0x20) : c; }

// The same for the four bytes of a word at once: a byte is an upper-case
// letter when its low seven bits are at least 0x41 and below 0x5B and its top
// bit is clear; adding 0x3F and 0x25 to the low seven bits sets bit 7 exactly
// at those bounds (no carry leaves a byte), and 0x80 >> 2 is the case bit.
__host__ __device__ inline uint32_t ascii_fold4(uint32_t w) {
  const uint32_t x = w & 0x7F7F7F7Fu;
  const uint32_t upper = (x + 0x3F3F3F3Fu) & ~(x + 0x25252525u) & ~w & 0x80808080u;
  return w | (upper >> 2);
}

constexpr uint32_t kBloom2Bits = 24;  // 2 MiB, read through L2
constexpr uint32_t kBigBits = 25;     // stage-1b table: 2^25 bytes, 32 MiB, read through L2
constexpr uint32_t kLeanBits = 20;    // stage 1 of the lean kernel: a 2^20-bit bitmap, 128 KiB of shared memory

// Blocked Bloom filter of stage 1 for long grams with the stage-1b table: the
// word of 32-bit gram hash hf (its top kLeanBits - 5 bits) and the two bits
// set in it (five-bit fields of a second multiplicative hash of hf).
__host__ __device__ inline uint32_t lean2_word(uint32_t hf) { return hf >> (32 - (kLeanBits - 5)); }
__host__ __device__ inline uint32_t lean2_mask(uint32_t hf) {
  const uint32_t h2 = hf * 0x2545F491u;
  return (1u << (h2 >> 27)) | (1u << ((h2 >> 22) & 31u));
}

// Gram hash of stage 1 (a multiplicative hash; the constant is 2^32 / phi).
inline uint32_t gram_hash(uint32_t gram, uint32_t bits) { return (gram * 0x9E3779B1u) >> (32 - bits); }

// Multiply-add hash of 2 or 4 words with a final avalanche (xor-shift,
// multiply, xor-shift), for long grams and 16-byte prefix keys.
__host__ __device__ inline uint32_t mix_words(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t salt) {
  uint32_t h = w0 * 0x9E3779B1u + w1 * 0x85EBCA77u + w2 * 0xC2B2AE3Du + w3 * 0x27D4EB2Fu + salt * 0x165667B1u;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  return h;
}

// Stage-1 key of a gram of 4, 8 or 16 bytes (g[0..gram_len/4)).
__host__ __device__ inline uint32_t long_gram_hash(uint32_t g0, uint32_t g1, uint32_t g2, uint32_t g3, uint32_t gram_len,
                                                   uint32_t bits) {
  return (gram_len == 8 ? mix_words(g0, g1, 0, 0, 8) : mix_words(g0, g1, g2, g3, 16)) >> (32 - bits);
}

// Word k of a key keeps only the bytes below pl.
__host__ __device__ inline uint32_t key_word(uint32_t x, uint32_t k, uint32_t pl) {
  if (pl >= 4 * k + 4) return x;
  if (pl <= 4 * k) return 0u;
  return x & ((1u << (8 * (pl - 4 * k))) - 1u);
}

// Stage-1.5b key of the first pl (1..16) bytes of the four words x.
__host__ __device__ inline uint32_t prefix16_key(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t pl) {
  return mix_words(key_word(x0, 0, pl), key_word(x1, 1, pl), key_word(x2, 2, pl), key_word(x3, 3, pl), pl) >>
         (32 - kBloom2Bits);
}

void plan_literals(const ws_pattern_tables& t, LiteralPlan& plan);

// Kernel launchers (ws_literal.cu).
struct LiteralLaunch {
  const uint8_t* data;
  uint64_t len;
  ws_match* out;
  uint64_t cap;
  unsigned long long* counter;  // device; incremented per match (true count)
  void* scratch;                // literal_scratch_bytes(survivor_cap) bytes
  uint64_t survivor_cap;
  // Batch scans: ascending exclusive end offsets of the items coalesced in
  // `data` (n_items of them); a match must end inside the item it starts in.
  const uint32_t* item_end = nullptr;
  uint32_t n_items = 0;
  // Stream scans: only matches ending after this offset are new.
  uint64_t min_end = 0;
  // Shard scans: only matches starting before this offset are this shard's.
  uint64_t max_start = ~0ull;
};

// Exclusive end of the item that contains offset `s` (the first end above s).
__host__ __device__ inline uint32_t item_end_of(const uint32_t* ends, uint32_t n, uint32_t s) {
  uint32_t lo = 0, hi = n;  // first index with ends[idx] > s
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (ends[mid] > s) hi = mid; else lo = mid + 1;
  }
  return lo < n ? ends[lo] : 0xFFFFFFFFu;
}

// Start of the item that contains offset `s` (the last end at or below s).
__host__ __device__ inline uint32_t item_start_of(const uint32_t* ends, uint32_t n, uint32_t s) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (ends[mid] > s) hi = mid; else lo = mid + 1;
  }
  return lo > 0 ? ends[lo - 1] : 0;
}
size_t literal_scratch_bytes(uint64_t survivor_cap);
inline uint64_t literal_survivor_cap(uint64_t len) { return len / 64 + 4096; }
void launch_literal_scan(const LiteralPlan& plan, const LiteralLaunch& a, cudaStream_t st, int sm_count);
size_t literal_smem_bytes(const LiteralPlan& plan);

}  // namespace ws
