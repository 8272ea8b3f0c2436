// Seeded synthetic workloads for the scan benchmarks and parity tests.
//
// Random numbers: xoshiro256** seeded through SplitMix64 (Blackman & Vigna's
// published generators).  Large inputs are produced in fixed 1 MiB segments,
// each from its own stream (seed, segment index), so the bytes do not depend on
// the number of threads used.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t x = seed;
    for (auto& v : s) v = splitmix64(x);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  inline uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  inline uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
  inline double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

constexpr uint64_t kSegment = 1ull << 20;

uint64_t stream_seed(uint64_t seed, uint64_t segment) {
  uint64_t x = seed ^ (segment * 0xD1B54A32D192ED03ull);
  return splitmix64(x);
}

template <class F>
void parallel_segments(uint64_t len, int threads, F&& fn) {
  uint64_t nseg = (len + kSegment - 1) / kSegment;
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  if (threads <= 0) threads = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) {
    th.emplace_back([&, t] {
      for (uint64_t g = (uint64_t)t; g < nseg; g += (uint64_t)threads) {
        uint64_t a = g * kSegment, b = std::min(len, a + kSegment);
        fn(g, a, b);
      }
    });
  }
  for (auto& x : th) x.join();
}

// Walker's alias tables for one discrete distribution.
struct Alias {
  std::vector<uint32_t> prob;   // threshold scaled to 2^32
  std::vector<uint32_t> alias;
  void build(const std::vector<double>& w) {
    size_t n = w.size();
    double sum = 0;
    for (double x : w) sum += x;
    std::vector<double> p(n);
    for (size_t i = 0; i < n; ++i) p[i] = w[i] * n / sum;
    prob.assign(n, 0);
    alias.assign(n, 0);
    std::vector<size_t> small, large;
    for (size_t i = 0; i < n; ++i) (p[i] < 1.0 ? small : large).push_back(i);
    while (!small.empty() && !large.empty()) {
      size_t s = small.back(); small.pop_back();
      size_t l = large.back();
      prob[s] = (uint32_t)std::min(4294967295.0, p[s] * 4294967296.0);
      alias[s] = (uint32_t)l;
      p[l] = (p[l] + p[s]) - 1.0;
      if (p[l] < 1.0) { large.pop_back(); small.push_back(l); }
    }
    for (size_t i : large) { prob[i] = 0xFFFFFFFFu; alias[i] = (uint32_t)i; }
    for (size_t i : small) { prob[i] = 0xFFFFFFFFu; alias[i] = (uint32_t)i; }
  }
  inline uint32_t draw(Xoshiro& r) const {
    uint64_t x = r.next();
    uint32_t col = (uint32_t)(((x >> 32) * (uint64_t)prob.size()) >> 32);
    return ((uint32_t)x <= prob[col]) ? col : alias[col];
  }
};

}  // namespace

extern "C" {

// iid uniform bytes over `alphabet`.
void wl_fill_uniform(uint8_t* out, uint64_t len, const uint8_t* alphabet, uint32_t n, uint64_t seed,
                     int threads) {
  parallel_segments(len, threads, [&](uint64_t g, uint64_t a, uint64_t b) {
    Xoshiro r(stream_seed(seed, g));
    for (uint64_t i = a; i < b; ++i) out[i] = alphabet[r.below(n)];
  });
}

// Order-1 Markov chain over `alphabet`: row i of the transition matrix has
// weights u^3 (u uniform in (0,1)) drawn from `matrix_seed`, normalised.  Each
// 1 MiB segment starts from a uniformly drawn symbol.
void wl_fill_markov(uint8_t* out, uint64_t len, const uint8_t* alphabet, uint32_t n, uint64_t seed,
                    uint64_t matrix_seed, int threads) {
  std::vector<Alias> rows(n);
  Xoshiro mr(matrix_seed);
  for (uint32_t i = 0; i < n; ++i) {
    std::vector<double> w(n);
    for (auto& x : w) { double u = mr.unit(); x = u * u * u + 1e-6; }
    rows[i].build(w);
  }
  parallel_segments(len, threads, [&](uint64_t g, uint64_t a, uint64_t b) {
    Xoshiro r(stream_seed(seed, g));
    uint32_t st = r.below(n);
    for (uint64_t i = a; i < b; ++i) {
      st = rows[st].draw(r);
      out[i] = alphabet[st];
    }
  });
}

// iid uniform ACGT with runs of 'N' (lengths uniform in [run_lo, run_hi]) that
// start at each position with probability p_run.
void wl_fill_acgt(uint8_t* out, uint64_t len, uint64_t seed, double p_run, uint32_t run_lo,
                  uint32_t run_hi, int threads) {
  static const uint8_t acgt[4] = {'A', 'C', 'G', 'T'};
  uint64_t thresh = (uint64_t)(p_run * 18446744073709551615.0);
  parallel_segments(len, threads, [&](uint64_t g, uint64_t a, uint64_t b) {
    Xoshiro r(stream_seed(seed, g));
    uint64_t i = a;
    while (i < b) {
      uint64_t x = r.next();
      if (x < thresh) {
        uint32_t rl = run_lo + r.below(run_hi - run_lo + 1);
        for (uint32_t k = 0; k < rl && i < b; ++k) out[i++] = 'N';
      } else {
        out[i++] = acgt[x & 3];
      }
    }
  });
}

// n literals, lengths uniform in [lmin, lmax], characters drawn from
// `alphabet` with the given weights.  Writes bytes back to back into out
// (capacity n*lmax) and the lengths into lens.
void wl_gen_literals(uint32_t n, uint32_t lmin, uint32_t lmax, const uint8_t* alphabet,
                     const double* weights, uint32_t na, uint64_t seed, uint8_t* out, uint32_t* lens) {
  Alias al;
  al.build(std::vector<double>(weights, weights + na));
  Xoshiro r(seed);
  uint64_t o = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t L = lmin + r.below(lmax - lmin + 1);
    lens[i] = L;
    for (uint32_t k = 0; k < L; ++k) out[o++] = alphabet[al.draw(r)];
  }
}

}  // extern "C"
