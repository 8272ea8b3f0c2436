// Learned boundary-state proposer of the speculative DFA walk.
//
// The speculative walk starts every chunk (after the first) from a guessed
// DFA state; the fix-up makes results exact whatever the guess, so a better
// guess only saves re-walk time.  The proposer is an MLP over the 16 bytes
// before the boundary, mapped to the joint byte classes of all DFA groups:
// 16 class ids -> 16-dim embeddings (256 values) -> 256 -> 256 (GELU) -> one
// head per group over that group's most frequent boundary states plus an
// "other" entry (other = the unanchored start).  Weights are BF16, every
// product accumulates in FP32 (hand-written mma.sync kernels).
#pragma once
#include "ws_internal.h"

namespace ws {

struct RegexPlan;
struct Proposer;

constexpr int kPropCtx = 16;     // context bytes
constexpr int kPropEmb = 16;     // embedding width
constexpr int kPropHid = 256;    // hidden width (= kPropCtx * kPropEmb)
constexpr int kPropVocab = 64;   // per-group outputs (63 states + other)

struct ProposerStats {
  double top1 = 0, top4 = 0;        // held-out hit rates of the MLP
  double start_rate = 0;            // hit rate of always guessing the unanchored start
  uint64_t samples = 0;
  uint32_t steps = 0;
  double final_loss = 0;
};

// Trains (or retrains) the proposer of `plan` on `corpus` (device pointer).
void proposer_train(RegexPlan& plan, const uint8_t* d_corpus, uint64_t len, uint64_t seed, int sm_count,
                    ProposerStats* stats);
void proposer_destroy(Proposer* p);
// Writes one guessed start state per (group, chunk) into guess (state rows,
// layout [group][chunk]; chunk 0 is not written).  Returns the number of
// launches.
uint32_t proposer_predict(Proposer& p, const uint8_t* data, uint64_t len, uint64_t chunk, uint64_t n_chunks,
                          uint32_t* guess, cudaStream_t st);

// ---------------------------------------------- tcgen05 inference (ws_proposer_tc.cu)
constexpr int kTcMaxGemms = 40;  // 2 hidden layers + up to 38 head chunks of 4 groups

// The MLP's weights packed for the tensor-core kernel: per GEMM, four K
// slices of N x 64 BF16 in the shared-memory operand layout, each slice one
// contiguous block for a single bulk copy.
struct TcPlan {
  DeviceBuffer blob, err;
  uint32_t n_gemm = 0;
  uint16_t gemm_n[kTcMaxGemms] = {};
  uint32_t gemm_off[kTcMaxGemms] = {};
  int sm_count = 0;
  bool ready = false;
};

struct TcInputs {
  const uint8_t* data;
  uint64_t chunk, n_chunks;
  const uint8_t* jmap;
  const void* E;  // BF16 embeddings [classes][16]
  uint32_t n_emb;  // classes (at most 64)
  const float *b1, *b2, *b3;
  const uint32_t* vocab;
  uint32_t G;
  uint32_t* guess;
};

// Packs W1T, W2T ([256][256]) and W3T ([n_out][256]) (device BF16) into tp.
// Leaves tp.ready false when the head count does not fit the kernel.
void tc_prepare(TcPlan& tp, const void* W1T, const void* W2T, const void* W3T, uint32_t n_out);
uint32_t tc_predict(const TcPlan& tp, const TcInputs& in, cudaStream_t st);

}  // namespace ws
