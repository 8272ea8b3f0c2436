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
// Writes one guessed start state per (group, chunk) into guess (premultiplied
// state offsets, layout [group][chunk]; chunk 0 is not written).  Returns the
// number of launches.
uint32_t proposer_predict(Proposer& p, const uint8_t* data, uint64_t len, uint64_t chunk, uint64_t n_chunks,
                          uint32_t* guess, cudaStream_t st);

}  // namespace ws
