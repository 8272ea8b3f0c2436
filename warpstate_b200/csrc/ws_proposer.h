// Learned boundary-state proposer of the speculative DFA walk.
#pragma once
#include "ws_internal.h"

namespace ws {

struct RegexPlan;
struct Proposer;

// Trains the proposer on a seeded synthetic corpus (returns nullptr when the
// plan has nothing to learn).  Fills plan.top1/top4 with held-out hit rates.
Proposer* proposer_train(RegexPlan& plan, const ws_config& cfg);
void proposer_destroy(Proposer* p);
// Writes one guessed start state per (group, chunk) into guess (premultiplied
// state offsets, layout [group][chunk]).  Returns the number of launches.
uint32_t proposer_predict(Proposer& p, const uint8_t* d_cls, const uint8_t* data, uint64_t len, uint64_t chunk,
                          uint64_t n_chunks, uint32_t* guess, cudaStream_t st);

}  // namespace ws
