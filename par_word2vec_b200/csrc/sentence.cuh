// Per-sentence learning rate and random-stream seed shared by the BATCHED kernels.
#pragma once
#include <cstdint>

#include "common.cuh"
#include "internal.h"

namespace parw2v {

// The epoch being trained lives in device memory, so that one captured epoch (a CUDA graph) can
// be replayed for every epoch: a kernel at the end of the epoch advances it.  Kernels read it
// once, at their start.
__device__ __forceinline__ int hogwild_epoch(const TrainArgs &a) { return (int) a.cnt->epoch; }

// alpha for a sentence that starts after kept_before kept tokens of this epoch: the reference's
// linear decay over iter * train_words words (PAR_Word2Vec_cpu.cpp:431-446), with the position in
// the epoch measured in kept tokens and scaled to raw tokens; floor alpha0 * 1e-4.
__device__ __forceinline__ float sentence_alpha_b(const TrainArgs &a, int epoch, uint64_t kept_before, uint64_t total_kept) {
    const double done = (double) epoch * (double) a.n_tokens +
                        (total_kept ? (double) kept_before / (double) total_kept : 0.0) * (double) a.n_tokens;
    float alpha = a.alpha0 * (float) (1.0 - done / ((double) a.iter * (double) a.train_words + 1.0));
    const float floor_a = a.alpha0 * 0.0001f;
    return alpha < floor_a ? floor_a : alpha;
}

// The sentence's LCG seed in the Hogwild modes: a hash of (seed, epoch, line, 1000-token piece).
__device__ __forceinline__ uint64_t sentence_seed_b(const TrainArgs &a, int epoch, uint64_t line, int piece) {
    return mix64(mix64(a.seed ^ (0xD1B54A32D192ED03ULL * (uint64_t) (epoch + 1))) ^ (line * 1024ULL + piece));
}

}  // namespace parw2v
