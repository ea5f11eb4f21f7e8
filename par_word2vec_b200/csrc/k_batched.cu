// BATCHED / BATCHED_BF16 modes (data-local persistent kernel) -- placeholder until implemented.
#include "common.cuh"
#include "internal.h"

namespace parw2v {

int batched_max_warps(int, int, int, int, bool, size_t *per_warp) {
    if (per_warp) *per_warp = 0;
    return 0;
}

cudaError_t launch_batched_train(const TrainArgs &, bool, int, int, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace parw2v
