// Internal declarations of libparw2v: the context and the kernel launchers.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "../../include/parw2v.h"

namespace parw2v {

// Device-side counters, one struct per context (zeroed before each training call).
struct DevCounters {
    unsigned long long words, kept, sentences, pairs, batches, negatives;
    unsigned long long n_keep, n_b, n_alpha, n_rep_b, n_neg;  // trace fill levels (DET)
    unsigned long long final_lcg;
    unsigned long long work;        // persistent-grid work counter
    unsigned long long n_lines;     // "</s>"-terminated lines in the corpus (set by packing)
    unsigned long long total_kept;  // kept tokens after subsampling (set by packing)
    float final_alpha;
    unsigned error;                 // kErr* bits
    unsigned epoch;                 // Hogwild modes: the epoch being trained (advanced on the device)
};

// Trace buffers on the device (DET mode)
struct DevTrace {
    uint8_t *keep = nullptr; int64_t keep_cap = 0;
    uint8_t *b = nullptr; int64_t b_cap = 0;
    float *alpha = nullptr; int64_t alpha_cap = 0;
    uint8_t *rep_b = nullptr; int64_t rep_b_cap = 0;
    int32_t *neg = nullptr; int64_t neg_cap = 0;
};

// Arguments common to every training kernel
struct TrainArgs {
    const int32_t *corpus;   // n_tokens ids + sentinel 0
    uint64_t n_tokens;
    const float *keep_thr;   // per word: sqrtf(r) + r, r = sample * train_words / cn
    const int32_t *table;    // unigram table
    const float *exp_table;  // 1001 entries
    void *w_in, *w_out;      // FP32 or BF16 [V][ld]
    int ld;                  // row stride in elements (16-byte multiple)
    int d, window, negative, batch, iter, vocab;
    float alpha0, sample;
    uint64_t train_words;
    uint64_t seed;
    DevCounters *cnt;
    // Hogwild packing products
    const int32_t *packed;   // kept tokens in corpus order
    const uint32_t *line_end;  // per "</s>": index into packed one past the line's last token
    float *scratch;          // per-warp workspace (PLAIN), per-context workspace (DET)
    size_t scratch_per_warp; // floats
    int64_t max_resample;
    int sync_window;         // window-synchronous attraction (PARW2V_ATTRACT_WINDOW)
    int stage_bulk;          // BATCHED repulsion staging: 1 bulk copies (TMA unit), 0 16-byte cp.async
    int lane_elems;          // streamed kernel: row elements per lane (0 = the smallest that holds d)
    int attr_pipe;           // streamed kernel: sequential attraction in its pipelined form
};

// Launchers (return a cudaError_t)
cudaError_t launch_build_thresholds(const uint32_t *counts, int V, float sample, uint64_t train_words,
                                    float *keep_thr, cudaStream_t s);
cudaError_t launch_build_table(const double *pow_cn, int V, int32_t *table, float *d_thr_f,
                               long long *start, double *total, cudaStream_t s);
cudaError_t launch_init_net(float *w_in, float *w_out, __nv_bfloat16 *b_in, __nv_bfloat16 *b_out, int V,
                            int d, int ld, cudaStream_t s);
cudaError_t launch_det_train(const TrainArgs &a, const DevTrace &tr, cudaStream_t s, size_t *smem_needed);
cudaError_t launch_advance_epoch(DevCounters *cnt, cudaStream_t s);
cudaError_t launch_count_zeros(const int32_t *corpus, uint64_t n, DevCounters *cnt, cudaStream_t s);
cudaError_t launch_pack(const TrainArgs &a, int32_t *packed, uint32_t *line_end, uint32_t *tile_kept,
                        uint32_t *tile_zero, uint64_t n_tiles, cudaStream_t s);
uint64_t pack_tiles(uint64_t n_tokens);
cudaError_t launch_plain_train(const TrainArgs &a, int grid, int warps_per_cta, cudaStream_t s);
cudaError_t launch_batched_train(const TrainArgs &a, bool bf16, bool stream, int grid, int warps_per_cta, cudaStream_t s);
size_t plain_scratch_floats(int ld, int batch, int window, int negative);
int plain_warps_per_cta(int requested);
int batched_max_warps(int ld, int window, int negative, int batch, bool bf16, size_t *smem_per_warp, bool stream);
bool batched_tensor_repulsion(int window, int negative, int batch);  // the BATCHED modes' repulsion path
// CTAs of `warps` warps of the BATCHED kernel that fit on one SM at once (shared memory, threads,
// registers at the kernel's 128-register bound)
int batched_ctas_per_sm(int ld, int window, int negative, int batch, bool bf16, bool stream, int warps);
// the streamed kernel's row elements per lane: the default for d, and the next larger one (0 if none)
int stream_lane_elems_default(int d);
int stream_lane_elems_next(int e);

// Loss / adjoint / finite differences
struct LossBatch {
    const int32_t *tgt, *ctx, *neg;
    int n_pairs, n_neg, ctx_per_window;
};
cudaError_t launch_loss(const LossBatch &b, const void *w_in, const void *w_out, bool bf16, int d, int ld,
                        double *out, cudaStream_t s);
cudaError_t launch_adjoint(const LossBatch &b, const void *w_in, const void *w_out, bool bf16, int d, int ld,
                           const float *exp_table, int exact, float *g_in, float *g_out, cudaStream_t s);
cudaError_t launch_loss_fd(const LossBatch &b, const void *w_in, const void *w_out, bool bf16, int d, int ld,
                           const int32_t *matrix, const int32_t *row, const int32_t *col, int n_probes, double h,
                           double *grad, cudaStream_t s);
// Records the text parw2v_last_error(NULL) returns; returns code.
int set_global_error(int code, const char *msg);
// Weight rows between the device layout (rows of ld elements, FP32 or BF16, padding zero) and dense
// FP32 rows of d elements (the caller's layout); `rows` rows starting at the given pointers.
cudaError_t launch_rows_to_dense(const void *dev, bool bf16, int ld, float *dst, int d, size_t rows, cudaStream_t s);
cudaError_t launch_rows_from_dense(const float *src, int d, void *dev, bool bf16, int ld, size_t rows, cudaStream_t s);

}  // namespace parw2v
