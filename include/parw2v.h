/*
 * parw2v.h -- C ABI of the B200-native PAR-Word2Vec training library (libparw2v.so).
 *
 * The reference has no library interface: its boundary is the command line, the text
 * files and the globals that Train_PAR_Word2Vec() works on.  Each entry point below
 * names the reference code it replaces.  File:line citations are into the reference
 * project (PAR_Word2Vec_cpu.cpp, PAR_Word2Vec_gpu_text.cu / _graph.cu).
 *
 * Conventions
 *   - Every function returns PARW2V_OK (0) or a negative PARW2V_ERR_* status; nothing
 *     calls exit() (the reference calls exit(0) on CUDA errors, gpu_text.cu:42-48, and
 *     exit(1) on a missing file, cpu.cpp:259-262).
 *   - Host pointers belong to the caller and are copied in or out during the call.
 *     All device memory belongs to the context.
 *   - A context is single-threaded: its calls are serialised on the context's own CUDA
 *     stream.  Distinct contexts may be used from distinct threads.
 *   - No CPU fallback: a context cannot be created without a CUDA device.
 */
#ifndef PARW2V_H
#define PARW2V_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PARW2V_OK 0
#define PARW2V_ERR_ARG (-1)      /* invalid argument or configuration */
#define PARW2V_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define PARW2V_ERR_OOM (-3)      /* device allocation failed or exceeds mem_cap_bytes */
#define PARW2V_ERR_CAPACITY (-4) /* an input exceeds a fixed limit of the library */
#define PARW2V_ERR_TIMEOUT (-5)  /* a bounded device loop gave up (e.g. negative resampling) */
#define PARW2V_ERR_STATE (-6)    /* call order violated (e.g. train before set_vocab) */
#define PARW2V_ERR_IO (-7)       /* file could not be read or written */
#define PARW2V_ERR_NODEV (-8)    /* no CUDA device / library built without one */

/* Execution modes of parw2v_train */
#define PARW2V_MODE_DET 0          /* one CTA walks the stream in reference order: bit-exact with
                                      PAR_Word2Vec_cpu at -threads 1 (cpu.cpp:430-687) */
#define PARW2V_MODE_PLAIN 1        /* FP32 Hogwild, a warp per sentence, rows in global memory */
#define PARW2V_MODE_BATCHED 2      /* FP32, persistent data-local kernel: sentence rows staged
                                      on chip, shared-negative repulsion per batch */
#define PARW2V_MODE_BATCHED_BF16 3 /* as BATCHED, W_in/W_out stored in BF16, FP32 accumulation,
                                      stochastic rounding on write-back */

typedef struct {
    int size;        /* -size: hidden size d (cpu.cpp:787-788) */
    int window;      /* -window (cpu.cpp:803-804) */
    int negative;    /* -negative (cpu.cpp:807-808) */
    int batch_size;  /* -batch-size (cpu.cpp:815-816); the reference CPU default is 24 */
    int iter;        /* -iter (cpu.cpp:811-812) */
    float alpha;     /* -alpha: starting learning rate (cpu.cpp:799-800) */
    float sample;    /* -sample: subsampling threshold, 0 = off (cpu.cpp:805-806) */
    int mode;        /* PARW2V_MODE_* */
    int device;      /* CUDA device ordinal */
    uint64_t seed;   /* DET: initial LCG state (the reference uses the OpenMP thread id, 0);
                        Hogwild modes: seed of the per-sentence LCG streams */
    int grid;        /* Hogwild modes: persistent CTAs, 0 = one wave of the device */
    int warps_per_cta; /* Hogwild modes: sentences in flight per CTA, 0 = tuned default */
    size_t mem_cap_bytes; /* refuse device allocations beyond this total, 0 = no cap */
    int min_rounds;  /* Hogwild modes: cap on sentences in flight, so that a small corpus is not
                        processed almost all at once from stale weights.  0 = default:
                        max(7,000 corpus tokens' worth of lines, lines / 8192); > 0: lines /
                        min_rounds; < 0: no cap */
    int attraction;  /* PARW2V_ATTRACT_*: how the contexts of one target are applied */
    int variant;     /* BATCHED modes: PARW2V_VARIANT_* kernel organisation */
    int staging;     /* BATCHED modes: PARW2V_STAGING_* copies of the repulsion's rows into
                        shared memory */
    int autotune;    /* BATCHED modes: 1 = on the first parw2v_train (and whenever the number of
                        sentences in flight changes), time short trials of the launch knobs that
                        do not change the result -- the kernel organisation (unless cfg.variant fixes
                        it), the split of the sentences in flight into CTAs
                        and warps, the row elements per lane of the streamed kernel, the staging
                        copies (unless cfg.staging fixes them) and, with PARW2V_ATTRACT_DEFAULT, the
                        sequential attraction's plain or pipelined form -- on a prefix of the first epoch, with
                        the weights restored after each trial, and keep the fastest (with the
                        environment variable PARW2V_AUTOTUNE_LOG set, each trial's time is printed
                        on stderr); 0 = the compiled-in choices */
} parw2v_config;

/* Repulsion staging of the BATCHED modes (cfg.staging); the result does not depend on it */
#define PARW2V_STAGING_AUTO 0     /* CPASYNC (measured faster for these 64-byte row chunks) */
#define PARW2V_STAGING_BULK 1     /* one bulk copy (cp.async.bulk, the TMA unit) per row and column
                                     chunk, completing on a shared-memory mbarrier, and one bulk
                                     store per row and chunk for the BF16 write-back */
#define PARW2V_STAGING_CPASYNC 2  /* 16-byte cp.async copies and 16-byte stores */

/* Kernel organisation of the BATCHED modes (cfg.variant) */
#define PARW2V_VARIANT_AUTO 0    /* STREAM */
#define PARW2V_VARIANT_WINDOW 1  /* the window's W_in rows held in shared memory as FP32 working
                                    copies, written back once per window exit */
#define PARW2V_VARIANT_STREAM 2  /* rows read and written in global memory (L1-resident while the
                                    window reuses them); more sentences in flight per SM */

/* Attraction variants (cfg.attraction) */
#define PARW2V_ATTRACT_DEFAULT 0    /* SEQUENTIAL */
#define PARW2V_ATTRACT_SEQUENTIAL 1 /* the reference: each context sees the target row as the
                                       previous context left it (cpu.cpp:536-567) */
#define PARW2V_ATTRACT_WINDOW 2     /* window-synchronous: all contexts of a target are scored
                                       against the same target row, then all updates are applied
                                       (the contexts x d by d x 1 contraction of the window) */
#define PARW2V_ATTRACT_PIPELINED 3  /* SEQUENTIAL's updates in SEQUENTIAL's order, with the score of
                                       each next context formed as x'.y + g (x'.x) while the current
                                       gradient g is looked up (equal up to FP32 rounding).  The
                                       BATCHED streamed kernel only; DET and PLAIN run SEQUENTIAL */

typedef struct {
    uint64_t words;      /* raw tokens read incl. "</s>" over all epochs: the reference's
                            word_count (cpu.cpp:456), the numerator of words/sec */
    uint64_t kept;       /* positions trained after subsampling */
    uint64_t sentences;  /* non-empty sentences trained */
    uint64_t pairs;      /* attraction (context, target) updates */
    uint64_t batches;    /* repulsion batches */
    uint64_t negatives;  /* shared negatives drawn */
    double kernel_ms;    /* device time of the training kernels (CUDA events) */
    double pack_ms;      /* device time of subsampling + packing (Hogwild modes) */
    float final_alpha;   /* learning rate at the end */
    int grid;            /* Hogwild modes: persistent CTAs of the training kernel's launch */
    int warps_per_cta;   /* Hogwild modes: sentences in flight per CTA */
    int repulsion;       /* PARW2V_REPULSION_* path the training kernel took for the batches */
    int lane_elems;      /* BATCHED streamed kernel: row elements each lane holds */
    int staging;         /* BATCHED modes: PARW2V_STAGING_BULK or _CPASYNC as launched */
    int attraction;      /* PARW2V_ATTRACT_* form the training kernel ran */
    int variant;         /* BATCHED modes: PARW2V_VARIANT_STREAM or _WINDOW as launched */
} parw2v_stats;

/* parw2v_stats.repulsion */
#define PARW2V_REPULSION_SERIAL 0   /* DET and PLAIN: the reference's three products in order */
#define PARW2V_REPULSION_TENSOR 1   /* BATCHED: warp-level tensor-core products (batch <= 32 rows,
                                       (2*window-1)*negative <= 96 negatives) */
#define PARW2V_REPULSION_CUDA 2     /* BATCHED: CUDA-core products (larger batches) */

/* Deterministic-mode trace: the random decisions of the run, for parity checks. Host
 * buffers; an entry beyond a capacity is counted but not stored. */
typedef struct {
    uint8_t *keep;   int64_t keep_cap;   int64_t n_keep;   /* per token read: 0 dropped, 1 kept, 2 "</s>" */
    uint8_t *b;      int64_t b_cap;      int64_t n_b;      /* per attraction step: window shrink b */
    float *alpha;    int64_t alpha_cap;  int64_t n_alpha;  /* per attraction step: learning rate */
    uint8_t *rep_b;  int64_t rep_b_cap;  int64_t n_rep_b;  /* per repulsion batch: rep_b */
    int32_t *neg;    int64_t neg_cap;    int64_t n_neg;    /* shared negatives in draw order */
    uint64_t final_lcg;                                    /* LCG state at the end */
} parw2v_trace;

typedef struct parw2v_ctx parw2v_ctx;

/* Library identification and error text. */
const char *parw2v_version(void);
const char *parw2v_strerror(int status);
/* Detail of the last error on this context.  With ctx NULL: the calling thread's last error of a
 * call that has no context (parw2v_create, parw2v_det_train_noalloc, parw2v_random_walks). */
const char *parw2v_last_error(const parw2v_ctx *ctx);

/* Replaces the globals set by main() + the device set-up of gpu_text.cu:1090-1100.
 * Validates the configuration, selects the device and creates the context's stream. */
int parw2v_create(const parw2v_config *cfg, parw2v_ctx **out);
void parw2v_destroy(parw2v_ctx *ctx);

/* Vocabulary counts in vocabulary order, index 0 = "</s>" (SortVocab, cpu.cpp:204-226).
 * Builds on the device: the 1e8-entry unigram^0.75 table (InitUnigramTable, cpu.cpp:96-117;
 * FP64 normalisation, byte-equal with the reference), expTable (cpu.cpp:822-826) and the
 * per-word subsampling thresholds (cpu.cpp:459-460).  train_words = sum of counts. */
int parw2v_set_vocab(parw2v_ctx *ctx, const uint32_t *counts, int vocab_size);

/* Copies of the device tables, for checks: table has 100,000,000 entries, exp_table 1001. */
int parw2v_get_table(parw2v_ctx *ctx, int32_t *table);
int parw2v_get_exp_table(parw2v_ctx *ctx, float *exp_table);

/* InitNet (cpu.cpp:337-357) on the device: W_in from the seed-1 LCG, W_out = 0. */
int parw2v_init_weights(parw2v_ctx *ctx);
/* Host <-> device copies of the vocab_size x size row-major FP32 matrices (either may be
 * NULL).  In BF16 mode set_weights rounds to nearest and get_weights widens exactly.  The
 * rows pass through a device staging buffer of at most 64 MiB, allocated on first use, kept
 * by the context and counted against mem_cap_bytes.  Host buffers may be pageable; pinned
 * buffers (cudaHostAlloc) move at the full host-link speed. */
int parw2v_set_weights(parw2v_ctx *ctx, const float *w_in, const float *w_out);
int parw2v_get_weights(parw2v_ctx *ctx, float *w_in, float *w_out);

/* The word-id stream loadStream produces (cpu.cpp:359-370): n_tokens ids in corpus
 * order, out-of-vocabulary words already dropped, 0 = "</s>".  The library appends the
 * sentinel 0 itself. */
int parw2v_set_corpus(parw2v_ctx *ctx, const int32_t *tokens, uint64_t n_tokens);

/* Train_PAR_Word2Vec's epoch loop (cpu.cpp:397-700; gpu_text.cu:879-952): cfg.iter
 * epochs over the corpus in the configured mode.  stats may be NULL. */
int parw2v_train(parw2v_ctx *ctx, parw2v_stats *stats);

/* DET mode only: record the random decisions of the next parw2v_train into trace
 * (host buffers, filled when train returns).  NULL switches tracing off. */
int parw2v_set_trace(parw2v_ctx *ctx, parw2v_trace *trace);

/* ---- SGNS loss and its adjoint (no reference counterpart as a function: the reference
 * applies the gradient in place, cpu.cpp:550-565 and :633-674) ----
 * A minibatch is n_pairs (target, context) pairs; pairs [w*ctx_per_window,
 * (w+1)*ctx_per_window) form window w and share the n_neg negatives
 * neg[w*n_neg .. (w+1)*n_neg).  All ids index the vocabulary.
 *   L = sum_p [ -log s(u_c . v_t) - sum_{k in window} log s(-u_c . v_k) ],
 * u = W_in rows, v = W_out rows, s = logistic.  Dot products are FP32 over the stored
 * weights (BF16 widened exactly in BF16 mode); log s and the reduction are FP64. */
int parw2v_loss(parw2v_ctx *ctx, const int32_t *tgt, const int32_t *ctxw, int n_pairs,
                const int32_t *neg, int n_neg, int ctx_per_window, double *loss);
/* dL/dW_in and dL/dW_out as dense vocab_size x size FP32 host matrices (either may be
 * NULL), all terms evaluated at the same weights.  exact = 1: s computed exactly (the
 * adjoint of parw2v_loss).  exact = 0: s from expTable with the +-6 clamp, i.e. -1/alpha
 * times the reference's update rule (cpu.cpp:554-559 attraction, :642-647 repulsion). */
int parw2v_loss_adjoint(parw2v_ctx *ctx, const int32_t *tgt, const int32_t *ctxw, int n_pairs,
                        const int32_t *neg, int n_neg, int ctx_per_window, int exact,
                        float *d_w_in, float *d_w_out);
/* FP64 central finite differences of L on the device: for each probe i,
 * (L(W + h e_i) - L(W - h e_i)) / (2h) where e_i is element (row[i], col[i]) of W_in
 * (matrix[i] == 0) or W_out (matrix[i] == 1).  Weights are widened to FP64 exactly. */
int parw2v_loss_fd(parw2v_ctx *ctx, const int32_t *tgt, const int32_t *ctxw, int n_pairs,
                   const int32_t *neg, int n_neg, int ctx_per_window, const int32_t *matrix,
                   const int32_t *row, const int32_t *col, int n_probes, double h, double *grad);

/* ---- Random walks for the graph workload (no counterpart in the reference: it trains on walk
 * files made by other tools, data.sh:7-11) ----
 * walks_per_node * n_nodes uniform random walks of walk_len nodes over the graph in CSR form
 * (indptr[n_nodes + 1] starting at 0, indices[indptr[n_nodes]] neighbour ids), computed on
 * the GPU `device`.  Walk w starts at node w mod n_nodes; step s picks neighbour
 * (hi32(h) * degree) >> 32 with h = mix64(seed ^ mix64(w * 2^20 + s)) (SplitMix64 finaliser), so
 * every walk is reproducible on its own.  A node without neighbours repeats to the walk's end.
 * out_nodes receives walks_per_node * n_nodes * walk_len ids, walk after walk (host memory). */
int parw2v_random_walks(const int64_t *indptr, const int32_t *indices, int n_nodes, int walks_per_node,
                        int walk_len, uint64_t seed, int device, int32_t *out_nodes);

/* ---- Allocation-free deterministic training (no counterpart in the reference) ----
 * For callers that cannot let a library allocate device memory: a framework whose caching
 * allocator owns the GPU's memory, or a service that reserves its memory at start-up and must not
 * meet an allocation failure later.  It runs the DET-mode training (bit-identical to parw2v_train
 * in PARW2V_MODE_DET) on device buffers the caller owns and calls no cudaMalloc/cudaFree: its
 * scratch is a 1 MiB array in the library's static device memory, held by every GPU that loads
 * the library until the process exits.  Limit: (batch_size + 2*window*negative) * ld * 4 bytes
 * must fit in that 1 MiB less 256 bytes, else PARW2V_ERR_CAPACITY.
 *   d_corpus     n_tokens word ids followed by one 0 (the "</s>" sentinel), device memory
 *   d_table      the 100,000,000-entry unigram table (as parw2v_get_table returns it)
 *   d_exp_table  the 1001-entry sigma table (as parw2v_get_exp_table returns it)
 *   d_keep_thr   per word: r = (sample * (float) train_words) / (float) count, sqrtf(r) + r, FP32
 *   d_w_in/out   vocab_size rows of ld floats, trained in place
 *   stream       a cudaStream_t (NULL = the default stream); the call returns after the stream
 *                has finished the training, with stats filled (may be NULL)
 * cfg.device selects the GPU (made current for the call).  Each call looks up the array's device
 * address in the current context, clears the counters at the array's start and waits for the
 * stream: the call is synchronous, and must not be made while its stream is being captured.  All
 * calls share the one array and it keeps the last call's contents, so calls that overlap on the
 * same GPU (from several threads or several streams) race: serialise them. */
int parw2v_det_train_noalloc(const parw2v_config *cfg, int vocab_size, uint64_t train_words,
                             const int32_t *d_corpus, uint64_t n_tokens, const int32_t *d_table,
                             const float *d_exp_table, const float *d_keep_thr, float *d_w_in,
                             float *d_w_out, int ld, void *stream, parw2v_stats *stats);

/* ---- Host front end (reference-identical text handling; no device needed) ---- */

/* LearnVocabFromTrainFile + SortVocab (cpu.cpp:253-292, :204-226): reads a text corpus
 * with the reference's tokenizer, keeps words with count >= min_count (plus "</s>"),
 * orders them exactly as the reference's qsort does.  On success *vocab holds the
 * handle used by the functions below. */
typedef struct parw2v_vocab parw2v_vocab;
int parw2v_vocab_learn(const char *train_file, int min_count, parw2v_vocab **vocab);
/* ReadVocab (cpu.cpp:301-335): a "word count" per line file, then SortVocab. */
int parw2v_vocab_read(const char *vocab_file, int min_count, parw2v_vocab **vocab);
void parw2v_vocab_free(parw2v_vocab *vocab);
int parw2v_vocab_size(const parw2v_vocab *vocab);
uint64_t parw2v_vocab_train_words(const parw2v_vocab *vocab);
/* counts[vocab_size] in vocabulary order */
int parw2v_vocab_counts(const parw2v_vocab *vocab, uint32_t *counts);
const char *parw2v_vocab_word(const parw2v_vocab *vocab, int index);
/* SaveVocab (cpu.cpp:294-299) */
int parw2v_vocab_save(const parw2v_vocab *vocab, const char *path);
/* loadStream for one reader over the whole file (cpu.cpp:359-370): the id stream of the
 * corpus without the sentinel.  Call with tokens == NULL to get the length first. */
int parw2v_load_stream(const parw2v_vocab *vocab, const char *train_file, int32_t *tokens,
                       uint64_t capacity, uint64_t *n_tokens);
/* saveModel (cpu.cpp:721-737): "V d" header, then per word its string and d values
 * ("%f " text, or raw float32 when binary != 0). */
int parw2v_save_model(const parw2v_vocab *vocab, const float *w_in, int size, int binary,
                      const char *path);

#ifdef __cplusplus
}
#endif
#endif
