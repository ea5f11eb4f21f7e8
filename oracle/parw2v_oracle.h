/*
 * oracle/parw2v_oracle.h -- TEST INFRASTRUCTURE ONLY.  Never linked into the product
 * library; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it,
 * and only as the checker.
 *
 * A single-threaded C restatement of PAR-Word2Vec's CPU training loop
 * (PAR_Word2Vec_cpu.cpp:372-711, thread id 0 of 1) and of its set-up tables
 * (expTable :822-826, unigram table :96-117, InitNet :337-357).  It is pinned
 * bit-for-bit against the reference compiled from its own source (oracle/_ref,
 * tests/golden/) and additionally emits a trace of every random decision, which the
 * CUDA deterministic mode is compared against.
 */
#ifndef PARW2V_ORACLE_H
#define PARW2V_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PWO_TABLE_SIZE 100000000
#define PWO_EXP_TABLE_SIZE 1000

typedef struct {
    int vocab_size;      /* V, including "</s>" at index 0 */
    int hidden_size;     /* -size */
    int window;          /* -window */
    int negative;        /* -negative */
    int batch_size;      /* -batch-size */
    int iter;            /* -iter */
    float alpha;         /* -alpha */
    float sample;        /* -sample */
    uint64_t seed;       /* initial LCG state; the reference uses the OpenMP thread id (0) */
    int sync_window;     /* 0: the reference's attraction (each context sees the target row as the
                            previous context left it); 1: window-synchronous variant (all contexts
                            of a target are scored against the same target row, then every update
                            is applied; repeated context words accumulate into one row) */
} pwo_config;

/* Optional trace.  Each array may be NULL; entries beyond *_cap are counted, not stored. */
typedef struct {
    uint8_t *keep;   int64_t keep_cap;   int64_t n_keep;   /* per token read: 0 dropped, 1 kept, 2 "</s>" */
    uint8_t *b;      int64_t b_cap;      int64_t n_b;      /* per attraction step: window shrink b */
    float *alpha;    int64_t alpha_cap;  int64_t n_alpha;  /* per attraction step: learning rate used */
    uint8_t *rep_b;  int64_t rep_b_cap;  int64_t n_rep_b;  /* per repulsion batch: rep_b */
    int32_t *neg;    int64_t neg_cap;    int64_t n_neg;    /* per shared negative, in draw order */
    int64_t n_pairs;                                       /* attraction (context, target) updates */
    int64_t n_sentences;                                   /* non-empty sentences trained */
    uint64_t words_read;                                   /* word_count summed over epochs */
    uint64_t final_lcg;                                    /* LCG state at exit */
} pwo_trace;

/* expTable[1001]: sigma on [-6, 6] (PAR_Word2Vec_cpu.cpp:822-826) */
void pwo_exp_table(float *exp_table);
/* unigram^0.75 table of PWO_TABLE_SIZE ints (PAR_Word2Vec_cpu.cpp:96-117) */
void pwo_unigram_table(const uint32_t *counts, int vocab_size, int32_t *table);
/* W_in LCG-uniform, W_out zero (PAR_Word2Vec_cpu.cpp:337-357) */
void pwo_init_net(float *w_in, float *w_out, int vocab_size, int hidden_size);
/* The training loop.  stream holds n_tokens vocab ids followed by one extra 0 (the
 * sentinel loadStream writes, PAR_Word2Vec_cpu.cpp:368).  Returns 0, or -1 on bad
 * arguments, or -2 if a negative resampling loop exceeded max_resample draws (the
 * reference would spin forever there). */
int pwo_train(const pwo_config *cfg, const uint32_t *counts, const int32_t *table,
              const float *exp_table, const int32_t *stream, uint64_t n_tokens,
              float *w_in, float *w_out, pwo_trace *trace, int64_t max_resample);

#ifdef __cplusplus
}
#endif
#endif
