/*
 * oracle/parw2v_oracle.c -- TEST INFRASTRUCTURE ONLY (see parw2v_oracle.h).
 *
 * Restates, for one thread, what PAR_Word2Vec_cpu.cpp does.  Floating-point
 * expressions keep the reference's types and evaluation order so that, built with
 * -ffp-contract=off, results are bit-identical to the reference built the same way:
 *   - dot products sum j = 0..d-1 in order, one rounding per multiply and per add;
 *   - the three repulsion GEMMs sum their inner index in ascending order, which is
 *     the order oracle/mkl.h fixes for cblas_sgemm.
 */
#include "parw2v_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAX_EXP 6
#define MAX_SENTENCE_LENGTH 1000
/* EXP_TABLE_SIZE / (MAX_EXP * 2.0f), PAR_Word2Vec_cpu.cpp:70 */
static const float kExpResolution = PWO_EXP_TABLE_SIZE / (MAX_EXP * 2.0f);

static inline uint64_t lcg_next(uint64_t x) { return x * (uint64_t) 25214903917ULL + 11ULL; }

/* PAR_Word2Vec_cpu.cpp:822-826.  The reference is C++: exp() of a float argument
 * resolves to the float overload, i.e. expf. */
void pwo_exp_table(float *t) {
    for (int i = 0; i < PWO_EXP_TABLE_SIZE + 1; i++) {
        float x = ((float) i / (float) PWO_EXP_TABLE_SIZE * 2.0f - 1.0f) * (float) MAX_EXP;
        float e = expf(x);
        t[i] = e / (e + 1.0f);
    }
}

/* PAR_Word2Vec_cpu.cpp:96-117.  pow(unsigned, float) promotes both to double; the
 * running threshold d1 is a float that absorbs double quotients; the slot position is
 * the float quotient a / 1e8f. */
void pwo_unigram_table(const uint32_t *cn, int V, int32_t *table) {
    const double power = (double) 0.75f;
    double total = 0.0;
    for (int i = 0; i < V; i++) total += pow((double) cn[i], power);
    int i = 0;
    float d1 = (float) (pow((double) cn[0], power) / total);
    for (int a = 0; a < PWO_TABLE_SIZE; a++) {
        table[a] = i;
        if ((float) a / (float) PWO_TABLE_SIZE > d1) {
            i++;
            /* the reference reads vocab[V] here once i == V; the table is clamped to V-1
               from then on whatever d1 becomes, so the value added does not matter */
            double q = (i < V) ? pow((double) cn[i], power) / total : 0.0;
            d1 = (float) ((double) d1 + q);
        }
        if (i >= V) i = V - 1;
    }
}

/* PAR_Word2Vec_cpu.cpp:337-357 */
void pwo_init_net(float *w_in, float *w_out, int V, int d) {
    const int64_t n = (int64_t) V * d;
    memset(w_out, 0, sizeof(float) * (size_t) n);
    uint64_t r = 1;
    for (int64_t i = 0; i < n; i++) {
        r = lcg_next(r);
        w_in[i] = (((float) (r & 0xFFFF) / 65536.f) - 0.5f) / (float) d;
    }
}

/* g = (label - sigma(f)) * alpha through the clamped table, PAR_Word2Vec_cpu.cpp:554-559 and :642-647 */
static inline float grad_of(float f, int label, float alpha, const float *exp_table) {
    if (f > (float) MAX_EXP) return (float) (label - 1) * alpha;
    if (f < -(float) MAX_EXP) return (float) label * alpha;
    int idx = (int) ((f + (float) MAX_EXP) * kExpResolution);
    return ((float) label - exp_table[idx]) * alpha;
}

static inline int in_sentence(const int *sen, int len, int w) {
    for (int i = 0; i < len; i++)
        if (sen[i] == w) return 1;
    return 0;
}

typedef struct {
    const pwo_config *cfg;
    const uint32_t *cn;
    const int32_t *table;
    const float *exp_table;
    float *w_in, *w_out;
    pwo_trace *tr;
    uint64_t rng;
    float alpha;
    int sen[MAX_SENTENCE_LENGTH];
    int len;
    /* repulsion scratch: M_in [B x d], M_out [2wn x d], M_out_update [2wn x d], M_grad [2wn x B] */
    float *m_in, *m_out, *m_out_upd, *m_grad;
    int *neg;
    int64_t max_resample;
    int failed;
} trainer;

static void trace_u8(uint8_t *arr, int64_t cap, int64_t *n, uint8_t v) {
    if (arr && *n < cap) arr[*n] = v;
    (*n)++;
}

/* Sentence read with subsampling, PAR_Word2Vec_cpu.cpp:447-471. Returns the updated word_count. */
static uint64_t read_sentence(trainer *t, const int32_t *stream, uint64_t word_count, uint64_t train_words) {
    const float sample = t->cfg->sample;
    t->len = 0;
    for (;;) {
        int w = stream[word_count];
        word_count++;
        if (w == 0) {
            if (t->tr) trace_u8(t->tr->keep, t->tr->keep_cap, &t->tr->n_keep, 2);
            break;
        }
        if (sample > 0) {
            float ratio = (sample * (float) train_words) / (float) t->cn[w];
            float ran = sqrtf(ratio) + ratio;
            t->rng = lcg_next(t->rng);
            if (ran < (float) (t->rng & 0xFFFF) / 65536.f) {
                if (t->tr) trace_u8(t->tr->keep, t->tr->keep_cap, &t->tr->n_keep, 0);
                continue;
            }
        }
        if (t->tr) trace_u8(t->tr->keep, t->tr->keep_cap, &t->tr->n_keep, 1);
        t->sen[t->len++] = w;
        if (t->len >= MAX_SENTENCE_LENGTH) break;
    }
    return word_count;
}

/* Window-synchronous attraction (the BATCHED modes' option): every context c of the target is
 * scored against the target row y as it was before this position, f_c = x_c . y (sequential sum),
 * g_c from the table; then y += sum_c g_c x_c (contexts in window order, x_c before update) and
 * x_c += g_c y for each distinct context word (a word occurring twice gets the sum of its g). */
static void attract_sync(trainer *t, int pos, int b, int target) {
    const int d = t->cfg->hidden_size, w = t->cfg->window;
    int ctx[256];
    float g[256];
    int n = 0;
    float *y = t->w_out + (int64_t) target * d;
    for (int i = b; i < 2 * w + 1 - b && n < 256; i++) {
        if (i == w) continue;
        const int c = pos - w + i;
        if (c < 0) continue;
        if (c >= t->len) break;
        const float *x = t->w_in + (int64_t) t->sen[c] * d;
        float f = 0.f;
        for (int j = 0; j < d; j++) {
            float p = x[j] * y[j];
            f = f + p;
        }
        ctx[n] = t->sen[c];
        g[n] = grad_of(f, 1, t->alpha, t->exp_table);
        n++;
        if (t->tr) t->tr->n_pairs++;
    }
    for (int i = 0; i < n; i++)  /* merge repeated context words into their first occurrence */
        for (int k = 0; k < i; k++)
            if (ctx[k] == ctx[i]) {
                g[k] = g[k] + g[i];
                g[i] = 0.f;
                break;
            }
    for (int j = 0; j < d; j++) {
        const float yj = y[j];
        float dy = 0.f;
        for (int i = 0; i < n; i++) {
            float *x = t->w_in + (int64_t) ctx[i] * d;
            float p = g[i] * x[j];
            dy = dy + p;
        }
        for (int i = 0; i < n; i++) {
            if (g[i] == 0.f) continue;
            float *x = t->w_in + (int64_t) ctx[i] * d;
            float p = g[i] * yj;
            x[j] = x[j] + p;
        }
        y[j] = yj + dy;
    }
}

/* One attraction step for sentence position pos, PAR_Word2Vec_cpu.cpp:529-568 */
static void attract(trainer *t, int pos) {
    const int d = t->cfg->hidden_size, w = t->cfg->window;
    const int target = t->sen[pos];  /* stale when len == 0; no context is visited then */
    t->rng = lcg_next(t->rng);
    const int b = (int) (t->rng % (uint64_t) w);
    if (t->tr) {
        trace_u8(t->tr->b, t->tr->b_cap, &t->tr->n_b, (uint8_t) b);
        if (t->tr->alpha && t->tr->n_alpha < t->tr->alpha_cap) t->tr->alpha[t->tr->n_alpha] = t->alpha;
        t->tr->n_alpha++;
    }
    if (t->cfg->sync_window) {
        attract_sync(t, pos, b, target);
        return;
    }
    for (int i = b; i < 2 * w + 1 - b; i++) {
        if (i == w) continue;
        const int c = pos - w + i;
        if (c < 0) continue;
        if (c >= t->len) break;
        float *x = t->w_in + (int64_t) t->sen[c] * d;
        float *y = t->w_out + (int64_t) target * d;
        float f = 0.f;
        for (int j = 0; j < d; j++) {
            float p = x[j] * y[j];
            f = f + p;
        }
        const float g = grad_of(f, 1, t->alpha, t->exp_table);
        for (int j = 0; j < d; j++) {
            float keep_y = g * y[j];
            float dy = g * x[j];
            y[j] = y[j] + dy;
            x[j] = x[j] + keep_y;
        }
        if (t->tr) t->tr->n_pairs++;
    }
}

/* C[M x N] = op(A) op(B), inner index ascending, fresh accumulator per element (oracle/mkl.h order) */
static void gemm_ordered(int M, int N, int K, const float *A, int a_rs, int a_cs,
                         const float *B, int b_rs, int b_cs, float *C, int ldc) {
    for (int i = 0; i < M; i++)
        for (int j = 0; j < N; j++) {
            float acc = 0.0f;
            for (int k = 0; k < K; k++) {
                float p = A[(int64_t) i * a_rs + (int64_t) k * a_cs] * B[(int64_t) k * b_rs + (int64_t) j * b_cs];
                acc = acc + p;
            }
            C[(int64_t) i * ldc + j] = acc;
        }
}

/* Shared-negative repulsion over the whole sentence, PAR_Word2Vec_cpu.cpp:571-679 */
static void repel(trainer *t) {
    const int d = t->cfg->hidden_size, w = t->cfg->window, n = t->cfg->negative;
    const int B = t->cfg->batch_size, V = t->cfg->vocab_size, L = t->len;
    if (L <= 0) return;
    const int num_batch = (L + B - 1) / B;
    for (int nb = 0; nb < num_batch; nb++) {
        const int lo = nb * B;
        const int hi = (lo + (B - 1) < L - 1) ? lo + (B - 1) : L - 1;
        const int rows = hi - lo + 1;
        if (rows <= 0) break;
        int rep_b;
        t->rng = lcg_next(t->rng);
        if (lo <= w - 1 || (L - 1) - lo <= w - 1)
            rep_b = (int) (t->rng % (uint64_t) w);
        else
            rep_b = (int) (t->rng % (uint64_t) (w * 2));
        if (t->tr) trace_u8(t->tr->rep_b, t->tr->rep_b_cap, &t->tr->n_rep_b, (uint8_t) rep_b);
        const int K = rep_b * n;
        for (int k = 0; k < K; k++) {
            t->rng = lcg_next(t->rng);
            int s = t->table[(t->rng >> 16) % (uint64_t) PWO_TABLE_SIZE];
            if (!s) s = (int) (t->rng % (uint64_t) (V - 1) + 1);
            int64_t tries = 0;
            while (in_sentence(t->sen, L, s)) {
                if (++tries > t->max_resample) {
                    t->failed = 1;
                    return;
                }
                t->rng = lcg_next(t->rng);
                s = (int) (t->rng % (uint64_t) (V - 1) + 1);
            }
            t->neg[k] = s;
            if (t->tr) {
                if (t->tr->neg && t->tr->n_neg < t->tr->neg_cap) t->tr->neg[t->tr->n_neg] = s;
                t->tr->n_neg++;
            }
        }
        for (int r = 0; r < rows; r++)
            memcpy(t->m_in + (int64_t) r * d, t->w_in + (int64_t) t->sen[lo + r] * d, sizeof(float) * d);
        for (int k = 0; k < K; k++)
            memcpy(t->m_out + (int64_t) k * d, t->w_out + (int64_t) t->neg[k] * d, sizeof(float) * d);
        /* MM1: grad[K x rows] = M_out . M_in^T */
        gemm_ordered(K, rows, d, t->m_out, d, 1, t->m_in, 1, d, t->m_grad, rows);
        for (int e = 0; e < K * rows; e++) t->m_grad[e] = grad_of(t->m_grad[e], 0, t->alpha, t->exp_table);
        /* MM2: M_out_update[K x d] = grad . M_in */
        gemm_ordered(K, d, rows, t->m_grad, rows, 1, t->m_in, d, 1, t->m_out_upd, d);
        /* MM3: M_in[rows x d] = grad^T . M_out (overwrites M_in, as the reference does) */
        gemm_ordered(rows, d, K, t->m_grad, 1, rows, t->m_out, d, 1, t->m_in, d);
        for (int r = 0; r < rows; r++) {
            float *dst = t->w_in + (int64_t) t->sen[lo + r] * d;
            const float *src = t->m_in + (int64_t) r * d;
            for (int j = 0; j < d; j++) dst[j] = dst[j] + src[j];
        }
        for (int k = 0; k < K; k++) {
            float *dst = t->w_out + (int64_t) t->neg[k] * d;
            const float *src = t->m_out_upd + (int64_t) k * d;
            for (int j = 0; j < d; j++) dst[j] = dst[j] + src[j];
        }
    }
}

int pwo_train(const pwo_config *cfg, const uint32_t *cn, const int32_t *table, const float *exp_table,
              const int32_t *stream, uint64_t n_tokens, float *w_in, float *w_out, pwo_trace *tr,
              int64_t max_resample) {
    if (!cfg || cfg->vocab_size < 2 || cfg->hidden_size < 1 || cfg->window < 1 || cfg->batch_size < 1 ||
        cfg->negative < 0 || cfg->iter < 1)
        return -1;
    if (stream[n_tokens] != 0) return -1;
    const int d = cfg->hidden_size, B = cfg->batch_size;
    const int kmax = 2 * cfg->window * cfg->negative;
    trainer t;
    memset(&t, 0, sizeof(t));
    t.cfg = cfg; t.cn = cn; t.table = table; t.exp_table = exp_table;
    t.w_in = w_in; t.w_out = w_out; t.tr = tr; t.rng = cfg->seed; t.alpha = cfg->alpha;
    t.max_resample = max_resample > 0 ? max_resample : ((int64_t) 1 << 40);
    t.m_in = (float *) malloc(sizeof(float) * (size_t) B * d);
    t.m_out = (float *) malloc(sizeof(float) * (size_t) (kmax > 0 ? kmax : 1) * d);
    t.m_out_upd = (float *) malloc(sizeof(float) * (size_t) (kmax > 0 ? kmax : 1) * d);
    t.m_grad = (float *) malloc(sizeof(float) * (size_t) (kmax > 0 ? kmax : 1) * B);
    t.neg = (int *) malloc(sizeof(int) * (size_t) (kmax > 0 ? kmax : 1));

    uint64_t train_words = 0;
    for (int i = 0; i < cfg->vocab_size; i++) train_words += cn[i];
    const float starting_alpha = cfg->alpha;
    const uint64_t local_train_words = n_tokens;  /* one thread loads the whole stream */
    uint64_t word_count = 0, last_word_count = 0, word_count_actual = 0, words_read = 0;
    int local_iter = cfg->iter;
    int pos = 0, rep_pos = 0;
    t.len = 0;

    /* PAR_Word2Vec_cpu.cpp:430-687: one attraction position per trip */
    for (;;) {
        if (word_count - last_word_count > 10000) {
            word_count_actual += word_count - last_word_count;
            last_word_count = word_count;
            t.alpha = starting_alpha * (1 - (float) word_count_actual /
                                                (float) ((uint64_t) cfg->iter * train_words + 1));
            if (t.alpha < starting_alpha * 0.0001f) t.alpha = starting_alpha * 0.0001f;
        }
        if (t.len == 0) {
            word_count = read_sentence(&t, stream, word_count, train_words);
            pos = 0;
            rep_pos = 0;
        }
        if (word_count > local_train_words) {
            word_count_actual += word_count - last_word_count;
            words_read += word_count;
            local_iter--;
            if (local_iter == 0) break;
            word_count = 0;
            last_word_count = 0;
            t.len = 0;
            continue;
        }
        attract(&t, pos);
        pos++;
        if (pos >= t.len) {
            rep_pos = 0;
            if (t.len > 0) {
                repel(&t);
                if (t.failed) break;
                rep_pos = t.len;
                if (tr) tr->n_sentences++;
            }
        }
        if (rep_pos >= t.len) {
            t.len = 0;
            continue;
        }
    }
    if (tr) {
        tr->words_read = words_read;
        tr->final_lcg = t.rng;
    }
    free(t.m_in); free(t.m_out); free(t.m_out_upd); free(t.m_grad); free(t.neg);
    return t.failed ? -2 : 0;
}
