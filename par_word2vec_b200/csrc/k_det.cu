// Deterministic single-stream mode: one CTA replays PAR_Word2Vec_cpu's training loop for thread
// 0 of 1 (PAR_Word2Vec_cpu.cpp:430-687) in the reference's order.  Scalar control flow (LCG,
// subsampling, sentence assembly, negative draws, learning-rate decay) runs on thread 0; the
// vector work is spread over the CTA without changing any floating-point order:
//   - a dot product's products are formed in parallel (each is one rounding) and summed
//     sequentially j = 0..d-1 by one thread, as the reference's scalar loop does;
//   - the attraction update is element-wise;
//   - each repulsion GEMM element sums its inner index in ascending order (the order the
//     oracle's cblas_sgemm fixes), and scatters of duplicate rows apply in the reference's order.
// The result is bit-identical to the reference built without FMA contraction.
#include <cstring>

#include "common.cuh"
#include "internal.h"

namespace parw2v {

namespace {

constexpr int kDetThreads = 256;

enum : int { kActAttract = 0, kActSkip = 1, kActDone = 2 };

struct DetShared {
    uint64_t rng;
    uint64_t word_count, last_word_count, word_count_actual, words_total;
    float alpha;
    int len, pos, local_iter, action, b;
    int rep_b, k, candidate, found;
    float g;
    int failed;
};

__device__ __forceinline__ void trace_put_u8(uint8_t *buf, int64_t cap, unsigned long long *n, uint8_t v) {
    unsigned long long i = *n;
    if (buf && (int64_t) i < cap) buf[i] = v;
    *n = i + 1;
}

// Sentence read with subsampling (PAR_Word2Vec_cpu.cpp:447-471), thread 0 only.
__device__ void det_read_sentence(const TrainArgs &a, const DevTrace &tr, DetShared &st, int *sen) {
    uint64_t wc = st.word_count;
    int len = 0;
    for (;;) {
        const int w = a.corpus[wc];
        wc++;
        if (w == 0) {
            trace_put_u8(tr.keep, tr.keep_cap, &a.cnt->n_keep, 2);
            break;
        }
        if (a.sample > 0) {
            st.rng = lcg_next(st.rng);
            const float u = __fdiv_rn((float) (st.rng & 0xFFFF), 65536.f);
            if (a.keep_thr[w] < u) {
                trace_put_u8(tr.keep, tr.keep_cap, &a.cnt->n_keep, 0);
                continue;
            }
        }
        trace_put_u8(tr.keep, tr.keep_cap, &a.cnt->n_keep, 1);
        sen[len++] = w;
        if (len >= kMaxSentence) break;
    }
    st.word_count = wc;
    st.len = len;
}

__global__ void __launch_bounds__(kDetThreads, 1) k_det_train(TrainArgs a, DevTrace tr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DetShared st;
    __shared__ int sen[kMaxSentence];
    __shared__ float s_g[256];   // window-synchronous variant: per-context gradients
    __shared__ int s_ctx[256];   // and context words
    const int tid = threadIdx.x;
    const int d = a.d, ld = a.ld, w = a.window, B = a.batch;
    const FastMod mod_w((uint32_t) w), mod_2w((uint32_t) (2 * w));  // r % w, r % 2w (:534, :591-600)
    const int kmax = 2 * w * a.negative;
    float *prod = reinterpret_cast<float *>(smem_raw);  // d
    float *grad = prod + ((d + 3) & ~3);                 // kmax * B
    int *neg = reinterpret_cast<int *>(grad + (size_t) kmax * B);  // kmax
    float *m_in = a.scratch;                             // B x ld
    float *m_out = a.scratch + (size_t) B * ld;          // kmax x ld
    float *w_in = static_cast<float *>(a.w_in);
    float *w_out = static_cast<float *>(a.w_out);
    const float starting_alpha = a.alpha0;
    const float denom = __ull2float_rn((uint64_t) a.iter * a.train_words + 1ULL);

    if (tid == 0) {
        st.rng = a.seed;
        st.word_count = st.last_word_count = st.word_count_actual = st.words_total = 0;
        st.alpha = a.alpha0;
        st.len = 0;
        st.pos = 0;
        st.local_iter = a.iter;
        st.failed = 0;
    }
    __syncthreads();

    for (;;) {
        if (tid == 0) {
            // learning-rate decay every >10k words (PAR_Word2Vec_cpu.cpp:431-446)
            if (st.word_count - st.last_word_count > 10000) {
                st.word_count_actual += st.word_count - st.last_word_count;
                st.last_word_count = st.word_count;
                float frac = __fdiv_rn(__ull2float_rn(st.word_count_actual), denom);
                st.alpha = __fmul_rn(starting_alpha, __fsub_rn(1.0f, frac));
                float floor_a = __fmul_rn(starting_alpha, 0.0001f);
                if (st.alpha < floor_a) st.alpha = floor_a;
            }
            if (st.len == 0) {
                det_read_sentence(a, tr, st, sen);
                st.pos = 0;
            }
            if (st.word_count > a.n_tokens) {  // end of the thread's stream (:472-527)
                st.word_count_actual += st.word_count - st.last_word_count;
                st.words_total += st.word_count;
                st.local_iter--;
                if (st.local_iter == 0) {
                    st.action = kActDone;
                } else {
                    st.word_count = 0;
                    st.last_word_count = 0;
                    st.len = 0;
                    st.action = kActSkip;
                }
            } else {
                st.rng = lcg_next(st.rng);
                st.b = (int) mod_w(st.rng);
                st.action = kActAttract;
                trace_put_u8(tr.b, tr.b_cap, &a.cnt->n_b, (uint8_t) st.b);
                unsigned long long i = a.cnt->n_alpha;
                if (tr.alpha && (int64_t) i < tr.alpha_cap) tr.alpha[i] = st.alpha;
                a.cnt->n_alpha = i + 1;
            }
        }
        __syncthreads();
        const int action = st.action;
        __syncthreads();  // everyone has read st before thread 0 may write it again
        if (action == kActDone) break;
        if (action == kActSkip) continue;

        // ---- attraction for sentence position pos (:529-568) ----
        const int len = st.len, pos = st.pos, b = st.b;
        const float alpha = st.alpha;
        const int target = sen[pos < len ? pos : 0];
        if (a.sync_window && len > 0) {
            // window-synchronous variant: all contexts scored against the same target row
            float *y = w_out + (size_t) target * ld;
            int n = 0;
            for (int i = b; i < 2 * w + 1 - b; i++) {
                if (i == w) continue;
                const int c = pos - w + i;
                if (c < 0) continue;
                if (c >= len) break;
                const float *x = w_in + (size_t) sen[c] * ld;
                for (int j = tid; j < d; j += kDetThreads) prod[j] = __fmul_rn(x[j], y[j]);
                __syncthreads();
                if (tid == 0) {
                    float f = 0.f;
                    for (int j = 0; j < d; j++) f = __fadd_rn(f, prod[j]);
                    s_g[n] = grad_from_table(f, 1, alpha, a.exp_table);
                    s_ctx[n] = sen[c];
                    a.cnt->pairs++;
                }
                n++;
                __syncthreads();
            }
            if (tid == 0)
                for (int i = 0; i < n; i++)
                    for (int k = 0; k < i; k++)
                        if (s_ctx[k] == s_ctx[i]) {
                            s_g[k] = __fadd_rn(s_g[k], s_g[i]);
                            s_g[i] = 0.f;
                            break;
                        }
            __syncthreads();
            for (int j = tid; j < d; j += kDetThreads) {
                const float yj = y[j];
                float dy = 0.f;
                for (int i = 0; i < n; i++) dy = __fadd_rn(dy, __fmul_rn(s_g[i], w_in[(size_t) s_ctx[i] * ld + j]));
                for (int i = 0; i < n; i++) {
                    if (s_g[i] == 0.f) continue;
                    float *xj = w_in + (size_t) s_ctx[i] * ld + j;
                    *xj = __fadd_rn(*xj, __fmul_rn(s_g[i], yj));
                }
                y[j] = __fadd_rn(yj, dy);
            }
            __syncthreads();
        } else
        for (int i = b; i < 2 * w + 1 - b; i++) {
            if (i == w) continue;
            const int c = pos - w + i;
            if (c < 0) continue;
            if (c >= len) break;
            float *x = w_in + (size_t) sen[c] * ld;
            float *y = w_out + (size_t) target * ld;
            for (int j = tid; j < d; j += kDetThreads) prod[j] = __fmul_rn(x[j], y[j]);
            __syncthreads();
            if (tid == 0) {
                float f = 0.f;
                for (int j = 0; j < d; j++) f = __fadd_rn(f, prod[j]);
                st.g = grad_from_table(f, 1, alpha, a.exp_table);
            }
            __syncthreads();
            const float g = st.g;
            for (int j = tid; j < d; j += kDetThreads) {
                const float xj = x[j], yj = y[j];
                const float keep_y = __fmul_rn(g, yj);
                y[j] = __fadd_rn(yj, __fmul_rn(g, xj));
                x[j] = __fadd_rn(xj, keep_y);
            }
            if (tid == 0) a.cnt->pairs++;
            __syncthreads();
        }

        // ---- repulsion once the sentence's last position is done (:571-679) ----
        if (pos + 1 >= len && len > 0) {
            const int num_batch = (len + B - 1) / B;
            for (int nb = 0; nb < num_batch; nb++) {
                const int lo = nb * B;
                const int hi = (lo + (B - 1) < len - 1) ? lo + (B - 1) : len - 1;
                const int rows = hi - lo + 1;
                if (tid == 0) {
                    st.rng = lcg_next(st.rng);
                    if (lo <= w - 1 || (len - 1) - lo <= w - 1) st.rep_b = (int) mod_w(st.rng);
                    else st.rep_b = (int) mod_2w(st.rng);
                    st.k = st.rep_b * a.negative;
                    trace_put_u8(tr.rep_b, tr.rep_b_cap, &a.cnt->n_rep_b, (uint8_t) st.rep_b);
                    a.cnt->batches++;
                }
                __syncthreads();
                const int K = st.k;
                // shared negatives: unigram draw, then uniform redraws while the word is in the sentence
                for (int k = 0; k < K; k++) {
                    if (tid == 0) {
                        st.rng = lcg_next(st.rng);
                        int s = a.table[(st.rng >> 16) % (uint64_t) kTableSize];
                        if (!s) s = (int) (st.rng % (uint64_t) (a.vocab - 1) + 1);
                        st.candidate = s;
                    }
                    __syncthreads();
                    for (int64_t tries = 0;; tries++) {
                        const int cand = st.candidate;
                        int hit = 0;
                        for (int q = tid; q < len; q += kDetThreads) hit |= (sen[q] == cand);
                        const int found = __syncthreads_or(hit);
                        if (!found) break;
                        if (tries >= a.max_resample) {
                            if (tid == 0) st.failed = 1;
                            break;
                        }
                        if (tid == 0) {
                            st.rng = lcg_next(st.rng);
                            st.candidate = (int) (st.rng % (uint64_t) (a.vocab - 1) + 1);
                        }
                        __syncthreads();
                    }
                    __syncthreads();
                    if (st.failed) break;
                    if (tid == 0) {
                        neg[k] = st.candidate;
                        unsigned long long i = a.cnt->n_neg;
                        if (tr.neg && (int64_t) i < tr.neg_cap) tr.neg[i] = st.candidate;
                        a.cnt->n_neg = i + 1;
                        a.cnt->negatives++;
                    }
                    __syncthreads();
                }
                if (st.failed) break;
                // gather M_in (rows x d) and M_out (K x d) (:624-631)
                for (int e = tid; e < rows * d; e += kDetThreads) {
                    const int r = e / d, j = e - r * d;
                    m_in[(size_t) r * ld + j] = w_in[(size_t) sen[lo + r] * ld + j];
                }
                for (int e = tid; e < K * d; e += kDetThreads) {
                    const int k = e / d, j = e - k * d;
                    m_out[(size_t) k * ld + j] = w_out[(size_t) neg[k] * ld + j];
                }
                __syncthreads();
                // MM1 + sigma/label 0 (:633-650): grad[k][r] = g(M_out[k] . M_in[r])
                for (int e = tid; e < K * rows; e += kDetThreads) {
                    const int k = e / rows, r = e - k * rows;
                    const float *p = m_out + (size_t) k * ld;
                    const float *q = m_in + (size_t) r * ld;
                    float acc = 0.0f;
                    for (int j = 0; j < d; j++) acc = __fadd_rn(acc, __fmul_rn(p[j], q[j]));
                    grad[e] = grad_from_table(acc, 0, alpha, a.exp_table);
                }
                __syncthreads();
                // MM2 + W_out scatter (:652-653, :667-674), MM3 + W_in scatter (:655-665)
                for (int j = tid; j < d; j += kDetThreads) {
                    for (int k = 0; k < K; k++) {
                        float acc = 0.0f;
                        for (int r = 0; r < rows; r++)
                            acc = __fadd_rn(acc, __fmul_rn(grad[k * rows + r], m_in[(size_t) r * ld + j]));
                        float *dst = w_out + (size_t) neg[k] * ld + j;
                        *dst = __fadd_rn(*dst, acc);
                    }
                    for (int r = 0; r < rows; r++) {
                        float acc = 0.0f;
                        for (int k = 0; k < K; k++)
                            acc = __fadd_rn(acc, __fmul_rn(grad[k * rows + r], m_out[(size_t) k * ld + j]));
                        float *dst = w_in + (size_t) sen[lo + r] * ld + j;
                        *dst = __fadd_rn(*dst, acc);
                    }
                }
                __syncthreads();
            }
            if (tid == 0) {
                a.cnt->sentences++;
                a.cnt->kept += (unsigned long long) len;
            }
        }
        __syncthreads();
        if (st.failed) break;
        if (tid == 0) {
            st.pos = pos + 1;
            if (st.pos >= len) st.len = 0;  // rep_sentence_position >= sentence_length (:682-685)
        }
        __syncthreads();
    }
    if (tid == 0) {
        a.cnt->words = st.words_total;
        a.cnt->final_lcg = st.rng;
        a.cnt->final_alpha = st.alpha;
        if (st.failed) atomicOr(&a.cnt->error, kErrResample);
    }
}

}  // namespace

cudaError_t launch_det_train(const TrainArgs &a, const DevTrace &tr, cudaStream_t s, size_t *smem_needed) {
    const int kmax = 2 * a.window * a.negative;
    size_t smem = sizeof(float) * (size_t) ((a.d + 3) & ~3) + sizeof(float) * (size_t) kmax * a.batch +
                  sizeof(int) * (size_t) kmax;
    if (smem_needed) *smem_needed = smem;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_det_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    k_det_train<<<1, kDetThreads, smem, s>>>(a, tr);
    return cudaGetLastError();
}

}  // namespace parw2v

// ---- Allocation-free entry point (parw2v_det_train_noalloc) ----
// Some callers cannot let a library call cudaMalloc: a framework whose caching allocator owns all
// device memory, or a service that sizes its device memory once at start-up and must not fail
// later on an allocation.  This entry point runs the deterministic training kernel on buffers the
// caller owns; its only scratch (the repulsion staging rows and the counters) lives in the array
// below, which every GPU that loads this library keeps for the life of the process.
namespace {

constexpr size_t kNoAllocScratchBytes = 1u << 20;  // 1 MiB: counters + (batch + 2*window*negative) x ld floats
constexpr size_t kNoAllocCounterBytes = 256;       // DevCounters, rounded up
static_assert(sizeof(parw2v::DevCounters) <= kNoAllocCounterBytes, "counters must fit their slot");
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

}  // namespace

extern "C" int parw2v_det_train_noalloc(const parw2v_config *cfg, int vocab_size, uint64_t train_words,
                                        const int32_t *d_corpus, uint64_t n_tokens, const int32_t *d_table,
                                        const float *d_exp_table, const float *d_keep_thr, float *d_w_in,
                                        float *d_w_out, int ld, void *stream, parw2v_stats *stats) {
    using namespace parw2v;
    if (!cfg || !d_corpus || !d_table || !d_exp_table || !d_keep_thr || !d_w_in || !d_w_out)
        return set_global_error(PARW2V_ERR_ARG, "null argument");
    const parw2v_config &k = *cfg;
    if (vocab_size < 2 || k.size < 1 || ld < k.size || k.window < 1 || k.window > 100 || k.negative < 0 ||
        k.negative > 100 || k.batch_size < 1 || k.batch_size > 1000 || k.iter < 1 || !(k.alpha > 0) || k.sample < 0 ||
        k.device < 0 || k.device >= kNoAllocMaxDevices)
        return set_global_error(PARW2V_ERR_ARG, "invalid configuration value");
    const size_t rows = (size_t) k.batch_size + 2 * (size_t) k.window * k.negative;
    if (kNoAllocCounterBytes + rows * (size_t) ld * sizeof(float) > kNoAllocScratchBytes)
        return set_global_error(PARW2V_ERR_CAPACITY,
                                "(batch_size + 2*window*negative) * ld * 4 bytes exceeds the 1 MiB static scratch");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return set_global_error(PARW2V_ERR_NODEV, "no CUDA device");
    if (prev != k.device && cudaSetDevice(k.device) != cudaSuccess)
        return set_global_error(PARW2V_ERR_ARG, "device ordinal out of range");
    int rc = PARW2V_OK;
    // The device address of the array in the current device's context, looked up on every call
    // (cheap once the module is loaded): an address kept from an earlier call would be stale
    // after cudaDeviceReset or under another context.  The host-side name g_noalloc_scratch is
    // not a device address and is never passed to a kernel.
    void *scratch = nullptr;
    {
        const cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            rc = set_global_error(PARW2V_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevCounters h{};
    if (rc == PARW2V_OK) {
        DevCounters *cnt = static_cast<DevCounters *>(scratch);
        TrainArgs a{};
        a.corpus = d_corpus;
        a.n_tokens = n_tokens;
        a.keep_thr = d_keep_thr;
        a.table = d_table;
        a.exp_table = d_exp_table;
        a.w_in = d_w_in;
        a.w_out = d_w_out;
        a.ld = ld;
        a.d = k.size;
        a.window = k.window;
        a.negative = k.negative;
        a.batch = k.batch_size;
        a.iter = k.iter;
        a.vocab = vocab_size;
        a.alpha0 = k.alpha;
        a.sample = k.sample;
        a.train_words = train_words;
        a.seed = k.seed;
        a.cnt = cnt;
        a.scratch = reinterpret_cast<float *>(static_cast<unsigned char *>(scratch) + kNoAllocCounterBytes);
        a.max_resample = 1LL << 20;
        a.sync_window = k.attraction == PARW2V_ATTRACT_WINDOW;
        // the counters start at zero on every call; the staging rows are written before read
        cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(DevCounters), s);
        size_t smem = 0;
        if (e == cudaSuccess) e = launch_det_train(a, DevTrace{}, s, &smem);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = set_global_error(smem > 200 * 1024 ? PARW2V_ERR_CAPACITY : PARW2V_ERR_CUDA, cudaGetErrorString(e));
        else if (h.error & kErrResample)
            rc = set_global_error(PARW2V_ERR_TIMEOUT, "negative resampling exceeded its draw limit");
    }
    if (rc == PARW2V_OK && stats) {
        memset(stats, 0, sizeof(*stats));
        stats->words = h.words;
        stats->kept = h.kept;
        stats->sentences = h.sentences;
        stats->pairs = h.pairs;
        stats->batches = h.batches;
        stats->negatives = h.negatives;
        stats->final_alpha = h.final_alpha;
    }
    if (prev != k.device) cudaSetDevice(prev);
    return rc;
}
