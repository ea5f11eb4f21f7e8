// C ABI of libparw2v: context management, set-up and the training dispatch (include/parw2v.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "internal.h"

using namespace parw2v;

struct parw2v_ctx {
    parw2v_config cfg{};
    int ld = 0;
    bool bf16 = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    std::string err;
    size_t allocated = 0;
    std::vector<void *> owned;
    // vocabulary and tables
    int vocab = 0;
    uint64_t train_words = 0;
    uint32_t *d_counts = nullptr;
    int32_t *d_table = nullptr;
    float *d_exp = nullptr;
    float *d_thr = nullptr;
    // weights
    void *d_w_in = nullptr, *d_w_out = nullptr;
    bool weights_ready = false;
    // corpus and packing
    int32_t *d_corpus = nullptr;
    uint64_t n_tokens = 0, corpus_cap = 0, n_lines = 0;
    int32_t *d_packed = nullptr;
    uint32_t *d_line_end = nullptr;
    uint64_t line_cap = 0;
    uint32_t *d_tile_kept = nullptr, *d_tile_zero = nullptr;
    uint64_t tile_cap = 0;
    // workspace
    float *d_scratch = nullptr;
    size_t scratch_floats = 0;
    float *d_stage = nullptr;  // dense FP32 rows for weight copies (see copy_weights)
    size_t stage_bytes = 0;
    DevCounters *d_cnt = nullptr;
    // trace
    parw2v_trace *trace = nullptr;
    DevTrace dtr;
    size_t trace_bytes = 0;
    void *d_trace_mem = nullptr;
    int last_grid = 0, last_warps = 0;  // launch shape of the last Hogwild training call
    bool corpus_checked = false;        // the corpus's ids were validated against this vocabulary
    // the two epoch graphs (packing; training + epoch advance) of the last Hogwild call, kept for
    // the next call with the same launch arguments
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    TrainArgs graph_args{};
    int graph_grid = 0, graph_warps = 0;
    // launch knobs chosen by the autotuner (cfg.autotune) for `inflight` sentences in flight
    struct {
        bool done = false;
        uint64_t inflight = 0;
        int grid = 0, warps = 0, stage_bulk = 0, lane_elems = 0, attr_pipe = 0;
        bool stream = true;
    } tuned;
};

static void drop_graphs(parw2v_ctx *c) {
    for (auto &g : c->graphs)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// Text of the last error not tied to a context (a failed create, the allocation-free entry point,
// the random walks), per calling thread: calls on different threads never share it.
static thread_local std::string g_create_error;

namespace parw2v {
int set_global_error(int code, const char *msg) {
    g_create_error = msg;
    return code;
}
}  // namespace parw2v

static int fail(parw2v_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

static int cuda_fail(parw2v_ctx *c, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return fail(c, PARW2V_ERR_OOM, m);
    return fail(c, PARW2V_ERR_CUDA, m);
}

#define CK(c, call, what)                               \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

// Device allocation against the context's memory cap.
static int dalloc(parw2v_ctx *c, void **p, size_t bytes, const char *what) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (c->cfg.mem_cap_bytes && c->allocated + bytes > c->cfg.mem_cap_bytes)
        return fail(c, PARW2V_ERR_OOM, std::string(what) + ": exceeds mem_cap_bytes");
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return cuda_fail(c, e, what);
    }
    c->allocated += bytes;
    c->owned.push_back(*p);
    return PARW2V_OK;
}

static void dfree(parw2v_ctx *c, void *p, size_t bytes) {
    if (!p) return;
    for (size_t i = 0; i < c->owned.size(); i++)
        if (c->owned[i] == p) {
            c->owned.erase(c->owned.begin() + (long) i);
            break;
        }
    cudaFree(p);
    c->allocated -= bytes < c->allocated ? bytes : c->allocated;
}

static int set_device(parw2v_ctx *c) {
    CK(c, cudaSetDevice(c->cfg.device), "cudaSetDevice");
    return PARW2V_OK;
}

static size_t welem(const parw2v_ctx *c) { return c->bf16 ? sizeof(__nv_bfloat16) : sizeof(float); }

extern "C" {

const char *parw2v_version(void) { return "parw2v-b200 0.1 (sm_100a)"; }

const char *parw2v_strerror(int s) {
    switch (s) {
        case PARW2V_OK: return "ok";
        case PARW2V_ERR_ARG: return "invalid argument";
        case PARW2V_ERR_CUDA: return "CUDA error";
        case PARW2V_ERR_OOM: return "out of device memory";
        case PARW2V_ERR_CAPACITY: return "input exceeds a library limit";
        case PARW2V_ERR_TIMEOUT: return "bounded device loop gave up";
        case PARW2V_ERR_STATE: return "call order violated";
        case PARW2V_ERR_IO: return "file I/O error";
        case PARW2V_ERR_NODEV: return "no CUDA device";
        default: return "unknown status";
    }
}

const char *parw2v_last_error(const parw2v_ctx *c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int parw2v_create(const parw2v_config *cfg, parw2v_ctx **out) {
    if (!cfg || !out) return fail(nullptr, PARW2V_ERR_ARG, "null argument");
    *out = nullptr;
    const parw2v_config &k = *cfg;
    if (k.size < 1 || k.window < 1 || k.negative < 0 || k.batch_size < 1 || k.iter < 1 || !(k.alpha > 0) ||
        k.sample < 0 || k.mode < PARW2V_MODE_DET || k.mode > PARW2V_MODE_BATCHED_BF16 || k.grid < 0 ||
        k.warps_per_cta < 0)
        return fail(nullptr, PARW2V_ERR_ARG, "invalid configuration value");
    if (k.variant < PARW2V_VARIANT_AUTO || k.variant > PARW2V_VARIANT_STREAM)
        return fail(nullptr, PARW2V_ERR_ARG, "invalid kernel variant");
    if (k.attraction < PARW2V_ATTRACT_DEFAULT || k.attraction > PARW2V_ATTRACT_PIPELINED)
        return fail(nullptr, PARW2V_ERR_ARG, "invalid attraction variant");
    if (k.staging < PARW2V_STAGING_AUTO || k.staging > PARW2V_STAGING_CPASYNC)
        return fail(nullptr, PARW2V_ERR_ARG, "invalid staging method");
    if (k.window > 100 || k.negative > 100 || k.batch_size > 1000)
        return fail(nullptr, PARW2V_ERR_CAPACITY, "window/negative/batch_size beyond the supported range");
    if (k.mode != PARW2V_MODE_DET && k.size > 512)
        return fail(nullptr, PARW2V_ERR_CAPACITY, "Hogwild modes support size <= 512");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, PARW2V_ERR_NODEV, "no CUDA device available");
    }
    if (k.device < 0 || k.device >= ndev) return fail(nullptr, PARW2V_ERR_ARG, "device ordinal out of range");
    parw2v_ctx *c = new parw2v_ctx();
    c->cfg = k;
    c->bf16 = (k.mode == PARW2V_MODE_BATCHED_BF16);
    // rows of whole 32-byte sectors: every column chunk of the repulsion is a whole number of
    // tensor-core k-steps, and a row starts on a sector
    const int align = c->bf16 ? 16 : 8;
    c->ld = (k.size + align - 1) / align * align;
    int rc = set_device(c);
    if (rc == PARW2V_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev2);
        if (e != cudaSuccess) rc = cuda_fail(c, e, "stream/event creation");
    }
    if (rc == PARW2V_OK) rc = dalloc(c, (void **) &c->d_cnt, sizeof(DevCounters), "counters");
    if (rc == PARW2V_OK) rc = dalloc(c, (void **) &c->d_exp, sizeof(float) * (kExpTableSize + 1), "expTable");
    if (rc != PARW2V_OK) {
        g_create_error = c->err;
        parw2v_destroy(c);
        return rc;
    }
    // expTable on the host with the reference's float expression (PAR_Word2Vec_cpu.cpp:822-826;
    // exp of a float argument is expf in the reference's C++)
    float h_exp[kExpTableSize + 1];
    for (int i = 0; i < kExpTableSize + 1; i++) {
        float x = ((float) i / (float) kExpTableSize * 2.0f - 1.0f) * (float) kMaxExp;
        float e = expf(x);
        h_exp[i] = e / (e + 1.0f);
    }
    cudaError_t e = cudaMemcpyAsync(c->d_exp, h_exp, sizeof(h_exp), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        rc = cuda_fail(c, e, "expTable upload");
        g_create_error = c->err;
        parw2v_destroy(c);
        return rc;
    }
    *out = c;
    return PARW2V_OK;
}

void parw2v_destroy(parw2v_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->cfg.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    for (void *p : c->owned) cudaFree(p);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev2) cudaEventDestroy(c->ev2);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int parw2v_set_vocab(parw2v_ctx *c, const uint32_t *counts, int V) {
    if (!c || !counts) return fail(c, PARW2V_ERR_ARG, "null argument");
    if (V < 2) return fail(c, PARW2V_ERR_ARG, "vocab_size must be >= 2 (\"</s>\" plus one word)");
    int rc = set_device(c);
    if (rc) return rc;
    if (c->vocab != V) {
        dfree(c, c->d_counts, sizeof(uint32_t) * (size_t) c->vocab);
        dfree(c, c->d_thr, sizeof(float) * (size_t) c->vocab);
        c->d_counts = nullptr;
        c->d_thr = nullptr;
        if (c->d_w_in) {
            dfree(c, c->d_w_in, welem(c) * (size_t) c->vocab * c->ld);
            dfree(c, c->d_w_out, welem(c) * (size_t) c->vocab * c->ld);
            c->d_w_in = c->d_w_out = nullptr;
        }
        c->weights_ready = false;
        if ((rc = dalloc(c, (void **) &c->d_counts, sizeof(uint32_t) * (size_t) V, "counts"))) return rc;
        if ((rc = dalloc(c, (void **) &c->d_thr, sizeof(float) * (size_t) V, "thresholds"))) return rc;
        c->vocab = V;
    }
    if (!c->d_table && (rc = dalloc(c, (void **) &c->d_table, sizeof(int32_t) * (size_t) kTableSize, "table")))
        return rc;
    uint64_t tw = 0;
    for (int i = 0; i < V; i++) tw += counts[i];
    c->train_words = tw;
    c->corpus_checked = false;
    // cn^0.75 as the reference computes it: pow(unsigned, float) promotes both to double
    std::vector<double> pw((size_t) V);
    for (int i = 0; i < V; i++) pw[(size_t) i] = pow((double) counts[i], (double) 0.75f);
    void *tmp = nullptr;
    const size_t tmp_bytes = sizeof(double) * (size_t) V + sizeof(float) * (size_t) V + sizeof(long long) * (size_t) V +
                             sizeof(double) + 16;  // + alignment slack for the int64 array
    if ((rc = dalloc(c, &tmp, tmp_bytes, "table workspace"))) return rc;
    double *d_pow = (double *) tmp;
    float *d_D = (float *) (d_pow + V);
    long long *d_g = (long long *) (((uintptr_t) (d_D + V) + 7) & ~(uintptr_t) 7);
    double *d_total = (double *) (d_g + V);
    cudaError_t e = cudaMemcpyAsync(d_pow, pw.data(), sizeof(double) * (size_t) V, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_counts, counts, sizeof(uint32_t) * (size_t) V, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_build_table(d_pow, V, c->d_table, d_D, d_g, d_total, c->stream);
    if (e == cudaSuccess) e = launch_build_thresholds(c->d_counts, V, c->cfg.sample, tw, c->d_thr, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, tmp, tmp_bytes);
    if (e != cudaSuccess) return cuda_fail(c, e, "unigram table / thresholds");
    return PARW2V_OK;
}

int parw2v_get_table(parw2v_ctx *c, int32_t *table) {
    if (!c || !table) return fail(c, PARW2V_ERR_ARG, "null argument");
    if (!c->vocab) return fail(c, PARW2V_ERR_STATE, "set_vocab first");
    int rc = set_device(c);
    if (rc) return rc;
    CK(c, cudaMemcpyAsync(table, c->d_table, sizeof(int32_t) * (size_t) kTableSize, cudaMemcpyDeviceToHost, c->stream),
       "table download");
    CK(c, cudaStreamSynchronize(c->stream), "table download");
    return PARW2V_OK;
}

int parw2v_get_exp_table(parw2v_ctx *c, float *t) {
    if (!c || !t) return fail(c, PARW2V_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (rc) return rc;
    CK(c, cudaMemcpyAsync(t, c->d_exp, sizeof(float) * (kExpTableSize + 1), cudaMemcpyDeviceToHost, c->stream),
       "expTable download");
    CK(c, cudaStreamSynchronize(c->stream), "expTable download");
    return PARW2V_OK;
}

static int ensure_weights(parw2v_ctx *c) {
    if (!c->vocab) return fail(c, PARW2V_ERR_STATE, "set_vocab first");
    if (c->d_w_in) return PARW2V_OK;
    const size_t bytes = welem(c) * (size_t) c->vocab * c->ld;
    int rc = dalloc(c, &c->d_w_in, bytes, "W_in");
    if (!rc) rc = dalloc(c, &c->d_w_out, bytes, "W_out");
    return rc;
}

int parw2v_init_weights(parw2v_ctx *c) {
    if (!c) return fail(c, PARW2V_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (!rc) rc = ensure_weights(c);
    if (rc) return rc;
    cudaError_t e;
    if (c->bf16)
        e = launch_init_net(nullptr, nullptr, (__nv_bfloat16 *) c->d_w_in, (__nv_bfloat16 *) c->d_w_out, c->vocab,
                            c->cfg.size, c->ld, c->stream);
    else
        e = launch_init_net((float *) c->d_w_in, (float *) c->d_w_out, nullptr, nullptr, c->vocab, c->cfg.size, c->ld,
                            c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "InitNet");
    c->weights_ready = true;
    return PARW2V_OK;
}

// Host [V][d] FP32 <-> device [V][ld] rows (FP32 or BF16).  The rows go through a staging buffer of
// dense FP32 rows, at most kStageBytes, kept for later calls: one kernel converts a chunk of rows
// between the two layouts and one linear copy moves the chunk across the host link.  (A pitched
// copy of V rows of d floats runs at a fraction of the link's speed.)
static constexpr size_t kStageBytes = 64ull << 20;

static int copy_rows(parw2v_ctx *c, const float *src_h, float *dst_h, void *dev, bool bf16) {
    const size_t V = (size_t) c->vocab, d = (size_t) c->cfg.size, ld = (size_t) c->ld;
    const size_t row_bytes = sizeof(float) * d;
    const size_t chunk = std::max<size_t>(1, std::min(V, kStageBytes / row_bytes));
    if (c->stage_bytes < chunk * row_bytes) {
        dfree(c, c->d_stage, c->stage_bytes);
        c->d_stage = nullptr;
        c->stage_bytes = 0;
        int rc = dalloc(c, (void **) &c->d_stage, chunk * row_bytes, "weights staging");
        if (rc) return rc;
        c->stage_bytes = chunk * row_bytes;
    }
    const size_t esz = bf16 ? sizeof(__nv_bfloat16) : sizeof(float);
    for (size_t r0 = 0; r0 < V; r0 += chunk) {
        const size_t rows = std::min(chunk, V - r0);
        void *drow = (char *) dev + r0 * ld * esz;
        if (src_h) {
            CK(c, cudaMemcpyAsync(c->d_stage, src_h + r0 * d, rows * row_bytes, cudaMemcpyHostToDevice, c->stream),
               "weights upload");
            CK(c, launch_rows_from_dense(c->d_stage, (int) d, drow, bf16, (int) ld, rows, c->stream),
               "weights layout");
        } else {
            CK(c, launch_rows_to_dense(drow, bf16, (int) ld, c->d_stage, (int) d, rows, c->stream),
               "weights layout");
            CK(c, cudaMemcpyAsync(dst_h + r0 * d, c->d_stage, rows * row_bytes, cudaMemcpyDeviceToHost, c->stream),
               "weights download");
        }
    }
    CK(c, cudaStreamSynchronize(c->stream), "weights copy");
    return PARW2V_OK;
}

static int copy_weights(parw2v_ctx *c, const float *src_h, float *dst_h, void *dev) {
    return copy_rows(c, src_h, dst_h, dev, c->bf16);
}

int parw2v_set_weights(parw2v_ctx *c, const float *w_in, const float *w_out) {
    if (!c) return fail(c, PARW2V_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (!rc) rc = ensure_weights(c);
    if (rc) return rc;
    if (!c->weights_ready && (!w_in || !w_out))
        return fail(c, PARW2V_ERR_STATE, "first set_weights needs both matrices (or call init_weights)");
    if (w_in && (rc = copy_weights(c, w_in, nullptr, c->d_w_in))) return rc;
    if (w_out && (rc = copy_weights(c, w_out, nullptr, c->d_w_out))) return rc;
    c->weights_ready = true;
    return PARW2V_OK;
}

int parw2v_get_weights(parw2v_ctx *c, float *w_in, float *w_out) {
    if (!c) return fail(c, PARW2V_ERR_ARG, "null argument");
    if (!c->weights_ready) return fail(c, PARW2V_ERR_STATE, "no weights on the device");
    int rc = set_device(c);
    if (rc) return rc;
    if (w_in && (rc = copy_weights(c, nullptr, w_in, c->d_w_in))) return rc;
    if (w_out && (rc = copy_weights(c, nullptr, w_out, c->d_w_out))) return rc;
    return PARW2V_OK;
}

int parw2v_set_corpus(parw2v_ctx *c, const int32_t *tokens, uint64_t n) {
    if (!c || (!tokens && n)) return fail(c, PARW2V_ERR_ARG, "null argument");
    if (n >= 0xFFFFFFF0ULL) return fail(c, PARW2V_ERR_CAPACITY, "corpus must hold fewer than 2^32 - 16 tokens");
    int rc = set_device(c);
    if (rc) return rc;
    if (n + 16 > c->corpus_cap) {
        dfree(c, c->d_corpus, sizeof(int32_t) * c->corpus_cap);
        c->d_corpus = nullptr;
        c->corpus_cap = 0;
        const uint64_t cap = n + 16;
        if ((rc = dalloc(c, (void **) &c->d_corpus, sizeof(int32_t) * cap, "corpus"))) return rc;
        c->corpus_cap = cap;
    }
    if (n) CK(c, cudaMemcpyAsync(c->d_corpus, tokens, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream), "corpus upload");
    CK(c, cudaMemsetAsync(c->d_corpus + n, 0, sizeof(int32_t) * 16, c->stream), "sentinel");
    c->n_tokens = n;
    c->corpus_checked = false;
    return PARW2V_OK;
}

int parw2v_set_trace(parw2v_ctx *c, parw2v_trace *t) {
    if (!c) return fail(c, PARW2V_ERR_ARG, "null argument");
    if (t && c->cfg.mode != PARW2V_MODE_DET) return fail(c, PARW2V_ERR_STATE, "traces exist in DET mode only");
    c->trace = t;
    return PARW2V_OK;
}

// Validation of token ids against the vocabulary (one pass, on the device).
// Validation of token ids against the vocabulary and count of "</s>"-terminated lines (one pass).
__global__ void k_validate(const int32_t *corpus, uint64_t n, int V, DevCounters *cnt) {
    bool bad = false;
    unsigned long long lines = 0;
    for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x) {
        const int w = corpus[i];
        bad |= (w < 0 || w >= V);
        lines += (w == 0);
    }
    for (int o = 16; o > 0; o >>= 1) lines += __shfl_xor_sync(0xffffffffu, lines, o);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&cnt->error, kErrCapacity);
    if ((threadIdx.x & 31) == 0 && lines) atomicAdd(&cnt->n_lines, lines);
}

static int read_counters(parw2v_ctx *c, DevCounters *h) {
    CK(c, cudaMemcpyAsync(h, c->d_cnt, sizeof(DevCounters), cudaMemcpyDeviceToHost, c->stream), "counters");
    CK(c, cudaStreamSynchronize(c->stream), "counters");
    return PARW2V_OK;
}

static int device_sms(parw2v_ctx *c) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->cfg.device);
    return sms;
}

static int train_det(parw2v_ctx *c, TrainArgs &a, parw2v_stats *st) {
    const size_t need = (size_t) (c->cfg.batch_size + 2 * c->cfg.window * c->cfg.negative) * c->ld;
    int rc;
    if (c->scratch_floats < need) {
        dfree(c, c->d_scratch, sizeof(float) * c->scratch_floats);
        c->d_scratch = nullptr;
        c->scratch_floats = 0;
        if ((rc = dalloc(c, (void **) &c->d_scratch, sizeof(float) * need, "DET workspace"))) return rc;
        c->scratch_floats = need;
    }
    a.scratch = c->d_scratch;
    // trace buffers on the device
    DevTrace dt;
    parw2v_trace *t = c->trace;
    void *tm = nullptr;
    size_t tb = 0;
    if (t) {
        tb = (size_t) (t->keep ? t->keep_cap : 0) + (size_t) (t->b ? t->b_cap : 0) + (size_t) (t->rep_b ? t->rep_b_cap : 0) +
             16 * 4 + sizeof(float) * (size_t) (t->alpha ? t->alpha_cap : 0) +
             sizeof(int32_t) * (size_t) (t->neg ? t->neg_cap : 0);
        if ((rc = dalloc(c, &tm, tb, "trace buffers"))) return rc;
        unsigned char *p = (unsigned char *) tm;
        auto take = [&](size_t bytes) {
            unsigned char *q = p;
            p += (bytes + 15) & ~(size_t) 15;
            return q;
        };
        if (t->alpha) { dt.alpha = (float *) take(sizeof(float) * t->alpha_cap); dt.alpha_cap = t->alpha_cap; }
        if (t->neg) { dt.neg = (int32_t *) take(sizeof(int32_t) * t->neg_cap); dt.neg_cap = t->neg_cap; }
        if (t->keep) { dt.keep = (uint8_t *) take(t->keep_cap); dt.keep_cap = t->keep_cap; }
        if (t->b) { dt.b = (uint8_t *) take(t->b_cap); dt.b_cap = t->b_cap; }
        if (t->rep_b) { dt.rep_b = (uint8_t *) take(t->rep_b_cap); dt.rep_b_cap = t->rep_b_cap; }
    }
    cudaError_t e = cudaEventRecord(c->ev0, c->stream);
    size_t smem = 0;
    if (e == cudaSuccess) e = launch_det_train(a, dt, c->stream, &smem);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        dfree(c, tm, tb);
        if (smem > 200 * 1024) return fail(c, PARW2V_ERR_CAPACITY, "DET mode: window*negative*batch too large");
        return cuda_fail(c, e, "DET training kernel");
    }
    DevCounters h;
    if ((rc = read_counters(c, &h))) {
        dfree(c, tm, tb);
        return rc;
    }
    if (t) {
        auto back = [&](void *dst, const void *src, int64_t n, size_t el) -> cudaError_t {
            if (!dst || !src || n <= 0) return cudaSuccess;
            return cudaMemcpy(dst, src, (size_t) n * el, cudaMemcpyDeviceToHost);
        };
        t->n_keep = (int64_t) h.n_keep;
        t->n_b = (int64_t) h.n_b;
        t->n_alpha = (int64_t) h.n_alpha;
        t->n_rep_b = (int64_t) h.n_rep_b;
        t->n_neg = (int64_t) h.n_neg;
        t->final_lcg = h.final_lcg;
        e = back(t->keep, dt.keep, std::min<int64_t>(t->n_keep, t->keep_cap), 1);
        if (e == cudaSuccess) e = back(t->b, dt.b, std::min<int64_t>(t->n_b, t->b_cap), 1);
        if (e == cudaSuccess) e = back(t->alpha, dt.alpha, std::min<int64_t>(t->n_alpha, t->alpha_cap), sizeof(float));
        if (e == cudaSuccess) e = back(t->rep_b, dt.rep_b, std::min<int64_t>(t->n_rep_b, t->rep_b_cap), 1);
        if (e == cudaSuccess) e = back(t->neg, dt.neg, std::min<int64_t>(t->n_neg, t->neg_cap), sizeof(int32_t));
        dfree(c, tm, tb);
        if (e != cudaSuccess) return cuda_fail(c, e, "trace download");
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (st) {
        st->words = h.words;
        st->kept = h.kept;
        st->sentences = h.sentences;
        st->pairs = h.pairs;
        st->batches = h.batches;
        st->negatives = h.negatives;
        st->kernel_ms = ms;
        st->pack_ms = 0;
        st->final_alpha = h.final_alpha;
    }
    if (h.error & kErrResample)
        return fail(c, PARW2V_ERR_TIMEOUT, "negative resampling exceeded its draw limit (every word is in the sentence?)");
    return PARW2V_OK;
}

static int ensure_packing(parw2v_ctx *c) {
    int rc;
    const uint64_t tiles = pack_tiles(c->n_tokens) + 1;
    if (c->corpus_cap > 0 && (!c->d_packed || c->line_cap < c->n_tokens + 1)) {
        dfree(c, c->d_packed, sizeof(int32_t) * c->line_cap);
        dfree(c, c->d_line_end, sizeof(uint32_t) * c->line_cap);
        c->d_packed = nullptr;
        c->d_line_end = nullptr;
        const uint64_t cap = c->n_tokens + 1;
        if ((rc = dalloc(c, (void **) &c->d_packed, sizeof(int32_t) * cap, "packed corpus"))) return rc;
        if ((rc = dalloc(c, (void **) &c->d_line_end, sizeof(uint32_t) * cap, "line offsets"))) return rc;
        c->line_cap = cap;
    }
    if (tiles > c->tile_cap) {
        dfree(c, c->d_tile_kept, sizeof(uint32_t) * c->tile_cap);
        dfree(c, c->d_tile_zero, sizeof(uint32_t) * c->tile_cap);
        c->d_tile_kept = c->d_tile_zero = nullptr;
        c->tile_cap = 0;
        if ((rc = dalloc(c, (void **) &c->d_tile_kept, sizeof(uint32_t) * tiles, "tile sums"))) return rc;
        if ((rc = dalloc(c, (void **) &c->d_tile_zero, sizeof(uint32_t) * tiles, "tile sums"))) return rc;
        c->tile_cap = tiles;
    }
    return PARW2V_OK;
}

static bool stream_variant(const parw2v_ctx *c) { return c->cfg.variant != PARW2V_VARIANT_WINDOW; }

// Sentences in flight for the Hogwild modes, 0 = no cap.  Concurrency acts like extra step size on
// frequently updated rows (every sentence in flight computes its update from values the others
// have not yet changed), so the final loss falls below the reference's as it grows.  Measured
// against the reference's 16-thread runs: ~7,000 corpus tokens in flight centres a small corpus
// (3M-token text, 8M-token graph walks) on the reference's loss, and an 800M-token corpus stays
// within 1% with every warp of the device busy.  Default: max(7,000 tokens' worth of lines,
// lines / 8192); min_rounds > 0 caps at lines / min_rounds instead; min_rounds < 0: no cap.
static uint64_t hogwild_cap(int min_rounds, uint64_t n_lines, uint64_t n_tokens) {
    if (min_rounds < 0) return 0;
    if (min_rounds > 0) return std::max<uint64_t>(1, n_lines / (uint64_t) min_rounds);
    const uint64_t per_line = std::max<uint64_t>(1, n_tokens / std::max<uint64_t>(1, n_lines));
    return std::max<uint64_t>(std::max<uint64_t>(1, 7000 / per_line), n_lines / 8192);
}

// The autotuner (cfg.autotune): short timed trials of the BATCHED launch knobs that leave the
// result unchanged -- how the sentences in flight split into CTAs and warps (their number stays),
// the row elements per lane of the streamed kernel, the staging copies -- each on a prefix of the
// first epoch's packed corpus, after a warm launch, with the weights and counters restored after
// every launch.  The fastest is kept in the context.  Returns an error only for a failed CUDA call;
// without the memory for the weight backup it keeps the compiled-in choices.
static int autotune(parw2v_ctx *c, TrainArgs a, int base_grid, int base_warps) {
    const parw2v_config &k = c->cfg;
    c->tuned = {};
    struct Cand {
        int grid, warps, bulk, elems, pipe;
        bool stream;
    };
    std::vector<int> bulks;
    if (k.staging != PARW2V_STAGING_AUTO) bulks = {k.staging == PARW2V_STAGING_BULK ? 1 : 0};
    else if (batched_tensor_repulsion(k.window, k.negative, k.batch_size)) bulks = {0, 1};
    else bulks = {0};
    std::vector<Cand> cands;
    // the kernel organisation: STREAM and, when the same sentences in flight fit its shared memory,
    // WINDOW (both run the reference's order), unless cfg.variant fixes one
    for (int v = 0; v < 2; v++) {
        const bool stream = v == 0;
        if ((stream && k.variant == PARW2V_VARIANT_WINDOW) || (!stream && k.variant == PARW2V_VARIANT_STREAM)) continue;
        if (!stream && (k.attraction == PARW2V_ATTRACT_PIPELINED ||
                        batched_max_warps(c->ld, k.window, k.negative, k.batch_size, c->bf16, nullptr, false) < base_warps))
            continue;
        std::vector<std::pair<int, int>> splits = {{base_grid, base_warps}};
        for (int f : {2, 4})
            if (base_warps % f == 0 &&
                batched_ctas_per_sm(c->ld, k.window, k.negative, k.batch_size, c->bf16, stream, base_warps / f) >= f)
                splits.push_back({base_grid * f, base_warps / f});
        std::vector<int> elems = {0};
        if (stream) {
            const int e0 = stream_lane_elems_default(k.size), e1 = stream_lane_elems_next(e0);
            elems = {e0};
            if (e1) elems.push_back(e1);
        }
        // the sequential attraction in its plain or pipelined form, unless cfg.attraction fixes one
        std::vector<int> pipes = {stream ? a.attr_pipe : 0};
        if (stream && k.attraction == PARW2V_ATTRACT_DEFAULT) pipes = {0, 1};
        for (auto &sp : splits)
            for (int e : elems)
                for (int b : bulks)
                    for (int pp : pipes) cands.push_back({sp.first, sp.second, b, e, pp, stream});
    }
    if (cands.empty()) return PARW2V_OK;
    // epoch 0's packed corpus
    CK(c, cudaMemsetAsync(&c->d_cnt->work, 0, sizeof(unsigned long long), c->stream), "autotune");
    CK(c, launch_pack(a, c->d_packed, c->d_line_end, c->d_tile_kept, c->d_tile_zero, pack_tiles(c->n_tokens), c->stream),
       "autotune packing");
    DevCounters h0;
    int rc = read_counters(c, &h0);
    if (rc) return rc;
    const uint64_t inflight = (uint64_t) base_grid * base_warps;
    if (h0.n_lines == 0 || cands.size() < 2) return PARW2V_OK;
    const uint64_t trial = std::min<uint64_t>(h0.n_lines, std::max<uint64_t>(h0.n_lines / 50, 8 * inflight));
    const uint64_t warm = std::min<uint64_t>(h0.n_lines, inflight);
    const size_t wbytes = welem(c) * (size_t) c->vocab * c->ld;
    void *backup = nullptr;
    if (dalloc(c, &backup, 2 * wbytes, "autotune weight backup") != PARW2V_OK) {
        c->err.clear();
        return PARW2V_OK;
    }
    auto copy = [&](void *dst, const void *src) {
        return cudaMemcpyAsync(dst, src, wbytes, cudaMemcpyDeviceToDevice, c->stream);
    };
    cudaError_t e = copy(backup, c->d_w_in);
    if (e == cudaSuccess) e = copy((char *) backup + wbytes, c->d_w_out);
    float best_ms = 0.f;
    Cand best = cands[0];
    // PARW2V_AUTOTUNE_LOG set: every trial's time on stderr (diagnostics; the choice is the same)
    const bool log_trials = getenv("PARW2V_AUTOTUNE_LOG") != nullptr;
    for (size_t i = 0; i < cands.size() && e == cudaSuccess; i++) {
        const Cand &cd = cands[i];
        a.stage_bulk = cd.bulk;
        a.lane_elems = cd.elems;
        a.attr_pipe = cd.pipe;
        float ms = 0.f;
        for (int pass = 0; pass < 2 && e == cudaSuccess; pass++) {
            DevCounters hc = h0;
            hc.n_lines = pass == 0 ? warm : trial;
            hc.work = 0;
            e = cudaMemcpyAsync(c->d_cnt, &hc, sizeof(hc), cudaMemcpyHostToDevice, c->stream);
            if (e == cudaSuccess) e = cudaEventRecord(c->ev0, c->stream);
            if (e == cudaSuccess) e = launch_batched_train(a, c->bf16, cd.stream, cd.grid, cd.warps, c->stream);
            if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
            if (e == cudaSuccess) e = copy(c->d_w_in, backup);
            if (e == cudaSuccess) e = copy(c->d_w_out, (char *) backup + wbytes);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
            if (e == cudaSuccess && pass == 1) e = cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        }
        if (e == cudaSuccess && log_trials)
            fprintf(stderr, "parw2v autotune: %s, grid %d x %d warps, %d elements per lane, staging %s, attraction %s: "
                            "%.3f ms for %llu lines\n",
                    cd.stream ? "stream" : "window", cd.grid, cd.warps,
                    cd.stream ? (cd.elems ? cd.elems : stream_lane_elems_default(k.size)) : 0,
                    cd.bulk ? "bulk" : "cp.async", cd.pipe ? "pipelined" : "sequential", ms,
                    (unsigned long long) trial);
        if (e == cudaSuccess && (i == 0 || ms < best_ms)) {
            best_ms = ms;
            best = cd;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_cnt, &h0, sizeof(h0), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, backup, 2 * wbytes);
    if (e != cudaSuccess) return cuda_fail(c, e, "autotune trials");
    c->tuned.done = true;
    c->tuned.inflight = inflight;
    c->tuned.grid = best.grid;
    c->tuned.warps = best.warps;
    c->tuned.stage_bulk = best.bulk;
    c->tuned.lane_elems = best.elems;
    c->tuned.attr_pipe = best.pipe;
    c->tuned.stream = best.stream;
    return PARW2V_OK;
}

static int train_hogwild(parw2v_ctx *c, TrainArgs &a, parw2v_stats *st) {
    int rc = ensure_packing(c);
    if (rc) return rc;
    const int sms = device_sms(c);
    int grid = c->cfg.grid;
    int warps = c->cfg.warps_per_cta;
    const bool plain = c->cfg.mode == PARW2V_MODE_PLAIN;
    bool stream = stream_variant(c);  // BATCHED kernel organisation (the autotuner may change it)
    if (plain) {
        warps = plain_warps_per_cta(warps);
        if (!grid) grid = sms * 2;
        const size_t per = plain_scratch_floats(c->ld, c->cfg.batch_size, c->cfg.window, c->cfg.negative);
        const size_t need = per * (size_t) grid * warps;
        if (c->scratch_floats < need) {
            dfree(c, c->d_scratch, sizeof(float) * c->scratch_floats);
            c->d_scratch = nullptr;
            c->scratch_floats = 0;
            if ((rc = dalloc(c, (void **) &c->d_scratch, sizeof(float) * need, "PLAIN workspace"))) return rc;
            c->scratch_floats = need;
        }
        a.scratch = c->d_scratch;
        a.scratch_per_warp = per;
    } else {
        size_t per_warp = 0;
        const int maxw = batched_max_warps(c->ld, c->cfg.window, c->cfg.negative, c->cfg.batch_size, c->bf16, &per_warp,
                                           stream_variant(c));
        if (maxw <= 0) return fail(c, PARW2V_ERR_CAPACITY, "BATCHED mode: rows do not fit in shared memory");
        if (!warps || warps > maxw) warps = maxw;
        if (!grid) grid = sms;
    }
    // cap the sentences in flight (see parw2v_config.min_rounds)
    const uint64_t cap = hogwild_cap(c->cfg.min_rounds, c->n_lines, c->n_tokens);
    if (cap) {
        if ((uint64_t) grid * warps > cap) {
            // spread the capped warps over the SMs, never more CTAs than one wave
            const int per_sm = (int) std::max<uint64_t>(1, cap / (uint64_t) std::min(grid, sms));
            warps = std::min(warps, per_sm);
            grid = (int) std::min<uint64_t>((uint64_t) std::min(grid, sms), std::max<uint64_t>(1, cap / (uint64_t) warps));
        }
    }
    if (!plain && c->cfg.autotune) {
        const uint64_t inflight = (uint64_t) grid * warps;
        if (!c->tuned.done || c->tuned.inflight != inflight) {
            if ((rc = autotune(c, a, grid, warps))) return rc;
        }
        if (c->tuned.done && c->tuned.inflight == inflight) {
            grid = c->tuned.grid;
            warps = c->tuned.warps;
            a.stage_bulk = c->tuned.stage_bulk;
            a.lane_elems = c->tuned.lane_elems;
            a.attr_pipe = c->tuned.attr_pipe;
            stream = c->tuned.stream;
        }
    }
    c->last_grid = grid;
    c->last_warps = warps;
    // One epoch is two CUDA graphs, captured once and replayed for every epoch: (reset the work
    // counter, subsample and pack) and (train, advance the epoch index in device memory).  The
    // timing events are recorded between the two launches, outside the graphs.
    CK(c, cudaMemsetAsync(&c->d_cnt->epoch, 0, sizeof(unsigned), c->stream), "counters");
    // the graphs of the previous call serve again when every launch argument is the same
    const bool reuse = c->graphs[0] && c->graphs[1] && grid == c->graph_grid && warps == c->graph_warps &&
                       memcmp(&a, &c->graph_args, sizeof(TrainArgs)) == 0;
    if (!reuse) drop_graphs(c);
    cudaGraphExec_t *exec = c->graphs;
    cudaError_t e = cudaSuccess;
    for (int part = 0; part < 2 && e == cudaSuccess && !reuse; part++) {
        cudaGraph_t graph = nullptr;
        e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) break;
        if (part == 0) {
            e = cudaMemsetAsync(&c->d_cnt->work, 0, sizeof(unsigned long long), c->stream);
            if (e == cudaSuccess)
                e = launch_pack(a, c->d_packed, c->d_line_end, c->d_tile_kept, c->d_tile_zero, pack_tiles(c->n_tokens),
                                c->stream);
        } else {
            e = plain ? launch_plain_train(a, grid, warps, c->stream)
                      : launch_batched_train(a, c->bf16, stream, grid, warps, c->stream);
            if (e == cudaSuccess) e = launch_advance_epoch(c->d_cnt, c->stream);
        }
        const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
        if (e == cudaSuccess) e = ec;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec[part], graph, 0);
        if (graph) cudaGraphDestroy(graph);
    }
    if (e != cudaSuccess) {
        drop_graphs(c);
        return cuda_fail(c, e, "capturing the epoch graphs");
    }
    c->graph_args = a;
    c->graph_grid = grid;
    c->graph_warps = warps;
    float pack_ms_total = 0.f, kernel_ms_total = 0.f;
    for (int ep = 0; ep < c->cfg.iter; ep++) {
        nvtxRangePushA("parw2v epoch");
        e = cudaEventRecord(c->ev0, c->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec[0], c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec[1], c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev2, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        nvtxRangePop();
        if (e != cudaSuccess) {
            drop_graphs(c);
            return cuda_fail(c, e, "training epoch");
        }
        float m0 = 0, m1 = 0;
        cudaEventElapsedTime(&m0, c->ev0, c->ev1);
        cudaEventElapsedTime(&m1, c->ev1, c->ev2);
        pack_ms_total += m0;
        kernel_ms_total += m1;
    }
    DevCounters h;
    if ((rc = read_counters(c, &h))) return rc;
    if (st) {
        st->words = (uint64_t) c->n_tokens * (uint64_t) c->cfg.iter;
        st->kept = h.kept;
        st->sentences = h.sentences;
        st->pairs = h.pairs;
        st->batches = h.batches;
        st->negatives = h.negatives;
        st->kernel_ms = kernel_ms_total;
        st->pack_ms = pack_ms_total;
        // the schedule's rate after all epochs (the kernels' per-sentence rate at the end of the
        // last epoch), floored at alpha * 1e-4 (PAR_Word2Vec_cpu.cpp:437-445)
        const double done = (double) c->cfg.iter * (double) c->n_tokens;
        const float end_alpha =
            c->cfg.alpha * (float) (1.0 - done / ((double) c->cfg.iter * (double) c->train_words + 1.0));
        st->final_alpha = std::max(end_alpha, c->cfg.alpha * 0.0001f);
        st->grid = grid;
        st->warps_per_cta = warps;
        st->lane_elems = plain || !stream ? 0 : (a.lane_elems ? a.lane_elems : stream_lane_elems_default(c->cfg.size));
        st->variant = plain ? 0 : (stream ? PARW2V_VARIANT_STREAM : PARW2V_VARIANT_WINDOW);
        st->staging = plain ? 0 : (a.stage_bulk ? PARW2V_STAGING_BULK : PARW2V_STAGING_CPASYNC);
        st->attraction = a.sync_window ? PARW2V_ATTRACT_WINDOW
                                       : (!plain && a.attr_pipe ? PARW2V_ATTRACT_PIPELINED : PARW2V_ATTRACT_SEQUENTIAL);
        st->repulsion = plain ? PARW2V_REPULSION_SERIAL
                              : (batched_tensor_repulsion(c->cfg.window, c->cfg.negative, c->cfg.batch_size)
                                     ? PARW2V_REPULSION_TENSOR
                                     : PARW2V_REPULSION_CUDA);
    }
    if (h.error & kErrStaging)
        return fail(c, PARW2V_ERR_TIMEOUT, "a bulk copy of the repulsion's rows did not complete in time");
    if (h.error & kErrResample)
        return fail(c, PARW2V_ERR_TIMEOUT, "negative resampling exceeded its draw limit (every word is in the sentence?)");
    return PARW2V_OK;
}

int parw2v_train(parw2v_ctx *c, parw2v_stats *st) {
    if (!c) return fail(c, PARW2V_ERR_ARG, "null argument");
    if (!c->vocab) return fail(c, PARW2V_ERR_STATE, "set_vocab first");
    if (!c->weights_ready) return fail(c, PARW2V_ERR_STATE, "init_weights or set_weights first");
    if (!c->d_corpus) return fail(c, PARW2V_ERR_STATE, "set_corpus first");
    if (st) memset(st, 0, sizeof(*st));
    int rc = set_device(c);
    if (rc) return rc;
    CK(c, cudaMemsetAsync(c->d_cnt, 0, sizeof(DevCounters), c->stream), "counters");
    if (!c->corpus_checked) {
        // ids against the vocabulary and the count of lines: once per corpus and vocabulary
        if (c->n_tokens) {
            k_validate<<<148 * 4, 256, 0, c->stream>>>(c->d_corpus, c->n_tokens, c->vocab, c->d_cnt);
            CK(c, cudaGetLastError(), "validation kernel");
        }
        DevCounters h;
        if ((rc = read_counters(c, &h))) return rc;
        if (h.error & kErrCapacity) return fail(c, PARW2V_ERR_ARG, "corpus holds ids outside [0, vocab_size)");
        c->n_lines = h.n_lines;
        c->corpus_checked = true;
        CK(c, cudaMemsetAsync(c->d_cnt, 0, sizeof(DevCounters), c->stream), "counters");
    }
    TrainArgs a;
    memset(&a, 0, sizeof(a));  // padding too: the arguments are compared bytewise to reuse graphs
    a.corpus = c->d_corpus;
    a.n_tokens = c->n_tokens;
    a.keep_thr = c->d_thr;
    a.table = c->d_table;
    a.exp_table = c->d_exp;
    a.w_in = c->d_w_in;
    a.w_out = c->d_w_out;
    a.ld = c->ld;
    a.d = c->cfg.size;
    a.window = c->cfg.window;
    a.negative = c->cfg.negative;
    a.batch = c->cfg.batch_size;
    a.iter = c->cfg.iter;
    a.vocab = c->vocab;
    a.alpha0 = c->cfg.alpha;
    a.sample = c->cfg.sample;
    a.train_words = c->train_words;
    a.seed = c->cfg.seed;
    a.cnt = c->d_cnt;
    a.packed = c->d_packed;
    a.line_end = c->d_line_end;
    a.max_resample = 1LL << 20;
    a.sync_window = c->cfg.attraction == PARW2V_ATTRACT_WINDOW;
    a.stage_bulk = c->cfg.staging == PARW2V_STAGING_BULK;
    a.attr_pipe = c->cfg.attraction == PARW2V_ATTRACT_PIPELINED;
    if (c->cfg.mode == PARW2V_MODE_DET) return train_det(c, a, st);
    rc = ensure_packing(c);
    if (rc) return rc;
    a.packed = c->d_packed;
    a.line_end = c->d_line_end;
    return train_hogwild(c, a, st);
}

// ---- loss / adjoint / finite differences ----
struct DevBatch {
    void *mem = nullptr;
    size_t bytes = 0;
    LossBatch b{};
};

static int upload_batch(parw2v_ctx *c, const int32_t *tgt, const int32_t *ctxw, int n_pairs, const int32_t *neg,
                        int n_neg, int cpw, DevBatch &db) {
    if (!tgt || !ctxw || n_pairs <= 0 || cpw <= 0 || n_neg < 0 || (n_neg > 0 && !neg))
        return fail(c, PARW2V_ERR_ARG, "invalid minibatch");
    if (!c->weights_ready) return fail(c, PARW2V_ERR_STATE, "no weights on the device");
    const int n_win = (n_pairs + cpw - 1) / cpw;
    for (int i = 0; i < n_pairs; i++)
        if (tgt[i] < 0 || tgt[i] >= c->vocab || ctxw[i] < 0 || ctxw[i] >= c->vocab)
            return fail(c, PARW2V_ERR_ARG, "minibatch id outside the vocabulary");
    for (long long i = 0; i < (long long) n_win * n_neg; i++)
        if (neg[i] < 0 || neg[i] >= c->vocab) return fail(c, PARW2V_ERR_ARG, "negative id outside the vocabulary");
    const size_t n_negs = (size_t) n_win * n_neg;
    db.bytes = sizeof(int32_t) * (2 * (size_t) n_pairs + n_negs + 4);
    int rc = dalloc(c, &db.mem, db.bytes, "minibatch");
    if (rc) return rc;
    int32_t *p = (int32_t *) db.mem;
    cudaError_t e = cudaMemcpyAsync(p, tgt, sizeof(int32_t) * n_pairs, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p + n_pairs, ctxw, sizeof(int32_t) * n_pairs, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && n_negs)
        e = cudaMemcpyAsync(p + 2 * n_pairs, neg, sizeof(int32_t) * n_negs, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) {
        dfree(c, db.mem, db.bytes);
        return cuda_fail(c, e, "minibatch upload");
    }
    db.b.tgt = p;
    db.b.ctx = p + n_pairs;
    db.b.neg = p + 2 * n_pairs;
    db.b.n_pairs = n_pairs;
    db.b.n_neg = n_neg;
    db.b.ctx_per_window = cpw;
    return PARW2V_OK;
}

int parw2v_loss(parw2v_ctx *c, const int32_t *tgt, const int32_t *ctxw, int n_pairs, const int32_t *neg, int n_neg,
                int cpw, double *loss) {
    if (!c || !loss) return fail(c, PARW2V_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (rc) return rc;
    DevBatch db;
    if ((rc = upload_batch(c, tgt, ctxw, n_pairs, neg, n_neg, cpw, db))) return rc;
    double *d_out = nullptr;
    if ((rc = dalloc(c, (void **) &d_out, sizeof(double), "loss"))) {
        dfree(c, db.mem, db.bytes);
        return rc;
    }
    cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(double), c->stream);
    if (e == cudaSuccess) e = launch_loss(db.b, c->d_w_in, c->d_w_out, c->bf16, c->cfg.size, c->ld, d_out, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss, d_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, d_out, sizeof(double));
    dfree(c, db.mem, db.bytes);
    if (e != cudaSuccess) return cuda_fail(c, e, "loss kernel");
    return PARW2V_OK;
}

int parw2v_loss_adjoint(parw2v_ctx *c, const int32_t *tgt, const int32_t *ctxw, int n_pairs, const int32_t *neg,
                        int n_neg, int cpw, int exact, float *d_w_in, float *d_w_out) {
    if (!c) return fail(c, PARW2V_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (rc) return rc;
    DevBatch db;
    if ((rc = upload_batch(c, tgt, ctxw, n_pairs, neg, n_neg, cpw, db))) return rc;
    const size_t V = (size_t) c->vocab, ld = (size_t) c->ld;
    const size_t bytes = sizeof(float) * V * ld * 2;
    float *g = nullptr;
    if ((rc = dalloc(c, (void **) &g, bytes, "gradient buffers"))) {
        dfree(c, db.mem, db.bytes);
        return rc;
    }
    cudaError_t e = cudaMemsetAsync(g, 0, bytes, c->stream);
    if (e == cudaSuccess)
        e = launch_adjoint(db.b, c->d_w_in, c->d_w_out, c->bf16, c->cfg.size, c->ld, c->d_exp, exact, g, g + V * ld,
                           c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess && d_w_in) rc = copy_rows(c, nullptr, d_w_in, g, false);
    if (e == cudaSuccess && !rc && d_w_out) rc = copy_rows(c, nullptr, d_w_out, g + V * ld, false);
    dfree(c, g, bytes);
    dfree(c, db.mem, db.bytes);
    if (e != cudaSuccess) return cuda_fail(c, e, "adjoint kernel");
    return rc;
}

int parw2v_loss_fd(parw2v_ctx *c, const int32_t *tgt, const int32_t *ctxw, int n_pairs, const int32_t *neg, int n_neg,
                   int cpw, const int32_t *matrix, const int32_t *row, const int32_t *col, int n_probes, double h,
                   double *grad) {
    if (!c || !matrix || !row || !col || !grad || n_probes <= 0 || !(h > 0)) return fail(c, PARW2V_ERR_ARG, "invalid probes");
    for (int i = 0; i < n_probes; i++)
        if ((matrix[i] != 0 && matrix[i] != 1) || row[i] < 0 || row[i] >= c->vocab || col[i] < 0 || col[i] >= c->cfg.size)
            return fail(c, PARW2V_ERR_ARG, "probe outside the weights");
    int rc = set_device(c);
    if (rc) return rc;
    DevBatch db;
    if ((rc = upload_batch(c, tgt, ctxw, n_pairs, neg, n_neg, cpw, db))) return rc;
    const size_t pb = sizeof(int32_t) * 3 * (size_t) n_probes + sizeof(double) * (size_t) n_probes + 16;
    void *pm = nullptr;
    if ((rc = dalloc(c, &pm, pb, "probes"))) {
        dfree(c, db.mem, db.bytes);
        return rc;
    }
    double *d_grad = (double *) pm;
    int32_t *d_m = (int32_t *) (d_grad + n_probes);
    cudaError_t e = cudaMemcpyAsync(d_m, matrix, sizeof(int32_t) * n_probes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_m + n_probes, row, sizeof(int32_t) * n_probes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_m + 2 * n_probes, col, sizeof(int32_t) * n_probes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = launch_loss_fd(db.b, c->d_w_in, c->d_w_out, c->bf16, c->cfg.size, c->ld, d_m, d_m + n_probes,
                           d_m + 2 * n_probes, n_probes, h, d_grad, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, d_grad, sizeof(double) * n_probes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, pm, pb);
    dfree(c, db.mem, db.bytes);
    if (e != cudaSuccess) return cuda_fail(c, e, "finite-difference kernel");
    return PARW2V_OK;
}

}  // extern "C"
