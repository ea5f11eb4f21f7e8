// BATCHED (FP32) and BATCHED_BF16 modes: the data-local persistent kernel.
//
// One CTA per SM, W warps per CTA, one sentence per warp at a time (an atomic counter hands out
// "</s>"-terminated lines of the packed corpus; lines are cut into 1000-token sentences).  The
// sentence is processed as PAR_Word2Vec_cpu does it (PAR_Word2Vec_cpu.cpp:529-679) -- attraction
// for every position, then shared-negative repulsion per batch -- but rows live on chip:
//
//  attraction  W_in rows of the window [p-w, p+w] sit in shared memory as FP32 working copies,
//              in a ring of 2w+1+P slots.  Rows are prefetched P positions ahead with 16-byte
//              cp.async copies, so the dependent dot/axpy chain never waits on HBM.  A word that
//              occurs twice in the window shares one copy (ownership moves to the newest
//              occurrence), which keeps the reference's sequential semantics inside the sentence.
//              A row is written back once, when its last occurrence leaves the window.  The
//              target's W_out row lives in registers for the position (prefetched too).
//  repulsion   per batch of `batch` positions: rep_b * negative shared negatives from the unigram
//              table (redrawn while they occur in the sentence).  G = sigma(M_out M_in^T) is
//              accumulated over d in column chunks staged in shared memory; then a second pass
//              over the chunks forms M_out + G M_in and M_in + G^T M_out and writes each distinct
//              row once (duplicate negatives / rows are merged into one gradient row first).
//
// Rows of the global tables are read at L2 (ld.global.cg or cp.async.cg), never from the SM's L1,
// which is not coherent with other SMs' writes: a hot row served from a stale L1 line would turn
// its concurrent updates into lost ones.
// Write-back is "value + own update" (overwrite), never an atomic add: with thousands of
// sentences in flight, adding updates computed from stale copies of a hot row multiplies its
// step size and diverges; overwriting loses colliding updates, as the reference's unsynchronised
// `+=` does.  In BF16 mode the global tables are BF16, working copies and accumulation are FP32,
// and every write-back rounds stochastically (per-lane LCG bits, the sm_100a cvt.rs conversion).
#include <algorithm>

#include "common.cuh"
#include "internal.h"
#include "mma.cuh"
#include "repel.cuh"
#include "sentence.cuh"

namespace parw2v {

namespace {

constexpr int kPrefetch = 2;                  // P: positions prefetched ahead
constexpr int kRing = kPrefetch + 1;          // landing buffers for targets / BF16 rows
constexpr int kMaxWarpsB = 16;
constexpr size_t kSmemBudget = 227 * 1024;

struct Layout {  // per-warp shared-memory carve-up, in bytes (all offsets 16-byte aligned)
    int ws;            // window slots 2w+1+P
    int ch;            // repulsion column chunk (multiple of 4), CUDA-core path
    int kmax;          // 2 * window * negative
    rep::Geom geo;     // tensor-core repulsion (geo.mma), inside the region
    size_t region;     // window cur rows (+ BF16 landing ring) | repulsion buffers
    size_t raw_off;    // BF16 landing ring inside the region
    size_t tgt_off, g_off, neg_off, dup_off, meta_off, ctx_off, exit_off, bar_off, per_warp;
};

__host__ __device__ inline size_t up16(size_t x) { return (x + 15) & ~(size_t) 15; }

// Head of a CTA's shared memory: the expTable (1,001 floats, padded) and 32 bytes of CTA-wide
// constants (STREAM variant: the 2w divisor, the line count and the kept-token count), read from
// there rather than held in registers; the warps' regions follow.
constexpr size_t kExpBytes = 1004 * sizeof(float);
constexpr size_t kSmemHead = kExpBytes + 32;
static_assert(sizeof(FastMod) == 16, "the 2w divisor takes 16 of the 32 bytes");
static_assert(kExpBytes % 16 == 0, "the constants after the expTable are 16-byte aligned");

__host__ __device__ inline Layout make_layout(int ld, int window, int negative, int batch, bool bf16) {
    Layout L;
    L.ws = 2 * window + 1 + kPrefetch;
    L.kmax = 2 * window * negative;
    const size_t row32 = (size_t) ld * 4, row_st = (size_t) ld * (bf16 ? 2 : 4);
    const size_t window_bytes = up16((size_t) L.ws * row32);
    L.raw_off = window_bytes;
    const size_t win_total = window_bytes + (bf16 ? up16((size_t) kRing * row_st) : 0);
    // the CUDA-core path's column chunk: as wide as fits in the window's bytes, at least 16 columns
    const size_t rows_rep = (size_t) (batch + L.kmax);
    long ch = (long) (win_total / (rows_rep * 4)) - 4;
    ch = ch / 4 * 4;
    if (ch > ((ld + 3) / 4) * 4) ch = ((ld + 3) / 4) * 4;
    if (ch < 16) ch = 16;
    L.ch = (int) ch;
    L.geo = rep::make_geom(window, negative, batch, bf16);
    const size_t rep_bytes = L.geo.mma ? L.geo.bytes : up16(rows_rep * (size_t) (L.ch + 4) * 4);
    L.region = win_total > rep_bytes ? win_total : rep_bytes;
    L.tgt_off = L.region;
    L.g_off = L.tgt_off + up16((size_t) kRing * row_st);
    const size_t g_floats = L.geo.mma ? 0 : (size_t) L.kmax * batch;
    L.neg_off = L.g_off + up16(g_floats * 4);
    L.dup_off = L.neg_off + up16((size_t) L.kmax * 4);
    L.meta_off = L.dup_off + up16((size_t) (L.kmax + 2 * batch) * 4);
    L.ctx_off = L.meta_off + up16((size_t) L.ws * 8);
    L.exit_off = L.ctx_off + up16((size_t) (2 * window) * 8);
    L.bar_off = L.exit_off + up16((size_t) kPrefetch * 4 + 16);
    L.per_warp = L.bar_off + 16;
    return L;
}

template <int NV4>
struct Row {
    float4 v[NV4];
};

__device__ __forceinline__ float4 f4_fma(float g, float4 x, float4 y) {  // g * x + y
    return make_float4(fmaf(g, x.x, y.x), fmaf(g, x.y, y.y), fmaf(g, x.z, y.z), fmaf(g, x.w, y.w));
}
__device__ __forceinline__ float f4_dot(float4 x, float4 y, float acc) {
    return fmaf(x.x, y.x, fmaf(x.y, y.y, fmaf(x.z, y.z, fmaf(x.w, y.w, acc))));
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prefetch() {
    asm volatile("cp.async.wait_group %0;" ::"n"(kPrefetch) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <bool BF16>
struct Store;

template <>
struct Store<false> {  // FP32 tables
    using T = float;
    static constexpr int kChunkElems = 4;  // elements per 16-byte copy
    __device__ static float2 load2(const float *row, int q) { return reinterpret_cast<const float2 *>(row)[q]; }
    __device__ static void store2(float *row, int q, float2 v, uint64_t) { reinterpret_cast<float2 *>(row)[q] = v; }
    __device__ static float4 load4(const float *row, int j4) { return reinterpret_cast<const float4 *>(row)[j4]; }
    // a row of the global tables: read at L2, never from this SM's (non-coherent) L1
    __device__ static float4 load4g(const float *row, int j4) { return __ldcg(reinterpret_cast<const float4 *>(row) + j4); }
    __device__ static void store4(float *row, int j4, float4 v, uint64_t) { reinterpret_cast<float4 *>(row)[j4] = v; }
    // 16-byte lane chunks as stored (read ahead and kept in this form until used)
    using Raw = float4;
    __device__ static Raw zero_raw() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ static Raw loadraw_g(const float *row, int j4) { return __ldcg(reinterpret_cast<const float4 *>(row) + j4); }
    __device__ static float4 widen(Raw r) { return r; }
    __device__ static Raw pack4(float4 v, uint64_t) { return v; }
    __device__ static void storeraw(float *row, int j4, Raw r) { reinterpret_cast<float4 *>(row)[j4] = r; }
};

template <>
struct Store<true> {  // BF16 tables
    using T = __nv_bfloat16;
    static constexpr int kChunkElems = 8;
    __device__ static float2 load2(const __nv_bfloat16 *row, int q) {
        return __bfloat1622float2(reinterpret_cast<const __nv_bfloat162 *>(row)[q]);
    }
    __device__ static void store2(__nv_bfloat16 *row, int q, float2 v, uint64_t h) {
        reinterpret_cast<unsigned *>(row)[q] = pack_sr2(v, h);
    }
    __device__ static float4 widen(uint2 u) {
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ static float4 load4(const __nv_bfloat16 *row, int j4) { return widen(reinterpret_cast<const uint2 *>(row)[j4]); }
    // a row of the global tables: read at L2, never from this SM's (non-coherent) L1
    __device__ static float4 load4g(const __nv_bfloat16 *row, int j4) {
        return widen(__ldcg(reinterpret_cast<const uint2 *>(row) + j4));
    }
    __device__ static void store4(__nv_bfloat16 *row, int j4, float4 v, uint64_t h) {
        reinterpret_cast<uint2 *>(row)[j4] = pack4(v, h);
    }
    // 4 BF16 as stored (read ahead and kept in this form until used: 2 registers, not 4)
    using Raw = uint2;
    __device__ static Raw zero_raw() { return make_uint2(0u, 0u); }
    __device__ static Raw loadraw_g(const __nv_bfloat16 *row, int j4) { return __ldcg(reinterpret_cast<const uint2 *>(row) + j4); }
    __device__ static Raw pack4(float4 v, uint64_t h) {
        uint2 u;
        u.x = pack_sr2(make_float2(v.x, v.y), h);
        u.y = pack_sr2(make_float2(v.z, v.w), h >> 32);
        return u;
    }
    __device__ static void storeraw(__nv_bfloat16 *row, int j4, Raw r) { reinterpret_cast<uint2 *>(row)[j4] = r; }
};


// Repulsion of one batch on the CUDA cores (FP32 tables, or shapes beyond the mma path): G is
// accumulated over column chunks staged as FP32, then a second pass writes the new rows.
template <bool BF16>
__device__ __noinline__ void repel_simt(const TrainArgs &a, const Layout &Lo, unsigned char *base, const int32_t *bw, int rows,
                           const int *negs, int K, float alpha, const float *s_exp, float *G, int *dup, int lane,
                           LaneBits &rb) {
    using S = Store<BF16>;
    using T = typename S::T;
    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const int ld = a.ld, B = a.batch;
    const int stride = Lo.ch + 4;
    float *s_in = reinterpret_cast<float *>(base);
    float *s_out = s_in + (size_t) B * stride;
    const int c4 = Lo.ch / 4;
    for (int e = lane; e < K * rows; e += 32) G[e] = 0.f;
    __syncwarp();
    auto stage_chunk = [&](int col0) {
        const int ncol4 = min(c4, (ld - col0 + 3) / 4);
        for (int rr = 0; rr < rows + K; rr++) {
            const T *src = rr < rows ? w_in + (size_t) __ldg(bw + rr) * ld : w_out + (size_t) negs[rr - rows] * ld;
            float *dst = rr < rows ? s_in + (size_t) rr * stride : s_out + (size_t) (rr - rows) * stride;
            for (int j4 = lane; j4 < c4; j4 += 32)
                reinterpret_cast<float4 *>(dst)[j4] = j4 < ncol4 ? S::load4g(src + col0, j4) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
    };
    for (int col0 = 0; col0 < ld; col0 += Lo.ch) {
        stage_chunk(col0);
        for (int e = lane; e < K * rows; e += 32) {
            const int k = e / rows, r = e - k * rows;
            const float4 *po = reinterpret_cast<const float4 *>(s_out + (size_t) k * stride);
            const float4 *pi = reinterpret_cast<const float4 *>(s_in + (size_t) r * stride);
            float acc = 0.f;
            for (int j4 = 0; j4 < c4; j4++) {
                const float4 u = po[j4], v = pi[j4];
                acc = fmaf(u.x, v.x, fmaf(u.y, v.y, fmaf(u.z, v.z, fmaf(u.w, v.w, acc))));
            }
            G[e] += acc;
        }
        __syncwarp();
    }
    for (int e = lane; e < K * rows; e += 32) G[e] = grad_from_table(G[e], 0, alpha, s_exp);
    __syncwarp();
    rep::mark_repeats(negs, K, bw, rows, dup, lane);
    rep::merge_marked(K, rows, G, rows, dup, lane);
    for (int col0 = 0; col0 < ld; col0 += Lo.ch) {
        stage_chunk(col0);
        const int ncol4 = min(c4, (ld - col0 + 3) / 4);
        for (int k = 0; k < K; k++) {
            if (dup[k] >= 0) continue;
            for (int j4 = lane; j4 < ncol4; j4 += 32) {
                float4 acc = reinterpret_cast<const float4 *>(s_out + (size_t) k * stride)[j4];
                for (int r = 0; r < rows; r++) {
                    const float gk = G[k * rows + r];
                    const float4 v = reinterpret_cast<const float4 *>(s_in + (size_t) r * stride)[j4];
                    acc = make_float4(fmaf(gk, v.x, acc.x), fmaf(gk, v.y, acc.y), fmaf(gk, v.z, acc.z), fmaf(gk, v.w, acc.w));
                }
                S::store4(w_out + (size_t) negs[k] * ld + col0, j4, acc, rb.next());
            }
        }
        for (int r = 0; r < rows; r++) {
            if (dup[K + r] >= 0) continue;
            const int word = __ldg(bw + r);
            for (int j4 = lane; j4 < ncol4; j4 += 32) {
                float4 acc = reinterpret_cast<const float4 *>(s_in + (size_t) r * stride)[j4];
                for (int k = 0; k < K; k++) {
                    const float gk = G[k * rows + r];
                    const float4 v = reinterpret_cast<const float4 *>(s_out + (size_t) k * stride)[j4];
                    acc = make_float4(fmaf(gk, v.x, acc.x), fmaf(gk, v.y, acc.y), fmaf(gk, v.z, acc.z), fmaf(gk, v.w, acc.w));
                }
                S::store4(w_in + (size_t) word * ld + col0, j4, acc, rb.next());
            }
        }
        __syncwarp();
    }
}

// The repulsion of one batch on the path its shapes allow (tensor cores for rows <= 32 and at most
// 96 negatives, else CUDA cores).  False if the staging could not complete: the caller stops.
template <bool BF16>
__device__ __forceinline__ bool repel_batch(const TrainArgs &a, const Layout &Lo, unsigned char *base, const int32_t *bw,
                                            int rows, const int *negs, int K, float alpha, const float *s_exp, float *G,
                                            int *dup, int lane, LaneBits &rb, rep::Stager &st) {
    if (Lo.geo.mma) {
        int *sbw = dup + Lo.kmax + a.batch;  // the batch's words, read once
        if (lane < rows) sbw[lane] = __ldg(bw + lane);
        __syncwarp();
        if constexpr (BF16) {
            return rep::repel_bf16(a, Lo.geo, base, sbw, rows, negs, K, alpha, s_exp, dup, lane, rb, st);
        } else {
            return Lo.geo.mt <= 3 ? rep::repel_f32<3>(a, Lo.geo, base, sbw, rows, negs, K, alpha, s_exp, dup, lane, st)
                                  : rep::repel_f32<6>(a, Lo.geo, base, sbw, rows, negs, K, alpha, s_exp, dup, lane, st);
        }
    }
    repel_simt<BF16>(a, Lo, base, bw, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
    return true;
}

// The warp's staging barrier, initialised once per warp before any copy uses it.
__device__ __forceinline__ rep::Stager make_stager(unsigned char *bar_mem, int stage_bulk, int lane) {
    uint64_t *bar = reinterpret_cast<uint64_t *>(bar_mem);
    if (lane == 0) mbar_init(bar, 1);
    __syncwarp();
    return rep::Stager{bar, 0u, stage_bulk != 0};
}

template <int NV4, bool BF16, bool SYNC>
__global__ void __launch_bounds__(kMaxWarpsB * 32, 1) k_batched_train(TrainArgs a, int warps) {
    using S = Store<BF16>;
    using T = typename S::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = a.window, B = a.batch, ld = a.ld, d = a.d;
    const FastMod mod_w((uint32_t) w), mod_2w((uint32_t) (2 * w));
    const int n4 = (d + 3) >> 2;  // float4 chunks that carry data (the padding stays zero)
    const Layout Lo = make_layout(ld, w, a.negative, B, BF16);
    float *s_exp = reinterpret_cast<float *>(smem_raw);
    for (int i = threadIdx.x; i <= kExpTableSize; i += blockDim.x) s_exp[i] = a.exp_table[i];
    __syncthreads();
    if (wid >= warps) return;

    unsigned char *base = smem_raw + kSmemHead + (size_t) wid * Lo.per_warp;
    float *cur = reinterpret_cast<float *>(base);                        // ws x ld FP32 (window)
    T *raw = reinterpret_cast<T *>(base + Lo.raw_off);                    // kRing x ld landing (BF16)
    T *tgt = reinterpret_cast<T *>(base + Lo.tgt_off);                    // kRing x ld target landing
    float *G = reinterpret_cast<float *>(base + Lo.g_off);
    int *negs = reinterpret_cast<int *>(base + Lo.neg_off);
    int *dup = reinterpret_cast<int *>(base + Lo.dup_off);
    int *slot_word = reinterpret_cast<int *>(base + Lo.meta_off);
    int *slot_alias = slot_word + Lo.ws;
    float *ctx_g = reinterpret_cast<float *>(base + Lo.ctx_off);        // 2w: window-synchronous gradients
    int *ctx_s = reinterpret_cast<int *>(ctx_g + 2 * w);                 // 2w: and context slots
    int *recent_exit = reinterpret_cast<int *>(base + Lo.exit_off);      // words written back lately
    rep::Stager st = make_stager(base + Lo.bar_off, a.stage_bulk, lane);

    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const uint64_t n_lines = a.cnt->n_lines, total_kept = a.cnt->total_kept;
    const int epoch = hogwild_epoch(a);
    const int row_chunks = ld / S::kChunkElems;  // 16-byte pieces per stored row
    // c mod ws for positions c < 2^16 by a multiply-high reciprocal (exact: ws <= 256)
    const unsigned ws_u = (unsigned) Lo.ws, ws_m = (unsigned) (0xFFFFFFFFULL / ws_u) + 1u;
    auto ring = [&](int c) { return (int) ((unsigned) c - __umulhi((unsigned) c, ws_m) * ws_u); };
    unsigned long long st_kept = 0, st_sent = 0, st_pairs = 0, st_batches = 0, st_negs = 0;
    bool failed = false;
    unsigned fail_bits = 0;

    for (;;) {
        unsigned long long line = 0;
        if (lane == 0) line = atomicAdd(&a.cnt->work, 1ULL);
        line = __shfl_sync(0xffffffffu, line, 0);
        if (line >= n_lines || failed) break;
        const uint32_t lo_line = line ? a.line_end[line - 1] : 0u, hi_line = a.line_end[line];
        int piece = 0;
        for (uint32_t c0 = lo_line; c0 < hi_line; c0 += kMaxSentence, piece++) {
            const int L = (int) min((uint32_t) kMaxSentence, hi_line - c0);
            const int32_t *sen = a.packed + c0;
            uint64_t rng = sentence_seed_b(a, epoch, line, piece);
            LaneBits rb{(uint32_t) mix64(rng ^ (0xA24BAED4963EE407ULL * (uint64_t) (lane + 1))) | 1u};
            const float alpha = sentence_alpha_b(a, epoch, c0, total_kept);

            // ---- attraction (:529-568) ----
            // One loop from p = -max(w, P) to L + w: positions join the window at step q - w (the
            // first max(w, P) of them synchronously, the rest from P-ahead cp.async copies), the
            // target of step p >= 0 is trained, and position q leaves at step q + w + 1.
            for (int i = lane; i < Lo.ws; i += 32) {
                slot_word[i] = -1;
                slot_alias[i] = -1;
            }
            if (lane < kPrefetch) recent_exit[lane] = -1;
            __syncwarp();
            Row<NV4> y;
            int prev_t = -1, prev2_t = -1;
            const int p_first = -max(w, kPrefetch);
            for (int p = p_first; p <= L + w; p++) {
                // leave: the row of position p - w - 1 goes back to the table once its last
                // occurrence in the window is done (overwrite; BF16 rounds stochastically)
                const int q_out = p - w - 1;
                if (q_out >= 0 && q_out < L) {
                    const int s = ring(q_out);
                    if (slot_alias[s] < 0) {
                        const int word = slot_word[s];
                        T *row = w_in + (size_t) word * ld;
                        const float4 *src = reinterpret_cast<const float4 *>(cur + (size_t) s * ld);
                        for (int c = lane; c < n4; c += 32) S::store4(row, c, src[c], rb.next());
                        if (lane == 0) {
                            for (int i = kPrefetch - 1; i > 0; i--) recent_exit[i] = recent_exit[i - 1];
                            recent_exit[0] = word;
                        }
                    }
                    __syncwarp();
                    if (lane == 0) {
                        slot_word[s] = -1;
                        slot_alias[s] = -1;
                    }
                }
                if (p >= L) continue;
                // prefetch: W_in row of position p + w + P, W_out row of target p + P
                if (p >= -kPrefetch) {
                    const int qi = p + w + kPrefetch, qt = p + kPrefetch;
                    if (qi < L) {
                        const unsigned char *src = reinterpret_cast<const unsigned char *>(w_in + (size_t) __ldg(sen + qi) * ld);
                        unsigned char *dst = BF16 ? reinterpret_cast<unsigned char *>(raw + (size_t) (qi % kRing) * ld)
                                                  : reinterpret_cast<unsigned char *>(cur + (size_t) ring(qi) * ld);
                        for (int m = lane; m < row_chunks; m += 32) cp_async16(dst + 16 * (size_t) m, src + 16 * (size_t) m);
                    }
                    if (qt >= 0 && qt < L) {
                        const unsigned char *src = reinterpret_cast<const unsigned char *>(w_out + (size_t) __ldg(sen + qt) * ld);
                        unsigned char *dst = reinterpret_cast<unsigned char *>(tgt + (size_t) (qt % kRing) * ld);
                        for (int m = lane; m < row_chunks; m += 32) cp_async16(dst + 16 * (size_t) m, src + 16 * (size_t) m);
                    }
                    cp_async_commit();
                }
                if (p >= 0) cp_async_wait_prefetch();
                __syncwarp();
                // enter: position p + w joins the window; a word already inside keeps one shared
                // copy (ownership moves to the newest occurrence)
                const int qn = p + w;
                if (qn >= 0 && qn < L) {
                    const int s = ring(qn);
                    const int word = __ldg(sen + qn);
                    int owner = -1;
                    for (int c = max(0, p - w) + lane; c < qn; c += 32) {
                        const int sc = ring(c);
                        if (slot_alias[sc] < 0 && slot_word[sc] == word) owner = sc;
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, owner >= 0);
                    bool recently_written = false;
                    for (int i = 0; i < kPrefetch; i++) recently_written |= (recent_exit[i] == word);
                    float4 *dst = reinterpret_cast<float4 *>(cur + (size_t) s * ld);
                    const bool landed = qn >= w;  // prefetched (else loaded here)
                    if (m) {
                        owner = __shfl_sync(0xffffffffu, owner, __ffs(m) - 1);
                        const float4 *src = reinterpret_cast<const float4 *>(cur + (size_t) owner * ld);
                        for (int c = lane; c < n4; c += 32) dst[c] = src[c];
                        for (int i = lane; i < Lo.ws; i += 32)
                            if (slot_alias[i] == owner) slot_alias[i] = s;
                        __syncwarp();
                        if (lane == 0) slot_alias[owner] = s;
                    } else if (BF16 || !landed || recently_written) {
                        // a landed copy can predate this sentence's own write-back of the word: reload
                        if (recently_written || !landed) {
                            const T *src = w_in + (size_t) word * ld;
                            for (int c = lane; c < n4; c += 32) dst[c] = S::load4g(src, c);
                        } else {
                            const T *src = raw + (size_t) (qn % kRing) * ld;
                            for (int c = lane; c < n4; c += 32) dst[c] = S::load4(src, c);
                        }
                    }
                    if (lane == 0) {
                        slot_word[s] = word;
                        slot_alias[s] = -1;
                    }
                    __syncwarp();
                }
                if (p < 0) continue;
                // the target row into registers (reused when the word repeats; reloaded when its
                // landed copy predates the write-back two positions ago)
                const int t = __ldg(sen + p);
                if (t != prev_t) {
                    const bool fresh = t == prev2_t;  // global row, else the landed copy in shared memory
                    const T *src = fresh ? w_out + (size_t) t * ld : tgt + (size_t) (p % kRing) * ld;
#pragma unroll
                    for (int i = 0; i < NV4; i++) {
                        const int c = lane + 32 * i;
                        y.v[i] = c < n4 ? (fresh ? S::load4g(src, c) : S::load4(src, c)) : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
                rng = lcg_next(rng);
                const int b = (int) mod_w(rng);
                const int lo_c = max(p - w + b, 0), hi_c = min(p + w - b, L - 1);
                const int n = hi_c - lo_c;  // contexts [lo_c, hi_c] without p, in window order
                if constexpr (SYNC) {
                    // window-synchronous: every context scored against the same target row
                    for (int i0 = 0; i0 < n; i0 += 2) {
                        float f[2] = {0.f, 0.f};
                        int sl[2] = {-1, -1};
#pragma unroll
                        for (int u = 0; u < 2; u++)
                            if (i0 + u < n) {
                                const int c = lo_c + i0 + u + (lo_c + i0 + u >= p ? 1 : 0);
                                const int s0 = ring(c), al = slot_alias[s0];
                                sl[u] = al < 0 ? s0 : al;
                                const float4 *x = reinterpret_cast<const float4 *>(cur + (size_t) sl[u] * ld);
#pragma unroll
                                for (int k = 0; k < NV4; k++) {
                                    const int cc = lane + 32 * k;
                                    if (cc < n4) f[u] = f4_dot(x[cc], y.v[k], f[u]);
                                }
                            }
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            f[0] += __shfl_xor_sync(0xffffffffu, f[0], o);
                            f[1] += __shfl_xor_sync(0xffffffffu, f[1], o);
                        }
                        if (lane == 0)
#pragma unroll
                            for (int u = 0; u < 2; u++)
                                if (i0 + u < n) {
                                    ctx_g[i0 + u] = grad_from_table(f[u], 1, alpha, s_exp);
                                    ctx_s[i0 + u] = sl[u];
                                }
                    }
                    __syncwarp();
                    if (lane == 0)  // a word twice among the contexts: one slot, summed gradient
                        for (int i = 1; i < n; i++)
                            for (int k = 0; k < i; k++)
                                if (ctx_s[k] == ctx_s[i]) {
                                    ctx_g[k] += ctx_g[i];
                                    ctx_g[i] = 0.f;
                                    break;
                                }
                    __syncwarp();
                    Row<NV4> dy;
#pragma unroll
                    for (int k = 0; k < NV4; k++) dy.v[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                    for (int i = 0; i < n; i++) {
                        const float g = ctx_g[i];
                        float4 *x = reinterpret_cast<float4 *>(cur + (size_t) ctx_s[i] * ld);
#pragma unroll
                        for (int k = 0; k < NV4; k++) {
                            const int cc = lane + 32 * k;
                            if (cc < n4) {
                                const float4 xv = x[cc];
                                dy.v[k] = f4_fma(g, xv, dy.v[k]);
                                if (g != 0.f) x[cc] = f4_fma(g, y.v[k], xv);
                            }
                        }
                    }
#pragma unroll
                    for (int k = 0; k < NV4; k++)
                        y.v[k] = make_float4(y.v[k].x + dy.v[k].x, y.v[k].y + dy.v[k].y, y.v[k].z + dy.v[k].z,
                                             y.v[k].w + dy.v[k].w);
                } else {
                    // the reference's order: each context sees the target row as the previous left it
                    for (int i = 0; i < n; i++) {
                        const int c = lo_c + i + (lo_c + i >= p ? 1 : 0);
                        const int s0 = ring(c), al = slot_alias[s0];
                        float4 *x = reinterpret_cast<float4 *>(cur + (size_t) (al < 0 ? s0 : al) * ld);
                        Row<NV4> xr;
                        float f = 0.f;
#pragma unroll
                        for (int k = 0; k < NV4; k++) {
                            const int cc = lane + 32 * k;
                            xr.v[k] = cc < n4 ? x[cc] : make_float4(0.f, 0.f, 0.f, 0.f);
                            f = f4_dot(xr.v[k], y.v[k], f);
                        }
                        f = warp_sum(f);
                        const float g = grad_from_table(f, 1, alpha, s_exp);
#pragma unroll
                        for (int k = 0; k < NV4; k++) {
                            const int cc = lane + 32 * k;
                            const float4 yv = y.v[k];
                            y.v[k] = f4_fma(g, xr.v[k], yv);
                            if (cc < n4) x[cc] = f4_fma(g, yv, xr.v[k]);
                        }
                    }
                }
                st_pairs += n;
                // target write-back
                T *trow = w_out + (size_t) t * ld;
#pragma unroll
                for (int i = 0; i < NV4; i++) {
                    const int c = lane + 32 * i;
                    if (c < n4) S::store4(trow, c, y.v[i], rb.next());
                }
                prev2_t = prev_t;
                prev_t = t;
                __syncwarp();
            }
            cp_async_wait_all();
            __threadfence_block();
            __syncwarp();

            // ---- repulsion (:571-679) ----
            const int num_batch = (L + B - 1) / B;
            for (int nb = 0; nb < num_batch && !failed; nb++) {
                const int lo_b = nb * B;
                const int rows = min(B, L - lo_b);
                rng = lcg_next(rng);
                const int rep_b = (int) ((lo_b <= w - 1 || (L - 1) - lo_b <= w - 1) ? mod_w(rng) : mod_2w(rng));
                const int K = rep_b * a.negative;
                if (!warp_draw_negatives(a.table, a.vocab, rng, sen, L, K, negs, lane, a.max_resample)) {
                    failed = true;  // unresolved negatives: leave the batch untouched
                    fail_bits |= kErrResample;
                    break;
                }
                st_batches++;
                st_negs += K;
                if (K > 0 && !repel_batch<BF16>(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb, st)) {
                    failed = true;  // a staging copy did not complete
                    fail_bits |= kErrStaging;
                    break;
                }
                __threadfence_block();
                __syncwarp();
            }
            st_kept += L;
            st_sent++;
        }
    }
    if (lane == 0) {
        atomicAdd(&a.cnt->kept, st_kept);
        atomicAdd(&a.cnt->sentences, st_sent);
        atomicAdd(&a.cnt->pairs, st_pairs);
        atomicAdd(&a.cnt->batches, st_batches);
        atomicAdd(&a.cnt->negatives, st_negs);
        if (fail_bits) atomicOr(&a.cnt->error, fail_bits);
    }
}

template <int NV4, bool BF16, bool SYNC>
cudaError_t launch_nvs(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    const Layout Lo = make_layout(a.ld, a.window, a.negative, a.batch, BF16);
    const size_t smem = kSmemHead + (size_t) warps * Lo.per_warp;
    cudaError_t e = cudaFuncSetAttribute(k_batched_train<NV4, BF16, SYNC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) smem);
    if (e != cudaSuccess) return e;
    k_batched_train<NV4, BF16, SYNC><<<grid, warps * 32, smem, s>>>(a, warps);
    return cudaGetLastError();
}

template <int NV4, bool BF16>
cudaError_t launch_nv(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    return a.sync_window ? launch_nvs<NV4, BF16, true>(a, grid, warps, s) : launch_nvs<NV4, BF16, false>(a, grid, warps, s);
}

// ---- STREAM variant: rows stay in global memory (L1-resident while a window reuses them) ----
// Attraction reads and writes W rows directly, as the PLAIN kernel does, in lanes of 16-byte
// chunks (BF16 tables rounded stochastically at every write); the repulsion is the same on-chip
// staged tensor-core (BF16) or CUDA-core (FP32) contraction as the WINDOW variant.  Without the
// window ring a warp needs ~11 KB of shared memory (d = 300, window 5, 5 negatives), so more
// sentences are in flight per SM and more of the unified L1 is left to cache rows.
constexpr int kMaxWarpsS = 16;
constexpr int kStreamStats = 5;  // kept, sentences, pairs, batches, negatives (per warp, in shared memory)
constexpr size_t kSimtStage = 6400;  // CUDA-core repulsion staging bytes (column chunk as wide as fits)

__host__ __device__ inline Layout make_layout_stream(int ld, int window, int negative, int batch, bool bf16) {
    Layout L;
    L.ws = 0;
    L.kmax = 2 * window * negative;
    L.geo = rep::make_geom(window, negative, batch, bf16);
    L.raw_off = 0;
    L.tgt_off = 0;
    L.meta_off = 0;
    const size_t rows_rep = (size_t) (batch + L.kmax);
    long ch = (long) (kSimtStage / (rows_rep * 4)) - 4;
    ch = ch / 4 * 4;
    if (ch > ((ld + 3) / 4) * 4) ch = ((ld + 3) / 4) * 4;
    if (ch < 16) ch = 16;
    L.ch = (int) ch;
    if (L.geo.mma) {
        L.region = L.geo.bytes;
        L.g_off = 0;  // unused: the tensor-core paths keep G inside the region
    } else {
        L.region = up16(rows_rep * (size_t) (L.ch + 4) * 4);
        L.g_off = L.region;
    }
    const size_t g_bytes = L.geo.mma ? 0 : up16((size_t) L.kmax * batch * 4);
    L.neg_off = L.region + g_bytes;
    L.dup_off = L.neg_off + up16((size_t) L.kmax * 4);
    L.ctx_off = L.dup_off + up16((size_t) (L.kmax + 2 * batch) * 4);
    L.exit_off = L.ctx_off + up16((size_t) (2 * window) * 8);
    L.bar_off = L.exit_off + up16(kStreamStats * sizeof(unsigned long long));  // after the warp's statistics
    L.per_warp = L.bar_off + 16;
    return L;
}

// A table row as one warp holds it in the streamed kernel: E elements per lane (d <= 32 E), in up to
// three chunks of 16, 8 and 4 bytes.  Chunk j of 16 bytes covers elements j * 32 * EA + lane * EA
// (EA = 8 BF16 / 4 FP32); the 8-byte chunk (EB = 4 / 2 elements) and the 4-byte chunk (EC = 2 / 1)
// follow them.  At d = 300, BF16, that is one 16-byte and one 4-byte chunk per lane: 10 elements,
// 320 slots for 300 values (a lane of only 16-byte... chunks would hold 12 or 16).  Chunks that lie
// beyond the row's ld elements are neither read nor written; elements in [d, ld) are the row's zero
// padding and stay zero (0 + g * 0).
template <bool BF16, int E>
struct LaneRow {
    using T = typename Store<BF16>::T;
    static constexpr int EA = BF16 ? 8 : 4, EB = BF16 ? 4 : 2, EC = BF16 ? 2 : 1;
    static constexpr int NA = E / EA;
    static constexpr int NB = (E - NA * EA) / EB;
    static constexpr int NC = (E - NA * EA - NB * EB) / EC;
    static_assert(NA * EA + NB * EB + NC * EC == E && NB <= 1 && NC <= 1, "E must split into the chunk sizes");
    static constexpr int W = NA * 4 + NB * 2 + NC;  // 32-bit words per lane as stored
    static constexpr int OFF_B = NA * 32 * EA, OFF_C = OFF_B + NB * 32 * EB;
    struct Raw {
        uint32_t w[W];
    };
    // which chunks of this lane lie inside a row of ld elements: bits 0..NA-1, NA (B), NA+1 (C)
    __device__ static unsigned valid_mask(int lane, int ld) {
        unsigned m = 0;
#pragma unroll
        for (int j = 0; j < NA; j++)
            if (j * 32 * EA + (lane + 1) * EA <= ld) m |= 1u << j;
        if (NB && OFF_B + (lane + 1) * EB <= ld) m |= 1u << NA;
        if (NC && OFF_C + (lane + 1) * EC <= ld) m |= 2u << NA;
        return m;
    }
    // the lane's chunks of a table row, read at L2 (never from this SM's non-coherent L1)
    __device__ static Raw load(const T *row, int lane, unsigned vm) {
        Raw r;
#pragma unroll
        for (int j = 0; j < NA; j++) {
            uint4 u = make_uint4(0u, 0u, 0u, 0u);
            if (vm & (1u << j)) u = __ldcg(reinterpret_cast<const uint4 *>(row + j * 32 * EA) + lane);
            r.w[4 * j] = u.x;
            r.w[4 * j + 1] = u.y;
            r.w[4 * j + 2] = u.z;
            r.w[4 * j + 3] = u.w;
        }
        if (NB) {
            uint2 u = make_uint2(0u, 0u);
            if (vm & (1u << NA)) u = __ldcg(reinterpret_cast<const uint2 *>(row + OFF_B) + lane);
            r.w[4 * NA] = u.x;
            r.w[4 * NA + 1] = u.y;
        }
        if (NC) {
            unsigned u = 0u;
            if (vm & (2u << NA)) u = __ldcg(reinterpret_cast<const unsigned *>(row + OFF_C) + lane);
            r.w[W - 1] = u;
        }
        return r;
    }
    __device__ static void store(T *row, const Raw &r, int lane, unsigned vm) {
#pragma unroll
        for (int j = 0; j < NA; j++)
            if (vm & (1u << j))
                reinterpret_cast<uint4 *>(row + j * 32 * EA)[lane] =
                    make_uint4(r.w[4 * j], r.w[4 * j + 1], r.w[4 * j + 2], r.w[4 * j + 3]);
        if (NB && (vm & (1u << NA)))
            reinterpret_cast<uint2 *>(row + OFF_B)[lane] = make_uint2(r.w[4 * NA], r.w[4 * NA + 1]);
        if (NC && (vm & (2u << NA))) reinterpret_cast<unsigned *>(row + OFF_C)[lane] = r.w[W - 1];
    }
    __device__ static void widen(const Raw &r, float (&v)[E]) {
        if constexpr (BF16) {
#pragma unroll
            for (int i = 0; i < W; i++) {
                v[2 * i] = __uint_as_float(r.w[i] << 16);
                v[2 * i + 1] = __uint_as_float(r.w[i] & 0xFFFF0000u);
            }
        } else {
#pragma unroll
            for (int i = 0; i < E; i++) v[i] = __uint_as_float(r.w[i]);
        }
    }
    // as stored: BF16 rounds stochastically (one 64-bit draw per four values), FP32 as is
    __device__ static Raw pack(const float (&v)[E], LaneBits &rb) {
        Raw r;
        if constexpr (BF16) {
#pragma unroll
            for (int i = 0; i < W; i += 2) {
                const uint64_t h = rb.next();
                r.w[i] = pack_sr2(make_float2(v[2 * i], v[2 * i + 1]), h);
                if (i + 1 < W) r.w[i + 1] = pack_sr2(make_float2(v[2 * i + 2], v[2 * i + 3]), h >> 32);
            }
        } else {
#pragma unroll
            for (int i = 0; i < E; i++) r.w[i] = __float_as_uint(v[i]);
        }
        return r;
    }
    // The lane's part of x . y with four independent partial sums (element i into sum i mod 4, a
    // chain of ceil(E/4) FMAs), formed two sums per instruction by the packed FP32 FMA of sm_100
    // (each element rounds exactly as fmaf).
    __device__ static float dot(const float (&x)[E], const float (&y)[E]) {
        float2 f01 = make_float2(0.f, 0.f), f23 = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < E; k += 2) {
            const float2 p = make_float2(x[k], x[k + 1]), q = make_float2(y[k], y[k + 1]);
            if (k & 2) f23 = __ffma2_rn(p, q, f23);
            else f01 = __ffma2_rn(p, q, f01);
        }
        return (f01.x + f01.y) + (f23.x + f23.y);
    }
    // out = g * a + b, two elements per packed FMA (out may be b)
    __device__ static void fma_scaled(float g, const float (&a)[E], const float (&b)[E], float (&out)[E]) {
        const float2 g2 = make_float2(g, g);
#pragma unroll
        for (int k = 0; k < E; k += 2) {
            const float2 r = __ffma2_rn(g2, make_float2(a[k], a[k + 1]), make_float2(b[k], b[k + 1]));
            out[k] = r.x;
            out[k + 1] = r.y;
        }
    }
};

// ATT: 0 the reference's sequential attraction; 1 window-synchronous; 2 sequential, pipelined (the
// same updates in the same order, with each pair's dot products taken before the previous pair's
// gradient is known).
template <bool BF16, int E, int ATT>
__global__ void __launch_bounds__(kMaxWarpsS * 32, 1) k_stream_train(TrainArgs a, int warps) {
    constexpr bool SYNC = ATT == 1;
    using LR = LaneRow<BF16, E>;
    using T = typename LR::T;
    using Raw = typename LR::Raw;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = a.window, B = a.batch, ld = a.ld;
    const FastMod mod_w((uint32_t) w);
    const Layout Lo = make_layout_stream(ld, w, a.negative, B, BF16);
    float *s_exp = reinterpret_cast<float *>(smem_raw);
    FastMod *s_mod_2w = reinterpret_cast<FastMod *>(smem_raw + kExpBytes);
    uint64_t *s_totals = reinterpret_cast<uint64_t *>(smem_raw + kExpBytes + sizeof(FastMod));  // lines, kept
    for (int i = threadIdx.x; i <= kExpTableSize; i += blockDim.x) s_exp[i] = a.exp_table[i];
    if (threadIdx.x == 0) {
        *s_mod_2w = FastMod((uint32_t) (2 * w));
        s_totals[0] = a.cnt->n_lines;
        s_totals[1] = a.cnt->total_kept;
    }
    __syncthreads();
    if (wid >= warps) return;
    unsigned char *base = smem_raw + kSmemHead + (size_t) wid * Lo.per_warp;
    float *G = reinterpret_cast<float *>(base + Lo.g_off);
    int *negs = reinterpret_cast<int *>(base + Lo.neg_off);
    int *dup = reinterpret_cast<int *>(base + Lo.dup_off);
    float *ctx_g = reinterpret_cast<float *>(base + Lo.ctx_off);
    int *ctx_w = reinterpret_cast<int *>(ctx_g + 2 * w);
    // statistics live in shared memory (lane 0 adds once per sentence), not in registers
    unsigned long long *wst = reinterpret_cast<unsigned long long *>(base + Lo.exit_off);
    if (lane == 0)
        for (int i = 0; i < kStreamStats; i++) wst[i] = 0;
    rep::Stager st = make_stager(base + Lo.bar_off, a.stage_bulk, lane);
    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const unsigned vm = LR::valid_mask(lane, ld);
    const int epoch = hogwild_epoch(a);
    bool failed = false;
    unsigned fail_bits = 0;

    for (;;) {
        unsigned long long line = 0;
        if (lane == 0) line = atomicAdd(&a.cnt->work, 1ULL);
        line = __shfl_sync(0xffffffffu, line, 0);
        if (line >= s_totals[0] || failed) break;
        const uint32_t lo_line = line ? a.line_end[line - 1] : 0u, hi_line = a.line_end[line];
        int piece = 0;
        for (uint32_t c0 = lo_line; c0 < hi_line; c0 += kMaxSentence, piece++) {
            const int L = (int) min((uint32_t) kMaxSentence, hi_line - c0);
            const int32_t *sen = a.packed + c0;
            uint64_t rng = sentence_seed_b(a, epoch, line, piece);
            LaneBits rb{(uint32_t) mix64(rng ^ (0xA24BAED4963EE407ULL * (uint64_t) (lane + 1))) | 1u};
            const float alpha = sentence_alpha_b(a, epoch, c0, s_totals[1]);
            unsigned pairs = 0, batches = 0, negs_drawn = 0;
            // ---- attraction (:529-568) ----
            // Rows are read one step ahead (the next target's row during this position, the next
            // context's row during this pair, and during a position's last pair the first context
            // row of the next position; BF16 tables only), so the L2 latency overlaps the
            // dependent chain.  A row read ahead that this warp writes before using it (the same
            // word again) is replaced by the value written.  Each position's b is drawn one
            // position ahead, from the same random stream, so the next position's first context
            // is known in time.  With FP32 tables the raw row is twice the registers, and keeping
            // it across positions measured slower: there a position reads its first row itself.
            Raw yn = LR::load(w_out + (size_t) __ldg(sen) * ld, lane, vm);
            rng = lcg_next(rng);
            int b_next = (int) mod_w(rng);
            Raw xn;
            int c_next = 1, w_next = 0;  // position 0's first context is position 1 (its window starts at 0)
            if constexpr (!SYNC && BF16) {
                if (L > 1) {
                    w_next = __ldg(sen + 1);
                    xn = LR::load(w_in + (size_t) w_next * ld, lane, vm);
                }
            }
            for (int p = 0; p < L; p++) {
                const int b = b_next;
                if (p + 1 < L) {
                    rng = lcg_next(rng);
                    b_next = (int) mod_w(rng);
                }
                const int t = __ldg(sen + p);
                T *yrow = w_out + (size_t) t * ld;
                float y[E];
                LR::widen(yn, y);
                const int t_next = p + 1 < L ? __ldg(sen + p + 1) : t;
                if (t_next != t) yn = LR::load(w_out + (size_t) t_next * ld, lane, vm);
                const int lo_c = max(p - w + b, 0), hi_c = min(p + w - b, L - 1);
                const int n = hi_c - lo_c;
                if constexpr (SYNC) {
                    // window-synchronous: every context scored against the same target row
                    for (int i0 = 0; i0 < n; i0 += 2) {
                        float f[2] = {0.f, 0.f};
                        int wd[2] = {-1, -1};
#pragma unroll
                        for (int u = 0; u < 2; u++)
                            if (i0 + u < n) {
                                const int c = lo_c + i0 + u + (lo_c + i0 + u >= p ? 1 : 0);
                                wd[u] = __ldg(sen + c);
                                float xv[E];
                                LR::widen(LR::load(w_in + (size_t) wd[u] * ld, lane, vm), xv);
                                f[u] = LR::dot(xv, y);
                            }
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            f[0] += __shfl_xor_sync(0xffffffffu, f[0], o);
                            f[1] += __shfl_xor_sync(0xffffffffu, f[1], o);
                        }
                        if (lane == 0)
#pragma unroll
                            for (int u = 0; u < 2; u++)
                                if (i0 + u < n) {
                                    ctx_g[i0 + u] = grad_from_table(f[u], 1, alpha, s_exp);
                                    ctx_w[i0 + u] = wd[u];
                                }
                    }
                    __syncwarp();
                    if (lane == 0)  // a word twice among the contexts: one update with the summed gradient
                        for (int i = 1; i < n; i++)
                            for (int k = 0; k < i; k++)
                                if (ctx_w[k] == ctx_w[i]) {
                                    ctx_g[k] += ctx_g[i];
                                    ctx_g[i] = 0.f;
                                    break;
                                }
                    __syncwarp();
                    float dy[E];
#pragma unroll
                    for (int k = 0; k < E; k++) dy[k] = 0.f;
                    for (int i = 0; i < n; i++) {
                        const float g = ctx_g[i];
                        T *x = w_in + (size_t) ctx_w[i] * ld;
                        float xv[E];
                        LR::widen(LR::load(x, lane, vm), xv);
                        LR::fma_scaled(g, xv, dy, dy);
                        LR::fma_scaled(g, y, xv, xv);
                        if (g != 0.f) LR::store(x, LR::pack(xv, rb), lane, vm);
                    }
#pragma unroll
                    for (int k = 0; k < E; k += 2) {
                        const float2 r = __fadd2_rn(make_float2(y[k], y[k + 1]), make_float2(dy[k], dy[k + 1]));
                        y[k] = r.x;
                        y[k + 1] = r.y;
                    }
                } else if (n > 0) {
                    // contexts c in [lo_c, hi_c] without p, in window order; the first one and its
                    // row were read during the previous position (L > 1 gives every position one)
                    int c = c_next;
                    int wc = w_next;
                    if constexpr (!BF16) {
                        c = lo_c == p ? lo_c + 1 : lo_c;
                        wc = __ldg(sen + c);
                        xn = LR::load(w_in + (size_t) wc * ld, lane, vm);
                    }
                    // the next position's first context: its window start, which is below it
                    // (b_next < w), so never the position itself
                    const bool has_next = p + 1 < L;
                    const int c_first_next = max(p + 1 - w + b_next, 0);
                    if constexpr (ATT == 2) {
                        // f_{i+1} = x_{i+1} . y_i = x_{i+1} . y_{i-1} + g_i (x_{i+1} . x_i): both dot
                        // products and their warp sums are formed while g_i is looked up, so one
                        // scalar FMA and the table lookup are all that each pair waits for.  The
                        // row of pair i+2 is read after pair i's store; a pair whose word repeats the
                        // previous pair's uses the value just stored and the sequential form.
                        int word = wc;
                        float xr[E];
                        LR::widen(xn, xr);
                        float f = warp_sum(LR::dot(xr, y));
                        if (1 < n || (BF16 && has_next)) {
                            c = 1 < n ? (c + 1 == p ? c + 2 : c + 1) : c_first_next;
                            wc = __ldg(sen + c);
                            if (wc != word) xn = LR::load(w_in + (size_t) wc * ld, lane, vm);
                        }
                        for (int i = 0; i < n; i++) {
                            const float g = grad_from_table(f, 1, alpha, s_exp);
                            const bool more = i + 1 < n;
                            const int word1 = wc;
                            float x1[E], P = 0.f, Q = 0.f;
                            if (more) {
                                LR::widen(xn, x1);
                                warp_sum2(LR::dot(x1, y), LR::dot(x1, xr), lane, P, Q);
                            }
                            T *x = w_in + (size_t) word * ld;
                            float xw[E];
                            LR::fma_scaled(g, y, xr, xw);  // from the entry values of y
                            LR::fma_scaled(g, xr, y, y);
                            const Raw r = LR::pack(xw, rb);
                            LR::store(x, r, lane, vm);
                            if (i + 2 < n || (BF16 && has_next && more)) {
                                c = i + 2 < n ? (c + 1 == p ? c + 2 : c + 1) : c_first_next;
                                wc = __ldg(sen + c);
                                if (wc != word1) xn = LR::load(w_in + (size_t) wc * ld, lane, vm);
                            }
                            if (more) {
                                if (word1 == word) {
                                    LR::widen(r, x1);
                                    f = warp_sum(LR::dot(x1, y));
                                } else {
                                    f = fmaf(g, Q, P);
                                }
#pragma unroll
                                for (int k = 0; k < E; k++) xr[k] = x1[k];
                                word = word1;
                            } else if (BF16 && has_next && wc == word) {
                                xn = r;  // the next position's first context is this row, just stored
                            }
                        }
                    } else {
                    for (int i = 0; i < n; i++) {
                        const int word = wc;
                        T *x = w_in + (size_t) word * ld;
                        float xr[E];
                        LR::widen(xn, xr);
                        float f = LR::dot(xr, y);
                        const bool more = i + 1 < n;
                        const bool ahead = more || (BF16 && has_next);
                        if (ahead) {
                            c = more ? (c + 1 == p ? c + 2 : c + 1) : c_first_next;
                            wc = __ldg(sen + c);
                            if (wc != word) xn = LR::load(w_in + (size_t) wc * ld, lane, vm);
                        }
                        f = BF16 ? warp_sum_fixed(f) : warp_sum(f);
                        const float g = grad_from_table(f, 1, alpha, s_exp);
                        float xw[E];
                        LR::fma_scaled(g, y, xr, xw);  // from the entry values of y
                        LR::fma_scaled(g, xr, y, y);
                        const Raw r = LR::pack(xw, rb);
                        LR::store(x, r, lane, vm);
                        if (ahead && wc == word) xn = r;
                    }
                    }
                    c_next = c;
                    w_next = wc;
                }
                pairs += n;
                const Raw r = LR::pack(y, rb);
                LR::store(yrow, r, lane, vm);
                if (t_next == t) yn = r;
            }
            __syncwarp();  // this sentence's row writes before any lane's staging reads
            // ---- repulsion (:571-679) ----
            const int num_batch = (L + B - 1) / B;
            for (int nb = 0; nb < num_batch && !failed; nb++) {
                const int lo_b = nb * B;
                const int rows = min(B, L - lo_b);
                rng = lcg_next(rng);
                const int rep_b = (int) ((lo_b <= w - 1 || (L - 1) - lo_b <= w - 1) ? mod_w(rng) : (*s_mod_2w)(rng));
                const int K = rep_b * a.negative;
                if (!warp_draw_negatives(a.table, a.vocab, rng, sen, L, K, negs, lane, a.max_resample)) {
                    failed = true;
                    fail_bits |= kErrResample;
                    break;
                }
                batches++;
                negs_drawn += K;
                if (K > 0 && !repel_batch<BF16>(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb, st)) {
                    failed = true;  // a staging copy did not complete
                    fail_bits |= kErrStaging;
                    break;
                }
                __syncwarp();
            }
            if (lane == 0) {
                wst[0] += L;
                wst[1] += 1;
                wst[2] += pairs;
                wst[3] += batches;
                wst[4] += negs_drawn;
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.cnt->kept, wst[0]);
        atomicAdd(&a.cnt->sentences, wst[1]);
        atomicAdd(&a.cnt->pairs, wst[2]);
        atomicAdd(&a.cnt->batches, wst[3]);
        atomicAdd(&a.cnt->negatives, wst[4]);
        if (fail_bits) atomicOr(&a.cnt->error, fail_bits);
    }
}

template <bool BF16, int E, int ATT>
cudaError_t launch_stream_e(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    const Layout Lo = make_layout_stream(a.ld, a.window, a.negative, a.batch, BF16);
    const size_t smem = kSmemHead + (size_t) warps * Lo.per_warp;
    cudaError_t e = cudaFuncSetAttribute(k_stream_train<BF16, E, ATT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    k_stream_train<BF16, E, ATT><<<grid, warps * 32, smem, s>>>(a, warps);
    return cudaGetLastError();
}

// Elements per lane of the streamed kernel's rows for a hidden size d (d <= 32 E).
inline int stream_lane_elems(int d) { return d <= 128 ? 4 : d <= 256 ? 8 : d <= 320 ? 10 : d <= 384 ? 12 : 16; }

template <bool BF16, int E>
cudaError_t launch_stream_es(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    if (a.sync_window) return launch_stream_e<BF16, E, 1>(a, grid, warps, s);
    return a.attr_pipe ? launch_stream_e<BF16, E, 2>(a, grid, warps, s) : launch_stream_e<BF16, E, 0>(a, grid, warps, s);
}

template <bool BF16>
cudaError_t launch_stream_mode(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    if (a.d > 512) return cudaErrorInvalidValue;
    const int e = a.lane_elems ? a.lane_elems : stream_lane_elems(a.d);
    if (32 * e < a.d) return cudaErrorInvalidValue;
    switch (e) {
        case 4: return launch_stream_es<BF16, 4>(a, grid, warps, s);
        case 8: return launch_stream_es<BF16, 8>(a, grid, warps, s);
        case 10: return launch_stream_es<BF16, 10>(a, grid, warps, s);
        case 12: return launch_stream_es<BF16, 12>(a, grid, warps, s);
        case 16: return launch_stream_es<BF16, 16>(a, grid, warps, s);
        default: return cudaErrorInvalidValue;
    }
}

template <bool BF16>
cudaError_t launch_mode(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    switch ((a.d + 127) / 128) {  // float4 chunks per lane
        case 1: return launch_nv<1, BF16>(a, grid, warps, s);
        case 2: return launch_nv<2, BF16>(a, grid, warps, s);
        case 3: return launch_nv<3, BF16>(a, grid, warps, s);
        case 4: return launch_nv<4, BF16>(a, grid, warps, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int batched_max_warps(int ld, int window, int negative, int batch, bool bf16, size_t *per_warp, bool stream) {
    const Layout Lo = stream ? make_layout_stream(ld, window, negative, batch, bf16) : make_layout(ld, window, negative, batch, bf16);
    if (per_warp) *per_warp = Lo.per_warp;
    const size_t avail = kSmemBudget - kSmemHead;
    long w = (long) (avail / Lo.per_warp);
    const long cap = stream ? kMaxWarpsS : kMaxWarpsB;
    if (w > cap) w = cap;
    return (int) w;
}

int batched_ctas_per_sm(int ld, int window, int negative, int batch, bool bf16, bool stream, int warps) {
    const Layout Lo = stream ? make_layout_stream(ld, window, negative, batch, bf16) : make_layout(ld, window, negative, batch, bf16);
    const size_t smem = kSmemHead + (size_t) warps * Lo.per_warp + 1024;  // + the CTA's reserved 1 KB
    const int by_smem = (int) ((228u * 1024u) / smem);
    const int by_threads = 2048 / (32 * warps);
    const int by_regs = 65536 / (128 * 32 * warps);
    return std::min(by_smem, std::min(by_threads, by_regs));
}

int stream_lane_elems_default(int d) { return stream_lane_elems(d); }
int stream_lane_elems_next(int e) { return e == 4 ? 8 : e == 8 ? 10 : e == 10 ? 12 : e == 12 ? 16 : 0; }

bool batched_tensor_repulsion(int window, int negative, int batch) {
    return rep::make_geom(window, negative, batch, true).mma;
}

cudaError_t launch_batched_train(const TrainArgs &a, bool bf16, bool stream, int grid, int warps_per_cta, cudaStream_t s) {
    if (stream)
        return bf16 ? launch_stream_mode<true>(a, grid, warps_per_cta, s) : launch_stream_mode<false>(a, grid, warps_per_cta, s);
    return bf16 ? launch_mode<true>(a, grid, warps_per_cta, s) : launch_mode<false>(a, grid, warps_per_cta, s);
}

}  // namespace parw2v
