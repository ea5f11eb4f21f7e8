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
// Write-back is "value + own update" (overwrite), never an atomic add: with thousands of
// sentences in flight, adding updates computed from stale copies of a hot row multiplies its
// step size and diverges; overwriting loses colliding updates, as the reference's unsynchronised
// `+=` does.  In BF16 mode the global tables are BF16, working copies and accumulation are FP32,
// and every write-back rounds stochastically (a counter-based hash supplies the 16 random bits).
#include "common.cuh"
#include "internal.h"

namespace parw2v {

namespace {

constexpr int kPrefetch = 2;                  // P: positions prefetched ahead
constexpr int kRing = kPrefetch + 1;          // landing buffers for targets / BF16 rows
constexpr int kMaxWarpsB = 16;
constexpr size_t kSmemBudget = 227 * 1024;

struct Layout {  // per-warp shared-memory carve-up, in bytes (all offsets 16-byte aligned)
    int ws;            // window slots 2w+1+P
    int ch;            // repulsion column chunk (multiple of 4)
    int kmax;          // 2 * window * negative
    size_t region;     // window cur rows (+ BF16 landing ring) | repulsion chunk staging
    size_t raw_off;    // BF16 landing ring inside the region
    size_t tgt_off, g_off, neg_off, dup_off, meta_off, exit_off, per_warp;
};

__host__ __device__ inline size_t up16(size_t x) { return (x + 15) & ~(size_t) 15; }

__host__ __device__ inline Layout make_layout(int ld, int window, int negative, int batch, bool bf16) {
    Layout L;
    L.ws = 2 * window + 1 + kPrefetch;
    L.kmax = 2 * window * negative;
    const size_t row32 = (size_t) ld * 4, row_st = (size_t) ld * (bf16 ? 2 : 4);
    const size_t window_bytes = up16((size_t) L.ws * row32);
    L.raw_off = window_bytes;
    const size_t win_total = window_bytes + (bf16 ? up16((size_t) kRing * row_st) : 0);
    // the column chunk: as wide as fits in the window's bytes, at least 16 columns
    const size_t rows_rep = (size_t) (batch + L.kmax);
    long ch = (long) (win_total / (rows_rep * 4)) - 4;
    ch = ch / 4 * 4;
    if (ch > ((ld + 3) / 4) * 4) ch = ((ld + 3) / 4) * 4;
    if (ch < 16) ch = 16;
    L.ch = (int) ch;
    const size_t rep_bytes = up16(rows_rep * (size_t) (L.ch + 4) * 4);
    L.region = win_total > rep_bytes ? win_total : rep_bytes;
    L.tgt_off = L.region;
    L.g_off = L.tgt_off + up16((size_t) kRing * row_st);
    L.neg_off = L.g_off + up16((size_t) L.kmax * batch * 4);
    L.dup_off = L.neg_off + up16((size_t) L.kmax * 4);
    L.meta_off = L.dup_off + up16((size_t) (L.kmax + batch) * 4);
    L.exit_off = L.meta_off + up16((size_t) L.ws * 8);
    L.per_warp = L.exit_off + up16((size_t) kPrefetch * 4 + 16);
    return L;
}

template <int NV2>
struct Row {
    float2 v[NV2];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prefetch() {
    asm volatile("cp.async.wait_group %0;" ::"n"(kPrefetch) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Stochastic rounding FP32 -> BF16: add 16 uniform bits below the kept mantissa, truncate.
__device__ __forceinline__ unsigned short sr_bf16(float x, unsigned bits16) {
    unsigned u = __float_as_uint(x);
    if ((u & 0x7f800000u) != 0x7f800000u) u += bits16 & 0xFFFFu;
    return (unsigned short) (u >> 16);
}
__device__ __forceinline__ unsigned pack_sr2(float2 v, uint64_t h) {
    return (unsigned) sr_bf16(v.x, (unsigned) h) | ((unsigned) sr_bf16(v.y, (unsigned) (h >> 16)) << 16);
}

template <bool BF16>
struct Store;

template <>
struct Store<false> {  // FP32 tables
    using T = float;
    static constexpr int kChunkElems = 4;  // elements per 16-byte copy
    __device__ static float2 load2(const float *row, int q) { return reinterpret_cast<const float2 *>(row)[q]; }
    __device__ static void store2(float *row, int q, float2 v, uint64_t) { reinterpret_cast<float2 *>(row)[q] = v; }
    __device__ static float4 load4(const float *row, int j4) { return reinterpret_cast<const float4 *>(row)[j4]; }
    __device__ static void store4(float *row, int j4, float4 v, uint64_t) { reinterpret_cast<float4 *>(row)[j4] = v; }
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
    __device__ static float4 load4(const __nv_bfloat16 *row, int j4) {
        const uint2 u = reinterpret_cast<const uint2 *>(row)[j4];
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ static void store4(__nv_bfloat16 *row, int j4, float4 v, uint64_t h) {
        uint2 u;
        u.x = pack_sr2(make_float2(v.x, v.y), h);
        u.y = pack_sr2(make_float2(v.z, v.w), h >> 32);
        reinterpret_cast<uint2 *>(row)[j4] = u;
    }
};

__device__ __forceinline__ float sentence_alpha_b(const TrainArgs &a, uint64_t kept_before, uint64_t total_kept) {
    const double done = (double) a.epoch * (double) a.n_tokens +
                        (total_kept ? (double) kept_before / (double) total_kept : 0.0) * (double) a.n_tokens;
    float alpha = a.alpha0 * (float) (1.0 - done / ((double) a.iter * (double) a.train_words + 1.0));
    const float floor_a = a.alpha0 * 0.0001f;
    return alpha < floor_a ? floor_a : alpha;
}

__device__ __forceinline__ uint64_t sentence_seed_b(const TrainArgs &a, uint64_t line, int piece) {
    return mix64(mix64(a.seed ^ (0xD1B54A32D192ED03ULL * (uint64_t) (a.epoch + 1))) ^ (line * 1024ULL + piece));
}

template <int NV2, bool BF16>
__global__ void __launch_bounds__(kMaxWarpsB * 32, 1) k_batched_train(TrainArgs a, int warps) {
    using S = Store<BF16>;
    using T = typename S::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = a.window, B = a.batch, ld = a.ld, d = a.d;
    const int n2 = (d + 1) >> 1;  // float2 chunks that carry data (the padding stays zero)
    const Layout Lo = make_layout(ld, w, a.negative, B, BF16);
    float *s_exp = reinterpret_cast<float *>(smem_raw);
    for (int i = threadIdx.x; i <= kExpTableSize; i += blockDim.x) s_exp[i] = a.exp_table[i];
    __syncthreads();
    if (wid >= warps) return;

    unsigned char *base = smem_raw + up16(1004 * sizeof(float)) + (size_t) wid * Lo.per_warp;
    float *cur = reinterpret_cast<float *>(base);                        // ws x ld FP32 (window)
    T *raw = reinterpret_cast<T *>(base + Lo.raw_off);                    // kRing x ld landing (BF16)
    float *stage = reinterpret_cast<float *>(base);                      // repulsion chunks (aliases)
    T *tgt = reinterpret_cast<T *>(base + Lo.tgt_off);                    // kRing x ld target landing
    float *G = reinterpret_cast<float *>(base + Lo.g_off);               // kmax x B
    int *negs = reinterpret_cast<int *>(base + Lo.neg_off);
    int *dup = reinterpret_cast<int *>(base + Lo.dup_off);
    int *slot_word = reinterpret_cast<int *>(base + Lo.meta_off);
    int *slot_alias = slot_word + Lo.ws;
    int *recent_exit = reinterpret_cast<int *>(base + Lo.exit_off);      // words written back lately

    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const uint64_t n_lines = a.cnt->n_lines, total_kept = a.cnt->total_kept;
    const int row_chunks = ld / S::kChunkElems;  // 16-byte pieces per stored row
    unsigned long long st_kept = 0, st_sent = 0, st_pairs = 0, st_batches = 0, st_negs = 0;
    bool failed = false;

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
            uint64_t rng = sentence_seed_b(a, line, piece);
            const float alpha = sentence_alpha_b(a, c0, total_kept);

            auto slot_of = [&](int c) {
                const int s = c % Lo.ws;
                const int al = slot_alias[s];
                return al < 0 ? s : al;
            };
            // a position joins the window: share the row with an occurrence already inside, else
            // take the landed copy (BF16: widen it into the slot)
            auto enter = [&](int q, int first_in_window, bool landed_in_slot, const T *landing) {
                const int s = q % Lo.ws;
                const int word = __ldg(sen + q);
                int owner = -1;
                for (int c = first_in_window + lane; c < q; c += 32) {
                    const int sc = c % Lo.ws;
                    if (slot_alias[sc] < 0 && slot_word[sc] == word) owner = sc;
                }
                const unsigned m = __ballot_sync(0xffffffffu, owner >= 0);
                bool recently_written = false;
                for (int i = 0; i < kPrefetch; i++) recently_written |= (recent_exit[i] == word);
                float *dst = cur + (size_t) s * ld;
                if (m) {
                    owner = __shfl_sync(0xffffffffu, owner, __ffs(m) - 1);
                    const float *src = cur + (size_t) owner * ld;
                    for (int qq = lane; qq < n2; qq += 32)
                        reinterpret_cast<float2 *>(dst)[qq] = reinterpret_cast<const float2 *>(src)[qq];
                    for (int i = lane; i < Lo.ws; i += 32)
                        if (slot_alias[i] == owner) slot_alias[i] = s;
                    __syncwarp();
                    if (lane == 0) slot_alias[owner] = s;
                } else if (!landed_in_slot || recently_written) {
                    // landed copy may predate this sentence's own write-back of the word: reload
                    const T *src = (recently_written || landing == nullptr) ? w_in + (size_t) word * ld : landing;
                    for (int qq = lane; qq < n2; qq += 32) reinterpret_cast<float2 *>(dst)[qq] = S::load2(src, qq);
                }
                if (lane == 0) {
                    slot_word[s] = word;
                    slot_alias[s] = -1;
                }
                __syncwarp();
            };
            auto leave = [&](int q, uint64_t salt) {
                const int s = q % Lo.ws;
                if (slot_alias[s] < 0) {
                    const int word = slot_word[s];
                    T *row = w_in + (size_t) word * ld;
                    const float *src = cur + (size_t) s * ld;
                    for (int qq = lane; qq < n2; qq += 32)
                        S::store2(row, qq, reinterpret_cast<const float2 *>(src)[qq], mix64(salt ^ ((uint64_t) word << 20 | qq)));
                    if (lane == 0) {
                        for (int i = kPrefetch - 1; i > 0; i--) recent_exit[i] = recent_exit[i - 1];
                        recent_exit[0] = word;
                    }
                }
                __syncwarp();  // orders this write-back before any lane's later read of the row
                if (lane == 0) {
                    slot_word[s] = -1;
                    slot_alias[s] = -1;
                }
                __syncwarp();
            };
            auto issue = [&](int qi, int qt) {  // prefetch W_in row of position qi, W_out row of target qt
                if (qi < L) {
                    const T *src = w_in + (size_t) __ldg(sen + qi) * ld;
                    unsigned char *dst = BF16 ? reinterpret_cast<unsigned char *>(raw + (size_t) (qi % kRing) * ld)
                                              : reinterpret_cast<unsigned char *>(cur + (size_t) (qi % Lo.ws) * ld);
                    for (int m = lane; m < row_chunks; m += 32)
                        cp_async16(dst + 16 * (size_t) m, reinterpret_cast<const unsigned char *>(src) + 16 * (size_t) m);
                }
                if (qt < L) {
                    const T *src = w_out + (size_t) __ldg(sen + qt) * ld;
                    unsigned char *dst = reinterpret_cast<unsigned char *>(tgt + (size_t) (qt % kRing) * ld);
                    for (int m = lane; m < row_chunks; m += 32)
                        cp_async16(dst + 16 * (size_t) m, reinterpret_cast<const unsigned char *>(src) + 16 * (size_t) m);
                }
                cp_async_commit();
            };

            // ---- attraction ----
            for (int i = lane; i < Lo.ws; i += 32) {
                slot_word[i] = -1;
                slot_alias[i] = -1;
            }
            if (lane < kPrefetch) recent_exit[lane] = -1;
            __syncwarp();
            const int pro = min(w, L);
            for (int q = 0; q < pro; q++) enter(q, 0, false, nullptr);  // synchronous loads
            for (int s = 0; s < kPrefetch; s++) issue(w + s, s);
            Row<NV2> y;
            int prev_t = -1, prev2_t = -1;
            for (int p = 0; p < L; p++) {
                if (p - w - 1 >= 0) leave(p - w - 1, rng ^ (uint64_t) p);
                issue(p + w + kPrefetch, p + kPrefetch);
                cp_async_wait_prefetch();
                __syncwarp();
                const int qn = p + w;
                if (qn < L && qn >= pro)
                    enter(qn, max(0, p - w), !BF16, BF16 ? raw + (size_t) (qn % kRing) * ld : nullptr);
                // target row into registers
                const int t = __ldg(sen + p);
                if (t != prev_t) {
                    const T *src = (t == prev2_t) ? w_out + (size_t) t * ld : tgt + (size_t) (p % kRing) * ld;
#pragma unroll
                    for (int i = 0; i < NV2; i++) {
                        const int qq = lane + 32 * i;
                        y.v[i] = qq < n2 ? S::load2(src, qq) : make_float2(0.f, 0.f);
                    }
                }
                rng = lcg_next(rng);
                const int b = (int) (rng % (uint64_t) w);
                for (int i = b; i < 2 * w + 1 - b; i++) {
                    if (i == w) continue;
                    const int c = p - w + i;
                    if (c < 0) continue;
                    if (c >= L) break;
                    float2 *x = reinterpret_cast<float2 *>(cur + (size_t) slot_of(c) * ld);
                    Row<NV2> xr;
                    float f = 0.f;
#pragma unroll
                    for (int k = 0; k < NV2; k++) {
                        const int qq = lane + 32 * k;
                        xr.v[k] = qq < n2 ? x[qq] : make_float2(0.f, 0.f);
                        f = fmaf(xr.v[k].x, y.v[k].x, fmaf(xr.v[k].y, y.v[k].y, f));
                    }
                    f = warp_sum(f);
                    const float g = grad_from_table(f, 1, alpha, s_exp);
#pragma unroll
                    for (int k = 0; k < NV2; k++) {
                        const int qq = lane + 32 * k;
                        const float2 xv = xr.v[k], yv = y.v[k];
                        y.v[k] = make_float2(fmaf(g, xv.x, yv.x), fmaf(g, xv.y, yv.y));
                        if (qq < n2) x[qq] = make_float2(fmaf(g, yv.x, xv.x), fmaf(g, yv.y, xv.y));
                    }
                    st_pairs++;
                }
                // target write-back
                T *trow = w_out + (size_t) t * ld;
                const uint64_t h0 = mix64(rng ^ ((uint64_t) t << 21));
#pragma unroll
                for (int i = 0; i < NV2; i++) {
                    const int qq = lane + 32 * i;
                    if (qq < n2) S::store2(trow, qq, y.v[i], mix64(h0 + (uint64_t) qq));
                }
                prev2_t = prev_t;
                prev_t = t;
                __syncwarp();
            }
            for (int q = max(0, L - w - 1); q < L; q++) leave(q, rng ^ (uint64_t) (q + 7919));
            cp_async_wait_all();
            __threadfence_block();
            __syncwarp();

            // ---- repulsion (:571-679) ----
            const int num_batch = (L + B - 1) / B;
            const int stride = Lo.ch + 4;
            float *s_in = stage;                         // rows x stride
            float *s_out = stage + (size_t) B * stride;  // K x stride
            for (int nb = 0; nb < num_batch && !failed; nb++) {
                const int lo_b = nb * B;
                const int rows = min(B, L - lo_b);
                rng = lcg_next(rng);
                const int rep_b = (lo_b <= w - 1 || (L - 1) - lo_b <= w - 1) ? (int) (rng % (uint64_t) w)
                                                                              : (int) (rng % (uint64_t) (2 * w));
                const int K = rep_b * a.negative;
                if (!warp_draw_negatives(a.table, a.vocab, rng, sen, L, K, negs, lane, a.max_resample)) {
                    failed = true;  // unresolved negatives: leave the batch untouched
                    break;
                }
                st_batches++;
                st_negs += K;
                for (int e = lane; e < K * rows; e += 32) G[e] = 0.f;
                __syncwarp();
                const int c4 = Lo.ch / 4;
                auto stage_chunk = [&](int col0) {
                    const int ncol4 = min(c4, (ld - col0 + 3) / 4);
                    for (int it = lane; it < (rows + K) * c4; it += 32) {
                        const int rr = it / c4, j4 = it - rr * c4;
                        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (j4 < ncol4) {
                            const T *src = rr < rows ? w_in + (size_t) __ldg(sen + lo_b + rr) * ld
                                                     : w_out + (size_t) negs[rr - rows] * ld;
                            v = S::load4(src + col0, j4);
                        }
                        float *dst = rr < rows ? s_in + (size_t) rr * stride : s_out + (size_t) (rr - rows) * stride;
                        reinterpret_cast<float4 *>(dst)[j4] = v;
                    }
                    __syncwarp();
                };
                // pass 1: G[k][r] = M_out[k] . M_in[r], chunk by chunk
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
                // merge duplicate negatives / rows so that each distinct row is written once
                for (int k = lane; k < K; k += 32) {
                    int first = -1;
                    for (int q = 0; q < k && first < 0; q++)
                        if (negs[q] == negs[k]) first = q;
                    dup[k] = first;
                }
                for (int r = lane; r < rows; r += 32) {
                    int first = -1;
                    const int wr = __ldg(sen + lo_b + r);
                    for (int q = 0; q < r && first < 0; q++)
                        if (__ldg(sen + lo_b + q) == wr) first = q;
                    dup[K + r] = first;
                }
                __syncwarp();
                for (int r = 0; r < rows; r++) {
                    const int f = dup[K + r];
                    if (f >= 0)
                        for (int k = lane; k < K; k += 32) {
                            G[k * rows + f] += G[k * rows + r];
                            G[k * rows + r] = 0.f;
                        }
                    __syncwarp();
                }
                for (int k = 0; k < K; k++) {
                    const int f = dup[k];
                    if (f >= 0)
                        for (int r = lane; r < rows; r += 32) {
                            G[f * rows + r] += G[k * rows + r];
                            G[k * rows + r] = 0.f;
                        }
                    __syncwarp();
                }
                // pass 2: new rows, chunk by chunk, from freshly staged values
                const uint64_t salt = mix64(rng ^ 0x9E3779B97F4A7C15ULL);
                for (int col0 = 0; col0 < ld; col0 += Lo.ch) {
                    stage_chunk(col0);
                    const int ncol4 = min(c4, (ld - col0 + 3) / 4);
                    for (int it = lane; it < K * ncol4; it += 32) {
                        const int k = it / ncol4, j4 = it - k * ncol4;
                        if (dup[k] >= 0) continue;
                        float4 acc = reinterpret_cast<const float4 *>(s_out + (size_t) k * stride)[j4];
                        for (int r = 0; r < rows; r++) {
                            const float gk = G[k * rows + r];
                            const float4 v = reinterpret_cast<const float4 *>(s_in + (size_t) r * stride)[j4];
                            acc = make_float4(fmaf(gk, v.x, acc.x), fmaf(gk, v.y, acc.y), fmaf(gk, v.z, acc.z),
                                              fmaf(gk, v.w, acc.w));
                        }
                        S::store4(w_out + (size_t) negs[k] * ld + col0, j4, acc,
                                  mix64(salt ^ ((uint64_t) negs[k] << 20) ^ (uint64_t) (col0 + 4 * j4)));
                    }
                    for (int it = lane; it < rows * ncol4; it += 32) {
                        const int r = it / ncol4, j4 = it - r * ncol4;
                        if (dup[K + r] >= 0) continue;
                        float4 acc = reinterpret_cast<const float4 *>(s_in + (size_t) r * stride)[j4];
                        for (int k = 0; k < K; k++) {
                            const float gk = G[k * rows + r];
                            const float4 v = reinterpret_cast<const float4 *>(s_out + (size_t) k * stride)[j4];
                            acc = make_float4(fmaf(gk, v.x, acc.x), fmaf(gk, v.y, acc.y), fmaf(gk, v.z, acc.z),
                                              fmaf(gk, v.w, acc.w));
                        }
                        const int word = __ldg(sen + lo_b + r);
                        S::store4(w_in + (size_t) word * ld + col0, j4, acc,
                                  mix64(salt ^ ((uint64_t) word << 21) ^ (uint64_t) (col0 + 4 * j4) ^ 1ULL));
                    }
                    __syncwarp();
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
        if (failed) atomicOr(&a.cnt->error, kErrResample);
    }
}

template <int NV2, bool BF16>
cudaError_t launch_nv(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    const Layout Lo = make_layout(a.ld, a.window, a.negative, a.batch, BF16);
    const size_t smem = up16(1004 * sizeof(float)) + (size_t) warps * Lo.per_warp;
    cudaError_t e = cudaFuncSetAttribute(k_batched_train<NV2, BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) smem);
    if (e != cudaSuccess) return e;
    k_batched_train<NV2, BF16><<<grid, warps * 32, smem, s>>>(a, warps);
    return cudaGetLastError();
}

template <bool BF16>
cudaError_t launch_mode(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    switch ((a.d + 63) / 64) {
        case 1: return launch_nv<1, BF16>(a, grid, warps, s);
        case 2: return launch_nv<2, BF16>(a, grid, warps, s);
        case 3: return launch_nv<3, BF16>(a, grid, warps, s);
        case 4: return launch_nv<4, BF16>(a, grid, warps, s);
        case 5: return launch_nv<5, BF16>(a, grid, warps, s);
        case 6: return launch_nv<6, BF16>(a, grid, warps, s);
        case 7: return launch_nv<7, BF16>(a, grid, warps, s);
        case 8: return launch_nv<8, BF16>(a, grid, warps, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int batched_max_warps(int ld, int window, int negative, int batch, bool bf16, size_t *per_warp) {
    const Layout Lo = make_layout(ld, window, negative, batch, bf16);
    if (per_warp) *per_warp = Lo.per_warp;
    const size_t avail = kSmemBudget - up16(1004 * sizeof(float));
    long w = (long) (avail / Lo.per_warp);
    if (w > kMaxWarpsB) w = kMaxWarpsB;
    return (int) w;
}

cudaError_t launch_batched_train(const TrainArgs &a, bool bf16, int grid, int warps_per_cta, cudaStream_t s) {
    return bf16 ? launch_mode<true>(a, grid, warps_per_cta, s) : launch_mode<false>(a, grid, warps_per_cta, s);
}

}  // namespace parw2v
