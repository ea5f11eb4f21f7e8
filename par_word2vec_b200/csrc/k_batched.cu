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
#include "common.cuh"
#include "internal.h"
#include "mma.cuh"
#include "sentence.cuh"

namespace parw2v {

namespace {

constexpr int kPrefetch = 2;                  // P: positions prefetched ahead
constexpr int kRing = kPrefetch + 1;          // landing buffers for targets / BF16 rows
constexpr int kMaxWarpsB = 16;
constexpr size_t kSmemBudget = 227 * 1024;

// Tensor-core repulsion (BF16 mode): shapes and staging geometry
constexpr int kMmaK = 48;        // negatives per batch handled by the mma path (3 m-tiles)
constexpr int kMmaR = 32;        // batch rows handled by the mma path (2 m-tiles / 4 n-tiles)
// The column chunk is narrow on purpose: shared memory and L1 are one 256 KB array per SM, and
// every byte of staging taken from it is a byte of L1 the streamed kernel's row reuse loses.
constexpr int kMmaCols = 32;     // column chunk of the staging
constexpr int kMmaStride = 40;   // staged row stride in bf16 (80 B: conflict-free ldmatrix rows)
constexpr int kGbStride = 40;    // bf16 G row stride (80 B)
__host__ __device__ constexpr size_t up16_c(size_t x) { return (x + 15) & ~(size_t) 15; }
// FP32 tables on the tensor cores (3xTF32): the same staging bytes hold 16 FP32 columns
constexpr int kF32Cols = 16;     // column chunk of the FP32 staging
constexpr int kF32Stride = 20;   // staged FP32 row stride in floats (80 B: conflict-free ldmatrix rows)
constexpr int kGps = 36;         // FP32 G row stride in floats (144 B: conflict-free ldmatrix rows)
static_assert(kF32Stride * 4 == kMmaStride * 2, "FP32 and BF16 staging rows take the same bytes");

__host__ __device__ inline bool mma_path(int kmax_eff, int batch) { return kmax_eff <= kMmaK && batch <= kMmaR; }
__host__ __device__ inline size_t mma_g_bytes(bool bf16) {  // G kept through pass 2
    return bf16 ? up16_c((size_t) kMmaK * kGbStride * 2) : up16_c((size_t) kMmaK * kGps * 4);
}

struct Layout {  // per-warp shared-memory carve-up, in bytes (all offsets 16-byte aligned)
    int ws;            // window slots 2w+1+P
    int ch;            // repulsion column chunk (multiple of 4), SIMT path
    int kmax;          // 2 * window * negative
    bool mma;          // tensor-core repulsion
    size_t region;     // window cur rows (+ BF16 landing ring) | repulsion staging
    size_t raw_off;    // BF16 landing ring inside the region
    size_t gb_off;     // mma path: bf16 G inside the region, after the staged chunk
    size_t tgt_off, g_off, neg_off, dup_off, meta_off, ctx_off, exit_off, per_warp;
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
    // the column chunk: as wide as fits in the window's bytes, at least 16 columns
    const size_t rows_rep = (size_t) (batch + L.kmax);
    long ch = (long) (win_total / (rows_rep * 4)) - 4;
    ch = ch / 4 * 4;
    if (ch > ((ld + 3) / 4) * 4) ch = ((ld + 3) / 4) * 4;
    if (ch < 16) ch = 16;
    L.ch = (int) ch;
    L.mma = mma_path((2 * window - 1) * negative, batch);
    size_t rep_bytes = up16(rows_rep * (size_t) (L.ch + 4) * 4);
    L.gb_off = 0;
    if (L.mma) {
        const size_t stage = up16((size_t) (kMmaR + kMmaK) * kMmaStride * 2);
        L.gb_off = stage;
        rep_bytes = stage + mma_g_bytes(bf16);
    }
    L.region = win_total > rep_bytes ? win_total : rep_bytes;
    L.tgt_off = L.region;
    L.g_off = L.tgt_off + up16((size_t) kRing * row_st);
    const size_t g_floats = L.mma ? (size_t) kMmaK * kMmaR : (size_t) L.kmax * batch;
    L.neg_off = L.g_off + up16(g_floats * 4);
    L.dup_off = L.neg_off + up16((size_t) L.kmax * 4);
    L.meta_off = L.dup_off + up16((size_t) (L.kmax + 2 * batch) * 4);
    L.ctx_off = L.meta_off + up16((size_t) L.ws * 8);
    L.exit_off = L.ctx_off + up16((size_t) (2 * window) * 8);
    L.per_warp = L.exit_off + up16((size_t) kPrefetch * 4 + 16);
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


// Repeated words of a batch: dup[k] (negatives) and dup[K + r] (batch rows) get the index of the
// word's first occurrence, or -1.  Generic form (any K, rows).
__device__ __noinline__ void mark_repeats(const int *negs, int K, const int32_t *batch_words, int rows, int *dup,
                                          int lane) {
    for (int k = lane; k < K; k += 32) {
        int first = -1;
        for (int q = 0; q < k && first < 0; q++)
            if (negs[q] == negs[k]) first = q;
        dup[k] = first;
    }
    for (int r = lane; r < rows; r += 32) {
        int first = -1;
        const int wr = __ldg(batch_words + r);
        for (int q = 0; q < r && first < 0; q++)
            if (__ldg(batch_words + q) == wr) first = q;
        dup[K + r] = first;
    }
    __syncwarp();
}

// The same marks for K <= 64 negatives and rows <= 32 (the tensor-core paths), by warp matching:
// lanes holding equal words find each other in one __match_any_sync; negatives 32..63 also look
// through the first 32 by shuffles.  Lanes without a word hold distinct negative sentinels.
__device__ __forceinline__ void mark_repeats_small(const int *negs, int K, const int *words, int rows, int *dup,
                                                   int lane) {
    const int wr = lane < rows ? words[lane] : -1 - lane;
    const unsigned mr = __match_any_sync(0xffffffffu, wr);
    if (lane < rows) dup[K + lane] = (__ffs(mr) - 1 == lane) ? -1 : __ffs(mr) - 1;
    const int v0 = lane < K ? negs[lane] : -1 - lane;
    const unsigned m0 = __match_any_sync(0xffffffffu, v0);
    if (lane < K) dup[lane] = (__ffs(m0) - 1 == lane) ? -1 : __ffs(m0) - 1;
    if (K > 32) {
        const int v1 = lane + 32 < K ? negs[lane + 32] : -100 - lane;
        int first = -1;
        for (int q = 0; q < 32; q++) {
            const int w = __shfl_sync(0xffffffffu, v0, q);
            if (first < 0 && q < K && w == v1) first = q;
        }
        const unsigned m1 = __match_any_sync(0xffffffffu, v1);
        if (first < 0 && __ffs(m1) - 1 != lane) first = 32 + __ffs(m1) - 1;
        if (lane + 32 < K) dup[lane + 32] = first;
    }
    __syncwarp();
}

// Merge the gradient columns of repeated batch rows, then the gradient rows of repeated negatives,
// into their first occurrence (G is K x rows with row stride gs), so each distinct row is written
// once.  Only the marked rows are visited, in ascending order (32 at a time by ballot).
__device__ __noinline__ void merge_marked(int K, int rows, float *G, int gs, const int *dup, int lane) {
    for (int r0 = 0; r0 < rows; r0 += 32) {
        for (unsigned m = __ballot_sync(0xffffffffu, r0 + lane < rows && dup[K + r0 + lane] >= 0); m; m &= m - 1) {
            const int r = r0 + __ffs(m) - 1, f = dup[K + r];
            for (int k = lane; k < K; k += 32) {
                G[k * gs + f] += G[k * gs + r];
                G[k * gs + r] = 0.f;
            }
            __syncwarp();
        }
    }
    for (int k0 = 0; k0 < K; k0 += 32) {
        for (unsigned m = __ballot_sync(0xffffffffu, k0 + lane < K && dup[k0 + lane] >= 0); m; m &= m - 1) {
            const int k = k0 + __ffs(m) - 1, f = dup[k];
            for (int r = lane; r < rows; r += 32) {
                G[f * gs + r] += G[k * gs + r];
                G[k * gs + r] = 0.f;
            }
            __syncwarp();
        }
    }
}

__device__ __forceinline__ void merge_repeats(const int *negs, int K, const int32_t *batch_words, int rows, float *G,
                                              int gs, int *dup, int lane) {
    mark_repeats(negs, K, batch_words, rows, dup, lane);
    merge_marked(K, rows, G, gs, dup, lane);
}

// Repulsion of one batch on the tensor cores (BF16 tables, K <= 48 negatives, rows <= 32).
// Column chunks of M_in (rows) and M_out (negatives) are staged as BF16 with cp.async.
// Pass 1 accumulates G = M_out M_in^T over all chunks in registers (m16n8k16, FP32 accumulate);
// G = alpha * (0 - sigma(G)) through the table, repeated words merged, G rounded to BF16.
// Pass 2 re-stages each chunk, forms M_out + G M_in and M_in + G^T M_out 8 columns at a time,
// rounds them stochastically into the staged tile in place and stores every distinct row's
// 16-byte pieces back to the tables.
__device__ __noinline__ void repel_mma(const TrainArgs &a, const Layout &Lo, unsigned char *base, const int32_t *bw,
                                       int rows, const int *negs, int K, float alpha, const float *s_exp, float *Gf,
                                       int *dup, int lane, LaneBits &rb) {
    using T = __nv_bfloat16;
    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const int ld = a.ld;
    T *sin = reinterpret_cast<T *>(base);                        // kMmaR x kMmaStride
    T *sout = sin + (size_t) kMmaR * kMmaStride;                  // kMmaK x kMmaStride
    T *Gb = reinterpret_cast<T *>(base + Lo.gb_off);              // kMmaK x kGbStride
    const int g = lane >> 2, t = lane & 3;
    const int mt1 = (K + 15) >> 4;        // m-tiles of negatives
    const int nt1 = (rows + 7) >> 3;      // n-tiles of batch rows (pass 1)
    const int kr = (rows + 15) >> 4;      // 16-row steps of the batch (pass 2)
    constexpr int kPieces = kMmaCols / 8; // 16-byte pieces per staged row
    float acc[3][4][4];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[i][j][e] = 0.f;
    // the batch's words, read once: the staging and write-back loops index them per piece
    int *sbw = dup + Lo.kmax + a.batch;
    if (lane < rows) sbw[lane] = __ldg(bw + lane);
    __syncwarp();
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        // zero the padding rows the products read (batch rows up to kMmaR, negatives up to the
        // m-tile), columns 0..kMmaCols-1; they stay zero for every chunk of the pass, since the
        // staging writes only the real rows (the FP32 G of pass 1 may share these bytes, see the
        // streamed kernel, so pass 2 zeroes them again)
        const int pad_in = kMmaR - rows, pad_out = 16 * mt1 - K;
        for (int i = lane; i < (pad_in + pad_out) * kPieces; i += 32) {
            const int pr = i / kPieces, q = i - pr * kPieces;
            T *row = pr < pad_in ? sin + (size_t) (rows + pr) * kMmaStride : sout + (size_t) (K + pr - pad_in) * kMmaStride;
            reinterpret_cast<uint4 *>(row)[q] = make_uint4(0, 0, 0, 0);
        }
        __syncwarp();
#pragma unroll 1
        for (int col0 = 0; col0 < ld; col0 += kMmaCols) {
            // stage columns [col0, col0 + kMmaCols) of the batch rows and the negatives' rows
            for (int it = lane; it < (rows + K) * kPieces; it += 32) {
                const int rr = it / kPieces, pc = it - rr * kPieces;
                T *dst = (rr < rows ? sin + (size_t) rr * kMmaStride : sout + (size_t) (rr - rows) * kMmaStride) + pc * 8;
                const int col = col0 + pc * 8;
                if (col < ld) {
                    const T *src = (rr < rows ? w_in + (size_t) sbw[rr] * ld : w_out + (size_t) negs[rr - rows] * ld) + col;
                    cp_async16(dst, src);
                } else {
                    *reinterpret_cast<uint4 *>(dst) = make_uint4(0, 0, 0, 0);
                }
            }
            cp_async_commit();
            cp_async_wait_all();
            __syncwarp();
            if (pass == 0) {
#pragma unroll 1
                for (int ks = 0; ks < kMmaCols / 16; ks++) {
                    unsigned bfr[4][2];
#pragma unroll
                    for (int np = 0; np < 2; np++) {  // n-tiles 2np, 2np+1 in one ldmatrix.x4
                        unsigned r[4];
                        const int n = np * 16 + (lane & 7) + ((lane >> 4) << 3);
                        ldsm_x4(r, sin + (size_t) n * kMmaStride + ks * 16 + ((lane >> 3) & 1) * 8);
                        bfr[2 * np][0] = r[0];
                        bfr[2 * np][1] = r[1];
                        bfr[2 * np + 1][0] = r[2];
                        bfr[2 * np + 1][1] = r[3];
                    }
#pragma unroll
                    for (int mt = 0; mt < 3; mt++)
                        if (mt < mt1) {
                            unsigned af[4];
                            ldsm_x4(af, sout + (size_t) (mt * 16 + (lane & 15)) * kMmaStride + ks * 16 + (lane >> 4) * 8);
#pragma unroll
                            for (int nt = 0; nt < 4; nt++)
                                if (nt < nt1) mma16816(acc[mt][nt], af, bfr[nt][0], bfr[nt][1]);
                        }
                }
            } else {
                const int ncols = min(kMmaCols, ld - col0);
#pragma unroll 1
                for (int nt = 0; nt < ncols / 8; nt++) {
                    float o[3][4], q[2][4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        o[0][e] = o[1][e] = o[2][e] = 0.f;
                        q[0][e] = q[1][e] = 0.f;
                    }
                    // M_out update: G (K x rows) . M_in (rows x 8 columns)
#pragma unroll 1
                    for (int ks = 0; ks < kr; ks++) {
                        unsigned b[2];
                        ldsm_x2_t(b, sin + (size_t) (ks * 16 + (lane & 15)) * kMmaStride + nt * 8);
#pragma unroll
                        for (int mt = 0; mt < 3; mt++)
                            if (mt < mt1) {
                                unsigned af[4];
                                ldsm_x4(af, Gb + (size_t) (mt * 16 + (lane & 15)) * kGbStride + ks * 16 + (lane >> 4) * 8);
                                mma16816(o[mt], af, b[0], b[1]);
                            }
                    }
                    // M_in update: G^T (rows x K) . M_out (K x 8 columns)
#pragma unroll 1
                    for (int ks = 0; ks < mt1; ks++) {
                        unsigned b[2];
                        ldsm_x2_t(b, sout + (size_t) (ks * 16 + (lane & 15)) * kMmaStride + nt * 8);
#pragma unroll
                        for (int mt = 0; mt < 2; mt++)
                            if (mt < kr) {
                                unsigned af[4];
                                ldsm_x4_t(af, Gb + (size_t) (ks * 16 + ((lane >> 4) << 3) + (lane & 7)) * kGbStride +
                                                  mt * 16 + ((lane >> 3) & 1) * 8);
                                mma16816(q[mt], af, b[0], b[1]);
                            }
                    }
                    // new values = staged + update, rounded stochastically, in place
                    const int j = nt * 8 + 2 * t;
#pragma unroll
                    for (int mt = 0; mt < 3; mt++)
                        if (mt < mt1) {
                            const uint64_t bits = rb.next();
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                __nv_bfloat162 *cell = reinterpret_cast<__nv_bfloat162 *>(sout + (size_t) (mt * 16 + g + 8 * h) * kMmaStride + j);
                                const float2 old = __bfloat1622float2(*cell);
                                *reinterpret_cast<unsigned *>(cell) =
                                    pack_sr2(make_float2(old.x + o[mt][2 * h], old.y + o[mt][2 * h + 1]), bits >> (32 * h));
                            }
                        }
#pragma unroll
                    for (int mt = 0; mt < 2; mt++)
                        if (mt < kr) {
                            const uint64_t bits = rb.next();
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                __nv_bfloat162 *cell = reinterpret_cast<__nv_bfloat162 *>(sin + (size_t) (mt * 16 + g + 8 * h) * kMmaStride + j);
                                const float2 old = __bfloat1622float2(*cell);
                                *reinterpret_cast<unsigned *>(cell) =
                                    pack_sr2(make_float2(old.x + q[mt][2 * h], old.y + q[mt][2 * h + 1]), bits >> (32 * h));
                            }
                        }
                }
                __syncwarp();
                // each distinct row's new chunk back to its table in 16-byte pieces
                for (int it = lane; it < (rows + K) * kPieces; it += 32) {
                    const int rr = it / kPieces, pc = it - rr * kPieces;
                    const int col = col0 + pc * 8;
                    if (col >= ld || dup[rr < rows ? K + rr : rr - rows] >= 0) continue;
                    const T *src = (rr < rows ? sin + (size_t) rr * kMmaStride : sout + (size_t) (rr - rows) * kMmaStride) + pc * 8;
                    T *dst = (rr < rows ? w_in + (size_t) sbw[rr] * ld : w_out + (size_t) negs[rr - rows] * ld) + col;
                    *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(src);
                }
            }
            __syncwarp();
        }
        if (pass == 0) {
            // raw dot products into Gf (kMmaK x kMmaR), sigma / label 0, merge repeats, BF16 copy
#pragma unroll
            for (int mt = 0; mt < 3; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (mt < mt1 && nt < nt1) {
                            const int k = mt * 16 + g + ((e >> 1) << 3), r = nt * 8 + 2 * t + (e & 1);
                            if (k < K && r < rows) Gf[k * kMmaR + r] = grad_from_table(acc[mt][nt][e], 0, alpha, s_exp);
                        }
            mark_repeats_small(negs, K, sbw, rows, dup, lane);
            merge_marked(K, rows, Gf, kMmaR, dup, lane);
            // BF16 G over the part pass 2 reads: negatives below 16 * mt1, batch rows below 16 * kr
            const int sh = kr == 1 ? 3 : 4;  // column pairs per row: 8 * kr
            for (int i = lane; i < (16 * mt1) << sh; i += 32) {
                const int k = i >> sh, r = 2 * (i & ((1 << sh) - 1));
                const float v0 = (k < K && r < rows) ? Gf[k * kMmaR + r] : 0.f;
                const float v1 = (k < K && r + 1 < rows) ? Gf[k * kMmaR + r + 1] : 0.f;
                reinterpret_cast<__nv_bfloat162 *>(Gb + (size_t) k * kGbStride)[r >> 1] = __floats2bfloat162_rn(v0, v1);
            }
            __syncwarp();
        }
    }
}

// Repulsion of one batch on the tensor cores with FP32 tables (K <= 48 negatives, rows <= 32): the
// structure of repel_mma with FP32 staging (16-column chunks) and 3xTF32 products, so the FP32 mode
// keeps FP32-level arithmetic.  G stays FP32 through pass 2 (kMmaK x kGps floats), and the new
// values (staged value + update) go from the accumulators straight to the rows.
__device__ __noinline__ void repel_mma_f32(const TrainArgs &a, const Layout &Lo, unsigned char *base, const int32_t *bw,
                                           int rows, const int *negs, int K, float alpha, const float *s_exp, float *Gf,
                                           int *dup, int lane) {
    float *w_in = static_cast<float *>(a.w_in);
    float *w_out = static_cast<float *>(a.w_out);
    const int ld = a.ld;
    float *sin = reinterpret_cast<float *>(base);             // kMmaR x kF32Stride
    float *sout = sin + (size_t) kMmaR * kF32Stride;          // kMmaK x kF32Stride
    float *Gp = reinterpret_cast<float *>(base + Lo.gb_off);  // kMmaK x kGps
    const int g = lane >> 2, t = lane & 3;
    const int mt1 = (K + 15) >> 4;  // m-tiles of negatives
    const int nt1 = (rows + 7) >> 3;  // n-tiles of batch rows (pass 1)
    const int kr8 = (rows + 7) >> 3;  // 8-row k-steps over the batch rows
    const int kk8 = (K + 7) >> 3;     // 8-row k-steps over the negatives
    const int mr = (rows + 15) >> 4;  // m-tiles of batch rows (pass 2)
    constexpr int kPieces = kF32Cols / 4;  // 16-byte pieces per staged row
    float acc[3][4][4];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[i][j][e] = 0.f;
    // the batch's words, read once: the staging and write-back loops index them per piece
    int *sbw = dup + Lo.kmax + a.batch;
    if (lane < rows) sbw[lane] = __ldg(bw + lane);
    __syncwarp();
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        // zero the staging: padding rows stay zero for every chunk of the pass
        for (int i = lane; i < (kMmaR + kMmaK) * kF32Stride / 4; i += 32)
            reinterpret_cast<float4 *>(sin)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
#pragma unroll 1
        for (int col0 = 0; col0 < ld; col0 += kF32Cols) {
            for (int it = lane; it < (rows + K) * kPieces; it += 32) {
                const int rr = it / kPieces, pc = it - rr * kPieces;
                float *dst = (rr < rows ? sin + (size_t) rr * kF32Stride : sout + (size_t) (rr - rows) * kF32Stride) + pc * 4;
                const int col = col0 + pc * 4;
                if (col < ld) {
                    const float *src = (rr < rows ? w_in + (size_t) sbw[rr] * ld : w_out + (size_t) negs[rr - rows] * ld) + col;
                    cp_async16(dst, src);
                } else {
                    *reinterpret_cast<float4 *>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            cp_async_commit();
            cp_async_wait_all();
            __syncwarp();
            if (pass == 0) {
                // S += M_out . M_in^T over these 16 columns: two k-steps of 8
#pragma unroll 1
                for (int ks = 0; ks < kF32Cols / 8; ks++) {
                    unsigned bb[4][2], bs[4][2];
#pragma unroll
                    for (int np = 0; np < 2; np++) {  // n-tiles 2np, 2np+1 in one ldmatrix.x4
                        float r[4];
                        const int n = np * 16 + (lane & 7) + ((lane >> 4) << 3);
                        ldsm_x4_f32(r, sin + (size_t) n * kF32Stride + ks * 8 + ((lane >> 3) & 1) * 4);
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            split_tf32(r[2 * h], bb[2 * np + h][0], bs[2 * np + h][0]);
                            split_tf32(r[2 * h + 1], bb[2 * np + h][1], bs[2 * np + h][1]);
                        }
                    }
#pragma unroll
                    for (int mt = 0; mt < 3; mt++)
                        if (mt < mt1) {
                            float af[4];
                            ldsm_x4_f32(af, sout + (size_t) (mt * 16 + (lane & 7) + ((lane >> 3) & 1) * 8) * kF32Stride + ks * 8 +
                                                (lane >> 4) * 4);
                            unsigned ab[4], as[4];
                            split_a(af, ab, as);
#pragma unroll
                            for (int nt = 0; nt < 4; nt++)
                                if (nt < nt1) mma3xtf32(acc[mt][nt], ab, as, bb[nt], bs[nt]);
                        }
                }
            } else {
#pragma unroll 1
                for (int nt = 0; nt < kF32Cols / 8; nt++) {
                    const int cb = nt * 8;
                    if (col0 + cb >= ld) break;
                    float o[3][4], q[2][4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        o[0][e] = o[1][e] = o[2][e] = 0.f;
                        q[0][e] = q[1][e] = 0.f;
                    }
                    // M_out update: G (K x rows) . M_in (rows x 8 columns)
#pragma unroll 1
                    for (int ks = 0; ks < kr8; ks++) {
                        unsigned bb[2], bs[2];
                        split_tf32(sin[(size_t) (ks * 8 + t) * kF32Stride + cb + g], bb[0], bs[0]);
                        split_tf32(sin[(size_t) (ks * 8 + t + 4) * kF32Stride + cb + g], bb[1], bs[1]);
#pragma unroll
                        for (int mt = 0; mt < 3; mt++)
                            if (mt < mt1) {
                                float af[4];
                                ldsm_x4_f32(af, Gp + (size_t) (mt * 16 + (lane & 7) + ((lane >> 3) & 1) * 8) * kGps + ks * 8 +
                                                    (lane >> 4) * 4);
                                unsigned ab[4], as[4];
                                split_a(af, ab, as);
                                mma3xtf32(o[mt], ab, as, bb, bs);
                            }
                    }
                    // M_in update: G^T (rows x K) . M_out (K x 8 columns)
#pragma unroll 1
                    for (int ks = 0; ks < kk8; ks++) {
                        unsigned bb[2], bs[2];
                        split_tf32(sout[(size_t) (ks * 8 + t) * kF32Stride + cb + g], bb[0], bs[0]);
                        split_tf32(sout[(size_t) (ks * 8 + t + 4) * kF32Stride + cb + g], bb[1], bs[1]);
#pragma unroll
                        for (int mt = 0; mt < 2; mt++)
                            if (mt < mr) {
                                const float *gk = Gp + (size_t) (ks * 8 + t) * kGps + mt * 16 + g;
                                const float af[4] = {gk[0], gk[8], gk[4 * kGps], gk[4 * kGps + 8]};
                                unsigned ab[4], as[4];
                                split_a(af, ab, as);
                                mma3xtf32(q[mt], ab, as, bb, bs);
                            }
                    }
                    // staged value + update, straight to the rows (each distinct word once)
                    const int c = cb + 2 * t;
                    if (col0 + c < ld) {
#pragma unroll
                        for (int mt = 0; mt < 3; mt++)
                            if (mt < mt1)
#pragma unroll
                                for (int h = 0; h < 2; h++) {
                                    const int row = mt * 16 + g + 8 * h;
                                    if (row < K && dup[row] < 0) {
                                        const float2 old = *reinterpret_cast<const float2 *>(sout + (size_t) row * kF32Stride + c);
                                        *reinterpret_cast<float2 *>(w_out + (size_t) negs[row] * ld + col0 + c) =
                                            make_float2(old.x + o[mt][2 * h], old.y + o[mt][2 * h + 1]);
                                    }
                                }
#pragma unroll
                        for (int mt = 0; mt < 2; mt++)
                            if (mt < mr)
#pragma unroll
                                for (int h = 0; h < 2; h++) {
                                    const int row = mt * 16 + g + 8 * h;
                                    if (row < rows && dup[K + row] < 0) {
                                        const float2 old = *reinterpret_cast<const float2 *>(sin + (size_t) row * kF32Stride + c);
                                        *reinterpret_cast<float2 *>(w_in + (size_t) sbw[row] * ld + col0 + c) =
                                            make_float2(old.x + q[mt][2 * h], old.y + q[mt][2 * h + 1]);
                                    }
                                }
                    }
                }
            }
            __syncwarp();
        }
        if (pass == 0) {
            // raw dot products into Gf (kMmaK x kMmaR), sigma / label 0, merge repeats, then the FP32
            // copy that pass 2 reads (zero outside K x rows)
#pragma unroll
            for (int mt = 0; mt < 3; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (mt < mt1 && nt < nt1) {
                            const int k = mt * 16 + g + ((e >> 1) << 3), r = nt * 8 + 2 * t + (e & 1);
                            if (k < K && r < rows) Gf[k * kMmaR + r] = grad_from_table(acc[mt][nt][e], 0, alpha, s_exp);
                        }
            mark_repeats_small(negs, K, sbw, rows, dup, lane);
            merge_marked(K, rows, Gf, kMmaR, dup, lane);
            for (int i = lane; i < kMmaK * kMmaR; i += 32) {
                const int k = i / kMmaR, r = i - k * kMmaR;
                Gp[(size_t) k * kGps + r] = (k < K && r < rows) ? Gf[i] : 0.f;
            }
            __syncwarp();
        }
    }
}

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
    merge_repeats(negs, K, bw, rows, G, rows, dup, lane);
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

    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const uint64_t n_lines = a.cnt->n_lines, total_kept = a.cnt->total_kept;
    const int epoch = hogwild_epoch(a);
    const int row_chunks = ld / S::kChunkElems;  // 16-byte pieces per stored row
    const bool use_mma = Lo.mma;
    // c mod ws for positions c < 2^16 by a multiply-high reciprocal (exact: ws <= 256)
    const unsigned ws_u = (unsigned) Lo.ws, ws_m = (unsigned) (0xFFFFFFFFULL / ws_u) + 1u;
    auto ring = [&](int c) { return (int) ((unsigned) c - __umulhi((unsigned) c, ws_m) * ws_u); };
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
                    break;
                }
                st_batches++;
                st_negs += K;
                if (K > 0) {
                    if constexpr (BF16) {
                        if (use_mma)
                            repel_mma(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
                        else
                            repel_simt<true>(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
                    } else {
                        if (use_mma)
                            repel_mma_f32(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane);
                        else
                            repel_simt<false>(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
                    }
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
constexpr size_t kStreamStage = (size_t) (kMmaR + kMmaK) * kMmaStride * 2;  // 6,400 bytes
static_assert(kStreamStage >= (size_t) kMmaK * kMmaR * 4, "the FP32 G of pass 1 shares the staging bytes");

__host__ __device__ inline Layout make_layout_stream(int ld, int window, int negative, int batch, bool bf16) {
    Layout L;
    L.ws = 0;
    L.kmax = 2 * window * negative;
    L.mma = mma_path((2 * window - 1) * negative, batch);
    L.raw_off = 0;
    L.tgt_off = 0;
    L.meta_off = 0;
    const size_t rows_rep = (size_t) (batch + L.kmax);
    long ch = (long) (kStreamStage / (rows_rep * 4)) - 4;
    ch = ch / 4 * 4;
    if (ch > ((ld + 3) / 4) * 4) ch = ((ld + 3) / 4) * 4;
    if (ch < 16) ch = 16;
    L.ch = (int) ch;
    if (L.mma) {
        L.gb_off = kStreamStage;
        L.region = kStreamStage + mma_g_bytes(bf16);
        L.g_off = 0;  // the FP32 G of pass 1 shares the staging bytes
    } else {
        L.gb_off = 0;
        L.region = up16(rows_rep * (size_t) (L.ch + 4) * 4);
        L.g_off = L.region;
    }
    const size_t g_bytes = L.mma ? 0 : up16((size_t) L.kmax * batch * 4);
    L.neg_off = L.region + g_bytes;
    L.dup_off = L.neg_off + up16((size_t) L.kmax * 4);
    L.ctx_off = L.dup_off + up16((size_t) (L.kmax + 2 * batch) * 4);
    L.exit_off = L.ctx_off + up16((size_t) (2 * window) * 8);
    L.per_warp = L.exit_off + up16(kStreamStats * sizeof(unsigned long long));  // the warp's statistics
    return L;
}

template <int NV4, bool BF16, bool SYNC>
__global__ void __launch_bounds__(kMaxWarpsS * 32, 1) k_stream_train(TrainArgs a, int warps) {
    using S = Store<BF16>;
    using T = typename S::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = a.window, B = a.batch, ld = a.ld, d = a.d;
    const FastMod mod_w((uint32_t) w);
    const int n4 = (d + 3) >> 2;
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
    T *w_in = static_cast<T *>(a.w_in);
    T *w_out = static_cast<T *>(a.w_out);
    const int epoch = hogwild_epoch(a);
    bool failed = false;

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
            // it across positions measured 5% slower: there a position reads its first row itself.
            typename S::Raw yn[NV4];
            {
                const T *yrow0 = w_out + (size_t) __ldg(sen) * ld;
#pragma unroll
                for (int k = 0; k < NV4; k++) yn[k] = lane + 32 * k < n4 ? S::loadraw_g(yrow0, lane + 32 * k) : S::zero_raw();
            }
            rng = lcg_next(rng);
            int b_next = (int) mod_w(rng);
            typename S::Raw xn[NV4];
            int c_next = 1, w_next = 0;  // position 0's first context is position 1 (its window starts at 0)
            if constexpr (!SYNC && BF16) {
                if (L > 1) {
                    w_next = __ldg(sen + 1);
                    const T *xrow0 = w_in + (size_t) w_next * ld;
#pragma unroll
                    for (int k = 0; k < NV4; k++) xn[k] = lane + 32 * k < n4 ? S::loadraw_g(xrow0, lane + 32 * k) : S::zero_raw();
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
                Row<NV4> y;
#pragma unroll
                for (int k = 0; k < NV4; k++) y.v[k] = S::widen(yn[k]);
                const int t_next = p + 1 < L ? __ldg(sen + p + 1) : t;
                if (t_next != t) {
                    const T *ynrow = w_out + (size_t) t_next * ld;
#pragma unroll
                    for (int k = 0; k < NV4; k++) yn[k] = lane + 32 * k < n4 ? S::loadraw_g(ynrow, lane + 32 * k) : S::zero_raw();
                }
                const int lo_c = max(p - w + b, 0), hi_c = min(p + w - b, L - 1);
                const int n = hi_c - lo_c;
                if constexpr (SYNC) {
                    for (int i0 = 0; i0 < n; i0 += 2) {
                        float f[2] = {0.f, 0.f};
                        int wd[2] = {-1, -1};
#pragma unroll
                        for (int u = 0; u < 2; u++)
                            if (i0 + u < n) {
                                const int c = lo_c + i0 + u + (lo_c + i0 + u >= p ? 1 : 0);
                                wd[u] = __ldg(sen + c);
                                const T *x = w_in + (size_t) wd[u] * ld;
#pragma unroll
                                for (int k = 0; k < NV4; k++) {
                                    const int cc = lane + 32 * k;
                                    if (cc < n4) f[u] = f4_dot(S::load4g(x, cc), y.v[k], f[u]);
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
                                    ctx_w[i0 + u] = wd[u];
                                }
                    }
                    __syncwarp();
                    if (lane == 0)
                        for (int i = 1; i < n; i++)
                            for (int k = 0; k < i; k++)
                                if (ctx_w[k] == ctx_w[i]) {
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
                        T *x = w_in + (size_t) ctx_w[i] * ld;
#pragma unroll
                        for (int k = 0; k < NV4; k++) {
                            const int cc = lane + 32 * k;
                            if (cc < n4) {
                                const float4 xv = S::load4g(x, cc);
                                dy.v[k] = f4_fma(g, xv, dy.v[k]);
                                if (g != 0.f) S::store4(x, cc, f4_fma(g, y.v[k], xv), rb.next());
                            }
                        }
                    }
#pragma unroll
                    for (int k = 0; k < NV4; k++)
                        y.v[k] = make_float4(y.v[k].x + dy.v[k].x, y.v[k].y + dy.v[k].y, y.v[k].z + dy.v[k].z,
                                             y.v[k].w + dy.v[k].w);
                } else if (n > 0) {
                    // contexts c in [lo_c, hi_c] without p, in window order; the first one and its
                    // row were read during the previous position (L > 1 gives every position one)
                    int c = c_next;
                    int wc = w_next;
                    if constexpr (!BF16) {
                        c = lo_c == p ? lo_c + 1 : lo_c;
                        wc = __ldg(sen + c);
                        const T *xrow0 = w_in + (size_t) wc * ld;
#pragma unroll
                        for (int k = 0; k < NV4; k++) xn[k] = lane + 32 * k < n4 ? S::loadraw_g(xrow0, lane + 32 * k) : S::zero_raw();
                    }
                    // the next position's first context: its window start, which is below it
                    // (b_next < w), so never the position itself
                    const bool has_next = p + 1 < L;
                    const int c_first_next = max(p + 1 - w + b_next, 0);
                    for (int i = 0; i < n; i++) {
                        const int word = wc;
                        T *x = w_in + (size_t) word * ld;
                        Row<NV4> xr;
                        float f = 0.f;
#pragma unroll
                        for (int k = 0; k < NV4; k++) {
                            xr.v[k] = S::widen(xn[k]);
                            f = f4_dot(xr.v[k], y.v[k], f);
                        }
                        const bool more = i + 1 < n;
                        const bool ahead = more || (BF16 && has_next);
                        if (ahead) {
                            c = more ? (c + 1 == p ? c + 2 : c + 1) : c_first_next;
                            wc = __ldg(sen + c);
                            if (wc != word) {
                                const T *xnrow = w_in + (size_t) wc * ld;
#pragma unroll
                                for (int k = 0; k < NV4; k++)
                                    xn[k] = lane + 32 * k < n4 ? S::loadraw_g(xnrow, lane + 32 * k) : S::zero_raw();
                            }
                        }
                        f = warp_sum(f);
                        const float g = grad_from_table(f, 1, alpha, s_exp);
                        const bool again = ahead && wc == word;
#pragma unroll
                        for (int k = 0; k < NV4; k++) {
                            const int cc = lane + 32 * k;
                            const float4 yv = y.v[k];
                            y.v[k] = f4_fma(g, xr.v[k], yv);
                            const typename S::Raw r = S::pack4(f4_fma(g, yv, xr.v[k]), rb.next());
                            if (cc < n4) S::storeraw(x, cc, r);
                            if (again) xn[k] = r;
                        }
                    }
                    c_next = c;
                    w_next = wc;
                }
                pairs += n;
#pragma unroll
                for (int k = 0; k < NV4; k++) {
                    const int cc = lane + 32 * k;
                    const typename S::Raw r = S::pack4(y.v[k], rb.next());
                    if (cc < n4) S::storeraw(yrow, cc, r);
                    if (t_next == t) yn[k] = r;
                }
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
                    break;
                }
                batches++;
                negs_drawn += K;
                if (K > 0) {
                    if constexpr (BF16) {
                        if (Lo.mma)
                            repel_mma(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
                        else
                            repel_simt<true>(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
                    } else {
                        if (Lo.mma)
                            repel_mma_f32(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane);
                        else
                            repel_simt<false>(a, Lo, base, sen + lo_b, rows, negs, K, alpha, s_exp, G, dup, lane, rb);
                    }
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
        if (failed) atomicOr(&a.cnt->error, kErrResample);
    }
}

template <int NV4, bool BF16, bool SYNC>
cudaError_t launch_stream_nvs(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    const Layout Lo = make_layout_stream(a.ld, a.window, a.negative, a.batch, BF16);
    const size_t smem = kSmemHead + (size_t) warps * Lo.per_warp;
    cudaError_t e = cudaFuncSetAttribute(k_stream_train<NV4, BF16, SYNC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    k_stream_train<NV4, BF16, SYNC><<<grid, warps * 32, smem, s>>>(a, warps);
    return cudaGetLastError();
}

template <bool BF16>
cudaError_t launch_stream_mode(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    const bool y = a.sync_window;
    switch ((a.d + 127) / 128) {
        case 1: return y ? launch_stream_nvs<1, BF16, true>(a, grid, warps, s) : launch_stream_nvs<1, BF16, false>(a, grid, warps, s);
        case 2: return y ? launch_stream_nvs<2, BF16, true>(a, grid, warps, s) : launch_stream_nvs<2, BF16, false>(a, grid, warps, s);
        case 3: return y ? launch_stream_nvs<3, BF16, true>(a, grid, warps, s) : launch_stream_nvs<3, BF16, false>(a, grid, warps, s);
        case 4: return y ? launch_stream_nvs<4, BF16, true>(a, grid, warps, s) : launch_stream_nvs<4, BF16, false>(a, grid, warps, s);
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

cudaError_t launch_batched_train(const TrainArgs &a, bool bf16, bool stream, int grid, int warps_per_cta, cudaStream_t s) {
    if (stream)
        return bf16 ? launch_stream_mode<true>(a, grid, warps_per_cta, s) : launch_stream_mode<false>(a, grid, warps_per_cta, s);
    return bf16 ? launch_mode<true>(a, grid, warps_per_cta, s) : launch_mode<false>(a, grid, warps_per_cta, s);
}

}  // namespace parw2v
