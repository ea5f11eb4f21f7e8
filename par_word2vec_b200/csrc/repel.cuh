// Shared-negative repulsion of one batch (PAR_Word2Vec_cpu.cpp:571-679) for the BATCHED kernels.
//
// A batch is `rows` consecutive kept positions of a sentence (M_in: their W_in rows) and K negatives
// drawn for it (M_out: their W_out rows).  The reference forms, with three SGEMMs,
//     G = alpha * (0 - sigma(M_out M_in^T))          (K x rows, sigma through the expTable)
//     W_out[negs] += G M_in,   W_in[batch] += G^T M_out
// (cpu.cpp:633-674).  Here one warp does it on chip in column chunks of the rows:
//   pass 1  stage chunks of M_in and M_out, accumulate M_out M_in^T on the tensor cores;
//           sigma/label 0 through the table; gradients of repeated words merged into their first
//           occurrence, so every distinct row is written once;
//   pass 2  re-stage each chunk (the rows' current values: "current value + own update", a
//           one-chunk read-to-write window like the reference's unsynchronised `+=`), form the new
//           values on the tensor cores and store them back.
// Staging is 16-byte cp.async copies and the BF16 write-back 16-byte stores (the default); or,
// selectable, one bulk copy (cp.async.bulk, the TMA unit) per row and chunk completing on the
// warp's mbarrier and one bulk store per row and chunk.  The BF16 path reads each row's address
// from a per-batch table in shared memory (which also marks the rows its write-back skips); the
// FP32 path forms them from the words.  Rows of the tables are never read through this SM's L1
// (bulk copies and cp.async.cg read at L2): L1 is not coherent with the other SMs' writes.
#pragma once
#include <cstdint>

#include "bulk.cuh"
#include "common.cuh"
#include "internal.h"
#include "mma.cuh"

namespace parw2v {
namespace rep {

constexpr int kRows = 32;       // batch rows on the tensor-core paths (staging rows of M_in)
constexpr int kSweepNeg = 48;   // negatives per pass-1 sweep (3 m-tiles of accumulators)
constexpr int kMaxMt = 6;       // m-tiles of negatives: K <= 96 on the tensor-core paths
constexpr int kStride = 40;     // staged row stride in BF16 (80 B: conflict-free ldmatrix rows)
constexpr int kCols = 32;       // BF16 columns per chunk (64 B per row)
constexpr int kF32Cols = 16;    // FP32 columns per chunk (the same 64 B per row)
constexpr int kF32Stride = 20;  // staged FP32 row stride in floats (80 B)
constexpr int kGbStride = 40;   // BF16 G row stride (80 B)
constexpr int kGps = 36;        // FP32 G row stride in floats (144 B: conflict-free ldmatrix rows)
static_assert(kF32Stride * 4 == kStride * 2, "FP32 and BF16 staging rows take the same bytes");

__host__ __device__ constexpr size_t up16(size_t x) { return (x + 15) & ~(size_t) 15; }

// Where the repulsion's buffers sit inside a warp's shared-memory region (byte offsets from the
// region's start, all 16-byte aligned).
struct Geom {
    int kcap;       // negatives a batch can draw: rep_b * negative with rep_b < 2 * window
    int mt;         // m-tiles of negatives: ceil(kcap / 16)
    bool mma;       // tensor-core path (rows <= kRows, kcap <= 16 * kMaxMt)
    size_t stage;   // staging: kRows batch rows, then 16 * mt negative rows, 80 B each
    size_t gb;      // G kept through pass 2: BF16 16*mt x kGbStride, or FP32 16*mt x kGps
    size_t gf;      // FP32 G, kcap x kRows, for the table lookup and merging (may alias the staging)
    size_t tab;     // BF16: row addresses, kRows batch rows then kcap negatives (8 B each)
    size_t bytes;   // region size
};

__host__ __device__ inline Geom make_geom(int window, int negative, int batch, bool bf16) {
    Geom g{};
    g.kcap = (2 * window - 1) * negative;
    g.mt = (g.kcap + 15) / 16;
    g.mma = batch <= kRows && g.kcap <= 16 * kMaxMt;
    if (!g.mma) return g;
    const size_t stage_bytes = up16((size_t) (kRows + 16 * g.mt) * kStride * 2);
    const size_t gf_bytes = up16((size_t) g.kcap * kRows * 4);
    const size_t gb_bytes = bf16 ? up16((size_t) 16 * g.mt * kGbStride * 2) : up16((size_t) 16 * g.mt * kGps * 4);
    g.stage = 0;
    if (g.mt * 16 <= kSweepNeg) {
        // one pass-1 sweep: G is written after the last staged chunk of pass 1 and read before the
        // first of pass 2, so it shares the staging bytes
        g.gf = 0;
        g.gb = stage_bytes > gf_bytes ? stage_bytes : gf_bytes;
    } else {
        // several sweeps: the staging of a later sweep would overwrite the G of an earlier one
        g.gf = stage_bytes;
        g.gb = stage_bytes + gf_bytes;
    }
    g.tab = g.gb + gb_bytes;
    // the FP32 path forms row addresses from the words instead: without the table its warps fit
    // 16 to an SM
    g.bytes = g.tab + (bf16 ? up16((size_t) (kRows + g.kcap) * 8) : 0);
    return g;
}

// Warp-uniform staging state: the mbarrier (in shared memory), its phase and the copy method.
struct Stager {
    uint64_t *bar;
    unsigned phase;
    bool bulk;
};

// Global addresses of the batch's rows: tab[r] = W_in row of sbw[r] (r < rows), tab[rows + k] =
// W_out row of negs[k] (k < K).  Bit 0 is set later on rows whose update merges into an earlier
// copy of the same word (they are staged but not written back); rows start on 16-byte boundaries.
template <typename T>
__device__ __forceinline__ void build_row_table(const T *w_in, const T *w_out, int ld, const int *sbw, int rows,
                                                const int *negs, int K, uint64_t *tab, int lane) {
    for (int i = lane; i < rows + K; i += 32) {
        const T *p = i < rows ? w_in + (size_t) sbw[i] * ld : w_out + (size_t) negs[i - rows] * ld;
        tab[i] = reinterpret_cast<uint64_t>(p);
    }
    __syncwarp();
}

// Tag the rows that mark_repeats_warp found repeated (dup[k] for negatives, dup[K + r] for batch
// rows): the write-back skips them.
__device__ __forceinline__ void tag_repeats(uint64_t *tab, const int *dup, int rows, int K, int lane) {
    for (int i = lane; i < rows + K; i += 32)
        if (dup[i < rows ? K + i : i - rows] >= 0) tab[i] |= 1u;
    __syncwarp();
}

// Staged rows are 80 bytes apart (kStride BF16 / kF32Stride FP32).
constexpr int kStageRowBytes = kStride * 2;

// Where stage_rows finds a batch row r (in) and negative k (out): the BF16 path's table (tag bit
// masked off), or the FP32 path's words and tables.
struct RowsFromTable {
    const uint64_t *tab;
    int rows;
    __device__ uint64_t in(int r) const { return tab[r] & ~(uint64_t) 1; }
    __device__ uint64_t out(int k) const { return tab[rows + k] & ~(uint64_t) 1; }
};
template <typename T>
struct RowsFromWords {
    const T *w_in, *w_out;
    int ld;
    const int *sbw, *negs;
    __device__ uint64_t in(int r) const { return reinterpret_cast<uint64_t>(w_in + (size_t) sbw[r] * ld); }
    __device__ uint64_t out(int k) const { return reinterpret_cast<uint64_t>(w_out + (size_t) negs[k] * ld); }
};

// Stage bytes [c0, c0 + bytes) of the batch rows (rows.in(0..rows)) into `sin` and of the
// negatives k0..k0+nk-1 (rows.out(k0..)) into `sout`.  bytes is 32 or 64: each lane copies the
// same 16-byte piece (lane mod pieces) of every (32 / pieces)-th row.  Returns false (warp-uniform)
// if a bulk copy did not complete in time.
template <typename Rows>
__device__ __forceinline__ bool stage_rows(Stager &st, const Rows &rowsrc, unsigned c0, unsigned bytes, int rows,
                                           int k0, int nk, void *sin, void *sout, int lane) {
    unsigned char *s_in = static_cast<unsigned char *>(sin), *s_out = static_cast<unsigned char *>(sout);
    bool ok = true;
    if (st.bulk) {
        // the previous chunk's bulk stores have read the staging; earlier generic accesses of the
        // staging (ldmatrix, stmatrix, zeroing) come before the bulk writes
        bulk_wait_read_all();
        fence_proxy_async_shared();
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(st.bar, (unsigned) (rows + nk) * bytes);
        for (int r = lane; r < rows + nk; r += 32) {
            const bool in = r < rows;
            const uint64_t src = in ? rowsrc.in(r) : rowsrc.out(k0 + r - rows);
            unsigned char *dst = in ? s_in + r * kStageRowBytes : s_out + (r - rows) * kStageRowBytes;
            bulk_load(dst, reinterpret_cast<const void *>(src + c0), bytes, st.bar);
        }
        ok = __all_sync(0xffffffffu, mbar_wait_bounded(st.bar, st.phase, kMaxBulkPolls));
        // a copy that did not complete in time: wait once more (bounded) for the copies in flight
        // before the caller gives up on the batch and its warp stops using the staging
        if (!ok) mbar_wait_bounded(st.bar, st.phase, kMaxBulkPolls);
        st.phase ^= 1u;
    } else {
        const int sh = bytes == 64u ? 2 : 1;  // log2 of the 16-byte pieces per row
        const int r0 = lane >> sh, step = 32 >> sh;
        const unsigned pc16 = 16u * (unsigned) (lane & ((1 << sh) - 1));
        const uint64_t goff = c0 + pc16;
        unsigned s = smem_u32(s_in) + (unsigned) r0 * kStageRowBytes + pc16;
        for (int r = r0; r < rows; r += step, s += step * kStageRowBytes)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(rowsrc.in(r) + goff) : "memory");
        s = smem_u32(s_out) + (unsigned) r0 * kStageRowBytes + pc16;
        for (int r = r0; r < nk; r += step, s += step * kStageRowBytes)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(rowsrc.out(k0 + r) + goff)
                         : "memory");
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncwarp();
    return ok;
}

// Repeated words of a batch: dup[k] (negatives, k < K) and dup[K + r] (batch rows, r < rows) get
// the index of the word's first occurrence, or -1.  K <= 96 and rows <= 32, by warp matching.
__device__ __forceinline__ void mark_repeats_warp(const int *negs, int K, const int *words, int rows, int *dup,
                                                  int lane) {
    const int wr = lane < rows ? words[lane] : -1 - lane;
    const unsigned mr = __match_any_sync(0xffffffffu, wr);
    if (lane < rows) dup[K + lane] = (__ffs(mr) - 1 == lane) ? -1 : __ffs(mr) - 1;
    int v[3];
#pragma unroll
    for (int j = 0; j < 3; j++) v[j] = 32 * j + lane < K ? negs[32 * j + lane] : -1000 * (j + 1) - lane;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        if (32 * j >= K) break;
        int first = -1;
#pragma unroll
        for (int jj = 0; jj < j; jj++)
            for (int q = 0; q < 32; q++) {
                const int w = __shfl_sync(0xffffffffu, v[jj], q);
                if (first < 0 && w == v[j]) first = 32 * jj + q;
            }
        const unsigned m = __match_any_sync(0xffffffffu, v[j]);
        if (first < 0 && __ffs(m) - 1 != lane) first = 32 * j + __ffs(m) - 1;
        if (32 * j + lane < K) dup[32 * j + lane] = first;
    }
    __syncwarp();
}

// Generic form of the marks (any K, rows), for the CUDA-core path.
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

// Zero `n` staged rows (80 B each) starting at row pointer p.
__device__ __forceinline__ void zero_rows(void *p, int n, int lane) {
    uint4 *q = reinterpret_cast<uint4 *>(p);
    for (int i = lane; i < n * 5; i += 32) q[i] = make_uint4(0u, 0u, 0u, 0u);
}

// ---- BF16 tables ----
// Pass 2 works on 16-column tiles of the chunk in transposed form, so that the rows of the batch
// and the negatives are the MMA's n dimension (multiples of 8, little padding):
//   new M_in^T  (16 x rows) = M_out^T (16 x K) . G (K x rows)  + I . M_in^T
//   new M_out^T (16 x K)    = M_in^T (16 x rows) . G^T (rows x K) + I . M_out^T
// The identity products add the staged values exactly in FP32, so the accumulators hold the new
// values; each 8-row slice is rounded stochastically to BF16 and written back into the staged tile
// with stmatrix.trans, and whole 16-byte pieces go back to the tables.  Per 16-column tile the old
// M_in^T fragments the M_out products need are read into registers first; then the M_in update is
// formed and stored two n-tiles at a time (it reads the old M_out), then the M_out update one
// n-tile at a time (each tile reads only those registers and its own old rows).
// Returns false if staging failed (the batch is then left partly applied: the caller stops).
__device__ __noinline__ bool repel_bf16(const TrainArgs &a, const Geom &geo, unsigned char *region, const int *sbw,
                                        int rows, const int *negs, int K, float alpha, const float *s_exp, int *dup,
                                        int lane, LaneBits &rb, Stager &st) {
    using T = __nv_bfloat16;
    const T *w_in_c = static_cast<const T *>(a.w_in);
    const T *w_out_c = static_cast<const T *>(a.w_out);
    const int ld = a.ld;
    T *sin = reinterpret_cast<T *>(region + geo.stage);  // kRows x kStride
    T *sout = sin + (size_t) kRows * kStride;            // 16*mt x kStride
    T *Gb = reinterpret_cast<T *>(region + geo.gb);      // 16*mt x kGbStride
    float *Gf = reinterpret_cast<float *>(region + geo.gf);  // K x kRows
    const int g = lane >> 2, t = lane & 3;
    const int nt1 = (rows + 7) >> 3;  // pass 1: n-tiles of batch rows
    uint64_t *tab = reinterpret_cast<uint64_t *>(region + geo.tab);
    build_row_table(w_in_c, w_out_c, ld, sbw, rows, negs, K, tab, lane);
    bool ok = true;
    // this warp's earlier plain stores to the tables (the sentence's attraction, the previous
    // batch's write-back) before the bulk copies read the same rows
    if (st.bulk) fence_proxy_async_global();

    // ---- pass 1: G = M_out M_in^T in sweeps of up to 48 negatives ----
#pragma unroll 1
    for (int k0 = 0; k0 < K && ok; k0 += kSweepNeg) {
        const int nk = min(kSweepNeg, K - k0);
        const int mts = (nk + 15) >> 4;
        float acc[3][4][4];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int e = 0; e < 4; e++) acc[i][j][e] = 0.f;
#pragma unroll 1
        for (int col0 = 0; col0 < ld; col0 += kCols) {
            const int ncols = min(kCols, ld - col0);
            if (!(ok = stage_rows(st, RowsFromTable{tab, rows}, 2u * col0, 2u * ncols, rows, k0, nk, sin, sout, lane)))
                break;
            // rows beyond `rows` / `nk` in the tiles hold stale data; they only reach accumulator
            // entries that are never read
#pragma unroll 1
            for (int ks = 0; ks < (ncols >> 4); ks++) {
                unsigned bfr[4][2];
#pragma unroll
                for (int np = 0; np < 2; np++) {  // n-tiles 2np, 2np+1 in one ldmatrix.x4
                    unsigned r[4];
                    const int n = np * 16 + (lane & 7) + ((lane >> 4) << 3);
                    ldsm_x4(r, sin + (size_t) n * kStride + ks * 16 + ((lane >> 3) & 1) * 8);
                    bfr[2 * np][0] = r[0];
                    bfr[2 * np][1] = r[1];
                    bfr[2 * np + 1][0] = r[2];
                    bfr[2 * np + 1][1] = r[3];
                }
#pragma unroll
                for (int mt = 0; mt < 3; mt++)
                    if (mt < mts) {
                        unsigned af[4];
                        ldsm_x4(af, sout + (size_t) (mt * 16 + (lane & 15)) * kStride + ks * 16 + (lane >> 4) * 8);
#pragma unroll
                        for (int nt = 0; nt < 4; nt++)
                            if (nt < nt1) mma16816(acc[mt][nt], af, bfr[nt][0], bfr[nt][1]);
                    }
            }
            __syncwarp();
        }
        if (!ok) break;
        // sigma / label 0 through the table into the FP32 G
#pragma unroll
        for (int mt = 0; mt < 3; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (mt < mts && nt < nt1) {
                        const int k = mt * 16 + g + ((e >> 1) << 3), r = nt * 8 + 2 * t + (e & 1);
                        if (k < nk && r < rows) Gf[(k0 + k) * kRows + r] = grad_from_table(acc[mt][nt][e], 0, alpha, s_exp);
                    }
        __syncwarp();
    }
    if (!ok) return false;
    mark_repeats_warp(negs, K, sbw, rows, dup, lane);
    merge_marked(K, rows, Gf, kRows, dup, lane);
    tag_repeats(tab, dup, rows, K, lane);
    // BF16 G, zero outside K x rows up to whole 16 x 16 blocks
    const int kp = 16 * ((K + 15) >> 4), rp = 16 * ((rows + 15) >> 4);
    const int hsh = rp == 32 ? 4 : 3;  // column pairs per G row: rp / 2
    for (int i = lane; i < kp << hsh; i += 32) {
        const int k = i >> hsh, r = 2 * (i & ((1 << hsh) - 1));
        const float v0 = (k < K && r < rows) ? Gf[k * kRows + r] : 0.f;
        const float v1 = (k < K && r + 1 < rows) ? Gf[k * kRows + r + 1] : 0.f;
        reinterpret_cast<__nv_bfloat162 *>(Gb + (size_t) k * kGbStride)[r >> 1] = __floats2bfloat162_rn(v0, v1);
    }
    __syncwarp();  // the FP32 G may share the staging bytes zeroed next
    // zero the padding rows the pass-2 products read as their k dimension (they stay zero: the
    // stores write zeros back into them)
    zero_rows(sin + (size_t) rows * kStride, rp - rows, lane);
    zero_rows(sout + (size_t) K * kStride, kp - K, lane);
    __syncwarp();

    // ---- pass 2 ----
    const int ntq = (rows + 7) >> 3, ksq = kp >> 4;  // M_in update: n-tiles of rows, k-steps of negatives
    const int nto = (K + 7) >> 3, kso = rp >> 4;     // M_out update: n-tiles of negatives, k-steps of rows
    // identity A fragment (16 x 16 BF16): a0 = a3 = {I[g][2t], I[g][2t+1]}, a1 = a2 = 0
    unsigned ident[4];
    ident[0] = (g == 2 * t ? 0x3F80u : 0u) | (g == 2 * t + 1 ? 0x3F800000u : 0u);
    ident[1] = ident[2] = 0u;
    ident[3] = ident[0];
    // lane address parts: transposed A loads and the 8-row slices (ldmatrix / stmatrix rows)
    const int a_row = (lane & 7) + ((lane >> 4) << 3), a_col = ((lane >> 3) & 1) * 8;
    const int s_row = lane & 7, s_col = ((lane >> 3) & 1) * 8;
#pragma unroll 1
    for (int col0 = 0; col0 < ld; col0 += kCols) {
        const int ncols = min(kCols, ld - col0);
        if (!stage_rows(st, RowsFromTable{tab, rows}, 2u * col0, 2u * ncols, rows, 0, K, sin, sout, lane)) return false;
#pragma unroll 1
        for (int c = 0; c < ncols; c += 16) {
            // the old M_in^T slices the M_out products take as A, read before the new M_in values
            // overwrite them
            unsigned ai[2][4];
#pragma unroll
            for (int ks = 0; ks < 2; ks++)
                if (ks < kso) ldsm_x4_t(ai[ks], sin + (size_t) (16 * ks + a_row) * kStride + c + a_col);
            // new M_in^T slices, two n-tiles (batch rows 16np..16np+15) at a time
#pragma unroll 1
            for (int np = 0; 2 * np < ntq; np++) {
                const bool two = 2 * np + 1 < ntq;
                float q0[4], q1[4];
                const T *gq = Gb + (size_t) (lane & 15) * kGbStride + 16 * np + ((lane >> 4) << 3);
                const T *aq = sout + (size_t) a_row * kStride + c + a_col;
                {
                    unsigned af[4], b[4];  // k-step 0: G rows 0..15 at columns 16np..16np+15
                    ldsm_x4_t(af, aq);
                    ldsm_x4_t(b, gq);
                    mma16816_z(q0, af, b[0], b[1]);
                    if (two) mma16816_z(q1, af, b[2], b[3]);
                }
#pragma unroll 1
                for (int ks = 1; ks < ksq; ks++) {
                    unsigned af[4], b[4];
                    ldsm_x4_t(af, aq + (size_t) 16 * ks * kStride);
                    ldsm_x4_t(b, gq + (size_t) 16 * ks * kGbStride);
                    mma16816(q0, af, b[0], b[1]);
                    if (two) mma16816(q1, af, b[2], b[3]);
                }
                T *srow = sin + (size_t) (16 * np + s_row) * kStride + c + s_col;
                unsigned bi[2];
                ldsm_x2(bi, srow);
                mma16816(q0, ident, bi[0], bi[1]);
                uint64_t bits = rb.next();
                stsm_x2_t(srow, pack_sr2(make_float2(q0[0], q0[1]), bits), pack_sr2(make_float2(q0[2], q0[3]), bits >> 32));
                if (two) {
                    ldsm_x2(bi, srow + 8 * kStride);
                    mma16816(q1, ident, bi[0], bi[1]);
                    bits = rb.next();
                    stsm_x2_t(srow + 8 * kStride, pack_sr2(make_float2(q1[0], q1[1]), bits),
                              pack_sr2(make_float2(q1[2], q1[3]), bits >> 32));
                }
            }
            // new M_out^T, one n-tile (8 negatives) at a time: each tile's product, sum and rounding
            // is independent of the others
#pragma unroll 1
            for (int nt = 0; nt < nto; nt++) {
                float o[4];
                unsigned b[4];  // G rows 8nt..8nt+7, columns 0..31 (k-steps 0 and 1)
                ldsm_x4(b, Gb + (size_t) (8 * nt + (lane & 7)) * kGbStride + ((lane >> 3) & 3) * 8);
                mma16816_z(o, ai[0], b[0], b[1]);
                if (kso > 1) mma16816(o, ai[1], b[2], b[3]);
                unsigned bo[2];
                T *srow = sout + (size_t) (8 * nt + s_row) * kStride + c + s_col;
                ldsm_x2(bo, srow);
                mma16816(o, ident, bo[0], bo[1]);
                const uint64_t bits = rb.next();
                const unsigned p0 = pack_sr2(make_float2(o[0], o[1]), bits);
                const unsigned p1 = pack_sr2(make_float2(o[2], o[3]), bits >> 32);
                stsm_x2_t(srow, p0, p1);
            }
        }
        __syncwarp();
        // every distinct row's new chunk back to its table
        if (st.bulk) {
            // one bulk store per row; the next staging waits until they have read the tile
            fence_proxy_async_shared();  // this lane's stmatrix writes before the bulk reads
            __syncwarp();
            for (int rr = lane; rr < rows + K; rr += 32) {
                const uint64_t ad = tab[rr];
                if (ad & 1u) continue;  // a repeated word: its first copy carries the merged update
                const T *src = rr < rows ? sin + (size_t) rr * kStride : sout + (size_t) (rr - rows) * kStride;
                bulk_store(reinterpret_cast<void *>(ad + 2u * col0), src, (unsigned) ncols * 2u);
            }
            bulk_commit();
        } else {
            // as in stage_rows: each lane stores the same 16-byte piece of every (32 / pieces)-th row
            const int sh = ncols == kCols ? 2 : 1;  // log2 of the 16-byte pieces per row
            const int r0 = lane >> sh, step = 32 >> sh;
            const unsigned pc16 = 16u * (unsigned) (lane & ((1 << sh) - 1));
            const uint64_t goff = 2u * (unsigned) col0 + pc16;
            const unsigned char *src = reinterpret_cast<const unsigned char *>(sin) + r0 * kStageRowBytes + pc16;
            for (int r = r0; r < rows; r += step, src += step * kStageRowBytes) {
                const uint64_t ad = tab[r];
                if (!(ad & 1u)) *reinterpret_cast<uint4 *>(ad + goff) = *reinterpret_cast<const uint4 *>(src);
            }
            src = reinterpret_cast<const unsigned char *>(sout) + r0 * kStageRowBytes + pc16;
            for (int r = r0; r < K; r += step, src += step * kStageRowBytes) {
                const uint64_t ad = tab[rows + r];
                if (!(ad & 1u)) *reinterpret_cast<uint4 *>(ad + goff) = *reinterpret_cast<const uint4 *>(src);
            }
        }
        __syncwarp();
    }
    if (st.bulk) {
        // the rows are in global memory before this warp reads them again (the next batch's bulk
        // copies, the next sentence's plain loads)
        bulk_wait_all();
        fence_proxy_async_global();
        __syncwarp();
    }
    return true;
}

// ---- FP32 tables: 3xTF32 products (FP32-level accuracy) ----
// The structure of repel_bf16's pass 1 with 16-column FP32 chunks; pass 2 keeps G in FP32
// (16*mt x kGps) and goes from the accumulators straight to the rows, 8 columns at a time, so the
// new values never pass through BF16.  MTC bounds the negatives' m-tiles (3: K <= 48, 6: K <= 96).
template <int MTC>
__device__ __noinline__ bool repel_f32(const TrainArgs &a, const Geom &geo, unsigned char *region, const int *sbw,
                                       int rows, const int *negs, int K, float alpha, const float *s_exp, int *dup,
                                       int lane, Stager &st) {
    const float *w_in_c = static_cast<const float *>(a.w_in);
    const float *w_out_c = static_cast<const float *>(a.w_out);
    float *w_in = static_cast<float *>(a.w_in);
    float *w_out = static_cast<float *>(a.w_out);
    const int ld = a.ld;
    float *sin = reinterpret_cast<float *>(region + geo.stage);  // kRows x kF32Stride
    float *sout = sin + (size_t) kRows * kF32Stride;             // 16*mt x kF32Stride
    float *Gp = reinterpret_cast<float *>(region + geo.gb);      // 16*mt x kGps
    float *Gf = reinterpret_cast<float *>(region + geo.gf);      // K x kRows
    const int g = lane >> 2, t = lane & 3;
    const int mt1 = (K + 15) >> 4;    // m-tiles of negatives
    const int nt1 = (rows + 7) >> 3;  // n-tiles of batch rows (pass 1)
    const int kr8 = (rows + 7) >> 3;  // 8-row k-steps over the batch rows
    const int kk8 = (K + 7) >> 3;     // 8-row k-steps over the negatives
    const int mr = (rows + 15) >> 4;  // m-tiles of batch rows (pass 2)
    const RowsFromWords<float> rowsrc{w_in_c, w_out_c, ld, sbw, negs};
    bool ok = true;
    if (st.bulk) fence_proxy_async_global();  // as in repel_bf16
#pragma unroll 1
    for (int k0 = 0; k0 < K && ok; k0 += kSweepNeg) {
        const int nk = min(kSweepNeg, K - k0);
        const int mts = (nk + 15) >> 4;
        float acc[3][4][4];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int e = 0; e < 4; e++) acc[i][j][e] = 0.f;
#pragma unroll 1
        for (int col0 = 0; col0 < ld; col0 += kF32Cols) {
            const int ncols = min(kF32Cols, ld - col0);
            if (!(ok = stage_rows(st, rowsrc, 4u * col0, 4u * ncols, rows, k0, nk, sin, sout, lane))) break;
#pragma unroll 1
            for (int ks = 0; ks < (ncols >> 3); ks++) {
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
                    if (mt < mts) {
                        float af[4];
                        ldsm_x4_f32(af, sout + (size_t) (mt * 16 + (lane & 7) + ((lane >> 3) & 1) * 8) * kF32Stride +
                                            ks * 8 + (lane >> 4) * 4);
                        unsigned ab[4], as[4];
                        split_a(af, ab, as);
#pragma unroll
                        for (int nt = 0; nt < 4; nt++)
                            if (nt < nt1) mma3xtf32(acc[mt][nt], ab, as, bb[nt], bs[nt]);
                    }
            }
            __syncwarp();
        }
        if (!ok) break;
#pragma unroll
        for (int mt = 0; mt < 3; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (mt < mts && nt < nt1) {
                        const int k = mt * 16 + g + ((e >> 1) << 3), r = nt * 8 + 2 * t + (e & 1);
                        if (k < nk && r < rows) Gf[(k0 + k) * kRows + r] = grad_from_table(acc[mt][nt][e], 0, alpha, s_exp);
                    }
        __syncwarp();
    }
    if (!ok) return false;
    mark_repeats_warp(negs, K, sbw, rows, dup, lane);
    merge_marked(K, rows, Gf, kRows, dup, lane);
    // the FP32 G pass 2 reads, zero outside K x rows
    for (int i = lane; i < 16 * mt1 * kRows; i += 32) {
        const int k = i >> 5, r = i & 31;
        Gp[(size_t) k * kGps + r] = (k < K && r < rows) ? Gf[k * kRows + r] : 0.f;
    }
    __syncwarp();  // the FP32 G may share the staging bytes zeroed next
    // padding rows the products read as their k dimension (8-row steps)
    zero_rows(sin + (size_t) rows * kF32Stride, 8 * kr8 - rows, lane);
    zero_rows(sout + (size_t) K * kF32Stride, 16 * mt1 - K, lane);
    __syncwarp();
#pragma unroll 1
    for (int col0 = 0; col0 < ld; col0 += kF32Cols) {
        const int ncols = min(kF32Cols, ld - col0);
        if (!stage_rows(st, rowsrc, 4u * col0, 4u * ncols, rows, 0, K, sin, sout, lane)) return false;
#pragma unroll 1
        for (int nt = 0; nt < (ncols >> 3); nt++) {
            const int cb = nt * 8;
            float o[MTC][4], q[2][4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
#pragma unroll
                for (int m = 0; m < MTC; m++) o[m][e] = 0.f;
                q[0][e] = q[1][e] = 0.f;
            }
            // M_out update: G (K x rows) . M_in (rows x 8 columns)
#pragma unroll 1
            for (int ks = 0; ks < kr8; ks++) {
                unsigned bb[2], bs[2];
                split_tf32(sin[(size_t) (ks * 8 + t) * kF32Stride + cb + g], bb[0], bs[0]);
                split_tf32(sin[(size_t) (ks * 8 + t + 4) * kF32Stride + cb + g], bb[1], bs[1]);
#pragma unroll
                for (int mt = 0; mt < MTC; mt++)
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
#pragma unroll
            for (int mt = 0; mt < MTC; mt++)
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
        __syncwarp();
    }
    return true;
}

}  // namespace rep
}  // namespace parw2v
