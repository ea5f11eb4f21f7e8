// PLAIN mode: FP32 Hogwild, one warp per sentence, every row read from and written to global
// memory at each use.  This is the straightforward GPU formulation of PAR_Word2Vec_cpu's thread
// loop (PAR_Word2Vec_cpu.cpp:529-679) and the baseline the data-local kernel is measured against.
//
// Per sentence (a "</s>"-terminated line of the packed corpus, cut every 1000 kept tokens):
//   attraction  for each position: b from the sentence's LCG; the target's W_out row lives in
//               registers (lane l owns float2 chunks l, l+32, ...); each context's W_in row is
//               loaded, dotted (warp shuffle reduction), updated and stored back;
//   repulsion   per batch of `batch` positions: rep_b and rep_b * negative shared negatives from
//               the unigram table, redrawn uniformly while they occur in the sentence; M_in and
//               M_out are staged in the warp's global workspace, the three products run on the
//               warp.  Each touched row is written back once, duplicates merged first, as (the
//               row as it is at write-back + this batch's update): the reference's unsynchronised
//               `+=` with one row's read-to-write window.
// Table rows are always read at L2 (ld.global.cg): an SM's L1 is not coherent with other SMs'
// writes, and at thousands of sentences in flight a hot row served from a stale L1 line turns
// most of its updates into lost ones (the final loss drifts far from the reference's).
// Random streams: the sentence's LCG starts from mix64(seed, epoch, line, piece); the learning
// rate decays linearly with the sentence's position in the corpus (the reference decays with the
// words processed so far, :443).
#include "common.cuh"
#include "internal.h"
#include "sentence.cuh"

namespace parw2v {

namespace {

constexpr int kPlainWarps = 8;

template <int NV2>
struct RowReg {
    float2 v[NV2];
};

template <int NV2>
__device__ __forceinline__ void load_row(RowReg<NV2> &r, const float *row, int n2, int lane) {
    const float2 *p = reinterpret_cast<const float2 *>(row);
#pragma unroll
    for (int i = 0; i < NV2; i++) {
        const int q = lane + 32 * i;
        r.v[i] = q < n2 ? p[q] : make_float2(0.f, 0.f);
    }
}
// a row of the global tables: read at L2, never from this SM's (non-coherent) L1, so a row that
// another SM has written is seen as written, not as this SM cached it earlier
template <int NV2>
__device__ __forceinline__ void load_row_g(RowReg<NV2> &r, const float *row, int n2, int lane) {
    const float2 *p = reinterpret_cast<const float2 *>(row);
#pragma unroll
    for (int i = 0; i < NV2; i++) {
        const int q = lane + 32 * i;
        r.v[i] = q < n2 ? __ldcg(p + q) : make_float2(0.f, 0.f);
    }
}
template <int NV2>
__device__ __forceinline__ void store_row(const RowReg<NV2> &r, float *row, int n2, int lane) {
    float2 *p = reinterpret_cast<float2 *>(row);
#pragma unroll
    for (int i = 0; i < NV2; i++) {
        const int q = lane + 32 * i;
        if (q < n2) p[q] = r.v[i];
    }
}
template <int NV2>
__device__ __forceinline__ float dot_row(const RowReg<NV2> &a, const RowReg<NV2> &b) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < NV2; i++) s = fmaf(a.v[i].x, b.v[i].x, fmaf(a.v[i].y, b.v[i].y, s));
    return warp_sum(s);
}


__host__ __device__ __forceinline__ size_t plain_warp_smem(int kmax, int B, int w) {
    return sizeof(int) * (size_t) (kMaxSentence + 2 * kmax + B) + sizeof(float) * (size_t) kmax * B +
           (sizeof(float) + sizeof(int)) * (size_t) (2 * w);
}

// Duplicate words among the batch's negatives (and among its rows) would write the same row twice;
// their gradient rows / columns are merged into the first occurrence, which then writes once.
__device__ __forceinline__ void merge_duplicates(const int *negs, int K, const int *sen_b, int rows, float *grad,
                                                 int *dup, int lane) {
    for (int k = lane; k < K; k += 32) {
        int first = -1;
        for (int q = 0; q < k && first < 0; q++)
            if (negs[q] == negs[k]) first = q;
        dup[k] = first;
    }
    for (int r = lane; r < rows; r += 32) {
        int first = -1;
        for (int q = 0; q < r && first < 0; q++)
            if (sen_b[q] == sen_b[r]) first = q;
        dup[K + r] = first;
    }
    __syncwarp();
    // columns (batch rows) first, then rows (negatives): each step keeps G consistent
    for (int r = 0; r < rows; r++) {
        const int f = dup[K + r];
        if (f >= 0)
            for (int k = lane; k < K; k += 32) {
                grad[k * rows + f] += grad[k * rows + r];
                grad[k * rows + r] = 0.f;
            }
        __syncwarp();
    }
    for (int k = 0; k < K; k++) {
        const int f = dup[k];
        if (f >= 0)
            for (int r = lane; r < rows; r += 32) {
                grad[f * rows + r] += grad[k * rows + r];
                grad[k * rows + r] = 0.f;
            }
        __syncwarp();
    }
}

template <int NV2>
__global__ void __launch_bounds__(kPlainWarps * 32) k_plain_train(TrainArgs a, int warps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w = a.window, B = a.batch, ld = a.ld;
    const FastMod mod_w((uint32_t) w), mod_2w((uint32_t) (2 * w));
    const int n2 = (a.d + 1) >> 1;
    const int kmax = 2 * w * a.negative;
    float *s_exp = reinterpret_cast<float *>(smem_raw);  // 1004
    unsigned char *warp_base = smem_raw + 1004 * sizeof(float) + (size_t) wid * plain_warp_smem(kmax, B, w);
    int *sen = reinterpret_cast<int *>(warp_base);
    int *negs = sen + kMaxSentence;
    int *dup = negs + kmax;  // kmax + B: duplicate marks of negatives, then of batch rows
    float *grad = reinterpret_cast<float *>(dup + kmax + B);
    float *ctx_g = grad + (size_t) kmax * B;                  // 2w: window-synchronous gradients
    int *ctx_w = reinterpret_cast<int *>(ctx_g + 2 * w);       // 2w: and context words
    for (int i = threadIdx.x; i <= kExpTableSize; i += blockDim.x) s_exp[i] = a.exp_table[i];
    __syncthreads();

    float *w_in = static_cast<float *>(a.w_in);
    float *w_out = static_cast<float *>(a.w_out);
    const size_t gwarp = (size_t) blockIdx.x * warps + wid;
    float *m_in = a.scratch + gwarp * a.scratch_per_warp;  // B x ld
    float *m_out = m_in + (size_t) B * ld;                  // kmax x ld
    const uint64_t n_lines = a.cnt->n_lines, total_kept = a.cnt->total_kept;
    const int epoch = hogwild_epoch(a);
    unsigned long long st_kept = 0, st_sent = 0, st_pairs = 0, st_batches = 0, st_negs = 0;
    bool failed = false;

    for (;;) {
        unsigned long long line = 0;
        if (lane == 0) line = atomicAdd(&a.cnt->work, 1ULL);
        line = __shfl_sync(0xffffffffu, line, 0);
        if (line >= n_lines || failed) break;
        const uint32_t lo = line ? a.line_end[line - 1] : 0u, hi = a.line_end[line];
        int piece = 0;
        for (uint32_t c0 = lo; c0 < hi; c0 += kMaxSentence, piece++) {
            const int L = (int) min((uint32_t) kMaxSentence, hi - c0);
            for (int i = lane; i < L; i += 32) sen[i] = a.packed[c0 + i];
            __syncwarp();
            uint64_t rng = sentence_seed_b(a, epoch, line, piece);
            const float alpha = sentence_alpha_b(a, epoch, c0, total_kept);

            // ---- attraction (:529-568) ----
            for (int pos = 0; pos < L; pos++) {
                rng = lcg_next(rng);
                const int b = (int) mod_w(rng);
                float *y = w_out + (size_t) sen[pos] * ld;
                RowReg<NV2> yr;
                load_row_g(yr, y, n2, lane);
                if (a.sync_window) {
                    // all contexts scored against the same target row, then all updates applied
                    int n = 0;
                    for (int i = b; i < 2 * w + 1 - b; i++) {
                        if (i == w) continue;
                        const int c = pos - w + i;
                        if (c < 0) continue;
                        if (c >= L) break;
                        RowReg<NV2> xr;
                        load_row_g(xr, w_in + (size_t) sen[c] * ld, n2, lane);
                        const float g = grad_from_table(dot_row(xr, yr), 1, alpha, s_exp);
                        if (lane == 0) {
                            ctx_g[n] = g;
                            ctx_w[n] = sen[c];
                        }
                        n++;
                    }
                    __syncwarp();
                    if (lane == 0)
                        for (int i = 0; i < n; i++)
                            for (int k = 0; k < i; k++)
                                if (ctx_w[k] == ctx_w[i]) {
                                    ctx_g[k] += ctx_g[i];
                                    ctx_g[i] = 0.f;
                                    break;
                                }
                    __syncwarp();
                    RowReg<NV2> dy;
#pragma unroll
                    for (int q = 0; q < NV2; q++) dy.v[q] = make_float2(0.f, 0.f);
                    for (int i = 0; i < n; i++) {
                        const float g = ctx_g[i];
                        float *x = w_in + (size_t) ctx_w[i] * ld;
                        RowReg<NV2> xr;
                        load_row_g(xr, x, n2, lane);
#pragma unroll
                        for (int q = 0; q < NV2; q++) {
                            dy.v[q] = make_float2(fmaf(g, xr.v[q].x, dy.v[q].x), fmaf(g, xr.v[q].y, dy.v[q].y));
                            xr.v[q] = make_float2(fmaf(g, yr.v[q].x, xr.v[q].x), fmaf(g, yr.v[q].y, xr.v[q].y));
                        }
                        if (g != 0.f) store_row(xr, x, n2, lane);
                    }
#pragma unroll
                    for (int q = 0; q < NV2; q++) yr.v[q] = make_float2(yr.v[q].x + dy.v[q].x, yr.v[q].y + dy.v[q].y);
                    st_pairs += n;
                    __syncwarp();
                } else
                for (int i = b; i < 2 * w + 1 - b; i++) {
                    if (i == w) continue;
                    const int c = pos - w + i;
                    if (c < 0) continue;
                    if (c >= L) break;
                    float *x = w_in + (size_t) sen[c] * ld;
                    RowReg<NV2> xr;
                    load_row_g(xr, x, n2, lane);
                    const float g = grad_from_table(dot_row(xr, yr), 1, alpha, s_exp);
#pragma unroll
                    for (int q = 0; q < NV2; q++) {
                        const float2 xv = xr.v[q], yv = yr.v[q];
                        xr.v[q] = make_float2(fmaf(g, yv.x, xv.x), fmaf(g, yv.y, xv.y));
                        yr.v[q] = make_float2(fmaf(g, xv.x, yv.x), fmaf(g, xv.y, yv.y));
                    }
                    store_row(xr, x, n2, lane);
                    st_pairs++;
                }
                store_row(yr, y, n2, lane);
            }

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
                __syncwarp();
                // stage pre-update copies of the batch rows and the negatives' rows
                for (int r = 0; r < rows; r++) {
                    RowReg<NV2> t;
                    load_row_g(t, w_in + (size_t) sen[lo_b + r] * ld, n2, lane);
                    store_row(t, m_in + (size_t) r * ld, n2, lane);
                }
                for (int k = 0; k < K; k++) {
                    RowReg<NV2> t;
                    load_row_g(t, w_out + (size_t) negs[k] * ld, n2, lane);
                    store_row(t, m_out + (size_t) k * ld, n2, lane);
                }
                __syncwarp();
                // MM1 + sigma / label 0
                for (int k = 0; k < K; k++) {
                    RowReg<NV2> o;
                    load_row(o, m_out + (size_t) k * ld, n2, lane);
                    for (int r = 0; r < rows; r++) {
                        RowReg<NV2> in;
                        load_row(in, m_in + (size_t) r * ld, n2, lane);
                        const float f = dot_row(o, in);
                        if (lane == 0) grad[k * rows + r] = grad_from_table(f, 0, alpha, s_exp);
                    }
                }
                __syncwarp();
                merge_duplicates(negs, K, sen + lo_b, rows, grad, dup, lane);
                // MM2: W_out[neg_k] += sum_r grad[k][r] M_in[r]  (each distinct word once, added to
                // the row as it is now, not to the staged copy)
                for (int k = 0; k < K; k++) {
                    if (dup[k] >= 0) continue;
                    RowReg<NV2> acc;
                    load_row_g(acc, w_out + (size_t) negs[k] * ld, n2, lane);
                    for (int r = 0; r < rows; r++) {
                        RowReg<NV2> in;
                        load_row(in, m_in + (size_t) r * ld, n2, lane);
                        const float g = grad[k * rows + r];
#pragma unroll
                        for (int q = 0; q < NV2; q++)
                            acc.v[q] = make_float2(fmaf(g, in.v[q].x, acc.v[q].x), fmaf(g, in.v[q].y, acc.v[q].y));
                    }
                    store_row(acc, w_out + (size_t) negs[k] * ld, n2, lane);
                }
                // MM3: W_in[sen[lo_b + r]] += sum_k grad[k][r] M_out[k]
                for (int r = 0; r < rows; r++) {
                    if (dup[K + r] >= 0) continue;
                    RowReg<NV2> acc;
                    load_row_g(acc, w_in + (size_t) sen[lo_b + r] * ld, n2, lane);
                    for (int k = 0; k < K; k++) {
                        RowReg<NV2> o;
                        load_row(o, m_out + (size_t) k * ld, n2, lane);
                        const float g = grad[k * rows + r];
#pragma unroll
                        for (int q = 0; q < NV2; q++)
                            acc.v[q] = make_float2(fmaf(g, o.v[q].x, acc.v[q].x), fmaf(g, o.v[q].y, acc.v[q].y));
                    }
                    store_row(acc, w_in + (size_t) sen[lo_b + r] * ld, n2, lane);
                }
                __syncwarp();
            }
            st_kept += L;
            st_sent++;
            __syncwarp();
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

template <int NV2>
cudaError_t launch_plain_nv(const TrainArgs &a, int grid, int warps, cudaStream_t s) {
    const int kmax = 2 * a.window * a.negative;
    const size_t smem = 1004 * sizeof(float) + (size_t) warps * plain_warp_smem(kmax, a.batch, a.window);
    cudaError_t e = cudaFuncSetAttribute(k_plain_train<NV2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    k_plain_train<NV2><<<grid, warps * 32, smem, s>>>(a, warps);
    return cudaGetLastError();
}

}  // namespace

size_t plain_scratch_floats(int ld, int batch, int window, int negative) {
    return (size_t) (batch + 2 * window * negative) * ld;
}

int plain_warps_per_cta(int requested) { return requested > 0 && requested < kPlainWarps ? requested : kPlainWarps; }

cudaError_t launch_plain_train(const TrainArgs &a, int grid, int warps_per_cta, cudaStream_t s) {
    const int nv2 = (a.d + 63) / 64;
    switch (nv2) {
        case 1: return launch_plain_nv<1>(a, grid, warps_per_cta, s);
        case 2: return launch_plain_nv<2>(a, grid, warps_per_cta, s);
        case 3: return launch_plain_nv<3>(a, grid, warps_per_cta, s);
        case 4: return launch_plain_nv<4>(a, grid, warps_per_cta, s);
        case 5: return launch_plain_nv<5>(a, grid, warps_per_cta, s);
        case 6: return launch_plain_nv<6>(a, grid, warps_per_cta, s);
        case 7: return launch_plain_nv<7>(a, grid, warps_per_cta, s);
        case 8: return launch_plain_nv<8>(a, grid, warps_per_cta, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace parw2v
