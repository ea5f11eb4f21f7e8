// SGNS loss forward, its hand-written adjoint, and FP64 central finite differences.
//
// Minibatch: pairs p = (t_p, c_p); window w = p / ctx_per_window shares negatives
// neg[w * n_neg .. (w + 1) * n_neg).
//   L = sum_p [ softplus(-f_p) + sum_k softplus(f_pk) ],  f_p = u_c . v_t,  f_pk = u_c . v_k
// (softplus(x) = log(1 + e^x) = -log s(-x)).  The adjoint is the attraction-repulsion update
// of the reference with alpha = 1 and every term taken at the same weights:
//   dL/df_p  = s(f_p) - 1    (the reference's g = (1 - s(f)) * alpha, PAR_Word2Vec_cpu.cpp:554-559)
//   dL/df_pk = s(f_pk)       (g = (0 - s(f)) * alpha, :642-647)
//   dL/du_c += dL/df * v,  dL/dv += dL/df * u_c.
// Layout: one warp per pair, lane l owns float2 chunks l, l + 32, ... of a row, dot products by
// warp shuffle; gradient rows are added with vector reductions into dense FP32 buffers.
#include "common.cuh"
#include "internal.h"

namespace parw2v {

namespace {

constexpr int kLossWarps = 8;

__device__ __forceinline__ float2 load2(const void *w, bool bf16, size_t off) {
    if (bf16) {
        const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(static_cast<const __nv_bfloat16 *>(w) + off);
        return __bfloat1622float2(v);
    }
    return *reinterpret_cast<const float2 *>(static_cast<const float *>(w) + off);
}

__device__ __forceinline__ float row_dot(const void *a, size_t ra, const void *b, size_t rb, bool bf16, int n2, int lane) {
    float s = 0.f;
    for (int q = lane; q < n2; q += 32) {
        const float2 x = load2(a, bf16, ra + 2 * (size_t) q), y = load2(b, bf16, rb + 2 * (size_t) q);
        s = fmaf(x.x, y.x, fmaf(x.y, y.y, s));
    }
    return warp_sum(s);
}

__device__ __forceinline__ double softplus(double x) { return x > 0 ? x + log1p(exp(-x)) : log1p(exp(x)); }
__device__ __forceinline__ double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }

__global__ void __launch_bounds__(kLossWarps * 32) k_loss(LossBatch b, const void *w_in, const void *w_out, bool bf16,
                                                          int d, int ld, double *out) {
    const int lane = threadIdx.x & 31;
    const int p = blockIdx.x * kLossWarps + (threadIdx.x >> 5);
    __shared__ double part[kLossWarps];
    double acc = 0.0;
    if (p < b.n_pairs) {
        const int n2 = (d + 1) >> 1;
        const size_t rc = (size_t) b.ctx[p] * ld;
        const int win = p / b.ctx_per_window;
        acc += softplus(-(double) row_dot(w_in, rc, w_out, (size_t) b.tgt[p] * ld, bf16, n2, lane));
        for (int k = 0; k < b.n_neg; k++)
            acc += softplus((double) row_dot(w_in, rc, w_out, (size_t) b.neg[(size_t) win * b.n_neg + k] * ld, bf16, n2, lane));
    }
    if (lane == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < kLossWarps; i++) s += part[i];
        atomicAdd(out, s);
    }
}

__device__ __forceinline__ float dl_df(float f, int label, bool exact, const float *exp_table) {
    if (exact) return (float) (sigmoid((double) f) - (double) label);
    return -grad_from_table(f, label, 1.0f, exp_table);
}

__global__ void __launch_bounds__(kLossWarps * 32) k_adjoint(LossBatch b, const void *w_in, const void *w_out, bool bf16,
                                                             int d, int ld, const float *exp_table, int exact,
                                                             float *g_in, float *g_out) {
    const int lane = threadIdx.x & 31;
    const int p = blockIdx.x * kLossWarps + (threadIdx.x >> 5);
    if (p >= b.n_pairs) return;
    const int n2 = (d + 1) >> 1;
    const size_t rc = (size_t) b.ctx[p] * ld;
    const int win = p / b.ctx_per_window;
    // every term's dL/df is taken at the current weights: the dense gradient buffers are separate
    const size_t rt = (size_t) b.tgt[p] * ld;
    const float gp = dl_df(row_dot(w_in, rc, w_out, rt, bf16, n2, lane), 1, exact, exp_table);
    // positive term rows
    for (int q = lane; q < n2; q += 32) {
        const size_t o = 2 * (size_t) q;
        const float2 u = load2(w_in, bf16, rc + o);
        const float2 vt = load2(w_out, bf16, rt + o);
        red_add_f2(g_in + rc + o, make_float2(gp * vt.x, gp * vt.y));
        red_add_f2(g_out + rt + o, make_float2(gp * u.x, gp * u.y));
    }
    // negatives: one dot each (all lanes), then row updates
    for (int k = 0; k < b.n_neg; k++) {
        const size_t rk = (size_t) b.neg[(size_t) win * b.n_neg + k] * ld;
        const float gk = dl_df(row_dot(w_in, rc, w_out, rk, bf16, n2, lane), 0, exact, exp_table);
        for (int q = lane; q < n2; q += 32) {
            const size_t o = 2 * (size_t) q;
            const float2 u = load2(w_in, bf16, rc + o);
            const float2 vk = load2(w_out, bf16, rk + o);
            red_add_f2(g_in + rc + o, make_float2(gk * vk.x, gk * vk.y));
            red_add_f2(g_out + rk + o, make_float2(gk * u.x, gk * u.y));
        }
    }
}

// FP64 central differences: for probe i, only the terms whose dot product contains the probed
// element change, so (L+ - L-) is summed over those terms alone (the others cancel exactly).
__global__ void k_loss_fd(LossBatch b, const void *w_in, const void *w_out, bool bf16, int d, int ld,
                          const int32_t *matrix, const int32_t *row, const int32_t *col, double h, double *grad) {
    const int probe = blockIdx.x;
    const int m = matrix[probe], r = row[probe], j = col[probe];
    __shared__ double part[256];
    double acc = 0.0;
    auto wv = [&](const void *w, size_t off) -> double {
        return bf16 ? (double) __bfloat162float(static_cast<const __nv_bfloat16 *>(w)[off])
                    : (double) static_cast<const float *>(w)[off];
    };
    auto dot64 = [&](size_t ra, size_t rb) -> double {
        double s = 0.0;
        for (int e = 0; e < d; e++) s += wv(w_in, ra + e) * wv(w_out, rb + e);
        return s;
    };
    const int terms_per_pair = 1 + b.n_neg;
    for (long long t = threadIdx.x; t < (long long) b.n_pairs * terms_per_pair; t += blockDim.x) {
        const int p = (int) (t / terms_per_pair), k = (int) (t % terms_per_pair) - 1;
        const int c = b.ctx[p];
        const int o = k < 0 ? b.tgt[p] : b.neg[(size_t) (p / b.ctx_per_window) * b.n_neg + k];
        double coef;  // d f / d (probed element)
        if (m == 0 && c == r) coef = wv(w_out, (size_t) o * ld + j);
        else if (m == 1 && o == r) coef = wv(w_in, (size_t) c * ld + j);
        else continue;
        const double f = dot64((size_t) c * ld, (size_t) o * ld);
        const double fp = f + h * coef, fm = f - h * coef;
        // positive term softplus(-f), negative term softplus(f)
        acc += k < 0 ? softplus(-fp) - softplus(-fm) : softplus(fp) - softplus(fm);
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) grad[probe] = part[0] / (2.0 * h);
}

}  // namespace

cudaError_t launch_loss(const LossBatch &b, const void *w_in, const void *w_out, bool bf16, int d, int ld, double *out,
                        cudaStream_t s) {
    const int blocks = (b.n_pairs + kLossWarps - 1) / kLossWarps;
    if (blocks > 0) k_loss<<<blocks, kLossWarps * 32, 0, s>>>(b, w_in, w_out, bf16, d, ld, out);
    return cudaGetLastError();
}

cudaError_t launch_adjoint(const LossBatch &b, const void *w_in, const void *w_out, bool bf16, int d, int ld,
                           const float *exp_table, int exact, float *g_in, float *g_out, cudaStream_t s) {
    const int blocks = (b.n_pairs + kLossWarps - 1) / kLossWarps;
    if (blocks > 0)
        k_adjoint<<<blocks, kLossWarps * 32, 0, s>>>(b, w_in, w_out, bf16, d, ld, exp_table, exact, g_in, g_out);
    return cudaGetLastError();
}

cudaError_t launch_loss_fd(const LossBatch &b, const void *w_in, const void *w_out, bool bf16, int d, int ld,
                           const int32_t *matrix, const int32_t *row, const int32_t *col, int n_probes, double h,
                           double *grad, cudaStream_t s) {
    if (n_probes > 0) k_loss_fd<<<n_probes, 256, 0, s>>>(b, w_in, w_out, bf16, d, ld, matrix, row, col, h, grad);
    return cudaGetLastError();
}

}  // namespace parw2v
