// Set-up kernels: subsampling thresholds, the unigram^0.75 table, InitNet, BF16 conversions.
#include "common.cuh"
#include "internal.h"

namespace parw2v {

// keep_thr[w] = sqrtf(ratio) + ratio, ratio = (sample * (float) train_words) / (float) cn[w]
// (PAR_Word2Vec_cpu.cpp:459-460).  A token is dropped when keep_thr < (rand & 0xFFFF) / 65536.
__global__ void k_thresholds(const uint32_t *cn, int V, float sample, uint64_t train_words, float *thr) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= V) return;
    float ratio = __fdiv_rn(__fmul_rn(sample, __ull2float_rn(train_words)), __uint2float_rn(cn[w]));
    thr[w] = __fadd_rn(__fsqrt_rn(ratio), ratio);
}

cudaError_t launch_build_thresholds(const uint32_t *counts, int V, float sample, uint64_t train_words,
                                    float *keep_thr, cudaStream_t s) {
    k_thresholds<<<(V + 255) / 256, 256, 0, s>>>(counts, V, sample, train_words, keep_thr);
    return cudaGetLastError();
}

// ---- unigram table (PAR_Word2Vec_cpu.cpp:96-117) ----
// The reference fills the table sequentially: slot a gets the current word i, then i advances
// when a / 1e8f > d1, where d1 is a float running sum of the double quotients cn^0.75 / total.
// Word i therefore owns slots [t_i, e_i] with e_i = max(t_i, g_i), g_i the first slot whose
// float position exceeds threshold D_i, and t_{i+1} = e_i + 1.  The FP64 total and the float
// running sum are sequential recurrences and run in the reference's order, one addition after the
// other, on one warp whose lanes load 32 values at a time and pass them along by shuffles (so the
// chain never waits for memory); the quotients, the 27-step threshold search per word, the
// max-plus start recurrence (as a prefix maximum) and the 1e8-slot fill run in parallel.

// total = sum of pow_cn in index order, the reference's double additions one by one; every lane
// runs the same chain on the shuffled values.
__global__ void k_table_total(const double *pow_cn, int V, double *total_out) {
    const int lane = threadIdx.x;
    double total = 0.0;
    int base = 0;
    for (; base + 32 <= V; base += 32) {  // whole groups: unrolled, so the shuffles run ahead of the chain
        const double v = pow_cn[base + lane];
#pragma unroll
        for (int j = 0; j < 32; j++) total += __shfl_sync(0xffffffffu, v, j);
    }
    const double v = base + lane < V ? pow_cn[base + lane] : 0.0;
    for (int j = 0; j < V - base; j++) total += __shfl_sync(0xffffffffu, v, j);
    if (lane == 0) *total_out = total;
}

// q_i = pow_cn_i / total (the same double division the recurrence below adds)
__global__ void k_table_quotients(const double *pow_cn, int V, const double *total, double *q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < V) q[i] = pow_cn[i] / *total;
}

// D_i, the value of the float d1 while word i is current: d1 = (float) q_0, then
// d1 = (float) ((double) d1 + q_i), in index order; lane j keeps step j's value of each 32.
__global__ void k_table_running(const double *q, int V, float *D) {
    const int lane = threadIdx.x;
    float d1 = (float) q[0];
    if (lane == 0) D[0] = d1;
    int base = 1;
    for (; base + 32 <= V; base += 32) {  // whole groups: unrolled, so the shuffles run ahead of the chain
        const double v = q[base + lane];
        float mine = 0.f;
#pragma unroll
        for (int j = 0; j < 32; j++) {
            d1 = (float) ((double) d1 + __shfl_sync(0xffffffffu, v, j));
            if (lane == j) mine = d1;
        }
        D[base + lane] = mine;
    }
    const double v = base + lane < V ? q[base + lane] : 0.0;
    float mine = 0.f;
    for (int j = 0; j < V - base; j++) {
        d1 = (float) ((double) d1 + __shfl_sync(0xffffffffu, v, j));
        if (lane == j) mine = d1;
    }
    if (base + lane < V) D[base + lane] = mine;
}

__device__ __forceinline__ float slot_position(int a) {  // a / (real) table_size
    return __fdiv_rn(__int2float_rn(a), (float) kTableSize);
}

// g_i = first slot a in [0, 1e8) with a / 1e8f > D_i, or 1e8 when there is none.
__global__ void k_table_first_slot(const float *D, int V, long long *g) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const float x = D[i];
    int lo = 0, hi = kTableSize;
    while (lo < hi) {
        int mid = lo + ((hi - lo) >> 1);
        if (slot_position(mid) > x) hi = mid;
        else lo = mid + 1;
    }
    g[i] = lo;
}

// t_0 = 0, t_{i+1} = max(t_i, g_i) + 1, written in place over g.  With u_i = t_i - i this is
// u_0 = 0, u_{i+1} = max(u_i, g_i - i): u_i is the exclusive prefix maximum of g_j - j (floored at
// 0), the same integers as the one-step-at-a-time recurrence.  One block: each thread scans a
// contiguous chunk, the chunk maxima are scanned in shared memory, then each chunk is written.
constexpr int kStartsThreads = 1024;
__global__ void __launch_bounds__(kStartsThreads) k_table_starts(long long *g_then_t, int V) {
    __shared__ long long part[kStartsThreads];
    const long long kNone = -(1LL << 62);
    const int tid = threadIdx.x;
    const int per = (V + kStartsThreads - 1) / kStartsThreads;
    const int lo = min(V, tid * per), hi = min(V, lo + per);
    long long m = kNone;  // max of g_j - j over this thread's chunk
    for (int i = lo; i < hi; i++) m = max(m, g_then_t[i] - i);
    part[tid] = m;
    __syncthreads();
    for (int off = 1; off < kStartsThreads; off <<= 1) {  // inclusive prefix maximum of the chunks
        const long long v = tid >= off ? part[tid - off] : kNone;
        __syncthreads();
        part[tid] = max(part[tid], v);
        __syncthreads();
    }
    long long u = tid == 0 ? 0 : max(0LL, part[tid - 1]);
    for (int i = lo; i < hi; i++) {
        const long long gi = g_then_t[i];
        g_then_t[i] = i + u;
        u = max(u, gi - i);
    }
}

// Fill: slot a holds the last word i with t_i <= a (word V-1 from t_{V-1} on: the clamp).
constexpr int kFillChunk = 1024;
__global__ void k_table_fill(const long long *t, int V, int32_t *table) {
    long long a0 = ((long long) blockIdx.x * blockDim.x + threadIdx.x) * kFillChunk;
    if (a0 >= kTableSize) return;
    int lo = 0, hi = V - 1;  // largest i with t_i <= a0 (t_0 = 0 <= a0)
    while (lo < hi) {
        int mid = lo + ((hi - lo + 1) >> 1);
        if (t[mid] <= a0) lo = mid;
        else hi = mid - 1;
    }
    int i = lo;
    long long a1 = a0 + kFillChunk < kTableSize ? a0 + kFillChunk : kTableSize;
    long long next = (i + 1 < V) ? t[i + 1] : (1LL << 62);
    for (long long a = a0; a < a1; a++) {
        while (a >= next) {
            i++;
            next = (i + 1 < V) ? t[i + 1] : (1LL << 62);
        }
        table[a] = i;
    }
}

cudaError_t launch_build_table(const double *pow_cn, int V, int32_t *table, float *D, long long *g,
                               double *total, cudaStream_t s) {
    double *q = reinterpret_cast<double *>(g);  // the quotients, until the first slots replace them
    k_table_total<<<1, 32, 0, s>>>(pow_cn, V, total);
    k_table_quotients<<<(V + 255) / 256, 256, 0, s>>>(pow_cn, V, total, q);
    k_table_running<<<1, 32, 0, s>>>(q, V, D);
    k_table_first_slot<<<(V + 255) / 256, 256, 0, s>>>(D, V, g);
    k_table_starts<<<1, kStartsThreads, 0, s>>>(g, V);
    const long long chunks = (kTableSize + kFillChunk - 1) / kFillChunk;
    k_table_fill<<<(unsigned) ((chunks + 255) / 256), 256, 0, s>>>(g, V, table);
    return cudaGetLastError();
}

// ---- InitNet (PAR_Word2Vec_cpu.cpp:337-357) ----
// Element i (row-major over [V][d]) takes the LCG state after i + 1 steps from seed 1; each
// thread jumps to the start of its chunk in O(log i) and then steps sequentially.
constexpr int kInitChunk = 256;
__global__ void k_init_net(float *w_in, __nv_bfloat16 *b_in, int V, int d, int ld) {
    const long long n = (long long) V * d;
    const long long s0 = ((long long) blockIdx.x * blockDim.x + threadIdx.x) * kInitChunk;
    if (s0 >= n) return;
    uint64_t r = lcg_jump(1ULL, (uint64_t) s0);
    const long long s1 = s0 + kInitChunk < n ? s0 + kInitChunk : n;
    const float fd = (float) d;
    for (long long i = s0; i < s1; i++) {
        r = lcg_next(r);
        float v = __fdiv_rn(__fsub_rn(__fdiv_rn((float) (r & 0xFFFF), 65536.f), 0.5f), fd);
        long long row = i / d, col = i - row * d;
        if (w_in) w_in[row * ld + col] = v;
        else b_in[row * ld + col] = __float2bfloat16_rn(v);
    }
}

cudaError_t launch_init_net(float *w_in, float *w_out, __nv_bfloat16 *b_in, __nv_bfloat16 *b_out, int V, int d,
                            int ld, cudaStream_t s) {
    const size_t elems = (size_t) V * ld;
    cudaError_t e;
    if (w_in) {
        if ((e = cudaMemsetAsync(w_in, 0, elems * sizeof(float), s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(w_out, 0, elems * sizeof(float), s)) != cudaSuccess) return e;
    } else {
        if ((e = cudaMemsetAsync(b_in, 0, elems * sizeof(__nv_bfloat16), s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(b_out, 0, elems * sizeof(__nv_bfloat16), s)) != cudaSuccess) return e;
    }
    const long long n = (long long) V * d;
    const long long threads = (n + kInitChunk - 1) / kInitChunk;
    k_init_net<<<(unsigned) ((threads + 255) / 256), 256, 0, s>>>(w_in, b_in, V, d, ld);
    return cudaGetLastError();
}

// ---- device rows (V x ld, FP32 or BF16, padding columns zero) <-> dense FP32 rows (V x d) ----
// One warp per row: lanes walk the columns, so both sides are read and written coalesced.
__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ void from_f32(float x, float *p) { *p = x; }
__device__ __forceinline__ void from_f32(float x, __nv_bfloat16 *p) { *p = __float2bfloat16_rn(x); }

template <typename T>
__global__ void k_rows_to_dense(const T *dev, int ld, float *dst, int d, size_t rows) {
    const int lane = threadIdx.x & 31;
    const size_t warps = (size_t) gridDim.x * (blockDim.x >> 5);
    for (size_t r = (size_t) blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
        const T *s = dev + r * (size_t) ld;
        float *o = dst + r * (size_t) d;
        for (int c = lane; c < d; c += 32) o[c] = to_f32(s[c]);
    }
}

template <typename T>
__global__ void k_rows_from_dense(const float *src, int d, T *dev, int ld, size_t rows) {
    const int lane = threadIdx.x & 31;
    const size_t warps = (size_t) gridDim.x * (blockDim.x >> 5);
    for (size_t r = (size_t) blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
        const float *s = src + r * (size_t) d;
        T *o = dev + r * (size_t) ld;
        for (int c = lane; c < ld; c += 32) from_f32(c < d ? s[c] : 0.f, o + c);
    }
}

static unsigned rows_grid(size_t rows) { return (unsigned) std::min<size_t>(148 * 8, (rows + 7) / 8); }

cudaError_t launch_rows_to_dense(const void *dev, bool bf16, int ld, float *dst, int d, size_t rows, cudaStream_t s) {
    if (!rows) return cudaSuccess;
    if (bf16)
        k_rows_to_dense<<<rows_grid(rows), 256, 0, s>>>((const __nv_bfloat16 *) dev, ld, dst, d, rows);
    else
        k_rows_to_dense<<<rows_grid(rows), 256, 0, s>>>((const float *) dev, ld, dst, d, rows);
    return cudaGetLastError();
}

cudaError_t launch_rows_from_dense(const float *src, int d, void *dev, bool bf16, int ld, size_t rows, cudaStream_t s) {
    if (!rows) return cudaSuccess;
    if (bf16)
        k_rows_from_dense<<<rows_grid(rows), 256, 0, s>>>(src, d, (__nv_bfloat16 *) dev, ld, rows);
    else
        k_rows_from_dense<<<rows_grid(rows), 256, 0, s>>>(src, d, (float *) dev, ld, rows);
    return cudaGetLastError();
}

}  // namespace parw2v
