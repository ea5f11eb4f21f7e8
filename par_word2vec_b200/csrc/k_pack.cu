// Subsampling + sentence packing for the Hogwild modes.
//
// The reference assembles sentences one at a time on each CPU thread (PAR_Word2Vec_cpu.cpp:447-471)
// and the GPU reference packs once, on the host, into CSR offsets (PAR_Word2Vec_gpu_text.cu:785-828).
// Here every epoch re-subsamples on the device (the CPU semantics) with a counter-based random
// stream, so the decision for token i depends only on (seed, epoch, i):
//   keep(i) = corpus[i] != 0  &&  !(keep_thr[w] < (mix64(key + i) & 0xFFFF) / 65536)
// which has the reference's keep probability (the same 16-bit quantised uniform).  Kept tokens
// are compacted in corpus order into `packed`, and for every "</s>" the number of kept tokens
// before it is written to `line_end`, so line L owns packed[line_end[L-1] .. line_end[L]).
// A trailing line without "</s>" is not trained, as the reference drops it (:472).  Lines longer
// than 1000 kept tokens are cut into 1000-token sentences by the trainers (:467).
//
// Two passes over the corpus (count, then write) with a one-CTA scan of per-tile totals in
// between: 3 x 4 bytes/token of HBM traffic for the corpus reads and packed writes.
#include "common.cuh"
#include "internal.h"

namespace parw2v {

namespace {

constexpr int kPackThreads = 256;
constexpr int kPerThread = 16;
constexpr int kTile = kPackThreads * kPerThread;  // 4096 tokens

__device__ __forceinline__ uint64_t keep_key(uint64_t seed, int epoch) {
    return mix64(seed ^ (0x5851F42D4C957F2DULL * (uint64_t) (epoch + 1)));
}

// Loads the thread's 16 tokens (zero past the end) and returns bit masks of kept / "</s>" tokens.
__device__ __forceinline__ void token_flags(const TrainArgs &a, uint64_t base, int tok[kPerThread],
                                            unsigned &kept_mask, unsigned &zero_mask) {
    const uint64_t key = keep_key(a.seed, (int) __ldg(&a.cnt->epoch));
    kept_mask = 0;
    zero_mask = 0;
    if (base + kPerThread <= a.n_tokens) {
        const int4 *p = reinterpret_cast<const int4 *>(a.corpus + base);
#pragma unroll
        for (int v = 0; v < kPerThread / 4; v++) {
            int4 q = __ldg(p + v);
            tok[4 * v] = q.x; tok[4 * v + 1] = q.y; tok[4 * v + 2] = q.z; tok[4 * v + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kPerThread; j++) tok[j] = (base + j < a.n_tokens) ? a.corpus[base + j] : -1;
    }
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
        const int w = tok[j];
        if (w == 0) {
            zero_mask |= 1u << j;
        } else if (w > 0) {
            bool keep = true;
            if (a.sample > 0) {
                const float u = __fdiv_rn((float) (mix64(key + base + j) & 0xFFFF), 65536.f);
                keep = !(__ldg(a.keep_thr + w) < u);
            }
            if (keep) kept_mask |= 1u << j;
        }
    }
}

// Exclusive block scan of two counters; the block totals come back through tot_a / tot_b.
__device__ __forceinline__ void block_scan2(unsigned va, unsigned vb, unsigned &ea, unsigned &eb, unsigned &tot_a,
                                            unsigned &tot_b) {
    constexpr int kWarps = kPackThreads / 32;
    __shared__ unsigned wa[kWarps], wb[kWarps], sum_a, sum_b;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned ia = va, ib = vb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned ta = __shfl_up_sync(0xffffffffu, ia, o), tb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o) { ia += ta; ib += tb; }
    }
    if (lane == 31) { wa[wid] = ia; wb[wid] = ib; }
    __syncthreads();
    if (wid == 0) {
        const unsigned xa = lane < kWarps ? wa[lane] : 0, xb = lane < kWarps ? wb[lane] : 0;
        unsigned sa = xa, sb = xb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned ta = __shfl_up_sync(0xffffffffu, sa, o), tb = __shfl_up_sync(0xffffffffu, sb, o);
            if (lane >= o) { sa += ta; sb += tb; }
        }
        if (lane < kWarps) { wa[lane] = sa - xa; wb[lane] = sb - xb; }
        if (lane == kWarps - 1) { sum_a = sa; sum_b = sb; }
    }
    __syncthreads();
    ea = wa[wid] + ia - va;
    eb = wb[wid] + ib - vb;
    tot_a = sum_a;
    tot_b = sum_b;
}

__global__ void __launch_bounds__(kPackThreads) k_pack_count(TrainArgs a, uint32_t *tile_kept, uint32_t *tile_zero) {
    const uint64_t base = (uint64_t) blockIdx.x * kTile + (uint64_t) threadIdx.x * kPerThread;
    int tok[kPerThread];
    unsigned km, zm;
    token_flags(a, base, tok, km, zm);
    unsigned ek, ez, tk = 0, tz = 0;
    block_scan2(__popc(km), __popc(zm), ek, ez, tk, tz);
    if (threadIdx.x == 0) {
        tile_kept[blockIdx.x] = tk;
        tile_zero[blockIdx.x] = tz;
    }
}

// One CTA: exclusive scans of the per-tile totals, in place; grand totals into the counters.
__global__ void __launch_bounds__(1024) k_pack_scan(uint32_t *tile_kept, uint32_t *tile_zero, uint64_t n_tiles,
                                                    DevCounters *cnt) {
    __shared__ unsigned long long sk[1024], sz[1024];
    const uint64_t per = (n_tiles + 1023) / 1024;
    const uint64_t t0 = threadIdx.x * per, t1 = t0 + per < n_tiles ? t0 + per : n_tiles;
    unsigned long long k = 0, z = 0;
    for (uint64_t t = t0; t < t1; t++) { k += tile_kept[t]; z += tile_zero[t]; }
    sk[threadIdx.x] = k;
    sz[threadIdx.x] = z;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // Hillis-Steele inclusive scan
        unsigned long long ak = threadIdx.x >= o ? sk[threadIdx.x - o] : 0;
        unsigned long long az = threadIdx.x >= o ? sz[threadIdx.x - o] : 0;
        __syncthreads();
        sk[threadIdx.x] += ak;
        sz[threadIdx.x] += az;
        __syncthreads();
    }
    unsigned long long rk = sk[threadIdx.x] - k, rz = sz[threadIdx.x] - z;
    for (uint64_t t = t0; t < t1; t++) {
        unsigned ck = tile_kept[t], cz = tile_zero[t];
        tile_kept[t] = (uint32_t) rk;
        tile_zero[t] = (uint32_t) rz;
        rk += ck;
        rz += cz;
    }
    if (threadIdx.x == 1023) {
        cnt->total_kept = sk[1023];
        cnt->n_lines = sz[1023];
    }
}

__global__ void __launch_bounds__(kPackThreads) k_pack_write(TrainArgs a, const uint32_t *tile_kept,
                                                            const uint32_t *tile_zero, int32_t *packed,
                                                            uint32_t *line_end) {
    const uint64_t base = (uint64_t) blockIdx.x * kTile + (uint64_t) threadIdx.x * kPerThread;
    int tok[kPerThread];
    unsigned km, zm;
    token_flags(a, base, tok, km, zm);
    unsigned ek, ez, tk, tz;
    block_scan2(__popc(km), __popc(zm), ek, ez, tk, tz);
    uint32_t ok = tile_kept[blockIdx.x] + ek, oz = tile_zero[blockIdx.x] + ez;
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
        if (km & (1u << j)) packed[ok++] = tok[j];
        if (zm & (1u << j)) line_end[oz++] = ok;
    }
}

__global__ void k_count_zeros(const int32_t *corpus, uint64_t n, DevCounters *cnt) {
    unsigned long long z = 0;
    for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x)
        z += (corpus[i] == 0);
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    if ((threadIdx.x & 31) == 0 && z) atomicAdd(&cnt->n_lines, z);
}

}  // namespace

uint64_t pack_tiles(uint64_t n_tokens) { return (n_tokens + kTile - 1) / kTile; }

static __global__ void k_advance_epoch(DevCounters *cnt) { cnt->epoch += 1; }

cudaError_t launch_advance_epoch(DevCounters *cnt, cudaStream_t s) {
    k_advance_epoch<<<1, 1, 0, s>>>(cnt);
    return cudaGetLastError();
}

cudaError_t launch_count_zeros(const int32_t *corpus, uint64_t n, DevCounters *cnt, cudaStream_t s) {
    k_count_zeros<<<148 * 4, 256, 0, s>>>(corpus, n, cnt);
    return cudaGetLastError();
}

cudaError_t launch_pack(const TrainArgs &a, int32_t *packed, uint32_t *line_end, uint32_t *tile_kept,
                        uint32_t *tile_zero, uint64_t n_tiles, cudaStream_t s) {
    if (n_tiles == 0) return cudaSuccess;
    k_pack_count<<<(unsigned) n_tiles, kPackThreads, 0, s>>>(a, tile_kept, tile_zero);
    k_pack_scan<<<1, 1024, 0, s>>>(tile_kept, tile_zero, n_tiles, a.cnt);
    k_pack_write<<<(unsigned) n_tiles, kPackThreads, 0, s>>>(a, tile_kept, tile_zero, packed, line_end);
    return cudaGetLastError();
}

}  // namespace parw2v
