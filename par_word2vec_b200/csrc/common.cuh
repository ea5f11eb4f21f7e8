// Device helpers shared by the PAR-Word2Vec kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace parw2v {

constexpr int kTableSize = 100000000;  // unigram table entries, PAR_Word2Vec_cpu.cpp:75
constexpr int kExpTableSize = 1000;    // PAR_Word2Vec_cpu.cpp:32
constexpr int kMaxExp = 6;             // PAR_Word2Vec_cpu.cpp:33
constexpr int kMaxSentence = 1000;     // PAR_Word2Vec_cpu.cpp:34
// EXP_TABLE_SIZE / (MAX_EXP * 2.0f) rounded to float, PAR_Word2Vec_cpu.cpp:70
constexpr float kExpResolution = 1000.0f / 12.0f;

// Error bits raised by kernels into the context's device status word.
constexpr unsigned kErrResample = 1u;  // a negative-resampling loop hit its draw limit
constexpr unsigned kErrCapacity = 2u;  // an input exceeded a kernel's fixed capacity
constexpr unsigned kErrStaging = 4u;   // a bulk copy into shared memory did not complete in time

// The reference's linear congruential generator, next = next * 25214903917 + 11 (mod 2^64),
// PAR_Word2Vec_cpu.cpp:461, :532, :591-612.
__host__ __device__ __forceinline__ uint64_t lcg_next(uint64_t x) {
    return x * 25214903917ULL + 11ULL;
}

// Affine map x -> a*x + c (mod 2^64); composing n LCG steps gives a jump-ahead in O(log n).
struct Affine {
    uint64_t a, c;
};
__host__ __device__ __forceinline__ Affine affine_then(Affine first, Affine second) {
    return Affine{second.a * first.a, second.a * first.c + second.c};
}
__host__ __device__ inline uint64_t lcg_jump(uint64_t x, uint64_t n) {
    Affine acc{1ULL, 0ULL}, step{25214903917ULL, 11ULL};
    while (n) {
        if (n & 1ULL) acc = affine_then(acc, step);
        step = affine_then(step, step);
        n >>= 1;
    }
    return acc.a * x + acc.c;
}

// The affine maps of 0..32 LCG steps, for the jumps of the negative draws (at most 32 draws a
// round): kLcgJump.a[n] * x + kLcgJump.c[n] is x after n steps.
struct LcgJumpTable {
    uint64_t a[33], c[33];
};
constexpr LcgJumpTable make_lcg_jump_table() {
    LcgJumpTable t{};
    t.a[0] = 1ULL;
    t.c[0] = 0ULL;
    for (int n = 1; n <= 32; n++) {
        t.a[n] = 25214903917ULL * t.a[n - 1];
        t.c[n] = 25214903917ULL * t.c[n - 1] + 11ULL;
    }
    return t;
}
static __device__ const LcgJumpTable kLcgJump = make_lcg_jump_table();
__device__ __forceinline__ uint64_t lcg_jump_small(uint64_t x, int n) {  // 0 <= n <= 32
    return __ldg(&kLcgJump.a[n]) * x + __ldg(&kLcgJump.c[n]);
}

// x mod m for a 64-bit x and 0 < m < 2^16, exactly, through 32-bit remainders:
// (hi * 2^32 + lo) mod m = ((hi mod m) * (2^32 mod m) + lo mod m) mod m, all terms < 2^32.
__host__ __device__ __forceinline__ uint32_t mod_small(uint64_t x, uint32_t m) {
    const uint32_t r32 = (uint32_t) (0x100000000ULL % m);
    const uint32_t hi = (uint32_t) (x >> 32) % m, lo = (uint32_t) x % m;
    return (hi * r32 % m + lo) % m;
}

// x mod d for a 64-bit x and a divisor 0 < d < 2^16 fixed for a launch, with multiplications
// only (no integer division on the device): Lemire, Kaser & Kurz, "Faster remainder by direct
// computation" (2019): for a 32-bit a, a mod d = high64(low64(M * a) * d), M = floor((2^64-1)/d) + 1;
// a 64-bit x is reduced through its 32-bit halves as in mod_small.  Build it once per thread.
struct FastMod {
    uint64_t M;
    uint32_t d, r32;
    __host__ __device__ explicit FastMod(uint32_t divisor)
        : M(~0ULL / divisor + 1), d(divisor), r32((uint32_t) (0x100000000ULL % divisor)) {}
    __device__ __forceinline__ uint32_t mod32(uint32_t a) const { return (uint32_t) __umul64hi(M * a, d); }
    __device__ __forceinline__ uint32_t operator()(uint64_t x) const {
        return mod32(mod32((uint32_t) (x >> 32)) * r32 + mod32((uint32_t) x));
    }
};

// SplitMix64 finaliser (Steele, Lea & Flood 2014): a bijective 64-bit mixer used to derive
// independent per-token / per-sentence random streams in the Hogwild modes.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// g = (label - sigma(f)) * alpha through the clamped expTable (PAR_Word2Vec_cpu.cpp:554-559 for
// label 1, :642-647 for label 0).  Explicit round-to-nearest intrinsics keep every operation a
// single IEEE rounding, as in the reference built without contraction.  The index is clamped
// into the table, which only matters for a NaN dot product (undefined in the reference).
__device__ __forceinline__ float grad_from_table(float f, int label, float alpha, const float *exp_table) {
    if (f > (float) kMaxExp) return __fmul_rn((float) (label - 1), alpha);
    if (f < -(float) kMaxExp) return __fmul_rn((float) label, alpha);
    int idx = __float2int_rz(__fmul_rn(__fadd_rn(f, (float) kMaxExp), kExpResolution));
    idx = idx < 0 ? 0 : (idx > kExpTableSize ? kExpTableSize : idx);
    return __fmul_rn(__fsub_rn((float) label, exp_table[idx]), alpha);
}

// Warp sum through one integer reduction (redux.sync): each lane's value is clamped to +-32 and
// rounded to a multiple of 2^-20, so the 32 lanes add exactly and in any order, with no overflow
// (32 x 32 x 2^20 = 2^30), and the result carries at most 32 x 2^-21 = 1.5e-5 absolute error.
// One dependent step instead of five shuffles and adds.  For BF16 tables, whose rows are rounded
// at 2^-9 relative, this is far below the storage precision (a dot product's inputs, not the
// reduction, set its accuracy there); FP32 tables keep warp_sum.
__device__ __forceinline__ float warp_sum_fixed(float v) {
    const float c = fminf(fmaxf(v, -32.f), 32.f);
    const int q = __float2int_rn(__fmul_rn(c, 1048576.f));
    return __fmul_rn(__int2float_rn(__reduce_add_sync(0xffffffffu, q)), 1.f / 1048576.f);
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Two warp sums at once: lanes 0-15 reduce p while lanes 16-31 reduce q, then the halves swap
// results; every lane ends with the same P = sum(p) and Q = sum(q) (butterfly additions are
// commutative pairs, so all lanes hold bit-identical sums).  Seven shuffles for two sums.
__device__ __forceinline__ void warp_sum2(float p, float q, int lane, float &P, float &Q) {
    const bool hi = lane & 16;
    float v = hi ? q : p;
    v += __shfl_xor_sync(0xffffffffu, hi ? p : q, 16);
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const float other = __shfl_xor_sync(0xffffffffu, v, 16);
    P = hi ? other : v;
    Q = hi ? v : other;
}

// Fire-and-forget vector reduction into global memory (sm_90+): one L2 atomic per 8 bytes.
__device__ __forceinline__ void red_add_f2(float *addr, float2 v) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(addr), "f"(v.x), "f"(v.y) : "memory");
}

}  // namespace parw2v

namespace parw2v {

// The shared negatives of one repulsion batch (PAR_Word2Vec_cpu.cpp:603-622), drawn by a warp with
// the reference's exact random stream.  Draw k uses LCG state rng_{k+1}; every lane jumps to its
// own state and reads the unigram table at once (one memory latency instead of K dependent ones).
// The candidates are checked against the sentence; the first one found in it is resolved the
// reference's way (uniform redraws until a word outside the sentence), which shifts the stream,
// so the draws after it are redone from the new state.  Returns false if a redraw loop exceeds
// max_resample draws (the reference would spin forever when every word is in the sentence).
static __device__ __noinline__ bool warp_draw_negatives(const int32_t *table, int vocab, uint64_t &rng, const int *sen,
                                                    int len, int K, int *negs, int lane, int64_t max_resample) {
    int k0 = 0;
    while (k0 < K) {
        const int nk = min(K - k0, 32);
        int cand = -1;
        if (lane < nk) {
            const uint64_t r = lcg_jump_small(rng, lane + 1);
            cand = __ldg(table + (r >> 16) % (uint64_t) kTableSize);
            if (!cand) cand = (int) (r % (uint64_t) (vocab - 1) + 1);
        }
        bool hit = false;
        for (int q = 0; q < len; q++) hit |= (sen[q] == cand);
        const unsigned m = __ballot_sync(0xffffffffu, hit && lane < nk);
        const int first = m ? __ffs(m) - 1 : nk;
        if (lane < first) negs[k0 + lane] = cand;
        if (first == nk) {
            rng = lcg_jump_small(rng, nk);
            k0 += nk;
            continue;
        }
        rng = lcg_jump_small(rng, first + 1);
        int s = 0;
        for (int64_t tries = 0;; tries++) {
            if (tries >= max_resample) return false;
            rng = lcg_next(rng);
            s = (int) (rng % (uint64_t) (vocab - 1) + 1);
            bool h2 = false;
            for (int q = lane; q < len; q += 32) h2 |= (sen[q] == s);
            if (!__any_sync(0xffffffffu, h2)) break;
        }
        if (lane == 0) negs[k0 + first] = s;
        k0 += first + 1;
    }
    __syncwarp();
    return true;
}

}  // namespace parw2v
