// Warp-level tensor-core and BF16 helpers shared by the BATCHED kernels (sm_100a): ldmatrix
// fragment loads, the m16n8k16 BF16 MMA with FP32 accumulation, stochastic rounding of FP32 pairs
// to BF16, and the per-lane random bits that rounding draws on.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace parw2v {

// Stochastic rounding of a pair FP32 -> BF16 with the sm_100a conversion cvt.rs: each element
// takes 16 random bits (v.x the low half of h, v.y the high half), adds them below the kept
// mantissa and truncates; Inf and NaN pass through.
__device__ __forceinline__ unsigned pack_sr2(float2 v, uint64_t h) {
    unsigned d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(v.y), "f"(v.x), "r"((unsigned) h));
    return d;
}

// Per-lane stream of random bits for stochastic rounding: a 32-bit LCG (multiplier 747796405,
// increment 2891336453) with its high half folded into the low half, so both 16-bit fields of a
// word carry high-order bits.  One step serves the four values of a float4 write-back: the second
// pair takes the word with its halves swapped, so each value still sees a uniform 16-bit field
// (each rounding stays unbiased; values 0 and 3, 1 and 2 share a field).  Against two steps per
// float4 this measured 1.5% faster with no loss of planted-cluster recall.
struct LaneBits {
    uint32_t s;
    __device__ __forceinline__ uint32_t step() {
        s = s * 747796405u + 2891336453u;
        return s ^ (s >> 16);
    }
    __device__ __forceinline__ uint64_t next() {
        const uint32_t lo = step();
        return ((uint64_t) __funnelshift_l(lo, lo, 16) << 32) | lo;
    }
};

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void *p) {
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const void *p) {
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned (&r)[2], const void *p) {
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(a));
}
__device__ __forceinline__ void ldsm_x2(unsigned (&r)[2], const void *p) {
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(a));
}
// Inverse of ldsm_x2_t: lane (g, t) holds {M[2t][g], M[2t+1][g]} of two 8x8 BF16 matrices and the
// lanes 0..15 give the addresses of their rows (lanes 0-7 matrix 0, 8-15 matrix 1).
__device__ __forceinline__ void stsm_x2_t(void *p, unsigned r0, unsigned r1) {
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("stmatrix.sync.aligned.m8n8.x2.trans.shared.b16 [%0], {%1, %2};" ::"r"(a), "r"(r0), "r"(r1) : "memory");
}
// D += A (16x16 bf16, row) * B (16x8 bf16, col), FP32 accumulate
__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// d = a b: the same product with a zero accumulator input (no registers to clear first)
__device__ __forceinline__ void mma16816_z(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%10,%10,%10,%10};"
                 : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(0.f));
}


// ---- FP32 operands on the tensor cores: 3xTF32 ----
// x = big + small with both parts TF32 (cvt.rna), and a*b ~ big_a*big_b + big_a*small_b +
// small_a*big_b: the products keep about FP32's precision (the dropped small*small term is below
// 2^-22 of the product) at three m16n8k8 TF32 MMAs.
__device__ __forceinline__ unsigned tf32_bits(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, unsigned &big, unsigned &small) {
    big = tf32_bits(x);
    small = tf32_bits(x - __uint_as_float(big));
}
// D += A (16x8 tf32, row) * B (8x8 tf32, col), FP32 accumulate
__device__ __forceinline__ void mma1688(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// split FP32 fragments for 3xTF32
__device__ __forceinline__ void split_a(const float (&a)[4], unsigned (&big)[4], unsigned (&small)[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) split_tf32(a[i], big[i], small[i]);
}
__device__ __forceinline__ void mma3xtf32(float (&d)[4], const unsigned (&abig)[4], const unsigned (&asmall)[4],
                                          const unsigned (&bbig)[2], const unsigned (&bsmall)[2]) {
    mma1688(d, asmall, bbig[0], bbig[1]);
    mma1688(d, abig, bsmall[0], bsmall[1]);
    mma1688(d, abig, bbig[0], bbig[1]);
}
// ldmatrix of 32-bit elements: an 8 x 4 block of floats is an 8 x 8 block of 16-bit halves, so a
// lane receives the float at (its row / 4, its lane % 4) of each block
__device__ __forceinline__ void ldsm_x4_f32(float (&r)[4], const void *p) {
    unsigned u[4];
    ldsm_x4(u, p);
#pragma unroll
    for (int i = 0; i < 4; i++) r[i] = __uint_as_float(u[i]);
}

}  // namespace parw2v
