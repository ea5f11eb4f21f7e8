/*
 * oracle/mkl.h -- TEST INFRASTRUCTURE ONLY (the oracle is the checker, never the
 * product).  A minimal stand-in for the three things PAR_Word2Vec_cpu.cpp takes
 * from Intel MKL (PAR_Word2Vec_cpu.cpp:27, :54, :375, :633-656):
 *
 *   _mm_malloc/_mm_free   -> GCC's <mm_malloc.h>
 *   mkl_set_num_threads   -> no-op (only reached under -DUSE_MKL)
 *   cblas_sgemm           -> a row-major SGEMM with a FIXED summation order
 *
 * MKL is not installed here, so the reference's SGEMM results are unpinned by
 * MKL itself.  This shim pins them: every output element is
 *
 *     acc = 0.0f;  for k = 0 .. K-1 ascending:  acc = acc + op(A)[i][k] * op(B)[k][j]
 *     C[i][j] = (alpha == 1 ? acc : alpha * acc) (+ beta * C[i][j] when beta != 0)
 *
 * with each multiply and add rounded separately (build with -ffp-contract=off).
 * The CUDA deterministic kernel and the C restatement (oracle/parw2v_oracle.c)
 * use exactly this order, which is what makes the repulsion phase bit-exact.
 *
 * The loops run i, k, j so that the innermost loop is over independent output
 * elements (vectorisable by the compiler) while each element still sums k in
 * ascending order; results are identical to the naive i, j, k triple loop.
 */
#ifndef PARW2V_ORACLE_MKL_SHIM_H
#define PARW2V_ORACLE_MKL_SHIM_H

#include <mm_malloc.h>
#include <stdlib.h>
#include <string.h>

enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

static inline void mkl_set_num_threads(int) {}

/* grow-only per-thread scratch (the reference calls this three times per batch) */
static inline float *parw2v_shim_buf(int which, size_t n) {
    static thread_local float *buf[3] = {0, 0, 0};
    static thread_local size_t cap[3] = {0, 0, 0};
    if (n > cap[which]) {
        free(buf[which]);
        buf[which] = (float *) malloc(sizeof(float) * n);
        cap[which] = n;
    }
    return buf[which];
}

static inline void cblas_sgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                               int M, int N, int K, float alpha, const float *A, int lda,
                               const float *B, int ldb, float beta, float *C, int ldc) {
    if (layout != CblasRowMajor || M <= 0 || N <= 0) return;
    const size_t kk = (size_t) (K > 0 ? K : 1);
    /* op(A) as a dense M x K row-major copy, op(B) as a dense K x N row-major copy */
    float *a = parw2v_shim_buf(0, (size_t) M * kk);
    float *b = parw2v_shim_buf(1, kk * (size_t) N);
    float *acc = parw2v_shim_buf(2, (size_t) N);
    for (int i = 0; i < M; i++)
        for (int k = 0; k < K; k++)
            a[(size_t) i * K + k] = (ta == CblasNoTrans) ? A[(size_t) i * lda + k] : A[(size_t) k * lda + i];
    for (int k = 0; k < K; k++)
        for (int j = 0; j < N; j++)
            b[(size_t) k * N + j] = (tb == CblasNoTrans) ? B[(size_t) k * ldb + j] : B[(size_t) j * ldb + k];
    for (int i = 0; i < M; i++) {
        for (int j = 0; j < N; j++) acc[j] = 0.0f;
        for (int k = 0; k < K; k++) {
            const float aik = a[(size_t) i * K + k];
            const float *brow = b + (size_t) k * N;
            for (int j = 0; j < N; j++) {
                float p = aik * brow[j];
                acc[j] = acc[j] + p;
            }
        }
        for (int j = 0; j < N; j++) {
            float v = (alpha == 1.0f) ? acc[j] : alpha * acc[j];
            if (beta != 0.0f) {
                float cb = beta * C[(size_t) i * ldc + j];
                v = v + cb;
            }
            C[(size_t) i * ldc + j] = v;
        }
    }
}

#endif
