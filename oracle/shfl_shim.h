/* oracle/shfl_shim.h -- TEST INFRASTRUCTURE ONLY.
 * Force-included when the reference's GPU graph program (PAR_Word2Vec_gpu_graph.cu) is built for
 * sm_100a: the reference calls the pre-Volta __shfl_down, which current CUDA does not offer for
 * sm_70 and later.  In the reference every call is made by all 32 lanes of warp 0, so the
 * full-mask synchronising form computes the same values. */
#pragma once
#define __shfl_down(v, delta) __shfl_down_sync(0xffffffffu, (v), (delta))
