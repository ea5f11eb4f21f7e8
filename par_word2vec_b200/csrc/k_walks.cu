// Uniform random walks over a graph on the GPU: the input of the graph workload
// (PAR_Word2Vec_gpu_graph trains on walk files made outside the reference, data.sh:7-11).
//
// Walk w (0 <= w < walks_per_node * n_nodes) starts at node w mod n_nodes, so every node starts
// walks_per_node walks, in rounds over the nodes.  Step s > 0 moves from the current node v to
// its neighbour indices[indptr[v] + j] with j = (hi32(h) * deg(v)) >> 32 and
// h = mix64(seed ^ mix64(w * 2^20 + s)): a counter-based draw, so any walk can be recomputed on its
// own (the tests restate it in numpy) and the result does not depend on the launch shape.  A node
// without neighbours ends its walk there: the remaining steps repeat it.
#include "common.cuh"
#include "internal.h"

namespace parw2v {
namespace {

__device__ __forceinline__ uint64_t walk_hash(uint64_t seed, uint64_t walk, int step) {
    return mix64(seed ^ mix64((walk << 20) + (uint64_t) step));
}

__global__ void k_random_walks(const int64_t *indptr, const int32_t *indices, int n_nodes, uint64_t n_walks,
                               int walk_len, uint64_t seed, int32_t *out) {
    for (uint64_t w = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; w < n_walks;
         w += (uint64_t) gridDim.x * blockDim.x) {
        int v = (int) (w % (uint64_t) n_nodes);
        int32_t *o = out + w * (uint64_t) walk_len;
        o[0] = v;
        for (int s = 1; s < walk_len; s++) {
            const int64_t lo = __ldg(indptr + v), deg = __ldg(indptr + v + 1) - lo;
            if (deg > 0) {
                const uint64_t h = walk_hash(seed, w, s);
                v = __ldg(indices + lo + (int64_t) (((h >> 32) * (uint64_t) deg) >> 32));
            }
            o[s] = v;
        }
    }
}

}  // namespace
}  // namespace parw2v

using namespace parw2v;

extern "C" int parw2v_random_walks(const int64_t *indptr, const int32_t *indices, int n_nodes, int walks_per_node,
                                   int walk_len, uint64_t seed, int device, int32_t *out_nodes) {
    if (!indptr || !indices || !out_nodes || n_nodes < 1 || walks_per_node < 1 || walk_len < 1 || walk_len > (1 << 20))
        return set_global_error(PARW2V_ERR_ARG, "random walks: invalid argument");
    const int64_t n_edges = indptr[n_nodes];
    if (indptr[0] != 0 || n_edges < 0) return set_global_error(PARW2V_ERR_ARG, "random walks: indptr must start at 0");
    for (int v = 0; v < n_nodes; v++)
        if (indptr[v + 1] < indptr[v]) return set_global_error(PARW2V_ERR_ARG, "random walks: indptr must not decrease");
    for (int64_t e = 0; e < n_edges; e++)
        if (indices[e] < 0 || indices[e] >= n_nodes)
            return set_global_error(PARW2V_ERR_ARG, "random walks: neighbour id outside [0, n_nodes)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_global_error(PARW2V_ERR_NODEV, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return set_global_error(PARW2V_ERR_ARG, "device ordinal out of range");
    cudaError_t e = cudaSetDevice(device);
    const uint64_t n_walks = (uint64_t) walks_per_node * (uint64_t) n_nodes;
    const size_t out_bytes = sizeof(int32_t) * n_walks * (uint64_t) walk_len;
    int64_t *d_indptr = nullptr;
    int32_t *d_indices = nullptr, *d_out = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&d_indptr, sizeof(int64_t) * ((size_t) n_nodes + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_indices, sizeof(int32_t) * (size_t) (n_edges > 0 ? n_edges : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, out_bytes);
    if (e == cudaSuccess)
        e = cudaMemcpy(d_indptr, indptr, sizeof(int64_t) * ((size_t) n_nodes + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n_edges > 0)
        e = cudaMemcpy(d_indices, indices, sizeof(int32_t) * (size_t) n_edges, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const uint64_t blocks = (n_walks + 255) / 256;
        k_random_walks<<<(unsigned) (blocks < 148 * 64 ? blocks : 148 * 64), 256>>>(d_indptr, d_indices, n_nodes, n_walks,
                                                                                  walk_len, seed, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out_nodes, d_out, out_bytes, cudaMemcpyDeviceToHost);
    cudaFree(d_indptr);
    cudaFree(d_indices);
    cudaFree(d_out);
    if (e != cudaSuccess) {
        const int code = e == cudaErrorMemoryAllocation ? PARW2V_ERR_OOM : PARW2V_ERR_CUDA;
        return set_global_error(code, (std::string("random walks: ") + cudaGetErrorString(e)).c_str());
    }
    return PARW2V_OK;
}
