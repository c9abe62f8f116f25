// common.cuh -- shared definitions for the sm_100a TLFEA hot path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "../../include/tlfea_b200.h"

namespace tlfea {

// Quadrature / topology constants (quadrature_utils.h:125-179).
constexpr int T10_NPE = 10;
constexpr int T10_NQP = 5;
constexpr int T4_NPE = 4;
constexpr int T4_NQP = 1;

// Elements per tile: one CTA thread per element.  Power of two (the in-tile
// incidence code packs slot*TE + element).
constexpr int TILE_ELEMS = 128;
constexpr int TILE_SHIFT = 7;
// a tile's block in the tile-ordered node record holds a multiple of this many entries:
// 8 doubles, ints or uint16 are each a multiple of 16 bytes (bulk-copy granularity)
constexpr int TILE_NODE_PAD = 8;

// Number of kernels this library has launched (the bench reports launches
// inside its timed region from the difference of two reads).
extern std::atomic<long long> g_launches;

// Thread-local text of the last error, returned by tlfea_last_error().
void set_error(const std::string& msg);

#define TLFEA_CUDA(call)                                                                              \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            ::tlfea::set_error(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " __FILE__); \
            return TLFEA_CUDA_ERROR;                                                                  \
        }                                                                                             \
    } while (0)

#define TLFEA_LAUNCHED(n) (::tlfea::g_launches.fetch_add((n), std::memory_order_relaxed))

#define TLFEA_CHECK_LAUNCH()                                                                  \
    do {                                                                                      \
        cudaError_t e_ = cudaGetLastError();                                                  \
        if (e_ != cudaSuccess) {                                                              \
            ::tlfea::set_error(std::string("kernel launch: ") + cudaGetErrorString(e_));      \
            return TLFEA_CUDA_ERROR;                                                          \
        }                                                                                     \
        TLFEA_LAUNCHED(1);                                                                    \
    } while (0)

template <typename T>
int dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
        *p = nullptr;
        return TLFEA_CUDA_ERROR;
    }
    return TLFEA_OK;
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// ------------------------------------------------------------ device helpers

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum: warp shuffles, then warp 0 folds the per-warp
// partials in warp order.  Result valid in thread 0.  `red` holds >= 32 T.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    T s = T(0);
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = (lane < nw) ? red[lane] : T(0);
        s = warp_sum(s);
    }
    return s;
}

}  // namespace tlfea
