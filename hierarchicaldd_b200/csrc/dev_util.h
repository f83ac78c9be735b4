// Small device-memory helpers shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "hdd_common.h"

namespace hdd {
namespace dev {

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(HDD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* upload(const std::vector<T>& h, cudaStream_t s, size_t& bytes) {
    if (h.empty()) return nullptr;
    T* p = nullptr;
    cudaError_t e = cudaMalloc(&p, h.size() * sizeof(T));
    if (e != cudaSuccess) throw Error(HDD_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ck(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    bytes += h.size() * sizeof(T);
    return p;
}

// Zeroed on the caller's stream: a legacy-stream memset would not be ordered
// before work on the solver's non-blocking stream.
template <class T>
T* alloc_zero(size_t n, size_t& bytes, cudaStream_t s) {
    if (n == 0) return nullptr;
    T* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) throw Error(HDD_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ck(cudaMemsetAsync(p, 0, n * sizeof(T), s), "memset");
    bytes += n * sizeof(T);
    return p;
}

template <class T>
void release(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

}  // namespace dev
}  // namespace hdd
