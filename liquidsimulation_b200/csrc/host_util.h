// Host-side helpers of the engines: the error type every entry point maps to a status code,
// an owning device array, and the CUDA call check.
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "../../include/lsp.h"

namespace lsp {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <typename T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count)
    {
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            throw Error(e == cudaErrorMemoryAllocation ? LSP_ERR_CAPACITY : LSP_ERR_CUDA,
                        std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) + " bytes: " +
                            cudaGetErrorString(e));
        }
        n = count;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
};

#define LSP_CK(call)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            throw ::lsp::Error(LSP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace lsp
