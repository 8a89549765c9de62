// Host-side CUDA helpers shared by the library's translation units: the
// exception that carries a CUDA error to the C-ABI boundary, the CK() check
// and an owning device buffer.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

namespace atrc {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(x)                                                                                     \
    do {                                                                                          \
        cudaError_t err_ = (x);                                                                   \
        if (err_ != cudaSuccess)                                                                  \
            throw ::atrc::CudaError(std::string(#x) + ": " + cudaGetErrorString(err_));           \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    void alloc(size_t b) {
        if (p) { cudaFree(p); p = nullptr; }
        bytes = b;
        if (b) {
            cudaError_t e = cudaMalloc(&p, b);
            if (e != cudaSuccess) {
                p = nullptr;
                bytes = 0;
                throw CudaError(std::string("cudaMalloc of ") + std::to_string(b) + " bytes: " + cudaGetErrorString(e));
            }
        }
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

template <class T>
const T* upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s) {
    if (v.empty()) return nullptr;
    b.alloc(v.size() * sizeof(T));
    CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return b.as<T>();
}

void set_last_error(const std::string& msg);  // capi_host.cpp

}  // namespace atrc
