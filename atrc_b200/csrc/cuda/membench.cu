// Streaming-read bandwidth of the device's memory hierarchy, the denominator
// of the traversal kernels' roofline.  No counterpart in the reference (which
// has no GPU code).
//
// A buffer of `bytes` is read `passes` times with 16-byte loads that bypass
// L1 (ld.global.cg), four independent loads in flight per thread, by a grid
// of resident blocks (the SM count x 4 blocks of 512 threads) striding over
// the buffer.  A buffer well inside the L2 cache (126 MB on B200; a few tens
// of MB) measures L2 read bandwidth after the first pass has loaded it; a
// buffer of several GB measures HBM read bandwidth.  Each thread folds what it
// read into one word and stores it only when it equals a value the caller can
// never make appear, so the loads cannot be optimised away and nothing else is
// written.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../../include/atrc_cuda.h"
#include "cuda_util.h"

namespace {

__global__ void __launch_bounds__(512) k_stream_read(const uint4* __restrict__ buf, size_t n, int passes,
                                                     unsigned* __restrict__ sink) {
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    unsigned acc = 0;
    for (int pass = 0; pass < passes; ++pass) {
        size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
        for (; i + 3 * stride < n; i += 4 * stride) {
            const uint4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride);
            const uint4 c = __ldcg(buf + i + 2 * stride), d = __ldcg(buf + i + 3 * stride);
            acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
        }
        for (; i < n; i += stride) {
            const uint4 a = __ldcg(buf + i);
            acc ^= a.x ^ a.y ^ a.z ^ a.w;
        }
        acc = acc * 2654435761u + unsigned(pass);
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;  // the buffer is zero-filled: never taken in practice
}

int fail_status(int code, const std::string& msg) {
    atrc::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int atrc_cuda_stream_read_gbs(int device, uint64_t bytes, int passes, double* gbs) {
    if (!gbs || passes < 2 || bytes < (1u << 20) || bytes % 16)
        return fail_status(ATRC_ERR_INVALID_ARG,
                                      "atrc_cuda_stream_read_gbs: need gbs, passes >= 2 and a multiple of 16 bytes >= 1 MiB");
    *gbs = 0;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail_status(ATRC_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    void* buf = nullptr;
    unsigned* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    auto cleanup = [&] {
        if (ev[0]) cudaEventDestroy(ev[0]);
        if (ev[1]) cudaEventDestroy(ev[1]);
        if (s) cudaStreamDestroy(s);
        if (buf) cudaFree(buf);
        if (sink) cudaFree(sink);
    };
    if ((e = cudaMalloc(&buf, bytes)) != cudaSuccess || (e = cudaMalloc(&sink, sizeof(unsigned))) != cudaSuccess) {
        cleanup();
        return fail_status(ATRC_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ev[0])) != cudaSuccess || (e = cudaEventCreate(&ev[1])) != cudaSuccess ||
        (e = cudaMemsetAsync(buf, 0, bytes, s)) != cudaSuccess) {
        cleanup();
        return fail_status(ATRC_ERR_CUDA, cudaGetErrorString(e));
    }
    const size_t n = bytes / 16;
    const int grid = std::max(1, sms) * 4;
    // one untimed pass loads the buffer into L2 (when it fits) and warms up
    k_stream_read<<<grid, 512, 0, s>>>(static_cast<const uint4*>(buf), n, 1, sink);
    cudaEventRecord(ev[0], s);
    k_stream_read<<<grid, 512, 0, s>>>(static_cast<const uint4*>(buf), n, passes, sink);
    cudaEventRecord(ev[1], s);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaEventSynchronize(ev[1])) != cudaSuccess) {
        cleanup();
        return fail_status(ATRC_ERR_CUDA, cudaGetErrorString(e));
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    cleanup();
    *gbs = double(bytes) * passes / (double(ms) * 1e-3) / 1e9;
    return ATRC_OK;
}
