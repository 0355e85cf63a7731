// Read-bandwidth probe of this GPU's memory hierarchy.  The roofline of the
// traversal kernel compares its algorithmic bytes with two denominators: the
// HBM copy bandwidth and the bandwidth at which the SMs can stream data that
// sits in L2.  This kernel measures the second (and, with a buffer larger
// than L2, the first): every thread of a persistent grid streams 16-byte
// loads over the buffer with L1 bypassed (ld.global.cg) and keeps a running
// sum, so no load can be dropped.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/tinypt_cuda.h"

namespace {

__global__ void __launch_bounds__(512) k_read(const uint4* __restrict__ p, size_t n16, int reps,
                                              unsigned* __restrict__ sink) {
    unsigned acc = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r) {
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride) {
            const uint4 v = __ldcg(p + i);
            acc += v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    // a data-dependent store: the loads cannot be optimised away
    if (acc == 0x9e3779b9u) sink[blockIdx.x] = acc;
}

struct Cleanup {
    void* buf = nullptr;
    unsigned* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Cleanup() {
        if (buf) cudaFree(buf);
        if (sink) cudaFree(sink);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

}  // namespace

extern "C" int tpt_probe_read_bandwidth(int64_t bytes, int reps, double* gbs_out) {
    if (bytes < (1 << 20) || bytes > (int64_t(1) << 34) || reps < 1 || reps > 1000 || !gbs_out) return TPT_ERR_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return TPT_ERR_CUDA;
    Cleanup c;
    const size_t n16 = (size_t)bytes / 16;
    if (cudaMalloc(&c.buf, n16 * 16) != cudaSuccess) return TPT_ERR_ALLOC;
    if (cudaMalloc(&c.sink, 4096 * sizeof(unsigned)) != cudaSuccess) return TPT_ERR_ALLOC;
    if (cudaMemset(c.buf, 0x5a, n16 * 16) != cudaSuccess) return TPT_ERR_CUDA;
    if (cudaEventCreate(&c.e0) != cudaSuccess || cudaEventCreate(&c.e1) != cudaSuccess) return TPT_ERR_CUDA;
    const int grid = sms * 4;  // 4 blocks of 512 threads per SM: 64 warps
    const uint4* p = static_cast<const uint4*>(c.buf);
    k_read<<<grid, 512>>>(p, n16, 1, c.sink);  // warm-up: brings the buffer into L2 if it fits
    cudaEventRecord(c.e0);
    k_read<<<grid, 512>>>(p, n16, reps, c.sink);
    cudaEventRecord(c.e1);
    if (cudaEventSynchronize(c.e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) return TPT_ERR_CUDA;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c.e0, c.e1);
    if (ms <= 0.0f) return TPT_ERR_CUDA;
    *gbs_out = (double)(n16 * 16) * reps / (ms * 1e-3) / 1e9;
    return TPT_OK;
}
