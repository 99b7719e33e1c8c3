// l2_atomic_peak.cu -- throughput of random 32-bit atomicOr on an L2-resident
// bitmap the size of the n = 28 level slot's (32 MiB): the roof of the level
// engine's wide levels, whose every image is one such test-and-set.  Built and
// run by tests/test_l2_atomic_peak.py.
//
// Every thread keeps kChains independent atomics in flight (the level kernel
// keeps four: two items, two images each) on addresses drawn from a xorshift
// generator; the returned words are folded into a sink so none is dead.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 4;

__global__ void __launch_bounds__(512) k_random_or(uint32_t *bits, uint32_t mask_words, int iters, uint32_t *sink)
{
    uint32_t x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 0x9E3779B9u * (c + 1);
    uint32_t acc = 0;
    for (int it = 0; it < iters; ++it) {
        uint32_t old[kChains];
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            x[c] ^= x[c] << 13;
            x[c] ^= x[c] >> 17;
            x[c] ^= x[c] << 5;
            old[c] = atomicOr(bits + (x[c] & mask_words), 1u << (x[c] >> 27));
        }
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc ^= old[c];
    }
    if (acc == 0x12345678u) sink[0] = acc;
}

}  // namespace

// Random atomicOr per second (billions) on a buffer of 2^log2_words 32-bit
// words, ctas_per_sm x 512 threads per SM; negative on a CUDA error.
extern "C" double l2_random_atomic_gops(int log2_words, int ctas_per_sm, int iters)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return -1.0;
    const size_t words = (size_t)1 << log2_words;
    uint32_t *bits = nullptr, *sink = nullptr;
    if (cudaMalloc(&bits, words * 4) != cudaSuccess) return -2.0;
    if (cudaMalloc(&sink, 4) != cudaSuccess) {
        cudaFree(bits);
        return -2.0;
    }
    cudaMemset(bits, 0, words * 4);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = -3.0;
    const int ctas = sms * ctas_per_sm;
    for (int rep = 0; rep < 3; ++rep) {   // the first pass warms the buffer into L2
        cudaEventRecord(e0);
        k_random_or<<<ctas, 512>>>(bits, (uint32_t)(words - 1), iters, sink);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double gops = (double)ctas * 512 * kChains * iters / (ms * 1e-3) / 1e9;
        if (rep > 0 && gops > best) best = gops;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(bits);
    cudaFree(sink);
    return best;
}
