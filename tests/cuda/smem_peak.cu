// smem_peak.cu -- shared-memory throughput of one SM, in bytes per SM clock:
// the denominator of the on-chip roofline of the BFS kernels.  Built and run by
// tests/test_smem_peak.py.
//
// One CTA of 1024 threads per SM.  Every lane reads 32-bit words of its own
// column of a lane-interleaved array ([element][lane]: the 32 lanes of a warp
// touch 32 different banks, as the per-lane BFS kernel's accesses do), eight
// independent loads per step so that the pipe, not latency, sets the rate.
// The SM's own cycle counter (clock64) brackets the loop, so the result does
// not depend on the clock frequency.  A second kernel measures 32-bit shared
// atomicOr the same way.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

constexpr int kThreads = 1024;
constexpr int kElems = 64;   // per lane: 64 x 32 x 4 B = 8 KiB

__device__ __forceinline__ uint32_t lds(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"((uint32_t)__cvta_generic_to_shared(p)));
    return v;
}

__device__ __forceinline__ uint32_t atom_or(uint32_t *p, uint32_t x)
{
    uint32_t v;
    asm volatile("atom.shared.or.b32 %0, [%1], %2;" : "=r"(v) : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(x));
    return v;
}

__global__ void __launch_bounds__(kThreads) k_read(int iters, unsigned long long *cycles, uint32_t *sink)
{
    __shared__ uint32_t buf[kElems * 32];
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kElems * 32; i += blockDim.x) buf[i] = (uint32_t)i * 2654435761u;
    __syncthreads();
    uint32_t a[8] = {};
    const long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] ^= lds(&buf[(((it << 3) + j) & (kElems - 1)) * 32 + lane]);
    }
    __syncthreads();
    const long long t1 = clock64();
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) x ^= a[j];
    if (x == 0x12345678u) sink[0] = x;
    if (threadIdx.x == 0) cycles[blockIdx.x] = (unsigned long long)(t1 - t0);
}

__global__ void __launch_bounds__(kThreads) k_atomic(int iters, unsigned long long *cycles, uint32_t *sink)
{
    __shared__ uint32_t buf[kElems * 32];
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kElems * 32; i += blockDim.x) buf[i] = 0u;
    __syncthreads();
    uint32_t a[8] = {};
    const long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
            a[j] ^= atom_or(&buf[(((it << 3) + j) & (kElems - 1)) * 32 + lane], 1u << ((it + j) & 31));
    }
    __syncthreads();
    const long long t1 = clock64();
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) x ^= a[j];
    if (x == 0x12345678u) sink[0] = x;
    if (threadIdx.x == 0) cycles[blockIdx.x] = (unsigned long long)(t1 - t0);
}

}  // namespace

// Bytes (32-bit lane-interleaved loads, or atomicOr operands) per SM clock,
// averaged over one CTA per SM; negative on a CUDA error.
extern "C" double smem_bytes_per_clk(int atomics, int iters)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return -1.0;
    unsigned long long *d_cycles = nullptr;
    uint32_t *d_sink = nullptr;
    if (cudaMalloc(&d_cycles, sizeof(unsigned long long) * sms) != cudaSuccess) return -2.0;
    if (cudaMalloc(&d_sink, sizeof(uint32_t)) != cudaSuccess) {
        cudaFree(d_cycles);
        return -2.0;
    }
    double result = -3.0;
    for (int rep = 0; rep < 2; ++rep) {   // the first launch warms up
        if (atomics) k_atomic<<<sms, kThreads>>>(iters, d_cycles, d_sink);
        else k_read<<<sms, kThreads>>>(iters, d_cycles, d_sink);
        if (cudaDeviceSynchronize() != cudaSuccess) break;
        unsigned long long *h = new unsigned long long[sms];
        if (cudaMemcpy(h, d_cycles, sizeof(unsigned long long) * sms, cudaMemcpyDeviceToHost) == cudaSuccess) {
            double cyc = 0;
            for (int i = 0; i < sms; ++i) cyc += (double)h[i];
            cyc /= sms;
            result = (double)kThreads * 8.0 * 4.0 * (double)iters / cyc;
        }
        delete[] h;
    }
    cudaFree(d_cycles);
    cudaFree(d_sink);
    return result;
}
