// k_classify.cu -- bucket a mixed-size batch by size class on the device.
//
// The reference bakes one n into the kernel at JIT time (GlobalVariableSymbol,
// GPGPU/GPU/SlimGPUQueue.cs:21,78,216) and therefore cannot run mixed sizes in
// one batch (AlgorithmCorrectnessTestProject/IntegrityTest.cs:68-70).  Here a
// batch with per-automaton n is split into size classes by three small
// kernels (histogram, offsets, scatter) whose output -- an order array and a
// (offset, count) pair per class -- feeds each class's persistent kernel
// without a round trip to the host, so the whole chain can be captured in a
// CUDA graph.
#include "classes.cuh"
#include "common.cuh"

namespace sbfs {
namespace {

__global__ void k_hist(const uint8_t *ns, int64_t count, unsigned long long *hist)
{
    __shared__ unsigned int h[kNumClasses];
    if (threadIdx.x < kNumClasses) h[threadIdx.x] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[class_of_n(ns[i])], 1u);
    __syncthreads();
    if (threadIdx.x < kNumClasses && h[threadIdx.x])
        atomicAdd(&hist[threadIdx.x], (unsigned long long)h[threadIdx.x]);
}

// hist[c] -> ranges[c] = {offset, count}; cursor[c] = offset
__global__ void k_offsets(const unsigned long long *hist, unsigned long long *ranges,
                          unsigned long long *cursor)
{
    if (threadIdx.x == 0) {
        unsigned long long off = 0;
        for (int c = 0; c < kNumClasses; ++c) {
            ranges[2 * c] = off;
            ranges[2 * c + 1] = hist[c];
            cursor[c] = off;
            off += hist[c];
        }
    }
}

__global__ void k_scatter(const uint8_t *ns, int64_t count, unsigned long long *cursor, int32_t *order)
{
    const int lane = threadIdx.x & 31;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) & ~31ll; base < count;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + lane;
        const int c = i < count ? class_of_n(ns[i]) : -1;
#pragma unroll
        for (int k = 0; k < kNumClasses; ++k) {
            const unsigned m = __ballot_sync(kFull, c == k);
            if (!m) continue;
            unsigned long long pos = 0;
            const int leader = __ffs(m) - 1;
            if (lane == leader) pos = atomicAdd(&cursor[k], (unsigned long long)__popc(m));
            pos = __shfl_sync(kFull, pos, leader);
            if (c == k) order[pos + __popc(m & ((1u << lane) - 1u))] = (int32_t)i;
        }
    }
}

// out += number of lengths >= 0 (synchronizing automata); one atomic per block
__global__ void k_count_sync(const int32_t *len, int64_t count, unsigned long long *out)
{
    __shared__ unsigned int part[32];
    unsigned int c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        c += __ldcg(len + i) >= 0;
    c = __reduce_add_sync(kFull, c);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned int v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0u;
        v = __reduce_add_sync(kFull, v);
        if (threadIdx.x == 0 && v) atomicAdd(out, (unsigned long long)v);
    }
}

}  // namespace

cudaError_t launch_count_sync(const int32_t *d_len, int64_t count, unsigned long long *out, int sm_count,
                              cudaStream_t st)
{
    const int threads = 256;
    const int64_t want = (count + threads - 1) / threads;
    const int blocks = (int)(want < 1 ? 1 : (want > 2 * sm_count ? 2 * sm_count : want));
    k_count_sync<<<blocks, threads, 0, st>>>(d_len, count, out);
    return cudaGetLastError();
}

cudaError_t launch_classify(const uint8_t *d_ns, int64_t count, ClassScratch sc, int sm_count,
                            cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(sc.hist, 0, kNumClasses * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int threads = 256;
    int64_t want = (count + threads - 1) / threads;
    const int blocks = (int)(want < 1 ? 1 : (want > 4 * sm_count ? 4 * sm_count : want));
    k_hist<<<blocks, threads, 0, st>>>(d_ns, count, sc.hist);
    k_offsets<<<1, 32, 0, st>>>(sc.hist, sc.ranges, sc.cursor);
    k_scatter<<<blocks, threads, 0, st>>>(d_ns, count, sc.cursor, sc.order);
    return cudaGetLastError();
}

}  // namespace sbfs
