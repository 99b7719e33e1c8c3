// classes.cuh -- size classes: which kernel and which visited-store placement
// serve an automaton with n states.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sbfs {

// class 0: n <= 8   warp-pooled kernel, 32-byte bitmap per automaton in shared memory
// class 1: n <= 12  warp-pooled kernel, 512-byte bitmap
// class 2: n <= 16  warp-pooled kernel, 8 KiB bitmap
// class 3: n <= 20  one automaton per CTA, bitmap (<= 128 KiB) in shared memory
// class 4: n <= 28  level-synchronous, bitmap (<= 32 MiB) and frontier in HBM
constexpr int kNumClasses = 5;
constexpr int kClassMaxN[kNumClasses] = {8, 12, 16, 20, 28};
// Out-of-range n (0 or > 28) is routed to class 0, whose kernel rejects it
// as a malformed record.

__host__ __device__ __forceinline__ int class_of_n(int n)
{
    return (n >= 1 && n <= 8) ? 0 : n <= 12 ? 1 : n <= 16 ? 2 : n <= 20 ? 3 : n <= 28 ? 4 : 0;
}

struct ClassScratch {
    unsigned long long *hist;     // kNumClasses
    unsigned long long *ranges;   // 2 * kNumClasses: {offset, count}
    unsigned long long *cursor;   // kNumClasses
    int32_t *order;               // count entries
};

// Adds the number of non-negative lengths in len[0..count) to *out.
cudaError_t launch_count_sync(const int32_t *d_len, int64_t count, unsigned long long *out, int sm_count,
                              cudaStream_t st);
cudaError_t launch_classify(const uint8_t *d_ns, int64_t count, ClassScratch sc, int sm_count,
                            cudaStream_t st);

}  // namespace sbfs
