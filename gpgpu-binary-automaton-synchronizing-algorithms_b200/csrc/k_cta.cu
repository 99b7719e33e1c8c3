// k_cta.cu -- power-set BFS with one automaton per CTA (n <= 20).
//
// The visited bitmap (2^n bits, up to 128 KiB at n = 20) lives in shared
// memory; the level-ordered queue lives in a per-CTA global area of 2^n
// 64-bit entries (subset | parent index << 32 | letter-is-b << 63), which is
// retained for the word (GPGPU/CPU/CPU.cs:203-205,262-269).  Images come from
// byte tables in shared memory: table[c][v] = (a-image << 32) | b-image of the
// states 8c..8c+7 selected by v, so an image is ceil(n/8) loads (the 4-bit
// table of GPGPU/CPU/SlimCPU4bits.cs:122-206 widened to bytes).  The CTA
// expands one level at a time (grid-stride over the level's queue slice),
// appends new subsets with one shared atomic per warp, and moves to the next
// level after a barrier -- the level-synchronous structure of
// GPGPU/GPU/SlimGPUQueue.cs:314-405 without its per-thread queue atomics.
#include <atomic>

#include "common.cuh"

namespace sbfs {
namespace {

// One barrier per level: every thread derives the next level's bounds from the
// entries the level appended, so the shared counters rotate and nothing a fast
// thread writes in level L+1 is read by a slow thread finishing level L:
//   * cnt[L % 3] counts level L's appends (positions lvl_end + count); level L
//     zeroes cnt[(L+1) % 3], which was last read at the start of level L-1;
//   * found[L & 1] takes level L's singleton hits; a hit ends the search, so
//     both are reset once per automaton.
struct CtaCtl {
    unsigned long long found[2];   // min over (queue index << 1 | letter) of singleton hits
    uint32_t cnt[3];
    int64_t k;
    int n;
    int bad;
};

__global__ void __launch_bounds__(1024) k_cta(Batch b, int nb_max, uint64_t *queues,
                                              unsigned long long *ticket)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *table = reinterpret_cast<uint64_t *>(smem_raw);            // 3 * 256
    uint32_t *bitmap = reinterpret_cast<uint32_t *>(table + 3 * 256);    // 2^nb_max bits
    __shared__ CtaCtl ctl;
    __shared__ uint32_t singles_a[32], singles_b[32];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    uint64_t *queue = queues + ((size_t)blockIdx.x << nb_max);
    int64_t count;
    const int32_t *order;
    resolve_work(b, count, order);
    unsigned long long expanded = 0;

    while (true) {
        if (tid == 0) {
            const unsigned long long pos = atomicAdd(ticket, 1ull);
            ctl.k = pos < (unsigned long long)count ? automaton_at(order, (int64_t)pos) : -1;
            ctl.bad = 0;
            if (ctl.k >= 0) {
                const int n = automaton_n(b, ctl.k);
                ctl.n = n;
                if (n < 1 || n > nb_max || n > b.lstride) ctl.bad = 1;
            }
        }
        __syncthreads();
        const int64_t k = ctl.k;
        if (k < 0) break;
        const int n = ctl.n;
        if (!ctl.bad && tid < n) {
            const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
            const uint32_t aj = rec[tid], bj = rec[b.lstride + tid];
            if (aj >= (uint32_t)n || bj >= (uint32_t)n) atomicOr(&ctl.bad, 1);
            singles_a[tid] = 1u << aj;
            singles_b[tid] = 1u << bj;
        }
        __syncthreads();
        if (ctl.bad) {
            if (tid == 0) {
                if (b.out_len) b.out_len[k] = kLenInvalid;
                atomicOr(b.error, kErrInvalid);
                publish_result(b, k);
            }
            __syncthreads();
            continue;
        }
        const int chunks = (n + 7) >> 3;
        for (int e = tid; e < chunks * 256; e += blockDim.x) {
            const int c = e >> 8, v = e & 255;
            uint32_t ta = 0, tb = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int st = 8 * c + j;
                if (((v >> j) & 1) && st < n) {
                    ta |= singles_a[st];
                    tb |= singles_b[st];
                }
            }
            table[e] = ((uint64_t)ta << 32) | tb;
        }
        const int words = n >= 5 ? (1 << (n - 5)) : 1;
        for (int w = tid; w < words; w += blockDim.x) bitmap[w] = 0u;
        __syncthreads();
        const uint32_t full = (1u << n) - 1u;
        if (tid == 0) {
            queue[0] = full;
            bitmap[full >> 5] |= 1u << (full & 31u);
            ctl.found[0] = ctl.found[1] = ~0ull;
            ctl.cnt[0] = ctl.cnt[1] = ctl.cnt[2] = 0u;
        }
        __syncthreads();

        int32_t len = kLenNonSync;
        uint32_t ls = 0, le = 1, level = 0;
        while (true) {
            uint32_t *cnt = &ctl.cnt[level % 3];
            unsigned long long *found = &ctl.found[level & 1];
            if (tid == 0) ctl.cnt[(level + 1) % 3] = 0u;
            // whole warps iterate so the push ballots stay converged
            for (uint32_t base = ls + (tid & ~31); base < le; base += blockDim.x) {
                const uint32_t i = base + lane;
                bool p0 = false, p1 = false;
                uint32_t y0 = 0, y1 = 0;
                if (i < le) {
                    const uint32_t x = (uint32_t)queue[i];
                    uint64_t t = table[x & 255u];
                    if (chunks > 1) t |= table[256 + ((x >> 8) & 255u)];
                    if (chunks > 2) t |= table[512 + ((x >> 16) & 255u)];
                    y0 = (uint32_t)(t >> 32);
                    y1 = (uint32_t)t;
                    const uint32_t m0 = 1u << (y0 & 31u);
                    const bool in0 = SBFS_CHECK((y0 >> nb_max) == 0u, b.error);
                    const bool in1 = SBFS_CHECK((y1 >> nb_max) == 0u, b.error);
                    if (in0 && !(atomicOr(&bitmap[y0 >> 5], m0) & m0)) {
                        if (is_singleton(y0))
                            atomicMin(found, ((unsigned long long)i << 1));
                        else
                            p0 = true;
                    }
                    const uint32_t m1 = 1u << (y1 & 31u);
                    if (in1 && !(atomicOr(&bitmap[y1 >> 5], m1) & m1)) {
                        if (is_singleton(y1))
                            atomicMin(found, ((unsigned long long)i << 1) | 1ull);
                        else
                            p1 = true;
                    }
                    ++expanded;
                }
                const unsigned m0 = __ballot_sync(kFull, p0), m1 = __ballot_sync(kFull, p1);
                const int c = __popc(m0) + __popc(m1);
                if (c) {
                    uint32_t pos = 0;
                    if (lane == 0) pos = le + atomicAdd(cnt, (uint32_t)c);
                    pos = __shfl_sync(kFull, pos, 0);
                    const unsigned lt = (1u << lane) - 1u;
                    pos += __popc(m0 & lt) + __popc(m1 & lt);
                    // every subset enters the queue at most once: 2^nb_max entries never overflow
                    if (p0 && SBFS_CHECK(pos < (1u << nb_max), b.error)) queue[pos] = y0 | ((uint64_t)i << 32);
                    pos += p0 ? 1u : 0u;
                    if (p1 && SBFS_CHECK(pos < (1u << nb_max), b.error))
                        queue[pos] = y1 | ((uint64_t)i << 32) | (1ull << 63);
                }
            }
            __syncthreads();
            const unsigned long long f = *found;
            const uint32_t added = *cnt;
            if (f != ~0ull) {
                len = (int32_t)level + 1;
                if (tid == 0) {
                    record_result(b, k, n, len);
                    if (b.out_words) {
                        uint64_t *w = b.out_words + (size_t)k * (size_t)b.word_stride;
                        for (int c = 0; c < b.word_stride; ++c) w[c] = 0ull;
                        if (len <= 64 * b.word_stride) {
                            int d = len - 1;
                            w[d >> 6] |= (uint64_t)(f & 1ull) << (d & 63);
                            uint64_t e = queue[f >> 1];
                            for (d = len - 2; d >= 0; --d) {
                                w[d >> 6] |= (uint64_t)(e >> 63) << (d & 63);
                                e = queue[(e >> 32) & 0x7FFFFFFFull];
                            }
                        }
                    }
                    publish_result(b, k);
                }
                break;
            }
            if (added == 0) {
                if (tid == 0) {
                    record_result(b, k, n, kLenNonSync);
                    if (b.out_words) {
                        uint64_t *w = b.out_words + (size_t)k * (size_t)b.word_stride;
                        for (int c = 0; c < b.word_stride; ++c) w[c] = 0ull;
                    }
                    publish_result(b, k);
                }
                break;
            }
            ls = le;
            le += added;
            ++level;
        }
        __syncthreads();
    }
    // one atomic per warp
    for (int o = 16; o; o >>= 1) expanded += __shfl_down_sync(kFull, expanded, o);
    if (lane == 0 && b.expanded) atomicAdd(b.expanded, expanded);
}

}  // namespace

size_t cta_smem_bytes(int nb_max)
{
    const size_t bitmap = nb_max >= 5 ? ((size_t)1 << nb_max) / 8 : 4;
    return 3 * 256 * sizeof(uint64_t) + bitmap;
}

size_t cta_queue_entries(int nb_max, int ctas)
{
    return (size_t)ctas << nb_max;
}

namespace {

constexpr int kMaxDevices = 16;

int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return dev;
}

// Raises the kernel's dynamic shared-memory cap once per device to the largest
// footprint any launch asks for (n = 20), so concurrent launches of different
// sizes never lower it under one another.
cudaError_t cta_allow_smem()
{
    static std::atomic<int> done[kMaxDevices];
    const int dev = current_device();
    const bool cached = dev >= 0 && dev < kMaxDevices;
    if (cached && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(k_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)cta_smem_bytes(20));
    if (e == cudaSuccess && cached) done[dev].store(1, std::memory_order_release);
    return e;
}

}  // namespace

int cta_max_ctas_per_sm(int nb_max, int threads)
{
    // resident CTAs per (device, n, width), measured once: enqueue paths ask on every launch
    static std::atomic<int> known[kMaxDevices][21][33];
    if (nb_max < 1 || nb_max > 20 || threads < 32 || threads > 1024 || (threads & 31)) return 0;
    const int dev = current_device();
    const bool cached = dev >= 0 && dev < kMaxDevices;
    if (cached) {
        const int v = known[dev][nb_max][threads >> 5].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    if (cta_allow_smem() != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_cta, threads, cta_smem_bytes(nb_max)) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cached && blocks > 0) known[dev][nb_max][threads >> 5].store(blocks, std::memory_order_relaxed);
    return blocks;
}

cudaError_t launch_cta(int nb_max, int threads, int ctas, const Batch &b, uint64_t *queues,
                       unsigned long long *ticket, cudaStream_t st)
{
    if (nb_max < 1 || nb_max > 20 || threads < 32 || threads > 1024 || (threads & 31) || ctas < 1)
        return cudaErrorInvalidValue;
    const size_t smem = cta_smem_bytes(nb_max);
    const cudaError_t e = cta_allow_smem();
    if (e != cudaSuccess) return e;
    k_cta<<<ctas, threads, smem, st>>>(b, nb_max, queues, ticket);
    return cudaGetLastError();
}

}  // namespace sbfs
