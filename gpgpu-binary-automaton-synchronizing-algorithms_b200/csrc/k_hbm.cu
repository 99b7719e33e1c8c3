// k_hbm.cu -- level-synchronous power-set BFS with the visited bitmap and
// the frontier in HBM (21 <= n <= 28).
//
// The whole grid works on one automaton at a time.  Per level every CTA takes a
// slice of the level's queue range, computes both images through byte tables
// held in its shared memory, test-and-sets the bits in the 2^n-bit global
// bitmap (32 MiB at n = 28; it stays resident in the 126 MB L2), and appends new
// subsets with one global atomic per warp.  A grid barrier separates levels.
// Queue entries are 64-bit: subset | parent index << 28 | letter-is-b << 63,
// retained for the word (GPGPU/CPU/CPU.cs:203-205,262-269).  Level semantics
// and the singleton-on-generation rule are those of
// GPGPU/CPU/SlimCPUUntweaked.cs:119-184; the reference itself stops at n <= 16
// (ushort masks, SlimCPUUntweaked.cs:61,69) and its GPU kernel at n <= 14
// (shared-memory size, GPGPU/GPU/SlimGPUQueue.cs:80-90).
//
// The kernel is launched cooperatively so that all CTAs are resident; the grid
// barrier still bounds its wait (kBarrierTimeoutNs) and, when it runs out, sets
// kErrTimeout and every CTA returns.
#include "common.cuh"

namespace sbfs {

constexpr int kErrTimeout = 4;

namespace {

constexpr unsigned long long kBarrierTimeoutNs = 20ull * 1000 * 1000 * 1000;

struct HbmCtl {
    unsigned int bar_count;
    unsigned int bar_gen;
    unsigned long long found;
    unsigned long long tail;
    unsigned long long lvl_start, lvl_end, level;
    long long k;
    int n;
    int bad;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Returns false when the barrier timed out or another CTA reported a timeout.
__device__ bool grid_barrier(HbmCtl *ctl, int *error)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned int *gen = &ctl->bar_gen;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(&ctl->bar_count, 1u) == gridDim.x - 1) {
            ctl->bar_count = 0;
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (*gen == g) {
                if (*(volatile int *)error & kErrTimeout) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicOr(error, kErrTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__global__ void __launch_bounds__(512) k_hbm(Batch b, uint32_t *bitmap, uint64_t *queue,
                                             HbmCtl *ctl, unsigned long long *ticket)
{
    __shared__ uint64_t table[4 * 256];
    __shared__ uint32_t singles_a[32], singles_b[32];
    __shared__ long long s_k;
    __shared__ int s_n;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + tid;
    const size_t gthreads = (size_t)gridDim.x * blockDim.x;
    int64_t count;
    const int32_t *order;
    resolve_work(b, count, order);
    unsigned long long expanded = 0;

    while (true) {
        // CTA 0 claims the next automaton and validates it; the barrier publishes it
        if (blockIdx.x == 0 && tid == 0) {
            const unsigned long long pos = atomicAdd(ticket, 1ull);
            long long k = pos < (unsigned long long)count ? automaton_at(order, (int64_t)pos) : -1;
            int bad = 0, n = 0;
            if (k >= 0) {
                n = automaton_n(b, k);
                if (n < 1 || n > 28 || n > b.lstride) {
                    bad = 1;
                } else {
                    const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
                    for (int j = 0; j < n; ++j)
                        if (rec[j] >= n || rec[b.lstride + j] >= n) bad = 1;
                }
                if (bad) {
                    if (b.out_len) b.out_len[k] = kLenInvalid;
                    atomicOr(b.error, kErrInvalid);
                }
            }
            ctl->k = k;
            ctl->n = n;
            ctl->bad = bad;
            ctl->found = ~0ull;
            ctl->lvl_start = 0;
            ctl->lvl_end = 1;
            ctl->tail = 1;
            ctl->level = 0;
        }
        if (!grid_barrier(ctl, b.error)) return;
        if (tid == 0) {
            s_k = *(volatile long long *)&ctl->k;
            s_n = *(volatile int *)&ctl->n;
        }
        __syncthreads();
        const long long k = s_k;
        const int n = s_n;
        if (k < 0) break;
        const bool bad = *(volatile int *)&ctl->bad != 0;
        if (bad) {
            if (!grid_barrier(ctl, b.error)) return;
            continue;
        }
        const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
        if (tid < n) {
            singles_a[tid] = 1u << rec[tid];
            singles_b[tid] = 1u << rec[b.lstride + tid];
        }
        __syncthreads();
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
        // clear the bitmap (2^n bits) with 16-byte stores
        const size_t words4 = ((size_t)1 << n) / 128;
        uint4 *bm4 = reinterpret_cast<uint4 *>(bitmap);
        for (size_t w = gtid; w < words4; w += gthreads) bm4[w] = make_uint4(0u, 0u, 0u, 0u);
        if (!grid_barrier(ctl, b.error)) return;
        const uint32_t full = (1u << n) - 1u;
        if (blockIdx.x == 0 && tid == 0) {
            queue[0] = full;
            bitmap[full >> 5] = 1u << (full & 31u);
        }
        if (!grid_barrier(ctl, b.error)) return;

        while (true) {
            const unsigned long long ls = *(volatile unsigned long long *)&ctl->lvl_start;
            const unsigned long long le = *(volatile unsigned long long *)&ctl->lvl_end;
            for (unsigned long long base = ls + (gtid & ~31ull); base < le; base += gthreads) {
                const unsigned long long i = base + lane;
                bool p0 = false, p1 = false;
                uint32_t y0 = 0, y1 = 0;
                if (i < le) {
                    const uint32_t x = (uint32_t)(__ldcg(queue + i) & 0x0FFFFFFFull);
                    uint64_t t = table[x & 255u];
                    if (chunks > 1) t |= table[256 + ((x >> 8) & 255u)];
                    if (chunks > 2) t |= table[512 + ((x >> 16) & 255u)];
                    if (chunks > 3) t |= table[768 + ((x >> 24) & 255u)];
                    y0 = (uint32_t)(t >> 32);
                    y1 = (uint32_t)t;
                    const uint32_t m0 = 1u << (y0 & 31u);
                    if (!(atomicOr(&bitmap[y0 >> 5], m0) & m0)) {
                        if (is_singleton(y0))
                            atomicMin(&ctl->found, i << 1);
                        else
                            p0 = true;
                    }
                    const uint32_t m1 = 1u << (y1 & 31u);
                    if (!(atomicOr(&bitmap[y1 >> 5], m1) & m1)) {
                        if (is_singleton(y1))
                            atomicMin(&ctl->found, (i << 1) | 1ull);
                        else
                            p1 = true;
                    }
                    ++expanded;
                }
                const unsigned m0 = __ballot_sync(kFull, p0), m1 = __ballot_sync(kFull, p1);
                const int cnt = __popc(m0) + __popc(m1);
                if (cnt) {
                    unsigned long long pos = 0;
                    if (lane == 0) pos = atomicAdd(&ctl->tail, (unsigned long long)cnt);
                    pos = __shfl_sync(kFull, pos, 0);
                    const unsigned lt = (1u << lane) - 1u;
                    pos += __popc(m0 & lt) + __popc(m1 & lt);
                    if (p0) __stcg(queue + pos++, (uint64_t)y0 | (i << 28));
                    if (p1) __stcg(queue + pos, (uint64_t)y1 | (i << 28) | (1ull << 63));
                }
            }
            if (!grid_barrier(ctl, b.error)) return;
            const unsigned long long f = *(volatile unsigned long long *)&ctl->found;
            const unsigned long long tail = *(volatile unsigned long long *)&ctl->tail;
            const unsigned long long level = *(volatile unsigned long long *)&ctl->level;
            const bool stop = (f != ~0ull) || (tail == le);
            if (stop) {
                if (blockIdx.x == 0 && tid == 0) {
                    const int32_t len = f != ~0ull ? (int32_t)level + 1 : kLenNonSync;
                    record_result(b, k, n, len);
                    if (b.out_words) {
                        uint64_t *w = b.out_words + (size_t)k * (size_t)b.word_stride;
                        for (int c = 0; c < b.word_stride; ++c) w[c] = 0ull;
                        if (len > 0 && len <= 64 * b.word_stride) {
                            int d = len - 1;
                            w[d >> 6] |= (uint64_t)(f & 1ull) << (d & 63);
                            uint64_t e = __ldcg(queue + (f >> 1));
                            for (d = len - 2; d >= 0; --d) {
                                w[d >> 6] |= (uint64_t)(e >> 63) << (d & 63);
                                e = __ldcg(queue + ((e >> 28) & 0x7FFFFFFFFull));
                            }
                        }
                    }
                }
                if (!grid_barrier(ctl, b.error)) return;
                break;
            }
            if (!grid_barrier(ctl, b.error)) return;   // everyone has read ctl before it moves on
            if (blockIdx.x == 0 && tid == 0) {
                ctl->lvl_start = le;
                ctl->lvl_end = tail;
                ctl->level = level + 1;
            }
            if (!grid_barrier(ctl, b.error)) return;
        }
    }
    for (int o = 16; o; o >>= 1) expanded += __shfl_down_sync(kFull, expanded, o);
    if (lane == 0 && b.expanded) atomicAdd(b.expanded, expanded);
}

}  // namespace

size_t hbm_ctl_bytes() { return 256; }

int hbm_max_ctas_per_sm(int threads)
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_hbm, threads, 0) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

cudaError_t launch_hbm(int threads, int ctas, const Batch &b, uint32_t *bitmap, uint64_t *queue,
                       void *ctl, unsigned long long *ticket, cudaStream_t st)
{
    if (threads < 32 || threads > 512 || (threads & 31) || ctas < 1) return cudaErrorInvalidValue;
    static_assert(sizeof(HbmCtl) <= 256, "control block");
    cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(HbmCtl), st);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HbmCtl *c = static_cast<HbmCtl *>(ctl);
    e = cudaLaunchKernelEx(&cfg, k_hbm, b, bitmap, queue, c, ticket);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace sbfs
