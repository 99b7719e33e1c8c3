// k_hash.cu -- power-set BFS of automata with 13..20 states (size classes 2
// and 3) with one warp per automaton and an open-addressed hash set as the
// visited store.
//
// A random automaton of 13..20 states is settled after a few hundred subsets
// over ~11 levels (its shortest word is at most ~36 letters), so neither a
// 2^n-bit bitmap (128 KiB at n = 20) nor a 1024-thread CTA (k_cta.cu) pays for
// itself: the CTA's per-level barriers and round trips dominate.  Here each
// warp keeps in shared memory
//   * nibble tables: table[c][v] = (a-image << 32) | b-image of the states
//     4c..4c+3 selected by v, so both images of a subset are 5 loads;
//   * a hash set of 2^CAP_BITS slots, each holding subset | generation << 20;
//     the generation changes with every automaton, so a slot from an earlier
//     automaton reads as empty and the set is cleared once per 4095 automata;
//   * a level-ordered queue of 16-bit entries, set slot | letter-is-b << 15
//     (a slot keeps its subset for the whole search), with a 16-bit parent
//     index per entry, retained for the word (GPGPU/CPU/CPU.cs:203-205).
// 15 KB per warp at 2048 slots: five warps per CTA, three CTAs per SM.
// The warp expands 32 subsets of the current level per step (level-
// synchronous, as GPGPU/CPU/SlimCPUUntweaked.cs:119-184), tests the images
// against the set (atomicCAS insert), and appends the new ones compacted by
// ballots in queue order.  An automaton that needs more than 3/4 of the set's
// slots or kHashLevelCap levels (a Cerny automaton: (n-1)^2 levels) is handed
// to the CTA-wide kernel through a list.  Random n = 17..20: 1.7 % of the
// automata pass 1536 subsets, 0.3 % pass 4096.
#include <atomic>

#include "common.cuh"

namespace sbfs {
namespace {

constexpr uint32_t kHashLevelCap = 48;         // random n <= 20: at most ~40 levels
constexpr uint32_t kSubsetMask = (1u << 20) - 1u;

template <int CAP_BITS>
struct HashGeom {
    static constexpr int kCap = 1 << CAP_BITS;                  // hash slots per warp
    static constexpr uint32_t kLimit = 3u * (1u << CAP_BITS) / 4u;   // subsets a warp keeps
    static constexpr int kWarps = CAP_BITS <= 11 ? 5 : 2;        // warps per CTA (~75 KB)
};

template <int CAP_BITS>
struct __align__(16) HashWarp {
    using G = HashGeom<CAP_BITS>;
    uint64_t table[5 * 16];
    uint32_t set[G::kCap];
    uint16_t queue[G::kLimit];    // set slot | letter-is-b << 15
    uint16_t parent[G::kLimit];
};

template <int CAP_BITS>
__device__ __forceinline__ uint32_t hash_slot(uint32_t x)
{
    return (x * 0x9E3779B1u) >> (32 - CAP_BITS);
}

// Inserts subset x (generation gen); returns its slot when it was not yet in
// the set, -1 otherwise.
template <int CAP_BITS>
__device__ __forceinline__ int set_insert(uint32_t *set, uint32_t x, uint32_t gen)
{
    constexpr int kCap = 1 << CAP_BITS;
    const uint32_t key = x | (gen << 20);
    uint32_t p = hash_slot<CAP_BITS>(x);
    for (int probe = 0; probe < kCap; ++probe) {
        uint32_t v = set[p];
        while ((v >> 20) != gen) {   // a slot of an earlier automaton: empty for this one
            const uint32_t prev = atomicCAS(&set[p], v, key);
            if (prev == v) return (int)p;
            v = prev;   // someone else took it: look at what is there now
        }
        if (v == key) return -1;
        p = (p + 1) & (kCap - 1);
    }
    return -1;   // unreachable: the set is never more than ~3/4 full
}

template <int CAP_BITS>
__global__ void __launch_bounds__(HashGeom<CAP_BITS>::kWarps * 32)
    k_hash(Batch b, int32_t *heavy_list, unsigned long long *heavy_count, unsigned long long *ticket)
{
    using G = HashGeom<CAP_BITS>;
    constexpr int kHashCap = G::kCap;
    constexpr uint32_t kHashLimit = G::kLimit;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    HashWarp<CAP_BITS> &W = reinterpret_cast<HashWarp<CAP_BITS> *>(smem_raw)[warp];
    int64_t count;
    const int32_t *order;
    resolve_work(b, count, order);
    // generation 0 marks never-used slots; each automaton takes the next one
    for (int i = lane; i < kHashCap; i += 32) W.set[i] = 0u;
    __syncwarp();
    uint32_t gen = 0;
    unsigned long long expanded = 0;

    while (true) {
        unsigned long long pos = 0;
        if (lane == 0) pos = atomicAdd(ticket, 1ull);
        pos = __shfl_sync(kFull, pos, 0);
        if (pos >= (unsigned long long)count) break;
        const int64_t k = automaton_at(order, (int64_t)pos);
        const int n = automaton_n(b, k);
        const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
        bool bad = n < 1 || n > 20 || n > b.lstride;
        uint64_t single = 0;
        if (!bad && lane < n) {
            const uint32_t av = rec[lane], bv = rec[b.lstride + lane];
            if (av >= (uint32_t)n || bv >= (uint32_t)n)
                bad = true;
            else
                single = ((uint64_t)(1u << av) << 32) | (1u << bv);
        }
        if (__any_sync(kFull, bad)) {
            if (lane == 0) {
                record_result(b, k, n, kLenInvalid);
                if (b.out_words)
                    for (int c = 0; c < b.word_stride; ++c) b.out_words[(size_t)k * b.word_stride + c] = 0ull;
                atomicOr(b.error, kErrInvalid);
                publish_result(b, k);
            }
            continue;
        }
        // nibble tables: 80 entries in three passes that every lane takes (the
        // shuffles need the whole warp), the third storing lanes 0..15 only
#pragma unroll
        for (int pass = 0; pass < 3; ++pass) {
            const int e = lane + 32 * pass;
            const int c = min(e >> 4, 4), v = e & 15;
            uint64_t acc = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint64_t sj = __shfl_sync(kFull, single, 4 * c + j);
                if (((v >> j) & 1) && 4 * c + j < n) acc |= sj;
            }
            if (e < 5 * 16) W.table[e] = acc;
        }
        if (++gen == (1u << 12)) {   // generations wrapped: clear once, start again at 1
            for (int i = lane; i < kHashCap; i += 32) W.set[i] = 0u;
            gen = 1;
            __syncwarp();
        }
        const uint32_t full = (1u << n) - 1u;
        if (lane == 0) W.queue[0] = (uint16_t)set_insert<CAP_BITS>(W.set, full, gen);
        __syncwarp();
        // n = 1: the visited root is the only singleton, the search generates nothing new
        uint32_t head = 0, lvl_end = n > 1 ? 1u : 0u, tail = lvl_end, level = 0;
        int32_t len = kLenNonSync;
        uint32_t found = 0, found_letter = 0;
        bool heavy = false;
        while (head < lvl_end) {
            const uint32_t idx = head + (uint32_t)lane;
            const bool has = idx < lvl_end;
            uint32_t ya = 0, yb = 0;
            if (has) {
                const uint32_t x = W.set[W.queue[idx] & 0x7FFFu] & kSubsetMask;
                uint64_t t = W.table[x & 15u] | W.table[16 + ((x >> 4) & 15u)] | W.table[32 + ((x >> 8) & 15u)] |
                             W.table[48 + ((x >> 12) & 15u)] | W.table[64 + ((x >> 16) & 15u)];
                ya = (uint32_t)(t >> 32);
                yb = (uint32_t)t;
            }
            expanded += has ? 1u : 0u;
            const bool sa = has && is_singleton(ya), sb = has && is_singleton(yb);
            const unsigned smask = __ballot_sync(kFull, sa || sb);
            if (smask) {
                // the first singleton in queue order (lowest lane, a before b)
                const int fl = __ffs(smask) - 1;
                found = head + (uint32_t)fl;
                found_letter = (uint32_t)__shfl_sync(kFull, sa ? 0 : 1, fl);
                len = (int32_t)level + 1;
                break;
            }
            const int sa_slot = has ? set_insert<CAP_BITS>(W.set, ya, gen) : -1;
            const int sb_slot = has ? set_insert<CAP_BITS>(W.set, yb, gen) : -1;
            bool fa = sa_slot >= 0, fb = sb_slot >= 0;
            const unsigned ma = __ballot_sync(kFull, fa), mb = __ballot_sync(kFull, fb);
            const uint32_t added = (uint32_t)(__popc(ma) + __popc(mb));
            if (tail + added > kHashLimit) {
                heavy = true;
                break;
            }
            const unsigned lt = (1u << lane) - 1u;
            uint32_t p = tail + (uint32_t)(__popc(ma & lt) + __popc(mb & lt));
            if (!SBFS_CHECK(p + (fa ? 1u : 0u) + (fb ? 1u : 0u) <= kHashLimit, b.error)) fa = fb = false;
            if (fa) {
                W.queue[p] = (uint16_t)sa_slot;
                W.parent[p++] = (uint16_t)idx;
            }
            if (fb) {
                W.queue[p] = (uint16_t)(sb_slot | 0x8000);
                W.parent[p] = (uint16_t)idx;
            }
            tail += added;
            head = min(head + 32u, lvl_end);
            __syncwarp();
            if (head == lvl_end && tail > lvl_end) {
                lvl_end = tail;
                if (++level >= kHashLevelCap) {
                    heavy = true;
                    break;
                }
            }
        }
        __syncwarp();
        if (heavy) {
            // a long or wide search: the CTA-wide kernel takes it from the start
            if (lane == 0) heavy_list[atomicAdd(heavy_count, 1ull)] = (int32_t)k;
            continue;
        }
        if (lane == 0) {
            record_result(b, k, n, len);
            if (b.out_words) {
                // letters from the root: the entry at depth d + 1 holds letter d
                // (a word here has at most kHashLevelCap <= 64 letters)
                uint64_t w0 = 0;
                if (len > 0) {
                    if (found_letter) w0 |= 1ull << level;
                    uint32_t i = found;
                    for (int d = (int)level - 1; d >= 0; --d) {
                        if (W.queue[i] >> 15) w0 |= 1ull << d;
                        i = W.parent[i];
                    }
                }
                uint64_t *w = b.out_words + (size_t)k * (size_t)b.word_stride;
                w[0] = w0;
                for (int c = 1; c < b.word_stride; ++c) w[c] = 0ull;
            }
            publish_result(b, k);
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) expanded += __shfl_down_sync(kFull, expanded, o);
    if (lane == 0 && b.expanded && expanded) atomicAdd(b.expanded, expanded);
}

// Counting sort of a hand-off list by n, largest first (one CTA): the
// persistent CTA-wide kernel then takes the longest searches first, and the
// short ones fill the SMs that free up (longest-processing-time order).
// With split, the sorted list is also described as two work ranges,
// {0, entries with n >= top_n} and {that, the rest}, so the entries below
// top_n can run in a launch sized for top_n - 1.
__global__ void __launch_bounds__(1024) k_sort_handoff(Batch b, const int32_t *list,
                                                       const unsigned long long *count, int32_t *out,
                                                       int top_n, unsigned long long *split)
{
    __shared__ unsigned int hist[SBFS_MAX_N + 2];
    const int tid = threadIdx.x;
    const int64_t cnt = (int64_t)*count;
    for (int i = tid; i < SBFS_MAX_N + 2; i += blockDim.x) hist[i] = 0u;
    __syncthreads();
    for (int64_t i = tid; i < cnt; i += blockDim.x) {
        const int n = min(max(automaton_n(b, list[i]), 0), SBFS_MAX_N + 1);
        atomicAdd(&hist[n], 1u);
    }
    __syncthreads();
    if (tid == 0) {
        unsigned int off = 0, top = 0;
        for (int n = SBFS_MAX_N + 1; n >= 0; --n) {
            const unsigned int c = hist[n];
            hist[n] = off;
            off += c;
            if (n == top_n) top = off;   // entries with n >= top_n
        }
        if (split) {
            split[0] = 0ull;
            split[1] = top;
            split[2] = top;
            split[3] = (unsigned long long)cnt - top;
        }
    }
    __syncthreads();
    for (int64_t i = tid; i < cnt; i += blockDim.x) {
        const int32_t k = list[i];
        const int n = min(max(automaton_n(b, k), 0), SBFS_MAX_N + 1);
        out[atomicAdd(&hist[n], 1u)] = k;
    }
}

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

// The shared-memory cap and the resident CTAs per SM are set and measured once
// per device: the enqueue paths ask on every launch.
template <int CAP_BITS>
struct HashLaunch {
    static size_t smem() { return (size_t)HashGeom<CAP_BITS>::kWarps * sizeof(HashWarp<CAP_BITS>); }
    static cudaError_t prepare()
    {
        static std::atomic<int> done[kMaxDevices];
        const int dev = current_device();
        const bool cached = dev >= 0 && dev < kMaxDevices;
        if (cached && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
        const cudaError_t e =
            cudaFuncSetAttribute(k_hash<CAP_BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
        if (e == cudaSuccess && cached) done[dev].store(1, std::memory_order_release);
        return e;
    }
    static int per_sm()
    {
        static std::atomic<int> known[kMaxDevices];
        const int dev = current_device();
        const bool cached = dev >= 0 && dev < kMaxDevices;
        if (cached) {
            const int v = known[dev].load(std::memory_order_relaxed);
            if (v > 0) return v;
        }
        if (prepare() != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_hash<CAP_BITS>, HashGeom<CAP_BITS>::kWarps * 32,
                                                          smem()) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        if (cached && blocks > 0) known[dev].store(blocks, std::memory_order_relaxed);
        return blocks;
    }
    static cudaError_t launch(int ctas, const Batch &b, int32_t *list, unsigned long long *count,
                              unsigned long long *ticket, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess) return e;
        k_hash<CAP_BITS><<<ctas, HashGeom<CAP_BITS>::kWarps * 32, smem(), st>>>(b, list, count, ticket);
        return cudaGetLastError();
    }
};

}  // namespace

// size 1: 2048 hash slots per warp (1536 subsets), size 2: 4096 (3072 subsets)
int hash_max_ctas_per_sm(int size)
{
    return size == 2 ? HashLaunch<12>::per_sm() : size == 1 ? HashLaunch<11>::per_sm() : 0;
}

cudaError_t launch_sort_handoff(const Batch &b, const int32_t *list, const unsigned long long *count, int32_t *out,
                                int top_n, unsigned long long *split, cudaStream_t st)
{
    k_sort_handoff<<<1, 1024, 0, st>>>(b, list, count, out, top_n, split);
    return cudaGetLastError();
}

cudaError_t launch_hash(int size, int ctas, const Batch &b, int32_t *heavy_list, unsigned long long *heavy_count,
                        unsigned long long *ticket, cudaStream_t st)
{
    if (ctas < 1 || !heavy_list || !heavy_count) return cudaErrorInvalidValue;
    if (size == 1) return HashLaunch<11>::launch(ctas, b, heavy_list, heavy_count, ticket, st);
    if (size == 2) return HashLaunch<12>::launch(ctas, b, heavy_list, heavy_count, ticket, st);
    return cudaErrorInvalidValue;
}

}  // namespace sbfs
