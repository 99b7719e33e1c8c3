// k_pool.cu -- power-set BFS for many small automata per warp (n <= 16).
//
// Replaces the per-CTA Alea kernel of GPGPU/GPU/SlimGPUQueue.cs:210-407, which
// runs one automaton at a time per CTA with 6-bit shared-memory counters as the
// visited store and two level queues.  Here one warp keeps S automata in
// flight ("slots"), each with
//   * a visited bitmap of 2^NMAX bits in shared memory (atomicOr is an exact
//     test-and-set, replacing the counter emulation at SlimGPUQueue.cs:334-362),
//   * a nibble table over 4-bit chunks of the subset, entry = (a-image << 16) |
//     b-image (the combined table of GPGPU/CPU/SlimCPU4bits.cs:122-206), so both
//     images come from ceil(n/4) shared-memory loads,
//   * a level-ordered queue of (subset | parent index << 16) entries, the first
//     Q in shared memory and the rest in a per-slot global spill area; the
//     retained queue gives the word by parent pointers (GPGPU/CPU/CPU.cs:203-205).
// Each step the warp scans the slots' remaining current-level work and hands
// one subset to each lane, whichever automaton it belongs to, so the 32 lanes
// stay busy even though one level of one automaton holds only a few subsets.
// Levels are strictly synchronous per automaton (a slot moves to the next
// level only after all of the current level has been expanded), so a subset
// is first discovered at its BFS depth and the first singleton generated gives
// the shortest length, as in GPGPU/CPU/SlimCPUUntweaked.cs:119-184.
#include <climits>

#include "common.cuh"

namespace sbfs {
namespace {

template <int NMAX>
struct PoolGeom {
    static constexpr int kBitmapWords = (1 << NMAX) / 32 > 0 ? (1 << NMAX) / 32 : 1;
    static constexpr int kChunks = (NMAX + 3) / 4;
    static constexpr int kTable = kChunks * 16;
    // bitmaps of up to 4 KiB (NMAX <= 15) are cleared by whole-bitmap stores;
    // larger ones by walking the queue of subsets that were marked
    static constexpr bool kWalkClear = kBitmapWords > 1024;
};

__host__ __device__ constexpr int region_words(int bitmap_words, int table, int slots, int q)
{
    // per-warp region: bitmaps, tables, queues, 32-entry start map; 16-byte multiple
    return ((slots * (bitmap_words + table + q) + 32) + 3) & ~3;
}

template <int NMAX>
__device__ __forceinline__ uint32_t table_image(const uint32_t *tb, uint32_t x)
{
    uint32_t t = tb[x & 15u];
    if (PoolGeom<NMAX>::kChunks > 1) t |= tb[16 + ((x >> 4) & 15u)];
    if (PoolGeom<NMAX>::kChunks > 2) t |= tb[32 + ((x >> 8) & 15u)];
    if (PoolGeom<NMAX>::kChunks > 3) t |= tb[48 + ((x >> 12) & 15u)];
    return t;
}

template <int NMAX, int S>
__global__ void __launch_bounds__(512) k_pool(Batch b, int q_smem, int grab, uint32_t *spill,
                                              unsigned long long *ticket, PoolHeavy heavy)
{
    using G = PoolGeom<NMAX>;
    constexpr int BW = G::kBitmapWords;
    constexpr int T = G::kTable;
    extern __shared__ __align__(16) uint32_t smem[];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const int Q = q_smem;
    uint32_t *region = smem + (size_t)warp * region_words(BW, T, S, Q);
    uint32_t *bitmap = region;                 // S * BW
    uint32_t *table = bitmap + S * BW;         // S * T
    uint32_t *queue = table + S * T;           // S * Q
    uint32_t *startmap = queue + S * Q;        // 32
    const uint32_t spill_per_slot = (1u << NMAX) > (uint32_t)Q ? (1u << NMAX) - (uint32_t)Q : 0u;
    uint32_t *spill_warp = spill + ((size_t)blockIdx.x * warps + warp) * S * spill_per_slot;

    auto qload = [&](int s, uint32_t i) -> uint32_t {
        return i < (uint32_t)Q ? queue[s * Q + i]
                               : __ldcg(spill_warp + (size_t)s * spill_per_slot + (i - (uint32_t)Q));
    };
    auto qstore = [&](int s, uint32_t i, uint32_t v) {
        if (!SBFS_CHECK(i < (uint32_t)Q + spill_per_slot, b.error)) return;
        if (i < (uint32_t)Q)
            queue[s * Q + i] = v;
        else
            __stcg(spill_warp + (size_t)s * spill_per_slot + (i - (uint32_t)Q), v);
    };

    for (int w = lane; w < S * BW; w += 32) bitmap[w] = 0u;
    __syncwarp();

    // Slot registers: lane s < S owns slot s.
    int my_active = 0;
    uint32_t my_head = 0, my_lvl_end = 0, my_tail = 0, my_level = 0;
    int my_n = 0;
    int64_t my_k = -1;

    int64_t count;
    const int32_t *order;
    resolve_work(b, count, order);
    int64_t cur = 0, lim = 0;   // warp-uniform claimed range of the work list
    bool more = true;
    unsigned long long expanded = 0;

    while (true) {
        // ---- refill free slots from the work list --------------------------
        unsigned free_mask = __ballot_sync(kFull, lane < S && !my_active);
        while (free_mask && more) {
            if (cur == lim) {
                unsigned long long got = 0;
                if (lane == 0) got = atomicAdd(ticket, (unsigned long long)grab);
                got = __shfl_sync(kFull, got, 0);
                cur = (int64_t)got;
                lim = min((int64_t)got + grab, count);
                if (cur >= count) {
                    more = false;
                    break;
                }
            }
            const int s = __ffs(free_mask) - 1;
            const int64_t k = automaton_at(order, cur);
            ++cur;
            const int n = automaton_n(b, k);
            const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
            bool bad = (n < 1 || n > NMAX || n > b.lstride);
            uint32_t single = 0;
            if (!bad && lane < n) {
                const uint32_t aj = rec[lane], bj = rec[b.lstride + lane];
                if (aj >= (uint32_t)n || bj >= (uint32_t)n)
                    bad = true;
                else
                    single = (1u << (aj + 16)) | (1u << bj);
            }
            if (__any_sync(kFull, bad)) {
                if (lane == 0) {
                    if (b.out_len) b.out_len[k] = kLenInvalid;
                    atomicOr(b.error, kErrInvalid);
                    publish_result(b, k);
                }
                continue;   // slot s stays free
            }
            free_mask &= free_mask - 1;
            // table[c*16 + v] = OR of single[4c + j] over the set bits j of v
#pragma unroll
            for (int r = 0; r < (T + 31) / 32; ++r) {
                const int e = r * 32 + lane;
                const int c = (e >> 4) & 3, v = e & 15;
                uint32_t acc = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t sj = __shfl_sync(kFull, single, c * 4 + j);
                    if ((v >> j) & 1) acc |= sj;
                }
                if (e < T) table[s * T + e] = acc;
            }
            const uint32_t full = (1u << n) - 1u;
            if (lane == 0) {
                queue[s * Q] = full;
                bitmap[s * BW + (full >> 5)] |= 1u << (full & 31u);
            }
            if (lane == s) {
                my_active = 1;
                my_head = 0;
                my_lvl_end = 1;
                my_tail = 1;
                my_level = 0;
                my_n = n;
                my_k = k;
            }
        }
        __syncwarp();
        if (!__any_sync(kFull, my_active)) {
            if (!more) break;
            continue;
        }

        // ---- hand out current-level subsets to lanes -----------------------
        const uint32_t avail = my_active ? (my_lvl_end - my_head) : 0u;
        uint32_t incl = avail;
#pragma unroll
        for (int d = 1; d < S; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += y;
        }
        const uint32_t excl = incl - avail;
        const uint32_t take = (lane < S && excl < 32u) ? min(avail, 32u - excl) : 0u;
        const uint32_t total = min(__shfl_sync(kFull, incl, S - 1), 32u);
        const unsigned starts = __reduce_or_sync(kFull, take ? (1u << excl) : 0u);
        if (take) startmap[excl] = (uint32_t)lane;
        __syncwarp();

        int s_item = -1;
        uint32_t off = 0;
        if ((uint32_t)lane < total) {
            const unsigned below = starts & (kFull >> (31 - lane));
            const int st = 31 - __clz(below);
            s_item = (int)startmap[st];
            off = (uint32_t)(lane - st);
        }
        const int src = s_item >= 0 ? s_item : lane;
        const uint32_t it_head = __shfl_sync(kFull, my_head, src);
        const uint32_t it_excl = __shfl_sync(kFull, excl, src);
        const uint32_t it_take = __shfl_sync(kFull, take, src);
        const uint32_t head_old = my_head;
        my_head += take;

        // ---- expand: both images, test-and-set, classify --------------------
        uint32_t img0 = 0, img1 = 0, idx = 0;
        bool push0 = false, push1 = false, fnd0 = false, fnd1 = false;
        if (s_item >= 0) {
            idx = it_head + off;
            const uint32_t x = qload(s_item, idx) & 0xFFFFu;
            const uint32_t t = table_image<NMAX>(table + s_item * T, x);
            img0 = t >> 16;
            img1 = t & 0xFFFFu;
            uint32_t *bm = bitmap + s_item * BW;
            const bool in = SBFS_CHECK((img0 >> 5) < (uint32_t)BW && (img1 >> 5) < (uint32_t)BW, b.error);
            const uint32_t bit0 = 1u << (img0 & 31u);
            if (in && !(atomicOr(&bm[img0 >> 5], bit0) & bit0)) {
                push0 = true;
                fnd0 = is_singleton(img0);
            }
            const uint32_t bit1 = 1u << (img1 & 31u);
            if (in && !(atomicOr(&bm[img1 >> 5], bit1) & bit1)) {
                push1 = true;
                fnd1 = is_singleton(img1);
            }
        }
        expanded += total;

        // ---- append new subsets (singletons too, so the walk-clear sees them)
        const unsigned pa = __ballot_sync(kFull, push0);
        const unsigned pb = __ballot_sync(kFull, push1);
        const unsigned own_range = take ? ((take >= 32u ? kFull : ((1u << take) - 1u)) << excl) : 0u;
        const uint32_t own_base = my_tail;
        if (take) my_tail += __popc(pa & own_range) + __popc(pb & own_range);
        const uint32_t it_base = __shfl_sync(kFull, own_base, src);
        if (s_item >= 0) {
            const unsigned rng = (it_take >= 32u ? kFull : ((1u << it_take) - 1u)) << it_excl;
            const unsigned lt = (1u << lane) - 1u;
            uint32_t pos = it_base + __popc(pa & rng & lt) + __popc(pb & rng & lt);
            if (push0) qstore(s_item, pos++, img0 | (idx << 16));
            if (push1) qstore(s_item, pos, img1 | (idx << 16));
        }

        // ---- per-slot bookkeeping (owner lanes) -----------------------------
        const unsigned fa = __ballot_sync(kFull, fnd0);
        const unsigned fb = __ballot_sync(kFull, fnd1);
        bool done = false, esc = false;
        int32_t res_len = kLenNonSync;
        uint32_t f_parent = 0, f_letter = 0;
        const unsigned fr = (fa | fb) & own_range;
        if (fr) {
            const int fl = __ffs(fr) - 1;   // earliest queue entry, letter a before b
            done = true;
            res_len = (int32_t)my_level + 1;
            f_parent = head_old + (uint32_t)(fl - (int)excl);
            f_letter = ((fa >> fl) & 1u) ? 0u : 1u;
        } else if (my_active && my_head == my_lvl_end) {
            if (my_tail == my_lvl_end) {
                done = true;   // no new subset at this level: not synchronizing
            } else {
                my_lvl_end = my_tail;
                ++my_level;
                // a long thin search (a Cerny automaton has (n-1)^2 levels; random
                // ones here stay far below the cap) goes to a CTA-wide kernel
                if (heavy.list && my_level >= (uint32_t)heavy.level_cap) esc = true;
            }
        }
        __syncwarp();

        const unsigned em = __ballot_sync(kFull, esc);
        if (em) {
            unsigned long long pos = 0;
            const int leader = __ffs(em) - 1;
            if (lane == leader) pos = atomicAdd(heavy.count, (unsigned long long)__popc(em));
            pos = __shfl_sync(kFull, pos, leader);
            if (esc) heavy.list[pos + __popc(em & ((1u << lane) - 1u))] = (int32_t)my_k;
        }

        // ---- finished slots: result, word, bitmap clear ---------------------
        if (done) {
            record_result(b, my_k, my_n, res_len);
            if (b.out_words) {
                uint64_t *w = b.out_words + (size_t)my_k * (size_t)b.word_stride;
                const int ws = b.word_stride;
                int top = -1;   // highest chunk written by the backtrack
                if (res_len > 0 && res_len <= 64 * ws) {
                    const uint32_t *tb = table + lane * T;
                    int d = res_len - 1;
                    int chunk = d >> 6;
                    top = chunk;
                    uint64_t acc = (uint64_t)f_letter << (d & 63);
                    uint32_t e = qload(lane, f_parent);
                    for (d = res_len - 2; d >= 0; --d) {
                        if ((d >> 6) != chunk) {
                            w[chunk] = acc;
                            acc = 0;
                            chunk = d >> 6;
                        }
                        const uint32_t x = e & 0xFFFFu;
                        const uint32_t pe = qload(lane, e >> 16);
                        const uint32_t aimg = table_image<NMAX>(tb, pe & 0xFFFFu) >> 16;
                        acc |= (uint64_t)(aimg == x ? 0u : 1u) << (d & 63);
                        e = pe;
                    }
                    w[chunk] = acc;
                }
                for (int c = top + 1; c < ws; ++c) w[c] = 0ull;
            }
            publish_result(b, my_k);
        }
        unsigned done_mask = __ballot_sync(kFull, done || esc);
        while (done_mask) {
            const int s = __ffs(done_mask) - 1;
            done_mask &= done_mask - 1;
            uint32_t *bm = bitmap + s * BW;
            const uint32_t tail = __shfl_sync(kFull, my_tail, s);
            if (!G::kWalkClear || tail > (uint32_t)BW) {
                if (BW % 128 == 0) {
                    uint4 *bm4 = reinterpret_cast<uint4 *>(bm);
                    for (int w = lane; w < BW / 4; w += 32) bm4[w] = make_uint4(0u, 0u, 0u, 0u);
                } else {
                    for (int w = lane; w < BW; w += 32) bm[w] = 0u;
                }
            } else {
                for (uint32_t i = lane; i < tail; i += 32) bm[(qload(s, i) & 0xFFFFu) >> 5] = 0u;
            }
        }
        if (done || esc) my_active = 0;
        __syncwarp();
    }
    if (lane == 0 && b.expanded) atomicAdd(b.expanded, expanded);
}

template <int NMAX, int S>
cudaError_t launch_t(const PoolShape &s, const Batch &b, uint32_t *spill,
                     unsigned long long *ticket, cudaStream_t st, const PoolHeavy &hv)
{
    const size_t smem = pool_smem_bytes(s);
    cudaError_t e = cudaFuncSetAttribute(k_pool<NMAX, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k_pool<NMAX, S><<<s.ctas, s.warps * 32, smem, st>>>(b, s.queue_smem, s.grab > 0 ? s.grab : 16, spill, ticket,
                                                         hv);
    return cudaGetLastError();
}

template <int NMAX>
cudaError_t launch_n(const PoolShape &s, const Batch &b, uint32_t *spill,
                     unsigned long long *ticket, cudaStream_t st, const PoolHeavy &hv)
{
    switch (s.slots) {
    case 4: return launch_t<NMAX, 4>(s, b, spill, ticket, st, hv);
    case 8: return launch_t<NMAX, 8>(s, b, spill, ticket, st, hv);
    case 16: return launch_t<NMAX, 16>(s, b, spill, ticket, st, hv);
    case 32: return launch_t<NMAX, 32>(s, b, spill, ticket, st, hv);
    default: return cudaErrorInvalidValue;
    }
}

template <int NMAX>
const void *kernel_ptr(int slots)
{
    switch (slots) {
    case 4: return (const void *)k_pool<NMAX, 4>;
    case 8: return (const void *)k_pool<NMAX, 8>;
    case 16: return (const void *)k_pool<NMAX, 16>;
    case 32: return (const void *)k_pool<NMAX, 32>;
    default: return nullptr;
    }
}

const void *pool_kernel(const PoolShape &s)
{
    switch (s.nmax) {
    case 8: return kernel_ptr<8>(s.slots);
    case 12: return kernel_ptr<12>(s.slots);
    case 16: return kernel_ptr<16>(s.slots);
    default: return nullptr;
    }
}

int bitmap_words(int nmax) { return (1 << nmax) / 32 > 0 ? (1 << nmax) / 32 : 1; }
int table_words(int nmax) { return ((nmax + 3) / 4) * 16; }

}  // namespace

size_t pool_smem_bytes(const PoolShape &s)
{
    return (size_t)s.warps * region_words(bitmap_words(s.nmax), table_words(s.nmax), s.slots, s.queue_smem) *
           sizeof(uint32_t);
}

size_t pool_spill_words(const PoolShape &s)
{
    const size_t per_slot = (size_t)1 << s.nmax > (size_t)s.queue_smem ? ((size_t)1 << s.nmax) - s.queue_smem : 0;
    return (size_t)s.ctas * s.warps * s.slots * per_slot;
}

int pool_max_ctas_per_sm(const PoolShape &s)
{
    const void *k = pool_kernel(s);
    if (!k) return 0;
    const size_t smem = pool_smem_bytes(s);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, s.warps * 32, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

cudaError_t launch_pool(const PoolShape &s, const Batch &b, uint32_t *spill,
                        unsigned long long *ticket, cudaStream_t st, const PoolHeavy &heavy)
{
    if (s.queue_smem < 32 || s.warps < 1 || s.warps > 16 || s.ctas < 1) return cudaErrorInvalidValue;
    if (heavy.list && (heavy.level_cap < 1 || !heavy.count)) return cudaErrorInvalidValue;
    switch (s.nmax) {
    case 8: return launch_n<8>(s, b, spill, ticket, st, heavy);
    case 12: return launch_n<12>(s, b, spill, ticket, st, heavy);
    case 16: return launch_n<16>(s, b, spill, ticket, st, heavy);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sbfs
