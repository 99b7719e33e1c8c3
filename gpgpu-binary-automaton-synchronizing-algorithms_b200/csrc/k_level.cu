// k_level.cu -- level-synchronous power-set BFS of many large automata at
// once, with every automaton's visited bitmap and frontier in HBM.
//
// State lives in device memory between launches ("slots"): each admitted
// automaton owns a 2^n-bit bitmap, a queue of 64-bit entries
// (subset | parent index << 28 | letter-is-b << 63, retained for the word as
// in GPGPU/CPU/CPU.cs:203-205,262-269) and byte tables of its images.  One
// launch of k_level advances every running slot by exactly one BFS level:
// all CTAs stride over the concatenation of the slots' current levels, test-
// and-set images in the bitmaps with global atomics, and append new subsets
// through a per-CTA staging buffer (one global atomic per slot per CTA round,
// coalesced writes).  The last CTA to finish (threadfence + ticket, no spin)
// then moves every slot to its next level, finishes the ones that found a
// singleton or ran dry, turns freshly admitted slots into running ones, and
// recomputes the prefix sums the next launch uses.  Level semantics are those
// of GPGPU/CPU/SlimCPUUntweaked.cs:119-184.
//
// Because state persists, the host (batch path or the serving loop) can admit
// new automata into free slots between launches and launch levels back to
// back (or from a CUDA graph) without waiting for the slowest automaton.
#include <cooperative_groups.h>

#include "level.cuh"

namespace sbfs {
namespace {

namespace cg = cooperative_groups;

constexpr int kThreads = 512;
constexpr int kNarrowCluster = 8;      // CTAs of the narrow-level kernel's cluster
// Items a thread of k_level expands per round: their queue loads, bitmap
// probes and atomics are issued together, so a wide level (C_28 has levels of
// up to 3.6M subsets) keeps K times more L2 requests in flight per thread.
constexpr int kWideItems = 2;

template <int K>
struct LevelSmem {
    static constexpr int kStage = 2 * K * kThreads;   // staged pushes per CTA round
    unsigned long long prefix[kMaxLevelSlots + 1];
    uint64_t stage[kStage];
    unsigned short stage_slot[kStage];
    unsigned short stage_rank[kStage];              // rank within its slot in this round (< kStage)
    unsigned int count;
    unsigned int slot_count[kMaxLevelSlots];
    unsigned long long slot_base[kMaxLevelSlots];
    unsigned long long warp_sum[kThreads / 32];
    unsigned long long lvl_start[kMaxLevelSlots];   // current level's first queue index per slot
    unsigned long long b_total;                     // narrow kernel: rank 0's transition results
    int b_running;
    int b_it;                                       // narrow kernel: levels run so far
    bool last;
};


__device__ __forceinline__ int find_slot(const unsigned long long *prefix, int nslots, unsigned long long item)
{
    // largest s with prefix[s] <= item (prefix[0] = 0, nondecreasing)
    int lo = 0, hi = nslots;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= item)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Expands this CTA's share of the current level of every running slot, over
// the concatenation of the slots' levels (sh.prefix).  A round gives each
// thread up to K items, ncta * blockDim apart (so a level narrower than a
// full round still spreads over every CTA, and the j-th items of a warp are
// consecutive: coalesced queue reads).  Returns the number of subsets expanded.
template <int K>
__device__ unsigned long long level_items(LevelSlot *slots, const uint64_t *tables, LevelSmem<K> &sh, int nslots,
                                          unsigned long long total, int cta, int ncta)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const unsigned long long gthreads = (unsigned long long)ncta * blockDim.x;
    // ---- one level of every running slot ------------------------------------
    // Pushes are staged per CTA round; positions come from one shared atomic per
    // warp and image batch (staging slot) and per warp and automaton (rank
    // within the automaton), so no shared address is hammered by every thread.
    unsigned long long expanded = 0;
    const unsigned lt = (1u << lane) - 1u;
    for (unsigned long long base = (unsigned long long)cta * blockDim.x; base < total; base += K * gthreads) {
        if (tid == 0) sh.count = 0;
        __syncthreads();
        int s[K];
        unsigned long long idx[K];
        uint32_t x[K];
        bool have[K];
        // queue entries first (K independent loads) ...
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const unsigned long long item = base + (unsigned long long)j * gthreads + tid;
            have[j] = item < total;
            s[j] = 0;
            idx[j] = 0;
            x[j] = 0;
            if (have[j]) {
                s[j] = find_slot(sh.prefix, nslots, item);
                idx[j] = sh.lvl_start[s[j]] + (item - sh.prefix[s[j]]);
                x[j] = (uint32_t)(__ldcg(slots[s[j]].queue + idx[j]) & kLevelSubsetMask);
            }
        }
        // ... then both images of each from the byte tables ...
        uint32_t y[2 * K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            uint64_t t = 0;
            if (have[j]) {
                const uint64_t *tb = tables + (size_t)s[j] * kLevelTable;
                t = __ldg(tb + (x[j] & 255u));
                t |= __ldg(tb + 256 + ((x[j] >> 8) & 255u));
                t |= __ldg(tb + 512 + ((x[j] >> 16) & 255u));
                t |= __ldg(tb + 768 + ((x[j] >> 24) & 255u));
                ++expanded;
            }
            y[2 * j] = (uint32_t)(t >> 32);
            y[2 * j + 1] = (uint32_t)t;
        }
        // ... then the atomic test-and-set of every image, issued back to back.
        // (A plain load of the bitmap word first, to skip the atomic for images
        // already visited -- about half of them on a Cerny level -- lengthens the
        // dependent chain more than it saves: C_28 took 15.4 ms with it, 13.2 ms
        // without.)
        bool push[2 * K];
#pragma unroll
        for (int c = 0; c < 2 * K; ++c) {
            const uint32_t m = 1u << (y[c] & 31u);
            push[c] = false;
            if (have[c >> 1]) {
                LevelSlot *sl = &slots[s[c >> 1]];
                if (!(atomicOr(sl->bitmap + (y[c] >> 5), m) & m)) {
                    if (is_singleton(y[c]))
                        atomicMin(&sl->found, (idx[c >> 1] << 1) | (unsigned long long)(c & 1));
                    else
                        push[c] = true;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 2 * K; ++c) {
            const unsigned pm = __ballot_sync(kFull, push[c]);
            if (pm) {
                unsigned int pos = 0;
                const int leader = __ffs(pm) - 1;
                if (lane == leader) pos = atomicAdd(&sh.count, (unsigned)__popc(pm));
                pos = __shfl_sync(kFull, pos, leader) + __popc(pm & lt);
                if (push[c]) {
                    const int q = s[c >> 1];
                    const unsigned grp = __match_any_sync(pm, q);
                    const int gl = __ffs(grp) - 1;
                    unsigned int r0 = 0;
                    if (lane == gl) r0 = atomicAdd(&sh.slot_count[q], (unsigned)__popc(grp));
                    const unsigned int rank = __shfl_sync(grp, r0, gl) + __popc(grp & lt);
                    sh.stage[pos] = (uint64_t)y[c] | (idx[c >> 1] << 28) | ((uint64_t)(c & 1) << 63);
                    sh.stage_slot[pos] = (unsigned short)q;
                    sh.stage_rank[pos] = (unsigned short)rank;
                }
            }
        }
        __syncthreads();
        // reserve space per slot: one global atomic per slot with pushes in this pass
        for (int q = tid; q < nslots; q += blockDim.x) {
            const unsigned int c = sh.slot_count[q];
            if (c) {
                sh.slot_base[q] = atomicAdd(&slots[q].tail, (unsigned long long)c);
                sh.slot_count[q] = 0;
            }
        }
        __syncthreads();
        const unsigned int cnt = sh.count;
        for (unsigned int p = tid; p < cnt; p += blockDim.x) {
            const int q = sh.stage_slot[p];
            const unsigned long long pos = sh.slot_base[q] + sh.stage_rank[p];
            LevelSlot &dst = slots[q];
            if (pos < dst.cap)
                __stcg(dst.queue + pos, sh.stage[p]);
            else
                atomicOr(&dst.overflow, 1);
        }
        __syncthreads();
    }
    return expanded;
}

// Moves every slot to its next level (all threads of one CTA): finishes the
// slots that found a singleton or ran dry (word by parent pointers), turns
// freshly admitted slots into running ones, and writes the prefix sums of the
// new levels to prefix_out.  Returns the new total (block-uniform); `running`
// receives the number of running slots.
template <int K>
__device__ unsigned long long level_transition(LevelSlot *slots, LevelCtl *ctl, const Batch &out, LevelSmem<K> &sh,
                                               int nslots, unsigned long long *prefix_out, int &running)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    for (int s = tid; s < nslots; s += blockDim.x) {
        LevelSlot &sl = slots[s];
        const int st = *(volatile int *)&sl.state;
        if (st == kSlotInit) {
            bool bad = sl.n < 1 || sl.n > 28;
            for (int j = 0; !bad && j < sl.n; ++j) {
                const uint32_t av = sl.rec ? sl.rec[j] : sl.a[j];
                const uint32_t bv = sl.rec ? sl.rec[sl.lstride + j] : sl.b[j];
                if (av >= (uint32_t)sl.n || bv >= (uint32_t)sl.n) bad = true;
            }
            if (bad) {
                sl.result_len = kLenInvalid;
                for (int c = 0; c < kLevelWordU64; ++c) sl.word[c] = 0ull;
                if (out.out_len && sl.tag >= 0) out.out_len[sl.tag] = kLenInvalid;
                if (out.error) atomicOr(out.error, kErrInvalid);
                sl.state = kSlotDone;
                atomicAdd(&ctl->finished, 1u);
                continue;
            }
            const uint32_t full = sl.n >= 32 ? 0xFFFFFFFFu : (1u << sl.n) - 1u;
            sl.queue[0] = full;
            sl.bitmap[full >> 5] = 1u << (full & 31u);
            sl.lvl_start = 0;
            sl.lvl_end = 1;
            sl.tail = 1;
            sl.level = 0;
            sl.found = ~0ull;
            sl.overflow = 0;
            sl.state = kSlotRun;
        } else if (st == kSlotRun) {
            const unsigned long long f = *(volatile unsigned long long *)&sl.found;
            const unsigned long long tail = *(volatile unsigned long long *)&sl.tail;
            int32_t len = 0;
            int next = kSlotRun;
            if (f != ~0ull) {
                len = (int32_t)sl.level + 1;
                next = kSlotDone;
            } else if (sl.overflow || tail > sl.cap) {
                len = kLenNonSync;
                next = kSlotFail;
            } else if (tail == sl.lvl_end) {
                len = kLenNonSync;
                next = kSlotDone;
            }
            if (next == kSlotRun) {
                sl.lvl_start = sl.lvl_end;
                sl.lvl_end = tail;
                ++sl.level;
            } else {
                sl.result_len = len;
                for (int c = 0; c < kLevelWordU64; ++c) sl.word[c] = 0ull;
                if (next == kSlotDone && len > 0 && len <= 64 * kLevelWordU64) {
                    int d = len - 1;
                    sl.word[d >> 6] |= (uint64_t)(f & 1ull) << (d & 63);
                    uint64_t e = __ldcg(sl.queue + (f >> 1));
                    for (d = len - 2; d >= 0; --d) {
                        sl.word[d >> 6] |= (uint64_t)(e >> 63) << (d & 63);
                        e = __ldcg(sl.queue + ((e >> 28) & 0x7FFFFFFFFull));
                    }
                }
                if (out.out_len && sl.tag >= 0 && next == kSlotDone) {
                    record_result(out, sl.tag, sl.n, len);
                    if (out.out_words) {
                        uint64_t *w = out.out_words + (size_t)sl.tag * (size_t)out.word_stride;
                        for (int c = 0; c < out.word_stride; ++c) w[c] = c < kLevelWordU64 ? sl.word[c] : 0ull;
                    }
                }
                sl.state = next;
                atomicAdd(&ctl->finished, 1u);
            }
        }
    }
    __syncthreads();
    unsigned long long w = 0;
    if (tid < nslots && slots[tid].state == kSlotRun) w = slots[tid].lvl_end - slots[tid].lvl_start;
    unsigned long long incl = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) sh.warp_sum[tid >> 5] = incl;
    __syncthreads();
    unsigned long long before = 0;
    for (int q = 0; q < (tid >> 5); ++q) before += sh.warp_sum[q];
    const unsigned long long excl = before + incl - w;
    running = __syncthreads_count(w > 0);
    if (tid <= nslots) prefix_out[tid] = excl;   // prefix_out[nslots] = total (w = 0 there)
    unsigned long long total_new = 0;
    for (int q = 0; q < kThreads / 32; ++q) total_new += sh.warp_sum[q];
    __syncthreads();
    return total_new;
}

__global__ void __launch_bounds__(kThreads) k_level(LevelSlot *slots, uint64_t *tables, LevelCtl *ctl,
                                                    Batch out, int par)
{
    __shared__ LevelSmem<kWideItems> sh;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int nslots = ctl->nslots;
    const unsigned long long total = ctl->total[par];
    // Only as many CTAs as the level needs take part (all of them while new
    // slots are being set up); the others leave at once, so a small level
    // does not pay for the whole grid's barriers and fences.
    const int n_init = ctl->n_init[par];
    const unsigned long long want = (total + blockDim.x - 1) / blockDim.x;
    const int need = n_init > 0 ? (int)gridDim.x : (int)max(1ull, min((unsigned long long)gridDim.x, want));
    if ((int)blockIdx.x >= need) return;
    // slots admitted since the last transition (index >= prefix_n) have no work yet
    const int pn = min(ctl->prefix_n[par], nslots);
    for (int i = tid; i <= nslots; i += blockDim.x) sh.prefix[i] = ctl->prefix[par][i <= pn ? i : pn];

    // ---- set-up of freshly admitted slots: clear bitmaps, build tables ------
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + tid;
    const size_t gthreads = (size_t)need * blockDim.x;
    for (int q = 0; q < n_init; ++q) {
        const int s = ctl->init_list[q];
        LevelSlot &sl = slots[s];
        const size_t words4 = sl.n >= 7 ? ((size_t)1 << sl.n) / 128 : 1;
        uint4 *bm4 = reinterpret_cast<uint4 *>(sl.bitmap);
        for (size_t w = gtid; w < words4; w += gthreads) bm4[w] = make_uint4(0u, 0u, 0u, 0u);
        uint64_t *tb = tables + (size_t)s * kLevelTable;
        for (size_t e = gtid; e < kLevelTable; e += gthreads) {
            const int c = (int)(e >> 8), v = (int)(e & 255);
            uint32_t ta = 0, tbv = 0;
            for (int j = 0; j < 8; ++j) {
                const int st = 8 * c + j;
                if (((v >> j) & 1) && st < sl.n) {
                    const uint32_t av = sl.rec ? sl.rec[st] : sl.a[st];
                    const uint32_t bv = sl.rec ? sl.rec[sl.lstride + st] : sl.b[st];
                    ta |= 1u << (av & 31u);
                    tbv |= 1u << (bv & 31u);
                }
            }
            tb[e] = ((uint64_t)ta << 32) | tbv;
        }
    }
    if (tid < kMaxLevelSlots) sh.slot_count[tid] = 0;
    for (int q = tid; q < nslots; q += blockDim.x) sh.lvl_start[q] = slots[q].lvl_start;
    __syncthreads();

    unsigned long long expanded = level_items<kWideItems>(slots, tables, sh, nslots, total, blockIdx.x, need);
    for (int o = 16; o; o >>= 1) expanded += __shfl_down_sync(kFull, expanded, o);
    if (lane == 0 && expanded) atomicAdd(&ctl->expanded, expanded);

    // ---- the last CTA moves every slot to its next level ---------------------
    __threadfence();
    __syncthreads();
    if (tid == 0) sh.last = atomicAdd(&ctl->done_ctas, 1u) == (unsigned)need - 1;
    __syncthreads();
    if (!sh.last) return;
    __threadfence();
    const int nxt = par ^ 1;
    int running = 0;
    const unsigned long long total_new = level_transition(slots, ctl, out, sh, nslots, ctl->prefix[nxt], running);
    if (tid == 0) {
        ctl->total[nxt] = total_new;
        ctl->prefix_n[nxt] = nslots;
        ctl->running = running;
        ctl->n_init[nxt] = 0;
        ctl->launches += 1;
        ctl->done_ctas = 0;
        __threadfence();
    }
}

// Narrow levels: one cluster of kNarrowCluster CTAs runs consecutive levels by
// itself -- all CTAs expand their share of the level, rank 0 moves every slot
// to its next level, the others take the new prefix sums from rank 0's shared
// memory -- with hardware cluster barriers instead of launches between levels,
// while the levels stay at most `narrow` subsets wide, up to `max_levels`
// levels.  Levels of at most one CTA round (the Cerny automata's long tails:
// 289 of C_28's levels have at most 512 subsets) are run by rank 0 alone with
// CTA barriers, the other CTAs waiting at one cluster barrier (C_28 12.8 ->
// 12.5 ms).  Launched as one cluster, and only when no slot awaits set-up.
__global__ void __cluster_dims__(kNarrowCluster, 1, 1) __launch_bounds__(kThreads)
    k_level_narrow(LevelSlot *slots, uint64_t *tables, LevelCtl *ctl, Batch out, int par, int max_levels,
                   unsigned long long narrow)
{
    __shared__ LevelSmem<1> sh;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int nslots = ctl->nslots;
    unsigned long long total = ctl->total[par];
    const int pn = min(ctl->prefix_n[par], nslots);
    for (int i = tid; i <= nslots; i += blockDim.x) sh.prefix[i] = ctl->prefix[par][i <= pn ? i : pn];
    for (int q = tid; q < nslots; q += blockDim.x) sh.lvl_start[q] = slots[q].lvl_start;
    if (tid < kMaxLevelSlots) sh.slot_count[tid] = 0;
    __syncthreads();
    unsigned long long expanded = 0;
    int running = 0;
    LevelSmem<1> *sh0 = cluster.map_shared_rank(&sh, 0);
    int it = 0;
    while (it < max_levels) {
        if (total <= (unsigned long long)kThreads) {
            // levels of at most one round: rank 0 runs them by itself with CTA
            // barriers only, while the other CTAs wait at one cluster barrier
            if (rank == 0) {
                while (it < max_levels) {
                    expanded += level_items<1>(slots, tables, sh, nslots, total, 0, 1);
                    __syncthreads();
                    total = level_transition(slots, ctl, out, sh, nslots, sh.prefix, running);
                    for (int q = tid; q < nslots; q += blockDim.x) sh.lvl_start[q] = slots[q].lvl_start;
                    __syncthreads();
                    ++it;
                    if (running == 0 || total > (unsigned long long)kThreads) break;
                }
                if (tid == 0) {
                    sh.b_total = total;
                    sh.b_running = running;
                    sh.b_it = it;
                }
            }
            cluster.sync();   // rank 0's levels are done and its results visible
            if (rank != 0) {
                for (int i = tid; i <= nslots; i += blockDim.x) sh.prefix[i] = sh0->prefix[i];
                for (int q = tid; q < nslots; q += blockDim.x) sh.lvl_start[q] = sh0->lvl_start[q];
            }
            total = sh0->b_total;
            running = sh0->b_running;
            it = sh0->b_it;
            __syncthreads();
            cluster.sync();   // every CTA has read rank 0's results before rank 0 writes again
            if (running == 0 || total > narrow) break;
            continue;
        }
        expanded += level_items<1>(slots, tables, sh, nslots, total, rank, kNarrowCluster);
        cluster.sync();   // every CTA's pushes of this level are in
        if (rank == 0) {
            total = level_transition(slots, ctl, out, sh, nslots, sh.prefix, running);
            if (tid == 0) {
                sh.b_total = total;
                sh.b_running = running;
            }
            for (int q = tid; q < nslots; q += blockDim.x) sh.lvl_start[q] = slots[q].lvl_start;
        }
        cluster.sync();   // rank 0's transition is visible
        if (rank != 0) {
            for (int i = tid; i <= nslots; i += blockDim.x) sh.prefix[i] = sh0->prefix[i];
            for (int q = tid; q < nslots; q += blockDim.x) sh.lvl_start[q] = sh0->lvl_start[q];
            total = sh0->b_total;
            running = sh0->b_running;
            __syncthreads();
        } else {
            __syncthreads();
            total = sh.b_total;
            running = sh.b_running;
        }
        ++it;
        if (running == 0 || total > narrow) break;
    }
    for (int o = 16; o; o >>= 1) expanded += __shfl_down_sync(kFull, expanded, o);
    if (lane == 0 && expanded) atomicAdd(&ctl->expanded, expanded);
    cluster.sync();   // rank 0's shared memory stays valid until every CTA is done reading it
    if (rank != 0) return;
    const int nxt = par ^ 1;
    for (int i = tid; i <= nslots; i += blockDim.x) ctl->prefix[nxt][i] = sh.prefix[i];
    if (tid == 0) {
        ctl->total[nxt] = total;
        ctl->prefix_n[nxt] = nslots;
        ctl->running = running;
        ctl->n_init[nxt] = 0;
        ctl->launches += 1;
        __threadfence();
    }
}

}  // namespace

int level_max_ctas_per_sm()
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_level, kThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

cudaError_t launch_level(int ctas, int parity, LevelSlot *slots, uint64_t *tables, LevelCtl *ctl, const Batch &out,
                         cudaStream_t st)
{
    if (ctas < 1) return cudaErrorInvalidValue;
    k_level<<<ctas, kThreads, 0, st>>>(slots, tables, ctl, out, parity & 1);
    return cudaGetLastError();
}

cudaError_t launch_level_narrow(int parity, int max_levels, unsigned long long narrow, LevelSlot *slots,
                                uint64_t *tables, LevelCtl *ctl, const Batch &out, cudaStream_t st)
{
    if (max_levels < 1) return cudaErrorInvalidValue;
    k_level_narrow<<<kNarrowCluster, kThreads, 0, st>>>(slots, tables, ctl, out, parity & 1, max_levels, narrow);
    return cudaGetLastError();
}

}  // namespace sbfs
