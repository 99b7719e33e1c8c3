// api.cu -- the C ABI of include/sbfs.h.
//
// Host flow of one sbfs_solve_batch call (the native counterpart of
// GPGPU/GPU/SlimGPUQueue.cs:32-208, which allocates, flattens and copies per
// call, launches one kernel per stream and copies back):
//   * device buffers are grow-only and owned by the handle, so steady-state
//     calls allocate nothing;
//   * the batch is cut into chunks that rotate over the handle's lanes
//     (streams): chunk c's host->device copy overlaps chunk c-1's kernels and
//     chunk c-2's device->host copy;
//   * per chunk: reset counters, bucket by size class when n varies, run each
//     class's kernel, copy lengths/words/counters back;
//   * caller buffers in pinned memory are copied directly; pageable ones go
//     through the lane's pinned staging buffers.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>

#include "runtime.cuh"

namespace sbfs {

size_t cta_smem_bytes(int nb_max);
size_t cta_queue_entries(int nb_max, int ctas);
int cta_max_ctas_per_sm(int nb_max, int threads);
cudaError_t launch_cta(int nb_max, int threads, int ctas, const Batch &b, uint64_t *queues,
                       unsigned long long *ticket, cudaStream_t st);
cudaError_t plan_autotune(sbfs_handle *h, Plan &plan);
int hash_max_ctas_per_sm(int size);
cudaError_t launch_sort_handoff(const Batch &b, const int32_t *list, const unsigned long long *count, int32_t *out,
                                int top_n, unsigned long long *split, cudaStream_t st);
cudaError_t launch_hash(int size, int ctas, const Batch &b, int32_t *heavy_list, unsigned long long *heavy_count,
                        unsigned long long *ticket, cudaStream_t st);

cudaError_t DevBuf::reserve(size_t want)
{
    if (want <= bytes && ptr) return cudaSuccess;
    release();
    size_t sz = std::max<size_t>(want, 256);
    cudaError_t e = cudaMalloc(&ptr, sz);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return e;
    }
    bytes = sz;
    return cudaSuccess;
}

void DevBuf::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

cudaError_t HostBuf::reserve(size_t want)
{
    if (want <= bytes && ptr) return cudaSuccess;
    release();
    size_t sz = std::max<size_t>(want, 256);
    // mapped, so kernels may store into it (the streamed host path's chunk flags)
    cudaError_t e = cudaHostAlloc(&ptr, sz, cudaHostAllocMapped);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return e;
    }
    bytes = sz;
    return cudaSuccess;
}

void HostBuf::release()
{
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

}  // namespace sbfs

using namespace sbfs;

namespace {

__global__ void finalize_violation(const DevCounters *c, int64_t *out)
{
    *out = c->first_violation == ULLONG_MAX ? -1ll : (int64_t)c->first_violation;
}

thread_local std::string g_create_error;

constexpr int kDefaultLanes = 4;
// levels a pooled warp spends on one automaton before handing it to the
// CTA-wide kernel: random automata with n <= 20 stay below 40 (max 36 in 20K
// samples at n = 20), a Cerny automaton needs (n-1)^2
constexpr int kPoolLevelCap = 48;
constexpr int kHandoffThreads16 = 256;   // CTA width of the CTA-wide kernel on n <= 16 hand-offs
constexpr int64_t kDefaultChunk = 1 << 18;

sbfs_status fail(sbfs_handle *h, sbfs_status st, const std::string &msg)
{
    if (h)
        h->last_error = msg;
    else
        g_create_error = msg;
    return st;
}

sbfs_status cuda_fail(sbfs_handle *h, cudaError_t e, const char *what)
{
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return fail(h, e == cudaErrorMemoryAllocation ? SBFS_ENOMEM : SBFS_ECUDA, msg);
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t _e = (call);                         \
        if (_e != cudaSuccess) return cuda_fail(h, _e, what); \
    } while (0)

bool is_pinned(const void *p)
{
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

struct Job {
    const uint8_t *maps;     // device
    int32_t lstride;
    const uint8_t *ns;       // device or null
    int32_t n_uniform;
    int32_t max_n;           // largest n in the job (bounds buffer sizes)
    int64_t count;
    int32_t *len;            // device or null
    uint64_t *words;         // device or null
    int32_t word_stride;
    unsigned int *done_flag = nullptr;   // per-automaton completion flags (serving)
    unsigned int done_tag = 0;
};

int class_present_mask(const Job &j)
{
    if (!j.ns) return 1 << class_of_n(j.n_uniform);
    int m = 0;
    for (int c = 0; c < kNumClasses; ++c)
        if (c == 0 || j.max_n > (c ? kClassMaxN[c - 1] : 0)) m |= 1 << c;
    return m;
}

size_t level_arena_bytes(sbfs_handle *h, int max_n)
{
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = (size_t)8 << 30;
    }
    size_t want = free_b / 2;
    const size_t cap = (size_t)64 << 30;
    if (want > cap) want = cap;
    if (h->cfg.level_arena_bytes > 0) want = (size_t)h->cfg.level_arena_bytes;
    const size_t one = LevelEngine::footprint(max_n);
    if (want < one) want = one;   // at least one automaton of the largest size
    return want;
}

// Automata with 21 <= n <= 28 run on the device-resident level slots: admit as
// many as the arena holds, advance them a few levels per launch batch, collect
// the finished ones, admit more.  Results land in the job's device outputs.
sbfs_status run_level_class(sbfs_handle *h, Lane &L, const Job &j, const Batch &bc, int *launches)
{
    std::vector<std::pair<int64_t, int>> items;
    if (!j.ns) {
        items.reserve((size_t)j.count);
        for (int64_t i = 0; i < j.count; ++i) items.push_back({i, j.n_uniform});
    } else {
        // class-4 members come from the device bucketing: read the range, the order slice and sizes
        unsigned long long range[2] = {0, 0};
        CK(cudaMemcpyAsync(range, bc.range_dev, sizeof(range), cudaMemcpyDeviceToHost, L.stream),
           "reading class range");
        CK(cudaStreamSynchronize(L.stream), "waiting for bucketing");
        if (range[1] == 0) return SBFS_OK;
        std::vector<int32_t> idx((size_t)range[1]);
        std::vector<uint8_t> ns((size_t)j.count);
        CK(cudaMemcpy(idx.data(), bc.order + range[0], idx.size() * sizeof(int32_t), cudaMemcpyDeviceToHost),
           "reading class members");
        CK(cudaMemcpy(ns.data(), j.ns, ns.size(), cudaMemcpyDeviceToHost), "reading sizes");
        for (int32_t i : idx) items.push_back({i, ns[(size_t)i]});
    }
    if (items.empty()) return SBFS_OK;
    int max_n = 0;
    for (auto &it : items) max_n = std::max(max_n, it.second);
    max_n = std::min(std::max(max_n, 1), SBFS_MAX_N);
    if (!L.level_ready) {
        CK(L.level.init(h->sm_count, level_arena_bytes(h, max_n), L.stream), "setting up level slots");
        L.level_ready = true;
    } else if (L.level.arena_capacity() < LevelEngine::footprint(max_n)) {
        L.level.destroy();
        CK(L.level.init(h->sm_count, level_arena_bytes(h, max_n), L.stream), "setting up level slots");
    }
    LevelEngine &E = L.level;
    const unsigned long long expanded0 = E.expanded();
    size_t next = 0;
    int levels = 4;
    std::vector<LevelEngine::Finished> done;
    const size_t rec = 2 * (size_t)j.lstride;
    while (next < items.size() || E.in_flight() > 0) {
        while (next < items.size()) {
            const int n = items[next].second;
            if (n < 1 || n > SBFS_MAX_N) return fail(h, SBFS_EINVAL, "n out of range");
            if (E.admit(j.maps + (size_t)items[next].first * rec, j.lstride, n, items[next].first, nullptr,
                        nullptr) < 0)
                break;
            ++next;
        }
        if (E.in_flight() == 0) return fail(h, SBFS_ENOMEM, "level-slot arena cannot hold one automaton");
        CK(E.launch(levels, bc, 4096), "launching level kernels");
        *launches += levels;
        done.clear();
        CK(E.collect(done), "collecting level slots");
        for (auto &f : done)
            if (f.state == kSlotFail) return fail(h, SBFS_ECUDA, "level slot queue overflow");
        // long-running automata: fewer host round trips -- but once the levels
        // have shrunk to a few narrow-level widths, short batches, so that the
        // host sees them become narrow and hands them to the one-cluster kernel
        // (a whole-grid launch costs ~11 us even for a narrow level; C_28 has
        // 112 levels between 256K and 16K subsets on its way down)
        const int cap = E.level_total() <= 16 * kNarrowLevel ? 16 : 256;
        levels = done.empty() ? std::min(levels * 2, cap) : 4;
    }
    L.level_expanded += E.expanded() - expanded0;
    return SBFS_OK;
}

// A uniform batch of n = 13 runs on the per-lane kernel k_lane<13>.
// (and of n = 14 on k_lane<14>); the shape, or null
const LaneShape *uniform_lane(const sbfs_handle *h, const uint8_t *ns, int32_t n_uniform)
{
    if (ns) return nullptr;
    if (n_uniform == 13 && h->plan.use_lane13) return &h->plan.lane13;
    if (n_uniform == 14 && h->plan.use_lane14) return &h->plan.lane14;
    return nullptr;
}

// Reserve the lane's work buffers for a job and enqueue its kernels on the lane's
// stream.  Counters must already be reset.
sbfs_status enqueue_kernels(sbfs_handle *h, Lane &L, const Job &j, int *launches, bool plain = false,
                            unsigned long long *ticket_override = nullptr)
{
    const Plan &P = h->plan;
    cudaStream_t st = L.stream;
    DevCounters *ctr = L.counters.as<DevCounters>();
    Batch b{};
    b.maps = j.maps;
    b.lstride = j.lstride;
    b.ns = j.ns;
    b.n_uniform = j.n_uniform;
    b.order = nullptr;
    b.count = j.count;
    b.range_dev = nullptr;
    b.out_len = j.len;
    b.out_words = j.words;
    b.word_stride = j.word_stride;
    b.slack = h->cfg.slack;
    b.first_violation = &ctr->first_violation;
    b.expanded = &ctr->expanded;
    b.error = &ctr->error;
    b.done_flag = j.done_flag;
    b.done_tag = j.done_tag;

    const int present = class_present_mask(j);
    const size_t escal_entries = (size_t)std::max<int64_t>(j.count, 1);
    // a mixed batch: classes 0..2 each on their own stream, forked after the bucketing
    const bool fork = j.ns && !plain && __builtin_popcount((unsigned)present) > 1 && L.aux[0];
    bool joined[3] = {false, false, false};
    if (j.ns) {
        CK(L.order.reserve((size_t)j.count * sizeof(int32_t)), "allocating order array");
        // hist[K] | ranges[2K] | cursor[K]
        CK(L.ranges.reserve(4 * kNumClasses * sizeof(unsigned long long)), "allocating class ranges");
        unsigned long long *r = L.ranges.as<unsigned long long>();
        ClassScratch sc{r, r + kNumClasses, r + 3 * kNumClasses, L.order.as<int32_t>()};
        CK(launch_classify(j.ns, j.count, sc, h->sm_count, st), "launching size-class bucketing");
        *launches += 3;
        b.order = sc.order;
        if (fork) CK(cudaEventRecord(L.ev_fork, st), "recording event");
    }
    for (int c = 0; c < kNumClasses; ++c) {
        if (!(present & (1 << c))) continue;
        Batch bc = b;
        if (j.ns) bc.range_dev = L.ranges.as<unsigned long long>() + kNumClasses + 2 * c;
        unsigned long long *ticket = ticket_override ? ticket_override : &ctr->ticket[c];
        cudaStream_t cs = st;
        if (fork && c < 3) {
            cs = L.aux[c];
            CK(cudaStreamWaitEvent(cs, L.ev_fork, 0), "ordering streams");
            joined[c] = true;
        }
        const LaneShape *ul = c == 2 && !plain && !ticket_override ? uniform_lane(h, j.ns, j.n_uniform) : nullptr;
        const bool lane13 = ul != nullptr;
        if ((c < 2 && !plain && !P.use_pool[c]) || lane13) {
            const LaneShape &ls = lane13 ? *ul : P.lane[c];
            // one escalation list per lane class (a uniform n = 13 batch has no
            // class 1 and takes its list and counters); entries read as -1 until stored
            const int lc = lane13 ? 1 : c;
            CK(L.escal.reserve(2 * escal_entries * sizeof(int32_t)), "allocating escalation list");
            int32_t *list = L.escal.as<int32_t>() + (size_t)lc * escal_entries;
            CK(cudaMemsetAsync(list, 0xFF, escal_entries * sizeof(int32_t), cs), "resetting escalation list");
            CK(launch_lane(ls.nmax, ls.warps, ls.ring, ls.refill_k, ls.tail_k, ls.ctas, bc, list, escal_entries,
                           &ctr->escal_count[lc], &ctr->escal_claim[lc], ticket, LaneStream{}, cs),
               "launching per-lane kernel");
        } else if ((c == 2 && P.class2_hash && !plain && !ticket_override) ||
                   (c == 3 && P.class3_hash && !P.class3_level)) {
            const int size = c == 2 ? P.class2_hash : P.class3_hash;
            const int nb = c == 2 ? kClassMaxN[2] : std::min(20, std::max(j.ns ? j.max_n : j.n_uniform, 17));
            // class 2's hand-offs (Cerny C_13..C_16: a few hundred subsets per level)
            // run 256-thread CTAs, several per SM; class 3 keeps the tuned width
            const int threads = c == 2 && !plain && !ticket_override ? std::min(P.cta.threads, kHandoffThreads16)
                                                                     : P.cta.threads;
            const int per_sm = cta_max_ctas_per_sm(nb, threads);
            if (per_sm < 1) return fail(h, SBFS_ECUDA, "CTA-wide kernel does not fit on an SM");
            const int ctas = std::min(P.cta.ctas, per_sm * h->sm_count);
            CK(L.heavy_queue[c].reserve(cta_queue_entries(nb, ctas) * sizeof(uint64_t)), "allocating CTA queues");
            if (plain || ticket_override) {
                CK(launch_cta(nb, threads, ctas, bc, L.heavy_queue[c].as<uint64_t>(), ticket, cs),
                   "launching CTA-wide kernel");
            } else {
                // one warp per automaton with a hash set; searches wider than its
                // set or longer than its level cap go to the CTA-wide kernel, same stream
                const int hper = hash_max_ctas_per_sm(size);
                if (hper < 1) return fail(h, SBFS_ECUDA, "hash-set kernel does not fit on an SM");
                // hand-off list | the same sorted by n, largest first (mixed sizes)
                CK(L.heavy[c].reserve(2 * escal_entries * sizeof(int32_t)), "allocating hand-off list");
                int32_t *list = L.heavy[c].as<int32_t>();
                CK(launch_hash(size, hper * h->sm_count, bc, list, &ctr->heavy_range[c][1], ticket, cs),
                   "launching hash-set kernel");
                Batch bh = bc;
                bh.order = list;
                bh.range_dev = ctr->heavy_range[c];
                // class 3, mixed sizes: the hand-offs below the class's top n run in a
                // second launch sized for n - 1, whose halved bitmap fits two CTAs per SM
                const bool split = j.ns && c == 3 && nb >= 18;
                if (j.ns) {
                    CK(launch_sort_handoff(bc, list, &ctr->heavy_range[c][1], list + escal_entries, nb,
                                           split ? ctr->heavy_split[c] : nullptr, cs),
                       "launching hand-off sort");
                    bh.order = list + escal_entries;
                    *launches += 1;
                }
                if (split) {
                    const int nb2 = nb - 1;
                    const int per_sm2 = cta_max_ctas_per_sm(nb2, threads);
                    if (per_sm2 < 1) return fail(h, SBFS_ECUDA, "CTA-wide kernel does not fit on an SM");
                    const int ctas2 = std::min(P.cta.ctas, per_sm2 * h->sm_count);
                    CK(L.heavy_queue[c].reserve(std::max(cta_queue_entries(nb, ctas), cta_queue_entries(nb2, ctas2)) *
                                                sizeof(uint64_t)),
                       "allocating CTA queues");
                    bh.range_dev = ctr->heavy_split[c];
                    CK(launch_cta(nb, threads, ctas, bh, L.heavy_queue[c].as<uint64_t>(), &ctr->heavy_ticket[c], cs),
                       "launching hand-off kernel");
                    bh.range_dev = ctr->heavy_split[c] + 2;
                    CK(launch_cta(nb2, threads, ctas2, bh, L.heavy_queue[c].as<uint64_t>(), &ctr->heavy_ticket2[c],
                                  cs),
                       "launching hand-off kernel");
                    *launches += 2;
                } else {
                    CK(launch_cta(nb, threads, ctas, bh, L.heavy_queue[c].as<uint64_t>(), &ctr->heavy_ticket[c], cs),
                       "launching hand-off kernel");
                    *launches += 1;
                }
            }
        } else if (c < 3) {
            const PoolShape &s = P.pool[c];
            DevBuf &spill = fork ? L.spill_c[c] : L.spill;
            CK(spill.reserve(pool_spill_words(s) * sizeof(uint32_t)), "allocating queue spill");
            if (plain || ticket_override) {
                CK(launch_pool(s, bc, spill.as<uint32_t>(), ticket, cs), "launching small-n kernel");
            } else {
                // long thin searches (Cerny automata: (n-1)^2 levels) leave the pooled
                // warp after kPoolLevelCap levels for the CTA-wide kernel, same stream
                CK(L.heavy[c].reserve(escal_entries * sizeof(int32_t)), "allocating hand-off list");
                PoolHeavy hv{kPoolLevelCap, L.heavy[c].as<int32_t>(), &ctr->heavy_range[c][1]};
                CK(launch_pool(s, bc, spill.as<uint32_t>(), ticket, cs, hv), "launching small-n kernel");
                Batch bh = bc;
                bh.order = L.heavy[c].as<int32_t>();
                bh.range_dev = ctr->heavy_range[c];
                const int nb = s.nmax;
                const int per_sm = cta_max_ctas_per_sm(nb, P.cta.threads);
                if (per_sm < 1) return fail(h, SBFS_ECUDA, "hand-off kernel does not fit on an SM");
                const int ctas = std::min(P.cta.ctas, per_sm * h->sm_count);
                CK(L.heavy_queue[c].reserve(cta_queue_entries(nb, ctas) * sizeof(uint64_t)), "allocating CTA queues");
                CK(launch_cta(nb, P.cta.threads, ctas, bh, L.heavy_queue[c].as<uint64_t>(), &ctr->heavy_ticket[c], cs),
                   "launching hand-off kernel");
                *launches += 1;
            }
        } else if (c == 3 && P.class3_level && !plain) {
            sbfs_status ls = run_level_class(h, L, j, bc, launches);
            if (ls) return ls;
            continue;
        } else if (c == 3) {
            const int nb = std::min(20, std::max(j.ns ? j.max_n : j.n_uniform, 17));
            const int per_sm = cta_max_ctas_per_sm(nb, P.cta.threads);
            if (per_sm < 1) return fail(h, SBFS_ECUDA, "class-3 kernel does not fit on an SM");
            const int ctas = std::min(P.cta.ctas, per_sm * h->sm_count);
            CK(L.cta_queue.reserve(cta_queue_entries(nb, ctas) * sizeof(uint64_t)), "allocating CTA queues");
            CK(launch_cta(nb, P.cta.threads, ctas, bc, L.cta_queue.as<uint64_t>(), ticket, st), "launching n<=20 kernel");
        } else {
            sbfs_status ls = run_level_class(h, L, j, bc, launches);
            if (ls) return ls;
            continue;
        }
        *launches += 1;
        if (c < 3 && joined[c]) CK(cudaEventRecord(L.ev_join[c], cs), "recording event");
    }
    for (int c = 0; c < 3; ++c)
        if (joined[c]) CK(cudaStreamWaitEvent(st, L.ev_join[c], 0), "ordering streams");
    if (!plain && j.len && j.count > 0 && !j.done_flag) {
        CK(launch_count_sync(j.len, j.count, &ctr->synchronizing, h->sm_count, st), "launching result count");
        *launches += 1;
    }
    return SBFS_OK;
}

sbfs_status ensure_plan(sbfs_handle *h)
{
    if (h->plan_ready) return SBFS_OK;
    Plan &P = h->plan;
    const int sms = h->sm_count;
    const int defaults[3][4] = {
        // slots, warps, queue_smem
        {16, 8, 64, 0},
        {8, 2, 64, 0},
        {4, 2, 256, 0},
    };
    for (int c = 0; c < 3; ++c) {
        // configured shapes apply to every small-n class whose shared memory they fit
        PoolShape &s = P.pool[c];
        s.nmax = kClassMaxN[c];
        s.slots = h->cfg.slots_per_warp > 0 ? h->cfg.slots_per_warp : defaults[c][0];
        s.warps = h->cfg.warps_per_cta > 0 ? h->cfg.warps_per_cta : defaults[c][1];
        s.queue_smem = h->cfg.queue_smem > 0 ? h->cfg.queue_smem : defaults[c][2];
        s.ctas = 1;
        int per_sm = pool_max_ctas_per_sm(s);
        if (per_sm < 1) {
            s.slots = defaults[c][0];
            s.warps = defaults[c][1];
            s.queue_smem = defaults[c][2];
            per_sm = pool_max_ctas_per_sm(s);
        }
        if (per_sm < 1) return fail(h, SBFS_EINVAL, "small-n kernel shape does not fit in shared memory");
        s.ctas = per_sm * sms;
    }
    const int lane_defaults[2][4] = {
        // warps, ring, refill_k, tail_k (the autotuner's picks on B200 for uniform n = 8 and n = 12)
        {8, 16, 16, 4},
        {1, 64, 16, 4},
    };
    for (int c = 0; c < 2; ++c) {
        LaneShape &ls = P.lane[c];
        ls.nmax = kClassMaxN[c];
        ls.warps = h->cfg.lane_warps > 0 ? h->cfg.lane_warps : lane_defaults[c][0];
        ls.ring = h->cfg.lane_ring > 0 ? h->cfg.lane_ring : lane_defaults[c][1];
        ls.refill_k = h->cfg.lane_refill > 0 ? h->cfg.lane_refill : lane_defaults[c][2];
        ls.tail_k = h->cfg.lane_tail > 0 ? std::min(h->cfg.lane_tail, 32) : h->cfg.lane_tail < 0 ? 0 : lane_defaults[c][3];
        if (lane_max_ctas_per_sm(ls.nmax, ls.warps, ls.ring) < 1) {
            ls.warps = lane_defaults[c][0];
            ls.ring = lane_defaults[c][1];
        }
        const int per_sm = lane_max_ctas_per_sm(ls.nmax, ls.warps, ls.ring);
        if (per_sm < 1) return fail(h, SBFS_EINVAL, "per-lane kernel shape does not fit in shared memory");
        ls.ctas = per_sm * sms;
    }
    {
        // uniform n = 13: 1 KB of bitmap per lane and a 128-entry ring, four
        // one-warp CTAs per SM.  2^21 automata: ring 32 3.47 ms, 64 2.48 ms,
        // 128 2.03 ms, 256 2.60 ms, 512 3.84 ms -- a small ring escalates more
        // searches to the whole-warp path, a large one costs resident warps
        LaneShape &ls = P.lane13;
        ls.nmax = 13;
        ls.warps = 1;
        ls.ring = 128;
        ls.refill_k = 16;
        ls.tail_k = 4;
        const int per_sm = lane_max_ctas_per_sm(13, ls.warps, ls.ring);
        ls.ctas = per_sm * sms;
        P.use_lane13 = per_sm > 0 && h->cfg.small_kernel != 2 ? 1 : 0;
    }
    {
        // uniform n = 14: 2 KB of bitmap per lane and a 256-entry ring, two
        // one-warp CTAs per SM.  2^21 automata: 4.83 ms (k_hash: 7.80 ms; ring
        // 128: 5.19 ms; ring 512, one CTA per SM: 9.48 ms)
        LaneShape &ls = P.lane14;
        ls.nmax = 14;
        ls.warps = 1;
        ls.ring = 256;
        ls.refill_k = 16;
        ls.tail_k = 4;
        const int per_sm = lane_max_ctas_per_sm(14, ls.warps, ls.ring);
        ls.ctas = per_sm * sms;
        P.use_lane14 = per_sm > 0 && h->cfg.small_kernel != 2 ? 1 : 0;
    }
    P.cta.threads = 1024;   // the autotuner's pick with Cerny members in the batch
    P.cta.ctas = sms * 4;
    P.hbm.threads = 512;
    P.hbm.ctas = sms * 4;
    P.use_pool[0] = P.use_pool[1] = h->cfg.small_kernel == 2 ? 1 : 0;
    P.class3_level = 0;
    P.class2_hash = h->cfg.small_kernel == 2 ? 0 : 1;   // small_kernel 2: the pooled kernel up to n = 16
    P.class3_hash = 1;
    P.tuned = 0;
    h->plan_ready = true;   // the tuner below runs batches with the defaults in place
    if (h->cfg.autotune) {
        cudaError_t e = plan_autotune(h, P);
        if (e != cudaSuccess) {
            h->plan_ready = false;
            return cuda_fail(h, e, "autotuning kernel shapes");
        }
    }
    return SBFS_OK;
}

sbfs_status check_records(sbfs_handle *h, const uint8_t *maps, int32_t lstride, const uint8_t *ns,
                          int32_t n_uniform, int64_t count, int32_t *max_n, int32_t *same_n = nullptr)
{
    if (same_n) *same_n = 0;
    if (count < 0) return fail(h, SBFS_EINVAL, "negative count");
    if (count > 0 && !maps) return fail(h, SBFS_EINVAL, "maps is NULL");
    if (lstride < 1 || lstride > 32) return fail(h, SBFS_EINVAL, "lstride must be in 1..32");
    if (!ns) {
        if (n_uniform < 1 || n_uniform > SBFS_MAX_N || n_uniform > lstride)
            return fail(h, SBFS_EINVAL, "n_uniform must be in 1..min(28, lstride)");
        *max_n = n_uniform;
    } else {
        int m = 0, lo = 255;
        for (int64_t i = 0; i < count; ++i) {
            m = std::max<int>(m, ns[i]);
            lo = std::min<int>(lo, ns[i]);
        }
        *max_n = std::min(m, SBFS_MAX_N);
        // every automaton has the same valid n: the batch is uniform
        if (same_n && count > 0 && lo == m && m >= 1 && m <= SBFS_MAX_N && m <= lstride) *same_n = m;
    }
    return SBFS_OK;
}

sbfs_status reset_counters(sbfs_handle *h, Lane &L)
{
    CK(L.counters.reserve(sizeof(DevCounters)), "allocating counters");
    CK(cudaMemsetAsync(L.counters.ptr, 0, sizeof(DevCounters), L.stream), "resetting counters");
    L.level_expanded = 0;
    CK(cudaMemsetAsync(&L.counters.as<DevCounters>()->first_violation, 0xFF, sizeof(unsigned long long),
                       L.stream),
       "resetting counters");
    return SBFS_OK;
}

struct Totals {
    int64_t first_violation = -1;
    int64_t expanded = 0;
    int64_t escalated = 0;
    int64_t synchronizing = 0;
    int error = 0;
    double kernel_ms = 0;
};

sbfs_status finish_lane(sbfs_handle *h, Lane &L, Totals &t)
{
    if (!L.busy) return SBFS_OK;
    L.busy = false;
    CK(cudaEventSynchronize(L.ev_done), "waiting for a chunk");
    const DevCounters *c = L.h_counters.as<DevCounters>();
    t.error |= c->error;
    t.expanded += (int64_t)(c->expanded + L.level_expanded);
    t.escalated += (int64_t)(c->escal_count[0] + c->escal_count[1]);
    t.synchronizing += (int64_t)c->synchronizing;
    if (c->first_violation != ULLONG_MAX) {
        const int64_t g = L.begin + (int64_t)c->first_violation;
        if (t.first_violation < 0 || g < t.first_violation) t.first_violation = g;
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, L.ev_k0, L.ev_k1) == cudaSuccess) t.kernel_ms += ms;
    cudaGetLastError();
    if (L.staged_out) {
        CopyPool::Group g;
        if (L.user_len) h->copy_pool().copy(L.user_len + L.begin, L.h_len.ptr, (size_t)L.count * sizeof(int32_t), g);
        if (L.user_words)
            h->copy_pool().copy(L.user_words + (size_t)L.begin * L.word_stride, L.h_words.ptr,
                                (size_t)L.count * L.word_stride * sizeof(uint64_t), g);
        h->copy_pool().wait(g);
    }
    return SBFS_OK;
}

// Runs `body` (stream work on L.stream) directly, or replays it from a CUDA
// graph.  A key's first run is direct (it sizes the lane's buffers); its second
// run is captured; later runs launch the graph.  A graph whose lane buffers
// moved since capture is rebuilt.
template <class F>
sbfs_status run_maybe_captured(sbfs_handle *h, Lane &L, const std::string &key, bool allow, int *launches, F &&body)
{
    if (!allow) return body();
    auto it = L.graphs.find(key);
    if (it != L.graphs.end()) {
        if (it->second.sig == L.signature()) {
            CK(cudaGraphLaunch(it->second.exec, L.stream), "launching graph");
            *launches += it->second.launches;
            return SBFS_OK;
        }
        cudaGraphExecDestroy(it->second.exec);
        L.graphs.erase(it);
    }
    if (!L.seen.count(key)) {
        L.seen.insert(key);
        return body();
    }
    const uint64_t sig = L.signature();
    const int before = *launches;
    CK(cudaStreamBeginCapture(L.stream, cudaStreamCaptureModeThreadLocal), "beginning capture");
    const sbfs_status s = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(L.stream, &g);
    if (s != SBFS_OK || e != cudaSuccess || L.signature() != sig) {
        // not capturable this time (or it reallocated): run it directly instead
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        *launches = before;
        return body();
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        cudaGetLastError();
        *launches = before;
        return body();
    }
    if (L.graphs.size() >= 64) L.drop_graphs();
    L.graphs[key] = {exec, sig, *launches - before};
    CK(cudaGraphLaunch(exec, L.stream), "launching graph");
    return SBFS_OK;
}

// Launch sequences that never wait on the host (no level-slot classes) can be captured.
bool graph_safe(sbfs_handle *h, int max_n)
{
    return max_n <= kClassMaxN[2] || (max_n <= kClassMaxN[3] && !h->plan.class3_level);
}

std::string graph_key(const void *a, const void *b, const void *c, const void *d, const void *e, int64_t cnt,
                      int lstride, int n_uniform, int max_n, int ws)
{
    char buf[256];
    std::snprintf(buf, sizeof buf, "%p|%p|%p|%p|%p|%lld|%d|%d|%d|%d", a, b, c, d, e, (long long)cnt, lstride,
                  n_uniform, max_n, ws);
    return buf;
}

// Streamed host path for a uniform batch of n <= 14 on the per-lane kernel:
// one kernel launch per job instead of one per chunk (each launch pays the
// BFS's longest tail), with the copies of both directions overlapping it.
//  - copy_in: records chunk by chunk, each followed by its chunk_ready flag;
//    the kernel waits (bounded) only for a chunk its ticket has reached;
//  - the kernel counts lane outcomes per chunk and the warp that completes a
//    chunk sets the chunk's flag in mapped host memory;
//  - this thread polls those flags and copies each finished chunk's lengths
//    and words out on copy_out while the kernel still runs;
//  - automata solved by the whole-warp search finish late: they are also
//    written to a compact array (by escalation slot) and, after the last
//    chunk's copy, stored into the host results by a small kernel through
//    mapped memory (pinned results) or by the host threads (pageable ones);
//  - a pageable caller's records are staged into pinned memory chunk by
//    chunk, and its results go on from pinned staging as each chunk lands,
//    both by the handle's host copy threads.
constexpr int64_t kStreamChunk = 1 << 17;   // x 2n bytes: whole 128-byte lines
// Chunk 0's size.  A 2^14-automaton first chunk (the kernel starts after a
// 0.4 MB copy instead of 3 MB) measured the same end to end with pinned buffers
// (0.913-0.946 ms against 0.923-0.941 ms per 10^6 automata at n = 12) and
// slower with pageable ones (2.06-2.20 ms against 1.44-1.63 ms): the kernel
// then waits on chunk 1 while the host stages it.
constexpr int64_t kStreamFirst = kStreamChunk;
constexpr int64_t kStreamJob = 1 << 24;     // automata per kernel launch

bool stream_eligible(sbfs_handle *h, const uint8_t *ns, int32_t n_uniform, int64_t count, bool plain)
{
    if (plain || ns || h->cfg.chunk != 0 || count < 2 * kStreamChunk) return false;
    const int c = class_of_n(n_uniform);
    return (c < 2 && !h->plan.use_pool[c]) || uniform_lane(h, ns, n_uniform) != nullptr;
}

struct StreamOut {
    int64_t expanded = 0, escalated = 0, synchronizing = 0, first_violation = -1;
    int error = 0;
    double kernel_ms = 0;
    int launches = 0;
};

sbfs_status solve_streamed_job(sbfs_handle *h, const uint8_t *maps, int32_t lstride, int32_t n, int64_t cnt,
                               int32_t *out_len, uint64_t *out_words, int32_t ws, bool pin_in, bool pin_out,
                               StreamOut &o)
{
    Lane &L = h->lanes[0];
    Streamer &S = h->streamer;
    const size_t rec = 2 * (size_t)lstride;
    LaneStream geo{};
    geo.chunk = kStreamChunk;
    geo.first = kStreamFirst;
    const int64_t nch = geo.chunks(cnt);
    const int c = class_of_n(n);
    // n = 13 (class 2) runs on k_lane<13> with class 1's escalation counters
    const int lc = c < 2 ? c : 1;
    const LaneShape &ls = c < 2 ? h->plan.lane[c] : *uniform_lane(h, nullptr, n);
    CK(L.maps.reserve(cnt * rec), "allocating records");
    if (out_len) CK(L.len.reserve(cnt * sizeof(int32_t)), "allocating lengths");
    if (out_words) CK(L.words.reserve((size_t)cnt * ws * sizeof(uint64_t)), "allocating words");
    CK(L.counters.reserve(sizeof(DevCounters)), "allocating counters");
    CK(L.h_counters.reserve(sizeof(DevCounters)), "allocating pinned counters");
    CK(L.escal.reserve((size_t)cnt * sizeof(int32_t)), "allocating escalation list");
    CK(S.flags.reserve(2 * (size_t)nch * sizeof(unsigned int)), "allocating chunk flags");
    CK(S.escal_out.reserve((size_t)cnt * sizeof(EscalResult)), "allocating escalated results");
    CK(S.h_flags.reserve(3 * (size_t)nch * sizeof(unsigned int)), "allocating host chunk flags");
    unsigned int *hf = S.h_flags.as<unsigned int>();   // host_flag | zeros | ones
    for (int64_t i = 0; i < nch; ++i) {
        hf[i] = 0u;
        hf[nch + i] = 0u;
        hf[2 * nch + i] = 1u;
    }
    unsigned int *d_host_flag = nullptr;
    CK(cudaHostGetDevicePointer((void **)&d_host_flag, hf, 0), "mapping host chunk flags");
    unsigned int *ready = S.flags.as<unsigned int>(), *done = ready + nch;
    const uint8_t *src = maps;
    if (!pin_in) {
        CK(L.h_maps.reserve(cnt * rec), "allocating pinned staging");
        src = L.h_maps.as<uint8_t>();
    }
    if (!pin_out && (int64_t)S.ev_out.size() < nch) {
        for (int64_t i = (int64_t)S.ev_out.size(); i < nch; ++i) {
            cudaEvent_t e = nullptr;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating events");
            S.ev_out.push_back(e);
        }
    }
    int32_t *dst_len = out_len;
    uint64_t *dst_words = out_words;
    if (!pin_out) {
        if (out_len) {
            CK(L.h_len.reserve(cnt * sizeof(int32_t)), "allocating pinned staging");
            dst_len = L.h_len.as<int32_t>();
        }
        if (out_words) {
            CK(L.h_words.reserve((size_t)cnt * ws * sizeof(uint64_t)), "allocating pinned staging");
            dst_words = L.h_words.as<uint64_t>();
        }
    }
    // flags through the copy engine only: a memset could need an SM that the
    // running kernel holds
    CK(cudaMemcpyAsync(ready, hf + nch, nch * sizeof(unsigned int), cudaMemcpyHostToDevice, h->copy_in),
       "clearing chunk flags");
    auto copy_chunk_in = [&](int64_t ci) -> sbfs_status {
        const int64_t a = geo.chunk_begin(ci), m = geo.chunk_size(ci, cnt);
        if (!pin_in) {
            // pageable records: this chunk into pinned staging first (host threads)
            CopyPool::Group g;
            h->copy_pool().copy(L.h_maps.as<uint8_t>() + a * rec, maps + a * rec, m * rec, g);
            h->copy_pool().wait(g);
        }
        CK(cudaMemcpyAsync(L.maps.as<uint8_t>() + a * rec, src + a * rec, m * rec, cudaMemcpyHostToDevice,
                           h->copy_in),
           "copying records");
        if (ci == h->skip_ready_chunk) return SBFS_OK;   // test hook: this chunk's flag never comes
        CK(cudaMemcpyAsync(ready + ci, hf + 2 * nch + ci, sizeof(unsigned int), cudaMemcpyHostToDevice, h->copy_in),
           "setting a chunk flag");
        return SBFS_OK;
    };
    sbfs_status st = copy_chunk_in(0);
    if (st) return st;
    CK(cudaEventRecord(S.ev_in0, h->copy_in), "recording event");
    // the kernel, behind chunk 0
    CK(cudaStreamWaitEvent(L.stream, S.ev_in0, 0), "ordering streams");
    CK(cudaMemsetAsync(L.counters.ptr, 0, sizeof(DevCounters), L.stream), "resetting counters");
    L.level_expanded = 0;
    CK(cudaMemsetAsync(&L.counters.as<DevCounters>()->first_violation, 0xFF, sizeof(unsigned long long), L.stream),
       "resetting counters");
    CK(cudaMemsetAsync(L.escal.ptr, 0xFF, (size_t)cnt * sizeof(int32_t), L.stream), "resetting escalation list");
    CK(cudaMemsetAsync(done, 0, nch * sizeof(unsigned int), L.stream), "resetting chunk counts");
    DevCounters *ctr = L.counters.as<DevCounters>();
    Batch b{};
    b.maps = L.maps.as<uint8_t>();
    b.lstride = lstride;
    b.n_uniform = n;
    b.count = cnt;
    b.out_len = out_len ? L.len.as<int32_t>() : nullptr;
    b.out_words = out_words ? L.words.as<uint64_t>() : nullptr;
    b.word_stride = out_words ? ws : 0;
    b.slack = h->cfg.slack;
    b.first_violation = &ctr->first_violation;
    b.expanded = &ctr->expanded;
    b.error = &ctr->error;
    LaneStream lsd = geo;
    lsd.chunk_ready = ready;
    lsd.chunk_done = done;
    lsd.host_flag = d_host_flag;
    lsd.escal_out = S.escal_out.as<EscalResult>();
    lsd.wait_polls = h->cfg.wait_polls > 0 ? h->cfg.wait_polls : (1 << 24);
    CK(cudaEventRecord(L.ev_k0, L.stream), "recording event");
    CK(launch_lane(ls.nmax, ls.warps, ls.ring, ls.refill_k, ls.tail_k, ls.ctas, b, L.escal.as<int32_t>(),
                   (unsigned long long)cnt, &ctr->escal_count[lc], &ctr->escal_claim[lc], &ctr->ticket[c], lsd,
                   L.stream),
       "launching per-lane kernel");
    CK(cudaEventRecord(L.ev_k1, L.stream), "recording event");
    o.launches += 1;
    // results out, chunk by chunk, as the kernel finishes them
    auto copy_chunk_out = [&](int64_t ci) -> sbfs_status {
        const int64_t a = geo.chunk_begin(ci), m = geo.chunk_size(ci, cnt);
        if (out_len)
            CK(cudaMemcpyAsync(dst_len + a, L.len.as<int32_t>() + a, m * sizeof(int32_t), cudaMemcpyDeviceToHost,
                               S.copy_out),
               "copying lengths");
        if (out_words)
            CK(cudaMemcpyAsync(dst_words + (size_t)a * ws, L.words.as<uint64_t>() + (size_t)a * ws,
                               (size_t)m * ws * sizeof(uint64_t), cudaMemcpyDeviceToHost, S.copy_out),
               "copying words");
        if (!pin_out) CK(cudaEventRecord(S.ev_out[ci], S.copy_out), "recording event");
        return SBFS_OK;
    };
    // pageable results: a chunk whose copy into pinned staging has completed is
    // copied on to the caller's buffers by the host threads, while later chunks
    // are still on the device
    CopyPool::Group g_out;
    CopyPool::Scope g_out_scope{pin_out ? nullptr : &h->copy_pool(), g_out};
    int64_t unstaged = 0;
    auto stage_out = [&](int64_t ci) {
        const int64_t a = geo.chunk_begin(ci), m = geo.chunk_size(ci, cnt);
        if (out_len) h->copy_pool().copy(out_len + a, dst_len + a, m * sizeof(int32_t), g_out);
        if (out_words)
            h->copy_pool().copy(out_words + (size_t)a * ws, dst_words + (size_t)a * ws,
                                (size_t)m * ws * sizeof(uint64_t), g_out);
    };
    int64_t next = 0;
    // non-blocking: copy out every chunk the kernel has finished, and stage on
    // every pageable chunk whose copy has landed
    auto poll_out = [&]() -> sbfs_status {
        sbfs_status ps;
        while (next < nch && *(volatile unsigned int *)(hf + next))
            if ((ps = copy_chunk_out(next++))) return ps;
        while (!pin_out && unstaged < next && cudaEventQuery(S.ev_out[unstaged]) == cudaSuccess)
            stage_out(unstaged++);
        return SBFS_OK;
    };
    // Every chunk copy is enqueued before anything else is launched behind the
    // kernel: the kernel waits for those chunks, and the first launch of a
    // kernel whose module is not loaded yet (CUDA loads modules lazily) can
    // block this thread until the device is idle -- which the running kernel
    // would then wait out to its bounded limit.
    // (Results of finished chunks go out in between: staging a pageable chunk
    // takes the host longer than the kernel takes to finish one.)
    for (int64_t ci = 1; ci < nch; ++ci) {
        if ((st = poll_out())) return st;
        if ((st = copy_chunk_in(ci))) return st;
    }
    if (out_len) {
        CK(launch_count_sync(b.out_len, cnt, &ctr->synchronizing, h->sm_count, L.stream), "launching result count");
        o.launches += 1;
    }
    CK(cudaMemcpyAsync(L.h_counters.ptr, L.counters.ptr, sizeof(DevCounters), cudaMemcpyDeviceToHost, L.stream),
       "copying counters");
    CK(cudaEventRecord(S.ev_kdone, L.stream), "recording event");
    const auto t_start = std::chrono::steady_clock::now();
    while (next < nch) {
        if (*(volatile unsigned int *)(hf + next)) {
            if ((st = copy_chunk_out(next))) return st;
            ++next;
            continue;
        }
        if (!pin_out && unstaged < next && cudaEventQuery(S.ev_out[unstaged]) == cudaSuccess) {
            stage_out(unstaged++);
            continue;
        }
        const cudaError_t q = cudaEventQuery(S.ev_kdone);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) CK(q, "waiting for the kernel");
        if (std::chrono::steady_clock::now() - t_start > std::chrono::seconds(600))
            return fail(h, SBFS_ETIMEOUT, "streamed solve: no progress for 600 s");
        std::this_thread::yield();
    }
    CK(cudaEventSynchronize(S.ev_kdone), "waiting for the kernel");
    for (; next < nch; ++next)
        if ((st = copy_chunk_out(next))) return st;
    // escalated automata finish after their chunk may have been copied: store
    // their results into the host output from the device, behind the copies
    // (pageable output: from the host, below, once the staged copies are done)
    int32_t *map_len = nullptr;
    uint64_t *map_words = nullptr;
    bool mapped = pin_out;
    if (mapped && dst_len && cudaHostGetDevicePointer((void **)&map_len, dst_len, 0) != cudaSuccess) mapped = false;
    if (mapped && dst_words && cudaHostGetDevicePointer((void **)&map_words, dst_words, 0) != cudaSuccess)
        mapped = false;
    cudaGetLastError();
    const DevCounters *hc = L.h_counters.as<DevCounters>();
    const int64_t esc = (int64_t)hc->escal_count[lc];
    if (esc > 0 && (out_len || out_words)) {
        if (mapped) {
            CK(launch_escal_patch(S.escal_out.as<EscalResult>(), &ctr->escal_count[lc], map_len, map_words, ws,
                                  h->sm_count, S.copy_out),
               "launching result patch");
            o.launches += 1;
        } else {
            CK(S.h_escal.reserve((size_t)esc * sizeof(EscalResult)), "allocating escalated results");
            CK(cudaMemcpyAsync(S.h_escal.ptr, S.escal_out.ptr, (size_t)esc * sizeof(EscalResult),
                               cudaMemcpyDeviceToHost, S.copy_out),
               "copying escalated results");
        }
    }
    CK(cudaStreamSynchronize(S.copy_out), "copying results");
    if (!pin_out) {
        while (unstaged < nch) stage_out(unstaged++);
        h->copy_pool().wait(g_out);
    }
    if (esc > 0 && (out_len || out_words) && !mapped) {
        // random stores into the caller's buffers, spread over the host threads
        const EscalResult *r = S.h_escal.as<EscalResult>();
        std::atomic<bool> corrupt{false};
        h->copy_pool().parallel_for((size_t)esc, 2048, [&](size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) {
                if (i + 16 < i1) {   // the stores miss the cache: keep several in flight
                    if (out_len) __builtin_prefetch(out_len + r[i + 16].k, 1);
                    if (out_words) __builtin_prefetch(out_words + (size_t)r[i + 16].k * ws, 1);
                }
                const int64_t k = r[i].k;
                if (k < 0 || k >= cnt) {
                    corrupt.store(true, std::memory_order_relaxed);
                    continue;
                }
                if (out_len) out_len[k] = r[i].len;
                if (out_words) {
                    uint64_t *w = out_words + (size_t)k * ws;
                    for (int j = 0; j < ws; ++j) w[j] = j < 3 ? r[i].word[j] : 0ull;
                }
            }
        });
        if (corrupt.load()) return fail(h, SBFS_ECUDA, "streamed solve: corrupt escalated result");
    }
    o.expanded += (int64_t)(hc->expanded + L.level_expanded);
    o.escalated += esc;
    o.synchronizing += (int64_t)hc->synchronizing;
    o.error |= hc->error;
    if (hc->first_violation != ULLONG_MAX && o.first_violation < 0) o.first_violation = (int64_t)hc->first_violation;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, L.ev_k0, L.ev_k1) == cudaSuccess) o.kernel_ms += ms;
    cudaGetLastError();
    return SBFS_OK;
}

sbfs_status solve_host(sbfs_handle *h, const uint8_t *maps, int32_t lstride, const uint8_t *ns,
                       int32_t n_uniform, int64_t count, int32_t *out_len, uint64_t *out_words,
                       int32_t word_stride, int64_t *out_first_violation, sbfs_stats *stats, bool plain)
{
    if (!h) return fail(nullptr, SBFS_EINVAL, "handle is NULL");
    std::lock_guard<std::mutex> lock(h->mu);
    h->last_error.clear();
    const auto t0 = std::chrono::steady_clock::now();
    int32_t max_n = 0, same_n = 0;
    sbfs_status s = check_records(h, maps, lstride, ns, n_uniform, count, &max_n, &same_n);
    if (s) return s;
    if (same_n) {
        // one n for every automaton (the IComputable mirrors always pass sizes):
        // the uniform-batch kernels and paths apply, and the sizes need not cross
        ns = nullptr;
        n_uniform = same_n;
    }
    if (out_words && word_stride < 1) return fail(h, SBFS_EINVAL, "word_stride must be >= 1");
    if (!out_len && out_words) return fail(h, SBFS_EINVAL, "words need out_len");
    CK(cudaSetDevice(h->device), "selecting device");
    if ((s = ensure_plan(h))) return s;

    if (h->device_pending) CK(cudaEventSynchronize(h->ev_device), "waiting for device work");
    if (stream_eligible(h, ns, n_uniform, count, plain)) {
        const bool s_pin_in = is_pinned(maps), s_pin_out = is_pinned(out_len) && is_pinned(out_words);
        const int32_t ws = out_words ? word_stride : 0;
        StreamOut so;
        for (int64_t begin = 0; begin < count; begin += kStreamJob) {
            const int64_t cnt = std::min(kStreamJob, count - begin);
            const int64_t fv_before = so.first_violation;
            so.first_violation = -1;
            s = solve_streamed_job(h, maps + (size_t)begin * 2 * lstride, lstride, n_uniform, cnt,
                                   out_len ? out_len + begin : nullptr,
                                   out_words ? out_words + (size_t)begin * ws : nullptr, ws, s_pin_in, s_pin_out, so);
            if (s) return s;
            so.first_violation =
                fv_before >= 0 ? fv_before : (so.first_violation >= 0 ? begin + so.first_violation : -1);
        }
        h->skip_ready_chunk = -1;   // the test hook is one-shot
        if (out_first_violation) *out_first_violation = so.first_violation;
        if (stats) {
            stats->automata = count;
            stats->expanded = so.expanded;
            stats->synchronizing = so.synchronizing;
            stats->h2d_bytes = count * 2 * (int64_t)lstride;
            stats->d2h_bytes = (out_len ? count * 4 : 0) + (out_words ? count * (int64_t)ws * 8 : 0);
            stats->launches = so.launches;
            stats->classes = 1;
            stats->kernel_ms = so.kernel_ms;
            stats->escalated = so.escalated;
            stats->total_ms =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        if (so.error & kErrInvalid) return fail(h, SBFS_EINVAL, "malformed automaton: a state index >= n");
        if (so.error & kErrBounds) return fail(h, SBFS_ECUDA, "a bounds check failed (checked build)");
        if (so.error) return fail(h, SBFS_ETIMEOUT, "a device-side bounded wait ran out");
        return SBFS_OK;
    }
    const int64_t chunk = plain ? std::max<int64_t>(count, 1)
                                : (h->cfg.chunk > 0 ? h->cfg.chunk : kDefaultChunk);
    const bool pin_in = is_pinned(maps) && is_pinned(ns);
    const bool pin_out = is_pinned(out_len) && is_pinned(out_words);
    const size_t rec = 2 * (size_t)lstride;
    Totals tot;
    int launches = 0;
    int64_t h2d = 0, d2h = 0;
    const int nlanes = plain ? 1 : (int)h->lanes.size();

    for (int64_t begin = 0, ci = 0; begin < count; begin += chunk, ++ci) {
        Lane &L = h->lanes[ci % nlanes];
        if ((s = finish_lane(h, L, tot))) return s;
        const int64_t cnt = std::min(chunk, count - begin);
        CK(L.maps.reserve(cnt * rec), "allocating records");
        if (ns) CK(L.ns.reserve(cnt), "allocating sizes");
        if (out_len) CK(L.len.reserve(cnt * sizeof(int32_t)), "allocating lengths");
        if (out_words) CK(L.words.reserve(cnt * word_stride * sizeof(uint64_t)), "allocating words");
        CK(L.h_counters.reserve(sizeof(DevCounters)), "allocating pinned counters");
        const uint8_t *src_maps = maps + begin * rec;
        const uint8_t *src_ns = ns ? ns + begin : nullptr;
        if (!pin_in) {
            CK(L.h_maps.reserve(cnt * rec), "allocating pinned staging");
            if (ns) CK(L.h_ns.reserve(cnt), "allocating pinned staging");
            CopyPool::Group g;
            h->copy_pool().copy(L.h_maps.ptr, src_maps, cnt * rec, g);
            src_maps = L.h_maps.as<uint8_t>();
            if (ns) {
                h->copy_pool().copy(L.h_ns.ptr, src_ns, cnt, g);
                src_ns = L.h_ns.as<uint8_t>();
            }
            h->copy_pool().wait(g);
        }
        L.staged_out = !pin_out;
        L.user_len = out_len;
        L.user_words = out_words;
        L.word_stride = word_stride;
        void *dst_len = nullptr, *dst_words = nullptr;
        const size_t wb = out_words ? (size_t)cnt * word_stride * sizeof(uint64_t) : 0;
        if (out_len) {
            dst_len = pin_out ? (void *)(out_len + begin) : nullptr;
            if (!pin_out) {
                CK(L.h_len.reserve(cnt * sizeof(int32_t)), "allocating pinned staging");
                dst_len = L.h_len.ptr;
            }
        }
        if (out_words) {
            dst_words = pin_out ? (void *)(out_words + (size_t)begin * word_stride) : nullptr;
            if (!pin_out) {
                CK(L.h_words.reserve(wb), "allocating pinned staging");
                dst_words = L.h_words.ptr;
            }
        }
        Job j{L.maps.as<uint8_t>(), lstride, ns ? L.ns.as<uint8_t>() : nullptr, n_uniform, max_n, cnt,
              out_len ? L.len.as<int32_t>() : nullptr, out_words ? L.words.as<uint64_t>() : nullptr,
              word_stride};
        h2d += cnt * rec + (ns ? cnt : 0);
        d2h += (out_len ? cnt * (int64_t)sizeof(int32_t) : 0) + (int64_t)wb;
        if (!plain) {
            // records in on the shared copy stream (chunk order), then the lane waits for them
            CK(cudaMemcpyAsync(L.maps.ptr, src_maps, cnt * rec, cudaMemcpyHostToDevice, h->copy_in),
               "copying records");
            if (ns) CK(cudaMemcpyAsync(L.ns.ptr, src_ns, cnt, cudaMemcpyHostToDevice, h->copy_in), "copying sizes");
            CK(cudaEventRecord(L.ev_in, h->copy_in), "recording event");
            CK(cudaStreamWaitEvent(L.stream, L.ev_in, 0), "ordering streams");
        }
        CK(cudaEventRecord(L.ev_k0, L.stream), "recording event");
        if (!plain) {
            // one chunk: counters, bucketing, class kernels, copies out
            auto body = [&]() -> sbfs_status {
                sbfs_status bs = reset_counters(h, L);
                if (bs) return bs;
                if ((bs = enqueue_kernels(h, L, j, &launches))) return bs;
                if (out_len)
                    CK(cudaMemcpyAsync(dst_len, L.len.ptr, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, L.stream),
                       "copying lengths");
                if (out_words)
                    CK(cudaMemcpyAsync(dst_words, L.words.ptr, wb, cudaMemcpyDeviceToHost, L.stream), "copying words");
                CK(cudaMemcpyAsync(L.h_counters.ptr, L.counters.ptr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                                   L.stream),
                   "copying counters");
                return SBFS_OK;
            };
            const bool graphable = h->cfg.use_graph && graph_safe(h, max_n);
            const std::string key = graphable ? graph_key(src_maps, src_ns, dst_len, dst_words, nullptr, cnt, lstride,
                                                          n_uniform, max_n, word_stride)
                                              : std::string();
            if ((s = run_maybe_captured(h, L, key, graphable, &launches, body))) return s;
            CK(cudaEventRecord(L.ev_k1, L.stream), "recording event");
        } else {
            CK(cudaMemcpyAsync(L.maps.ptr, src_maps, cnt * rec, cudaMemcpyHostToDevice, L.stream), "copying records");
            if (ns) CK(cudaMemcpyAsync(L.ns.ptr, src_ns, cnt, cudaMemcpyHostToDevice, L.stream), "copying sizes");
            if ((s = reset_counters(h, L))) return s;
            // one launch per automaton, same kernels, one-CTA grid
            Plan saved = h->plan;
            for (int c = 0; c < 3; ++c) h->plan.pool[c].ctas = 1;
            h->plan.cta.ctas = 1;
            CK(L.tickets.reserve((size_t)cnt * sizeof(unsigned long long)), "allocating tickets");
            CK(cudaMemsetAsync(L.tickets.ptr, 0, (size_t)cnt * sizeof(unsigned long long), L.stream),
               "resetting tickets");
            CK(cudaEventRecord(L.ev_k0, L.stream), "recording event");
            for (int64_t i = 0; i < cnt; ++i) {
                Job one = j;
                one.maps = j.maps + i * rec;
                one.ns = nullptr;
                one.n_uniform = ns ? ns[begin + i] : n_uniform;
                one.max_n = one.n_uniform;
                one.count = 1;
                one.len = j.len ? j.len + i : nullptr;
                one.words = j.words ? j.words + i * word_stride : nullptr;
                if (one.n_uniform < 1 || one.n_uniform > SBFS_MAX_N) {
                    h->plan = saved;
                    return fail(h, SBFS_EINVAL, "n out of range");
                }
                if ((s = enqueue_kernels(h, L, one, &launches, true, L.tickets.as<unsigned long long>() + i))) {
                    h->plan = saved;
                    return s;
                }
            }
            h->plan = saved;
            CK(cudaEventRecord(L.ev_k1, L.stream), "recording event");
            if (out_len)
                CK(cudaMemcpyAsync(dst_len, L.len.ptr, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, L.stream),
                   "copying lengths");
            if (out_words)
                CK(cudaMemcpyAsync(dst_words, L.words.ptr, wb, cudaMemcpyDeviceToHost, L.stream), "copying words");
            CK(cudaMemcpyAsync(L.h_counters.ptr, L.counters.ptr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                               L.stream),
               "copying counters");
        }
        CK(cudaEventRecord(L.ev_done, L.stream), "recording event");
        L.busy = true;
        L.begin = begin;
        L.count = cnt;
    }
    for (auto &L : h->lanes)
        if ((s = finish_lane(h, L, tot))) return s;
    if (out_first_violation) *out_first_violation = tot.first_violation;
    if (stats) {
        stats->automata = count;
        stats->expanded = tot.expanded;
        stats->synchronizing = tot.synchronizing;
        if (plain && out_len) {
            stats->synchronizing = 0;
            for (int64_t i = 0; i < count; ++i) stats->synchronizing += out_len[i] >= 0;
        }
        stats->h2d_bytes = h2d;
        stats->d2h_bytes = d2h;
        stats->launches = launches;
        stats->classes = 0;
        stats->kernel_ms = tot.kernel_ms;
        stats->escalated = tot.escalated;
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    if (tot.error & kErrInvalid) return fail(h, SBFS_EINVAL, "malformed automaton: a state index >= n");
    if (tot.error & kErrBounds) return fail(h, SBFS_ECUDA, "a bounds check failed (checked build)");
    if (tot.error) return fail(h, SBFS_ETIMEOUT, "a device-side bounded wait ran out");
    return SBFS_OK;
}

}  // namespace

namespace sbfs {

// Enqueue one solve of device-resident records on lane L's stream (counters
// reset, size-class bucketing, class kernels).  Shared with the serving loop.
sbfs_status engine_enqueue(sbfs_handle *h, Lane &L, const uint8_t *d_maps, int32_t lstride, const uint8_t *d_ns,
                           int32_t n_uniform, int32_t max_n, int64_t count, int32_t *d_len, uint64_t *d_words,
                           int32_t word_stride, int *launches, unsigned int *done_flag, unsigned int done_tag)
{
    sbfs_status s = ensure_plan(h);
    if (s) return s;
    if ((s = reset_counters(h, L))) return s;
    Job j{d_maps, lstride, d_ns, n_uniform, max_n, count, d_len, d_words, d_words ? word_stride : 0, done_flag,
          done_tag};
    return enqueue_kernels(h, L, j, launches);
}

}  // namespace sbfs

extern "C" {

int32_t sbfs_abi_version(void) { return SBFS_ABI_VERSION; }

sbfs_status sbfs_config_default(sbfs_config *cfg)
{
    if (!cfg) return SBFS_EINVAL;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = -1;
    cfg->use_graph = 0;
    cfg->autotune = 0;
    return SBFS_OK;
}

const char *sbfs_status_string(sbfs_status s)
{
    switch (s) {
    case SBFS_OK: return "ok";
    case SBFS_EINVAL: return "invalid argument";
    case SBFS_ENOMEM: return "out of memory";
    case SBFS_ETIMEOUT: return "timed out";
    case SBFS_ECUDA: return "CUDA error";
    case SBFS_EBUSY: return "busy";
    case SBFS_ENOTFOUND: return "not found";
    case SBFS_ECANCELED: return "cancelled";
    case SBFS_ESTOPPED: return "stopped";
    }
    return "unknown status";
}

sbfs_status sbfs_create(const sbfs_config *cfg, sbfs_handle **out)
{
    if (!out) return fail(nullptr, SBFS_EINVAL, "out is NULL");
    *out = nullptr;
    sbfs_config c;
    sbfs_config_default(&c);
    if (cfg) c = *cfg;
    int dev = c.device;
    cudaError_t e;
    if (dev < 0) {
        e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return cuda_fail(nullptr, e, "no CUDA device");
    }
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "selecting device");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "reading device properties");
    if (prop.major < 10) return fail(nullptr, SBFS_ECUDA, "libsbfs is built for sm_100a (B200)");
    sbfs_handle *h = new (std::nothrow) sbfs_handle();
    if (!h) return fail(nullptr, SBFS_ENOMEM, "allocating handle");
    h->device = dev;
    h->sm_count = prop.multiProcessorCount;
    h->smem_optin = prop.sharedMemPerBlockOptin;
    h->cfg = c;
    if (const char *skip = std::getenv("SBFS_TEST_SKIP_CHUNK_READY")) h->skip_ready_chunk = std::atoll(skip);
    h->lanes.resize(c.streams > 0 ? std::min(c.streams, 16) : kDefaultLanes);
    if ((e = cudaEventCreateWithFlags(&h->ev_device, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev_dk0)) != cudaSuccess || (e = cudaEventCreate(&h->ev_dk1)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->copy_in, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->streamer.copy_out, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&h->streamer.ev_in0, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&h->streamer.ev_kdone, cudaEventDisableTiming)) != cudaSuccess) {
        sbfs_destroy(h);
        return cuda_fail(nullptr, e, "creating events");
    }
    // lane i runs chunks i, i + lanes, ...: earlier lanes get higher stream
    // priority, so an older chunk's pending CTAs (a hand-off launch after its
    // pooled kernel) are scheduled ahead of a younger chunk's and chunks
    // complete in order
    int prio_least = 0, prio_greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess) {
        cudaGetLastError();
        prio_least = prio_greatest = 0;
    }
    int lane_index = 0;
    for (auto &L : h->lanes) {
        const int prio = std::min(prio_least, prio_greatest + lane_index++);
        if ((e = cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, prio)) != cudaSuccess ||
            (e = cudaEventCreate(&L.ev_k0)) != cudaSuccess || (e = cudaEventCreate(&L.ev_k1)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&L.ev_done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&L.ev_in, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&L.ev_fork, cudaEventDisableTiming)) != cudaSuccess) {
            sbfs_destroy(h);
            return cuda_fail(nullptr, e, "creating streams");
        }
        for (int c = 0; c < 3; ++c)
            if ((e = cudaStreamCreateWithPriority(&L.aux[c], cudaStreamNonBlocking, prio)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&L.ev_join[c], cudaEventDisableTiming)) != cudaSuccess) {
                sbfs_destroy(h);
                return cuda_fail(nullptr, e, "creating streams");
            }
    }
    *out = h;
    return SBFS_OK;
}

sbfs_status sbfs_destroy(sbfs_handle *h)
{
    if (!h) return SBFS_OK;
    cudaSetDevice(h->device);
    for (auto &L : h->lanes) {
        if (L.stream) cudaStreamSynchronize(L.stream);
        for (cudaStream_t a : L.aux)
            if (a) cudaStreamSynchronize(a);
        L.drop_graphs();
        for (DevBuf *d : {&L.maps, &L.ns, &L.len, &L.words, &L.spill, &L.order, &L.counters, &L.ranges,
                          &L.cta_queue, &L.hbm_bitmap, &L.hbm_queue, &L.escal, &L.tickets})
            d->release();
        for (HostBuf *b : {&L.h_counters, &L.h_maps, &L.h_ns, &L.h_len, &L.h_words}) b->release();
        if (L.ev_k0) cudaEventDestroy(L.ev_k0);
        if (L.ev_k1) cudaEventDestroy(L.ev_k1);
        if (L.ev_done) cudaEventDestroy(L.ev_done);
        if (L.ev_in) cudaEventDestroy(L.ev_in);
        if (L.ev_fork) cudaEventDestroy(L.ev_fork);
        for (int c = 0; c < 3; ++c) {
            if (L.aux[c]) cudaStreamDestroy(L.aux[c]);
            if (L.ev_join[c]) cudaEventDestroy(L.ev_join[c]);
            L.spill_c[c].release();
        }
        for (int c = 0; c < 4; ++c) {
            L.heavy[c].release();
            L.heavy_queue[c].release();
        }
        if (L.level_ready) L.level.destroy();
        if (L.stream) cudaStreamDestroy(L.stream);
    }
    if (h->copy_in) {
        cudaStreamSynchronize(h->copy_in);
        cudaStreamDestroy(h->copy_in);
    }
    {
        Streamer &S = h->streamer;
        if (S.copy_out) {
            cudaStreamSynchronize(S.copy_out);
            cudaStreamDestroy(S.copy_out);
        }
        if (S.ev_in0) cudaEventDestroy(S.ev_in0);
        if (S.ev_kdone) cudaEventDestroy(S.ev_kdone);
        for (cudaEvent_t e : S.ev_out) cudaEventDestroy(e);
        S.ev_out.clear();
        S.flags.release();
        S.escal_out.release();
        S.h_flags.release();
        S.h_escal.release();
    }
    if (h->ev_device) cudaEventDestroy(h->ev_device);
    if (h->ev_dk0) cudaEventDestroy(h->ev_dk0);
    if (h->ev_dk1) cudaEventDestroy(h->ev_dk1);
    delete h;
    return SBFS_OK;
}

const char *sbfs_last_error(const sbfs_handle *h)
{
    return h ? h->last_error.c_str() : g_create_error.c_str();
}

int32_t sbfs_best_parallelism(const sbfs_handle *h) { return h ? (int32_t)h->lanes.size() : 0; }

int32_t sbfs_word_stride(int32_t max_n)
{
    if (max_n < 2) return 1;
    const int64_t bits = (int64_t)(max_n - 1) * (max_n - 1);
    return (int32_t)std::max<int64_t>(1, (bits + 63) / 64);
}

sbfs_status sbfs_solve_batch(sbfs_handle *h, const uint8_t *maps, int32_t lstride, const uint8_t *ns,
                             int32_t n_uniform, int64_t count, int32_t *out_len, uint64_t *out_words,
                             int32_t word_stride, int64_t *out_first_violation, sbfs_stats *stats)
{
    if (!out_len) return fail(h, SBFS_EINVAL, "out_len is NULL (use sbfs_verify_batch)");
    return solve_host(h, maps, lstride, ns, n_uniform, count, out_len, out_words, word_stride,
                      out_first_violation, stats, false);
}

sbfs_status sbfs_verify_batch(sbfs_handle *h, const uint8_t *maps, int32_t lstride, const uint8_t *ns,
                              int32_t n_uniform, int64_t count, int32_t *out_len,
                              int64_t *out_first_violation, sbfs_stats *stats)
{
    return solve_host(h, maps, lstride, ns, n_uniform, count, out_len, nullptr, 0, out_first_violation, stats,
                      false);
}

sbfs_status sbfs_solve_plain(sbfs_handle *h, const uint8_t *maps, int32_t lstride, const uint8_t *ns,
                             int32_t n_uniform, int64_t count, int32_t *out_len, uint64_t *out_words,
                             int32_t word_stride, int64_t *out_first_violation, sbfs_stats *stats)
{
    if (!out_len) return fail(h, SBFS_EINVAL, "out_len is NULL");
    return solve_host(h, maps, lstride, ns, n_uniform, count, out_len, out_words, word_stride,
                      out_first_violation, stats, true);
}

sbfs_status sbfs_solve_batch_device(sbfs_handle *h, const uint8_t *d_maps, int32_t lstride,
                                    const uint8_t *d_ns, int32_t n_uniform, int32_t max_n, int64_t count,
                                    int32_t *d_len, uint64_t *d_words, int32_t word_stride,
                                    int64_t *d_first_violation, void *stream)
{
    if (!h) return fail(nullptr, SBFS_EINVAL, "handle is NULL");
    std::lock_guard<std::mutex> lock(h->mu);
    h->last_error.clear();
    if (count < 0 || (count > 0 && !d_maps)) return fail(h, SBFS_EINVAL, "bad records");
    if (lstride < 1 || lstride > 32) return fail(h, SBFS_EINVAL, "lstride must be in 1..32");
    if (!d_ns && (n_uniform < 1 || n_uniform > SBFS_MAX_N || n_uniform > lstride))
        return fail(h, SBFS_EINVAL, "n_uniform must be in 1..min(28, lstride)");
    if (d_words && word_stride < 1) return fail(h, SBFS_EINVAL, "word_stride must be >= 1");
    if (!d_first_violation) return fail(h, SBFS_EINVAL, "d_first_violation is NULL");
    CK(cudaSetDevice(h->device), "selecting device");
    sbfs_status s = ensure_plan(h);
    if (s) return s;
    Lane &L = h->lanes[0];
    if (L.busy) {
        Totals t;
        if ((s = finish_lane(h, L, t))) return s;
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : L.stream;
    if (st != L.stream) {
        // lane 0's buffers may still be read by earlier work on its own stream
        CK(cudaEventRecord(L.ev_done, L.stream), "recording event");
        CK(cudaStreamWaitEvent(st, L.ev_done, 0), "ordering streams");
    }
    CK(L.h_counters.reserve(sizeof(DevCounters)), "allocating pinned counters");
    cudaStream_t saved = L.stream;
    L.stream = st;
    Job j{d_maps, lstride, d_ns, n_uniform, d_ns ? (max_n > 0 ? std::min(max_n, SBFS_MAX_N) : SBFS_MAX_N) : n_uniform,
          count, d_len, d_words, d_words ? word_stride : 0};
    int launches = 0;
    // counters, bucketing, class kernels, the violation index, counters back to the host
    auto body = [&]() -> sbfs_status {
        sbfs_status bs = reset_counters(h, L);
        if (bs) return bs;
        if (count > 0 && (bs = enqueue_kernels(h, L, j, &launches))) return bs;
        launches += 1;
        finalize_violation<<<1, 1, 0, L.stream>>>(L.counters.as<DevCounters>(), d_first_violation);
        CK(cudaGetLastError(), "launching finalize");
        CK(cudaMemcpyAsync(L.h_counters.ptr, L.counters.ptr, sizeof(DevCounters), cudaMemcpyDeviceToHost, L.stream),
           "copying counters");
        return SBFS_OK;
    };
    const bool graphable = h->cfg.use_graph && graph_safe(h, j.max_n);
    const std::string key = graphable ? graph_key(d_maps, d_ns, d_len, d_words, d_first_violation, count, lstride,
                                                  n_uniform, j.max_n, word_stride)
                                      : std::string();
    CK(cudaEventRecord(h->ev_dk0, st), "recording event");
    s = run_maybe_captured(h, L, key, graphable, &launches, body);
    L.stream = saved;
    if (s) return s;
    CK(cudaEventRecord(h->ev_dk1, st), "recording event");
    CK(cudaEventRecord(h->ev_device, st), "recording event");
    if (st != L.stream) CK(cudaStreamWaitEvent(L.stream, h->ev_device, 0), "ordering streams");
    h->device_pending = true;
    h->device_count = count;
    h->device_launches = launches;
    return SBFS_OK;
}

sbfs_status sbfs_device_wait(sbfs_handle *h, sbfs_stats *stats)
{
    if (!h) return fail(nullptr, SBFS_EINVAL, "handle is NULL");
    std::lock_guard<std::mutex> lock(h->mu);
    if (!h->device_pending) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return SBFS_OK;
    }
    CK(cudaEventSynchronize(h->ev_device), "waiting for device work");
    h->device_pending = false;
    const DevCounters *c = h->lanes[0].h_counters.as<DevCounters>();
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->automata = h->device_count;
        stats->expanded = (int64_t)(c->expanded + h->lanes[0].level_expanded);
        stats->escalated = (int64_t)(c->escal_count[0] + c->escal_count[1]);
        stats->synchronizing = (int64_t)c->synchronizing;
        stats->launches = h->device_launches;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, h->ev_dk0, h->ev_dk1) == cudaSuccess) stats->kernel_ms = ms;
        cudaGetLastError();
    }
    if (c->error & kErrInvalid) return fail(h, SBFS_EINVAL, "malformed automaton: a state index >= n");
    if (c->error & kErrBounds) return fail(h, SBFS_ECUDA, "a bounds check failed (checked build)");
    if (c->error) return fail(h, SBFS_ETIMEOUT, "a device-side bounded wait ran out");
    return SBFS_OK;
}

int32_t sbfs_describe_plan(sbfs_handle *h, char *buf, int32_t len)
{
    if (!h) return 0;
    std::lock_guard<std::mutex> lock(h->mu);
    if (cudaSetDevice(h->device) != cudaSuccess || ensure_plan(h) != SBFS_OK) {
        cudaGetLastError();
        return 0;
    }
    const Plan &P = h->plan;
    std::string js = "{\"tuned\":";
    js += P.tuned ? "true" : "false";
    js += ",\"classes\":[";
    char tmp[256];
    for (int c = 0; c < 3; ++c) {
        const bool lane = c < 2 && !P.use_pool[c];
        if (c == 2 && P.class2_hash && P.use_lane13) {
            std::snprintf(tmp, sizeof tmp,
                          "{\"class\":2,\"max_n\":16,\"kernel\":\"k_hash+k_cta\",\"slots\":%d,"
                          "\"uniform_n13\":\"k_lane<13>\",\"ring13\":%d,\"ctas13\":%d,"
                          "\"uniform_n14\":\"%s\",\"ring14\":%d,\"ctas14\":%d},",
                          P.class2_hash == 2 ? 4096 : 2048, P.lane13.ring, P.lane13.ctas,
                          P.use_lane14 ? "k_lane<14>" : "k_hash+k_cta", P.lane14.ring, P.lane14.ctas);
        } else if (lane) {
            const LaneShape &l = P.lane[c];
            std::snprintf(tmp, sizeof tmp,
                          "{\"class\":%d,\"max_n\":%d,\"kernel\":\"k_lane<%d>\",\"warps\":%d,\"ring\":%d,"
                          "\"refill\":%d,\"ctas\":%d},",
                          c, kClassMaxN[c], l.nmax, l.warps, l.ring, l.refill_k, l.ctas);
        } else if (c == 2 && P.class2_hash) {
            std::snprintf(tmp, sizeof tmp, "{\"class\":2,\"max_n\":16,\"kernel\":\"k_hash+k_cta\",\"slots\":%d},",
                          P.class2_hash == 2 ? 4096 : 2048);
        } else {
            const PoolShape &q = P.pool[c];
            std::snprintf(tmp, sizeof tmp,
                          "{\"class\":%d,\"max_n\":%d,\"kernel\":\"k_pool<%d,%d>\",\"warps\":%d,"
                          "\"queue_smem\":%d,\"ctas\":%d},",
                          c, kClassMaxN[c], q.nmax, q.slots, q.warps, q.queue_smem, q.ctas);
        }
        js += tmp;
    }
    std::snprintf(tmp, sizeof tmp,
                  "{\"class\":3,\"max_n\":20,\"kernel\":\"%s\",\"threads\":%d,\"ctas\":%d},"
                  "{\"class\":4,\"max_n\":28,\"kernel\":\"k_level\",\"threads\":512,\"slots\":%d}]}",
                  P.class3_level ? "k_level" : P.class3_hash ? "k_hash+k_cta" : "k_cta", P.cta.threads, P.cta.ctas,
                  kMaxLevelSlots);
    js += tmp;
    if (buf && len > 0) {
        std::strncpy(buf, js.c_str(), (size_t)len - 1);
        buf[len - 1] = '\0';
    }
    return (int32_t)js.size() + 1;
}

sbfs_status sbfs_host_alloc(size_t bytes, void **out)
{
    if (!out) return SBFS_EINVAL;
    *out = nullptr;
    cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return SBFS_ENOMEM;
    }
    return SBFS_OK;
}

sbfs_status sbfs_host_free(void *p)
{
    if (p && cudaFreeHost(p) != cudaSuccess) {
        cudaGetLastError();
        return SBFS_EINVAL;
    }
    return SBFS_OK;
}

}  // extern "C"
